"""Trajectory output in the dataset schema of the reference's HDF5 writer.

The reference's ParallelHybridSolver writes one HDF5 file per experiment
(CaSim/ParallelHybridSolver.cpp:13-57 creates it, :234-337 fill it): groups
/Dyad /Cytosol /SR /Channels /IonsChannels, one dataset per output species,
each dataset [time index, scenario, ...] extended as the run goes, written
every "Iterations for <group>" time steps (time index j / cadence for step j,
j = 0 after the batch's first Update), scenarios batch after batch along the
second axis. This module runs the same scenario loop on a ReleaseSiteBatch
(CaSim/ParallelHybridSolver.cpp:339-437: per batch ResetSystem, InitOpening
of channel (S*batch + site) / sc_per_channel, Update, then n_iter steps) and
writes the same datasets, with the same names, shapes, element types and
cadences, as NumPy .npy files under <directory>/Output/<group>/<name>.npy
(no HDF5 library is linked; each file is a full dataset, allocated at its
final extent up front), next to the echoed Parameters.json as the reference
writes it (:40-45).

Dataset contents (the reference's Get* maps):
  /Dyad/<ion>, /Dyad/<ion>-<buffer>  [T, scenarios, nx, ny(, nz)] float64, for the
      ions and buffers named in "Outputs" (DyadRD2DCPU::GetConcentrations,
      CaSim/DyadRD2DCPU.cpp:500-523; node order y fastest in 2D, z fastest in 3D)
  /Cytosol/<species>                 [T, scenarios] float64 for the well-mixed pool
      (CytosolPool::GetConcentrations, CaSim/CytosolPool.cpp:331-357); for the 3D
      cytosol of this library, [T, scenarios, mc, mc, mc] (x fastest)
  /SR/<ion>                          [T, scenarios, channels] float64 (SRPool::
      GetConcentrations, CaSim/SRPool.cpp:91-101: the site's jSR value at every channel)
  /Channels/RyR                      [T, scenarios, channels] int32: the model state
      of each RyR (0/1, or the micro-state 0..59 of 60-state models)
  /IonsChannels/<ion>                [T, scenarios, channels] float64, every ion
      (DyadRD2DCPU::GetIonsNearChannels, CaSim/DyadRD2DCPU.cpp:536-544)
"""
import json
import os

import numpy as np

CADENCE_KEYS = {"Dyad": "Iterations for Dyad", "Cytosol": "Iterations for Cytosol", "SR": "Iterations for SR",
                "Channels": "Iterations for IonChannels", "IonsChannels": "Iterations for IonsNearChannels"}


def n_iterations(params):
    """n_iter = time_max / dt (int) as the reference computes it (CaSim/ParallelHybridSolver.cpp:14-18)."""
    dt = float(params["dt, ns"]) * 1e-6
    return int(float(params["Max Time, ms"]) / dt)


def first_channels(n_sites, n_batches, n_channels, batch):
    """Initially opened RyR of every site of a batch (CaSim/ParallelHybridSolver.cpp:411-417)."""
    sc_per_channel = n_batches * n_sites // n_channels
    if sc_per_channel < 1:
        sc_per_channel += 1
    return np.array([(n_sites * batch + j) // sc_per_channel for j in range(n_sites)], dtype=np.int32)


class ScenarioOutput:
    """Runs NumScenarios scenarios in batches of the handle's sites and writes the
    reference's datasets. The handle's sites must all have the same RyR count
    (the reference has one channel layout per run)."""

    def __init__(self, sim, params, directory, n_scenarios=None):
        self.sim, self.params, self.dir = sim, params, directory
        self.S = sim.S
        self.n_ch = int(np.max(sim.n_ch))
        if int(np.min(sim.n_ch)) != self.n_ch:
            raise ValueError("scenario output needs one RyR count for every site")
        self.n_scen = int(n_scenarios if n_scenarios is not None else params.get("NumScenarios", self.S))
        self.n_batches = max(1, self.n_scen // self.S)
        self.n_scen = self.n_batches * self.S
        self.n_iter = n_iterations(params)
        self.cad = {g: int(params.get(k, 0)) for g, k in CADENCE_KEYS.items()}
        outputs = set(params.get("Outputs", []))
        info = sim.info
        nsp = info.n_ions + info.n_pairs
        names = [sim.species_name(k) for k in range(nsp)]
        ions = names[:info.n_ions]
        # /Dyad: ions named in Outputs, and the ion-buffer pairs of the buffers named there
        self.dyad = [(n, k) for k, n in enumerate(names)
                     if (k < info.n_ions and n in outputs) or (k >= info.n_ions and n.split("-", 1)[1] in outputs)]
        self.rd3d = info.cyto_nodes > 0
        cnames = [sim.cyto_species_name(k) for k in range(info.n_cyto_species)]
        self.cyto = [(n, k) for k, n in enumerate(cnames)
                     if (k < info.n_ions and n in outputs) or (k >= info.n_ions and n.split("-", 1)[1] in outputs)]
        self.sr = [(n, k) for k, n in enumerate(ions) if n in outputs]
        self.mouth = [(n, k) for k, n in enumerate(ions)]
        self.micro = False
        ch = params["Dyad"]["Channels"]
        self.micro = any(c.get("Model") == "SingleSiteMWC" for c in ch.values())
        self.files = {}

    def _T(self, group):
        c = self.cad[group]
        return self.n_iter // c + 1 if c > 0 else 0

    def _open(self, group, name, tail, dtype):
        path = os.path.join(self.dir, "Output", group, name + ".npy")
        os.makedirs(os.path.dirname(path), exist_ok=True)
        arr = np.lib.format.open_memmap(path, mode="w+", dtype=dtype, shape=(self._T(group), self.n_scen) + tuple(tail))
        self.files[(group, name)] = arr
        return arr

    def _create(self):
        dims = self.sim._site_dims[0]
        dyad_tail = dims[:2] if self.sim.info.dim == 2 else dims
        if self._T("Dyad"):
            for n, _ in self.dyad:
                self._open("Dyad", n, dyad_tail, np.float64)
        if self._T("Cytosol"):
            mc = round(self.sim.info.cyto_nodes ** (1.0 / 3.0)) if self.rd3d else 0
            for n, _ in self.cyto:
                self._open("Cytosol", n, (mc, mc, mc) if self.rd3d else (), np.float64)
        if self._T("SR"):
            for n, _ in self.sr:
                self._open("SR", n, (self.n_ch,), np.float64)
        if self._T("Channels"):
            self._open("Channels", "RyR", (self.n_ch,), np.int32)
        if self._T("IonsChannels"):
            for n, _ in self.mouth:
                self._open("IonsChannels", n, (self.n_ch,), np.float64)

    def _write(self, j, batch):
        sim, S = self.sim, self.S
        sl = slice(batch * S, (batch + 1) * S)
        if self.cad["Dyad"] and j % self.cad["Dyad"] == 0:
            t = j // self.cad["Dyad"]
            for n, k in self.dyad:
                arr = self.files[("Dyad", n)]
                for s in range(S):
                    arr[t, batch * S + s] = sim.field(s, k).reshape(arr.shape[2:])
        if self.cad["Cytosol"] and j % self.cad["Cytosol"] == 0:
            t = j // self.cad["Cytosol"]
            for n, k in self.cyto:
                arr = self.files[("Cytosol", n)]
                for s in range(S):
                    if self.rd3d:
                        arr[t, batch * S + s] = sim.cyto_field(s, k).reshape(arr.shape[2:][::-1]).transpose(2, 1, 0)
                    else:
                        arr[t, batch * S + s] = sim.cyto(s)[k]
        if self.cad["SR"] and j % self.cad["SR"] == 0:
            t = j // self.cad["SR"]
            for n, k in self.sr:
                arr = self.files[("SR", n)]
                for s in range(S):
                    arr[t, batch * S + s, :] = sim.jsr(s)[k]
        if self.cad["Channels"] and j % self.cad["Channels"] == 0:
            t = j // self.cad["Channels"]
            arr = self.files[("Channels", "RyR")]
            for s in range(S):
                arr[t, batch * S + s] = sim.micro_states(s) if self.micro else sim.states(s)
        if self.cad["IonsChannels"] and j % self.cad["IonsChannels"] == 0:
            t = j // self.cad["IonsChannels"]
            for n, k in self.mouth:
                arr = self.files[("IonsChannels", n)]
                arr[t, sl] = sim.all_mouth(k).reshape(S, self.n_ch)

    def run(self):
        """All batches; returns the dataset paths by (group, name)."""
        os.makedirs(self.dir, exist_ok=True)
        with open(os.path.join(self.dir, "Parameters.json"), "w") as f:
            json.dump(self.params, f, indent=4)
        self._create()
        marks = sorted({j for c in self.cad.values() if c > 0 for j in range(0, self.n_iter + 1, c)} | {self.n_iter})
        for b in range(self.n_batches):
            self.sim.start(first_channels(self.S, self.n_batches, self.n_ch, b))
            self._write(0, b)
            done = 0
            for j in marks:
                if j == 0:
                    continue
                self.sim.step(j - done)
                done = j
                self._write(j, b)
        for arr in self.files.values():
            arr.flush()
        return {k: os.path.join(self.dir, "Output", k[0], k[1] + ".npy") for k in self.files}

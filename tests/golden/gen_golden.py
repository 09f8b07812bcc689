"""Generate the golden fixtures in this directory from the reference's OWN CPU
classes (oracle/_ref/libcasim_ref.so, built by `make -C oracle ref` from the
reference tree). Run where the reference tree is present, naming it:

    python tests/golden/gen_golden.py --ref <reference tree>
    CASIM_REFERENCE=<reference tree> python tests/golden/gen_golden.py

Each fixture is one NumBatch = 1 reference run (CaSim/ParallelHybridSolver.cpp:408-437
loop body, driven by oracle/ref_capi.cpp) with snapshots of the dyad fields,
RyR states, mouth Ca, jSR and cytosol pool after given step counts, plus the
first draws of RngStream::RandU01 for a few seeds. The example fixtures
(ex_*.npz) also hold the reference's example Parameters.json text and the
files it names, byte for byte, so that the tests can load them unchanged.
"""
import argparse
import ctypes
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402

REF_DIR = None  # the reference tree, from --ref or CASIM_REFERENCE


def ref_file(*parts):
    return os.path.join(REF_DIR, *parts)


def reference_params():
    with open(ref_file("CaSim", "test_input", "Parameters.json")) as f:
        return json.load(f)


def coords_text():
    with open(ref_file("CaSim", "test_input", "Jayasinghe.txt")) as f:
        return f.read()


def spline_tables():
    """Synthetic rate tables (this project's, 1/ms against Ca in uM) for the
    TwoStateSpline case: a saturating opening rate and a slowly falling
    closing rate on uneven knots."""
    ca = np.concatenate([np.linspace(0.0, 20.0, 11), np.linspace(25.0, 150.0, 26), np.linspace(175.0, 600.0, 18)])
    x = ca / 20.0
    kopen = 2.0 + 200.0 * x * x / (1.0 + x * x)
    kclose = 5.0 + 5.0 * np.exp(-ca / 100.0)
    return np.c_[ca, kopen], np.c_[ca, kclose]


def run_case(name, params, coords, steps, seed, first=0, tables=None):
    """Run the reference and store snapshots after each entry of `steps` (cumulative).
    tables: (kopen, kclose) arrays for a TwoStateSpline model, stored in the fixture."""
    with tempfile.TemporaryDirectory() as td:
        cpath = os.path.join(td, "coords.txt")
        with open(cpath, "w") as f:
            f.write(coords)
        p = json.loads(json.dumps(params))
        p["Dyad"]["Channels"]["RyR"]["Coordinates"] = cpath
        if tables is not None:
            for key, tab, fn in zip(("Kopen filename", "Kclose filename"), tables, ("kopen.txt", "kclose.txt")):
                np.savetxt(os.path.join(td, fn), tab, fmt="%.17g")
                p["Dyad"]["Channels"]["RyR"][key] = os.path.join(td, fn)
        p["Dyad"]["Seed"] = list(seed)
        sim = ref.RefSim(p, 1, 1)
        sim.start([first])
        out = {"params": np.frombuffer(json.dumps(params).encode(), dtype=np.uint8),
               "coords": np.loadtxt(cpath), "seed": np.asarray(seed, dtype=np.uint32),
               "first": np.int32(first), "steps": np.asarray(steps, dtype=np.int64), "dims": np.asarray(sim.dims)}
        if tables is not None:
            out["sp_open"], out["sp_close"] = tables
        ions = sorted(p["Dyad"]["Ions"].keys())
        bufs = sorted(p["Dyad"]["Buffers"].keys())
        done = 0
        for k, n in enumerate(steps):
            sim.step(n - done)
            done = n
            for ion in ions:
                out["f%d_%s" % (k, ion)] = sim.get("dyad:" + ion)
                out["m%d_%s" % (k, ion)] = sim.get("mouth:" + ion)
            for b in bufs:
                for ion in ions:
                    if ion in p["Dyad"]["Buffers"][b]["Ions"]:
                        out["f%d_%s-%s" % (k, ion, b)] = sim.get("dyadbuf:%s|%s-%s" % (b, ion, b))
            out["s%d" % k] = sim.states()
            out["sr%d" % k] = sim.get("sr")
            out["cy%d" % k] = sim.get("cyto:Calcium")
            out["tc%d" % k] = sim.get("total_sr_current")
        sim.close()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print("wrote", name, {k: v.shape for k, v in out.items() if hasattr(v, "shape") and v.size > 6})


def run_trajectory(name, params, coords, n_steps, every, seed, first=0):
    """States of every RyR (and mouth Ca, jSR Ca) every `every` steps, fields at the end."""
    with tempfile.TemporaryDirectory() as td:
        cpath = os.path.join(td, "coords.txt")
        with open(cpath, "w") as f:
            f.write(coords)
        p = json.loads(json.dumps(params))
        p["Dyad"]["Channels"]["RyR"]["Coordinates"] = cpath
        p["Dyad"]["Seed"] = list(seed)
        sim = ref.RefSim(p, 1, 1)
        sim.start([first])
        states, mouth, jsr = [], [], []
        for k in range(n_steps // every):
            sim.step(every)
            states.append(sim.states())
            mouth.append(sim.get("mouth:Calcium"))
            jsr.append(sim.get("sr")[0])
        out = {"params": np.frombuffer(json.dumps(params).encode(), dtype=np.uint8),
               "coords": np.loadtxt(cpath), "seed": np.asarray(seed, dtype=np.uint32), "first": np.int32(first),
               "every": np.int64(every), "states": np.asarray(states, dtype=np.int8),
               "mouth": np.asarray(mouth), "jsr": np.asarray(jsr), "dims": np.asarray(sim.dims),
               "ca_final": sim.get("dyad:Calcium")}
        sim.close()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    flips = int(np.abs(np.diff(out["states"].astype(int), axis=0)).sum())
    print("wrote", name, "transitions", flips)


def rng_fixture():
    L = ref.lib()
    seeds = [[3] * 6, [1, 2, 3, 4, 5, 6], [4294967086, 4294967086, 4294967086, 4294944442, 4294944442, 4294944442]]
    out = {}
    for k, s in enumerate(seeds):
        n = 4096
        arr = np.zeros(n)
        L.casimref_rng_draws((ctypes.c_ulong * 6)(*s), n, arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        out["seed%d" % k] = np.asarray(s, dtype=np.uint32)
        out["draws%d" % k] = arr
    np.savez_compressed(os.path.join(HERE, "rng.npz"), **out)
    print("wrote rng")


def run_example(name, example, steps, n_fields_every=None):
    """One NumBatch = 1 reference run of examples/<example>/Parameters.json as shipped
    (no seed: the reference falls back to the package seed, stream 0 for one thread),
    with the JSON text and the files it names stored byte for byte."""
    edir = ref_file("examples", example)
    with open(os.path.join(edir, "Parameters.json"), "rb") as f:
        text = f.read()
    params = json.loads(text)
    ch = params["Dyad"]["Channels"]["RyR"]
    names = [ch["Coordinates"]] + [ch[k] for k in ("Kopen filename", "Kclose filename") if k in ch]
    files = {}
    for fn in names:
        with open(os.path.join(edir, fn), "rb") as f:
            files[fn] = f.read()
    out = {"json_text": np.frombuffer(text, dtype=np.uint8), "file_names": np.array(names),
           "steps": np.asarray(steps, dtype=np.int64)}
    for k, fn in enumerate(names):
        out["file%d" % k] = np.frombuffer(files[fn], dtype=np.uint8)
    with tempfile.TemporaryDirectory() as td:
        for fn, data in files.items():
            with open(os.path.join(td, fn), "wb") as f:
                f.write(data)
        p = json.loads(text)
        c = p["Dyad"]["Channels"]["RyR"]
        for key in ("Coordinates", "Kopen filename", "Kclose filename"):
            if key in c:
                c[key] = os.path.join(td, c[key])
        # the reference's own GPU type names select its CPU classes here (same arithmetic in FP64)
        p["Dyad"]["Type"] = "CPU3D" if "3D" in p["Dyad"]["Type"] else "CPU2D"
        sim = ref.RefSim(p, 1, 1)
        sim.start([0])
        out["dims"] = np.asarray(sim.dims)
        ions = sorted(p["Dyad"]["Ions"].keys())
        bufs = sorted(p["Dyad"]["Buffers"].keys())
        done = 0
        for k, n in enumerate(steps):
            sim.step(n - done)
            done = n
            for ion in ions:
                out["f%d_%s" % (k, ion)] = sim.get("dyad:" + ion)
                out["m%d_%s" % (k, ion)] = sim.get("mouth:" + ion)
            for b in bufs:
                for ion in ions:
                    if ion in p["Dyad"]["Buffers"][b]["Ions"]:
                        out["f%d_%s-%s" % (k, ion, b)] = sim.get("dyadbuf:%s|%s-%s" % (b, ion, b))
            out["s%d" % k] = sim.states()
            out["sr%d" % k] = sim.get("sr")
            out["cy%d" % k] = sim.get("cyto:Calcium")
            out["tc%d" % k] = sim.get("total_sr_current")
        sim.close()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print("wrote", name, "transitions over", steps, [int(out["s%d" % k].sum()) for k in range(len(steps))])


def qs_fixture(name, n_scen=40):
    """The reference's own quasi-stationary Gillespie loop (CaSim/QuasyStationaryReleaseSite.cpp)
    over n_scen scenarios on one stream (a one-thread ParallelSolver), with the increments
    of the CPU restatement installed in place of the Eigen-based LinearNaraghiNeher
    constructor (oracle/ref_qs.cpp): the channel-state rows of every scenario."""
    from casim_b200 import configs
    from oracle import qs_oracle
    qs_params, coords = configs.quasi_stationary(20, seed=1)
    with tempfile.TemporaryDirectory() as td:
        np.savetxt(os.path.join(td, "coords.txt"), coords, fmt="%.17g")
        p = json.loads(json.dumps(qs_params))
        p["Calcium Release Site"]["Parameters"]["Channels"]["RyR"]["Coordinates"] = os.path.join(td, "coords.txt")
        added = np.ascontiguousarray(qs_oracle.naraghi_neher(qs_oracle.parse(p)))
        L = ref.lib()
        L.qsref_set_increments.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.qsref_run.restype = ctypes.c_long
        L.qsref_run.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_ulong), ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                ctypes.c_long]
        L.qsref_set_increments(len(coords), added.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        first = (np.arange(n_scen) % len(coords)).astype(np.int32)
        mr = 200000
        rt = np.zeros(mr)
        rs = np.zeros(mr * len(coords), dtype=np.int32)
        rps = np.zeros(n_scen, dtype=np.int32)
        seed = (ctypes.c_ulong * 6)(*([12345] * 6))
        tot = L.qsref_run(json.dumps(p).encode(), seed, n_scen, first.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                          rt.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), rs.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                          rps.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), mr)
        assert 0 < tot <= mr
    out = {"params": np.frombuffer(json.dumps(qs_params).encode(), dtype=np.uint8), "coords": coords,
           "increments": added, "first": first, "rows_per_scenario": rps, "row_t": rt[:tot],
           "row_states": rs[:tot * len(coords)].reshape(tot, len(coords)).astype(np.int8)}
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print("wrote", name, "rows", tot)


def main():
    global REF_DIR
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("CASIM_REFERENCE"), help="the reference tree (CaSim/, examples/)")
    ap.add_argument("--only", default=None, help="comma-separated fixture names")
    ap.add_argument("--here", action="store_true", help="run the example fixtures in this process")
    args = ap.parse_args()
    if not args.ref or not os.path.isdir(os.path.join(args.ref, "CaSim")):
        raise SystemExit("name the reference tree with --ref or CASIM_REFERENCE")
    REF_DIR = args.ref
    if not ref.available():
        raise SystemExit("oracle/_ref/libcasim_ref.so missing: run `make -C oracle ref`")
    only = set(args.only.split(",")) if args.only else None

    def want(n):
        return only is None or n in only
    if want("rng"):
        rng_fixture()
    base = reference_params()
    # 2D test config of the reference (SheepCannell, Ca + Mg, 3 buffers, sarcolemmal buffer)
    if want("ref2d_sheep"):
        run_case("ref2d_sheep", base, coords_text(), [1, 500, 3000], [7] * 6)
    # the same run longer with another seed (gating events inside the window)
    if want("ref2d_sheep_s3"):
        run_case("ref2d_sheep_s3", base, coords_text(), [12000, 16000], [3] * 6, first=5)
    # 3D cleft: 3 layers (dz = 7.5 nm keeps the explicit step stable)
    p3 = json.loads(json.dumps(base))
    p3["Dyad"]["Type"] = "CPU3D"
    p3["Dyad"]["dz"] = 7.5
    if want("ref3d_sheep"):
        run_case("ref3d_sheep", p3, coords_text(), [1, 400, 1500], [5] * 6)
    # two-state MWC gating with Mg inhibition (CaSim/TwoStateMWC.cpp)
    pm = json.loads(json.dumps(base))
    pm["Dyad"]["Channels"]["RyR"]["Model"] = "TwoStateMWC"
    pm["Dyad"]["Channels"]["RyR"]["Parameters"] = {"fCa": 0.00583687, "KCa": 4.1834575, "fMg": 3.2517014,
                                                    "KMg": 92.2954937, "KO0": 10800, "KMgI": 546.4, "kclose": 0.59}
    if want("ref2d_mwc"):
        run_case("ref2d_mwc", pm, coords_text(), [1, 2000], [11] * 6, first=3)
    # allosteric two-state gating with Mg inhibition (CaSim/TwoStateaHTG.cpp)
    pa = json.loads(json.dumps(base))
    pa["Dyad"]["Channels"]["RyR"]["Model"] = "TwoStateaHTG"
    pa["Dyad"]["Channels"]["RyR"]["Parameters"] = {"fCa": 0.00583687, "KCa": 4.1834575, "fMg": 3.2517014, "KMg": 92.2954937,
                                                    "KO0": 10800, "KMgI": 546.4, "KCL": 0.1, "KI": 0.01, "KOL": 10.0,
                                                    "kclose": 200.0}
    if want("ref2d_ahtg"):
        run_case("ref2d_ahtg", pa, coords_text(), [1, 2000], [13] * 6, first=4)
    # spline-tabulated rates (CaSim/TwoStateSplineModel.cpp, tk::spline)
    ps = json.loads(json.dumps(base))
    ps["Dyad"]["Channels"]["RyR"]["Model"] = "TwoStateSpline"
    ps["Dyad"]["Channels"]["RyR"]["Parameters"] = {}
    ps["Dyad"]["Channels"]["RyR"]["Kopen filename"] = "kopen.txt"
    ps["Dyad"]["Channels"]["RyR"]["Kclose filename"] = "kclose.txt"
    if want("ref2d_spline"):
        run_case("ref2d_spline", ps, coords_text(), [1, 1500, 3000], [17] * 6, first=6, tables=spline_tables())
    # fast gating: many open/close events in 4000 steps (identical trajectories expected)
    pf = json.loads(json.dumps(base))
    pf["Dyad"]["Channels"]["RyR"]["Parameters"].update({"kopen0": 4e5, "ncaopen": 0.5, "kopenmax": 8e5, "kclose0": 245.0 * 40})
    if want("ref2d_fastgating"):
        run_trajectory("ref2d_fastgating", pf, coords_text(), 4000, 50, [21] * 6, first=2)
    if want("qs_mwc"):
        qs_fixture("qs_mwc")
    # the reference's own example configs, loaded unchanged (two ions, three buffers,
    # spline-tabulated and 60-state MWC gating)
    # spline-tabulated and 60-state MWC gating). They name no seed, so the reference
    # takes the next stream of RngStream's process-wide package seed: each one runs in
    # a fresh process, where that is the first stream of the default package seed.
    for name, example in (("ex_spline_gpu", "SplineGPU"), ("ex_iaparov_gpu", "IaparovGPU")):
        if not want(name):
            continue
        if args.here:
            run_example(name, example, [1, 1000, 3000])
        else:
            import subprocess
            subprocess.run([sys.executable, os.path.abspath(__file__), "--ref", REF_DIR, "--only", name, "--here"], check=True)


if __name__ == "__main__":
    main()

"""Synthetic release-site workloads with the shapes of the benchmark configs.

Each builder returns ``(params, sites)``: ``params`` is a reference-schema
Parameters.json dict (the schema of CaSim/test_input/Parameters.json) and
``sites`` the per-site table (grid extents, RyR coordinates in nm, seeds,
jSR initial values, initially opened RyR). All randomness is seeded.

Units follow the reference: nm, ms, uM; D in nm^2/ms; dt in ns.
"""
import json
import math

import numpy as np

RYR_PITCH_NM = 31.0
FARADAY = 96485.33212


def ryr_conductance(pA_per_mM, v_elem_nm3):
    """Flux coefficient g (1/ms) such that J = g*(jSR - cleft) uM/ms in one
    grid element carries `pA_per_mM` picoampere per mM gradient (Ca2+, z=2)."""
    mol_per_s = pA_per_mM * 1e-12 / (2 * FARADAY)
    litres = v_elem_nm3 * 1e-24
    uM_per_ms_at_1mM = mol_per_s / litres * 1e6 * 1e-3
    return uM_per_ms_at_1mM / 1000.0


def sheep_cannell_power_law(k0_per_ms=0.1, k_half_uM=15.0, n=2.5, kclose_per_ms=1.0):
    """SheepCannell parameters for kopen = k0*(Ca/k_half)^n, kclose constant
    (CaSim/SheepCannell.cpp:12-18: rates in 1/s of Ca in mM)."""
    return {
        "kopen0": k0_per_ms * 1000.0 * (1000.0 / k_half_uM) ** n,
        "ncaopen": n,
        "kopenmax": 1e15,
        "kclose0": kclose_per_ms * 1000.0,
        "ncaclose": 0.0,
    }


# 60-state single-site MWC RyR of the reference's example (examples/IaparovGPU/Parameters.json)
SINGLE_SITE_MWC = {"KCa": 4.1834575, "KMg": 92.2954937, "KMgI": 546.4, "KO0": 10800, "alphaCa": 0, "alphaI": 0, "alphaMg": 0,
                   "alphaMgI": 0, "alphakco": 0.67057446, "alphakcoI": 0.67057446, "fCa": 0.00583687, "fCa4I": 0.00583687,
                   "fICa": 0.00583687, "fIMg": 3.2517014, "fMg": 3.2517014, "gCa": 1, "gMg": 1, "kco": 0.00110487,
                   "konCa": 0.71, "konMg": 0.0071, "konmgI": 5.9002e-07}


def with_single_site_mwc(params, speed=1.0):
    """A copy of `params` gated by the 60-state SingleSiteMWC model (CaSim/SingleSiteMWC.cpp):
    adds a Magnesium ion (1 mM, no conductance) to the dyad, jSR and NSR; `speed`
    scales the binding and opening rate constants (faster gating for short tests)."""
    p = json.loads(json.dumps(params))
    d = p["Dyad"]
    d["Ions"]["Magnesium"] = {"Concentration": 1000.0, "D": 160000.0, "Extracell": 1000.0}
    ch = d["Channels"]["RyR"]
    ch["Model"] = "SingleSiteMWC"
    par = dict(SINGLE_SITE_MWC)
    for k in ("konCa", "konMg", "kco", "konmgI"):
        par[k] *= speed
    ch["Parameters"] = par
    ch["Conductance"]["Magnesium"] = 0.0
    p["jSR"]["Ions"]["Magnesium"] = {"Binding sites of CQ": 1, "Concentration": 1000.0, "K CQ (uM)": 1.0e6, "T refill (ms)": 10.0}
    p["nSR"]["Ions"]["Magnesium"] = {"Concentration (uM)": 1000.0}
    return p


def lattice(n, cx, cy, rng, pitch=RYR_PITCH_NM, jitter=3.0):
    cols = int(math.ceil(math.sqrt(n)))
    rows = int(math.ceil(n / cols))
    xs, ys = [], []
    for k in range(n):
        i, j = k % cols, k // cols
        xs.append(cx + (i - (cols - 1) / 2.0) * pitch + rng.uniform(-jitter, jitter))
        ys.append(cy + (j - (rows - 1) / 2.0) * pitch + rng.uniform(-jitter, jitter))
    return xs, ys


def base_params(dim=2, nx=64, ny=64, dx=10.0, height=15.0, dz=7.5, dt_ns=50.0, cytosol="Pool", g=None,
                jsr_uM=1000.0, tau_refill=10.0, gating=None, sarcolemma=False):
    v_elem = dx * dx * height if dim == 2 else 0.5 * dx * dx * dz
    if g is None:
        g = ryr_conductance(0.35, dx * dx * height)
    dyad = {
        "Type": "3D" if dim == 3 else "2D",
        "dx": dx, "dy": dx, "dz": dz if dim == 3 else 5.0,
        "x": (nx - 1) * dx, "y": (ny - 1) * dx, "z": height,
        "Radius": 1000.0, "Voltage": 0.0, "Start": "Equilibrium",
        "Ions": {"Calcium": {"D": 220000.0, "Concentration": 0.1, "Extracell": 1000.0}},
        "Buffers": {
            "ATP": {"Total Concentration": 2000.0, "Ions": {"Calcium": {"D": 140000.0, "kon": 0.225, "koff": 45.0}}},
            "Fixed": {"Total Concentration": 50.0, "Ions": {"Calcium": {"D": 0.0, "kon": 0.1, "koff": 1.0}}},
        },
        "Channels": {"RyR": {
            "Model": "SheepCannell",
            "Parameters": gating or sheep_cannell_power_law(),
            "Conductance": {"Calcium": g},
            "Coordinates": "",
        }},
    }
    if sarcolemma:
        dyad["Sarcolemma"] = {"Calcium": {"N1": 0.0, "K1": 1100.0, "N2": 10666.65, "K2": 13.0}}
    if cytosol == "Pool":
        cyto = {
            "Type": "Pool", "Leak mult": 2e-06,
            "Buffers": {"Troponin": {"Total Concentration": 70.0, "Ions": {"Calcium": {"D": 0.0, "kon": 0.039, "koff": 0.02}}}},
            "SERCA": {"Calcium": {"Jmax": 0.2, "Kup": 0.2}},
        }
    else:
        cyto = {
            "Type": "RD3D", "Nodes": 25, "dx": 40.0,
            "Buffers": {"Calmodulin": {"Total Concentration": 24.0, "Ions": {"Calcium": {"D": 25000.0, "kon": 0.1, "koff": 0.038}}}},
            "SERCA": {"Calcium": {"Jmax": 0.2, "Kup": 0.2}},
        }
    return {
        "Solver": "ParallelHybridSolver",
        "dt, ns": dt_ns,
        "NumBatch": 1,
        "Dyad": dyad,
        "Cytosol": cyto,
        "jSR": {
            "Type": "Pool", "Constant": False, "Total CQ (uM)": 800.0, "V jSR (nm3)": 1e7,
            "Ions": {"Calcium": {"Binding sites of CQ": 15, "Concentration": jsr_uM, "K CQ (uM)": 600.0, "T refill (ms)": tau_refill}},
        },
        "nSR": {"Type": "ConstPool", "Ions": {"Calcium": {"Concentration (uM)": 1000.0}}},
        "_v_elem": v_elem,
    }


def _clean(params):
    return {k: v for k, v in params.items() if not k.startswith("_")}


def sites_table(nx, ny, nz, nch, xs, ys, seeds, jsr_init=None, first=None):
    S = len(nx)
    return {
        "nx": np.asarray(nx, dtype=np.int32), "ny": np.asarray(ny, dtype=np.int32), "nz": np.asarray(nz, dtype=np.int32),
        "n_ch": np.asarray(nch, dtype=np.int32),
        "ch_x": np.asarray(xs, dtype=np.float64), "ch_y": np.asarray(ys, dtype=np.float64),
        "seeds": np.asarray(seeds, dtype=np.uint32).reshape(S, 6),
        "jsr_init": None if jsr_init is None else np.asarray(jsr_init, dtype=np.float64).reshape(S, -1),
        "first_channel": np.asarray(first if first is not None else np.zeros(S), dtype=np.int32),
    }


def config1(n_sites=100, seed0=1, nx=64, ny=64, n_ryr=20):
    """2D 64x64 cleft, dx = 10 nm, 15 nm high; 20 RyRs on a 31 nm lattice with
    +-3 nm jitter; Ca + mobile ATP + fixed sites; power-law SheepCannell; one
    site per seed s = seed0 .. seed0 + n_sites - 1, seeds [s]*6."""
    p = base_params(dim=2, nx=nx, ny=ny)
    xs, ys, seeds = [], [], []
    for k in range(n_sites):
        s = seed0 + k
        rng = np.random.default_rng(s)
        x, y = lattice(n_ryr, (nx - 1) * 5.0, (ny - 1) * 5.0, rng)
        xs += x
        ys += y
        seeds.append([s] * 6)
    # RunSimulations opens channel (n_threads*i + j)/sc_per_channel (CaSim/ParallelHybridSolver.cpp:411-417)
    first = [0] * n_sites
    return _clean(p), sites_table([nx] * n_sites, [ny] * n_sites, [1] * n_sites, [n_ryr] * n_sites, xs, ys, seeds, first=first)


def config2(n_sites=4096, seed=2024, side=(40, 120), ryr=(10, 100), cytosol="RD3D"):
    """4096 3D clefts of uneven size: side ~ U{40..120} nodes at 10 nm, 3 z
    layers (dz = 7.5 nm of a 15 nm cleft); RyR count ~ U{10..100} on the
    jittered 31 nm lattice; coupled 25^3 cytosol at 40 nm with Ca, ATP, CaM."""
    p = base_params(dim=3, nx=64, ny=64, cytosol=cytosol)
    rng = np.random.default_rng(seed)
    n = rng.integers(side[0], side[1] + 1, size=n_sites)
    nr = rng.integers(ryr[0], ryr[1] + 1, size=n_sites)
    xs, ys, seeds, first = [], [], [], []
    for k in range(n_sites):
        x, y = lattice(int(nr[k]), (n[k] - 1) * 5.0, (n[k] - 1) * 5.0, rng)
        xs += x
        ys += y
        seeds.append([int(v) for v in rng.integers(1, 4294944443, size=6)])
        first.append(int(rng.integers(0, nr[k])))
    return _clean(p), sites_table(n, n, [3] * n_sites, nr, xs, ys, seeds, first=first)


def config3(n_sites=1024, seed=3, n_ryr=50):
    """1024 C1-like sites with 50 RyRs and jSR Ca ~ U[500, 1500] uM per site."""
    p = base_params(dim=2, nx=64, ny=64)
    rng = np.random.default_rng(seed)
    xs, ys, seeds, jsr = [], [], [], []
    for k in range(n_sites):
        x, y = lattice(n_ryr, 315.0, 315.0, rng)
        xs += x
        ys += y
        seeds.append([int(v) for v in rng.integers(1, 4294944443, size=6)])
        jsr.append([rng.uniform(500.0, 1500.0)])
    return _clean(p), sites_table([64] * n_sites, [64] * n_sites, [1] * n_sites, [n_ryr] * n_sites, xs, ys, seeds, jsr_init=jsr)


def with_magnesium(params):
    """A copy of `params` with a Magnesium ion (1 mM, no RyR conductance) in the
    dyad, the jSR and the NSR (the second ion of the reference's Mg-aware models)."""
    p = json.loads(json.dumps(params))
    p["Dyad"]["Ions"]["Magnesium"] = {"Concentration": 1000.0, "D": 160000.0, "Extracell": 1000.0}
    p["Dyad"]["Channels"]["RyR"]["Conductance"]["Magnesium"] = 0.0
    p["jSR"]["Ions"]["Magnesium"] = {"Binding sites of CQ": 1, "Concentration": 1000.0, "K CQ (uM)": 1.0e6, "T refill (ms)": 10.0}
    p["nSR"]["Ions"]["Magnesium"] = {"Concentration (uM)": 1000.0}
    return p


# Tetrameric MWC gating of the large sweep: Ca activation Kd 10 uM, allosteric
# coupling factor 0.1, 1 mM Mg competing at the activation site and inhibiting
# (the Po law of CaSim/TwoStateMWC.cpp:15-23; fMg, KMg, KMgI as the reference's
# example model, KO0 and kclose chosen for the sweep)
SWEEP_MWC = {"fCa": 0.1, "KCa": 10.0, "fMg": 3.2517014, "KMg": 92.2954937, "KO0": 1000.0, "KMgI": 546.4, "kclose": 1.0}


def mwc_open_rate(ca, mg=1000.0, par=SWEEP_MWC):
    """kopen(Ca) of the TwoStateMWC law: kclose * Po / (1 - Po) (1/ms)."""
    ca = np.asarray(ca, dtype=np.float64)
    inac = par["KMgI"] ** 2 / (par["KMgI"] ** 2 + mg * mg)
    a = (ca + par["KCa"] * par["fCa"] * (1 + mg / (par["fMg"] * par["KMg"]))) ** 4
    b = par["KO0"] * (par["fCa"] * (ca + par["KCa"] * (1 + mg / par["KMg"]))) ** 4
    po = inac * a / (a + b)
    return par["kclose"] * po / (1 - po)


def sweep_spline_tables(directory):
    """Rate tables of the spline-gated half: kopen(Ca) tabulated from the MWC law
    at 0 and 160 log-spaced Ca values in [0.01, 5000] uM, kclose constant.
    Returns the (kopen, kclose) file paths."""
    import os
    ca = np.concatenate([[0.0], np.logspace(-2, np.log10(5000.0), 160)])
    paths = []
    for name, y in (("kopen_mwc.txt", mwc_open_rate(ca)), ("kclose_mwc.txt", np.full(ca.size, SWEEP_MWC["kclose"]))):
        path = os.path.join(directory, name)
        np.savetxt(path, np.column_stack([ca, y]), fmt="%.17g")
        paths.append(path)
    return paths


def subset_sites(sites, idx):
    """The sites table restricted to the sites `idx`, in that order."""
    idx = np.asarray(idx, dtype=np.int64)
    off = np.concatenate([[0], np.cumsum(sites["n_ch"])])
    ch = np.concatenate([np.arange(off[k], off[k + 1]) for k in idx]) if idx.size else np.zeros(0, np.int64)
    out = {k: (None if sites.get(k) is None else np.asarray(sites[k])[idx])
           for k in ("nx", "ny", "nz", "n_ch", "seeds", "jsr_init", "first_channel")}
    out["ch_x"] = np.asarray(sites["ch_x"])[ch]
    out["ch_y"] = np.asarray(sites["ch_y"])[ch]
    return out


def config5(n_sites=16384, seed=5, side=(40, 120), ryr=(10, 150), cytosol="RD3D", table_dir=None):
    """Large sweep: 3D clefts as config 2 (side ~ U{40..120} x 3 layers, 25^3
    RD cytosol) with RyR count ~ U{10..150}, capped at the jittered 31 nm
    lattice that fits inside the rim; 1 mM Mg. Returns two halves, each
    (params, sites): the first gated by the tetrameric MWC law (SWEEP_MWC),
    the second by the same law tabulated for TwoStateSpline (tables written
    to `table_dir`, a temporary directory by default)."""
    import tempfile
    rng = np.random.default_rng(seed)
    n = rng.integers(side[0], side[1] + 1, size=n_sites)
    fit = (np.floor((n - 5) * 10.0 / RYR_PITCH_NM) + 1) ** 2
    nr = np.minimum(rng.integers(ryr[0], ryr[1] + 1, size=n_sites), fit).astype(np.int64)
    xs, ys, seeds, first = [], [], [], []
    for k in range(n_sites):
        x, y = lattice(int(nr[k]), (n[k] - 1) * 5.0, (n[k] - 1) * 5.0, rng)
        xs.append(x)
        ys.append(y)
        seeds.append([int(v) for v in rng.integers(1, 4294944443, size=6)])
        first.append(int(rng.integers(0, nr[k])))
    base = with_magnesium(base_params(dim=3, nx=64, ny=64, cytosol=cytosol))
    pm = json.loads(json.dumps(base))
    pm["Dyad"]["Channels"]["RyR"]["Model"] = "TwoStateMWC"
    pm["Dyad"]["Channels"]["RyR"]["Parameters"] = dict(SWEEP_MWC)
    ps = json.loads(json.dumps(base))
    kopen, kclose = sweep_spline_tables(table_dir or tempfile.mkdtemp(prefix="casim_sweep_"))
    ps["Dyad"]["Channels"]["RyR"]["Model"] = "TwoStateSpline"
    ps["Dyad"]["Channels"]["RyR"]["Parameters"] = {}
    ps["Dyad"]["Channels"]["RyR"]["Kopen filename"] = kopen
    ps["Dyad"]["Channels"]["RyR"]["Kclose filename"] = kclose
    halves = []
    for p, idx in ((pm, range(0, n_sites // 2)), (ps, range(n_sites // 2, n_sites))):
        idx = list(idx)
        cx = [v for k in idx for v in xs[k]]
        cy = [v for k in idx for v in ys[k]]
        halves.append((_clean(p), sites_table(n[idx], n[idx], [3] * len(idx), nr[idx], cx, cy, [seeds[k] for k in idx],
                                              first=[first[k] for k in idx])))
    return halves


def small_mixed(n_sites=6, seed=11, dim=2, cytosol="Pool", side=(12, 24), ryr=(2, 9)):
    """Small uneven sites for parity tests at sizes the oracle finishes in seconds."""
    p = base_params(dim=dim, nx=16, ny=16, cytosol=cytosol, sarcolemma=True)
    if cytosol == "RD3D":
        p["Cytosol"]["Nodes"] = 9
    rng = np.random.default_rng(seed)
    n = rng.integers(side[0], side[1] + 1, size=n_sites)
    m = rng.integers(side[0], side[1] + 1, size=n_sites)
    nr = rng.integers(ryr[0], ryr[1] + 1, size=n_sites)
    xs, ys, seeds, first, jsr = [], [], [], [], []
    for k in range(n_sites):
        cols = int(math.ceil(math.sqrt(nr[k])))
        pitch = min(RYR_PITCH_NM, (min(n[k], m[k]) - 5) * 10.0 / max(cols, 1))
        x, y = lattice(int(nr[k]), (n[k] - 1) * 5.0, (m[k] - 1) * 5.0, rng, pitch=pitch, jitter=2.0)
        xs += x
        ys += y
        seeds.append([int(v) for v in rng.integers(1, 4294944443, size=6)])
        first.append(int(rng.integers(0, nr[k])))
        jsr.append([rng.uniform(700.0, 1300.0)])
    nz = [3] * n_sites
    return _clean(p), sites_table(n, m, nz, nr, xs, ys, seeds, jsr_init=jsr, first=first)


def quasi_stationary(n_ryr=20, seed=1, max_time=50.0, coordinates="coords.txt"):
    """A quasi-stationary release site in the reference's ParallelSolver schema
    ("Calcium Release Site", LinearNaraghiNeher): n_ryr RyRs on the jittered lattice,
    TwoStateMWC gating at 1 mM Mg, ATP and calmodulin buffering, 4 pA per open RyR.
    Returns (params, coords [n_ryr, 2] in nm); write coords to `coordinates`, relative
    to the base directory given to QuasiStationarySites."""
    xs, ys = lattice(n_ryr, 150.0, 150.0, np.random.default_rng(seed))
    params = {"Calcium Release Site": {
        "Type": "QuasyStationary", "Name": "LinearNaraghiNeher", "Max Time": float(max_time),
        "Parameters": {
            "Channels": {"RyR": {"Coordinates": coordinates, "Model": "TwoStateMWC", "Current": 4.0,
                                 "Parameters": {"fCa": 0.00583687, "KCa": 4.1834575, "fMg": 3.2517014, "KMg": 92.2954937,
                                                "KO0": 10800, "KMgI": 546.4, "kclose": 0.59}}},
            "Dyadic Cleft": {"Ions": {"Calcium": {"Concentration": 0.1, "D": 2.2e-6}, "Magnesium": {"Concentration": 1000.0}},
                             "Buffers": {"ATP": {"kon": 0.225, "koff": 45.0, "D": 1.408e-6, "Total Concentration": 2000.0},
                                         "Calmodulin": {"kon": 0.1, "koff": 0.038, "D": 2.42e-7, "Total Concentration": 24.0}}},
            "Open Concentration": 100.0}}}
    return params, np.c_[xs, ys]

"""Python front end of the CPU restatement (oracle/casim_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the checker, never by the product package.

`build_model(params)` resolves a reference-schema Parameters.json dict into the
flat `or_model` struct, independently of the product's own C++ parser:
  * JSON objects iterate in sorted key order, as nlohmann::json's default
    std::map does in the reference (e.g. CaSim/DyadRD2DCPU.cpp:34-41);
  * ion-buffer pairs are ordered ion-major, buffer-minor
    (CaSim/DyadRD2DCPU.cpp:83-99);
  * equilibrium bound concentrations come from the reference's Gauss
    elimination (CaSim/DyadRD2DCPU.cpp:157-187) with a floating abs();
  * RyR positions snap to the grid with Point::GetCoordsOnGrid
    (CaSim/Point.cpp:17-23).
"""
import ctypes
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")

MAX_IONS, MAX_BUF, MAX_PAIRS, MAX_CBUF, MAX_CPAIRS, MAX_CHPAR, MAX_SPLINE = 4, 8, 16, 12, 24, 32, 1024
SHEEP_CANNELL, TWO_STATE_MWC, TWO_STATE_AHTG, TWO_STATE_SPLINE, FOUR_STATE_MWC, SINGLE_SITE_MWC = 0, 1, 2, 3, 4, 5
CYTO_POOL, CYTO_RD3D = 0, 1

_D = ctypes.c_double
_I = ctypes.c_int


class OrModel(ctypes.Structure):
    _fields_ = [
        ("dim", _I),
        ("dx", _D), ("dy", _D), ("dz", _D), ("z", _D), ("R", _D), ("dt", _D), ("voltage", _D),
        ("n_ions", _I),
        ("D_ion", _D * MAX_IONS), ("Cb_ion", _D * MAX_IONS), ("extracell", _D * MAX_IONS),
        ("has_sl", _I * MAX_IONS),
        ("N1", _D * MAX_IONS), ("K1", _D * MAX_IONS), ("N2", _D * MAX_IONS), ("K2", _D * MAX_IONS),
        ("n_buf", _I),
        ("Ctot", _D * MAX_BUF),
        ("binds", _I * (MAX_BUF * MAX_IONS)),
        ("n_pairs", _I),
        ("pair_ion", _I * MAX_PAIRS), ("pair_buf", _I * MAX_PAIRS),
        ("D_pair", _D * MAX_PAIRS), ("kon", _D * MAX_PAIRS), ("koff", _D * MAX_PAIRS), ("pair_init", _D * MAX_PAIRS),
        ("ch_model", _I),
        ("ch_par", _D * MAX_CHPAR),
        ("g", _D * MAX_IONS),
        ("ca_idx", _I), ("mg_idx", _I),
        ("sp_n", _I * 2),
        ("sp_x", (_D * MAX_SPLINE) * 2),
        ("sp_c", ((_D * 4) * MAX_SPLINE) * 2),
        ("sp_left", (_D * 3) * 2), ("sp_right", (_D * 3) * 2),
        ("jsr_const", _I),
        ("CQ", _D), ("V_jsr", _D),
        ("nCQ", _I * MAX_IONS),
        ("K_CQ", _D * MAX_IONS), ("tau_refill", _D * MAX_IONS), ("jsr0", _D * MAX_IONS),
        ("nsr", _D * MAX_IONS),
        ("cyto_type", _I),
        ("c_bg", _D * MAX_IONS), ("c_onetau_ion", _D * MAX_IONS),
        ("c_n_buf", _I),
        ("c_Ctot", _D * MAX_CBUF),
        ("c_binds", _I * (MAX_CBUF * MAX_IONS)),
        ("c_n_pairs", _I),
        ("c_kon", _D * MAX_CPAIRS), ("c_koff", _D * MAX_CPAIRS), ("c_init", _D * MAX_CPAIRS),
        ("c_onetau_pair", _D * MAX_CPAIRS),
        ("c_D_pair", _D * MAX_CPAIRS),
        ("c_in_dyad", _I * MAX_CPAIRS),
        ("c_dyad_pair", _I * MAX_CPAIRS),
        ("c_serca", _I * MAX_IONS),
        ("c_Jmax", _D * MAX_IONS), ("c_Kup", _D * MAX_IONS),
        ("mc", _I),
        ("hc", _D),
    ]


def gauss_elimination(a):
    """CaSim/DyadRD2DCPU.cpp:157-187 with floating |.| (the MSVC meaning)."""
    a = [list(map(float, r)) for r in a]
    n = len(a)
    m = len(a[0]) - 1
    where = [-1] * m
    row = 0
    for col in range(m):
        if row >= n:
            break
        sel = row
        for i in range(row, n):
            if abs(a[i][col]) > abs(a[sel][col]):
                sel = i
        if abs(a[sel][col]) < 1e-10:
            continue
        for i in range(col, m + 1):
            a[sel][i], a[row][i] = a[row][i], a[sel][i]
        where[col] = row
        for i in range(n):
            if i != row:
                c = a[i][col] / a[row][col]
                for j in range(col, m + 1):
                    a[i][j] -= a[row][j] * c
        row += 1
    ans = [0.0] * m
    for i in range(m):
        if where[i] != -1:
            ans[i] = a[where[i]][m] / a[where[i]][i]
    return ans


def _sorted_items(d):
    return sorted((d or {}).items(), key=lambda kv: kv[0])


def _equilibrium(ions, buf, start_equilibrium):
    """Bound concentrations of one buffer (CaSim/DyadRD2DCPU.cpp:47-81)."""
    kin = buf["Ions"]
    bound = [(iname, Cb) for iname, Cb in ions if iname in kin]
    n = len(kin)
    out = {}
    if not start_equilibrium or n == 0:
        return {iname: 0.0 for iname, _ in bound}
    a = [[0.0] * (n + 1) for _ in range(n)]
    for it, (iname, Cb) in enumerate(bound):
        k = kin[iname]
        for I in range(n):
            a[it][I] = k["kon"] * Cb
            if I == it:
                a[it][I] += k["koff"]
        a[it][n] = k["kon"] * Cb * buf["Total Concentration"]
    c = gauss_elimination(a)
    for t, (iname, _) in enumerate(bound):
        out[iname] = c[t]
    return out


def grid_index(coord, h):
    """Point::GetCoordsOnGrid (CaSim/Point.cpp:17-23)."""
    return int((coord + 0.5 * h) / h)


def natural_spline(x, y):
    """Natural cubic spline (zero second derivative at both ends) through (x, y):
    per interval [a, b, c, d] with y(x_i + h) = a + b h + c h^2 + d h^3, from the
    tridiagonal system for c_i = y''(x_i) / 2; plus the value, slope and c at the
    last knot for extrapolation."""
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    n = len(x)
    h = np.diff(x)
    A = np.zeros((n, n))
    r = np.zeros(n)
    A[0, 0] = A[n - 1, n - 1] = 2.0
    for i in range(1, n - 1):
        A[i, i - 1] = h[i - 1] / 3.0
        A[i, i] = 2.0 * (h[i - 1] + h[i]) / 3.0
        A[i, i + 1] = h[i] / 3.0
        r[i] = (y[i + 1] - y[i]) / h[i] - (y[i] - y[i - 1]) / h[i - 1]
    c = np.linalg.solve(A, r)
    b = np.zeros(n)
    d = np.zeros(n)
    for i in range(n - 1):
        d[i] = (c[i + 1] - c[i]) / (3.0 * h[i])
        b[i] = (y[i + 1] - y[i]) / h[i] - h[i] * (2.0 * c[i] + c[i + 1]) / 3.0
    hl = h[-1]
    b[n - 1] = 3.0 * d[n - 2] * hl * hl + 2.0 * c[n - 2] * hl + b[n - 2]
    return np.c_[y, b, c, d], (y[0], b[0], 0.0), (y[n - 1], b[n - 1], 0.0)


def _set_spline(m, w, x, y):
    if len(x) > MAX_SPLINE:
        raise ValueError("spline table longer than the oracle holds")
    coef, left, right = natural_spline(x, y)
    m.sp_n[w] = len(x)
    for i in range(len(x)):
        m.sp_x[w][i] = x[i]
        for k in range(4):
            m.sp_c[w][i][k] = coef[i, k]
    for k in range(3):
        m.sp_left[w][k] = left[k]
        m.sp_right[w][k] = right[k]


def build_model(params):
    d = params["Dyad"]
    m = OrModel()
    dtype = d.get("Type", "2D")
    m.dim = 3 if dtype in ("3D", "CPU3D") else 2
    m.dx, m.dy = float(d["dx"]), float(d["dy"])
    m.dz = float(d.get("dz", 1.0))
    m.z = float(d["z"])
    m.R = float(d["Radius"])
    m.voltage = float(d.get("Voltage", 0.0))
    m.dt = float(params["dt, ns"]) * 1e-6
    ions = _sorted_items(d["Ions"])
    m.n_ions = len(ions)
    ion_names = [k for k, _ in ions]
    m.ca_idx = ion_names.index("Calcium") if "Calcium" in ion_names else -1
    m.mg_idx = ion_names.index("Magnesium") if "Magnesium" in ion_names else -1
    for i, (name, p) in enumerate(ions):
        m.D_ion[i] = p["D"]
        m.Cb_ion[i] = p["Concentration"]
        m.extracell[i] = p.get("Extracell", 0.0)
    sl = d.get("Sarcolemma", {})
    for i, name in enumerate(ion_names):
        if name in sl:
            m.has_sl[i] = 1
            m.N1[i], m.K1[i], m.N2[i], m.K2[i] = sl[name]["N1"], sl[name]["K1"], sl[name]["N2"], sl[name]["K2"]
    start_eq = d.get("Start") == "Equilibrium"
    ion_cb = [(k, v["Concentration"]) for k, v in ions]
    bufs = _sorted_items(d["Buffers"])
    m.n_buf = len(bufs)
    eq = {}
    for b, (bname, bp) in enumerate(bufs):
        m.Ctot[b] = bp["Total Concentration"]
        eq[bname] = _equilibrium(ion_cb, bp, start_eq)
    pairs = []
    for i, iname in enumerate(ion_names):
        for b, (bname, bp) in enumerate(bufs):
            if iname in bp["Ions"]:
                m.binds[b + i * m.n_buf] = 1
                k = bp["Ions"][iname]
                p = len(pairs)
                m.pair_ion[p], m.pair_buf[p] = i, b
                m.D_pair[p], m.kon[p], m.koff[p] = k["D"], k["kon"], k["koff"]
                m.pair_init[p] = eq[bname][iname]
                pairs.append((iname, bname))
    m.n_pairs = len(pairs)
    # channels
    ch = list(_sorted_items(d["Channels"]))[0][1]
    model = ch["Model"]
    par = ch.get("Parameters", {})
    if model == "SheepCannell":
        m.ch_model = SHEEP_CANNELL
        vals = [par["kopen0"], par["ncaopen"], par["kopenmax"], par["kclose0"], par["ncaclose"]]
    elif model == "TwoStateMWC":
        m.ch_model = TWO_STATE_MWC
        vals = [par[k] for k in ("fCa", "KCa", "fMg", "KMg", "KO0", "KMgI", "kclose")]
    elif model == "TwoStateaHTG":
        m.ch_model = TWO_STATE_AHTG
        vals = [par[k] for k in ("fCa", "KCa", "fMg", "KMg", "KO0", "KMgI", "KCL", "KI", "KOL", "kclose")]
    elif model == "TwoStateSpline":
        # CaSim/TwoStateSplineModel.cpp:4-34: natural cubic splines through the
        # (Ca, rate) tables, linear extrapolation beyond the ends
        m.ch_model = TWO_STATE_SPLINE
        vals = []
        for w, key in enumerate(("Kopen filename", "Kclose filename")):
            tab = np.loadtxt(ch[key]).reshape(-1, 2)
            _set_spline(m, w, tab[:, 0], tab[:, 1])
    elif model == "SingleSiteMWC":
        # CaSim/SingleSiteMWC.cpp:5-37 (names absent from the map read as 0)
        m.ch_model = SINGLE_SITE_MWC
        vals = [float(par.get(k, 0.0)) for k in ("fCa4I", "fCa", "KCa", "alphaCa", "konCa", "fMg", "KMg", "konMg", "alphaMg",
                                                 "alphaMgI", "KO0", "alphakco", "alphakcoI", "kco", "KMgI", "konmgI", "fICa",
                                                 "fIMg", "gMg", "gCa")]
    else:
        raise ValueError("gating model not supported by the oracle: " + model)
    for k, v in enumerate(vals):
        m.ch_par[k] = v
    cond = dict(ch["Conductance"])
    for i, name in enumerate(ion_names):
        m.g[i] = cond.get(name, 0.0)
    # jSR
    j = params["jSR"]
    m.jsr_const = 1 if j.get("Constant", False) else 0
    m.CQ = j["Total CQ (uM)"]
    m.V_jsr = j["V jSR (nm3)"]
    for i, name in enumerate(ion_names):
        if name in j["Ions"]:
            p = j["Ions"][name]
            m.nCQ[i], m.K_CQ[i], m.tau_refill[i], m.jsr0[i] = p["Binding sites of CQ"], p["K CQ (uM)"], p["T refill (ms)"], p["Concentration"]
        else:
            m.nCQ[i], m.K_CQ[i], m.tau_refill[i], m.jsr0[i] = 0, 0.0, 1.0, 0.0
    nsr = [v["Concentration (uM)"] for _, v in _sorted_items(params["nSR"]["Ions"])]
    for i in range(m.n_ions):
        m.nsr[i] = nsr[i] if i < len(nsr) else 0.0
    # cytosol (CaSim/CytosolPool.cpp:1-155)
    c = params["Cytosol"]
    ctype = c.get("Type", "Pool")
    m.cyto_type = CYTO_RD3D if ctype == "RD3D" else CYTO_POOL
    leak = float(c.get("Leak mult", 0.0))
    for i, (name, p) in enumerate(ions):
        m.c_bg[i] = p["Concentration"]
        m.c_onetau_ion[i] = leak * p["D"]
    # RD3D keeps only diffusing dyad buffers in the cytosol (this project's definition)
    dyad_cb = [(n, b, True) for n, b in bufs
               if m.cyto_type == CYTO_POOL or any(k["D"] > 0 for k in b["Ions"].values())]
    cbufs = dyad_cb + [(n, b, False) for n, b in _sorted_items(c.get("Buffers", {}))]
    m.c_n_buf = len(cbufs)
    ceq = {n: _equilibrium(ion_cb, b, start_eq) for n, b, _ in cbufs}
    cp = 0
    dyad_pair_of = {pr: k for k, pr in enumerate(pairs)}
    for i, iname in enumerate(ion_names):
        for b, (bname, bp, indyad) in enumerate(cbufs):
            m.c_Ctot[b] = bp["Total Concentration"]
            if iname in bp["Ions"]:
                m.c_binds[b + i * m.c_n_buf] = 1
                k = bp["Ions"][iname]
                m.c_kon[cp], m.c_koff[cp] = k["kon"], k["koff"]
                m.c_D_pair[cp] = k["D"]
                m.c_init[cp] = ceq[bname][iname]
                m.c_onetau_pair[cp] = leak * k["D"]
                m.c_in_dyad[cp] = 1 if indyad else 0
                m.c_dyad_pair[cp] = dyad_pair_of[(iname, bname)] if indyad else -1
                cp += 1
    m.c_n_pairs = cp
    serca = c.get("SERCA", {})
    s = 0
    for i, name in enumerate(ion_names):
        if name in serca:
            m.c_serca[i] = 1
            m.c_Jmax[s], m.c_Kup[s] = serca[name]["Jmax"], serca[name]["Kup"]
            s += 1
    if m.cyto_type == CYTO_RD3D:
        m.mc = int(c["Nodes"])
        m.hc = float(c["dx"])
    return m


def _lib():
    L = ctypes.CDLL(LIB_PATH)
    vp, ip, dp, up = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint32)
    L.or_create.restype = vp
    L.or_create.argtypes = [ctypes.POINTER(OrModel), _I, ip, ip, ip, ip, ip, up, dp]
    L.or_destroy.argtypes = [vp]
    L.or_reset.argtypes = [vp]
    L.or_init_opening.argtypes = [vp, _I, _I]
    L.or_update.argtypes = [vp]
    L.or_start.argtypes = [vp, ip]
    L.or_step.argtypes = [vp, ctypes.c_long, _I]
    L.or_site_nodes.argtypes = [vp, _I]
    L.or_site_nodes.restype = ctypes.c_long
    for f in ("or_get_field", "or_get_mouth"):
        getattr(L, f).argtypes = [vp, _I, _I, dp]
    L.or_get_states.argtypes = [vp, _I, ip]
    L.or_get_micro.argtypes = [vp, _I, ip]
    for f in ("or_get_jsr", "or_get_total_current", "or_get_efflux", "or_get_cyto"):
        getattr(L, f).argtypes = [vp, _I, dp]
    L.or_get_cyto_field.argtypes = [vp, _I, _I, dp]
    L.or_get_cyto_field.restype = ctypes.c_long
    L.or_draws.argtypes = [vp, _I]
    L.or_draws.restype = ctypes.c_uint64
    L.or_release.argtypes = [vp, _I]
    L.or_release.restype = ctypes.c_double
    L.or_mrg_u01d.argtypes = [up, ctypes.c_long, dp]
    L.or_mrg_jump.argtypes = [up, _I, ctypes.c_long, up]
    return L


_L = None


def lib():
    global _L
    if _L is None:
        _L = _lib()
    return _L


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def mrg_u01d(seed, n):
    s = np.asarray(seed, dtype=np.uint32)
    out = np.zeros(n, dtype=np.float64)
    lib().or_mrg_u01d(_p(s, ctypes.c_uint32), n, _p(out, ctypes.c_double))
    return out


def mrg_jump(seed, log2_steps, mult=1):
    s = np.asarray(seed, dtype=np.uint32)
    out = np.zeros(6, dtype=np.uint32)
    lib().or_mrg_jump(_p(s, ctypes.c_uint32), log2_steps, mult, _p(out, ctypes.c_uint32))
    return out


class OracleSim:
    """Batch of independent sites stepped by the CPU restatement.

    sites: dict with int arrays nx, ny, nz, n_ch; ch_x, ch_y (nm, concatenated
    per site); seeds (S x 6 uint32); optional jsr_init (S x n_ions)."""

    def __init__(self, params, sites):
        self.model = build_model(params)
        m = self.model
        self.S = len(sites["nx"])
        nx = np.asarray(sites["nx"], dtype=np.int32)
        ny = np.asarray(sites["ny"], dtype=np.int32)
        nz = np.asarray(sites.get("nz", np.ones(self.S)), dtype=np.int32)
        nch = np.asarray(sites["n_ch"], dtype=np.int32)
        cx = np.asarray(sites["ch_x"], dtype=np.float64)
        cy = np.asarray(sites["ch_y"], dtype=np.float64)
        xyz = np.zeros((len(cx), 3), dtype=np.int32)
        for k in range(len(cx)):
            xyz[k, 0] = grid_index(cx[k], m.dx)
            xyz[k, 1] = grid_index(cy[k], m.dy)
            xyz[k, 2] = 0
        self.ch_xyz = xyz
        seeds = np.ascontiguousarray(np.asarray(sites["seeds"], dtype=np.uint32).reshape(self.S, 6))
        jsr = sites.get("jsr_init")
        jsr_arr = None if jsr is None else np.ascontiguousarray(np.asarray(jsr, dtype=np.float64).reshape(self.S, m.n_ions))
        self._keep = (nx, ny, nz, nch, xyz, seeds, jsr_arr)
        self.nx, self.ny, self.nz, self.nch = nx, ny, (nz if m.dim == 3 else np.ones_like(nz)), nch
        self.h = lib().or_create(ctypes.byref(m), self.S, _p(nx, _I), _p(ny, _I), _p(nz, _I), _p(nch, _I),
                                 _p(xyz, _I), _p(seeds, ctypes.c_uint32),
                                 None if jsr_arr is None else _p(jsr_arr, ctypes.c_double))

    def close(self):
        if getattr(self, "h", None):
            lib().or_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def start(self, first_channel):
        fc = np.asarray(first_channel, dtype=np.int32)
        lib().or_start(self.h, _p(fc, _I))

    def step(self, n, threads=1):
        lib().or_step(self.h, int(n), int(threads))

    @property
    def n_species(self):
        return self.model.n_ions + self.model.n_pairs + self.model.n_buf

    def field(self, site, species):
        """Site field in reference node order (y fastest in 2D, z fastest in 3D)."""
        n = lib().or_site_nodes(self.h, site)
        out = np.zeros(n, dtype=np.float64)
        lib().or_get_field(self.h, site, species, _p(out, ctypes.c_double))
        return out

    def mouth(self, site, species):
        out = np.zeros(int(self.nch[site]), dtype=np.float64)
        lib().or_get_mouth(self.h, site, species, _p(out, ctypes.c_double))
        return out

    def states(self, site):
        out = np.zeros(int(self.nch[site]), dtype=np.int32)
        lib().or_get_states(self.h, site, _p(out, _I))
        return out

    def micro_states(self, site):
        out = np.zeros(int(self.nch[site]), dtype=np.int32)
        lib().or_get_micro(self.h, site, _p(out, _I))
        return out

    def _vec(self, fn, site, n):
        out = np.zeros(n, dtype=np.float64)
        getattr(lib(), fn)(self.h, site, _p(out, ctypes.c_double))
        return out

    def jsr(self, site):
        return self._vec("or_get_jsr", site, self.model.n_ions)

    def total_current(self, site):
        return self._vec("or_get_total_current", site, self.model.n_ions)

    def efflux(self, site):
        return self._vec("or_get_efflux", site, self.model.n_ions + self.model.n_pairs)

    def cyto(self, site):
        return self._vec("or_get_cyto", site, self.model.n_ions + self.model.c_n_pairs)

    def cyto_field(self, site, species):
        n = lib().or_get_cyto_field(self.h, site, species, None)
        out = np.zeros(n, dtype=np.float64)
        lib().or_get_cyto_field(self.h, site, species, _p(out, ctypes.c_double))
        return out

    def draws(self, site):
        return int(lib().or_draws(self.h, site))

    def release(self, site):
        return float(lib().or_release(self.h, site))

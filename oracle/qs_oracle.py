"""CPU restatement of the reference's quasi-stationary release-site path
(CaSim/ParallelSolver.cpp:51-143, CaSim/QuasyStationaryReleaseSite.cpp:89-133,
CaSim/LinearNaraghiNeher.cpp:9-75). Test infrastructure: the checker of the
device path (casim_b200.QuasiStationarySites).

* naraghi_neher: the increments added[i][j] as the reference forms them: B =
  -D^-1 A, its eigen-decomposition (numpy's general eigensolver here, the
  reference's Eigen EigenSolver there; both take real parts), the smallest
  eigenvalue swapped to the last position with the reference's arithmetic swap,
  amplitudes a = E^-1 (0, .., I / (4 pi F D_Ca)), and the sum over the modes.
* run: one scenario of the Gillespie loop, in C (or_qs_run in casim_oracle.c),
  with the oracle's rate laws (the reference's pow forms).
"""
import ctypes
import json
import os

import numpy as np

from . import oracle

FAR = 96485.33e-6


def parse(params, base_dir=None):
    """(model, n_ch, positions, background Ca, Mg, max_time, increment inputs) of a
    ParallelSolver config ("Calcium Release Site")."""
    crs = params["Calcium Release Site"]
    par = crs["Parameters"]
    (name, ch), = par["Channels"].items()
    path = ch["Coordinates"]
    if base_dir and not os.path.isabs(path):
        path = os.path.join(base_dir, path)
    xy = np.loadtxt(path, ndmin=2)
    ions = par["Dyadic Cleft"]["Ions"]
    buffers = sorted(par["Dyadic Cleft"].get("Buffers", {}).items())
    m = oracle.OrModel()
    keys = {"TwoStateMWC": (1, ("fCa", "KCa", "fMg", "KMg", "KO0", "KMgI", "kclose")),
            "TwoStateaHTG": (2, ("fCa", "KCa", "fMg", "KMg", "KO0", "KMgI", "KCL", "KI", "KOL", "kclose")),
            "SheepCannell": (0, ("kopen0", "ncaopen", "kopenmax", "kclose0", "ncaclose"))}
    code, names = keys[ch["Model"]]
    m.ch_model = code
    for k, nm in enumerate(names):
        m.ch_par[k] = float(ch["Parameters"][nm])
    m.ca_idx, m.mg_idx = 0, 1
    return {"model": m, "xy": xy, "bg": float(ions["Calcium"]["Concentration"]), "dca": float(ions["Calcium"]["D"]),
            "mg": float(ions.get("Magnesium", {}).get("Concentration", 0.0)), "max_time": float(crs["Max Time"]),
            "current": float(ch["Current"]), "ca_open": float(par["Open Concentration"]), "buffers": buffers}


def naraghi_neher(cfg):
    """added[i][j], CaSim/LinearNaraghiNeher.cpp:9-75."""
    c0, dca = cfg["bg"], cfg["dca"]
    k, tau, d = [], [], []
    for _, b in cfg["buffers"]:
        K = b["koff"] / b["kon"]
        k.append(b["Total Concentration"] * K / ((K + c0) * (K + c0)))
        tau.append(1 / (b["koff"] + b["kon"] * c0))
        d.append(b["D"])
    nb = len(k)
    Dm = np.zeros((nb + 1, nb + 1))
    for i in range(nb):
        Dm[i, i] = d[i]
    Dm[nb, nb] = dca
    AA = np.zeros((nb + 1, nb + 1))
    for i in range(nb):
        AA[i, i] = -1 / tau[i]
        AA[i, nb] = k[i] / tau[i]
        AA[nb, i] = -AA[i, i]
        AA[nb, nb] -= AA[i, nb]
    B = -np.linalg.inv(Dm) @ AA
    mu_c, vec_c = np.linalg.eig(B)
    mu = np.real(mu_c).copy()
    eigv = np.real(vec_c).copy()
    mi = int(np.argmin(mu))
    # the reference's arithmetic swap of mu(min) and mu(last), and of their columns
    mu[mi] += mu[nb]
    mu[nb] = mu[mi] - mu[nb]
    mu[mi] -= mu[nb]
    eigv[:, [mi, nb]] = eigv[:, [nb, mi]]
    u = np.zeros(nb + 1)
    u[nb] = cfg["current"] / (4 * np.arccos(-1.0) * FAR * dca)
    aa = np.linalg.solve(eigv, u)
    xy = cfg["xy"]
    n = len(xy)
    added = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            r = float(np.sqrt((xy[i, 0] - xy[j, 0]) ** 2 + (xy[i, 1] - xy[j, 1]) ** 2))
            if r > 1e-6:
                added[i, j] = sum(1 / r * aa[q] * np.exp(-r * np.sqrt(abs(mu[q])) * 1e-8) * eigv[nb, q] * 1e-4
                                  for q in range(nb + 1))
            else:
                added[i, j] = cfg["ca_open"]
    return added


def _qs_lib():
    L = oracle.lib()
    if not hasattr(L, "_qs_ready"):
        L.or_qs_run.restype = ctypes.c_long
        L.or_qs_run.argtypes = [ctypes.POINTER(oracle.OrModel), ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                                ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_uint32), ctypes.c_int, ctypes.c_long,
                                ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                ctypes.POINTER(ctypes.c_uint64)]
        L._qs_ready = True
    return L


def run(cfg, added, seed6, first, max_events=1 << 16):
    """One scenario; returns (times, channels, states, draws, seed6 after the run)."""
    L = _qs_lib()
    n = len(cfg["xy"])
    a = np.ascontiguousarray(added, dtype=np.float64)
    s = np.ascontiguousarray(seed6, dtype=np.uint32).copy()
    t = np.zeros(max_events)
    c = np.zeros(max_events, dtype=np.int32)
    st = np.zeros(max_events, dtype=np.int32)
    draws = ctypes.c_uint64()
    P = lambda x, ty: x.ctypes.data_as(ctypes.POINTER(ty))
    ne = L.or_qs_run(ctypes.byref(cfg["model"]), n, P(a, ctypes.c_double), cfg["bg"], cfg["mg"], cfg["max_time"],
                     P(s, ctypes.c_uint32), int(first), max_events, P(t, ctypes.c_double), P(c, ctypes.c_int),
                     P(st, ctypes.c_int), ctypes.byref(draws))
    ne = min(ne, max_events)
    return t[:ne].copy(), c[:ne].copy(), st[:ne].copy(), int(draws.value), s


def stream_seeds(n, package=(12345,) * 6):
    """Stream s of the package seed, s < n (2^127 apart)."""
    out = np.zeros((n, 6), dtype=np.uint32)
    cur = np.asarray(package, dtype=np.uint32)
    L = oracle.lib()
    for k in range(n):
        out[k] = cur
        nxt = np.zeros(6, dtype=np.uint32)
        L.or_mrg_jump(cur.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), 127, 1, nxt.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
        cur = nxt
    return out


def naraghi_neher_exact(cfg, digits=50):
    """naraghi_neher in mpmath at `digits` significant digits, the same steps: the
    yardstick for the two double-precision eigen-solves (one mode of B is the
    conserved total, eigenvalue 0, so either solve carries ~1e-11 relative error)."""
    import mpmath as mp
    mp.mp.dps = digits
    F = mp.mpf
    c0, dca = F(cfg["bg"]), F(cfg["dca"])
    nb = len(cfg["buffers"])
    n = nb + 1
    AA, Dinv = mp.zeros(n, n), mp.zeros(n, n)
    for i, (_, b) in enumerate(cfg["buffers"]):
        K = F(b["koff"]) / F(b["kon"])
        k = F(b["Total Concentration"]) * K / ((K + c0) ** 2)
        tau = 1 / (F(b["koff"]) + F(b["kon"]) * c0)
        AA[i, i] = -1 / tau
        AA[i, nb] = k / tau
        AA[nb, i] = 1 / tau
        AA[nb, nb] -= k / tau
        Dinv[i, i] = 1 / F(b["D"])
    Dinv[nb, nb] = 1 / dca
    ev, er = mp.eig(-Dinv * AA)
    mu = [mp.re(e) for e in ev]
    perm = list(range(n))
    mi = min(perm, key=lambda q: mu[q])
    perm[mi], perm[nb] = perm[nb], perm[mi]
    mu = [mu[q] for q in perm]
    V = mp.matrix(n, n)
    for i in range(n):
        for q in range(n):
            V[i, q] = mp.re(er[i, perm[q]])
    u = mp.zeros(n, 1)
    u[nb] = F(cfg["current"]) / (4 * mp.pi * F("96485.33e-6") * dca)
    a = mp.lu_solve(V, u)
    xy = cfg["xy"]
    nc = len(xy)
    out = np.zeros((nc, nc))
    for i in range(nc):
        for j in range(nc):
            r = mp.sqrt((F(xy[i, 0]) - F(xy[j, 0])) ** 2 + (F(xy[i, 1]) - F(xy[j, 1])) ** 2)
            if r > F("1e-6"):
                out[i, j] = float(sum(a[q] / r * mp.exp(-r * mp.sqrt(abs(mu[q])) * F("1e-8")) * V[nb, q] * F("1e-4")
                                      for q in range(n)))
            else:
                out[i, j] = cfg["ca_open"]
    return out

"""ctypes wrapper for oracle/_ref/libcasim_ref.so: the reference's OWN CPU classes
(CaSim/DyadRD2DCPU.cpp, DyadRDCPU.cpp, DyadChannels.cpp, SRPool.cpp, CytosolPool.cpp,
NSRConstPool.cpp, rngstream.cpp, ...) compiled in place by oracle/Makefile.

Test infrastructure only: imported by tests/, the golden-fixture generator and the
CPU-baseline leg of bench.py, never by the product package.
"""
import ctypes
import json
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libcasim_ref.so")
_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        vp, cp, i, l, d = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_long, ctypes.c_double
        L.casimref_create.restype = vp
        L.casimref_create.argtypes = [cp, i, i]
        L.casimref_destroy.argtypes = [vp]
        L.casimref_last_error.restype = cp
        L.casimref_num_channels.argtypes = [vp]
        L.casimref_element_volume.argtypes = [vp]
        L.casimref_element_volume.restype = d
        L.casimref_dims.argtypes = [vp, ctypes.POINTER(l), i]
        L.casimref_reset.argtypes = [vp]
        L.casimref_init_opening.argtypes = [vp, i, i]
        L.casimref_update.argtypes = [vp]
        L.casimref_start.argtypes = [vp, ctypes.POINTER(i)]
        L.casimref_step.argtypes = [vp, l]
        L.casimref_get.argtypes = [vp, cp, ctypes.POINTER(d), l]
        L.casimref_get.restype = l
        L.casimref_get_states.argtypes = [vp, ctypes.POINTER(i), l]
        L.casimref_get_states.restype = l
        _lib = L
    return _lib


class RefSim:
    """One reference run of `n_batch` sites (NumBatch) driven like
    ParallelHybridSolver::RunSimulationsCPU (CaSim/ParallelHybridSolver.cpp:408-437)."""

    def __init__(self, params: dict, n_batch: int = 1, n_cores: int = 1):
        L = lib()
        self.params = params
        self.n_batch = n_batch
        self.h = L.casimref_create(json.dumps(params).encode(), n_batch, n_cores)
        if not self.h:
            raise RuntimeError("reference create failed: " + L.casimref_last_error().decode())
        self.n_channels = L.casimref_num_channels(self.h)
        dims = (ctypes.c_long * 8)()
        nd = L.casimref_dims(self.h, dims, 8)
        self.dims = [int(dims[k]) for k in range(nd)]

    def close(self):
        if self.h:
            lib().casimref_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def start(self, first_channel):
        arr = (ctypes.c_int * self.n_batch)(*[int(c) for c in first_channel])
        lib().casimref_start(self.h, arr)

    def step(self, n):
        lib().casimref_step(self.h, int(n))

    def get(self, what, n=None):
        L = lib()
        total = L.casimref_get(self.h, what.encode(), None, 0) if n is None else n
        if total < 0:
            raise KeyError(what)
        out = np.zeros(total, dtype=np.float64)
        L.casimref_get(self.h, what.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), total)
        return out

    def states(self):
        L = lib()
        n = L.casimref_get_states(self.h, None, 0)
        out = np.zeros(n, dtype=np.int32)
        L.casimref_get_states(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n)
        return out


def cre_analysis(times, states, max_time, nadir):
    """The reference's own IndChannelCREAnalyzer::RunAnalysis
    (CaSim/IndChannelCREAnalyzer.cpp:53-138) on traces given as events: times[i] (n_i,)
    and states[i] (n_i, n_channels) of 0/1. Returns what it writes: the per-scenario
    table and the four time histograms (first column of the files, the bin time, dropped)."""
    import tempfile
    L = lib()
    n_ch = int(np.asarray(states[0]).shape[1])
    n_ev = np.array([len(t) for t in times], dtype=np.int32)
    tt = np.ascontiguousarray(np.concatenate([np.asarray(t, dtype=np.float64) for t in times]))
    ss = np.ascontiguousarray(np.concatenate([np.asarray(s, dtype=np.int32).reshape(-1, n_ch) for s in states]))
    with tempfile.TemporaryDirectory() as d:
        os.makedirs(os.path.join(d, "analysis"))
        f = L.casimref_cre_analysis
        f.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                      ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_double, ctypes.c_int]
        rc = f(d.encode(), len(times), n_ev.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
               tt.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ss.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
               n_ch, float(max_time), int(nadir))
        if rc:
            raise RuntimeError("reference analysis failed: " + L.casimref_last_error().decode())

        def table(name):
            rows = [ln.split() for ln in open(os.path.join(d, "analysis", name)) if ln.strip()]
            return np.array([[float(v) for v in r] for r in rows])
        out = {"per_trace": table("scenarios.txt")}
        for key, name in (("hist", "time_hist.txt"), ("hist_quark", "time_hist_quarks.txt"),
                          ("hist_blip", "time_hist_blips.txt"), ("hist_spark", "time_hist_sparks.txt")):
            out[key] = table(name)[:, 1:].astype(np.int64)
    return out

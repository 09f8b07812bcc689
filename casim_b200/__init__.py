"""casim_b200: B200-native release-site hot path of CaSim.

The compute runs in libcasim_b200.so (CUDA, sm_100a) behind the C ABI declared
in include/casim_b200.h; this module is a thin ctypes mirror of it. There is no
CPU fallback: if the library cannot be loaded every call raises.

    from casim_b200 import ReleaseSiteBatch, configs
    params, sites = configs.config1(n_sites=100)
    sim = ReleaseSiteBatch(params, sites, precision="fp32")
    sim.start(sites["first_channel"])
    sim.step(20000)               # 1 ms at dt = 50 ns
    ca = sim.field(0, 0)          # Ca of site 0, reference node order
"""
import ctypes
import json
import os

import numpy as np

from . import configs  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcasim_b200.so")

OK, EINVAL, ECUDA, ENOMEM, EUNSTABLE, ETIMEOUT, ENONFINITE, EUNSUPPORTED = range(8)
FP64, FP32 = 0, 1
PATH_AUTO, PATH_PLAIN, PATH_RESIDENT = 0, 1, 2
_STATUS = {OK: "OK", EINVAL: "EINVAL", ECUDA: "ECUDA", ENOMEM: "ENOMEM", EUNSTABLE: "EUNSTABLE",
           ETIMEOUT: "ETIMEOUT", ENONFINITE: "ENONFINITE", EUNSUPPORTED: "EUNSUPPORTED"}

# every extern "C" symbol of include/casim_b200.h
EXPORTS = (
    "casim_b200_create", "casim_b200_destroy", "casim_b200_info", "casim_b200_species_name", "casim_b200_cyto_species_name",
    "casim_b200_qs_create", "casim_b200_qs_destroy", "casim_b200_qs_last_error", "casim_b200_qs_info", "casim_b200_qs_increments",
    "casim_b200_qs_run", "casim_b200_qs_last_run_ms", "casim_b200_qs_event_count", "casim_b200_qs_events", "casim_b200_qs_draws",
    "casim_b200_qs_analysis",
    "casim_b200_last_error", "casim_b200_set_stream", "casim_b200_reset", "casim_b200_init_opening",
    "casim_b200_update", "casim_b200_start", "casim_b200_step", "casim_b200_synchronize",
    "casim_b200_get_field", "casim_b200_set_field", "casim_b200_get_mouth", "casim_b200_get_states",
    "casim_b200_get_jsr", "casim_b200_get_total_current", "casim_b200_get_efflux", "casim_b200_get_cyto",
    "casim_b200_get_cyto_field", "casim_b200_set_cyto_field", "casim_b200_get_draws", "casim_b200_get_release", "casim_b200_check_finite",
    "casim_b200_get_all_mouth", "casim_b200_get_all_states", "casim_b200_last_step_ms",
    "casim_b200_last_step_launches", "casim_b200_profile_step", "casim_b200_set_site_gating", "casim_b200_debug_rng", "casim_b200_set_site_jsr",
    "casim_b200_rng_draws_static", "casim_b200_path_note",
    "casim_b200_set_all_states", "casim_b200_sg_features", "casim_b200_sg_set_mouth",
    "casim_b200_sg_gate_steps", "casim_b200_sg_run", "casim_b200_sg_create", "casim_b200_sg_destroy", "casim_b200_sg_set_stream", "casim_b200_sg_num_params",
    "casim_b200_sg_get_params", "casim_b200_sg_set_params", "casim_b200_sg_forward", "casim_b200_sg_gradients",
    "casim_b200_sg_train_step", "casim_b200_sg_check", "casim_b200_sg_launches", "casim_b200_sg_last_error",
    "casim_b200_sg_gemm", "casim_b200_trace_enable", "casim_b200_trace_count", "casim_b200_get_open_traces",
    "casim_b200_release_analysis", "casim_b200_get_micro_states", "casim_b200_sg_hybrid_run", "casim_b200_autotune",
)


class HybridStats(ctypes.Structure):
    """casim_sg_hybrid_stats"""
    _fields_ = [("surrogate_steps", ctypes.c_int64), ("rd_steps", ctypes.c_int64), ("checks", ctypes.c_int64),
                ("fallbacks", ctypes.c_int64), ("last_residual", ctypes.c_double), ("last_fail_fraction", ctypes.c_double)]


class CasimError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s: %s" % (_STATUS.get(status, str(status)), message))
        self.status = status


class SiteTable(ctypes.Structure):
    _fields_ = [
        ("n_sites", ctypes.c_int32),
        ("nx", ctypes.POINTER(ctypes.c_int32)), ("ny", ctypes.POINTER(ctypes.c_int32)),
        ("nz", ctypes.POINTER(ctypes.c_int32)), ("n_channels", ctypes.POINTER(ctypes.c_int32)),
        ("ch_x", ctypes.POINTER(ctypes.c_double)), ("ch_y", ctypes.POINTER(ctypes.c_double)),
        ("seeds", ctypes.POINTER(ctypes.c_uint32)), ("jsr_init", ctypes.POINTER(ctypes.c_double)),
    ]


class Info(ctypes.Structure):
    _fields_ = [
        ("n_sites", ctypes.c_int32), ("dim", ctypes.c_int32), ("n_ions", ctypes.c_int32),
        ("n_pairs", ctypes.c_int32), ("n_buffers", ctypes.c_int32), ("n_cyto_species", ctypes.c_int32),
        ("cyto_nodes", ctypes.c_int32), ("precision", ctypes.c_int32), ("path", ctypes.c_int32),
        ("max_channels", ctypes.c_int32), ("total_nodes", ctypes.c_int64), ("dt_ms", ctypes.c_double),
        ("element_volume", ctypes.c_double),
    ]


_lib = None


def lib():
    """Load libcasim_b200.so; raise if it is missing (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libcasim_b200.so is not built; run `python -m casim_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
        dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32)
        for name in EXPORTS:
            getattr(L, name).restype = ctypes.c_int
        L.casim_b200_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(SiteTable), ctypes.POINTER(vp)]
        L.casim_b200_destroy.argtypes = [vp]
        L.casim_b200_info.argtypes = [vp, ctypes.POINTER(Info)]
        L.casim_b200_species_name.argtypes = [vp, i32, ctypes.c_char_p, ctypes.c_size_t]
        L.casim_b200_cyto_species_name.argtypes = [vp, i32, ctypes.c_char_p, ctypes.c_size_t]
        u32p = ctypes.POINTER(ctypes.c_uint32)
        L.casim_b200_qs_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, i32, u32p, i64, ctypes.POINTER(vp)]
        L.casim_b200_qs_destroy.argtypes = [vp]
        L.casim_b200_qs_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
        L.casim_b200_qs_info.argtypes = [vp, ip, ip, dp]
        L.casim_b200_qs_increments.argtypes = [vp, dp]
        L.casim_b200_qs_run.argtypes = [vp, ip]
        L.casim_b200_qs_last_run_ms.argtypes = [vp, dp]
        L.casim_b200_qs_event_count.argtypes = [vp, i32, ctypes.POINTER(i64)]
        L.casim_b200_qs_events.argtypes = [vp, i32, dp, ip, ip]
        L.casim_b200_qs_draws.argtypes = [vp, i32, ctypes.POINTER(ctypes.c_uint64)]
        L.casim_b200_qs_analysis.argtypes = [vp, i32, dp, ip]
        L.casim_b200_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
        L.casim_b200_set_stream.argtypes = [vp, vp]
        L.casim_b200_reset.argtypes = [vp]
        L.casim_b200_init_opening.argtypes = [vp, i32, i32]
        L.casim_b200_update.argtypes = [vp]
        L.casim_b200_start.argtypes = [vp, ip]
        L.casim_b200_step.argtypes = [vp, i64]
        L.casim_b200_synchronize.argtypes = [vp]
        for f in ("get_field", "get_mouth", "get_cyto_field"):
            getattr(L, "casim_b200_" + f).argtypes = [vp, i32, i32, dp]
        L.casim_b200_set_field.argtypes = [vp, i32, i32, dp]
        L.casim_b200_set_cyto_field.argtypes = [vp, i32, i32, dp]
        L.casim_b200_get_states.argtypes = [vp, i32, ip]
        L.casim_b200_get_micro_states.argtypes = [vp, i32, ip]
        L.casim_b200_autotune.argtypes = [vp, i64, ctypes.c_char_p, ctypes.c_size_t]
        for f in ("get_jsr", "get_total_current", "get_efflux", "get_cyto", "get_release"):
            getattr(L, "casim_b200_" + f).argtypes = [vp, i32, dp]
        L.casim_b200_get_draws.argtypes = [vp, i32, ctypes.POINTER(ctypes.c_uint64)]
        L.casim_b200_check_finite.argtypes = [vp, ip]
        L.casim_b200_get_all_mouth.argtypes = [vp, i32, dp]
        L.casim_b200_get_all_states.argtypes = [vp, ip]
        L.casim_b200_set_all_states.argtypes = [vp, ip]
        L.casim_b200_sg_features.argtypes = [vp, i32, i32, vp]
        L.casim_b200_sg_set_mouth.argtypes = [vp, vp, i32, ctypes.c_double]
        L.casim_b200_sg_gate_steps.argtypes = [vp, i64]
        L.casim_b200_sg_run.argtypes = [vp, vp, i32, i64, i32, ctypes.c_double]
        L.casim_b200_sg_hybrid_run.argtypes = [vp, vp, i32, i64, i32, i32, i32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                               ctypes.POINTER(HybridStats)]
        L.casim_b200_last_step_ms.argtypes = [vp, dp]
        L.casim_b200_last_step_launches.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.casim_b200_profile_step.argtypes = [vp, dp, i32, ip]
        L.casim_b200_set_site_gating.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p, ip, i32]
        L.casim_b200_debug_rng.argtypes = [ctypes.POINTER(ctypes.c_uint32), i64, dp]
        L.casim_b200_set_site_jsr.argtypes = [vp, dp]
        L.casim_b200_path_note.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
        L.casim_b200_rng_draws_static.argtypes = [ctypes.POINTER(ctypes.c_uint32), i64, dp]
        L.casim_b200_trace_enable.argtypes = [vp, i64, i64]
        L.casim_b200_trace_count.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.casim_b200_get_open_traces.argtypes = [vp, ctypes.POINTER(ctypes.c_uint16)]
        L.casim_b200_release_analysis.argtypes = [vp, ctypes.c_double, ctypes.c_double, i32, dp, ip, ip, ip, ip, ip]
        fp = ctypes.POINTER(ctypes.c_float)
        L.casim_b200_sg_create.argtypes = [i32, i32, i32, i32, ctypes.c_uint64, ctypes.POINTER(vp)]
        L.casim_b200_sg_destroy.argtypes = [vp]
        L.casim_b200_sg_set_stream.argtypes = [vp, vp]
        L.casim_b200_sg_num_params.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.casim_b200_sg_get_params.argtypes = [vp, fp]
        L.casim_b200_sg_set_params.argtypes = [vp, fp]
        L.casim_b200_sg_forward.argtypes = [vp, vp, i32, vp]
        L.casim_b200_sg_gradients.argtypes = [vp, vp, vp, i32, fp, fp]
        L.casim_b200_sg_train_step.argtypes = [vp, vp, vp, i32, ctypes.c_float, fp]
        L.casim_b200_sg_check.argtypes = [vp]
        L.casim_b200_sg_launches.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.casim_b200_sg_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
        L.casim_b200_sg_gemm.argtypes = [vp, vp, i32, i32, i32, vp]
        _lib = L
    return _lib


def last_error(h=None):
    buf = ctypes.create_string_buffer(4096)
    lib().casim_b200_last_error(h, buf, 4096)
    return buf.value.decode()


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def debug_rng(seed, n):
    """n runif() draws of an MRG32k3a stream, generated on the device."""
    s = np.ascontiguousarray(seed, dtype=np.uint32)
    out = np.zeros(n, dtype=np.float64)
    st = lib().casim_b200_debug_rng(_p(s, ctypes.c_uint32), n, _p(out, ctypes.c_double))
    if st:
        raise CasimError(st, last_error())
    return out


class ReleaseSiteBatch:
    """A batch of independent release sites on the current CUDA device.

    Mirrors the reference's compartment interfaces for the RD path:
    DyadSeries (CaSim/DyadSeries.h:9-44), SRSeries (CaSim/SRSeries.h:7-16),
    CytosolSeries (CaSim/CytosolSeries.h:10-21), NSRSeries (CaSim/NSRSeries.h:5-12),
    stepped together as ParallelHybridSolver does (CaSim/ParallelHybridSolver.cpp:408-437).
    """

    def __init__(self, params=None, sites=None, precision="fp64", path="auto", base_dir=None, json_text=None):
        """params: a Parameters.json dict, or json_text: its text, passed to the library
        unchanged (relative file names in it resolve from base_dir)."""
        L = lib()
        if json_text is not None:
            params = json.loads(json_text)
            raw = json_text.encode() if isinstance(json_text, str) else bytes(json_text)
        else:
            raw = json.dumps(params).encode()
        self.params = params
        prec = {"fp64": FP64, "fp32": FP32}[precision]
        pth = {"auto": PATH_AUTO, "plain": PATH_PLAIN, "resident": PATH_RESIDENT}[path]
        self._keep = []
        tab = None
        if sites is not None:
            tab = SiteTable()
            S = len(sites["nx"])
            tab.n_sites = S

            def arr(key, dt, ct):
                v = sites.get(key)
                if v is None:
                    return None
                a = np.ascontiguousarray(v, dtype=dt).reshape(-1)
                self._keep.append(a)
                return _p(a, ct)
            tab.nx = arr("nx", np.int32, ctypes.c_int32)
            tab.ny = arr("ny", np.int32, ctypes.c_int32)
            tab.nz = arr("nz", np.int32, ctypes.c_int32)
            tab.n_channels = arr("n_ch", np.int32, ctypes.c_int32)
            tab.ch_x = arr("ch_x", np.float64, ctypes.c_double)
            tab.ch_y = arr("ch_y", np.float64, ctypes.c_double)
            tab.seeds = arr("seeds", np.uint32, ctypes.c_uint32)
            tab.jsr_init = arr("jsr_init", np.float64, ctypes.c_double)
        h = ctypes.c_void_p()
        st = L.casim_b200_create(raw, (base_dir or "").encode(), prec, pth,
                                 ctypes.byref(tab) if tab is not None else None, ctypes.byref(h))
        if st:
            raise CasimError(st, last_error())
        self.h = h
        self.info = Info()
        L.casim_b200_info(self.h, ctypes.byref(self.info))
        self.S = self.info.n_sites
        nch = np.zeros(self.S, dtype=np.int64)
        if sites is not None and sites.get("n_ch") is not None:
            nch[:] = np.asarray(sites["n_ch"])
        else:
            nch[:] = self.info.max_channels
        self.n_ch = nch
        d = params["Dyad"]
        if sites is not None:
            nz = sites.get("nz")
            self._site_dims = [(int(sites["nx"][k]), int(sites["ny"][k]),
                                int(nz[k]) if (self.info.dim == 3 and nz is not None) else 1) for k in range(self.S)]
        else:
            nx = int(d["x"] / d["dx"] + 1)
            ny = int(d["y"] / d["dy"] + 1)
            nz = int(d["z"] / d["dz"] + 1) if self.info.dim == 3 else 1
            self._site_dims = [(nx, ny, nz)] * self.S

    # -- lifecycle --------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            lib().casim_b200_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, st):
        if st:
            raise CasimError(st, last_error(self.h))

    @property
    def path(self):
        return {PATH_PLAIN: "plain", PATH_RESIDENT: "resident"}.get(self.info.path, "?")

    def path_note(self):
        """How the resident path splits the batch into cluster classes, or why it runs plain."""
        buf = ctypes.create_string_buffer(1024)
        self._ck(lib().casim_b200_path_note(self.h, buf, 1024))
        return buf.value.decode()

    def species_name(self, k):
        buf = ctypes.create_string_buffer(256)
        self._ck(lib().casim_b200_species_name(self.h, k, buf, 256))
        return buf.value.decode()

    def cyto_species_name(self, k):
        buf = ctypes.create_string_buffer(256)
        self._ck(lib().casim_b200_cyto_species_name(self.h, k, buf, 256))
        return buf.value.decode()

    @property
    def n_species(self):
        return self.info.n_ions + self.info.n_pairs + self.info.n_buffers

    def set_stream(self, cuda_stream):
        """Run all work of this batch on the given cudaStream_t (an integer handle)."""
        self._ck(lib().casim_b200_set_stream(self.h, ctypes.c_void_p(cuda_stream)))

    def set_site_jsr(self, jsr_init):
        """Initial jSR concentrations (sites x ions) for the next reset/start."""
        v = np.ascontiguousarray(jsr_init, dtype=np.float64).reshape(self.S, self.info.n_ions)
        self._ck(lib().casim_b200_set_site_jsr(self.h, _p(v, ctypes.c_double)))

    def reset(self):
        self._ck(lib().casim_b200_reset(self.h))

    def init_opening(self, site, channel):
        self._ck(lib().casim_b200_init_opening(self.h, site, channel))

    def update(self):
        self._ck(lib().casim_b200_update(self.h))

    def start(self, first_channel=None):
        fc = np.zeros(self.S, dtype=np.int32) if first_channel is None else np.ascontiguousarray(first_channel, dtype=np.int32)
        self._ck(lib().casim_b200_start(self.h, _p(fc, ctypes.c_int32)))

    def step(self, n):
        self._ck(lib().casim_b200_step(self.h, int(n)))

    def synchronize(self):
        self._ck(lib().casim_b200_synchronize(self.h))

    def last_step_ms(self):
        v = ctypes.c_double()
        self._ck(lib().casim_b200_last_step_ms(self.h, ctypes.byref(v)))
        return v.value

    def last_step_launches(self):
        v = ctypes.c_int64()
        self._ck(lib().casim_b200_last_step_launches(self.h, ctypes.byref(v)))
        return v.value

    def set_site_gating(self, params, sites, base_dir=None, json_text=None):
        """Gate the listed sites by the two-state RyR model of `params` (a Parameters
        dict of the same ions); the other sites keep theirs. Plain path only."""
        raw = json_text.encode() if json_text is not None else json.dumps(params).encode()
        idx = np.ascontiguousarray(sites, dtype=np.int32)
        self._ck(lib().casim_b200_set_site_gating(self.h, raw, (base_dir or "").encode(), _p(idx, ctypes.c_int32), int(idx.size)))

    def profile_step(self):
        """One time step with each kernel timed: {kernel: ms} (plain path: gating, cytosol,
        cleft, update; resident path: the one launch)."""
        ms = np.zeros(4)
        n = ctypes.c_int32()
        self._ck(lib().casim_b200_profile_step(self.h, _p(ms, ctypes.c_double), 4, ctypes.byref(n)))
        names = ("k_resident",) if self.path == "resident" else ("gating", "cytosol", "cleft", "update")
        return {k: float(ms[i]) for i, k in enumerate(names[:n.value])}

    # -- getters ---------------------------------------------------------
    def field(self, site, species):
        nx, ny, nz = self._dims(site)
        out = np.zeros(nx * ny * nz, dtype=np.float64)
        self._ck(lib().casim_b200_get_field(self.h, site, species, _p(out, ctypes.c_double)))
        return out

    def set_field(self, site, species, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        self._ck(lib().casim_b200_set_field(self.h, site, species, _p(v, ctypes.c_double)))

    def _dims(self, site):
        return self._site_dims[site]

    def mouth(self, site, species):
        out = np.zeros(int(self.n_ch[site]), dtype=np.float64)
        self._ck(lib().casim_b200_get_mouth(self.h, site, species, _p(out, ctypes.c_double)))
        return out

    def states(self, site):
        out = np.zeros(int(self.n_ch[site]), dtype=np.int32)
        self._ck(lib().casim_b200_get_states(self.h, site, _p(out, ctypes.c_int32)))
        return out

    def trace_enable(self, every_steps, max_samples):
        """Record the open-RyR count of every site now and every `every_steps` time
        steps of step() from here on (at most `max_samples` samples)."""
        self._ck(lib().casim_b200_trace_enable(self.h, int(every_steps), int(max_samples)))
        self._trace_every = int(every_steps)

    def open_traces(self):
        """[sites, samples] uint16 open-RyR counts recorded since trace_enable."""
        n = ctypes.c_int64(0)
        self._ck(lib().casim_b200_trace_count(self.h, ctypes.byref(n)))
        out = np.zeros((self.S, n.value), dtype=np.uint16)
        self._ck(lib().casim_b200_get_open_traces(self.h, _p(out, ctypes.c_uint16)))
        return out

    def release_analysis(self, max_time_ms, nadir, hist_dt_ms=0.01):
        """Release-event analysis of the recorded traces on the device (the
        arithmetic of CaSim/IndChannelCREAnalyzer.cpp:53-138): per site amplitude,
        time to peak, time to end, integral and mean of the open count, and the
        time histograms of the open count over all sites, quarks, blips, sparks."""
        nh = int(max_time_ms / hist_dt_ms)
        mch = int(self.info.max_channels)
        per_site = np.zeros((self.S, 5))
        h_all = np.zeros((nh + 1, mch + 1), dtype=np.int32)
        h_q = np.zeros((nh + 1, 2), dtype=np.int32)
        h_b = np.zeros((nh + 1, int(nadir) + 1), dtype=np.int32)
        h_s = np.zeros((nh + 1, mch + 1), dtype=np.int32)
        counts = np.zeros(3, dtype=np.int32)
        i32p = ctypes.c_int32
        self._ck(lib().casim_b200_release_analysis(self.h, float(hist_dt_ms), float(max_time_ms), int(nadir), _p(per_site, ctypes.c_double),
                                                   _p(h_all, i32p), _p(h_q, i32p), _p(h_b, i32p), _p(h_s, i32p), _p(counts, i32p)))
        return {"amp": per_site[:, 0], "ttp": per_site[:, 1], "tte": per_site[:, 2], "integral": per_site[:, 3],
                "mean": per_site[:, 4], "hist": h_all, "hist_quark": h_q, "hist_blip": h_b, "hist_spark": h_s,
                "quarks": int(counts[0]), "blips": int(counts[1]), "sparks": int(counts[2])}

    def autotune(self, steps_per_trial=20):
        """Choose block and cluster sizes by measurement (resident path); returns the choices."""
        buf = ctypes.create_string_buffer(4096)
        self._ck(lib().casim_b200_autotune(self.h, int(steps_per_trial), buf, 4096))
        return buf.value.decode()

    def micro_states(self, site):
        """60-state RyR models: the micro-state 0..59 of each RyR (45-59 open)."""
        out = np.zeros(int(self.n_ch[site]), dtype=np.int32)
        self._ck(lib().casim_b200_get_micro_states(self.h, site, _p(out, ctypes.c_int32)))
        return out

    def all_states(self):
        out = np.zeros(int(self.n_ch.sum()), dtype=np.int32)
        self._ck(lib().casim_b200_get_all_states(self.h, _p(out, ctypes.c_int32)))
        return out

    def set_all_states(self, states):
        st = np.ascontiguousarray(states, dtype=np.int32).reshape(-1)
        assert st.size == int(self.n_ch.sum())
        self._ck(lib().casim_b200_set_all_states(self.h, _p(st, ctypes.c_int32)))

    def all_mouth(self, species):
        out = np.zeros(int(self.n_ch.sum()), dtype=np.float64)
        self._ck(lib().casim_b200_get_all_mouth(self.h, species, _p(out, ctypes.c_double)))
        return out

    def _vec(self, fn, site, n):
        out = np.zeros(n, dtype=np.float64)
        self._ck(getattr(lib(), "casim_b200_" + fn)(self.h, site, _p(out, ctypes.c_double)))
        return out

    def jsr(self, site):
        return self._vec("get_jsr", site, self.info.n_ions)

    def total_current(self, site):
        return self._vec("get_total_current", site, self.info.n_ions)

    def efflux(self, site):
        return self._vec("get_efflux", site, self.info.n_ions + self.info.n_pairs)

    def cyto(self, site):
        return self._vec("get_cyto", site, self.info.n_cyto_species)

    def cyto_field(self, site, species):
        out = np.zeros(self.info.cyto_nodes, dtype=np.float64)
        self._ck(lib().casim_b200_get_cyto_field(self.h, site, species, _p(out, ctypes.c_double)))
        return out

    def set_cyto_field(self, site, species, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        assert v.size == self.info.cyto_nodes
        self._ck(lib().casim_b200_set_cyto_field(self.h, site, species, _p(v, ctypes.c_double)))

    def release(self, site):
        return float(self._vec("get_release", site, 1)[0])

    def draws(self, site):
        v = ctypes.c_uint64()
        self._ck(lib().casim_b200_get_draws(self.h, site, ctypes.byref(v)))
        return int(v.value)

    def check_finite(self):
        bad = ctypes.c_int32(-1)
        st = lib().casim_b200_check_finite(self.h, ctypes.byref(bad))
        return st == OK, bad.value


class QuasiStationarySites:
    """Quasi-stationary release sites simulated with Gillespie's method on the device:
    the reference's ParallelSolver path (CaSim/ParallelSolver.cpp:51-143,
    CaSim/QuasyStationaryReleaseSite.cpp:89-133) with the mouth Ca of the linearised
    Naraghi-Neher model (CaSim/LinearNaraghiNeher.cpp:9-75), one scenario per warp."""

    def __init__(self, params, n_scenarios, base_dir=None, seeds=None, max_events=4096, json_text=None):
        L = lib()
        raw = json_text.encode() if json_text is not None else json.dumps(params).encode()
        sd = None
        if seeds is not None:
            self._seeds = np.ascontiguousarray(seeds, dtype=np.uint32).reshape(n_scenarios, 6)
            sd = _p(self._seeds, ctypes.c_uint32)
        h = ctypes.c_void_p()
        st = L.casim_b200_qs_create(raw, (base_dir or "").encode(), int(n_scenarios), sd, int(max_events), ctypes.byref(h))
        if st:
            raise CasimError(st, self._err(None))
        self.h = h
        self.S = int(n_scenarios)
        nc, ns, mt = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_double()
        L.casim_b200_qs_info(self.h, ctypes.byref(nc), ctypes.byref(ns), ctypes.byref(mt))
        self.n_ch, self.max_time = nc.value, mt.value
        self.max_events = int(max_events)

    @staticmethod
    def _err(h):
        buf = ctypes.create_string_buffer(1024)
        lib().casim_b200_qs_last_error(h, buf, 1024)
        return buf.value.decode()

    def _ck(self, st):
        if st:
            raise CasimError(st, self._err(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib().casim_b200_qs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def increments(self):
        out = np.zeros((self.n_ch, self.n_ch))
        self._ck(lib().casim_b200_qs_increments(self.h, _p(out, ctypes.c_double)))
        return out

    def run(self, first_channel):
        fc = np.ascontiguousarray(first_channel, dtype=np.int32).reshape(self.S)
        self._ck(lib().casim_b200_qs_run(self.h, _p(fc, ctypes.c_int32)))

    def last_run_ms(self):
        v = ctypes.c_double()
        self._ck(lib().casim_b200_qs_last_run_ms(self.h, ctypes.byref(v)))
        return v.value

    def events(self, scenario):
        """(times, channels, new states) of the scenario's stored events, in order
        (the first max_events of them)."""
        k = min(self.event_count(scenario), self.max_events)
        t = np.zeros(k)
        c = np.zeros(k, dtype=np.int32)
        s = np.zeros(k, dtype=np.int32)
        self._ck(lib().casim_b200_qs_events(self.h, scenario, _p(t, ctypes.c_double), _p(c, ctypes.c_int32), _p(s, ctypes.c_int32)))
        return t, c, s

    def event_count(self, scenario):
        """Events of the scenario's last run, stored or not."""
        n = ctypes.c_int64()
        self._ck(lib().casim_b200_qs_event_count(self.h, scenario, ctypes.byref(n)))
        return n.value

    def draws(self, scenario):
        v = ctypes.c_uint64()
        self._ck(lib().casim_b200_qs_draws(self.h, scenario, ctypes.byref(v)))
        return int(v.value)

    def analysis(self, nadir):
        """per scenario [amplitude, time to peak, time to end, integral, mean] and the
        class counts (quarks, blips, sparks)."""
        out = np.zeros((self.S, 5))
        cls = np.zeros(3, dtype=np.int32)
        self._ck(lib().casim_b200_qs_analysis(self.h, int(nadir), _p(out, ctypes.c_double), _p(cls, ctypes.c_int32)))
        return out, cls

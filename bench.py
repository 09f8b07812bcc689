#!/usr/bin/env python
"""Benchmark of the release-site hot path: simulated site-milliseconds per second.

Workload (default): 4096 3D dyads of uneven size (cleft side ~U{40..120}
nodes at 10 nm x 3 z-layers, 10..100 RyRs on a jittered 31 nm lattice),
each coupled to a 25^3 cytosol at 40 nm with Ca, ATP and calmodulin,
two-state power-law RyR gating, dt = 50 ns, FP32 fields with FP64 pools.
Inputs are seeded synthetic sites (the reference ships no dataset).

One bench step advances every site by --chunk time steps. `value` is timed on
the device (CUDA events on the library's stream, max over ranks); `e2e` runs
one batch scenario per step through the public API the way the reference's
RunSimulations loop does (ResetSystem + InitOpening + Update, --chunk steps,
outputs read back): host->device the per-site initial jSR Ca and opened RyR,
device->host every RyR's mouth Ca and state.

    python bench.py                      # 1 GPU
    python bench.py --impl reference     # reference CPU classes on the host cores
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=["c1", "c2", "c3"])
    ap.add_argument("--sites", type=int, default=0, help="override the number of sites")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--path", default="auto", choices=["auto", "plain", "resident"])
    ap.add_argument("--chunk", type=int, default=200, help="time steps per bench step")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the surrogate-versus-RD report")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the mouth-Ca error check against FP64")
    ap.add_argument("--no-qs", action="store_true", help="skip the quasi-stationary (Gillespie) report")
    ap.add_argument("--surrogate-frontier", action="store_true",
                    help="print only the surrogate report over the tolerance frontier (one GPU)")
    return ap.parse_args()


def workload(args, world=1):
    """The global site table of a run on `world` GPUs: `--sites` (default: the
    config's size) sites per GPU, drawn by one seeded generator, so every rank
    builds the same table and takes its cost-balanced share (weak scaling)."""
    from casim_b200 import configs
    per = args.sites
    if args.config == "c1":
        p, s = configs.config1(n_sites=(per or 100) * world, seed0=1)
        name = "2D 64x64 cleft, 20 RyR, pool cytosol (config 1 geometry)"
    elif args.config == "c3":
        p, s = configs.config3(n_sites=(per or 1024) * world, seed=3)
        name = "1024 2D 64x64 clefts, 50 RyR, jSR Ca ~U[0.5,1.5] mM"
    else:
        p, s = configs.config2(n_sites=(per or 4096) * world, seed=2024)
        name = "4096 3D dyads side~U{40..120}x3 layers, 10..100 RyR, 25^3 RD cytosol"
    return p, s, name


def cyto_nodes_of(params):
    c = params.get("Cytosol", {})
    return int(c.get("Nodes", 0)) ** 3 if c.get("Type") == "RD3D" else 0


def sharded_run(params, sites, world, rank, make_sim, run):
    """One rank of a multi-GPU run: this rank's share of the global site table
    (casim_b200.dist.partition by node-steps), a batch of it from make_sim, the
    work run(sim, shard) does on it, and the per-site outputs of every rank
    gathered on rank 0 (None elsewhere). There is no exchange inside the time
    loop: sites are independent. Returns (sim, shard, run's result, outputs)."""
    from casim_b200 import dist as cdist
    idx, mine = cdist.shard_of_rank(sites, cyto_nodes_of(params), world, rank)
    sim = make_sim(params, mine)
    res = run(sim, mine)
    full = cdist.gather_sites(cdist.site_outputs(sim, len(idx)), idx, len(sites["nx"]))
    return sim, mine, res, full


def outputs_summary(full):
    from casim_b200.dist import SITE_OUTPUT_COLUMNS
    return {"sites": int(full.shape[0]),
            **{"sum_" + c: float(full[:, k].sum()) for k, c in enumerate(SITE_OUTPUT_COLUMNS)}}


def launch_ranks(args):
    """`--gpus N` without a torchrun environment: start N ranks of this script
    under torch.distributed.run (one process per GPU, rendezvous on 127.0.0.1),
    bounded by a timeout, and return their exit status."""
    import socket
    so = socket.socket()
    so.bind(("127.0.0.1", 0))
    port = so.getsockname()[1]
    so.close()
    cmd = ["timeout", "-k", "60", "1800", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", str(args.gpus), "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(cmd).returncode


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu_index=0):
        self.samples = []
        self.proc = None
        self.idx = gpu_index

    def __enter__(self):
        q = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + q, "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if "Active" in s[3 + k] and "Not" not in s[3 + k]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ncu dram__bytes_read.sum + dram__bytes_write.sum of the k_resident launches of one
# bench step on 512 sites of the config-2 workload, per site (FP32): each launch loads
# and stores every site once, so the traffic scales with the sites, not with the steps
RESIDENT_DRAM_BYTES_PER_SITE = 319.7e6 / 512
# ncu DRAM bytes (read + write) of one k_rd_s launch per cleft node (fp32, config-2 sites):
# 129.3 MB + 78.5 MB on the 10 352 496 cleft nodes of 512 sites of this workload
STREAM_CLEFT_DRAM_BYTES_PER_NODE = (129.278464e6 + 78.518016e6) / 10352496


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def algorithmic_bytes_per_step(sim, sites, params):
    """Each stored field read once and written once per node-step: cleft
    (ions + ion-buffer pairs) plus the RD3D cytosol species."""
    w = 4 if sim.info.precision == 1 else 8
    F = sim.info.n_ions + sim.info.n_pairs
    cleft = int(sim.info.total_nodes)
    cyto = sim.S * sim.info.cyto_nodes
    CS = sim.info.n_cyto_species if sim.info.cyto_nodes else 0
    return 2 * w * (cleft * F + cyto * CS)


def dominant_kernel(args, sim, sites, bytes_step, peak):
    """Roofline of the kernel that takes the largest share of a time step, from CUDA
    events on the library's stream: achieved = its algorithmic bytes per launch / its
    launch time (plain path: the average of 5 profiled time steps, every kernel timed;
    resident path: one launch of --chunk time steps)."""
    w = 4 if sim.info.precision == 1 else 8
    F = sim.info.n_ions + sim.info.n_pairs
    cleft_nodes = int(np.sum(np.asarray(sites["nx"], np.int64) * np.asarray(sites["ny"]) * np.asarray(sites["nz"])))
    CS = sim.info.n_cyto_species if sim.info.cyto_nodes else 0
    if sim.path == "resident":
        sim.step(args.chunk)
        sim.synchronize()
        kms = sim.last_step_ms()
        achieved = bytes_step * args.chunk / (kms / 1e3) / 1e9
        traffic = (RESIDENT_DRAM_BYTES_PER_SITE * sim.S
                   if args.precision == "fp32" and args.config == "c2" else None)
        return {"bound": "hbm", "kernel": "k_resident", "achieved": achieved, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "launch_ms": kms,
                "note": "achieved = algorithmic bytes (2 x field bytes per node-step) of one launch (--chunk time steps) / "
                        "its device time; the resident path keeps fields on chip, so this is an effective bandwidth; "
                        "traffic = ncu DRAM bytes of one launch (0.63 MB per site, measured on 512 sites of this "
                        "workload and scaled by sites)"}
    prof = {}
    for _ in range(5):
        for k, v in sim.profile_step().items():
            prof[k] = prof.get(k, 0.0) + v / 5
    kbytes = {"cleft": 2 * w * F * cleft_nodes, "cytosol": 2 * w * CS * sim.S * sim.info.cyto_nodes}
    names = {"gating": "k_pre_r (RyR gating, pools)", "cytosol": "k_cyto_m (RD3D cytosol)", "cleft": "k_rd_s (cleft stencil)",
             "update": "k_update_s (Update)"}
    dom = max(prof, key=prof.get)
    step_ms = sum(prof.values())
    kernels = {names[k]: {"ms": v, "share": v / step_ms,
                          "achieved_gbs": (kbytes[k] / (v / 1e3) / 1e9 if k in kbytes and v > 0 else None)}
               for k, v in prof.items()}
    achieved = kbytes.get(dom, bytes_step) / (prof[dom] / 1e3) / 1e9
    traffic = (STREAM_CLEFT_DRAM_BYTES_PER_NODE * cleft_nodes
               if STREAM_CLEFT_DRAM_BYTES_PER_NODE and dom == "cleft" and args.precision == "fp32" and args.config == "c2"
               else None)
    return {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "launch_ms": prof[dom], "kernels": kernels,
            "step_achieved_gbs": bytes_step / (step_ms / 1e3) / 1e9,
            "note": "achieved = the kernel's algorithmic bytes per launch (each stored value of its field read and "
                    "written once per node-step) / its CUDA-event launch time; traffic = ncu DRAM bytes per launch "
                    "(measured on 512 sites of this workload, scaled by cleft nodes)"}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_baseline(args, params, sites, budget_s):
    """The CPU restatement (oracle/) on a bounded sample of the same sites,
    all host threads (one site per thread), timed by wall clock; then one site
    on one thread, the per-core figure."""
    from oracle import oracle
    n_threads = os.cpu_count() or 1
    S = len(sites["nx"])
    sample = min(S, max(n_threads, 8))
    from casim_b200.configs import subset_sites

    def timed(idx, threads, budget):
        sub = subset_sites(sites, idx)
        o = oracle.OracleSim(params, sub)
        o.start(sub["first_channel"])
        o.step(2, threads)
        steps, t0 = 0, time.time()
        n = 5
        while time.time() - t0 < budget:
            o.step(n, threads)
            steps += n
            n = min(n * 2, 200)
        dt = time.time() - t0
        o.close()
        return len(idx) * steps * params_dt_ms(params) / dt, steps

    v_all, steps = timed(np.arange(sample), n_threads, budget_s)
    v_one, steps1 = timed(np.arange(1), 1, max(budget_s / 3, 3.0))
    return {"value": v_all, "unit": "site-ms/s", "cores": n_threads, "kind": "port", "cpu_model": cpu_model(),
            "sample": "%d of the workload's sites x %d time steps (CPU restatement, OpenMP over sites, %d threads)"
                      % (sample, steps, n_threads),
            "one_thread": {"value": v_one, "unit": "site-ms/s",
                           "sample": "site 0 of the workload x %d time steps on 1 thread" % steps1}}


# hybrid arms of the surrogate report: name -> (windows per check, RD correction steps,
# residual tolerance, largest fraction of sites allowed above it)
HYBRID_ARMS = {"hybrid_tol_1pct": (10, 20, 0.01, 0.0), "hybrid_tol_20pct": (10, 20, 0.2, 0.2)}
# the tolerance frontier (--surrogate-frontier)
FRONTIER_ARMS = {"tol_%g_fail_%g" % (t, f): (10, 20, t, f) for t in (0.01, 0.03, 0.1, 0.3) for f in (0.0, 0.2)}


def surrogate_report(sites=2048, sim_steps=20000, batches=8, train_steps=4000, hybrid=None):
    """Surrogate-gated versus plain-RD release sites on config-1 geometry: the
    network is trained on the device from RD snapshots (frozen open sets), its
    held-out mouth-Ca error is measured, then the same sites (same seeds, one
    RyR opened) run 1 ms with RD gating, with surrogate gating (network
    every 1 us, no RD step) and with the hybrid run (a 1 us full-RD correction
    after every 10 us of surrogate gating, residual check at the open RyRs,
    fallback to RD) at a 1 % and a 20 % tolerance. All arms are timed by wall
    clock around synchronised device work."""
    import torch
    from scipy.stats import ks_2samp
    import casim_b200 as cb
    from casim_b200 import configs, surrogate as sg
    Xs, Ys = [], []
    for b in range(batches):
        X, Y, _ = sg.rd_snapshots(4096, seed=100 + b)
        Xs.append(X)
        Ys.append(Y)
    X, Y = np.concatenate(Xs), np.concatenate(Ys)
    Xv, Yv, _ = sg.rd_snapshots(2048, seed=999)
    net = sg.Surrogate(X.shape[1], Y.shape[1], seed=3)
    sg.train(net, X, Y, train_steps, batch=8192, lr=2e-3)
    rel = np.abs(10.0 ** sg.predict(net, Xv) - 10.0 ** Yv) / 10.0 ** Yv
    p, s = configs.config1(n_sites=sites)
    first = np.random.default_rng(5).integers(0, 20, size=sites).astype(np.int32)
    out, stats = {}, {}
    hybrid = HYBRID_ARMS if hybrid is None else hybrid
    for mode in ("rd", "surrogate") + tuple(hybrid):
        sim = cb.ReleaseSiteBatch(p, s, precision="fp32", path="auto")
        sim.start(first)
        gate = sg.SurrogateGating(net, sim, window=20)
        torch.cuda.synchronize()
        t0 = time.time()
        if mode == "rd":
            sim.step(sim_steps)
        elif mode == "surrogate":
            gate.step(sim_steps)
        else:
            stats[mode] = gate.hybrid_step(sim_steps, *hybrid[mode])
        sim.synchronize()
        el = time.time() - t0
        out[mode] = (sites * sim_steps * sim.info.dt_ms / el, sim.all_states().reshape(sites, -1).sum(1),
                     np.array([sim.release(k) for k in range(sites)]))
        sim.close()
    net.close()
    hyb = {}
    for mode, (wpc, rds, tol, frac) in hybrid.items():
        st = stats[mode]
        hyb[mode] = {"site_ms_per_s": out[mode][0], "speedup_vs_rd": out[mode][0] / out["rd"][0],
                     "windows_per_check": wpc, "rd_correction_steps": rds, "tol": tol, "max_fail_fraction": frac,
                     "surrogate_step_fraction": st["surrogate_steps"] / max(1, st["surrogate_steps"] + st["rd_steps"]),
                     "fallbacks": st["fallbacks"], "checks": st["checks"],
                     "open_count_ks_p": float(ks_2samp(out["rd"][1], out[mode][1]).pvalue),
                     "release_ks_p": float(ks_2samp(out["rd"][2], out[mode][2]).pvalue),
                     "release_mean_ratio": float(out[mode][2].mean() / out["rd"][2].mean())}
    return {"workload": "%d config-1 sites, 1 ms from one open RyR, fp32" % sites,
            "rd_site_ms_per_s": out["rd"][0], "surrogate_site_ms_per_s": out["surrogate"][0],
            "speedup": out["surrogate"][0] / out["rd"][0],
            "held_out_mouth_rel_err_median": float(np.median(rel)), "held_out_mouth_rel_err_p90": float(np.percentile(rel, 90)),
            "open_count_ks_p": float(ks_2samp(out["rd"][1], out["surrogate"][1]).pvalue),
            "release_ks_p": float(ks_2samp(out["rd"][2], out["surrogate"][2]).pvalue),
            "release_mean_ratio": float(out["surrogate"][2].mean() / out["rd"][2].mean()),
            "training": "%d RD snapshots (0.25 ms relaxation), %d Adam steps of 8192 on the device" % (X.shape[0], train_steps),
            "hybrid": hyb}


def accuracy_report(args, params, sites, n_sites=64, steps=2000):
    """Mouth-Ca error of the benchmarked precision on the bench's own workload:
    the first `n_sites` sites run `steps` time steps in the bench's precision
    and all in FP64 from the same seeds (the FP64 device path matches the C
    restatement of the reference to 1e-11); errors over the sites still in
    lockstep (identical RyR states and draw counts)."""
    import casim_b200 as cb
    from casim_b200 import configs
    from casim_b200.precision import compare, snapshot
    idx = np.arange(min(n_sites, len(sites["nx"])))
    sub = configs.subset_sites(sites, idx)
    snaps = []
    for prec in (args.precision, "fp64"):
        sim = cb.ReleaseSiteBatch(params, sub, precision=prec, path="auto")
        sim.start(sub["first_channel"])
        sim.step(steps)
        sim.synchronize()
        snaps.append(snapshot(sim))
        sim.close()
    if sub.get("jsr_init") is None:
        jsr0 = np.full(idx.size, float(params["jSR"]["Ions"]["Calcium"]["Concentration"]))
    else:
        jsr0 = np.asarray(sub["jsr_init"], dtype=np.float64)[:, 0]
    r = compare(snaps[0], snaps[1], np.asarray(sub["n_ch"]), jsr0)
    return {"against": "fp64 device path, same seeds", "sites": int(idx.size), "time_steps": steps,
            "lockstep_sites": r["lockstep_sites"], "mouth_ca_rel_err_max": r["mouth_ca_rel_err"]["max"],
            "mouth_ca_rel_err_median": r["mouth_ca_rel_err"]["median"], "release_rel_err_max": r["release_rel_err"]["max"]}


def qs_cpu_baseline(params, coords, added, budget_s):
    """Scenarios per second of one host thread: the reference's own quasi-stationary
    loop (oracle/_ref) where it was built, else the CPU restatement."""
    import tempfile
    td = tempfile.mkdtemp()
    np.savetxt(os.path.join(td, "coords.txt"), coords, fmt="%.17g")
    from oracle import ref
    p = json.loads(json.dumps(params))
    p["Calcium Release Site"]["Parameters"]["Channels"]["RyR"]["Coordinates"] = os.path.join(td, "coords.txt")
    L = ref.lib() if ref.available() else None
    s6 = (12345,) * 6  # every chunk replays the package seed's stream from its start
    if L is not None and hasattr(L, "qsref_run"):
        L.qsref_set_increments.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.qsref_run.restype = ctypes.c_long
        L.qsref_run.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_ulong), ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                ctypes.c_long]
        a = np.ascontiguousarray(added)
        L.qsref_set_increments(len(coords), a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        n, done, t0 = 64, 0, time.time()
        while time.time() - t0 < budget_s:
            mr = 400 * n
            rt, rs, rps = np.zeros(mr), np.zeros(mr * len(coords), np.int32), np.zeros(n, np.int32)
            fc = (np.arange(done, done + n) % len(coords)).astype(np.int32)
            seed = (ctypes.c_ulong * 6)(*s6)
            L.qsref_run(json.dumps(p).encode(), seed, n, fc.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                        rt.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), rs.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                        rps.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), mr)
            done += n
            n *= 2
        kind = "reference"
        what = "the reference's QuasyStationaryReleaseSite loop (oracle/_ref), trace rows recorded as its solver does"
    else:
        from oracle import qs_oracle
        cfg = qs_oracle.parse(p, td)
        g = np.asarray(s6, np.uint32)
        done, t0 = 0, time.time()
        while time.time() - t0 < budget_s:
            g = qs_oracle.run(cfg, added, g, done % len(coords), max_events=4096)[4]
            done += 1
        kind = "port"
        what = "the CPU restatement of the reference's loop"
    el = time.time() - t0
    cpu = done / el
    return {"value": cpu, "unit": "scenarios/s", "cores": 1, "kind": kind, "cpu_model": cpu_model(),
            "sample": "%d scenarios on one stream, one thread: %s" % (done, what)}


def qs_report(n_scen=1048576, runs=3, cpu_budget_s=8.0):
    """Quasi-stationary release sites (Gillespie gating, casim_b200.QuasiStationarySites)
    on the 20-RyR MWC site of configs.quasi_stationary: scenarios per second on the
    device (CUDA events around each run, inputs resident), against the reference's own
    QuasyStationaryReleaseSite loop (oracle/_ref, one thread, as one ParallelSolver
    thread runs it) or, where that was not built, the CPU restatement, on a bounded
    sample of scenarios."""
    import tempfile
    import casim_b200 as cb
    from casim_b200 import configs
    params, coords = configs.quasi_stationary(20, seed=1)
    td = tempfile.mkdtemp()
    np.savetxt(os.path.join(td, "coords.txt"), coords, fmt="%.17g")
    q = cb.QuasiStationarySites(params, n_scen, base_dir=td, max_events=512)
    first = (np.arange(n_scen) % q.n_ch).astype(np.int32)
    for _ in range(2):
        q.run(first)
    ms = []
    for _ in range(runs):
        q.run(first)
        ms.append(q.last_run_ms())
    events = sum(q.event_count(s) for s in range(0, n_scen, 64)) * 64
    per, cls = q.analysis(nadir=3)
    added = q.increments()
    q.close()
    dev = n_scen / (np.median(ms) * 1e-3)
    out = {"workload": "%d scenarios of a 20-RyR TwoStateMWC site, 50 ms limit, 1 mM Mg, ATP + calmodulin, "
                       "first RyR s %% 20" % n_scen,
           "scenarios_per_s": dev, "events_per_s": events / (np.median(ms) * 1e-3), "run_ms": ms,
           "mean_events_per_scenario": events / n_scen, "classes": {"quarks": int(cls[0]), "blips": int(cls[1]),
                                                                    "sparks": int(cls[2])}}
    out["cpu_baseline"] = qs_cpu_baseline(params, coords, added, cpu_budget_s)
    out["device_vs_one_cpu_thread"] = dev / out["cpu_baseline"]["value"]
    return out


def params_dt_ms(params):
    return float(params["dt, ns"]) * 1e-6


def reference_arm(args):
    """The reference's own CPU classes (oracle/_ref) on the host cores, on the
    same sites. The reference has no 3D cytosol, so each site runs the
    reference's 3D cleft (DyadRDCPU) with its well-mixed cytosol pool."""
    from oracle import ref
    p, s, name = workload(args)
    dt_ms = params_dt_ms(p)
    if not ref.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libcasim_ref.so was not built on this machine"}
    import tempfile
    from concurrent.futures import ThreadPoolExecutor
    n_threads = os.cpu_count() or 1
    S = len(s["nx"])
    sample = min(S, n_threads)
    off = np.concatenate([[0], np.cumsum(s["n_ch"])])
    td = tempfile.mkdtemp()
    sims = []
    for i in range(sample):
        q = json.loads(json.dumps(p))
        cpath = os.path.join(td, "c%d.txt" % i)
        np.savetxt(cpath, np.c_[s["ch_x"][off[i]:off[i + 1]], s["ch_y"][off[i]:off[i + 1]]])
        d = q["Dyad"]
        d["Channels"]["RyR"]["Coordinates"] = cpath
        d["x"] = (int(s["nx"][i]) - 1) * d["dx"]
        d["y"] = (int(s["ny"][i]) - 1) * d["dy"]
        d["Seed"] = [int(v) for v in s["seeds"][i]]
        if "3D" in d["Type"]:
            d["Type"] = "CPU3D"
        if q["Cytosol"].get("Type") != "Pool":
            q["Cytosol"] = {"Type": "Pool", "Leak mult": 2e-06,
                            "Buffers": q["Cytosol"].get("Buffers", {}), "SERCA": q["Cytosol"].get("SERCA", {})}
        sim = ref.RefSim(q, 1, 1)
        sim.start([int(s["first_channel"][i])])
        sims.append(sim)
    pool = ThreadPoolExecutor(max_workers=sample)
    chunk = 20
    # calibrate the per-step sample so the whole run stays within a few minutes
    t0 = time.time()
    list(pool.map(lambda x: x.step(chunk), sims))
    per = max(time.time() - t0, 1e-3)
    budget = 10.0
    per_step = max(chunk, int(chunk * budget / per / max(args.steps + args.warmup, 1)))
    for _ in range(args.warmup):
        list(pool.map(lambda x: x.step(per_step), sims))
    t0 = time.time()
    for _ in range(args.steps):
        list(pool.map(lambda x: x.step(per_step), sims))
    dt = time.time() - t0
    value = sample * per_step * args.steps * dt_ms / dt
    sample_txt = "%d sites of the workload (3D clefts, reference pool cytosol) x %d time steps per step" % (sample, per_step)
    return {
        "impl": "reference", "metric": "simulated site-ms/s", "value": value, "unit": "site-ms/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": name, "cpu_sample": sample_txt,
                   "cytosol": "the reference's well-mixed cytosol pool (CaSim/CytosolPool.cpp) in place of the 25^3 RD3D "
                              "grid, which the reference does not have: about 43 % fewer node-steps per site than the GPU arm"
                   if cyto_nodes_of(p) else "the reference's well-mixed cytosol pool, as the GPU arm"},
        "cpu_baseline": {"value": value, "unit": "site-ms/s", "cores": sample, "kind": "reference", "sample": sample_txt,
                         "cpu_model": cpu_model()},
        "e2e": {"value": value, "unit": "site-ms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    env_world = int(os.environ.get("WORLD_SIZE", "0"))
    rank = int(os.environ.get("RANK", "0"))
    if args.surrogate_frontier:
        print(json.dumps(surrogate_report(hybrid=FRONTIER_ARMS)))
        return 0
    if args.impl == "reference":
        # the reference's CPU classes on the host cores: rank 0 alone (the others exit 0)
        if rank == 0:
            print(json.dumps(reference_arm(args)))
        return 0
    if args.gpus > 1 and env_world == 0:
        return launch_ranks(args)
    world = env_world or 1
    if world != args.gpus:
        sys.stderr.write("bench.py: --gpus %d but WORLD_SIZE %d\n" % (args.gpus, world))
        return 2
    import torch
    import casim_b200 as cb
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    p, s_global, name = workload(args, world)
    stream = torch.cuda.Stream()
    timing = {}

    def make_sim(params, sites):
        sim = cb.ReleaseSiteBatch(params, sites, precision=args.precision, path=args.path)
        sim.set_stream(stream.cuda_stream)
        return sim

    def run(sim, sites):
        sim.start(sites["first_channel"])
        for _ in range(args.warmup):
            sim.step(args.chunk)
        sim.synchronize()
        timing["launches_per"] = sim.last_step_launches()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        with Clocks(local) as clk:
            with torch.cuda.stream(stream):
                ev0.record(stream)
                for _ in range(args.steps):
                    sim.step(args.chunk)
                ev1.record(stream)
            torch.cuda.synchronize()
        if dist:
            dist.barrier()
        from casim_b200 import dist as cdist
        timing["ms"] = cdist.max_over_ranks(ev0.elapsed_time(ev1), device="cuda")
        timing["clocks"] = clk.summary()

    sim, s, _, outputs = sharded_run(p, s_global, world, rank, make_sim, run)
    ms = timing["ms"]
    dt_ms = sim.info.dt_ms
    total_sites = len(s_global["nx"])
    value = total_sites * args.chunk * args.steps * dt_ms / (ms / 1e3)
    ok_finite, _ = sim.check_finite()
    bytes_step = algorithmic_bytes_per_step(sim, s, p)
    peak, peak_kind = measured_peak_hbm()
    roof = dominant_kernel(args, sim, s, bytes_step, peak)
    result = {
        "metric": "simulated site-ms/s", "value": value, "unit": "site-ms/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic",
        "config": {"workload": name, "sites_per_gpu": sim.S, "sites_total": total_sites,
                   "sharding": "one global table, cost-balanced partition by node-steps (casim_b200.dist.partition); "
                               "no exchange in the time loop",
                   "time_steps_per_bench_step": args.chunk,
                   "dt_ns": float(p["dt, ns"]), "path": sim.path, "precision": args.precision,
                   "l2": "state of %.2f GB per GPU is larger than the 126 MB L2" % (bytes_step / 2 / 1e9)},
        "gpu_launches": int(timing["launches_per"] * args.steps),
        "finite": bool(ok_finite),
        "outputs": outputs_summary(outputs) if rank == 0 else None,
        "roofline": dict(roof, peak=peak, peak_kind=peak_kind),
        "clocks": timing["clocks"],
    }
    if not args.no_e2e:
        # batch scenarios through the public API: new initial conditions in,
        # outputs out, as one RunSimulations batch of --chunk steps
        rng = np.random.default_rng(7 + rank)
        h2d = d2h = 0
        n_e2e = max(1, min(args.steps, 5))
        t0 = time.time()
        for k in range(n_e2e):
            first = rng.integers(0, np.asarray(s["n_ch"])).astype(np.int32)
            jsr = rng.uniform(900.0, 1100.0, size=(sim.S, sim.info.n_ions))
            sim.set_site_jsr(jsr)
            sim.start(first)
            sim.step(args.chunk)
            mouth = sim.all_mouth(0)
            states = sim.all_states()
            h2d = first.nbytes + jsr.nbytes
            d2h = mouth.nbytes + states.nbytes
        el = time.time() - t0
        if dist:
            from casim_b200 import dist as cdist
            el = cdist.max_over_ranks(el, device="cuda")
        result["e2e"] = {"value": total_sites * args.chunk * n_e2e * dt_ms / el, "unit": "site-ms/s",
                         "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": n_e2e}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            result["cpu_baseline"] = cpu_baseline(args, p, s, args.cpu_seconds)
        except Exception as e:  # the baseline is reported, never required
            result["cpu_baseline"] = {"error": str(e)}
    if rank == 0 and world == 1 and not args.no_accuracy:
        try:
            result["accuracy"] = accuracy_report(args, p, s)
        except Exception as e:  # reported next to the headline, never required
            result["accuracy"] = {"error": str(e)}
    if rank == 0 and world == 1 and not args.no_qs:
        try:
            result["quasi_stationary"] = qs_report()
        except Exception as e:  # reported next to the headline, never required
            result["quasi_stationary"] = {"error": str(e)}
    if rank == 0 and world == 1 and not args.no_surrogate:
        try:
            result["surrogate"] = surrogate_report()
        except Exception as e:  # reported next to the headline, never required
            result["surrogate"] = {"error": str(e)}
    sim.close()
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result))
    return 0


if __name__ == "__main__":
    sys.exit(main())

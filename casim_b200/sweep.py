"""Large sweep (config 5): 16384 3D release sites with 10..150 RyRs and 1 mM
Mg, half gated by the tetrameric MWC law (TwoStateMWC) and half by the same
law tabulated for TwoStateSpline, run side by side on one GPU.

The two halves are two batches (a batch holds one gating model), each on its
own CUDA stream; the simulated site-ms/s counts both. After the run the open
RyR counts and the released Ca of the halves are compared by two-sample KS
tests: the tabulated law is the analytic one up to the spline's interpolation
error, so the distributions should agree.

    python -m casim_b200.sweep --sites 16384 --ms 0.2
"""
import argparse
import json
import time

import numpy as np

from . import ReleaseSiteBatch, configs


def run_sweep(n_sites=16384, t_ms=0.2, chunk=200, precision="fp32", seed=5, path="auto"):
    import torch
    from scipy.stats import ks_2samp
    halves = configs.config5(n_sites=n_sites, seed=seed)
    sims, streams = [], []
    for p, s in halves:
        sim = ReleaseSiteBatch(p, s, precision=precision, path=path)
        st = torch.cuda.Stream()
        sim.set_stream(st.cuda_stream)
        sim.start(s["first_channel"])
        sims.append(sim)
        streams.append(st)
    dt_ms = sims[0].info.dt_ms
    n_steps = int(round(t_ms / dt_ms))
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for st in streams:
        st.wait_event(ev0)
    done = 0
    launches = 0
    while done < n_steps:
        k = min(chunk, n_steps - done)
        for sim in sims:
            sim.step(k)
            launches += sim.last_step_launches()
        done += k
    for st in streams:
        torch.cuda.current_stream().wait_stream(st)
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    out = {"workload": "%d 3D dyads side~U{40..120}x3, 10..150 RyR, 25^3 RD cytosol, 1 mM Mg; "
                       "half TwoStateMWC, half TwoStateSpline (config 5)" % n_sites,
           "precision": precision, "paths": [sim.path for sim in sims], "t_ms": n_steps * dt_ms,
           "device_ms": ms, "site_ms_per_s": n_sites * n_steps * dt_ms / (ms / 1e3), "gpu_launches": launches,
           "finite": [bool(sim.check_finite()[0]) for sim in sims], "halves": []}
    opens, rels = [], []
    for sim, (p, s) in zip(sims, halves):
        off = np.concatenate([[0], np.cumsum(s["n_ch"])])
        st = sim.all_states()
        oc = np.add.reduceat(st, off[:-1])
        rel = np.array([sim.release(k) for k in range(sim.S)])
        opens.append(oc)
        rels.append(rel)
        out["halves"].append({"model": p["Dyad"]["Channels"]["RyR"]["Model"], "sites": sim.S,
                              "mean_open": float(oc.mean()), "mean_release": float(rel.mean())})
    out["ks_p_open"] = float(ks_2samp(opens[0], opens[1]).pvalue)
    out["ks_p_release"] = float(ks_2samp(rels[0], rels[1]).pvalue)
    for sim in sims:
        sim.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sites", type=int, default=16384)
    ap.add_argument("--ms", type=float, default=0.2, help="simulated time per site")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    a = ap.parse_args()
    t0 = time.time()
    res = run_sweep(a.sites, a.ms, precision=a.precision)
    res["wall_s"] = time.time() - t0
    print(json.dumps(res))


if __name__ == "__main__":
    main()

"""Precision study of the mixed-precision path (config 3).

The production precision keeps the cleft stencil and buffer kinetics in FP32
and the jSR pool, the cytosol pool and the accumulated release flux in FP64.
This module runs the same sites twice on the device, once in that mixed mode
and once all in FP64 (the FP64 device path matches the C restatement of the
reference's CPU classes to 1e-11 and draw for draw; a CPU run of 1024 sites
for 100 ms, 8e12 node-steps, is out of reach), and reports at each horizon:

* mouth Ca: relative error of the Ca at every RyR mouth;
* jSR depletion: relative error of jSR_init - jSR(t);
* total release: relative error of the accumulated RyR flux of the site.

Both runs draw the same MRG32k3a numbers, but a draw that falls within the
rounding difference of a transition probability takes the two runs apart.
Errors are therefore taken over the sites still in lockstep (identical RyR
states and identical draw counts), and every site enters a two-sample
Kolmogorov-Smirnov comparison of the release and jSR distributions.

    python -m casim_b200.precision --sites 1024 --horizons 10,100
    python -m casim_b200.precision --distributions 2000
"""
import argparse
import json
import time

import numpy as np

from . import ReleaseSiteBatch, configs


def _rel(a, b, floor):
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


def _summary(x):
    if x.size == 0:
        return {"median": None, "p99": None, "max": None}
    return {"median": float(np.median(x)), "p99": float(np.quantile(x, 0.99)), "max": float(np.max(x))}


def snapshot(sim):
    """Per-site state of a batch: RyR states, mouth Ca, jSR Ca, release, draws."""
    S = sim.S
    return {
        "states": sim.all_states(),
        "mouth": sim.all_mouth(0),
        "jsr": np.array([sim.jsr(s)[0] for s in range(S)]),
        "release": np.array([sim.release(s) for s in range(S)]),
        "draws": np.array([sim.draws(s) for s in range(S)], dtype=np.int64),
    }


def compare(a, b, n_ch, jsr_init):
    """Errors of snapshot `a` (mixed precision) against snapshot `b` (FP64)."""
    from scipy.stats import ks_2samp
    off = np.concatenate([[0], np.cumsum(n_ch)])
    S = len(n_ch)
    same = np.array([a["draws"][s] == b["draws"][s] and np.array_equal(a["states"][off[s]:off[s + 1]], b["states"][off[s]:off[s + 1]])
                     for s in range(S)])
    ch_same = np.repeat(same, n_ch)
    mouth = _rel(a["mouth"][ch_same], b["mouth"][ch_same], 1e-30)
    open_mouth = _rel(a["mouth"][ch_same & (b["states"] == 1)], b["mouth"][ch_same & (b["states"] == 1)], 1e-30)
    dep_a, dep_b = jsr_init - a["jsr"], jsr_init - b["jsr"]
    # depletion relative to its own size, floored at 1e-6 of the initial jSR Ca
    dep = _rel(dep_a[same], dep_b[same], 1e-6 * jsr_init[same])
    rel = _rel(a["release"][same], b["release"][same], 1e-30)
    openc_a = np.add.reduceat(a["states"], off[:-1])
    openc_b = np.add.reduceat(b["states"], off[:-1])
    return {
        "lockstep_sites": int(same.sum()), "sites": S,
        "mouth_ca_rel_err": _summary(mouth), "open_mouth_ca_rel_err": _summary(open_mouth),
        "jsr_depletion_rel_err": _summary(dep), "release_rel_err": _summary(rel),
        "ks_p_release": float(ks_2samp(a["release"], b["release"]).pvalue),
        "ks_p_jsr": float(ks_2samp(a["jsr"], b["jsr"]).pvalue),
        "ks_p_open": float(ks_2samp(openc_a, openc_b).pvalue),
        "mean_release": [float(a["release"].mean()), float(b["release"].mean())],
        "mean_jsr_depletion": [float(dep_a.mean()), float(dep_b.mean())],
    }


def precision_study(n_sites=1024, horizons_ms=(10.0, 100.0), seed=3, chunk=20000, path="auto"):
    """Config 3: `n_sites` 2D 64x64 clefts with 50 RyRs and jSR Ca ~ U[0.5, 1.5]
    mM, one RyR opened at t = 0; mixed precision against FP64 at each horizon."""
    p, s = configs.config3(n_sites=n_sites, seed=seed)
    jsr_init = s["jsr_init"][:, 0].copy()
    sims = {prec: ReleaseSiteBatch(p, s, precision=prec, path=path) for prec in ("fp32", "fp64")}
    for sim in sims.values():
        sim.start(s["first_channel"])
    dt_ms = sims["fp32"].info.dt_ms
    done = {k: 0 for k in sims}
    dev_ms = {k: 0.0 for k in sims}
    out = {"workload": "%d 2D 64x64 clefts, 50 RyR, jSR Ca ~U[0.5,1.5] mM (config 3)" % n_sites,
           "paths": {k: v.path for k, v in sims.items()}, "horizons": []}
    for h in horizons_ms:
        target = int(round(h / dt_ms))
        for k, sim in sims.items():
            while done[k] < target:
                n = min(chunk, target - done[k])
                sim.step(n)
                sim.synchronize()
                dev_ms[k] += sim.last_step_ms()
                done[k] += n
        row = {"t_ms": h}
        row.update(compare(snapshot(sims["fp32"]), snapshot(sims["fp64"]), np.asarray(s["n_ch"]), jsr_init))
        row["site_ms_per_s"] = {k: n_sites * done[k] * dt_ms / (dev_ms[k] / 1e3) for k in sims}
        out["horizons"].append(row)
    for sim in sims.values():
        sim.close()
    return out


def distribution_study(n_sites=2000, t_ms=1.0, every=100, nadir=2):
    """Config 1 (2D 64 x 64, 20 RyRs, one RyR opened at t = 0) run `n_sites`
    times in the mixed precision and `n_sites` times all in FP64 from
    disjoint seeds; two-sample KS tests of the per-run release-event metrics
    of the device analysis (peak open RyRs, time to peak, time to end,
    integral, open probability = mean open count / RyRs) and of the released
    Ca. Open-RyR counts are sampled every `every` time steps."""
    from scipy.stats import ks_2samp
    runs = {}
    for prec, seed0 in (("fp32", 1), ("fp64", 1 + 10 * n_sites)):
        p, s = configs.config1(n_sites=n_sites, seed0=seed0)
        sim = ReleaseSiteBatch(p, s, precision=prec, path="auto")
        sim.start(s["first_channel"])
        steps = int(round(t_ms / sim.info.dt_ms))
        sim.trace_enable(every, steps // every + 1)
        sim.step(steps)
        an = sim.release_analysis(t_ms, nadir, hist_dt_ms=every * sim.info.dt_ms)
        runs[prec] = {"amplitude": an["amp"], "time_to_peak": an["ttp"], "time_to_end": an["tte"],
                      "integral": an["integral"], "open_probability": an["mean"] / float(s["n_ch"][0]),
                      "release": np.array([sim.release(k) for k in range(sim.S)])}
        sim.close()
    out = {"workload": "config 1, %d runs per precision, %.3g ms, seeds disjoint" % (n_sites, t_ms), "metrics": {}}
    rng = np.random.default_rng(12345)
    for k in runs["fp32"]:
        a, b = np.asarray(runs["fp32"][k], float), np.asarray(runs["fp64"][k], float)
        row = {"mean_fp32": float(np.mean(a)), "mean_fp64": float(np.mean(b))}
        if k == "time_to_end" and np.all(a >= t_ms - 1e-9) and np.all(b >= t_ms - 1e-9):
            # no event ended inside the window: censored at t_ms in every run, no test
            row["censored_at_ms"] = t_ms
        else:
            row["ks_p"] = float(ks_2samp(a, b).pvalue)
            row.update(bootstrap_mean_difference(a, b, rng))
        out["metrics"][k] = row
    return out


def bootstrap_mean_difference(a, b, rng, n_boot=2000, level=0.95):
    """Percentile bootstrap interval of mean(a) - mean(b) (the two samples resampled
    independently): whether a difference of the means is inside sampling noise."""
    d = np.empty(n_boot)
    for i in range(n_boot):
        d[i] = np.mean(rng.choice(a, a.size)) - np.mean(rng.choice(b, b.size))
    lo, hi = np.percentile(d, [50 * (1 - level), 50 * (1 + level)])
    return {"mean_difference": float(np.mean(a) - np.mean(b)), "ci95": [float(lo), float(hi)],
            "difference_inside_noise": bool(lo <= 0.0 <= hi)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sites", type=int, default=1024)
    ap.add_argument("--horizons", default="10,100", help="report times in ms, comma separated")
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--distributions", type=int, default=0,
                    help="instead: release-event distributions of this many config-1 runs per precision")
    a = ap.parse_args()
    import torch
    torch.cuda.init()
    t0 = time.time()
    if a.distributions:
        res = distribution_study(a.distributions)
    else:
        res = precision_study(a.sites, tuple(float(x) for x in a.horizons.split(",")), seed=a.seed)
    res["wall_s"] = time.time() - t0
    print(json.dumps(res))


if __name__ == "__main__":
    main()

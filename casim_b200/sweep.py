"""Large sweep (config 5): 16384 3D release sites with 10..150 RyRs and 1 mM
Mg, half gated by the tetrameric MWC law (TwoStateMWC) and half by the same
law tabulated for TwoStateSpline, run side by side on one GPU.

By default (--path mixed) both halves are one batch, the second half's sites
gated by their own law (casim_b200_set_site_gating). With --path auto each half
is one batch on the path the library picks (a batch this large streams its
fields from HBM). With
--path split each half is ordered by size and split at the largest cleft side
whose sites the resident path still takes (the largest sites with the second
ion fit no 16-block cluster): the smaller sites run resident, the rest
streaming. The batches run on their own CUDA streams; the simulated
site-ms/s counts all of them. After the run the open RyR counts and the
released Ca of the halves are
compared by two-sample KS tests: the tabulated law is the analytic one up to
the spline's interpolation error, so the distributions should agree.

    python -m casim_b200.sweep --sites 16384 --ms 0.2
"""
import argparse
import json
import time

import numpy as np

from . import EUNSUPPORTED, CasimError, ReleaseSiteBatch, configs


def split_by_side(sides_of_sites, n_ch, fits):
    """[(site indices, path)]: the sites ordered by cleft side and RyR count,
    split at the largest side for which fits(indices of the sites with that
    side or less) holds (bisection over the distinct sides, so fits is
    called O(log sides) times and must be monotone); the rest run plain."""
    order = np.lexsort((np.asarray(n_ch), np.asarray(sides_of_sites)))
    side = np.asarray(sides_of_sites)[order]
    sides = np.unique(side)
    if sides.size == 0:
        return []
    if fits(order[side <= sides[-1]]):
        return [(order, "resident")]
    lo, hi = -1, len(sides) - 1  # fits for lo (no site, trivially), not for hi
    while hi - lo > 1:
        mid = (lo + hi) // 2
        if fits(order[side <= sides[mid]]):
            lo = mid
        else:
            hi = mid
    if lo < 0:
        return [(order, "plain")]
    cut = int(np.searchsorted(side, sides[lo], side="right"))
    return [(order[:cut], "resident"), (order[cut:], "plain")]


def split_resident(params, sites, precision):
    """split_by_side with the resident path's own answer: each probe builds a
    batch of the candidate sites on the resident path and releases it."""
    def fits(idx):
        try:
            ReleaseSiteBatch(params, configs.subset_sites(sites, idx), precision=precision, path="resident").close()
            return True
        except CasimError as e:
            if e.status != EUNSUPPORTED:
                raise
            return False

    return split_by_side(sites["nx"], sites["n_ch"], fits)


def run_sweep(n_sites=16384, t_ms=0.2, chunk=200, precision="fp32", seed=5, path="auto"):
    halves = configs.config5(n_sites=n_sites, seed=seed)
    sims, parts = [], []
    if path == "mixed":
        # one batch, the second half's sites gated by the second half's law
        (p0, s0), (p1, s1) = halves
        both = {k: (None if s0.get(k) is None else np.concatenate([np.asarray(s0[k]), np.asarray(s1[k])]))
                for k in ("nx", "ny", "nz", "n_ch", "seeds", "jsr_init", "first_channel", "ch_x", "ch_y")}
        sim = ReleaseSiteBatch(p0, both, precision=precision, path="plain")
        n0 = len(s0["nx"])
        sim.set_site_gating(p1, np.arange(n0, n0 + len(s1["nx"])))
        halves_of = np.r_[np.zeros(n0, int), np.ones(len(s1["nx"]), int)]
        return _run(sims=[sim], parts=[(None, both)], halves=halves, half_of=[halves_of], n_sites=n_sites, t_ms=t_ms,
                    chunk=chunk, precision=precision)
    for h, (p, s) in enumerate(halves):
        # "auto": one batch per half and the library's choice (large 3D batches stream);
        # "split": the sites that fit a cluster resident, the rest streaming
        split = split_resident(p, s, precision) if path == "split" else [(np.arange(len(s["nx"])), path)]
        for idx, pth in split:
            if idx.size == 0:
                continue
            sub = configs.subset_sites(s, idx)
            sim = ReleaseSiteBatch(p, sub, precision=precision, path=pth)
            sims.append(sim)
            parts.append((h, sub))
    return _run(sims, parts, halves, [np.full(sub_["nx"].size, h_, int) for h_, sub_ in parts], n_sites, t_ms, chunk, precision)


def _run(sims, parts, halves, half_of, n_sites, t_ms, chunk, precision):
    """Step the batches side by side on their own streams; half_of[b][k]: the half of
    batch b's site k."""
    import torch
    from scipy.stats import ks_2samp
    streams = []
    for sim, (_, sub) in zip(sims, parts):
        st = torch.cuda.Stream()
        sim.set_stream(st.cuda_stream)
        sim.start(sub["first_channel"])
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
           "precision": precision, "batches": [{"half": h if h is not None else "both", "sites": sim.S, "path": sim.path,
                                                "max_side": int(sub["nx"].max())}
                                               for sim, (h, sub) in zip(sims, parts)], "t_ms": n_steps * dt_ms,
           "device_ms": ms, "site_ms_per_s": n_sites * n_steps * dt_ms / (ms / 1e3), "gpu_launches": launches,
           "finite": [bool(sim.check_finite()[0]) for sim in sims], "halves": []}
    opens, rels = [[], []], [[], []]
    for sim, (_, sub), hof in zip(sims, parts, half_of):
        off = np.concatenate([[0], np.cumsum(sub["n_ch"])])
        o = np.add.reduceat(sim.all_states(), off[:-1])
        r = np.array([sim.release(k) for k in range(sim.S)])
        for h in (0, 1):
            opens[h].append(o[hof == h])
            rels[h].append(r[hof == h])
    opens = [np.concatenate(o) for o in opens]
    rels = [np.concatenate(r) for r in rels]
    for h, (p, _) in enumerate(halves):
        out["halves"].append({"model": p["Dyad"]["Channels"]["RyR"]["Model"], "sites": int(opens[h].size),
                              "mean_open": float(opens[h].mean()), "mean_release": float(rels[h].mean())})
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
    ap.add_argument("--path", default="mixed", choices=["auto", "mixed", "split", "plain", "resident"])
    a = ap.parse_args()
    t0 = time.time()
    res = run_sweep(a.sites, a.ms, precision=a.precision, path=a.path)
    res["wall_s"] = time.time() - t0
    print(json.dumps(res))


if __name__ == "__main__":
    main()

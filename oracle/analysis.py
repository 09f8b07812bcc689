"""CPU restatement of the reference's release-event analysis
(CaSim/IndChannelCREAnalyzer.cpp:53-138). Test infrastructure: the checker of the
device analysis (casim_b200_release_analysis), pinned against the reference's own
IndChannelCREAnalyzer compiled into oracle/_ref (tests/test_analysis_cpu.py).

A trace is a list of events: times t_j and the open-RyR count at each event. The
reference's events carry per-channel states and count the open ones
(FindNo, :10-16); with two-state channels that count is all the analysis uses.
"""
import numpy as np


def cre_analysis(times, opens, n_channels, max_time, nadir, dt=0.01):
    """times, opens: one sequence per trace (scenario). Returns per-trace
    [amp, ttp, tte, integral, mean] and the four time histograms with the
    reference's column-0 rule, and the class counts."""
    n_scen = len(times)
    nh = int(max_time / dt)  # long long n_time_hist = Max_time / dt (:58), truncation
    h_all = np.zeros((nh + 1, n_channels + 1), dtype=np.int64)
    h_q = np.zeros((nh + 1, 2), dtype=np.int64)
    h_b = np.zeros((nh + 1, nadir + 1), dtype=np.int64)
    h_s = np.zeros((nh + 1, n_channels + 1), dtype=np.int64)
    out = np.zeros((n_scen, 5))
    counts = [0, 0, 0]

    def fill(h, t, o):
        # WriteIntoHistogram over [cur_idx, min(next_idx, nh)] per event (:17-21, :78-82)
        cur = 0
        n = len(t)
        for j in range(n):
            nx = min(j + 1, n - 1)
            nxt = int(float(t[nx]) / dt)  # long long next_idx = t_next / dt
            for k in range(cur, min(nxt, nh) + 1):
                h[k, int(o[j])] += 1
            cur = nxt + 1

    for i in range(n_scen):
        t = [float(v) for v in times[i]]
        o = [int(v) for v in opens[i]]
        n = len(t)
        amp, ttp, q = 0.0, 0.0, 0.0
        for j in range(n):  # :71-83
            if o[j] > amp:
                amp = float(o[j])
                ttp = t[j]
            nx = min(j + 1, n - 1)
            q += o[j] * (t[nx] - t[j])
        fill(h_all, t, o)
        if amp == 1:  # :85-123 quark / blip / spark
            counts[0] += 1
            fill(h_q, t, o)
        elif amp <= nadir:
            counts[1] += 1
            fill(h_b, t, o)
        else:
            counts[2] += 1
            fill(h_s, t, o)
        tte = t[-1]
        with np.errstate(divide="ignore", invalid="ignore"):
            mean = np.float64(q) / np.float64(tte)
        out[i] = [amp, ttp, tte, q, mean]
    # CalculateGlobalHist: column 0 = class count minus the other columns (:32-38)
    for h, c in ((h_all, n_scen), (h_q, counts[0]), (h_b, counts[1]), (h_s, counts[2])):
        h[:, 0] = c - h[:, 1:].sum(axis=1)
    return {"per_trace": out, "hist": h_all, "hist_quark": h_q, "hist_blip": h_b, "hist_spark": h_s,
            "quarks": counts[0], "blips": counts[1], "sparks": counts[2]}

"""The CPU restatement of the release-event analysis (oracle/analysis.py) against the
reference's own IndChannelCREAnalyzer::RunAnalysis (CaSim/IndChannelCREAnalyzer.cpp:53-138,
compiled into oracle/_ref): per-trace amplitude, time to peak, time to end, integral and
mean (the reference prints 6 significant digits) and the four time histograms (exact)."""
import math

import numpy as np
import pytest

from oracle import analysis, ref

pytestmark = pytest.mark.skipif(not ref.available(), reason="reference library not built")


def _traces(seed, n_scen, n_ch, t_end, max_events=60, uniform=None):
    rng = np.random.default_rng(seed)
    times, states = [], []
    for i in range(n_scen):
        if uniform is not None:
            n = int(t_end / uniform) + 1
            t = np.arange(n) * uniform
        else:
            n = int(rng.integers(1, max_events))
            t = np.sort(rng.uniform(0, t_end, size=n))
            t[0] = 0.0
        st = (rng.uniform(size=(n, n_ch)) < rng.uniform(0, 0.5)).astype(np.int32)
        k = i % 6
        if k == 0:
            st[:] = 0  # never opens: amplitude 0, counted as a blip
        elif k == 1:
            st[:, 1:] = 0  # quark at most
        elif k == 2:
            st[:, 3:] = 0  # amplitude at most 3
        times.append(t)
        states.append(st)
    return times, states


def _compare(r, o):
    a, b = r["per_trace"], o["per_trace"]
    assert a.shape == b.shape
    both_nan = np.isnan(a) & np.isnan(b)
    scale = np.maximum(np.abs(b), 1e-300)
    ok = both_nan | (np.abs(a - b) <= 5e-6 * scale) | (np.abs(a - b) <= 1e-12)
    assert ok.all(), np.argwhere(~ok)[:5]
    for k in ("hist", "hist_quark", "hist_blip", "hist_spark"):
        assert np.array_equal(r[k], o[k]), k


@pytest.mark.parametrize("seed,max_time,nadir", [(1, 0.4, 3), (2, 0.2, 1), (3, 1.0, 5), (4, 0.333, 2)])
def test_oracle_analysis_matches_reference_random_events(seed, max_time, nadir):
    times, states = _traces(seed, 48, 7, 0.5)
    r = ref.cre_analysis(times, states, max_time, nadir)
    o = analysis.cre_analysis(times, [s.sum(axis=1) for s in states], 7, max_time, nadir)
    _compare(r, o)


@pytest.mark.parametrize("step", [0.001, 0.01, 0.03, 0.0025])
def test_oracle_analysis_matches_reference_uniform_samples(step):
    # samples on a grid, as the device records them: bin edges meet sample times exactly
    times, states = _traces(5, 24, 5, 0.3, uniform=step)
    r = ref.cre_analysis(times, states, 0.3, 2)
    o = analysis.cre_analysis(times, [s.sum(axis=1) for s in states], 5, 0.3, 2)
    _compare(r, o)


def test_oracle_analysis_single_event_traces():
    # one event: time to end 0, mean 0/0 (NaN in both)
    times = [np.array([0.0]), np.array([0.0])]
    states = [np.array([[1, 0, 0]], dtype=np.int32), np.array([[0, 0, 0]], dtype=np.int32)]
    r = ref.cre_analysis(times, states, 0.05, 1)
    o = analysis.cre_analysis(times, [s.sum(axis=1) for s in states], 3, 0.05, 1)
    _compare(r, o)
    assert math.isnan(o["per_trace"][0, 4]) and o["quarks"] == 1 and o["blips"] == 1

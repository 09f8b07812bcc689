"""Open-RyR traces recorded on the device and the release-event analysis run on them
(casim_b200_trace_enable / casim_b200_release_analysis) against, respectively, the
channel states read back at the same times and the CPU restatement of
CaSim/IndChannelCREAnalyzer.cpp:53-138 (oracle/analysis.py, pinned against the
reference's own analyzer in test_analysis_cpu.py)."""
import numpy as np
import pytest

import casim_b200 as cb
from casim_b200 import configs
from oracle import analysis

pytestmark = pytest.mark.gpu

N_SITES, N_RYR, SIDE, EVERY = 96, 6, 16, 20


def _sites(seed):
    p = configs.base_params(dim=2, nx=SIDE, ny=SIDE)
    # fast kinetics, so that 0.15 ms holds quarks, blips and sparks
    p["Dyad"]["Channels"]["RyR"]["Parameters"] = configs.sheep_cannell_power_law(k0_per_ms=2.0, kclose_per_ms=20.0)
    rng = np.random.default_rng(seed)
    xs, ys, seeds = [], [], []
    for k in range(N_SITES):
        x, y = configs.lattice(N_RYR, (SIDE - 1) * 5.0, (SIDE - 1) * 5.0, rng, pitch=25.0, jitter=0.0)
        xs += x
        ys += y
        seeds.append([int(v) for v in rng.integers(1, 4294944443, size=6)])
    first = rng.integers(0, N_RYR, size=N_SITES)
    return configs._clean(p), configs.sites_table([SIDE] * N_SITES, [SIDE] * N_SITES, [1] * N_SITES, [N_RYR] * N_SITES, xs, ys,
                                                  seeds, first=first)


@pytest.mark.parametrize("path", ["resident", "plain"])
def test_trace_matches_states_read_at_the_sample_times(cuda_device, path):
    p, s = _sites(3)
    a = cb.ReleaseSiteBatch(p, s, precision="fp32", path=path)
    b = cb.ReleaseSiteBatch(p, s, precision="fp32", path=path)
    for sim in (a, b):
        sim.start(s["first_channel"])
    a.trace_enable(EVERY, 1000)
    for n in (7, 33, 500, 1, 259, 1200):  # step calls that do not meet the sample times
        a.step(n)
    want = [np.array([b.states(k).sum() for k in range(N_SITES)])]
    for _ in range(2000 // EVERY):
        b.step(EVERY)
        want.append(np.array([b.states(k).sum() for k in range(N_SITES)]))
    got = a.open_traces()
    assert got.shape == (N_SITES, 2000 // EVERY + 1)
    assert np.array_equal(got, np.stack(want, axis=1))
    a.close()
    b.close()


@pytest.mark.parametrize("hist_dt,max_time,nadir", [(0.01, 0.15, 2), (0.002, 0.1, 3), (0.0035, 0.2, 1)])
def test_device_analysis_matches_oracle(cuda_device, hist_dt, max_time, nadir):
    p, s = _sites(4)
    sim = cb.ReleaseSiteBatch(p, s, precision="fp32", path="resident")
    sim.start(s["first_channel"])
    sim.trace_enable(EVERY, 400)
    sim.step(3000)
    tr = sim.open_traces()
    got = sim.release_analysis(max_time, nadir, hist_dt_ms=hist_dt)
    ts = EVERY * sim.info.dt_ms
    times = [np.arange(tr.shape[1]) * ts for _ in range(N_SITES)]
    want = analysis.cre_analysis(times, list(tr), int(sim.info.max_channels), max_time, nadir, dt=hist_dt)
    per = np.stack([got[k] for k in ("amp", "ttp", "tte", "integral", "mean")], axis=1)
    np.testing.assert_allclose(per, want["per_trace"], rtol=1e-12, atol=0)
    for k in ("hist", "hist_quark", "hist_blip", "hist_spark"):
        assert np.array_equal(got[k], want[k]), k
    assert (got["quarks"], got["blips"], got["sparks"]) == (want["quarks"], want["blips"], want["sparks"])
    assert got["quarks"] > 0 and got["sparks"] > 0  # the kinetics give every class
    sim.close()

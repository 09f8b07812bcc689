"""Statistical agreement over many runs: the FP32 resident GPU path and the
FP64 CPU restatement (oracle/) simulate 2000 release sites each from
independent seeds (the GPU seeds and the oracle seeds do not overlap); the
distributions of the released Ca, of the number of RyR transitions and of the
number of open RyRs at the end must be statistically indistinguishable
(two-sample Kolmogorov-Smirnov, p > 0.05). Small 16 x 16 clefts with 4 RyRs
keep the oracle's 2000 runs to seconds."""
import numpy as np
import pytest
from scipy.stats import ks_2samp

import casim_b200 as cb
from casim_b200 import configs
from oracle import oracle

pytestmark = pytest.mark.gpu

N_RUNS, STEPS, N_RYR, SIDE = 2000, 3000, 4, 16


def _sites(seed0):
    p = configs.base_params(dim=2, nx=SIDE, ny=SIDE)
    # faster RyR kinetics than the benchmark configs so that 0.15 ms holds transitions
    p["Dyad"]["Channels"]["RyR"]["Parameters"] = configs.sheep_cannell_power_law(k0_per_ms=2.0, kclose_per_ms=20.0)
    rng = np.random.default_rng(seed0)
    xs, ys, seeds = [], [], []
    for k in range(N_RUNS):
        x, y = configs.lattice(N_RYR, (SIDE - 1) * 5.0, (SIDE - 1) * 5.0, rng, pitch=40.0, jitter=0.0)
        xs += x
        ys += y
        seeds.append([int(v) for v in rng.integers(1, 4294944443, size=6)])
    first = rng.integers(0, N_RYR, size=N_RUNS)
    return configs._clean(p), configs.sites_table([SIDE] * N_RUNS, [SIDE] * N_RUNS, [1] * N_RUNS, [N_RYR] * N_RUNS, xs, ys,
                                                  seeds, first=first)


def _observables(sim):
    release = np.array([sim.release(k) for k in range(N_RUNS)])
    # one draw per RyR per step, one more per transition; the opening at start took N_RYR + 1
    transitions = np.array([sim.draws(k) for k in range(N_RUNS)]) - N_RYR * STEPS - (N_RYR + 1)
    n_open = np.array([int(np.sum(sim.states(k))) for k in range(N_RUNS)])
    return release, transitions, n_open


def test_gpu_fp32_and_oracle_fp64_distributions_agree(cuda_device):
    import os
    pg, sg_ = _sites(1)
    po, so = _sites(2)
    sim = cb.ReleaseSiteBatch(pg, sg_, precision="fp32", path="resident")
    sim.start(sg_["first_channel"])
    sim.step(STEPS)
    gpu = _observables(sim)
    sim.close()
    orc = oracle.OracleSim(po, so)
    orc.start(so["first_channel"])
    orc.step(STEPS, os.cpu_count() or 1)
    cpu = _observables(orc)
    assert np.std(gpu[0]) > 0 and np.mean(gpu[1]) > 1.0  # the runs do vary and do gate
    for name, a, b in zip(("release", "transitions", "open at end"), gpu, cpu):
        p = ks_2samp(a, b).pvalue
        assert p > 0.05, (name, p, np.mean(a), np.mean(b))


EVERY = 100  # time steps between open-count samples (5 us)


def test_release_event_distributions_agree(cuda_device):
    """Release-event amplitude (peak open RyRs) and latency (time to peak)
    from the device's traces and device analysis against the same metrics
    of FP64 oracle runs from other seeds (the oracle's open counts sampled at
    the same times, analysed by the CPU restatement of the reference's
    analyzer): two-sample KS, p > 0.05."""
    import os
    from oracle import analysis
    pg, sg_ = _sites(3)
    po, so = _sites(4)
    n_samples = STEPS // EVERY + 1
    sim = cb.ReleaseSiteBatch(pg, sg_, precision="fp32", path="resident")
    sim.start(sg_["first_channel"])
    sim.trace_enable(EVERY, n_samples)
    sim.step(STEPS)
    ts = EVERY * sim.info.dt_ms
    max_time = STEPS * sim.info.dt_ms
    gpu = sim.release_analysis(max_time, 2, hist_dt_ms=ts)
    sim.close()
    orc = oracle.OracleSim(po, so)
    orc.start(so["first_channel"])
    opens = np.zeros((N_RUNS, n_samples), dtype=np.int64)
    opens[:, 0] = [int(np.sum(orc.states(k))) for k in range(N_RUNS)]
    for j in range(1, n_samples):
        orc.step(EVERY, os.cpu_count() or 1)
        opens[:, j] = [int(np.sum(orc.states(k))) for k in range(N_RUNS)]
    times = [np.arange(n_samples) * ts for _ in range(N_RUNS)]
    cpu = analysis.cre_analysis(times, list(opens), N_RYR, max_time, 2, dt=ts)["per_trace"]
    assert np.std(gpu["amp"]) > 0 and np.std(gpu["ttp"]) > 0
    for name, a, b in (("amplitude", gpu["amp"], cpu[:, 0]), ("time to peak", gpu["ttp"], cpu[:, 1])):
        p = ks_2samp(a, b).pvalue
        assert p > 0.05, (name, p, np.mean(a), np.mean(b))

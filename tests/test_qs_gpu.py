"""Quasi-stationary release sites on the device (one scenario per warp) against the CPU
restatement, which reproduces the reference's own Gillespie loop (tests/test_qs_cpu.py):
every scenario on its own stream, identical event sequences (channels, states, draw
counts), event times to 1e-12; the release-event metrics of the device analysis equal
the restatement of IndChannelCREAnalyzer on the same traces; a second run continues
the streams."""
import json
import os

import numpy as np
import pytest

import casim_b200 as cb
from oracle import analysis, qs_oracle
from tests.helpers import load_golden

pytestmark = pytest.mark.gpu


def _setup(tmp_path, n_scen):
    z = load_golden("qs_mwc")
    p = json.loads(bytes(z["params"]).decode())
    np.savetxt(os.path.join(str(tmp_path), "coords.txt"), z["coords"], fmt="%.17g")
    q = cb.QuasiStationarySites(p, n_scen, base_dir=str(tmp_path), max_events=8192)
    cfg = qs_oracle.parse(p, str(tmp_path))
    return q, cfg, q.increments()


def test_device_gillespie_matches_restatement(cuda_device, tmp_path):
    S = 512
    q, cfg, added = _setup(tmp_path, S)
    seeds = qs_oracle.stream_seeds(S)
    first = (np.arange(S) % q.n_ch).astype(np.int32)
    for rnd in range(2):  # the second run continues every scenario's stream
        q.run(first)
        times, opens = [], []
        for s in range(S):
            t, c, st = q.events(s)
            to, co, so, d, seeds[s] = qs_oracle.run(cfg, added, seeds[s], int(first[s]))
            assert np.array_equal(c, co) and np.array_equal(st, so), (rnd, s)
            assert q.draws(s) == d
            if len(t):
                assert np.max(np.abs(t - to) / np.abs(to)) <= 1e-12, (rnd, s)
            times.append(np.concatenate([[0.0], to]))
            opens.append(1 + np.concatenate([[0], np.cumsum(np.where(so == 1, 1, -1))]))
        per, cls = q.analysis(nadir=3)
        ref = analysis.cre_analysis(times, opens, q.n_ch, cfg["max_time"], 3)
        want = ref["per_trace"]
        ok = np.isfinite(want)
        assert np.allclose(per[ok], want[ok], rtol=1e-12, atol=0)
        assert list(cls) == [ref["quarks"], ref["blips"], ref["sparks"]]
    assert ref["sparks"] > 0 and ref["quarks"] > 0
    q.close()


def test_odd_batches_and_storage_limits(cuda_device, tmp_path):
    # fewer scenarios than resident warps, not a multiple of the warps per block
    q, cfg, added = _setup(tmp_path, 37)
    first = ((np.arange(37) * 7) % q.n_ch).astype(np.int32)
    q.run(first)
    seeds = qs_oracle.stream_seeds(37)
    for s in range(37):
        t, c, st = q.events(s)
        to, co, so, d, _ = qs_oracle.run(cfg, added, seeds[s], int(first[s]))
        assert np.array_equal(c, co) and np.array_equal(st, so), s
    q.close()
    # 2 stored events: most traces are truncated (EUNSUPPORTED) and the stored ones are the
    # first events; the run goes on to each scenario's end below 64 x 2 events
    z = load_golden("qs_mwc")
    p = json.loads(bytes(z["params"]).decode())
    q = cb.QuasiStationarySites(p, 64, base_dir=str(tmp_path), max_events=2)
    first = (np.arange(64) % q.n_ch).astype(np.int32)
    with pytest.raises(cb.CasimError) as e:
        q.run(first)
    assert e.value.status in (cb.EUNSUPPORTED, cb.ETIMEOUT)
    seeds = qs_oracle.stream_seeds(64)
    capped = False
    for s in range(64):
        t, c, st = q.events(s)
        to, co, so, d, _ = qs_oracle.run(cfg, added, seeds[s], int(first[s]))
        n = q.event_count(s)
        assert len(t) == min(n, 2) and np.array_equal(c, co[:2]) and np.array_equal(st, so[:2]), s
        if len(to) > 128:
            capped = True
            assert n == 128
        else:
            assert n == len(to) and q.draws(s) == d
    if capped:
        assert e.value.status == cb.ETIMEOUT
    q.close()


def test_warp_kernel_for_large_sites(cuda_device, tmp_path):
    """Sites of more than 32 RyRs run one scenario per warp (k_qs_run): a 40-RyR site
    against the restatement, scenario by scenario."""
    from casim_b200 import configs
    p, coords = configs.quasi_stationary(40, seed=3, max_time=20.0)
    np.savetxt(os.path.join(str(tmp_path), "coords.txt"), coords, fmt="%.17g")
    S = 96
    q = cb.QuasiStationarySites(p, S, base_dir=str(tmp_path), max_events=8192)
    assert q.n_ch == 40
    cfg = qs_oracle.parse(p, str(tmp_path))
    added = q.increments()
    seeds = qs_oracle.stream_seeds(S)
    first = ((np.arange(S) * 11) % q.n_ch).astype(np.int32)
    q.run(first)
    for s in range(S):
        t, c, st = q.events(s)
        to, co, so, d, _ = qs_oracle.run(cfg, added, seeds[s], int(first[s]))
        assert np.array_equal(c, co) and np.array_equal(st, so), s
        assert q.draws(s) == d
        if len(t):
            assert np.max(np.abs(t - to) / np.abs(to)) <= 1e-12, s
    q.close()

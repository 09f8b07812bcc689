"""Large-sweep workload (config 5 shapes at sizes the oracle finishes in
seconds): 3D clefts with 1 mM Mg and the RD3D cytosol, one half gated by the
tetrameric MWC law and one by its spline tabulation. Each half is checked
against the C restatement in FP64 on both device paths, and the side-by-side
sweep runner must keep every field finite."""
import numpy as np
import pytest

import casim_b200 as cb
from casim_b200 import configs
from oracle import oracle
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu


FP32_TOL = 1e-5  # FP32 fields: max abs error over the species' largest value


@pytest.mark.parametrize("path,precision", [("plain", "fp64"), ("resident", "fp32")])
def test_config5_halves_match_oracle(cuda_device, tmp_path, path, precision):
    halves = configs.config5(n_sites=4, seed=9, side=(40, 44), ryr=(10, 150), table_dir=str(tmp_path))
    for params, sites in halves:
        model = params["Dyad"]["Channels"]["RyR"]["Model"]
        sim = cb.ReleaseSiteBatch(params, sites, precision=precision, path=path)
        assert sim.path == path
        orc = oracle.OracleSim(params, sites)
        sim.start(sites["first_channel"])
        orc.start(sites["first_channel"])
        sim.step(150)
        orc.step(150)
        for s in range(sim.S):
            # stored species: ions and ion-buffer pairs, then the RD3D cytosol's Ca
            pairs = [(sim.field(s, sp), orc.field(s, sp)) for sp in range(sim.info.n_ions + sim.info.n_pairs)]
            pairs.append((sim.cyto_field(s, 0), orc.cyto_field(s, 0)))
            for k, (a, b) in enumerate(pairs):
                if precision == "fp64":
                    assert rel_err(a, b) < 1e-11, (model, s, k)
                else:
                    assert np.max(np.abs(a - b)) <= FP32_TOL * np.max(np.abs(b)), (model, s, k)
            if precision == "fp64":
                assert np.array_equal(sim.states(s), orc.states(s))
        sim.close()


@pytest.mark.parametrize("path", ["auto", "split", "mixed"])
def test_sweep_runner_small(cuda_device, path):
    from casim_b200.sweep import run_sweep
    res = run_sweep(n_sites=64, t_ms=0.02, chunk=100, path=path)
    assert all(res["finite"]), res
    assert res["site_ms_per_s"] > 0
    assert [h["model"] for h in res["halves"]] == ["TwoStateMWC", "TwoStateSpline"]
    # every site runs in exactly one batch; resident batches hold the smaller sites of their half
    assert sum(b["sites"] for b in res["batches"]) == 64
    assert [h["sites"] for h in res["halves"]] == [32, 32]
    if path == "mixed":
        assert [b["half"] for b in res["batches"]] == ["both"]
        return
    for half in (0, 1):
        bs = [b for b in res["batches"] if b["half"] == half]
        assert sum(b["sites"] for b in bs) == 32
        if path == "auto":
            assert len(bs) == 1
        elif len(bs) == 2:
            assert [b["path"] for b in bs] == ["resident", "plain"]

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


def test_config5_halves_match_oracle(cuda_device, tmp_path, path="plain"):
    halves = configs.config5(n_sites=4, seed=9, side=(40, 44), ryr=(10, 150), table_dir=str(tmp_path))
    for params, sites in halves:
        sim = cb.ReleaseSiteBatch(params, sites, precision="fp64", path=path)
        orc = oracle.OracleSim(params, sites)
        sim.start(sites["first_channel"])
        orc.start(sites["first_channel"])
        sim.step(150)
        orc.step(150)
        for s in range(sim.S):
            # stored species: ions and ion-buffer pairs, then the RD3D cytosol's Ca
            for sp in range(sim.info.n_ions + sim.info.n_pairs):
                assert rel_err(sim.field(s, sp), orc.field(s, sp)) < 1e-11, (params["Dyad"]["Channels"]["RyR"]["Model"], s, sp)
            assert rel_err(sim.cyto_field(s, 0), orc.cyto_field(s, 0)) < 1e-11
            assert np.array_equal(sim.states(s), orc.states(s))
        sim.close()


def test_sweep_runner_small(cuda_device):
    from casim_b200.sweep import run_sweep
    res = run_sweep(n_sites=64, t_ms=0.02, chunk=100)
    assert all(res["finite"]), res
    assert res["site_ms_per_s"] > 0
    assert [h["model"] for h in res["halves"]] == ["TwoStateMWC", "TwoStateSpline"]

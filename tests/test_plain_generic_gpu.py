"""The plain path's specialised streaming kernels against its generic ones (the
kernels that serve layouts the specialised ones do not: JSON "B200":
{"GenericKernels": true}) on the same sites and seeds: config-2 sites (3D, RD3D
cytosol) and small uneven 2D sites with the pool cytosol. FP64: identical RyR
trajectories and draw counts, fields within 1e-12 (only the block sums of the Update
differ in order); FP32 (the specialised stencils divide with the approximate
reciprocal): the sites whose trajectories stay identical within 1e-5 of each
species' scale."""
import json

import numpy as np
import pytest

import casim_b200 as cb
from casim_b200 import configs

pytestmark = pytest.mark.gpu


def _cases():
    p2, s2 = configs.config2(n_sites=6, seed=77, side=(40, 56), ryr=(10, 40))
    p1, s1 = configs.small_mixed(n_sites=6, seed=5, dim=2, cytosol="Pool")
    return [("config2", p2, s2), ("small2d", p1, s1)]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("case", ["config2", "small2d"])
def test_specialised_equals_generic(cuda_device, precision, case):
    name, params, sites = [c for c in _cases() if c[0] == case][0]
    gen = json.loads(json.dumps(params))
    gen.setdefault("B200", {})["GenericKernels"] = True
    a = cb.ReleaseSiteBatch(params, sites, precision=precision, path="plain")
    b = cb.ReleaseSiteBatch(gen, sites, precision=precision, path="plain")
    for sim in (a, b):
        sim.start(sites["first_channel"])
        sim.step(300)
    ta, tb = a.profile_step(), b.profile_step()  # one more step each, kernels timed
    assert set(ta) == set(tb) == {"gating", "cytosol", "cleft", "update"}
    same = [s for s in range(a.S) if np.array_equal(a.states(s), b.states(s)) and a.draws(s) == b.draws(s)]
    # FP64: every site in lockstep; FP32 (other rounding): nearly every one
    assert len(same) == a.S if precision == "fp64" else len(same) >= a.S - 1
    for s in same:
        for sp in range(a.info.n_ions + a.info.n_pairs):
            fa, fb = a.field(s, sp), b.field(s, sp)
            if precision == "fp64":
                assert np.max(np.abs(fa - fb) / np.maximum(np.abs(fb), 1e-300)) < 1e-12, (s, sp)
            else:
                assert np.max(np.abs(fa - fb)) <= 1e-5 * np.max(np.abs(fb)), (s, sp)
    a.close()
    b.close()

"""Per-site RyR gating models in one batch: config-5 sites, half gated by the
tetrameric MWC law and half by its spline tabulation, run as one plain-path handle
(the MWC model of the JSON, the spline model set on the second half) must give, site
for site, exactly what the two single-model batches give: every site has its own
fields, pools and MRG32k3a stream, so only the gating law differs between them."""
import numpy as np
import pytest

import casim_b200 as cb
from casim_b200 import configs

pytestmark = pytest.mark.gpu


def _concat(a, b):
    out = {}
    for k in ("nx", "ny", "nz", "n_ch", "seeds", "jsr_init", "first_channel", "ch_x", "ch_y"):
        if a.get(k) is None:
            out[k] = None
        else:
            out[k] = np.concatenate([np.asarray(a[k]), np.asarray(b[k])])
    return out


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_mixed_batch_equals_single_model_batches(cuda_device, tmp_path, precision):
    (p_mwc, s_mwc), (p_spl, s_spl) = configs.config5(n_sites=8, seed=9, side=(40, 48), ryr=(10, 150), table_dir=str(tmp_path))
    n0 = len(s_mwc["nx"])
    both = _concat(s_mwc, s_spl)
    mixed = cb.ReleaseSiteBatch(p_mwc, both, precision=precision, path="plain")
    mixed.set_site_gating(p_spl, np.arange(n0, n0 + len(s_spl["nx"])))
    singles = [cb.ReleaseSiteBatch(p, s, precision=precision, path="plain") for p, s in ((p_mwc, s_mwc), (p_spl, s_spl))]
    mixed.start(both["first_channel"])
    for sim, (_, s) in zip(singles, ((p_mwc, s_mwc), (p_spl, s_spl))):
        sim.start(s["first_channel"])
    for sim in [mixed] + singles:
        sim.step(400)
    for h, sim in enumerate(singles):
        for k in range(sim.S):
            m = h * n0 + k
            assert np.array_equal(mixed.states(m), sim.states(k)), (h, k)
            assert mixed.draws(m) == sim.draws(k), (h, k)
            for sp in range(sim.info.n_ions + sim.info.n_pairs):
                assert np.array_equal(mixed.field(m, sp), sim.field(k, sp)), (h, k, sp)
            assert np.array_equal(mixed.cyto_field(m, 0), sim.cyto_field(k, 0))
            assert np.array_equal(mixed.jsr(m), sim.jsr(k))
    for sim in [mixed] + singles:
        sim.close()


def test_site_gating_limits(cuda_device, tmp_path):
    (p_mwc, s_mwc), (p_spl, s_spl) = configs.config5(n_sites=4, seed=9, side=(40, 44), ryr=(10, 150), table_dir=str(tmp_path))
    res = cb.ReleaseSiteBatch(p_mwc, s_mwc, precision="fp32", path="resident")
    with pytest.raises(cb.CasimError) as e:
        res.set_site_gating(p_spl, [0])
    assert e.value.status == cb.EUNSUPPORTED
    res.close()
    sim = cb.ReleaseSiteBatch(p_mwc, s_mwc, precision="fp32", path="plain")
    with pytest.raises(cb.CasimError) as e:
        sim.set_site_gating(p_spl, [len(s_mwc["nx"])])  # no such site
    assert e.value.status == cb.EINVAL
    sim.set_site_gating(p_spl, [0])
    sim.start(s_mwc["first_channel"])
    sim.step(10)
    assert sim.check_finite()[0]
    sim.close()

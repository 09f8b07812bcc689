"""Precision study (config 3 shapes, shortened): the mixed-precision path (FP32
stencil and buffers, FP64 pools and release accumulator) against the all-FP64
device path, which the parity tests pin to the C restatement of the
reference's CPU classes. Same seeds, so most sites stay in lockstep; on those
the mouth Ca, the jSR depletion and the total release must agree within 1 %
(mouth Ca) and 0.1 % (pool quantities)."""
import pytest

from casim_b200.precision import precision_study

pytestmark = pytest.mark.gpu

MOUTH_TOL = 1e-2   # relative, every RyR mouth of the lockstep sites
POOL_TOL = 1e-3    # relative, jSR depletion and accumulated release


def test_mixed_precision_within_one_percent_of_fp64(cuda_device):
    res = precision_study(n_sites=64, horizons_ms=(0.5, 2.0), seed=5)
    for row in res["horizons"]:
        assert row["lockstep_sites"] >= row["sites"] // 2, row
        assert row["mouth_ca_rel_err"]["max"] < MOUTH_TOL, row
        assert row["jsr_depletion_rel_err"]["max"] < POOL_TOL, row
        assert row["release_rel_err"]["max"] < POOL_TOL, row

"""Host-side checks of the C-ABI library that need no GPU: it loads, exports
every symbol include/casim_b200.h declares, and rejects bad input with the
documented status codes before touching the device."""
import json
import os
import re

import pytest

import casim_b200 as cb
from casim_b200 import configs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    with open(os.path.join(ROOT, "include", "casim_b200.h")) as f:
        return sorted(set(re.findall(r"casim_status\s+(casim_b200_\w+)\s*\(", f.read())))


def test_library_exports_every_header_symbol():
    L = cb.lib()
    names = header_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    assert sorted(cb.EXPORTS) == names


def test_malformed_json_is_einval():
    with pytest.raises(cb.CasimError) as e:
        cb.ReleaseSiteBatch({"Dyad": {"dx": 10}})
    assert e.value.status == cb.EINVAL


def test_unstable_dt_is_rejected_before_launch():
    params, sites = configs.small_mixed(n_sites=2, dim=3)
    params["Dyad"]["dz"] = 3.0  # dt*D*sum(2/h^2) > 1
    with pytest.raises(cb.CasimError) as e:
        cb.ReleaseSiteBatch(params, sites)
    assert e.value.status == cb.EUNSTABLE


def test_ryr_outside_grid_is_einval():
    params, sites = configs.small_mixed(n_sites=2)
    sites["ch_x"][0] = 1e6
    with pytest.raises(cb.CasimError) as e:
        cb.ReleaseSiteBatch(params, sites)
    assert e.value.status == cb.EINVAL
    assert "outside the grid" in str(e.value)


def test_bad_seed_is_einval():
    params, sites = configs.small_mixed(n_sites=2)
    sites["seeds"][1] = [5, 0, 0, 0, 0, 0]
    with pytest.raises(cb.CasimError) as e:
        cb.ReleaseSiteBatch(params, sites)
    assert e.value.status == cb.EINVAL


def test_unknown_gating_model_is_einval():
    params, sites = configs.small_mixed(n_sites=1)
    params["Dyad"]["Channels"]["RyR"]["Model"] = "NoSuchModel"
    with pytest.raises(cb.CasimError) as e:
        cb.ReleaseSiteBatch(params, sites)
    assert e.value.status == cb.EINVAL


@pytest.mark.parametrize("entry", ["casim_b200_debug_rng", "casim_b200_rng_draws_static"])
@pytest.mark.parametrize("seed", [[0, 0, 0, 1, 1, 1], [1, 1, 1, 0, 0, 0], [4294967087, 1, 1, 1, 1, 1],
                                  [1, 1, 1, 1, 4294944443, 1]])
def test_generator_entry_points_apply_checkseed(entry, seed):
    """RngStream's CheckSeed rules (CaSim/rngstream.cpp:200-234) hold for the stand-alone
    generator entry points: an invalid seed is EINVAL before any device work."""
    import ctypes
    import numpy as np
    s = np.asarray(seed, dtype=np.uint32)
    out = np.zeros(4)
    st = getattr(cb.lib(), entry)(s.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), 4,
                                  out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert st == cb.EINVAL
    assert "seed" in cb.last_error()

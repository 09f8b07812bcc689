"""casim_b200_rng_draws_static: the MRG32k3a generator for callers that cannot
allocate device memory (its staging buffer is a fixed device array). It must
give exactly the draws of casim_b200_debug_rng, which allocates its buffer,
on consecutive calls that reuse the shared array, leave the device's free
memory unchanged on every call after the first, and reject counts beyond the
array and seeds that RngStream's CheckSeed rejects."""
import ctypes

import numpy as np
import pytest

import casim_b200 as cb

pytestmark = pytest.mark.gpu

MAX_DRAWS = 262144


def _static_draws(seed, n):
    s = np.ascontiguousarray(seed, dtype=np.uint32)
    out = np.full(n, -1.0)
    st = cb.lib().casim_b200_rng_draws_static(s.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), n,
                                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return st, out


def _free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_static_scratch_draws_match_allocating_entry_point(cuda_device):
    for seed, n in (([3] * 6, 50000), ([1, 2, 3, 4, 5, 6], 12345)):
        expected = cb.debug_rng(seed, n)
        for _ in range(2):  # the second call reuses the array the first one filled
            st, got = _static_draws(seed, n)
            assert st == cb.OK, cb.last_error()
            assert np.array_equal(got, expected)


def test_static_scratch_allocates_nothing(cuda_device):
    """After the first call (which may load the module onto the device), repeated
    calls leave the device's free memory exactly where it was."""
    st, _ = _static_draws([7] * 6, 1000)
    assert st == cb.OK, cb.last_error()
    before = _free_bytes()
    for n in (1000, MAX_DRAWS, 77):
        st, _ = _static_draws([7] * 6, n)
        assert st == cb.OK, cb.last_error()
        assert _free_bytes() == before


def test_static_scratch_rejects_oversize(cuda_device):
    st, _ = _static_draws([3] * 6, MAX_DRAWS + 1)
    assert st == cb.EINVAL
    assert "exceed" in cb.last_error()


@pytest.mark.parametrize("seed", [[0, 0, 0, 1, 1, 1], [1, 1, 1, 0, 0, 0], [4294967087, 1, 1, 1, 1, 1],
                                  [1, 1, 1, 1, 4294944443, 1]])
def test_static_scratch_rejects_invalid_seed(cuda_device, seed):
    st, _ = _static_draws(seed, 10)
    assert st == cb.EINVAL
    assert "seed" in cb.last_error()

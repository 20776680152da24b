"""nbExtAccelerationNoAllocCUDA: the external potential with no device allocation.

Callers that cannot call cudaMalloc/cudaFree (cudaFree waits for the whole device;
cudaMalloc can fail under a fixed memory budget) evaluate the potential through a fixed
static device array instead.  Checked through the C ABI against nbExtAccelerationCUDA, which
allocates, on two calls in a row with different points (the shared array keeps the previous
call's contents, so a stale read would show), bit for bit like every potential check here.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_POINTS = 65536


def _call(fn, pot, pos):
    from milkywayathome_client_b200 import _lib
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    acc = np.full_like(pos, np.nan)
    rc = fn(ctypes.byref(pot), _lib.ptr(pos), _lib.ptr(acc), len(pos), 0)
    return rc, acc


def test_no_alloc_matches_allocating_entry_point_twice():
    from milkywayathome_client_b200 import _lib, nbody
    lib = _lib.load()
    pot = nbody.milky_way_potential()
    rng = np.random.default_rng(31)
    first = rng.normal(scale=20.0, size=(MAX_POINTS, 3))          # fills the whole array
    second = rng.normal(scale=5.0, size=(1000, 3))                  # then a smaller call
    for pos in (first, second):
        rc_ref, want = _call(lib.nbExtAccelerationCUDA, pot, pos)
        rc, got = _call(lib.nbExtAccelerationNoAllocCUDA, pot, pos)
        assert rc == rc_ref == 0
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


def test_no_alloc_leaves_device_memory_unchanged():
    """The property the entry point exists for: repeated calls take no device memory (the
    device's free memory, as cudaMemGetInfo reports it, is the same before and after)."""
    import torch
    from milkywayathome_client_b200 import _lib, nbody
    lib = _lib.load()
    pot = nbody.milky_way_potential()
    pos = np.random.default_rng(7).normal(scale=15.0, size=(4096, 3))
    assert _call(lib.nbExtAccelerationNoAllocCUDA, pot, pos)[0] == 0      # set-up call
    torch.cuda.synchronize(0)
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(200):
        assert _call(lib.nbExtAccelerationNoAllocCUDA, pot, pos)[0] == 0
    torch.cuda.synchronize(0)
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0


def test_no_alloc_rejects_more_points_than_the_array_holds():
    from milkywayathome_client_b200 import _lib, nbody
    lib = _lib.load()
    pos = np.zeros((MAX_POINTS + 1, 3))
    rc, _ = _call(lib.nbExtAccelerationNoAllocCUDA, nbody.milky_way_potential(), pos)
    assert rc == _lib.NBODY_USER_ERROR
    assert "exceed" in _lib.last_error()

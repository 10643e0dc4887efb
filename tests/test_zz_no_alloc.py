"""pppm_spatial_hash_noalloc: the spatial hash for callers that cannot
allocate device memory (a simulation loop whose frame budget cannot absorb the
device synchronisation of cudaMalloc, an allocator of fixed size, or a device
heap owned by another framework's pool).  It must give exactly what the
allocating entry point pppm_hasher_run gives — sorted keys, sorted indices and
cell start/end tables are integer results, so the comparison is bit-exact —
on two calls in a row, whatever the shared scratch holds from before.  A small
case is also checked against the CPU oracle's hash (its own keys, stable sort
and cell tables), so a fault shared by both GPU entry points cannot hide, and
a call made while every library allocation is armed to fail must still
succeed: it allocates nothing.

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pppm_vortex_bouyant_flow_sample_b200 import _lib
    lib = _lib.load()
    lib.pppm_spatial_hash_noalloc.restype = C.c_int
    lib.pppm_spatial_hash_noalloc.argtypes = [C.c_uint32, C.c_void_p, C.c_uint32, C.c_float,
                                              C.POINTER(C.c_float), C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.c_void_p, C.c_void_p]
    return lib, torch


def _reference_tables(lib, torch, pos, n, h, origin):
    """The allocating path: pppm_hasher_create + pppm_hasher_run."""
    from pppm_vortex_bouyant_flow_sample_b200 import _lib
    N = pos.shape[0]
    handle = C.c_void_p()
    _lib.check(lib.pppm_hasher_create(N, n, None, C.byref(handle)), "pppm_hasher_create")
    try:
        o = (C.c_float * 3)(*origin)
        _lib.check(lib.pppm_hasher_run(handle, N, C.c_void_p(pos.data_ptr()), C.c_float(h), o), "pppm_hasher_run")
        ptrs = [C.c_void_p() for _ in range(4)]
        _lib.check(lib.pppm_hasher_tables(handle, *[C.byref(p) for p in ptrs]), "pppm_hasher_tables")
        torch.cuda.synchronize()
        out = []
        for p, count in zip(ptrs, (N, N, n ** 3, n ** 3)):
            t = torch.empty(count, dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            _copy_dev(torch, t, p.value, count)
            out.append(t.cpu().numpy().view(np.uint32))
        return out
    finally:
        lib.pppm_hasher_destroy(handle)


def _copy_dev(torch, dst, src_ptr, count):
    class View:
        __cuda_array_interface__ = {"shape": (count,), "typestr": "<i4", "data": (src_ptr, False),
                                    "version": 2, "strides": None}
    dst.copy_(torch.as_tensor(View(), device="cuda"))


def _noalloc(lib, torch, pos, n, h, origin):
    N = pos.shape[0]
    outs = [torch.full((c,), -7, dtype=torch.int32, device="cuda") for c in (N, N, n ** 3, n ** 3)]
    o = (C.c_float * 3)(*origin)
    rc = lib.pppm_spatial_hash_noalloc(N, C.c_void_p(pos.data_ptr()), n, C.c_float(h), o,
                                       *[C.c_void_p(t.data_ptr()) for t in outs], None)
    assert rc == 0, lib.pppm_last_error()
    torch.cuda.synchronize()
    return [t.cpu().numpy().view(np.uint32) for t in outs]


@pytest.mark.parametrize("n", [64, 128])
def test_noalloc_matches_allocating_hash_twice(env, n):
    lib, torch = env
    rng = np.random.default_rng(n)
    cases = []
    for N, spread in ((300_000, 1.0), (120_000, 0.4)):
        pos = np.zeros((N, 4), np.float32)
        pos[:, :3] = rng.random((N, 3), dtype=np.float32) * np.float32(spread) + np.float32(0.1)
        cases.append(torch.from_numpy(pos).cuda())
    h, origin = 1.3 / n, (0.05, 0.02, 0.08)
    for pos in cases:  # two calls in a row with different inputs and sizes
        got = _noalloc(lib, torch, pos, n, h, origin)
        ref = _reference_tables(lib, torch, pos, n, h, origin)
        for g, r, name in zip(got, ref, ("sorted_key", "sorted_idx", "cell_start", "cell_end")):
            assert np.array_equal(g, r), name


def test_noalloc_rejects_oversize_without_touching_gpu(env):
    lib, torch = env
    from pppm_vortex_bouyant_flow_sample_b200 import _lib
    N = _lib.NOALLOC_MAX_PARTICLES + 1
    o = (C.c_float * 3)(0.0, 0.0, 0.0)
    # real (small) buffers; the size check rejects the call before any use
    pos = torch.zeros((16, 4), dtype=torch.float32, device="cuda")
    outs = [torch.zeros(64 ** 3, dtype=torch.int32, device="cuda") for _ in range(4)]
    rc = lib.pppm_spatial_hash_noalloc(N, C.c_void_p(pos.data_ptr()), 64, C.c_float(0.01), o,
                                       *[C.c_void_p(t.data_ptr()) for t in outs], None)
    assert rc == 1  # PPPM_ERR_INVALID
    assert b"exceeds the fixed scratch limit" in lib.pppm_last_error()


def test_noalloc_matches_oracle_and_allocates_nothing(env):
    lib, torch = env
    from oracle import pyoracle as O
    n, N = 32, 20_000
    rng = np.random.default_rng(7)
    pos = np.zeros((N, 4), np.float32)
    pos[:, :3] = rng.random((N, 3), dtype=np.float32) * np.float32(0.9) + np.float32(0.03)
    h, origin = np.float32(1.0 / n), np.array([0.0, 0.0, 0.0], np.float32)
    dpos = torch.from_numpy(pos).cuda()
    _noalloc(lib, torch, dpos, n, float(h), origin)  # warm: the scratch address is looked up once
    key, idx = O.calc_hash(pos, n, h, origin)
    skey, sidx = O.sort_by_key(key, idx)
    start, end = O.find_cell_start(skey, n ** 3)
    lib.pppm_debug_fail_allocation.argtypes = [C.c_int64]
    lib.pppm_debug_fail_allocation(0)  # the next library allocation, if any, fails
    try:
        got = _noalloc(lib, torch, dpos, n, float(h), origin)
    finally:
        lib.pppm_debug_fail_allocation(-1)
    for g, r, name in zip(got, (skey, sidx, start, end), ("sorted_key", "sorted_idx", "cell_start", "cell_end")):
        assert np.array_equal(g, r), name

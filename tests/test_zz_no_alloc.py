"""sph3_morton_sort_noalloc: the Morton sort for callers that cannot allocate
device memory (a caller-owned pool or arena, a host framework that owns the
allocator, or a loop that cannot pay for cudaMalloc).  It keeps its scratch
in a fixed static device array, so it must give exactly what the allocating
entry point (sph3_set_particles + sph3_morton_order) gives -- integer keys
and indices, compared bit for bit -- on two calls in a row that share that
array.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_sort(pos_np, max_level, want_order=True, want_keys=True):
    import torch
    from sph_3_b200 import _lib
    lib = _lib.load()
    n = pos_np.shape[0]
    pos = torch.from_numpy(np.ascontiguousarray(pos_np)).cuda()
    order = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    keys = torch.zeros(n, dtype=torch.int64, device="cuda")
    status = torch.full((1,), 0x5A5A, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.sph3_morton_sort_noalloc(ctypes.c_void_p(pos.data_ptr()), n, max_level,
                                      ctypes.c_void_p(order.data_ptr()) if want_order else None,
                                      ctypes.c_void_p(keys.data_ptr()) if want_keys else None,
                                      ctypes.c_void_p(status.data_ptr()), ctypes.c_void_p(stream))
    assert rc == 0, _lib.error_string(rc)
    torch.cuda.synchronize()
    return (order.cpu().numpy() if want_order else None,
            keys.cpu().numpy().view(np.uint64) if want_keys else None, int(status.cpu()[0]))


def _allocating_sort(pos_np, max_level):
    from sph_3_b200 import Config, Context
    ctx = Context(Config(max_level=max_level))
    try:
        ctx.set_particles(pos_np, np.full(pos_np.shape[0], 1.0 / pos_np.shape[0]))
        return ctx.morton_order()
    finally:
        ctx.close()


def test_noalloc_sort_matches_allocating_entry_point_twice():
    from sph_3_b200.ic import evrard
    cases = [(evrard(50000, seed=21)["pos"], 16), (evrard(65536, seed=22)["pos"] * 3.0 + 0.25, 21)]
    for pos, lvl in cases:  # two calls in a row on the shared static scratch
        o1, k1, st = _noalloc_sort(pos, lvl)
        o2, k2 = _allocating_sort(pos, lvl)
        assert st == 0
        assert np.array_equal(k1, k2)
        assert np.array_equal(o1, o2)


@pytest.mark.parametrize("n", [1, 7, 4095, 4097])
def test_noalloc_sort_small_sizes_and_single_outputs(n):
    """Sizes below and around one sort tile (4,096 keys), with each output
    alone, against the allocating path."""
    pos = np.random.default_rng(n).normal(size=(n, 3))
    o2, k2 = _allocating_sort(pos, 16)
    o1, k1, st = _noalloc_sort(pos, 16)
    assert st == 0 and np.array_equal(o1, o2) and np.array_equal(k1, k2)
    o1, _, _ = _noalloc_sort(pos, 16, want_keys=False)
    _, k1, _ = _noalloc_sort(pos, 16, want_order=False)
    assert np.array_equal(o1, o2) and np.array_equal(k1, k2)


def test_noalloc_sort_reports_non_finite_input():
    pos = np.random.default_rng(3).random((1000, 3))
    pos[17, 1] = np.nan
    _, _, st = _noalloc_sort(pos, 16)
    from sph_3_b200 import _lib
    assert st & _lib.C["SPH3_STATUS_NAN_INPUT"]
    _, _, st = _noalloc_sort(pos[:17], 16)  # cleared by the next call
    assert st == 0


def test_noalloc_sort_rejects_bad_arguments():
    import torch
    from sph_3_b200 import _lib
    lib = _lib.load()
    n = 65537
    pos = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    order = torch.zeros(n, dtype=torch.int64, device="cuda")
    p, o = ctypes.c_void_p(pos.data_ptr()), ctypes.c_void_p(order.data_ptr())
    assert lib.sph3_morton_sort_noalloc(p, n, 16, o, None, None, None) == _lib.C["SPH3_ERR_TOO_LARGE"]
    for lvl in (3, 22):
        assert lib.sph3_morton_sort_noalloc(p, 100, lvl, o, None, None, None) == _lib.C["SPH3_ERR_INVALID_ARG"]
    assert lib.sph3_morton_sort_noalloc(p, 100, 16, None, None, None, None) == _lib.C["SPH3_ERR_INVALID_ARG"]

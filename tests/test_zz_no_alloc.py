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


def _noalloc_sort(pos_np, max_level):
    import torch
    from sph_3_b200 import _lib
    lib = _lib.load()
    n = pos_np.shape[0]
    pos = torch.from_numpy(np.ascontiguousarray(pos_np)).cuda()
    order = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    keys = torch.zeros(n, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.sph3_morton_sort_noalloc(ctypes.c_void_p(pos.data_ptr()), n, max_level,
                                      ctypes.c_void_p(order.data_ptr()), ctypes.c_void_p(keys.data_ptr()),
                                      ctypes.c_void_p(stream))
    assert rc == 0, _lib.error_string(rc)
    torch.cuda.synchronize()
    return order.cpu().numpy(), keys.cpu().numpy().view(np.uint64)


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
        o1, k1 = _noalloc_sort(pos, lvl)
        o2, k2 = _allocating_sort(pos, lvl)
        assert np.array_equal(k1, k2)
        assert np.array_equal(o1, o2)


def test_noalloc_sort_rejects_sizes_above_its_maximum():
    import torch
    from sph_3_b200 import _lib
    lib = _lib.load()
    n = 65537
    pos = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    order = torch.zeros(n, dtype=torch.int64, device="cuda")
    rc = lib.sph3_morton_sort_noalloc(ctypes.c_void_p(pos.data_ptr()), n, 16, ctypes.c_void_p(order.data_ptr()),
                                      None, None)
    assert rc == _lib.C["SPH3_ERR_TOO_LARGE"]

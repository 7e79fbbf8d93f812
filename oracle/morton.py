"""NumPy restatement of the GPU's Morton keys and sort order -- test
infrastructure only.

The reference's GPU code has no Morton keys (it inserts bodies into a pointer
octree with locks, Particles_in_BH_Tree_III/Evrard_Collapse_2024/
bh_tree_iteration_v2.h:149-367), so the definition checked here is this
project's: per system, a power-of-two root cube [origin, origin + size) that
contains the particles, origin on the size/2 grid; coordinates quantised to
2^L cells with floor((x - origin) * 2^L / size), clamped; bits interleaved
x, y, z from the least significant end; the system index above the 3 L
Morton bits; a stable sort (ties keep the input order).
"""
from __future__ import annotations

import numpy as np


def root_cube(pos, periodic_box=None):
    if periodic_box is not None and max(periodic_box) > 0:
        L = max(periodic_box)
        _, e = np.frexp(L)
        size = float(np.ldexp(1.0, int(e)))
        if size * 0.5 >= L:
            size *= 0.5
        return np.zeros(3), size
    if pos.shape[0] == 0:
        lo = hi = np.zeros(3)
    else:
        lo = pos.min(axis=0)
        hi = pos.max(axis=0)
    ext = float(np.max(hi - lo))
    if not (ext > 0.0) or not np.isfinite(ext):
        ext = 1.0
    _, e = np.frexp(ext)
    size = float(np.ldexp(1.0, int(e)))
    for _ in range(64):
        half = 0.5 * size
        org = np.floor(lo / half) * half
        if np.all(org + size > hi):
            break
        size *= 2.0
    return org, size


def _spread3(v):
    v = v.astype(np.uint64) & np.uint64(0x1FFFFF)
    v = (v | (v << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
    v = (v | (v << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
    v = (v | (v << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
    v = (v | (v << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
    v = (v | (v << np.uint64(2))) & np.uint64(0x1249249249249249)
    return v


def keys(pos, max_level=16, cloud=0, periodic_box=None):
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    org, size = root_cube(pos, periodic_box)
    inv_cell = np.ldexp(1.0, max_level) / size
    maxq = (1 << max_level) - 1
    t = (pos - org) * inv_cell
    q = np.where(t > 0.0, np.floor(np.where(t > 0.0, t, 0.0)), 0.0)
    q = np.minimum(q, float(maxq)).astype(np.uint64)
    mort = _spread3(q[:, 0]) | (_spread3(q[:, 1]) << np.uint64(1)) | (_spread3(q[:, 2]) << np.uint64(2))
    return (np.uint64(cloud) << np.uint64(3 * max_level)) | mort


def order(pos, max_level=16, counts=None, periodic_box=None):
    """Sorted order (indices into pos) and the sorted keys, systems in order."""
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    if counts is None:
        counts = [pos.shape[0]]
    allk = []
    beg = 0
    for c, cnt in enumerate(counts):
        allk.append(keys(pos[beg:beg + cnt], max_level, c, periodic_box))
        beg += cnt
    k = np.concatenate(allk) if allk else np.zeros(0, dtype=np.uint64)
    o = np.argsort(k, kind="stable")
    return o, k[o]

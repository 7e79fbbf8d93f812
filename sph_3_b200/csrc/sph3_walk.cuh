// Warp-per-group tree walk shared by the SPH and gravity passes.
//
// A group is up to 32 consecutive Morton-sorted particles of one cloud (one
// target per lane).  The warp walks the octree once for the whole group with
// a LIFO stack in shared memory: each iteration pops up to 32 nodes (one per
// lane), tests them against the group's bounding box, queues accepted leaves
// with a ballot and pushes the children of opened nodes with a warp scan.
// Queued leaves are flushed in 32-particle tiles: lanes load one source
// particle each (coalesced), convert it to the group frame and store it in
// shared memory, then every lane runs its target against the whole tile.
//
// Stack bound.  Children are pushed 8 at most per popped node and the tree
// depth is at most max_level + 1, so a single-node pop at depth d can grow the
// stack by at most 7 (max_depth - d) before it shrinks.  Wide pops are only
// taken while top + 7 p <= cap - 7 max_depth; below that the walk pops one
// node at a time.  With cap >= 7 (max_depth + 1) + 1 the stack never
// overflows; the check that raises SPH3_STATUS_STACK_OVERFLOW stays anyway.
#pragma once

#include "sph3_internal.cuh"

namespace sph3 {

struct WarpMem {
    int *stack;
    int *leafq;
    int *lfirst;  // [32]
    int *lpre;    // [32]
    void *tile;
};

__host__ __device__ constexpr size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline size_t warp_mem_bytes(int stack_cap, size_t tile_bytes) {
    return align16(sizeof(int) * stack_cap) + align16(sizeof(int) * kLeafQ) +
           align16(sizeof(int) * 64) + align16(tile_bytes);
}

__device__ inline WarpMem carve_warp_mem(unsigned char *base, int stack_cap, size_t tile_bytes) {
    const int w = threadIdx.x >> 5;
    unsigned char *p = base + (size_t)w * warp_mem_bytes(stack_cap, tile_bytes);
    WarpMem m;
    m.stack = reinterpret_cast<int *>(p);
    p += align16(sizeof(int) * stack_cap);
    m.leafq = reinterpret_cast<int *>(p);
    p += align16(sizeof(int) * kLeafQ);
    m.lfirst = reinterpret_cast<int *>(p);
    m.lpre = m.lfirst + 32;
    p += align16(sizeof(int) * 64);
    m.tile = p;
    return m;
}

// next group index for this warp (one atomic per group)
__device__ __forceinline__ int next_group(int *work) {
    int g = 0;
    if (lane_id() == 0) g = atomicAdd(work, 1);
    return __shfl_sync(kFull, g, 0);
}

// Group geometry in the FP32 frame of the reference cell `ref`.
struct GroupBox {
    float3 c;   // centre
    float3 hw;  // half widths
    int ref;
    float s10;
};

__device__ __forceinline__ GroupBox group_box(float3 p, bool active, int ref, float s10) {
    // inactive lanes contribute the first target (lane 0 is always active)
    float3 p0 = make_float3(__shfl_sync(kFull, p.x, 0), __shfl_sync(kFull, p.y, 0),
                            __shfl_sync(kFull, p.z, 0));
    if (!active) p = p0;
    float lx = warp_min(p.x), ly = warp_min(p.y), lz = warp_min(p.z);
    float hx = warp_max(p.x), hy = warp_max(p.y), hz = warp_max(p.z);
    GroupBox g;
    g.c = make_float3(0.5f * (lx + hx), 0.5f * (ly + hy), 0.5f * (lz + hz));
    // half widths padded so that rounding of the centre cannot shrink the box
    const float pad = 1e-6f * s10 * 1024.f;
    g.hw = make_float3(0.5f * (hx - lx) + pad + 1e-6f * fabsf(g.c.x),
                       0.5f * (hy - ly) + pad + 1e-6f * fabsf(g.c.y),
                       0.5f * (hz - lz) + pad + 1e-6f * fabsf(g.c.z));
    g.ref = ref;
    g.s10 = s10;
    return g;
}

// squared distance between the group box and a node box (0 if they overlap)
__device__ __forceinline__ float box_gap2(const GroupBox &g, float3 nc, float3 nh) {
    float dx = fmaxf(fabsf(nc.x - g.c.x) - (nh.x + g.hw.x), 0.f);
    float dy = fmaxf(fabsf(nc.y - g.c.y) - (nh.y + g.hw.y), 0.f);
    float dz = fmaxf(fabsf(nc.z - g.c.z) - (nh.z + g.hw.z), 0.f);
    return dx * dx + dy * dy + dz * dz;
}

// squared distance from a point to the group box
__device__ __forceinline__ float point_gap2(const GroupBox &g, float3 p) {
    float dx = fmaxf(fabsf(p.x - g.c.x) - g.hw.x, 0.f);
    float dy = fmaxf(fabsf(p.y - g.c.y) - g.hw.y, 0.f);
    float dz = fmaxf(fabsf(p.z - g.c.z) - g.hw.z, 0.f);
    return dx * dx + dy * dy + dz * dz;
}

// Push the children of the opened nodes (nch each, first child cf) onto the
// stack; returns the new top.  Warp-uniform.
__device__ __forceinline__ int push_children(int *stack, int top, int cap, int nch, int cf,
                                             unsigned *status) {
    const int incl = warp_incl_scan(nch);
    const int tot = __shfl_sync(kFull, incl, 31);
    const int off = incl - nch;
    if (top + tot > cap) {  // cannot happen with a valid cap (see header)
        if (lane_id() == 0) set_status(status, SPH3_STATUS_STACK_OVERFLOW);
        // keep what fits, in lane order
        for (int k = 0; k < nch; ++k)
            if (top + off + k < cap) stack[top + off + k] = cf + k;
        __syncwarp();
        return cap;
    }
    for (int k = 0; k < nch; ++k) stack[top + off + k] = cf + k;
    __syncwarp();
    return top + tot;
}

// number of nodes to pop this iteration (warp-uniform)
__device__ __forceinline__ int pop_width(int top, int cap, int max_depth) {
    int room = (cap - 7 * (max_depth + 1) - top) / 7;
    int p = min(32, top);
    if (room < p) p = room < 1 ? 1 : room;
    return p;
}

// Runs `visit` over every particle of the queued leaves in tiles of 32:
// stage(lane_slot, j) fills the tile entry of sorted particle j, then
// interact(ne) runs every lane's target against the ne staged entries.
template <class Stage, class Interact>
__device__ __forceinline__ void flush_leaves(const int2 *range, const int *leafq, int nleaf,
                                             int *lfirst, int *lpre, Stage &stage,
                                             Interact &interact) {
    const int lane = lane_id();
    for (int base = 0; base < nleaf; base += 32) {
        int cnt = 0, fst = 0;
        if (base + lane < nleaf) {
            int2 r = range[leafq[base + lane]];
            fst = r.x;
            cnt = r.y;
        }
        const int incl = warp_incl_scan(cnt);
        const int tot = __shfl_sync(kFull, incl, 31);
        __syncwarp();
        lfirst[lane] = fst;
        lpre[lane] = incl - cnt;
        __syncwarp();
        const int nl = min(32, nleaf - base);
        for (int c0 = 0; c0 < tot; c0 += 32) {
            const int t = c0 + lane;
            if (t < tot) {
                int lo = 0, hi = nl - 1;
                while (lo < hi) {
                    int mid = (lo + hi + 1) >> 1;
                    if (lpre[mid] <= t) lo = mid;
                    else hi = mid - 1;
                }
                stage(lane, lfirst[lo] + (t - lpre[lo]));
            }
            __syncwarp();
            interact(min(32, tot - c0));
            __syncwarp();
        }
    }
}

// Periodic images needed by a group whose reach is R: shifts in {-L, 0, L}
// per periodic axis where the reach crosses the domain boundary.  Returns
// the number of images and fills sh[] (first entry is the identity).
__device__ __forceinline__ int group_images(const GroupBox &g, float R, const double *box,
                                            int periodic, float3 *sh) {
    if (!periodic) {
        sh[0] = make_float3(0.f, 0.f, 0.f);
        return 1;
    }
    float opt[3][3];
    int no[3];
    const float gc[3] = {g.c.x, g.c.y, g.c.z};
    const float gh[3] = {g.hw.x, g.hw.y, g.hw.z};
    const int rc[3] = {g.ref & 1023, (g.ref >> 10) & 1023, g.ref >> 20};
    for (int d = 0; d < 3; ++d) {
        no[d] = 1;
        opt[d][0] = 0.f;
        const float L = (float)box[d];
        if (L > 0.f) {
            // absolute coordinate of the box edges (periodic root cube starts at 0)
            const float corner = rc[d] * g.s10;
            const float lo = corner + gc[d] - gh[d], hi = corner + gc[d] + gh[d];
            if (lo - R < 0.f) opt[d][no[d]++] = -L;
            if (hi + R > L) opt[d][no[d]++] = L;
        }
    }
    int k = 0;
    for (int a = 0; a < no[0]; ++a)
        for (int b = 0; b < no[1]; ++b)
            for (int c = 0; c < no[2]; ++c) sh[k++] = make_float3(opt[0][a], opt[1][b], opt[2][c]);
    return k;
}

}  // namespace sph3

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
    void *tile;
};

__host__ __device__ constexpr size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline size_t warp_mem_bytes(int stack_cap, size_t tile_bytes) {
    return align16(sizeof(int) * stack_cap) + align16(sizeof(int) * kLeafQ) + align16(tile_bytes);
}

__device__ inline WarpMem carve_warp_mem(unsigned char *base, int stack_cap, size_t tile_bytes) {
    const int w = threadIdx.x >> 5;
    unsigned char *p = base + (size_t)w * warp_mem_bytes(stack_cap, tile_bytes);
    WarpMem m;
    m.stack = reinterpret_cast<int *>(p);
    p += align16(sizeof(int) * stack_cap);
    m.leafq = reinterpret_cast<int *>(p);
    p += align16(sizeof(int) * kLeafQ);
    m.tile = p;
    return m;
}

// next group index for this warp (one atomic per group); no work at all once
// non-finite input has been flagged, so garbage cannot turn into an
// all-pairs walk over a degenerate tree
__device__ __forceinline__ int next_group(int *work, const unsigned *status) {
    int g = 0;
    if (lane_id() == 0) {
        const unsigned s = *reinterpret_cast<const volatile unsigned *>(status);
        g = (s & SPH3_STATUS_NAN_INPUT) ? 0x7fffffff : atomicAdd(work, 1);
    }
    return __shfl_sync(kFull, g, 0);
}

// Group geometry in the FP32 frame of the reference cell `ref`.
struct GroupBox {
    float3 c;   // centre
    float3 hw;  // half widths
    int ref;
    float s10;
    int first = -1;  // first sorted particle of the group (walk statistics)
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

// 4-wide tile component: one 128-bit (FP32) or two 128-bit (FP64) shared
// loads per entry field group; every lane reads the same entry (broadcast).
template <typename R>
struct alignas(4 * sizeof(R)) V4 {
    R x, y, z, w;
};

// Source particle of slot c0 + lane of a flush batch whose leaves are held
// one per lane (first particle fst, exclusive prefix pre of the counts).
// Every queued leaf holds at least one particle (the walks never take an
// empty node), so the prefixes strictly increase: the leaf holding slot c0 is
// the last lane starting at or before it, and each leaf starting inside the
// chunk moves the later slots on by one leaf -- a ballot and an OR-reduction
// instead of a dependent binary search through shared memory per slot.
__device__ __forceinline__ int leaf_source(int c0, int pre, int fst, bool is_leaf) {
    const int lane = lane_id();
    const unsigned at_or_before = __ballot_sync(kFull, is_leaf && pre <= c0);
    const int l0 = 31 - __clz((int)at_or_before);
    const unsigned starts =
        __reduce_or_sync(kFull, (is_leaf && pre > c0 && pre - c0 < 32) ? 1u << (pre - c0) : 0u);
    const int leaf = l0 + __popc(starts & (0xffffffffu >> (31 - lane)));
    return __shfl_sync(kFull, fst, leaf) + (c0 + lane - __shfl_sync(kFull, pre, leaf));
}

// Streams every particle of the queued leaves through a double-buffered
// 32-entry tile (tile[0..63]): the loads of the next 32 candidates are in
// flight while the lanes run the current ones.  load(j) returns the tile
// entry of sorted particle j (global loads + conversion to the group frame);
// interact(tile, ne) runs every lane's target against ne staged entries.
template <class E, class Load, class Interact>
__device__ __forceinline__ void flush_leaves(const int2 *range, const int *leafq, int nleaf, E *tile, Load &load,
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
        const int pre = incl - cnt;
        const bool is_leaf = base + lane < nleaf;
        auto fetch = [&](int c0, E &out) -> bool {
            const int t = c0 + lane;
            const int j = leaf_source(c0, pre, fst, is_leaf);
            if (t >= tot) return false;
            out = load(j);
            return true;
        };
        E cur;
        bool have = fetch(0, cur);
        int buf = 0;
        for (int c0 = 0; c0 < tot; c0 += 32) {
            if (have) tile[buf * 32 + lane] = cur;
            __syncwarp();
            have = c0 + 32 < tot ? fetch(c0 + 32, cur) : false;
            interact(tile + buf * 32, min(32, tot - c0));
            buf ^= 1;
        }
        __syncwarp();
    }
}

// As flush_leaves, with the tile layout left to the caller:
// store(buf, slot, entry, have) writes slot `slot` (0..31) of buffer `buf`
// (0 or 1) and is called for every slot, with have = false (write padding)
// where no candidate is left; interact(buf, ne) runs the targets against the
// first ne entries of buffer buf.  Padded slots let the interaction run
// whole pairs of entries without bounds checks.
template <class E, class Load, class Store, class Interact>
__device__ __forceinline__ void flush_leaves_st(const int2 *range, const int *leafq, int nleaf, Load &load,
                                                Store &store, Interact &interact) {
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
        const int pre = incl - cnt;
        const bool is_leaf = base + lane < nleaf;
        auto fetch = [&](int c0, E &out) -> bool {
            const int t = c0 + lane;
            const int j = leaf_source(c0, pre, fst, is_leaf);
            if (t >= tot) return false;
            out = load(j);
            return true;
        };
        E cur{};
        bool have = fetch(0, cur);
        int buf = 0;
        for (int c0 = 0; c0 < tot; c0 += 32) {
            store(buf, lane, cur, have);
            __syncwarp();
            have = c0 + 32 < tot ? fetch(c0 + 32, cur) : false;
            interact(buf, min(32, tot - c0));
            buf ^= 1;
        }
        __syncwarp();
    }
}

// As flush_leaves, but load(j, keep) also says whether candidate j can reach
// the group at all (tested once per candidate by the lane that loads it);
// kept candidates are compacted so that every interact() call but the last
// sees a full tile of 32.  The tile holds 64 entries: up to 31 left over
// plus one freshly loaded chunk.
template <class E, class Load, class Interact>
__device__ __forceinline__ void flush_leaves_compact(const int2 *range, const int *leafq, int nleaf, E *tile,
                                                     Load &load, Interact &interact) {
    const int lane = lane_id();
    int fill = 0;
    for (int base = 0; base < nleaf; base += 32) {
        int cnt = 0, fst = 0;
        if (base + lane < nleaf) {
            int2 r = range[leafq[base + lane]];
            fst = r.x;
            cnt = r.y;
        }
        const int incl = warp_incl_scan(cnt);
        const int tot = __shfl_sync(kFull, incl, 31);
        const int pre = incl - cnt;
        const bool is_leaf = base + lane < nleaf;
        auto fetch = [&](int c0, E &out) -> bool {
            const int t = c0 + lane;
            const int j = leaf_source(c0, pre, fst, is_leaf);
            if (t >= tot) return false;
            bool keep = true;
            out = load(j, keep);
            return keep;
        };
        E cur;
        bool have = fetch(0, cur);
        for (int c0 = 0; c0 < tot; c0 += 32) {
            const unsigned kb = __ballot_sync(kFull, have);
            if (have) tile[fill + __popc(kb & lanemask_lt())] = cur;
            fill += __popc(kb);
            __syncwarp();
            have = c0 + 32 < tot ? fetch(c0 + 32, cur) : false;
            if (fill >= 32) {
                interact(tile, 32);
                __syncwarp();
                E rest;
                const bool mv = lane < fill - 32;
                if (mv) rest = tile[32 + lane];
                __syncwarp();
                if (mv) tile[lane] = rest;
                fill -= 32;
                __syncwarp();
            }
        }
        __syncwarp();
    }
    if (fill > 0) interact(tile, fill);
    __syncwarp();
}

// A staged candidate as NF 32-bit fields (coordinates, h, mass, an index
// carried as float bits, ...).
template <int NF>
struct SoaV {
    float v[NF];
};

// As flush_leaves_compact, with the staged candidates kept as NF arrays of 64
// floats (field f of slot e at tile[64 f + e]) instead of 4-wide entries:
// load(j, keep) returns the fields of candidate j.  interact(ne) sees entries
// [0, ne); an odd last batch gets one pad entry (slot ne) with every field
// set to pad[f], so the entries can be run in pairs, two consecutive entries
// loading as one float2 per field: a ready packed FP32 operand.
template <int NF, class Load, class Interact>
__device__ __forceinline__ void flush_leaves_compact_soa(const int2 *range, const int *leafq, int nleaf, float *tile,
                                                         const SoaV<NF> &pad, Load &load, Interact &interact) {
    const int lane = lane_id();
    int fill = 0;
    for (int base = 0; base < nleaf; base += 32) {
        int cnt = 0, fst = 0;
        if (base + lane < nleaf) {
            int2 r = range[leafq[base + lane]];
            fst = r.x;
            cnt = r.y;
        }
        const int incl = warp_incl_scan(cnt);
        const int tot = __shfl_sync(kFull, incl, 31);
        const int pre = incl - cnt;
        const bool is_leaf = base + lane < nleaf;
        auto fetch = [&](int c0, SoaV<NF> &out) -> bool {
            const int t = c0 + lane;
            const int j = leaf_source(c0, pre, fst, is_leaf);
            if (t >= tot) return false;
            bool keep = true;
            out = load(j, keep);
            return keep;
        };
        SoaV<NF> cur;
        bool have = fetch(0, cur);
        for (int c0 = 0; c0 < tot; c0 += 32) {
            const unsigned kb = __ballot_sync(kFull, have);
            if (have) {
                const int at = fill + __popc(kb & lanemask_lt());
#pragma unroll
                for (int f = 0; f < NF; ++f) tile[64 * f + at] = cur.v[f];
            }
            fill += __popc(kb);
            __syncwarp();
            have = c0 + 32 < tot ? fetch(c0 + 32, cur) : false;
            if (fill >= 32) {
                interact(32);
                __syncwarp();
                const bool mv = lane < fill - 32;
                SoaV<NF> rest;
                if (mv) {
#pragma unroll
                    for (int f = 0; f < NF; ++f) rest.v[f] = tile[64 * f + 32 + lane];
                }
                __syncwarp();
                if (mv) {
#pragma unroll
                    for (int f = 0; f < NF; ++f) tile[64 * f + lane] = rest.v[f];
                }
                fill -= 32;
                __syncwarp();
            }
        }
        __syncwarp();
    }
    if (fill > 0) {
        if ((fill & 1) && lane == 0) {
#pragma unroll
            for (int f = 0; f < NF; ++f) tile[64 * f + fill] = pad.v[f];
        }
        __syncwarp();
        interact(fill);
    }
    __syncwarp();
}

// Periodic images needed by a group whose reach is R.  Per axis a 3-bit
// mask: bit 0 the identity, bit 1 the shift -L (reach crosses 0), bit 2 the
// shift +L (reach crosses L).  Image codes 0..26 combine one option per axis
// (code = ox + 3 oy + 9 oz); code 0 is the identity.  No arrays, so nothing
// lands in local memory.
struct Images {
    int mask;  // 3 bits per axis
};

__device__ __forceinline__ Images group_images(const GroupBox &g, float R, const double *box, int periodic) {
    Images im;
    im.mask = 1 | (1 << 3) | (1 << 6);
    if (!periodic) return im;
    const float gc[3] = {g.c.x, g.c.y, g.c.z};
    const float gh[3] = {g.hw.x, g.hw.y, g.hw.z};
    const int rc[3] = {g.ref & 1023, (g.ref >> 10) & 1023, g.ref >> 20};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float L = (float)box[d];
        if (L > 0.f) {
            // absolute coordinate of the box edges (periodic root cube starts at 0)
            const float corner = rc[d] * g.s10;
            const float lo = corner + gc[d] - gh[d], hi = corner + gc[d] + gh[d];
            if (lo - R < 0.f) im.mask |= 2 << (3 * d);
            if (hi + R > L) im.mask |= 4 << (3 * d);
        }
    }
    return im;
}

// shift of image `code` if the group needs it
__device__ __forceinline__ bool image_shift(const Images &im, int code, const double *box, float3 &s) {
    const int o[3] = {code % 3, (code / 3) % 3, code / 9};
    float v[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (!((im.mask >> (3 * d + o[d])) & 1)) return false;
        v[d] = o[d] == 0 ? 0.f : (o[d] == 1 ? -(float)box[d] : (float)box[d]);
    }
    s = make_float3(v[0], v[1], v[2]);
    return true;
}

}  // namespace sph3

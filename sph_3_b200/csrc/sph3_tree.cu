// Linear octree from Morton-sorted keys, built top-down one depth at a time,
// then moments bottom-up.
//
// A node is a contiguous run [first, first + count) of sorted particles whose
// keys share a common prefix; its level is the deepest level whose cell holds
// the whole run.  A node with more than leaf_size particles (and level below
// max_level) is split on the next 3-bit digit into its 2..8 non-empty
// sub-runs (digits are non-decreasing inside a run, so each digit's start is
// one boundary: a warp per node finds the 8 starts once and keeps them).
// Single-child chains never appear, so nodes < 2 * particles.  Children of a
// node are stored contiguously and each depth is compacted with an exclusive
// scan, so the layout, and every sum over it, is deterministic.  One launch
// per depth does the octant search, the scan (decoupled look-back between
// tiles taken in order) and the child writes.
// Compared with the reference's pointer octree (bh_tree_iteration_v2.h:149-450:
// one block, atomicCAS locks, a DFS sort that spins on its parent) there are
// no locks; the one wait, a tile reading its predecessors' published counts,
// waits only on running blocks and is bounded.
#include <algorithm>
#include <cfloat>

#include "sph3_internal.cuh"

namespace sph3 {

__device__ __forceinline__ int common_level(uint64_t a, uint64_t b, int max_level) {
    uint64_t x = a ^ b;
    if (x == 0) return max_level;
    int hb = 63 - __clzll((long long)x);
    return max_level - 1 - hb / 3;
}

__global__ void k_tree_roots(Tree T, Cloud *clouds, int ncloud, const uint64_t *key, int max_level) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) {
        T.depth_begin[0] = 0;
        T.depth_begin[1] = ncloud;
        T.lvl[kLvlEpoch] += 1;  // a new tag for this build's look-back words
    }
    if (c < kLvlEpoch) T.lvl[c] = 0;  // the per-depth tile counters
    if (c >= ncloud) return;
    Cloud &cl = clouds[c];
    int first = (int)cl.begin, count = (int)(cl.end - cl.begin);
    int lvl = count > 0 ? common_level(key[first], key[first + count - 1], max_level) : max_level;
    T.range[c] = make_int2(first, count);
    T.child[c] = make_int2(-1, lvl << 8);
    T.parent[c] = -1;
    cl.root = c;
}

// Children of each node of depth d: one warp per node finds where each
// 3-bit digit of the next level starts inside the node's sorted key run (8
// starts, -1 for an empty octant) and the number of non-empty octants (0 for
// a leaf).  Digits are non-decreasing inside a run, so the start of digit g
// is the first index whose digit is >= g.  Runs of up to 128 keys are read whole (4 coalesced loads per lane)
// and each start is the run start plus a ballot count; longer runs are
// searched 5-ary, 4 lanes per digit probing 4 points per round (about
// log5(count) dependent rounds instead of log2).
constexpr int kTreeScanMax = 128;  // runs up to this size are read whole

// The octant starts of node i (warp-collective): lane g < 8 gets the first
// index of the node's run whose next 3-bit digit is g (-1 for an empty
// octant); returns the number of non-empty octants, 0 for a node that stays
// a leaf (at most leaf_size particles, or at the deepest level).
__device__ __forceinline__ int node_octants(const Tree &T, const uint64_t *key, int i, int leaf_size, int max_level,
                                            int &start) {
    const int lane = threadIdx.x & 31;
    const int2 r = T.range[i];
    const int lvl = T.child[i].y >> 8;
    start = -1;
    if (!(r.y > leaf_size && lvl < max_level)) return 0;
    const int shift = 3 * (max_level - lvl - 1);
    const int s = r.x, e = r.x + r.y;
    int first;  // lanes 0..7: first index of the run with digit >= lane
    if (r.y <= kTreeScanMax) {
        int dg[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = s + 32 * q + lane;
            dg[q] = k < e ? (int)((key[k] >> shift) & 7u) : 8;
        }
        first = s;
#pragma unroll
        for (int g = 1; g < 8; ++g) {
            int below = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) below += __popc(__ballot_sync(kFull, dg[q] < g));
            if (lane == g) first = s + below;
        }
    } else {
        const int g = lane >> 2, sub = lane & 3;
        int a = s, b = e;  // the answer for digit g lies in [a, b]
        while (__any_sync(kFull, a < b)) {
            const int p = a + (int)((long long)(b - a) * (sub + 1) / 5);  // a <= p < b when a < b
            const bool pred = a < b && (int)((key[p] >> shift) & 7u) < g;
            const int t = __popc((__ballot_sync(kFull, pred) >> (4 * g)) & 0xFu);
            const int pl = __shfl_sync(kFull, p, 4 * g + (t > 0 ? t - 1 : 0));
            const int pr = __shfl_sync(kFull, p, 4 * g + (t < 4 ? t : 3));
            if (a < b) {
                if (t > 0) a = pl + 1;
                if (t < 4) b = pr;
            }
        }
        first = __shfl_sync(kFull, a, 4 * (lane & 7));
    }
    const int nxt = __shfl_down_sync(kFull, first, 1);
    const int stop = lane == 7 ? e : nxt;
    start = lane < 8 && first < stop ? first : -1;
    return __popc(__ballot_sync(kFull, start >= 0));
}

// Children of node i from its octant starts st[8] (-1: empty), written at
// cf, cf + 1, ... (a thread per node; nch = 0 marks a leaf).
__device__ __forceinline__ void emit_children(const Tree &T, const uint64_t *key, int i, int nch, const int *st,
                                              int cf, int max_level) {
    const int lvl = T.child[i].y >> 8;
    if (nch == 0) {
        T.child[i] = make_int2(-1, lvl << 8);
        return;
    }
    const int2 r = T.range[i];
    const int e = r.x + r.y;
    // all 16 key loads before any store, so they are in flight together
    int stops[8];
    uint64_t kf[8], kl[8];
#pragma unroll
    for (int dg = 0; dg < 8; ++dg) {
        int stop = e;
#pragma unroll
        for (int q = 7; q > dg; --q)
            if (st[q] >= 0) stop = st[q];
        stops[dg] = stop;
        kf[dg] = st[dg] >= 0 ? __ldg(key + st[dg]) : 0;
        kl[dg] = st[dg] >= 0 ? __ldg(key + stop - 1) : 0;
    }
    T.child[i] = make_int2(cf, nch | (lvl << 8));
    int c = 0;
#pragma unroll
    for (int dg = 0; dg < 8; ++dg) {
        if (st[dg] < 0) continue;
        const int stop = stops[dg];
        const int cl = common_level(kf[dg], kl[dg], max_level);
        T.range[cf + c] = make_int2(st[dg], stop - st[dg]);
        T.child[cf + c] = make_int2(-1, cl << 8);
        T.parent[cf + c] = i;
        ++c;
    }
}

// Decoupled look-back over the tiles of one depth (single thread): publishes
// the tile's child count, adds up the predecessors' counts until one that
// already knows its inclusive prefix, publishes the tile's own inclusive
// prefix and returns the exclusive one.  Words are tagged with (build, depth),
// so words of earlier passes read as "not yet published".  Tiles are taken in
// order from an atomic counter by running blocks, so every predecessor is
// running or done and each wait ends; the waits are bounded all the same and
// raise SPH3_STATUS_TREE_CAPACITY if one ever ran out.
constexpr unsigned kLbAgg = 1u, kLbIncl = 2u;
constexpr int kLbMaxSpin = 1 << 22;

__device__ __forceinline__ unsigned long long lb_word(unsigned tag, unsigned flag, int v) {
    return ((unsigned long long)tag << 32) | ((unsigned long long)flag << 30) | (unsigned long long)(unsigned)v;
}

__device__ int tile_lookback(unsigned long long *state, int tile, int tot, unsigned tag, unsigned *status) {
    if (tile == 0) {
        atomicExch(state, lb_word(tag, kLbIncl, tot));
        return 0;
    }
    atomicExch(state + tile, lb_word(tag, kLbAgg, tot));
    int excl = 0, j = tile - 1, spins = 0;
    while (j >= 0) {
        const unsigned long long w = atomicAdd(state + j, 0ull);
        const unsigned flag = (unsigned)(w >> 30) & 3u;
        if ((unsigned)(w >> 32) != tag || flag == 0u) {
            if (++spins > kLbMaxSpin) {
                atomicOr(status, SPH3_STATUS_TREE_CAPACITY);
                break;
            }
            __nanosleep(32);
            continue;
        }
        excl += (int)(w & 0x3fffffffull);
        if (flag == kLbIncl) break;
        --j;
    }
    atomicExch(state + tile, lb_word(tag, kLbIncl, excl + tot));
    return excl;
}

// One depth of the top-down build in one launch: blocks take tiles of
// consecutive nodes of depth d in order; a warp per node finds its
// octant starts (node_octants), the tile's child counts are scanned in the
// block and offset by the look-back prefix over earlier tiles, and a thread
// per node writes the children.  The children of the depth come out compacted
// in node order -- the layout of a global exclusive scan -- so the tree is
// deterministic.  The last tile sets depth_begin[d + 2].  Tiles hold up to
// kTreeTile nodes, fewer (down to one per warp) at the shallow depths, whose
// few nodes have long key runs to search: there the depth's nodes spread
// over all blocks instead of queueing eight deep behind one block's warps.
constexpr int kTreeTile = 64;
constexpr int kTreeTileMin = 8;

__global__ void __launch_bounds__(256) k_tree_level(Tree T, const uint64_t *key, int d, int leaf_size, int max_level,
                                                    unsigned *status) {
    __shared__ int s_tile, s_base;
    __shared__ int s_nch[kTreeTile], s_off[kTreeTile];
    __shared__ int s_st[kTreeTile * 8];
    const int beg = T.depth_begin[d], end = T.depth_begin[d + 1];
    const int m = end - beg;
    if (m <= 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) T.depth_begin[d + 2] = end;
        return;
    }
    const int per_block = (m + gridDim.x - 1) / gridDim.x;
    // nodes per tile: 64, or down to 8 when the depth is too small to give
    // every block a tile of 16
    const int ts = per_block <= 16 ? max(kTreeTileMin, (per_block + 7) & ~7) : kTreeTile;
    const int ntiles = (m + ts - 1) / ts;
    const unsigned tag = (unsigned)T.lvl[kLvlEpoch] * 32u + (unsigned)d;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(T.lvl + d, 1);
        __syncthreads();
        const int tile = s_tile;
        if (tile >= ntiles) break;
        const int t0 = tile * ts;
        const int tn = min(ts, m - t0);
        for (int q = w; q < tn; q += 8) {
            int start;
            const int nch = node_octants(T, key, beg + t0 + q, leaf_size, max_level, start);
            if (lane < 8) s_st[q * 8 + lane] = start;
            if (lane == 0) s_nch[q] = nch;
        }
        __syncthreads();
        if (w == 0) {
            const int a = 2 * lane < tn ? s_nch[2 * lane] : 0;
            const int b = 2 * lane + 1 < tn ? s_nch[2 * lane + 1] : 0;
            const int incl = warp_incl_scan(a + b);
            if (2 * lane < tn) s_off[2 * lane] = incl - a - b;
            if (2 * lane + 1 < tn) s_off[2 * lane + 1] = incl - b;
            const int tot = __shfl_sync(kFull, incl, 31);
            if (lane == 0) {
                int base = tile_lookback(T.lb, tile, tot, tag, status);
                if (end + base + tot > T.cap) {  // cannot happen: nodes < 2n + clouds + 64
                    atomicOr(status, SPH3_STATUS_TREE_CAPACITY);
                    base = -1;
                }
                s_base = base;
                if (tile == ntiles - 1) T.depth_begin[d + 2] = base >= 0 ? end + base + tot : end;
            }
        }
        __syncthreads();
        if (threadIdx.x < tn) {
            const int q = threadIdx.x;
            const int nch = s_base >= 0 ? s_nch[q] : 0;
            emit_children(T, key, beg + t0 + q, nch, s_st + 8 * q, end + s_base + s_off[q], max_level);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ moments
struct MomArgs {
    const double *pos, *m, *h, *eps;
    int64_t n;
    const Cloud *clouds;
    const uint64_t *key;
    int max_level;
    double inv_theta;  // 1/theta (inf for theta = 0)
    int mac_offset;    // add the com offset to the opening radius
};

// Four threads per node: a leaf's particles and an internal node's children
// are shared out round-robin and the partial sums (FP64), minima and maxima
// are combined with two shuffles, so a warp reads eight nodes' particle runs
// four consecutive entries at a time.  The combination order is fixed, so the
// moments are deterministic.
__global__ void k_tree_moments(Tree T, MomArgs a, int d, int quad) {
    const int beg = T.depth_begin[d], end = T.depth_begin[d + 1];
    const int cap = T.cap;
    const int64_t n = a.n;
    const int qt = threadIdx.x & 3;
    const unsigned qmask = 0xFu << (threadIdx.x & 28);
    auto qsum = [&](double v) {
        v += __shfl_xor_sync(qmask, v, 1);
        return v + __shfl_xor_sync(qmask, v, 2);
    };
    auto qmin = [&](double v) {
        v = fmin(v, __shfl_xor_sync(qmask, v, 1));
        return fmin(v, __shfl_xor_sync(qmask, v, 2));
    };
    auto qmax = [&](double v) {
        v = fmax(v, __shfl_xor_sync(qmask, v, 1));
        return fmax(v, __shfl_xor_sync(qmask, v, 2));
    };
    for (int i = beg + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 2); i < end;
         i += (int)((gridDim.x * blockDim.x) >> 2)) {
        const int2 r = T.range[i];
        const int2 ch = T.child[i];
        const int nch = ch.y & 255;
        double M = 0, sx = 0, sy = 0, sz = 0;
        double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
        double hm = 0, em = 0;
        if (nch == 0) {
#pragma unroll 4
            for (int k = r.x + qt; k < r.x + r.y; k += 4) {
                const double mk = a.m[k];
                const double x = a.pos[k], y = a.pos[n + k], z = a.pos[2 * n + k];
                M += mk;
                sx += mk * x;
                sy += mk * y;
                sz += mk * z;
                lo[0] = fmin(lo[0], x); hi[0] = fmax(hi[0], x);
                lo[1] = fmin(lo[1], y); hi[1] = fmax(hi[1], y);
                lo[2] = fmin(lo[2], z); hi[2] = fmax(hi[2], z);
                hm = fmax(hm, a.h[k]);
                em = fmax(em, a.eps[k]);
            }
        } else {
            // fixed trip count with a guard: the loads of all children are
            // issued together (a node has at most 8), same summation order
#pragma unroll
            for (int q8 = qt; q8 < 8; q8 += 4) {
                if (q8 >= nch) continue;
                const int c = ch.x + q8;
                const double mc = T.mass[c];
                M += mc;
                sx += mc * T.com[c];
                sy += mc * T.com[cap + c];
                sz += mc * T.com[2 * cap + c];
                for (int q = 0; q < 3; ++q) {
                    lo[q] = fmin(lo[q], T.bmin[q * cap + c]);
                    hi[q] = fmax(hi[q], T.bmax[q * cap + c]);
                }
                hm = fmax(hm, T.hmax[c]);
                em = fmax(em, T.epsmax[c]);
            }
        }
        M = qsum(M);
        sx = qsum(sx);
        sy = qsum(sy);
        sz = qsum(sz);
        for (int q = 0; q < 3; ++q) {
            lo[q] = qmin(lo[q]);
            hi[q] = qmax(hi[q]);
        }
        hm = qmax(hm);
        em = qmax(em);
        if (r.y == 0) {
            lo[0] = lo[1] = lo[2] = 0.0;
            hi[0] = hi[1] = hi[2] = 0.0;
        }
        double cx, cy, cz;
        if (M > 0) {
            cx = sx / M; cy = sy / M; cz = sz / M;
        } else {
            cx = 0.5 * (lo[0] + hi[0]); cy = 0.5 * (lo[1] + hi[1]); cz = 0.5 * (lo[2] + hi[2]);
        }
        if (qt == 0) {
            T.mass[i] = M;
            T.com[i] = cx; T.com[cap + i] = cy; T.com[2 * cap + i] = cz;
            for (int q = 0; q < 3; ++q) {
                T.bmin[q * cap + i] = lo[q];
                T.bmax[q * cap + i] = hi[q];
            }
            T.hmax[i] = hm;
            T.epsmax[i] = em;
        }
        double Q[6] = {0, 0, 0, 0, 0, 0};
        if (quad) {
            if (nch == 0) {
#pragma unroll 4
                for (int k = r.x + qt; k < r.x + r.y; k += 4) {
                    const double mk = a.m[k];
                    const double dx = a.pos[k] - cx, dy = a.pos[n + k] - cy, dz = a.pos[2 * n + k] - cz;
                    const double d2 = dx * dx + dy * dy + dz * dz;
                    Q[0] += mk * (3 * dx * dx - d2);
                    Q[1] += mk * (3 * dx * dy);
                    Q[2] += mk * (3 * dx * dz);
                    Q[3] += mk * (3 * dy * dy - d2);
                    Q[4] += mk * (3 * dy * dz);
                    Q[5] += mk * (3 * dz * dz - d2);
                }
            } else {
#pragma unroll
                for (int q8 = qt; q8 < 8; q8 += 4) {
                    if (q8 >= nch) continue;
                    const int c = ch.x + q8;
                    const double mc = T.mass[c];
                    const double dx = T.com[c] - cx, dy = T.com[cap + c] - cy, dz = T.com[2 * cap + c] - cz;
                    const double d2 = dx * dx + dy * dy + dz * dz;
                    Q[0] += T.quad[c] + mc * (3 * dx * dx - d2);
                    Q[1] += T.quad[cap + c] + mc * (3 * dx * dy);
                    Q[2] += T.quad[2 * cap + c] + mc * (3 * dx * dz);
                    Q[3] += T.quad[3 * cap + c] + mc * (3 * dy * dy - d2);
                    Q[4] += T.quad[4 * cap + c] + mc * (3 * dy * dz);
                    Q[5] += T.quad[5 * cap + c] + mc * (3 * dz * dz - d2);
                }
            }
        }
        for (int q = 0; q < 6; ++q) Q[q] = qsum(Q[q]);
        if (qt != 0) continue;  // one thread of the four writes the node
        for (int q = 0; q < 6; ++q) T.quad[q * cap + i] = Q[q];

        // FP32 packs for the walks
        const Cloud &cl = a.clouds[r.y > 0 ? (int)(a.key[r.x] >> (3 * a.max_level)) : 0];
        const double bcx = 0.5 * (lo[0] + hi[0]), bcy = 0.5 * (lo[1] + hi[1]), bcz = 0.5 * (lo[2] + hi[2]);
        const double hx = 0.5 * (hi[0] - lo[0]), hy = 0.5 * (hi[1] - lo[1]), hz = 0.5 * (hi[2] - lo[2]);
        const double pad = 1e-6 * cl.size;
        CellRel b = make_cellrel(bcx, bcy, bcz, cl);
        T.box_c[i] = make_float4(b.ox, b.oy, b.oz, __int_as_float(b.cell));
        T.box_h[i] = make_float4((float)(hx + pad), (float)(hy + pad), (float)(hz + pad),
                                 (float)(hm * (1.0 + 1e-6)));
        CellRel cm = make_cellrel(cx, cy, cz, cl);
        T.com_c[i] = make_float4(cm.ox, cm.oy, cm.oz, __int_as_float(cm.cell));
        const double ex = fmax(fabs(hi[0] - cx), fabs(cx - lo[0]));
        const double ey = fmax(fabs(hi[1] - cy), fabs(cy - lo[1]));
        const double ez = fmax(fabs(hi[2] - cz), fabs(cz - lo[2]));
        const double bmax = sqrt(ex * ex + ey * ey + ez * ez);
        const double side = 2.0 * fmax(hx, fmax(hy, hz));
        const double delta = sqrt((cx - bcx) * (cx - bcx) + (cy - bcy) * (cy - bcy) + (cz - bcz) * (cz - bcz));
        // s/d < theta (d > s/theta), optionally plus the offset of the centre of
        // mass from the box centre (d > s/theta + delta); theta = 0 never
        // accepts a node (exact sum).  The walks also require d > r_soft
        // (bmax + eps), so an accepted node's particles always lie outside the
        // group's box, whatever theta.
        double r_open = isinf(a.inv_theta) ? (double)FLT_MAX : side * a.inv_theta + (a.mac_offset ? delta : 0.0);
        r_open = fmin(r_open * (1.0 + 1e-5) + pad, (double)FLT_MAX);
        const double r_soft = fmin((bmax + em) * (1.0 + 1e-5) + pad, (double)FLT_MAX);
        T.mono[i] = make_float4((float)M, (float)r_open, (float)r_soft, 0.f);
        T.quad4[i] = make_float4((float)Q[0], (float)Q[1], (float)Q[2], (float)Q[3]);
        T.quad1[i] = (float)Q[4];
        // walk records: everything one node test needs in one contiguous
        // record, so a walk step is a single round trip to L2
        const int chy = r.y > 0 ? ch.y : -1;  // -1: empty node, never taken
        T.gw[2 * i] = T.com_c[i];
        T.gw[2 * i + 1] = make_float4((float)r_open, (float)r_soft, __int_as_float(ch.x), __int_as_float(chy));
        T.sw[3 * i] = T.box_c[i];
        T.sw[3 * i + 1] = T.box_h[i];
        T.sw[3 * i + 2] = make_float4(__int_as_float(ch.x), __int_as_float(chy), __int_as_float(r.y), 0.f);
    }
}

__global__ void k_tree_totals(Tree T, int max_depth, unsigned long long *counters) {
    // counters[6] = nodes, counters[7] = leaves
    const int nn = T.depth_begin[max_depth];
    unsigned long long leaves = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
        leaves += (T.child[i].y & 255) == 0;
    leaves = warp_sum(leaves);
    if ((threadIdx.x & 31) == 0 && leaves) atomicAdd(&counters[7], leaves);
    if (blockIdx.x == 0 && threadIdx.x == 0) counters[6] = (unsigned long long)nn;
}

// Last-arrival climb: after finishing node c, a thread counts itself in at
// c's parent; the thread that completes the parent's count (its children's
// results are all written and fenced) goes on with the parent.  No thread
// ever waits, and each internal node is done exactly once.  The counter is
// put back to zero for the next pass.
__device__ __forceinline__ int climb(const Tree &T, int c) {
    const int p = T.parent[c];
    if (p < 0) return -1;
    __threadfence();
    const int nch = T.child[p].y & 255;
    if (atomicAdd(T.arrive + p, 1) != nch - 1) return -1;
    __threadfence();
    T.arrive[p] = 0;
    return p;
}

// Node hmax from the current h (after an h search): a leaf from its
// particles, an internal node from its children (read through L2: they were
// written by other threads of the same launch).  With eps = h (eps_from_h)
// the softening maximum and the softening reach r_soft = bmax + eps_max
// follow as well.
__device__ void node_refit_h(const Tree &T, const double *h, int i, int refit_eps, const uint64_t *key,
                             const Cloud *clouds, int max_level) {
    const int cap = T.cap;
    const int2 r = T.range[i];
    const int2 ch = T.child[i];
    const int nch = ch.y & 255;
    double hm = 0;
    if (nch == 0) {
        for (int k = r.x; k < r.x + r.y; ++k) hm = fmax(hm, h[k]);
    } else {
        for (int c = ch.x; c < ch.x + nch; ++c) hm = fmax(hm, __ldcg(T.hmax + c));
    }
    T.hmax[i] = hm;
    T.box_h[i].w = (float)(hm * (1.0 + 1e-6));
    T.sw[3 * i + 1].w = (float)(hm * (1.0 + 1e-6));
    if (refit_eps && r.y > 0) {
        T.epsmax[i] = hm;
        const Cloud &cl = clouds[(int)(key[r.x] >> (3 * max_level))];
        const double cx = T.com[i], cy = T.com[cap + i], cz = T.com[2 * cap + i];
        const double ex = fmax(fabs(T.bmax[i] - cx), fabs(cx - T.bmin[i]));
        const double ey = fmax(fabs(T.bmax[cap + i] - cy), fabs(cy - T.bmin[cap + i]));
        const double ez = fmax(fabs(T.bmax[2 * cap + i] - cz), fabs(cz - T.bmin[2 * cap + i]));
        const double bmax = sqrt(ex * ex + ey * ey + ez * ez);
        const float r_soft = (float)fmin((bmax + hm) * (1.0 + 1e-5) + 1e-6 * cl.size, (double)FLT_MAX);
        T.mono[i].z = r_soft;
        T.gw[2 * i + 1].y = r_soft;
    }
}

// one launch: a thread per leaf, then up the last-arrival chain (hmax is a
// maximum, so the order in which children finish does not matter)
__global__ void k_tree_refit_h(Tree T, const double *h, int max_depth, int refit_eps, const uint64_t *key,
                               const Cloud *clouds, int max_level) {
    const int nn = T.depth_begin[max_depth];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        if ((T.child[i].y & 255) != 0) continue;
        node_refit_h(T, h, i, refit_eps, key, clouds, max_level);
        int c = i;
        for (int up = 0; up < max_depth; ++up) {
            c = climb(T, c);
            if (c < 0) break;
            node_refit_h(T, h, c, refit_eps, key, clouds, max_level);
        }
    }
}

void launch_tree_refit_h(State &S, const Params &P, cudaStream_t st) {
    if (S.ncloud == 0) return;
    k_tree_refit_h<<<S.num_sms * 8, 128, 0, st>>>(S.tree, S.h, S.max_level + 2, P.eps_from_h, S.key, S.clouds,
                                                   S.max_level);
}

// ------------------------------------------------------------ h start guess
// A starting h for the Newton search when none is given: every particle of a
// leaf gets the h at which a sphere of radius 2h would hold n_ngb particles
// at the leaf's number density (its count over its octree cell's volume).
// The search then converges in a few passes; the exact bootstrap of the
// reference (k-th nearest neighbour, k_boot_h) stays for the reference rule.
__global__ void k_h_guess(Tree T, const Cloud *clouds, const uint64_t *key, int max_level, int n_ngb, double *h,
                          float4 *pk_hme) {
    const int nn = T.depth_begin[max_level + 2];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        const int2 r = T.range[i];
        const int2 ch = T.child[i];
        if ((ch.y & 255) != 0 || r.y == 0) continue;  // leaves only
        const Cloud &cl = clouds[(int)(key[r.x] >> (3 * max_level))];
        const int lvl = ch.y >> 8;
        const double side = ldexp(cl.size, -lvl);
        const double dens = (double)r.y / (side * side * side);
        const double hg = 0.5 * cbrt(3.0 * (double)n_ngb / (4.0 * M_PI * dens));
        for (int k = r.x; k < r.x + r.y; ++k) {
            h[k] = hg;
            pk_hme[k].x = (float)hg;
        }
    }
}

void launch_h_guess(State &S, const Params &P, cudaStream_t st) {
    if (S.ncloud == 0 || S.n == 0) return;
    S.list_valid = false;
    k_h_guess<<<S.num_sms * 4, 256, 0, st>>>(S.tree, S.clouds, S.key, S.max_level, P.n_ngb, S.h, S.pk_hme);
}

// ------------------------------------------------------------ walk groups
// Target groups for the walks: runs of at most kGroup consecutive particles
// whose bounding box is small on the scale of their smoothing lengths (a
// walk's work grows with (group extent + 2h)^3, so one sprawling group can
// stall a whole persistent kernel).
//
// A node is *compact* if it holds <= kGroup particles and its bbox extent is
// at most kGroupSpan * hmax (or it holds one particle, or no h is known yet).
// Every non-compact internal node acts as a parent: it packs its consecutive
// compact children greedily into groups while the merged bbox stays within
// kGroupSpan * (largest hmax) and the count within kGroup; a non-compact leaf
// child is split into kGroup-sized chunks if it is only too populous, or into
// one group per particle if it is sprawling.  A compact root is one group.
// Every particle lands in exactly one group: the first compact node on its
// root-to-leaf chain is packed by its (non-compact) parent, and a chain
// without one ends in a non-compact leaf that its parent splits.  The order
// of the group table does not affect any result.
constexpr double kGroupSpan = 4.0;

__device__ __forceinline__ void emit_group(int2 *groups, int *gcl, int *ng, int first, int count, int cloud) {
    const int g = atomicAdd(ng, 1);
    groups[g] = make_int2(first, count);
    gcl[g] = cloud;
}

__device__ __forceinline__ double node_extent(const Tree &T, int i) {
    const int cap = T.cap;
    return fmax(T.bmax[i] - T.bmin[i],
                fmax(T.bmax[cap + i] - T.bmin[cap + i], T.bmax[2 * cap + i] - T.bmin[2 * cap + i]));
}

// length scale of a node: its largest h, or "any size" before h is known
__device__ __forceinline__ double node_scale(const Tree &T, int i) {
    const double h = T.hmax[i];
    return h > 0.0 ? kGroupSpan * h : DBL_MAX;
}

__device__ __forceinline__ bool compact_node(const Tree &T, int i) {
    const int cnt = T.range[i].y;
    return cnt <= kGroup && (cnt == 1 || node_extent(T, i) <= node_scale(T, i));
}

// a leaf that is not compact: kGroup-sized chunks if it is only too populous,
// one group per particle if it sprawls
__device__ __forceinline__ void split_leaf(const Tree &T, int c, int2 *groups, int *gcl, int *ng, int cloud) {
    const int2 r = T.range[c];
    const int step = node_extent(T, c) <= node_scale(T, c) ? kGroup : 1;
    for (int f = r.x; f < r.x + r.y; f += step) emit_group(groups, gcl, ng, f, min(step, r.x + r.y - f), cloud);
}

__global__ void k_make_groups(Tree T, int ncloud, int max_depth, const uint64_t *key, int max_level,
                              int2 *groups, int *gcl, int *ng) {
    const int nn = T.depth_begin[max_depth];
    const int cap = T.cap;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        const int2 r = T.range[i];
        if (r.y == 0) continue;
        const int cloud = (int)(key[r.x] >> (3 * max_level));
        const int2 ch = T.child[i];
        const int nch = ch.y & 255;
        const bool ci = compact_node(T, i);
        if (i < ncloud) {  // a cloud root: nobody packs it
            if (ci) {
                emit_group(groups, gcl, ng, r.x, r.y, cloud);
                continue;
            }
            if (nch == 0) {
                split_leaf(T, i, groups, gcl, ng, cloud);
                continue;
            }
        }
        if (nch == 0 || ci) continue;  // leaves and compact nodes are handled by their parent
        int open_first = -1, open_count = 0;
        double lo[3], hi[3], scale = 0.0;
        auto flush = [&]() {
            if (open_first >= 0) emit_group(groups, gcl, ng, open_first, open_count, cloud);
            open_first = -1;
            open_count = 0;
        };
        for (int c = ch.x; c < ch.x + nch; ++c) {
            const int2 cr = T.range[c];
            if (cr.y == 0) continue;
            if (compact_node(T, c)) {
                bool merged = false;
                if (open_first >= 0 && open_count + cr.y <= kGroup) {
                    double ext = 0.0;
                    for (int d = 0; d < 3; ++d)
                        ext = fmax(ext, fmax(hi[d], T.bmax[d * cap + c]) - fmin(lo[d], T.bmin[d * cap + c]));
                    const double sc = fmax(scale, node_scale(T, c));
                    if (ext <= sc) {
                        open_count += cr.y;
                        for (int d = 0; d < 3; ++d) {
                            lo[d] = fmin(lo[d], T.bmin[d * cap + c]);
                            hi[d] = fmax(hi[d], T.bmax[d * cap + c]);
                        }
                        scale = sc;
                        merged = true;
                    }
                }
                if (!merged) {
                    flush();
                    open_first = cr.x;
                    open_count = cr.y;
                    for (int d = 0; d < 3; ++d) {
                        lo[d] = T.bmin[d * cap + c];
                        hi[d] = T.bmax[d * cap + c];
                    }
                    scale = node_scale(T, c);
                }
            } else {
                flush();
                if ((T.child[c].y & 255) == 0) split_leaf(T, c, groups, gcl, ng, cloud);
                // a non-compact internal child packs its own children
            }
        }
        flush();
    }
}

void launch_groups(State &S, cudaStream_t st) {
    cudaMemsetAsync(S.ngroups_dev, 0, sizeof(int), st);
    if (S.ncloud == 0 || S.n == 0) return;
    k_make_groups<<<S.num_sms * 4, 256, 0, st>>>(S.tree, S.ncloud, S.max_level + 2, S.key, S.max_level,
                                                S.groups, S.group_cloud, S.ngroups_dev);
}

void launch_tree_build(State &S, const Params &P, cudaStream_t st) {
    S.list_valid = false;  // a new order invalidates the neighbour lists
    if (S.ncloud == 0) return;
    Tree &T = S.tree;
    const int maxd = S.max_level + 1;  // depths 0..max_level
    k_tree_roots<<<(S.ncloud + 127) / 128, 128, 0, st>>>(T, S.clouds, S.ncloud, S.key, S.max_level);
    const int blocks = S.num_sms * 4;
    for (int d = 0; d < maxd; ++d)
        k_tree_level<<<blocks, 256, 0, st>>>(T, S.key, d, P.leaf_size, S.max_level, S.status);
    MomArgs a;
    a.pos = S.pos; a.m = S.m; a.h = S.h; a.eps = S.eps; a.n = S.n;
    a.clouds = S.clouds; a.key = S.key; a.max_level = S.max_level;
    a.inv_theta = P.theta > 0 ? 1.0 / P.theta : __builtin_inf();
    a.mac_offset = P.mac == SPH3_MAC_BH_OFFSET;
    for (int d = maxd; d >= 0; --d) k_tree_moments<<<blocks * 4, 128, 0, st>>>(T, a, d, P.quadrupole);
    k_tree_totals<<<blocks, 256, 0, st>>>(T, maxd + 1, S.counters);
    launch_groups(S, st);
}

}  // namespace sph3

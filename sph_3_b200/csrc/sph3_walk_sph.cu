// SPH walks: bootstrap h, h search, density (+ div/curl v, EOS) and the fused
// hydro acceleration + du/dt pass, plus the neighbour-set export used by the
// parity tests.
//
// Every pass is one persistent kernel: warps pull compact particle groups
// (<= 32, built from the octree) from an atomic counter, walk the octree once
// per group (sph3_walk.cuh) and stream the candidate leaves through a
// double-buffered 32-entry shared-memory tile of 4-wide entries.  Two
// instantiations per pass:
//   float  -- mixed precision: positions in the FP32 frame of the group's
//             reference cell (exact integer cell offsets + FP32 in-cell
//             offsets), FP32 kernel arithmetic, FP64 results;
//   double -- the plain FP64 path: absolute FP64 positions and the
//             reference's own expressions for every predicate (no FMA
//             contraction in them), so neighbour sets and the reference h
//             rule are bit-exact.
// The kernel formulas follow sph_code/libsx.py (M4 kernel, sigma = 1/pi,
// hbar_ij = (h_i + h_j) / 2, support q <= 2) and sph_code/shear.py.
#include <cfloat>
#include <mutex>
#include <set>
#include <vector>

#include "sph3_walk.cuh"

namespace sph3 {

constexpr double kSig = 0.31830988618379067154;  // 1/pi
constexpr float kSigF = 0.31830988618379067154f;

// ------------------------------------------------------------ arguments
struct WalkArgs {
    const int2 *groups;
    const int *ngroups_dev;
    const int *group_cloud;
    const Cloud *clouds;
    int ncloud;
    const int2 *range;
    const int2 *child;
    const float4 *box_c;
    const float4 *box_h;
    const float4 *sw;  // walk records [node][3]
    const float4 *pk_pos;
    const double *pos;
    int64_t n;
    int stack_cap;
    int max_depth;
    int node_cap;
    int periodic;
    double box[3];
    int *work;
    unsigned *status;
    unsigned long long *counters;
    int visit_slot;  // counter that accumulates this pass's node visits
};

// division in the pass precision: the FP32 path uses the approximate
// hardware reciprocal, the FP64 path IEEE division
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }

// exact FP64 distance as the reference writes it: sqrt(dx*dx + dy*dy + dz*dz)
__device__ __forceinline__ double exact_dist(double dx, double dy, double dz) {
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
}

// The SPH walks take a node with at most kSphLeaf particles whole, as if it
// were a leaf: below that size descending costs more walk steps than the
// extra candidates it saves (the per-candidate reach test still drops them;
// the gravity walk keeps the tree's own leaves).
constexpr int kSphLeaf = 64;

// Walk the tree for one group, calling flush(nleaf) on full leaf queues.
// A node is kept if the gap between its bbox and the group bbox is at most
// reach = Rg + (node_h ? hmax_node : 0) (times a 4e-5 safety margin; the
// exact pair predicate decides); images shift the nodes by `shift`.
template <class Flush>
__device__ void collect_leaves(const WalkArgs &a, const WarpMem &wm, int root, const GroupBox &gb,
                               float Rg, bool node_h, float3 shift, Flush &flush) {
    const int lane = lane_id();
    int top = 1;
    if (lane == 0) wm.stack[0] = root;
    __syncwarp();
    int nleaf = 0;
    const float margin = 1.0f + 4e-5f;
    // every node is popped at most once per walk; the bound only trips on a
    // corrupted tree, which then raises a status bit instead of spinning
    unsigned long long visits = 0;
    int guard = 0;
    for (; top > 0; ++guard) {
        if (guard > a.node_cap) {
            if (lane == 0) set_status(a.status, SPH3_STATUS_STACK_OVERFLOW);
            break;
        }
        const int p = pop_width(top, a.stack_cap, a.max_depth);
        visits += p;
        int node = -1;
        if (lane < p) node = wm.stack[top - 1 - lane];
        __syncwarp();
        top -= p;
        bool take = false;
        int nch = 0, cf = 0;
        if (node >= 0) {
            // one record per node: box, half widths + hmax, children (one round trip)
            const float4 bc = a.sw[3 * node], bh = a.sw[3 * node + 1], w2 = a.sw[3 * node + 2];
            const int chy = __float_as_int(w2.y);
            float3 c = rel_to(bc, gb.ref, gb.s10);
            c.x += shift.x;
            c.y += shift.y;
            c.z += shift.z;
            const float reach = (Rg + (node_h ? bh.w : 0.f)) * margin;
            const float g2 = box_gap2(gb, c, make_float3(bh.x, bh.y, bh.z));
            if (chy >= 0 && g2 <= reach * reach) {
                const int k = chy & 255;
                if (k == 0 || __float_as_int(w2.z) <= kSphLeaf) {
                    take = true;
                } else {
                    nch = k;
                    cf = __float_as_int(w2.x);
                }
            }
        }
        const unsigned tb = __ballot_sync(kFull, take);
        if (take) wm.leafq[nleaf + __popc(tb & lanemask_lt())] = node;
        nleaf += __popc(tb);
        top = push_children(wm.stack, top, a.stack_cap, nch, cf, a.status);
        if (nleaf > kLeafQ - 32) {
            __syncwarp();
            flush(nleaf);
            nleaf = 0;
        }
    }
    __syncwarp();
    if (nleaf > 0) flush(nleaf);
    if (lane == 0) {  // walk statistics: node visits per pass, longest walk (and where)
        atomicAdd(&a.counters[a.visit_slot], visits);
        atomicMax(&a.counters[kCntWalkMaxIter], (unsigned long long)guard);
        atomicMax(&a.counters[kCntWalkMaxWhere],
                  ((unsigned long long)guard << 40) | ((unsigned long long)a.visit_slot << 32) |
                      (unsigned long long)(unsigned)gb.first);
    }
}

// ------------------------------------------------------------ group setup
struct GroupInfo {
    int first, count, cloud, i;
    bool active;
    int ref;
    float s10;
    int root;
    float3 prel;  // target in the group frame (FP32)
};

__device__ __forceinline__ GroupInfo group_info(const WalkArgs &a, int g) {
    GroupInfo gi;
    const int2 gr = a.groups[g];
    gi.first = gr.x;
    gi.count = gr.y;
    gi.cloud = a.group_cloud[g];
    const Cloud &cl = a.clouds[gi.cloud];
    gi.s10 = cl.s10;
    gi.root = cl.root;
    gi.ref = __float_as_int(a.pk_pos[gi.first].w);
    const int lane = lane_id();
    gi.active = lane < gi.count;
    gi.i = gi.first + (gi.active ? lane : 0);
    gi.prel = rel_to(a.pk_pos[gi.i], gi.ref, gi.s10);
    return gi;
}

// source position in the group frame: FP32 relative (mixed) or absolute FP64
template <typename R>
__device__ __forceinline__ V4<R> src_pos(const WalkArgs &a, const GroupInfo &gi, int j, float3 s, R w) {
    V4<R> p;
    if (sizeof(R) == 8) {
        p.x = (R)(a.pos[j] + (double)s.x);
        p.y = (R)(a.pos[a.n + j] + (double)s.y);
        p.z = (R)(a.pos[2 * a.n + j] + (double)s.z);
    } else {
        const float3 q = rel_to(a.pk_pos[j], gi.ref, gi.s10);
        p.x = (R)(q.x + s.x);
        p.y = (R)(q.y + s.y);
        p.z = (R)(q.z + s.z);
    }
    p.w = w;
    return p;
}

// group-frame FP32 position of source j shifted by s (for the reach filter)
__device__ __forceinline__ float3 frame_pos(const WalkArgs &a, const GroupInfo &gi, int j, float3 s) {
    const float3 q = rel_to(a.pk_pos[j], gi.ref, gi.s10);
    return make_float3(q.x + s.x, q.y + s.y, q.z + s.z);
}

// can a source at p with smoothing length hj reach any target of the group
// (gap to the group box <= reach + hj, with the walk's 4e-5 safety margin)?
__device__ __forceinline__ bool reaches(const GroupBox &gb, float3 p, float reach) {
    const float r = reach * (1.0f + 4e-5f);
    return point_gap2(gb, p) <= r * r;
}

// ================================================================= h search
struct HArgs {
    WalkArgs w;
    double *h;
    float4 *pk_hme;
    int *nngb;
    int n_ngb, tol, max_iter;
};

constexpr int kHK = 16;  // thresholds per pass in the reference-step mode
constexpr double kNewtonDelta = 0.08;

template <typename R, int MODE>
__device__ __forceinline__ void h_search_body(const HArgs &A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const WalkArgs &a = A.w;
    using E = V4<R>;
    WarpMem wm = carve_warp_mem(smem, a.stack_cap, sizeof(E) * 64);
    E *tile = reinterpret_cast<E *>(wm.tile);
    const int lane = lane_id();
    constexpr int K = MODE == SPH3_H_REFSTEP ? kHK : 2;
    const int up = A.n_ngb + A.tol, low = A.n_ngb - A.tol;
    unsigned long long pairs = 0, passes = 0;
    for (int g = next_group(a.work, a.status); g < *a.ngroups_dev; g = next_group(a.work, a.status)) {
        GroupInfo gi = group_info(a, g);
        const Cloud &cl = a.clouds[gi.cloud];
        const int64_t ncl = cl.end - cl.begin;
        GroupBox gb = group_box(gi.prel, gi.active, gi.ref, gi.s10);
        gb.first = gi.first;
        R tx, ty, tz;
        if (sizeof(R) == 8) {
            tx = (R)a.pos[gi.i];
            ty = (R)a.pos[a.n + gi.i];
            tz = (R)a.pos[2 * a.n + gi.i];
        } else {
            tx = (R)gi.prel.x;
            ty = (R)gi.prel.y;
            tz = (R)gi.prel.z;
        }
        double h = A.h[gi.i];
        if (!(h > 0.0) || !isfinite(h)) h = (double)gi.s10;  // no usable start: one level-10 cell
        bool conv = !gi.active;
        int ncount = 0;
        int steps = 0;  // reference-rule steps taken
        int dir = 0;    // reference rule: -1 down, +1 up, 0 unknown (first pass)
        double lb = 0.0, hb = DBL_MAX;
        int n_hb = 0;  // count at hb
        bool failed = false;
        const double hcap = 4.0 * cl.size;
        for (int pass = 0; pass < A.max_iter + 2; ++pass) {
            if (__all_sync(kFull, conv)) break;
            double thr[K];
            if (MODE == SPH3_H_REFSTEP) {
                if (dir == 0) {
#pragma unroll
                    for (int k = 0; k < K; ++k) thr[k] = __dmul_rn(2.0, h);
                } else {
                    double hk = h;
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const double t = __dmul_rn(0.003, hk);
                        hk = dir < 0 ? __dsub_rn(hk, t) : __dadd_rn(hk, t);
                        thr[k] = __dmul_rn(2.0, hk);
                    }
                }
            } else {
                thr[0] = 2.0 * h;
                // the first pass counts at 2h only (a smaller reach: most groups
                // are already in the window with the previous step's h); later
                // passes also count at 2h (1 + delta) for the measured slope
                thr[1] = pass == 0 ? thr[0] : 2.0 * h * (1.0 + kNewtonDelta);
            }
            float reach = 0.f;
            if (!conv) {
#pragma unroll
                for (int k = 0; k < K; ++k) reach = fmaxf(reach, (float)thr[k]);
            }
            reach = warp_max(reach) * (1.0f + 1e-5f);
            float thr2f[K];
#pragma unroll
            for (int k = 0; k < K; ++k) thr2f[k] = (float)(thr[k] * thr[k]);
            int cnt[K];
#pragma unroll
            for (int k = 0; k < K; ++k) cnt[k] = 0;
            const Images ims = group_images(gb, reach, a.box, a.periodic);
            for (int im = 0; im < 27; ++im) {
                float3 s;
                if (!image_shift(ims, im, a.box, s)) continue;
                auto load = [&](int j, bool &keep) {
                    const V4<R> p = src_pos<R>(a, gi, j, s, (R)0);
                    const float3 f = sizeof(R) == 8 ? frame_pos(a, gi, j, s)
                                                    : make_float3((float)p.x, (float)p.y, (float)p.z);
                    keep = reaches(gb, f, reach);
                    return p;
                };
                auto interact = [&](const E *t, int ne) {
                    if (conv) return;
                    pairs += ne;
                    for (int e = 0; e < ne; ++e) {
                        const E q = t[e];
                        if (sizeof(R) == 8) {
                            const double d = exact_dist((double)q.x - (double)tx, (double)q.y - (double)ty,
                                                        (double)q.z - (double)tz);
#pragma unroll
                            for (int k = 0; k < K; ++k) cnt[k] += d < thr[k];
                        } else {
                            const float dx = (float)q.x - (float)tx;
                            const float dy = (float)q.y - (float)ty;
                            const float dz = (float)q.z - (float)tz;
                            const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
#pragma unroll
                            for (int k = 0; k < K; ++k) cnt[k] += d2 < thr2f[k];
                        }
                    }
                };
                // FP32: candidates staged as coordinate arrays and tested two per
                // packed instruction (d2 bit for bit as in the scalar loop above)
                float *xs = reinterpret_cast<float *>(wm.tile), *ys = xs + 64, *zs = ys + 64;
                auto load_xyz = [&](int j, bool &keep) {
                    const float3 q = rel_to(a.pk_pos[j], gi.ref, gi.s10);
                    SoaV<3> f;
                    f.v[0] = q.x + s.x;
                    f.v[1] = q.y + s.y;
                    f.v[2] = q.z + s.z;
                    keep = reaches(gb, make_float3(f.v[0], f.v[1], f.v[2]), reach);
                    return f;
                };
                auto interact_xyz = [&](int ne) {
                    if (conv) return;
                    pairs += ne;
                    const float2 ntx = make_float2(-(float)tx, -(float)tx);
                    const float2 nty = make_float2(-(float)ty, -(float)ty);
                    const float2 ntz = make_float2(-(float)tz, -(float)tz);
                    for (int e = 0; e < ne; e += 2) {
                        const float2 dx = __fadd2_rn(*reinterpret_cast<const float2 *>(xs + e), ntx);
                        const float2 dy = __fadd2_rn(*reinterpret_cast<const float2 *>(ys + e), nty);
                        const float2 dz = __fadd2_rn(*reinterpret_cast<const float2 *>(zs + e), ntz);
                        float2 d2 = __fmul2_rn(dz, dz);
                        d2 = __ffma2_rn(dy, dy, d2);
                        d2 = __ffma2_rn(dx, dx, d2);
#pragma unroll
                        for (int k = 0; k < K; ++k) cnt[k] += (d2.x < thr2f[k]) + (d2.y < thr2f[k]);
                    }
                };
                auto flush = [&](int nl) {
                    if constexpr (sizeof(R) == 4)
                        flush_leaves_compact_soa<3>(a.range, wm.leafq, nl, xs,
                                                    SoaV<3>{{1e18f, 1e18f, 1e18f}}, load_xyz, interact_xyz);
                    else
                        flush_leaves_compact(a.range, wm.leafq, nl, tile, load, interact);
                };
                collect_leaves(a, wm, gi.root, gb, reach, false, s, flush);
            }
            ++passes;
            // ---- update (lanes already converged keep their h)
            if (conv) {
            } else if (MODE == SPH3_H_REFSTEP) {
                if (dir == 0) {
                    ncount = cnt[0];
                    if (ncount <= up && ncount >= low) conv = true;
                    else dir = ncount > up ? -1 : 1;
                } else {
                    double hk = h;
                    for (int k = 0; k < K; ++k) {
                        if (steps >= A.max_iter) {
                            failed = true;
                            conv = true;
                            break;
                        }
                        const double t = __dmul_rn(0.003, hk);
                        hk = dir < 0 ? __dsub_rn(hk, t) : __dadd_rn(hk, t);
                        ++steps;
                        ncount = cnt[k];
                        h = hk;
                        if (ncount <= up && ncount >= low) {
                            conv = true;
                            break;
                        }
                        const int nd = ncount > up ? -1 : 1;
                        if (nd != dir) {  // crossed the window: the rule turns around
                            dir = nd;
                            break;
                        }
                    }
                }
            } else {
                const int n0 = cnt[0], n1 = cnt[1];
                ncount = n0;
                if (n0 <= up && n0 >= low) {
                    conv = true;
                } else if (pass >= A.max_iter || (n0 < low && (int64_t)n0 >= ncl)) {
                    // out of iterations, or the whole system is inside 2h already
                    failed = true;
                    conv = true;
                } else {
                    // Newton step on ln N(ln h) with the slope measured between
                    // h and h (1 + delta), safeguarded by the bracket [lb, hb]
                    if (n0 > up && h < hb) {
                        hb = h;
                        n_hb = n0;
                    } else if (n0 < low) {
                        lb = fmax(lb, h);
                    }
                }
                if (!conv && lb > 0.0 && hb < DBL_MAX && hb - lb <= 1e-6 * hb) {
                    // the count jumps over the whole window at one radius (a
                    // shell of equidistant neighbours, e.g. on a lattice): no h
                    // reaches the window, take the smallest h above the jump
                    h = hb;
                    ncount = n_hb;
                    conv = true;
                } else if (!conv) {
                    double hn;
                    if (n0 == 0) {
                        hn = 2.0 * h;
                    } else {
                        // slope of ln N over ln h: measured, or 3 (uniform density) on the first pass
                        double sl = pass > 0 && n1 > n0 ? log((double)n1 / (double)n0) / log1p(kNewtonDelta) : 3.0;
                        sl = fmin(fmax(sl, 1.0), 6.0);
                        hn = h * exp((log((double)A.n_ngb) - log((double)n0)) / sl);
                    }
                    hn = fmin(fmax(hn, 0.5 * h), 2.0 * h);
                    if (!(hn > lb && hn < hb)) {
                        if (lb > 0.0 && hb < DBL_MAX) hn = sqrt(lb * hb);
                        else if (hb < DBL_MAX) hn = hb * 0.8;
                        else hn = lb * 1.25;
                    }
                    h = fmin(hn, hcap);
                }
            }
        }
        if (!conv) failed = true;
        if (gi.active) {
            A.h[gi.i] = h;
            A.nngb[gi.i] = ncount;
            A.pk_hme[gi.i].x = (float)h;
            // minimum-image counting needs the kernel support inside half the box
            bool big = false;
            for (int d = 0; d < 3; ++d) big |= a.box[d] > 0.0 && 2.0 * h > 0.5 * a.box[d];
            if (big) set_status(a.status, SPH3_STATUS_BOX_TOO_SMALL);
        }
        const unsigned fb = __ballot_sync(kFull, gi.active && failed);
        if (fb && lane == 0) set_status(a.status, SPH3_STATUS_H_NOT_CONVERGED);
    }
    pairs = warp_sum(pairs);
    if (lane == 0) {
        atomicAdd(&a.counters[4], pairs);
        atomicAdd(&a.counters[5], passes);
    }
}

template <typename R, int MODE>
__global__ void __launch_bounds__(kWalkWarps * 32, kWalkMinBlocks) k_h_search(HArgs A) {
    h_search_body<R, MODE>(A);
}

// The mixed Newton search (the per-step path) capped at 96 registers: 20
// resident warps per SM instead of 16 (its walk is latency-bound).
__global__ void __maxnreg__(96) k_h_search_f32_newton(HArgs A) { h_search_body<float, SPH3_H_NEWTON>(A); }

// ============================================================ bootstrap h
// h = 0.5 * (k-th smallest distance, self included), the reference's
// smoothing_length_mpi / do_smoothingX (sph_code/libsx.py:752-800), exact:
// a radius that holds k+1 particles, then a 17-way bisection on the bit
// pattern of the FP64 distance.
struct BootArgs {
    WalkArgs w;
    double *h;
    float4 *pk_hme;
    int k;
};

__global__ void __launch_bounds__(kWalkWarps * 32, kWalkMinBlocks) k_boot_h(BootArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const WalkArgs &a = A.w;
    using E = V4<double>;
    WarpMem wm = carve_warp_mem(smem, a.stack_cap, sizeof(E) * 64);
    E *tile = reinterpret_cast<E *>(wm.tile);
    for (int g = next_group(a.work, a.status); g < *a.ngroups_dev; g = next_group(a.work, a.status)) {
        GroupInfo gi = group_info(a, g);
        const Cloud &cl = a.clouds[gi.cloud];
        const int64_t ncl = cl.end - cl.begin;
        const int need = (int)std::min<int64_t>((int64_t)A.k, ncl - 1) + 1;
        GroupBox gb = group_box(gi.prel, gi.active, gi.ref, gi.s10);
        gb.first = gi.first;
        const double tx = a.pos[gi.i], ty = a.pos[a.n + gi.i], tz = a.pos[2 * a.n + gi.i];
        // phase 1: grow a common radius until every target has `need` particles within it
        double Rg = 2.0 * (double)fmaxf(gb.hw.x, fmaxf(gb.hw.y, gb.hw.z)) + (double)gi.s10;
        for (int it = 0; it < 64; ++it) {
            int cnt = 0;
            const Images ims = group_images(gb, (float)Rg, a.box, a.periodic);
            for (int im = 0; im < 27; ++im) {
                float3 s;
                if (!image_shift(ims, im, a.box, s)) continue;
                auto load = [&](int j) { return src_pos<double>(a, gi, j, s, 0.0); };
                auto interact = [&](const E *t, int ne) {
                    for (int e = 0; e < ne; ++e) {
                        const E q = t[e];
                        cnt += exact_dist(q.x - tx, q.y - ty, q.z - tz) <= Rg;
                    }
                };
                auto flush = [&](int nl) {
                    flush_leaves(a.range, wm.leafq, nl, tile, load, interact);
                };
                collect_leaves(a, wm, gi.root, gb, (float)Rg * 1.0001f, false, s, flush);
            }
            if (__all_sync(kFull, !gi.active || cnt >= need)) break;
            Rg *= 2.0;
        }
        // phase 2: bisection on the distance bits, 16 thresholds per pass
        unsigned long long lo = 0ull, hi = (unsigned long long)__double_as_longlong(Rg);
        for (int it = 0; it < 40; ++it) {
            if (__all_sync(kFull, !gi.active || lo == hi)) break;
            unsigned long long t[16];
            const unsigned long long span = hi - lo;
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                if (span > 16ull) t[m] = lo + (span / 17ull) * (unsigned long long)(m + 1);
                else t[m] = (unsigned long long)m < span ? lo + m : hi;
            }
            double tv[16];
#pragma unroll
            for (int m = 0; m < 16; ++m) tv[m] = __longlong_as_double((long long)t[m]);
            int c[16];
#pragma unroll
            for (int m = 0; m < 16; ++m) c[m] = 0;
            const Images ims = group_images(gb, (float)Rg, a.box, a.periodic);
            for (int im = 0; im < 27; ++im) {
                float3 s;
                if (!image_shift(ims, im, a.box, s)) continue;
                auto load = [&](int j) { return src_pos<double>(a, gi, j, s, 0.0); };
                auto interact = [&](const E *tl, int ne) {
                    if (lo == hi) return;
                    for (int e = 0; e < ne; ++e) {
                        const E q = tl[e];
                        const double d = exact_dist(q.x - tx, q.y - ty, q.z - tz);
#pragma unroll
                        for (int m = 0; m < 16; ++m) c[m] += d <= tv[m];
                    }
                };
                auto flush = [&](int nl) {
                    flush_leaves(a.range, wm.leafq, nl, tile, load, interact);
                };
                collect_leaves(a, wm, gi.root, gb, (float)Rg * 1.0001f, false, s, flush);
            }
            if (lo != hi) {
                int m = 0;
                while (m < 16 && c[m] < need) ++m;
                if (m == 16) {
                    lo = t[15] + 1;
                } else {
                    const unsigned long long nlo = m > 0 ? t[m - 1] + 1 : lo;
                    hi = t[m];
                    lo = nlo;
                }
                if (lo > hi) lo = hi;
            }
        }
        if (gi.active) {
            const double hv = __longlong_as_double((long long)hi) * 0.5;
            A.h[gi.i] = hv;
            A.pk_hme[gi.i].x = (float)hv;
        }
    }
}

// =================================================== density, EOS, div/curl
struct DArgs {
    WalkArgs w;
    const float4 *pk_hme, *pk_vel;
    const double *h, *m, *vel, *u;
    double *rho, *P, *c, *divV, *curlV, *bal;
    float4 *pk_thm;
    double gamma;
    int keep_rho;
    // neighbour lists for the hydro pass (null: none kept)
    int *list, *nlist;
    int list_cap;
    int *ovf;  // particles with more pairs than list_cap
};

// tile entry: p = {x, y, z, h}, q = {m, vx, vy, vz}, and the sorted source
// index j for the neighbour lists: in the unused q.y without div/curl (no
// velocities staged), in a field of its own with them
template <typename R, bool DC>
struct DE {
    V4<R> p, q;
    int j;
    __device__ void set_j(int v) { j = v; }
    __device__ int get_j() const { return j; }
};

template <typename R>
struct DE<R, false> {
    V4<R> p, q;
    __device__ void set_j(int v) { q.y = sizeof(R) == 4 ? (R)__int_as_float(v) : (R)v; }
    __device__ int get_j() const { return sizeof(R) == 4 ? __float_as_int((float)q.y) : (int)q.y; }
};

// Neighbour lists are written particle-major (row i holds list_cap slots,
// list_cap a multiple of 8): each lane stages its pairs in shared memory and
// writes them 8 at a time (two 16-byte stores, one full 32-byte sector).
constexpr int kListChunk = 8;
constexpr size_t kListStageBytes = sizeof(int) * kListChunk * 32;
// task list of the balanced density pass: one (target lane, tile entry) pair
// per in-support candidate of a tile, at most 32 x 32
constexpr size_t kTaskBytes = sizeof(unsigned short) * 32 * 32;
constexpr size_t kDensityExtraBytes = kListStageBytes + kTaskBytes;

template <typename R, bool DC>
__device__ __forceinline__ void density_body(const DArgs &A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const WalkArgs &a = A.w;
    using E = DE<R, DC>;
    WarpMem wm = carve_warp_mem(smem, a.stack_cap, sizeof(E) * 64 + kDensityExtraBytes);
    // neighbour-list staging: slot x of lane l at stage[x * 32 + l] (conflict-free)
    int *stage = reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(wm.tile) + sizeof(E) * 64);
    unsigned short *tasks = reinterpret_cast<unsigned short *>(stage + kListChunk * 32);
    E *tile = reinterpret_cast<E *>(wm.tile);
    const int lane = lane_id();
    unsigned long long pairs = 0;
    for (int g = next_group(a.work, a.status); g < *a.ngroups_dev; g = next_group(a.work, a.status)) {
        GroupInfo gi = group_info(a, g);
        GroupBox gb = group_box(gi.prel, gi.active, gi.ref, gi.s10);
        gb.first = gi.first;
        R tx, ty, tz, th, tvx = 0, tvy = 0, tvz = 0;
        if (sizeof(R) == 8) {
            tx = (R)a.pos[gi.i]; ty = (R)a.pos[a.n + gi.i]; tz = (R)a.pos[2 * a.n + gi.i];
            th = (R)A.h[gi.i];
            if (DC) { tvx = (R)A.vel[gi.i]; tvy = (R)A.vel[a.n + gi.i]; tvz = (R)A.vel[2 * a.n + gi.i]; }
        } else {
            tx = (R)gi.prel.x; ty = (R)gi.prel.y; tz = (R)gi.prel.z;
            th = (R)A.pk_hme[gi.i].x;
            if (DC) { const float4 v = A.pk_vel[gi.i]; tvx = (R)v.x; tvy = (R)v.y; tvz = (R)v.z; }
        }
        const float hmax_g = warp_max(gi.active ? (float)th : 0.f);
        R rho = 0, sdiv = 0, cx = 0, cy = 0, cz = 0;
        int nkept = 0;  // in-support pairs found (kept in the list while < list_cap)
        const Images ims = group_images(gb, hmax_g + a.box_h[gi.root].w, a.box, a.periodic);
        for (int im = 0; im < 27; ++im) {
            float3 s;
            if (!image_shift(ims, im, a.box, s)) continue;
            auto load = [&](int j, bool &keep) {
                E en;
                float3 f;
                if (sizeof(R) == 8) {
                    en.p = src_pos<R>(a, gi, j, s, (R)A.h[j]);
                    en.q.x = (R)A.m[j];
                    if (DC) { en.q.y = (R)A.vel[j]; en.q.z = (R)A.vel[a.n + j]; en.q.w = (R)A.vel[2 * a.n + j]; }
                    f = frame_pos(a, gi, j, s);
                } else {
                    const float4 hm = A.pk_hme[j];
                    en.p = src_pos<R>(a, gi, j, s, (R)hm.x);
                    en.q.x = (R)hm.y;
                    if (DC) { const float4 v = A.pk_vel[j]; en.q.y = (R)v.x; en.q.z = (R)v.y; en.q.w = (R)v.z; }
                    f = make_float3((float)en.p.x, (float)en.p.y, (float)en.p.z);
                }
                en.set_j(j);
                keep = reaches(gb, f, hmax_g + (float)en.p.w);
                return en;
            };
            auto interact = [&](const E *t, int ne) {
                if (!gi.active) return;
                pairs += ne;
                // pass 1: which staged sources lie inside this target's support
                unsigned mask = 0;
                for (int e = 0; e < ne; ++e) {
                    const V4<R> p = t[e].p;
                    bool in;
                    if (sizeof(R) == 8) {
                        const double dx = __dsub_rn((double)tx, (double)p.x);
                        const double dy = __dsub_rn((double)ty, (double)p.y);
                        const double dz = __dsub_rn((double)tz, (double)p.z);
                        const double hij = __dmul_rn(0.5, __dadd_rn((double)th, (double)p.w));
                        in = __ddiv_rn(exact_dist(dx, dy, dz), hij) <= 2.0;
                    } else {
                        const float dx = (float)tx - (float)p.x;
                        const float dy = (float)ty - (float)p.y;
                        const float dz = (float)tz - (float)p.z;
                        const float hs = (float)th + (float)p.w;
                        in = fmaf(dx, dx, fmaf(dy, dy, dz * dz)) <= hs * hs;
                    }
                    mask |= (unsigned)in << e;
                }
                // pass 2: each lane runs the kernel only on its own neighbours
                while (mask) {
                    const int e = __ffs(mask) - 1;
                    mask &= mask - 1;
                    const E en = t[e];
                    if (A.list) {  // keep the pair for the hydro pass
                        if (nkept < A.list_cap) {
                            const int x = nkept & (kListChunk - 1);
                            stage[x * 32 + lane] = en.get_j();
                            if (x == kListChunk - 1) {
                                int4 *dst = reinterpret_cast<int4 *>(A.list + (size_t)gi.i * A.list_cap +
                                                                     (nkept - x));
                                dst[0] = make_int4(stage[lane], stage[32 + lane], stage[64 + lane], stage[96 + lane]);
                                dst[1] = make_int4(stage[128 + lane], stage[160 + lane], stage[192 + lane],
                                                   stage[224 + lane]);
                            }
                        }
                        ++nkept;
                    }
                    if (sizeof(R) == 8) {
                        // reference order: dx = x_i - x_j, q = |r| / hbar
                        const double dx = __dsub_rn((double)tx, (double)en.p.x);
                        const double dy = __dsub_rn((double)ty, (double)en.p.y);
                        const double dz = __dsub_rn((double)tz, (double)en.p.z);
                        const double rr = exact_dist(dx, dy, dz);
                        const double hij = __dmul_rn(0.5, __dadd_rn((double)th, (double)en.p.w));
                        const double q = __ddiv_rn(rr, hij);
                        {
                            const double ih = 1.0 / hij;
                            const double ih3 = ih * ih * ih;
                            double W;
                            if (q <= 1.0) W = kSig * ih3 * (1.0 - 1.5 * q * q + 0.75 * q * q * q);
                            else { const double tq = 2.0 - q; W = kSig * ih3 * 0.25 * tq * tq * tq; }
                            const double mj = (double)en.q.x;
                            rho += (R)(mj * W);
                            if (DC) {
                                double nW;
                                const double ih5 = ih3 * ih * ih;
                                if (q <= 1.0) nW = kSig * ih5 * (-3.0 + 2.25 * q);
                                else { const double tq = 2.0 - q; nW = -0.75 * kSig * ih5 * tq * tq / (q + 1e-20); }
                                const double gx = nW * dx, gy = nW * dy, gz = nW * dz;
                                const double vx = (double)tvx - (double)en.q.y;
                                const double vy = (double)tvy - (double)en.q.z;
                                const double vz = (double)tvz - (double)en.q.w;
                                sdiv += (R)(-mj * (vx * gx + vy * gy + vz * gz));
                                cx += (R)(mj * (vy * gz - vz * gy));
                                cy += (R)(mj * (vz * gx - vx * gz));
                                cz += (R)(mj * (vx * gy - vy * gx));
                            }
                        }
                    } else {
                        const float dx = (float)tx - (float)en.p.x;
                        const float dy = (float)ty - (float)en.p.y;
                        const float dz = (float)tz - (float)en.p.z;
                        const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                        const float hs = (float)th + (float)en.p.w;  // = 2 hbar
                        {
                            const float ih = __fdividef(2.0f, hs);
                            // |r| as d2 * rsqrt(d2) (0 for the self pair), and both
                            // branches of the kernel evaluated and selected: no
                            // divergence inside the warp
                            const float q = (d2 > 0.f ? d2 * rsqrtf(d2) : 0.f) * ih;
                            const float ih3 = ih * ih * ih;
                            const float tq = 2.0f - q;
                            const float w_in = fmaf(q * q, fmaf(0.75f, q, -1.5f), 1.0f);
                            const float w_out = 0.25f * tq * tq * tq;
                            const float W = kSigF * ih3 * (q <= 1.0f ? w_in : w_out);
                            rho = fmaf((float)en.q.x, W, (float)rho);
                            if (DC) {
                                float nW;
                                const float ih5 = ih3 * ih * ih;
                                if (q <= 1.0f) nW = kSigF * ih5 * fmaf(2.25f, q, -3.0f);
                                else { const float tq = 2.0f - q; nW = -0.75f * kSigF * ih5 * tq * tq * __fdividef(1.0f, q + 1e-20f); }
                                const float mj = (float)en.q.x * nW;
                                const float vx = (float)tvx - (float)en.q.y;
                                const float vy = (float)tvy - (float)en.q.z;
                                const float vz = (float)tvz - (float)en.q.w;
                                sdiv -= mj * fmaf(vx, dx, fmaf(vy, dy, vz * dz));
                                cx += mj * (vy * dz - vz * dy);
                                cy += mj * (vz * dx - vx * dz);
                                cz += mj * (vx * dy - vy * dx);
                            }
                        }
                    }
                }
            };
            // Mixed path without div/curl: pass 2 balanced over the warp.  The
            // in-support (target, entry) pairs of the tile become a task list
            // ordered by target; lane k runs task k of each chunk of 32 (target
            // values by shuffle), writes the pair into the target's neighbour
            // list, and the density terms are summed per target with a
            // segmented warp reduction (fixed order: deterministic).  Lanes no
            // longer idle while the lane with the most neighbours finishes.
            // the balanced pass's tile: six arrays of 64 floats (x, y, z, h, m and
            // the source index as float bits), so pass 1 tests two candidates
            // per packed FP32 instruction (the same roundings as pass 1 above)
            float *sx = reinterpret_cast<float *>(wm.tile), *sy = sx + 64, *sz = sy + 64, *sh = sz + 64,
                  *sm = sh + 64, *sj = sm + 64;
            auto load_soa = [&](int j, bool &keep) {
                const float4 hm = A.pk_hme[j];
                const float3 q = rel_to(a.pk_pos[j], gi.ref, gi.s10);
                SoaV<6> v;
                v.v[0] = q.x + s.x;
                v.v[1] = q.y + s.y;
                v.v[2] = q.z + s.z;
                v.v[3] = hm.x;
                v.v[4] = hm.y;
                v.v[5] = __int_as_float(j);
                keep = reaches(gb, make_float3(v.v[0], v.v[1], v.v[2]), hmax_g + hm.x);
                return v;
            };
            // Mixed path without div/curl: pass 2 balanced over the warp.  The
            // in-support (target, entry) pairs of the tile become a task list
            // ordered by target; lane k runs task k of each chunk of 32 (target
            // values by shuffle), writes the pair into the target's neighbour
            // list, and the density terms are summed per target with a
            // segmented warp reduction (fixed order: deterministic).  Lanes no
            // longer idle while the lane with the most neighbours finishes.
            auto interact_bal = [&](int ne) {
                if (gi.active) pairs += ne;
                unsigned mask = 0;
                if (gi.active) {
                    const float2 ntx = make_float2(-(float)tx, -(float)tx);
                    const float2 nty = make_float2(-(float)ty, -(float)ty);
                    const float2 ntz = make_float2(-(float)tz, -(float)tz);
                    const float2 th2 = make_float2((float)th, (float)th);
                    for (int e = 0; e < ne; e += 2) {
                        const float2 dx = __fadd2_rn(*reinterpret_cast<const float2 *>(sx + e), ntx);
                        const float2 dy = __fadd2_rn(*reinterpret_cast<const float2 *>(sy + e), nty);
                        const float2 dz = __fadd2_rn(*reinterpret_cast<const float2 *>(sz + e), ntz);
                        const float2 hs = __fadd2_rn(th2, *reinterpret_cast<const float2 *>(sh + e));
                        const float2 hs2 = __fmul2_rn(hs, hs);
                        float2 d2 = __fmul2_rn(dz, dz);
                        d2 = __ffma2_rn(dy, dy, d2);
                        d2 = __ffma2_rn(dx, dx, d2);
                        mask |= ((unsigned)(d2.x <= hs2.x) | ((unsigned)(d2.y <= hs2.y) << 1)) << e;
                    }
                    if (ne < 32) mask &= (1u << ne) - 1u;  // the pad entry of an odd batch
                }
                const int c = __popc(mask);
                const int incl = warp_incl_scan(c);
                const int total = __shfl_sync(kFull, incl, 31);
                const int off = incl - c;
                {
                    int o = off;
                    unsigned mm = mask;
                    while (mm) {
                        const int e = __ffs(mm) - 1;
                        mm &= mm - 1;
                        tasks[o++] = (unsigned short)((lane << 5) | e);
                    }
                }
                __syncwarp();
                for (int k0 = 0; k0 < total; k0 += 32) {
                    const int k = k0 + lane;
                    const bool valid = k < total;
                    const int task = valid ? (int)tasks[k] : 0;
                    const int tl = valid ? task >> 5 : 32;  // key: target lane (32 past the end)
                    const int e = task & 31;
                    const float qx = __shfl_sync(kFull, (float)tx, tl & 31);
                    const float qy = __shfl_sync(kFull, (float)ty, tl & 31);
                    const float qz = __shfl_sync(kFull, (float)tz, tl & 31);
                    const float qh = __shfl_sync(kFull, (float)th, tl & 31);
                    const int base = __shfl_sync(kFull, nkept, tl & 31);
                    const int toff = __shfl_sync(kFull, off, tl & 31);
                    float v = 0.f;
                    if (valid) {
                        if (A.list) {
                            const int slot = base + (k - toff);
                            if (slot < A.list_cap)
                                A.list[(size_t)(gi.first + tl) * A.list_cap + slot] = __float_as_int(sj[e]);
                        }
                        const float dx = qx - sx[e];
                        const float dy = qy - sy[e];
                        const float dz = qz - sz[e];
                        const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                        const float ih = __fdividef(2.0f, qh + sh[e]);
                        const float q = (d2 > 0.f ? d2 * rsqrtf(d2) : 0.f) * ih;
                        const float ih3 = ih * ih * ih;
                        const float tq = 2.0f - q;
                        const float w_in = fmaf(q * q, fmaf(0.75f, q, -1.5f), 1.0f);
                        const float w_out = 0.25f * tq * tq * tq;
                        v = sm[e] * (kSigF * ih3 * (q <= 1.0f ? w_in : w_out));
                    }
                    // segmented suffix sums over equal keys (keys are non-decreasing)
#pragma unroll
                    for (int d = 1; d < 32; d <<= 1) {
                        const float ov = __shfl_down_sync(kFull, v, d);
                        const int ot = __shfl_down_sync(kFull, tl, d);
                        if (lane + d < 32 && ot == tl) v += ov;
                    }
                    // each target takes the sum of its run inside this chunk
                    const int first_pos = off > k0 ? off - k0 : 0;
                    const float got = __shfl_sync(kFull, v, first_pos & 31);
                    if (c > 0 && off < k0 + 32 && off + c > k0) rho += (R)got;
                }
                nkept += c;
                __syncwarp();
            };
            auto flush = [&](int nl) {
                if constexpr (sizeof(R) == 4 && !DC)
                    flush_leaves_compact_soa<6>(a.range, wm.leafq, nl, sx,
                                                SoaV<6>{{1e18f, 1e18f, 1e18f, 0.f, 0.f, 0.f}}, load_soa,
                                                interact_bal);
                else
                    flush_leaves_compact(a.range, wm.leafq, nl, tile, load, interact);
            };
            collect_leaves(a, wm, gi.root, gb, hmax_g, true, s, flush);
        }
        if (gi.active) {
            const int i = gi.i;
            if (A.list) {
                A.nlist[i] = nkept;
                if (nkept > A.list_cap) atomicAdd(A.ovf, 1);
                if constexpr (!(sizeof(R) == 4 && !DC)) {  // the staged path: write the last partial chunk
                    const int kept = min(nkept, A.list_cap);
                    const int base = kept & ~(kListChunk - 1);
                    for (int x = 0; x < kept - base; ++x)
                        A.list[(size_t)i * A.list_cap + base + x] = stage[x * 32 + lane];
                }
            }
            double r, P, c;
            if (A.keep_rho) {  // div/curl only: divide by the caller's rho
                r = A.rho[i];
                P = A.P[i];
                c = A.c[i];
            } else {
                r = (double)rho;
                const double u = A.u[i];
                P = (A.gamma - 1.0) * r * u;
                c = sqrt(A.gamma * (A.gamma - 1.0) * u);
                A.rho[i] = r;
                A.P[i] = P;
                A.c[i] = c;
            }
            double f = 0.0;
            if (DC) {
                const double inv = r > 0.0 ? 1.0 / r : 0.0;
                const double dv = fabs((double)sdiv) * inv;
                const double cv = sqrt((double)cx * (double)cx + (double)cy * (double)cy + (double)cz * (double)cz) * inv;
                A.divV[i] = dv;
                A.curlV[i] = cv;
                f = dv / (dv + cv + 0.0001 * c / A.h[i]);
                A.bal[i] = f;
            }
            const double pr = r > 0.0 ? P / (r * r) : 0.0;
            A.pk_thm[i] = make_float4((float)r, (float)pr, (float)c, (float)f);
            if (!(r > 0.0)) set_status(a.status, SPH3_STATUS_ZERO_DENSITY);
        }
    }
    pairs = warp_sum(pairs);
    if (lane == 0) atomicAdd(&a.counters[2], pairs);
}

template <typename R, bool DC>
__global__ void __launch_bounds__(kWalkWarps * 32, kWalkMinBlocks) k_density(DArgs A) {
    density_body<R, DC>(A);
}

// The mixed density pass of every step capped at 96 registers: 20 resident
// warps per SM instead of 16.
__global__ void __maxnreg__(96) k_density_f32(DArgs A) { density_body<float, false>(A); }

// ============================================================ hydro
struct YArgs {
    WalkArgs w;
    const float4 *pk_hme, *pk_vel, *pk_thm;
    const double *h, *m, *vel, *rho, *P, *c, *bal;
    double *acc_sph, *dudt;
    double *vsig;  // max signal velocity over the pairs (written with the acceleration)
    double alpha, beta, eta;
    // only_overflow: walk only for particles whose neighbour list overflowed
    const int *nlist;
    int list_cap;
    int only_overflow;
    const int *ovf;  // number of overflowed lists (only_overflow: nothing to do when 0)
};

// tile entry: p = {x, y, z, h}, v = {vx, vy, vz, m}, t = {rho, P/rho^2, c, f}
template <typename R>
struct YE {
    V4<R> p, v, t;
};

// One hydro pair, after the pair geometry (d = r_i - r_j, |d|, hbar_ij,
// q = |d| / hbar_ij): the reference's acceleration and du/dt terms
// (sph_code/libsx.py:117-165, :364-417; MG83 :236-246; Balsara
// sph_code/shear.py:193-215) and the pair's signal velocity.  sv = {vx, vy,
// vz, m} and st = {rho, P/rho^2, c, f} of the source.  Shared by the walk and
// the list passes, so both run the same arithmetic.
template <typename R, int VISC, bool ACC, bool DU>
__device__ __forceinline__ void hydro_pair(R dx, R dy, R dz, R rr, R hij, R q, R tvx, R tvy, R tvz, R trho, R tpr,
                                           R tc, R tf, const V4<R> &sv, const V4<R> &st, R alpha, R beta, R eta2,
                                           R &ax, R &ay, R &az, R &du, R &vmax) {
    const R ih = fdiv((R)1, hij);
    const R ih5 = ih * ih * ih * ih * ih;
    R nW;
    if (q <= (R)1) nW = (R)kSig * ih5 * ((R)-3 + (R)2.25 * q);
    else { const R tq = (R)2 - q; nW = fdiv((R)(-0.75 * kSig) * ih5 * tq * tq, q + (R)1e-20); }
    const R gx = nW * dx, gy = nW * dy, gz = nW * dz;
    const R vx = tvx - sv.x, vy = tvy - sv.y, vz = tvz - sv.z;
    const R vr = vx * dx + vy * dy + vz * dz;
    const R rhoij = (R)0.5 * (trho + st.x);
    R PI = 0;
    R vsig;  // signal velocity (time-step estimate)
    if (VISC == SPH3_VISC_MG83) {
        const R cij = (R)0.5 * (tc + st.z);
        const R mu = fdiv(hij * vr, rr * rr + hij * hij * eta2);
        if (vr <= (R)0) PI = fdiv(-alpha * cij * mu + beta * mu * mu, rhoij);
        if (ACC) vsig = tc + st.z - (R)3 * fdiv(vr, rr + (R)1e-5);
    } else {
        const R w = fdiv(vr, rr + (R)1e-5);
        vsig = tc + st.z - (R)3 * w;
        if (vr <= (R)0) PI = fdiv((R)-0.5 * alpha * vsig * w, rhoij);
        if (VISC == SPH3_VISC_BALSARA) PI = (R)0.5 * (tf + st.w) * PI;
    }
    if (ACC && vsig > vmax) vmax = vsig;
    const R mj = sv.w;
    if (ACC) {
        const R pt = mj * (tpr + st.y + PI);
        ax -= pt * gx;
        ay -= pt * gy;
        az -= pt * gz;
    }
    if (DU) du += mj * (tpr + (R)0.5 * PI) * (vx * gx + vy * gy + vz * gz);
}

template <typename R, int VISC, bool ACC, bool DU>
__global__ void __launch_bounds__(kWalkWarps * 32, kWalkMinBlocks) k_hydro(YArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const WalkArgs &a = A.w;
    using E = YE<R>;
    if (A.only_overflow && *A.ovf == 0) return;  // every list fitted
    WarpMem wm = carve_warp_mem(smem, a.stack_cap, sizeof(E) * 64);
    E *tile = reinterpret_cast<E *>(wm.tile);
    const int lane = lane_id();
    unsigned long long pairs = 0;
    const R alpha = (R)A.alpha, beta = (R)A.beta, eta2 = (R)(A.eta * A.eta);
    for (int g = next_group(a.work, a.status); g < *a.ngroups_dev; g = next_group(a.work, a.status)) {
        GroupInfo gi = group_info(a, g);
        const bool mine = !A.only_overflow || (gi.active && A.nlist[gi.i] > A.list_cap);
        if (A.only_overflow && !__any_sync(kFull, mine)) continue;
        GroupBox gb = group_box(gi.prel, gi.active, gi.ref, gi.s10);
        gb.first = gi.first;
        const int i = gi.i;
        R tx, ty, tz, tvx, tvy, tvz, th, trho, tpr, tc, tf;
        if (sizeof(R) == 8) {
            tx = (R)a.pos[i]; ty = (R)a.pos[a.n + i]; tz = (R)a.pos[2 * a.n + i];
            tvx = (R)A.vel[i]; tvy = (R)A.vel[a.n + i]; tvz = (R)A.vel[2 * a.n + i];
            th = (R)A.h[i]; trho = (R)A.rho[i];
            tpr = (R)(A.P[i] / (A.rho[i] * A.rho[i]));
            tc = (R)A.c[i]; tf = (R)A.bal[i];
        } else {
            tx = (R)gi.prel.x; ty = (R)gi.prel.y; tz = (R)gi.prel.z;
            const float4 v = A.pk_vel[i];
            tvx = (R)v.x; tvy = (R)v.y; tvz = (R)v.z;
            th = (R)A.pk_hme[i].x;
            const float4 t = A.pk_thm[i];
            trho = (R)t.x; tpr = (R)t.y; tc = (R)t.z; tf = (R)t.w;
        }
        const float hmax_g = warp_max(gi.active ? (float)th : 0.f);
        R ax = 0, ay = 0, az = 0, du = 0, vmax = 0;
        const Images ims = group_images(gb, hmax_g + a.box_h[gi.root].w, a.box, a.periodic);
        for (int im = 0; im < 27; ++im) {
            float3 s;
            if (!image_shift(ims, im, a.box, s)) continue;
            auto load = [&](int j, bool &keep) {
                E en;
                float3 f;
                if (sizeof(R) == 8) {
                    f = frame_pos(a, gi, j, s);
                    en.p = src_pos<R>(a, gi, j, s, (R)A.h[j]);
                    en.v.x = (R)A.vel[j]; en.v.y = (R)A.vel[a.n + j]; en.v.z = (R)A.vel[2 * a.n + j];
                    en.v.w = (R)A.m[j];
                    const double rj = A.rho[j];
                    en.t.x = (R)rj;
                    en.t.y = (R)(A.P[j] / (rj * rj));
                    en.t.z = (R)A.c[j];
                    en.t.w = (R)A.bal[j];
                } else {
                    const float4 hm = A.pk_hme[j];
                    en.p = src_pos<R>(a, gi, j, s, (R)hm.x);
                    const float4 v = A.pk_vel[j];
                    en.v.x = (R)v.x; en.v.y = (R)v.y; en.v.z = (R)v.z; en.v.w = (R)hm.y;
                    const float4 t = A.pk_thm[j];
                    en.t.x = (R)t.x; en.t.y = (R)t.y; en.t.z = (R)t.z; en.t.w = (R)t.w;
                    f = make_float3((float)en.p.x, (float)en.p.y, (float)en.p.z);
                }
                keep = reaches(gb, f, hmax_g + (float)en.p.w);
                return en;
            };
            auto interact = [&](const E *tl, int ne) {
                if (!gi.active) return;
                pairs += ne;
                // pass 1: which staged sources lie inside this target's support
                unsigned mask = 0;
                for (int e = 0; e < ne; ++e) {
                    const V4<R> p = tl[e].p;
                    bool in;
                    if (sizeof(R) == 8) {
                        const double ddx = __dsub_rn((double)tx, (double)p.x);
                        const double ddy = __dsub_rn((double)ty, (double)p.y);
                        const double ddz = __dsub_rn((double)tz, (double)p.z);
                        const double dh = __dmul_rn(0.5, __dadd_rn((double)th, (double)p.w));
                        in = __ddiv_rn(exact_dist(ddx, ddy, ddz), dh) <= 2.0;
                    } else {
                        const float fx = (float)tx - (float)p.x;
                        const float fy = (float)ty - (float)p.y;
                        const float fz = (float)tz - (float)p.z;
                        const float hs = (float)th + (float)p.w;
                        in = fmaf(fx, fx, fmaf(fy, fy, fz * fz)) <= hs * hs;
                    }
                    mask |= (unsigned)in << e;
                }
                // pass 2: each lane runs the pair terms only on its own neighbours
                while (mask) {
                    const int e = __ffs(mask) - 1;
                    mask &= mask - 1;
                    const E en = tl[e];
                    R dx, dy, dz, rr, hij, q;
                    bool in;
                    if (sizeof(R) == 8) {
                        const double ddx = __dsub_rn((double)tx, (double)en.p.x);
                        const double ddy = __dsub_rn((double)ty, (double)en.p.y);
                        const double ddz = __dsub_rn((double)tz, (double)en.p.z);
                        const double drr = exact_dist(ddx, ddy, ddz);
                        const double dh = __dmul_rn(0.5, __dadd_rn((double)th, (double)en.p.w));
                        const double dq = __ddiv_rn(drr, dh);
                        in = dq <= 2.0;
                        dx = (R)ddx; dy = (R)ddy; dz = (R)ddz; rr = (R)drr; hij = (R)dh; q = (R)dq;
                    } else {
                        dx = tx - en.p.x;
                        dy = ty - en.p.y;
                        dz = tz - en.p.z;
                        const R d2 = dx * dx + dy * dy + dz * dz;
                        const R hs = th + en.p.w;
                        in = d2 <= hs * hs;
                        rr = d2 > (R)0 ? (R)((float)d2 * rsqrtf((float)d2)) : (R)0;  // as the list pass
                        hij = (R)0.5 * hs;
                        q = (R)((float)rr * __fdividef(1.0f, (float)hij));
                    }
                    (void)in;
                    hydro_pair<R, VISC, ACC, DU>(dx, dy, dz, rr, hij, q, tvx, tvy, tvz, trho, tpr, tc, tf, en.v, en.t,
                                                 alpha, beta, eta2, ax, ay, az, du, vmax);
                }
            };
            auto flush = [&](int nl) {
                flush_leaves_compact(a.range, wm.leafq, nl, tile, load, interact);
            };
            collect_leaves(a, wm, gi.root, gb, hmax_g, true, s, flush);
        }
        if (gi.active && mine) {
            if (ACC) {
                A.acc_sph[i] = (double)ax;
                A.acc_sph[a.n + i] = (double)ay;
                A.acc_sph[2 * a.n + i] = (double)az;
                A.vsig[i] = (double)vmax;
            }
            if (DU) A.dudt[i] = (double)du;
        }
    }
    pairs = warp_sum(pairs);
    if (lane == 0) atomicAdd(&a.counters[3], pairs);
}

// ============================================================ hydro over lists
// Mixed path: the hydro pass over the neighbour lists kept by the density
// walk, one thread per particle.  The lists hold exactly the in-support pairs
// (|r| <= h_i + h_j in FP32, the same test as the walks' first pass) in the
// order the density walk met them, so this is the walk's pair loop without
// the walk: no tree traversal, no candidate tests.  Pair terms are the
// reference's (sph_code/libsx.py:117-165 acceleration, :364-417 du/dt; MG83
// :236-246; Balsara sph_code/shear.py:193-215) in FP32 on positions relative
// to the target's level-10 cell.  Periodic boxes use the minimum image (a
// unique image within the support: 2h < L/2 is checked by the h search).
// Particles whose list overflowed are skipped here and walked instead.
struct LArgs {
    const int *list, *nlist;
    int list_cap;
    const float4 *pk_pos, *pk_hme, *pk_vel, *pk_thm;
    float4 *hrec;  // [n][3] source records, packed by k_pack_hrec
    const uint64_t *key;
    int cloud_shift;
    const Cloud *clouds;
    int64_t n;
    int periodic;
    float box[3];
    double *acc_sph, *dudt, *vsig;
    float alpha, beta, eta2;
    unsigned long long *counters;
    // FP64 path: the masters
    const double *pos, *vel, *h, *m, *rho, *P, *c, *bal;
    double boxd[3];
    double alpha_d, beta_d, eta2_d;
};

// one 48-byte record per source: everything a hydro pair reads from it, in
// two 32-byte sectors instead of four (pk_pos, pk_hme, pk_vel, pk_thm)
__global__ void k_pack_hrec(LArgs A) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < A.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float4 hm = A.pk_hme[i], v = A.pk_vel[i], t = A.pk_thm[i];
        A.hrec[3 * i] = A.pk_pos[i];
        A.hrec[3 * i + 1] = make_float4(v.x, v.y, v.z, hm.y);
        A.hrec[3 * i + 2] = make_float4(t.x, t.y, t.z, hm.x);
    }
}

__device__ __forceinline__ float min_image(float d, float L) {
    if (L > 0.f) d -= L * rintf(d * (1.0f / L));
    return d;
}

template <int VISC, bool ACC, bool DU>
__global__ void __launch_bounds__(128, 7) k_hydro_list(LArgs A) {
    unsigned long long pairs = 0;
    const float alpha = A.alpha, beta = A.beta, eta2 = A.eta2;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < A.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int cnt = A.nlist[i];
        if (cnt > A.list_cap) continue;  // walked instead
        const float s10 = A.clouds[(int)(A.key[i] >> A.cloud_shift)].s10;
        const float4 pi = A.hrec[3 * i], tv = A.hrec[3 * i + 1], tt = A.hrec[3 * i + 2];  // tt = {rho, P/rho^2, c, h}
        const int ref = __float_as_int(pi.w);
        const float3 t = rel_to(pi, ref, s10);
        const float th = tt.w;
        const float tf = VISC == SPH3_VISC_BALSARA ? A.pk_thm[i].w : 0.f;
        float ax = 0.f, ay = 0.f, az = 0.f, du = 0.f, vmax = 0.f;
        // The row's indices come 4 at a time (16-byte loads, one chunk ahead:
        // a row holds list_cap slots, a multiple of 8, so whole chunks stay
        // inside it) and the next source's record is in flight while this
        // pair runs, so a pair waits on one load, not on an index load followed
        // by a record load.
        const int4 *row4 = reinterpret_cast<const int4 *>(A.list + (size_t)i * A.list_cap);
        int4 ids = cnt > 0 ? row4[0] : make_int4(0, 0, 0, 0);
        int4 ids_next = cnt > 4 ? row4[1] : ids;
        int jn = ids.x;
        float4 q0, q1, q2;
        if (cnt > 0) {
            q0 = A.hrec[3 * jn];
            q1 = A.hrec[3 * jn + 1];
            q2 = A.hrec[3 * jn + 2];
        }
        for (int k = 0; k < cnt; ++k) {
            const float4 r0 = q0, r1 = q1, r2 = q2;  // {pos}, {vx, vy, vz, m}, {rho, P/rho^2, c, h}
            const int j = jn;
            const int kn = k + 1;
            if (kn < cnt) {
                const int u = kn & 3;
                if (u == 0) {
                    ids = ids_next;
                    if (kn + 4 < cnt) ids_next = row4[(kn >> 2) + 1];
                }
                jn = u == 0 ? ids.x : (u == 1 ? ids.y : (u == 2 ? ids.z : ids.w));
                q0 = A.hrec[3 * jn];
                q1 = A.hrec[3 * jn + 1];
                q2 = A.hrec[3 * jn + 2];
            }
            const float3 p = rel_to(r0, ref, s10);
            const float hj = r2.w, mj = r1.w;
            float dx = t.x - p.x, dy = t.y - p.y, dz = t.z - p.z;
            if (A.periodic) {
                dx = min_image(dx, A.box[0]);
                dy = min_image(dy, A.box[1]);
                dz = min_image(dz, A.box[2]);
            }
            const float d2 = dx * dx + dy * dy + dz * dz;
            const float hs = th + hj;
            const float rr = d2 > 0.f ? d2 * rsqrtf(d2) : 0.f;  // as the density pass computes |r|
            const float hij = 0.5f * hs;
            const float q = rr * __fdividef(1.0f, hij);
            const V4<float> sv{r1.x, r1.y, r1.z, mj};
            const V4<float> st{r2.x, r2.y, r2.z, VISC == SPH3_VISC_BALSARA ? A.pk_thm[j].w : 0.f};
            hydro_pair<float, VISC, ACC, DU>(dx, dy, dz, rr, hij, q, tv.x, tv.y, tv.z, tt.x, tt.y, tt.z, tf, sv, st,
                                             alpha, beta, eta2, ax, ay, az, du, vmax);
        }
        pairs += (unsigned long long)cnt;
        if (ACC) {
            A.acc_sph[i] = (double)ax;
            A.acc_sph[A.n + i] = (double)ay;
            A.acc_sph[2 * A.n + i] = (double)az;
            A.vsig[i] = (double)vmax;
        }
        if (DU) A.dudt[i] = (double)du;
    }
    pairs = warp_sum(pairs);
    if ((threadIdx.x & 31) == 0 && pairs) atomicAdd(&A.counters[3], pairs);
}

// FP64 path over the same lists: the walk's FP64 pair arithmetic (the
// reference's operation order, correctly rounded predicates) on the FP64
// masters, with the periodic image the walk uses (source shifted by the
// FP32-rounded box length), so the results equal the walk's.
template <int VISC, bool ACC, bool DU>
__global__ void __launch_bounds__(256) k_hydro_list_f64(LArgs A) {
    unsigned long long pairs = 0;
    const int64_t n = A.n;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int cnt = A.nlist[i];
        if (cnt > A.list_cap) continue;  // walked instead
        const double tx = A.pos[i], ty = A.pos[n + i], tz = A.pos[2 * n + i], th = A.h[i];
        const double tvx = A.vel[i], tvy = A.vel[n + i], tvz = A.vel[2 * n + i];
        const double trho = A.rho[i], tpr = A.P[i] / (A.rho[i] * A.rho[i]), tc = A.c[i], tf = A.bal[i];
        double ax = 0, ay = 0, az = 0, du = 0, vmax = 0;
        const int *row = A.list + (size_t)i * A.list_cap;
        for (int k = 0; k < cnt; ++k) {
            const int j = row[k];
            double pj[3] = {A.pos[j], A.pos[n + j], A.pos[2 * n + j]};
            const double ti[3] = {tx, ty, tz};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double L = A.boxd[d];
                if (L > 0.0) {
                    const double dd = ti[d] - pj[d];
                    if (dd > 0.5 * L) pj[d] += (double)(float)L;
                    else if (dd < -0.5 * L) pj[d] += (double)(-(float)L);
                }
            }
            const double ddx = __dsub_rn(tx, pj[0]);
            const double ddy = __dsub_rn(ty, pj[1]);
            const double ddz = __dsub_rn(tz, pj[2]);
            const double drr = exact_dist(ddx, ddy, ddz);
            const double dh = __dmul_rn(0.5, __dadd_rn(th, A.h[j]));
            const double dq = __ddiv_rn(drr, dh);
            const double rj = A.rho[j];
            const V4<double> sv{A.vel[j], A.vel[n + j], A.vel[2 * n + j], A.m[j]};
            const V4<double> st{rj, A.P[j] / (rj * rj), A.c[j], A.bal[j]};
            hydro_pair<double, VISC, ACC, DU>(ddx, ddy, ddz, drr, dh, dq, tvx, tvy, tvz, trho, tpr, tc, tf, sv, st,
                                              A.alpha_d, A.beta_d, A.eta2_d, ax, ay, az, du, vmax);
        }
        pairs += (unsigned long long)cnt;
        if (ACC) {
            A.acc_sph[i] = ax;
            A.acc_sph[n + i] = ay;
            A.acc_sph[2 * n + i] = az;
            A.vsig[i] = vmax;
        }
        if (DU) A.dudt[i] = du;
    }
    pairs = warp_sum(pairs);
    if ((threadIdx.x & 31) == 0 && pairs) atomicAdd(&A.counters[3], pairs);
}

// ============================================================ neighbours
// Exact FP64 neighbour sets {j : q_ij <= 2} of selected particles; pass 0
// counts, pass 1 writes caller indices at the given offsets.  One warp per
// row, each lane testing its own staged candidate.
struct NArgs {
    WalkArgs w;
    const double *h;
    const int64_t *orig;
    const int64_t *rows;  // sorted indices
    int64_t nrows;
    int64_t *offsets;     // [nrows + 1]
    int64_t *out;
    int64_t cap;
    int *cursor;          // [nrows]
    int pass;
};

__global__ void __launch_bounds__(kWalkWarps * 32, kWalkMinBlocks) k_neighbours(NArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const WalkArgs &a = A.w;
    using E = V4<double>;
    WarpMem wm = carve_warp_mem(smem, a.stack_cap, sizeof(E) * 64);
    E *tile = reinterpret_cast<E *>(wm.tile);
    const int lane = lane_id();
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int64_t r = gw; r < A.nrows; r += nw) {
        const int i = (int)A.rows[r];
        int cloud = 0;
        {
            int lo = 0, hi = a.ncloud - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (a.clouds[mid].begin <= i) lo = mid;
                else hi = mid - 1;
            }
            cloud = lo;
        }
        const Cloud &cl = a.clouds[cloud];
        const int ref = __float_as_int(a.pk_pos[i].w);
        const float3 prel = rel_to(a.pk_pos[i], ref, cl.s10);
        GroupBox gb = group_box(prel, lane == 0, ref, cl.s10);
        const double tx = a.pos[i], ty = a.pos[a.n + i], tz = a.pos[2 * a.n + i];
        const double th = A.h[i];
        int found = 0;
        const Images ims = group_images(gb, (float)th + a.box_h[cl.root].w, a.box, a.periodic);
        for (int im = 0; im < 27; ++im) {
            float3 s;
            if (!image_shift(ims, im, a.box, s)) continue;
            auto load = [&](int j) {
                const double dx = __dsub_rn(tx, a.pos[j] + (double)s.x);
                const double dy = __dsub_rn(ty, a.pos[a.n + j] + (double)s.y);
                const double dz = __dsub_rn(tz, a.pos[2 * a.n + j] + (double)s.z);
                const double rr = exact_dist(dx, dy, dz);
                const double hij = __dmul_rn(0.5, __dadd_rn(th, A.h[j]));
                if (__ddiv_rn(rr, hij) <= 2.0) {
                    ++found;
                    if (A.pass == 1) {
                        const int k = atomicAdd(&A.cursor[r], 1);
                        const int64_t at = A.offsets[r] + k;
                        if (at < A.cap) A.out[at] = A.orig[j];
                        else set_status(a.status, SPH3_STATUS_LIST_OVERFLOW);
                    }
                }
                return E{};
            };
            auto interact = [&](const E *t, int ne) {
                (void)t;
                (void)ne;
            };
            auto flush = [&](int nl) {
                flush_leaves(a.range, wm.leafq, nl, tile, load, interact);
            };
            collect_leaves(a, wm, cl.root, gb, (float)th, true, s, flush);
        }
        found = warp_sum(found);
        if (A.pass == 0 && lane == 0) A.offsets[r] = found;
    }
}

// ============================================================ launchers
static WalkArgs walk_args(State &S, const Params &P, int slot) {
    WalkArgs a;
    a.groups = S.groups;
    a.ngroups_dev = S.ngroups_dev;
    a.group_cloud = S.group_cloud;
    a.clouds = S.clouds;
    a.ncloud = S.ncloud;
    a.range = S.tree.range;
    a.child = S.tree.child;
    a.box_c = S.tree.box_c;
    a.box_h = S.tree.box_h;
    a.sw = S.tree.sw;
    a.pk_pos = S.pk_pos;
    a.pos = S.pos;
    a.n = S.n;
    a.stack_cap = P.stack_cap;
    a.max_depth = S.max_level + 1;
    a.node_cap = S.tree.cap;
    a.periodic = P.periodic;
    for (int d = 0; d < 3; ++d) a.box[d] = P.box[d];
    a.work = S.work + slot;
    a.status = S.status;
    a.counters = S.counters;
    // node-visit counters: boot h / h search / density / hydro / neighbours
    static const int kVisitSlot[5] = {kCntVisitsH, kCntVisitsH, kCntVisitsDensity, kCntVisitsHydro, kCntVisitsH};
    a.visit_slot = kVisitSlot[slot];
    return a;
}

// dynamic shared memory of a walk block whose tile entries are E (double buffered)
template <typename E>
static size_t walk_smem(const Params &P) {
    return warp_mem_bytes(P.stack_cap, sizeof(E) * 64) * P.walk_warps;
}

// as walk_smem, with `extra` bytes per warp after the tile
template <typename E>
static size_t walk_smem_x(const Params &P, size_t extra) {
    return warp_mem_bytes(P.stack_cap, sizeof(E) * 64 + extra) * P.walk_warps;
}

static void allow_smem(const void *kern) {
    static std::mutex mu;
    static std::set<const void *> done;
    std::lock_guard<std::mutex> lk(mu);
    if (done.insert(kern).second)
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

template <typename Args>
static void run_walk(void (*kern)(Args), const Args &args, size_t smem, State &S, cudaStream_t st, int slot) {
    allow_smem((const void *)kern);
    cudaMemsetAsync(S.work + slot, 0, sizeof(int), st);
    // persistent grid: 32 warps' worth of blocks per SM
    kern<<<S.num_sms * (32 / S.walk_warps), S.walk_warps * 32, smem, st>>>(args);
}

void launch_boot_h(State &S, const Params &P, cudaStream_t st) {
    S.list_valid = false;
    if (S.n == 0) return;
    BootArgs A;
    A.w = walk_args(S, P, 0);
    A.h = S.h;
    A.pk_hme = S.pk_hme;
    A.k = P.n_boot;
    run_walk(k_boot_h, A, walk_smem<V4<double>>(P), S, st, 0);
}

// eps = h (the reference GPU driver's set_eps_of_gas_to_h)
__global__ void k_eps_from_h(int64_t n, const double *h, double *eps, float4 *pk_hme) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        eps[i] = h[i];
        pk_hme[i].z = (float)h[i];
    }
}

void launch_h_search(State &S, const Params &P, cudaStream_t st) {
    S.list_valid = false;  // new h: the supports change
    if (S.n == 0) return;
    HArgs A;
    A.w = walk_args(S, P, 1);
    A.h = S.h;
    A.pk_hme = S.pk_hme;
    A.nngb = S.nngb;
    A.n_ngb = P.n_ngb;
    A.tol = P.n_ngb_tol;
    A.max_iter = P.h_max_iter;
    if (P.precision == SPH3_PREC_FP64) {
        if (P.h_mode == SPH3_H_REFSTEP)
            run_walk(k_h_search<double, SPH3_H_REFSTEP>, A, walk_smem<V4<double>>(P), S, st, 1);
        else
            run_walk(k_h_search<double, SPH3_H_NEWTON>, A, walk_smem<V4<double>>(P), S, st, 1);
    } else {
        if (P.h_mode == SPH3_H_REFSTEP)
            run_walk(k_h_search<float, SPH3_H_REFSTEP>, A, walk_smem<V4<float>>(P), S, st, 1);
        else
            run_walk(k_h_search_f32_newton, A, walk_smem<V4<float>>(P), S, st, 1);
    }
    if (P.eps_from_h) {
        const int blocks = (int)std::min<int64_t>((S.n + 255) / 256, (int64_t)S.num_sms * 8);
        k_eps_from_h<<<blocks, 256, 0, st>>>(S.n, S.h, S.eps, S.pk_hme);
    }
}

void launch_density(State &S, const Params &P, bool divcurl, cudaStream_t st, bool keep_rho) {
    if (S.n == 0) return;
    DArgs A;
    A.keep_rho = keep_rho ? 1 : 0;
    A.w = walk_args(S, P, 2);
    A.pk_hme = S.pk_hme; A.pk_vel = S.pk_vel;
    A.h = S.h; A.m = S.m; A.vel = S.vel; A.u = S.u;
    A.rho = S.rho; A.P = S.P; A.c = S.c; A.divV = S.divV; A.curlV = S.curlV; A.bal = S.bal;
    A.pk_thm = S.pk_thm;
    A.gamma = P.gamma;
    A.list = S.list_cap > 0 ? S.list : nullptr;
    A.nlist = S.nlist;
    A.list_cap = S.list_cap;
    A.ovf = S.ovf;
    if (A.list) cudaMemsetAsync(S.ovf, 0, sizeof(int), st);
    S.list_valid = A.list != nullptr;
    if (P.precision == SPH3_PREC_FP64) {
        if (divcurl) run_walk(k_density<double, true>, A, walk_smem_x<DE<double, true>>(P, kDensityExtraBytes), S, st, 2);
        else run_walk(k_density<double, false>, A, walk_smem_x<DE<double, false>>(P, kDensityExtraBytes), S, st, 2);
    } else {
        if (divcurl) run_walk(k_density<float, true>, A, walk_smem_x<DE<float, true>>(P, kDensityExtraBytes), S, st, 2);
        else run_walk(k_density_f32, A, walk_smem_x<DE<float, false>>(P, kDensityExtraBytes), S, st, 2);
    }
}

template <typename R, int V>
static void hydro_dispatch(const YArgs &A, bool acc, bool du, const Params &P, State &S, cudaStream_t st) {
    const size_t sm = walk_smem<YE<R>>(P);
    if (acc && du) run_walk(k_hydro<R, V, true, true>, A, sm, S, st, 3);
    else if (acc) run_walk(k_hydro<R, V, true, false>, A, sm, S, st, 3);
    else run_walk(k_hydro<R, V, false, true>, A, sm, S, st, 3);
}

template <int V>
static void list_dispatch(const LArgs &L, bool fp64, bool acc, bool du, int blocks, cudaStream_t st) {
    if (fp64) {
        if (acc && du) k_hydro_list_f64<V, true, true><<<blocks, 256, 0, st>>>(L);
        else if (acc) k_hydro_list_f64<V, true, false><<<blocks, 256, 0, st>>>(L);
        else k_hydro_list_f64<V, false, true><<<blocks, 256, 0, st>>>(L);
        return;
    }
    // 128-thread blocks at <= 72 registers: 7 blocks (28 warps) per SM
    const int b128 = (int)std::min<int64_t>((L.n + 127) / 128, (int64_t)blocks * 2);
    if (acc && du) k_hydro_list<V, true, true><<<b128, 128, 0, st>>>(L);
    else if (acc) k_hydro_list<V, true, false><<<b128, 128, 0, st>>>(L);
    else k_hydro_list<V, false, true><<<b128, 128, 0, st>>>(L);
}

void launch_hydro(State &S, const Params &P, bool want_acc, bool want_dudt, cudaStream_t st) {
    if (S.n == 0 || (!want_acc && !want_dudt)) return;
    YArgs A;
    A.w = walk_args(S, P, 3);
    A.pk_hme = S.pk_hme; A.pk_vel = S.pk_vel; A.pk_thm = S.pk_thm;
    A.h = S.h; A.m = S.m; A.vel = S.vel; A.rho = S.rho; A.P = S.P; A.c = S.c; A.bal = S.bal;
    A.acc_sph = S.acc_sph; A.dudt = S.dudt; A.vsig = S.vsig;
    A.alpha = P.alpha; A.beta = P.beta; A.eta = P.eta;
    A.nlist = S.nlist;
    A.list_cap = S.list_cap;
    A.only_overflow = 0;
    A.ovf = S.ovf;
    if (S.list_valid) {
        // the list pass, then a walk for the particles whose lists overflowed
        const bool fp64 = P.precision == SPH3_PREC_FP64;
        LArgs L;
        L.list = S.list; L.nlist = S.nlist; L.list_cap = S.list_cap;
        L.pk_pos = S.pk_pos; L.pk_hme = S.pk_hme; L.pk_vel = S.pk_vel; L.pk_thm = S.pk_thm;
        L.key = S.key; L.cloud_shift = 3 * S.max_level; L.clouds = S.clouds;
        L.n = S.n;
        L.periodic = P.periodic;
        for (int d = 0; d < 3; ++d) L.box[d] = (float)P.box[d];
        L.acc_sph = S.acc_sph; L.dudt = S.dudt; L.vsig = S.vsig;
        L.alpha = (float)P.alpha; L.beta = (float)P.beta; L.eta2 = (float)(P.eta * P.eta);
        L.counters = S.counters;
        L.hrec = S.hrec;
        L.pos = S.pos; L.vel = S.vel; L.h = S.h; L.m = S.m; L.rho = S.rho; L.P = S.P; L.c = S.c; L.bal = S.bal;
        for (int d = 0; d < 3; ++d) L.boxd[d] = P.box[d];
        L.alpha_d = P.alpha; L.beta_d = P.beta; L.eta2_d = P.eta * P.eta;
        const int blocks = (int)std::min<int64_t>((S.n + 255) / 256, (int64_t)S.num_sms * 16);
        if (!fp64) k_pack_hrec<<<blocks, 256, 0, st>>>(L);
        if (P.visc == SPH3_VISC_MG83) list_dispatch<SPH3_VISC_MG83>(L, fp64, want_acc, want_dudt, blocks, st);
        else if (P.visc == SPH3_VISC_BALSARA)
            list_dispatch<SPH3_VISC_BALSARA>(L, fp64, want_acc, want_dudt, blocks, st);
        else list_dispatch<SPH3_VISC_SIGNAL>(L, fp64, want_acc, want_dudt, blocks, st);
        A.only_overflow = 1;
    }
    if (P.precision == SPH3_PREC_FP64) {
        if (P.visc == SPH3_VISC_MG83) hydro_dispatch<double, SPH3_VISC_MG83>(A, want_acc, want_dudt, P, S, st);
        else if (P.visc == SPH3_VISC_BALSARA) hydro_dispatch<double, SPH3_VISC_BALSARA>(A, want_acc, want_dudt, P, S, st);
        else hydro_dispatch<double, SPH3_VISC_SIGNAL>(A, want_acc, want_dudt, P, S, st);
    } else {
        if (P.visc == SPH3_VISC_MG83) hydro_dispatch<float, SPH3_VISC_MG83>(A, want_acc, want_dudt, P, S, st);
        else if (P.visc == SPH3_VISC_BALSARA) hydro_dispatch<float, SPH3_VISC_BALSARA>(A, want_acc, want_dudt, P, S, st);
        else hydro_dispatch<float, SPH3_VISC_SIGNAL>(A, want_acc, want_dudt, P, S, st);
    }
}

// P and c from the stored rho and u (getPressure, sph_serial.py:116), plus
// the Balsara factor from the stored div/curl (shear.py:212-213)
__global__ void k_eos(int64_t n, double gamma, const double *rho, const double *u, const double *divV,
                      const double *curlV, const double *h, double *P, double *c, double *bal,
                      float4 *pk_thm) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double r = rho[i];
        const double p = (gamma - 1.0) * r * u[i];
        const double cc = sqrt(gamma * (gamma - 1.0) * u[i]);
        P[i] = p;
        c[i] = cc;
        const double f = divV[i] / (divV[i] + curlV[i] + 0.0001 * cc / h[i]);
        bal[i] = f;
        pk_thm[i] = make_float4((float)r, (float)(r > 0 ? p / (r * r) : 0.0), (float)cc, (float)f);
    }
}

void launch_eos(State &S, const Params &P, cudaStream_t st) {
    if (S.n == 0) return;
    int blocks = (int)std::min<int64_t>((S.n + 255) / 256, (int64_t)S.num_sms * 8);
    k_eos<<<blocks, 256, 0, st>>>(S.n, P.gamma, S.rho, S.u, S.divV, S.curlV, S.h, S.P, S.c, S.bal, S.pk_thm);
}

__global__ void k_balsara(int64_t n, const double *divV, const double *curlV, const double *c,
                          const double *h, double *bal, float4 *pk_thm) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double f = divV[i] / (divV[i] + curlV[i] + 0.0001 * c[i] / h[i]);
        bal[i] = f;
        pk_thm[i].w = (float)f;
    }
}

void launch_balsara(State &S, cudaStream_t st) {
    if (S.n == 0) return;
    int blocks = (int)std::min<int64_t>((S.n + 255) / 256, (int64_t)S.num_sms * 8);
    k_balsara<<<blocks, 256, 0, st>>>(S.n, S.divV, S.curlV, S.c, S.h, S.bal, S.pk_thm);
}

int launch_neighbours(State &S, const Params &P, const int64_t *rows_sorted_dev, int64_t nrows,
                      int64_t *offsets_dev, int64_t *idx_dev, int64_t cap, cudaStream_t st) {
    if (nrows == 0) return 0;
    NArgs A;
    A.w = walk_args(S, P, 4);
    A.h = S.h;
    A.orig = S.orig;
    A.rows = rows_sorted_dev;
    A.nrows = nrows;
    A.offsets = offsets_dev;
    A.out = idx_dev;
    A.cap = cap;
    A.cursor = nullptr;
    const size_t sm = walk_smem<V4<double>>(P);
    allow_smem((const void *)k_neighbours);
    int blocks = (int)std::min<int64_t>((nrows + S.walk_warps - 1) / S.walk_warps, (int64_t)S.num_sms * 8);
    // pass 0: counts into offsets[0..nrows)
    A.pass = 0;
    k_neighbours<<<blocks, S.walk_warps * 32, sm, st>>>(A);
    // exclusive scan on the host (few rows)
    std::vector<int64_t> hv(nrows + 1);
    cudaMemcpyAsync(hv.data(), offsets_dev, sizeof(int64_t) * nrows, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    int64_t run = 0;
    for (int64_t r = 0; r < nrows; ++r) {
        const int64_t v = hv[r];
        hv[r] = run;
        run += v;
    }
    hv[nrows] = run;
    cudaMemcpyAsync(offsets_dev, hv.data(), sizeof(int64_t) * (nrows + 1), cudaMemcpyHostToDevice, st);
    int *cursor = nullptr;
    cudaMallocAsync(&cursor, sizeof(int) * nrows, st);
    cudaMemsetAsync(cursor, 0, sizeof(int) * nrows, st);
    A.cursor = cursor;
    A.pass = 1;
    k_neighbours<<<blocks, S.walk_warps * 32, sm, st>>>(A);
    cudaFreeAsync(cursor, st);
    cudaStreamSynchronize(st);
    return 0;
}

}  // namespace sph3

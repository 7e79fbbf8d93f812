// Barnes-Hut gravity with spline softening, and the FP64 direct sum.
//
// One warp per compact group (<= 32 particles) walks the octree once.  A node
// is accepted as a multipole for the whole group when the distance d from its
// centre of mass to the group's bounding box satisfies
//     d > s / theta + delta          (s: node bbox side, delta: |com - bbox centre|)
//     d > b_max + eps_max_node + eps_max_group   (outside every softening kernel)
// otherwise a leaf is opened into particle-particle terms with the reference's
// softened kernel (sph_code/libsx.py:640-652 force, :609-616 potential) and an
// internal node is opened into its children.  theta = 0 never accepts a node,
// so the walk becomes the exact direct sum.  Multipoles are monopole +
// traceless quadrupole about the centre of mass.  Accepted nodes and opened
// leaves are queued and streamed through double-buffered shared-memory tiles
// of 4-wide entries (broadcast reads).
#include <cfloat>
#include <mutex>
#include <set>

#include "sph3_walk.cuh"

namespace sph3 {

struct GArgs {
    const int2 *groups;
    const int *ngroups_dev;
    const int *group_cloud;
    const Cloud *clouds;
    const int2 *range;
    const int2 *child;
    const float4 *com_c;
    const float4 *mono;
    const float4 *gw;  // walk records
    const float4 *quad4;
    const float *quad1;
    const double *tcom;   // FP64 node com [3][cap]
    const double *tmass;
    const double *tquad;  // [6][cap]
    int cap;
    const float4 *pk_pos;
    const float4 *pk_hme;  // {h, m, eps}
    const double *pos, *m, *eps;
    int64_t n;
    double G;
    int quad;
    int stack_cap, max_depth;
    double *acc_g, *phi;
    int *work;
    unsigned *status;
    unsigned long long *counters;
};

// node entry: a = {com (group frame), mass}, b = {qxx, qxy, qxz, qyy}, qyz
template <typename R>
struct GN {
    V4<R> a, b;
    R qyz;
};

// particle entry: p = {pos (group frame), mass}, e = softening length
template <typename R>
struct GP {
    V4<R> p;
    R e;
};

template <typename R>
struct GTile {
    GN<R> nd[64];
    GP<R> pt[64];
    int nodeq[kNodeQ];
};

__device__ __forceinline__ float rsq(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsq(double x) { return 1.0 / sqrt(x); }

template <typename R>
__device__ __forceinline__ void spline_force(R r2, R dx, R dy, R dz, R mj, R epsij, R &ax, R &ay,
                                             R &az, R &ph) {
    // r2 > 0 here
    const R rinv = rsq(r2);
    const R r = r2 * rinv;
    const R rinv3 = rinv * rinv * rinv;
    R fk, pk;
    if (r >= (R)2 * epsij) {
        fk = rinv3;
        pk = rinv;
    } else {
        const R ie = (R)1 / epsij;
        const R q = r * ie;
        const R q2 = q * q, q3 = q2 * q;
        if (q <= (R)1) {
            fk = ie * ie * ie * ((R)(4.0 / 3.0) - (R)(6.0 / 5.0) * q2 + (R)0.5 * q3);
            pk = (R)-2 * ie * ((R)(1.0 / 3.0) * q2 - (R)(3.0 / 20.0) * q2 * q2 + (R)(1.0 / 20.0) * q2 * q3) +
                 (R)(7.0 / 5.0) * ie;
        } else {
            const R q4 = q2 * q2;
            fk = rinv3 * ((R)(-1.0 / 15.0) + (R)(8.0 / 3.0) * q3 - (R)3 * q4 + (R)(6.0 / 5.0) * q4 * q -
                          (R)(1.0 / 6.0) * q3 * q3);
            pk = (R)(-1.0 / 15.0) * rinv - ie * ((R)(4.0 / 3.0) * q2 - q3 + (R)(3.0 / 10.0) * q4 - (R)(1.0 / 30.0) * q4 * q) +
                 (R)(8.0 / 5.0) * ie;
        }
    }
    const R mf = mj * fk;
    ax -= mf * dx;
    ay -= mf * dy;
    az -= mf * dz;
    ph -= mj * pk;
}

// The walk of one group, shared by both precisions.  Pops up to 32 nodes per
// iteration, accepts a node as a multipole when the group's bbox lies outside
// both its opening radius and its softening reach, queues accepted nodes
// (nodeq) and opened leaves, and hands full queues to flush_nodes(count) /
// flush_leaves(count) / flush_far(count).  An opened leaf that still passes
// the softening test (it fails only the opening radius) goes to its own
// queue (farq): every pair it gives lies outside the softened kernel
// (r >= eps_i + eps_j), so its flush needs no spline.  Others go to
// wm.leafq.  Without FAR_QUEUE every opened leaf goes to wm.leafq.  Returns
// the iteration count.
template <bool FAR_QUEUE, class FlushNodes, class FlushLeaves, class FlushFar>
__device__ __forceinline__ int grav_walk(const GArgs &A, const WarpMem &wm, int *nodeq, int *farq, const Cloud &cl,
                                         int ref, const GroupBox &gb, float eps_g, FlushNodes &flush_nodes,
                                         FlushLeaves &flush_leaves_fn, FlushFar &flush_far,
                                         unsigned long long &visits) {
    const int lane = lane_id();
    int top = 1;
    if (lane == 0) wm.stack[0] = cl.root;
    __syncwarp();
    int nleaf = 0, nnode = 0, nfar = 0;
    int guard = 0;
    // each node is popped at most once; the bound only trips on a corrupted tree
    for (; top > 0; ++guard) {
        if (guard > A.cap) {
            if (lane == 0) set_status(A.status, SPH3_STATUS_STACK_OVERFLOW);
            break;
        }
        const int p = pop_width(top, A.stack_cap, A.max_depth);
        visits += p;
        int node = -1;
        if (lane < p) node = wm.stack[top - 1 - lane];
        __syncwarp();
        top -= p;
        bool take_leaf = false, take_node = false, take_far = false;
        int nch = 0, cf = 0;
        if (node >= 0) {
            const float4 w0 = A.gw[2 * node], w1 = A.gw[2 * node + 1];  // one record, one round trip
            const int chy = __float_as_int(w1.w);
            if (chy >= 0) {
                const float3 c = rel_to(w0, ref, cl.s10);
                const float d2 = point_gap2(gb, c);
                const float rs = w1.y + eps_g;
                if (d2 > w1.x * w1.x && d2 > rs * rs) {
                    take_node = true;
                } else {
                    const int k = chy & 255;
                    if (k == 0) {
                        if (FAR_QUEUE && d2 > rs * rs) take_far = true;
                        else take_leaf = true;
                    } else {
                        nch = k;
                        cf = __float_as_int(w1.z);
                    }
                }
            }
        }
        const unsigned nb = __ballot_sync(kFull, take_node);
        if (take_node) nodeq[nnode + __popc(nb & lanemask_lt())] = node;
        nnode += __popc(nb);
        const unsigned lb = __ballot_sync(kFull, take_leaf);
        if (take_leaf) wm.leafq[nleaf + __popc(lb & lanemask_lt())] = node;
        nleaf += __popc(lb);
        if (FAR_QUEUE) {
            const unsigned fb = __ballot_sync(kFull, take_far);
            if (take_far) farq[nfar + __popc(fb & lanemask_lt())] = node;
            nfar += __popc(fb);
        }
        top = push_children(wm.stack, top, A.stack_cap, nch, cf, A.status);
        __syncwarp();
        if (nnode > kNodeQ - 32) {
            flush_nodes(nnode);
            nnode = 0;
        }
        if (nleaf > kLeafQ - 32) {
            flush_leaves_fn(nleaf);
            nleaf = 0;
        }
        if (FAR_QUEUE && nfar > kLeafQ - 32) {
            flush_far(nfar);
            nfar = 0;
        }
    }
    __syncwarp();
    if (nnode > 0) flush_nodes(nnode);
    if (nleaf > 0) flush_leaves_fn(nleaf);
    if (FAR_QUEUE && nfar > 0) flush_far(nfar);
    return guard;
}

// FP64 path: one target per lane, AoS tiles of the FP64 masters.  PHI: also
// the potential (only the node terms are skipped without it; a near pair's
// softened potential comes with its force).
template <bool QUAD, bool PHI>
__global__ void __launch_bounds__(kWalkWarps * 32, kWalkMinBlocks) k_gravity_f64(GArgs A) {
    using R = double;
    extern __shared__ __align__(16) unsigned char smem[];
    WarpMem wm = carve_warp_mem(smem, A.stack_cap, sizeof(GTile<R>));
    GTile<R> &tile = *reinterpret_cast<GTile<R> *>(wm.tile);
    const int lane = lane_id();
    unsigned long long n_node = 0, n_part = 0, n_grp = 0;
    for (int g = next_group(A.work, A.status); g < *A.ngroups_dev; g = next_group(A.work, A.status)) {
        const int2 gr = A.groups[g];
        const Cloud &cl = A.clouds[A.group_cloud[g]];
        const int ref = __float_as_int(A.pk_pos[gr.x].w);
        ++n_grp;
        const bool active = lane < gr.y;
        const int i = gr.x + (active ? lane : 0);
        const float3 prel = rel_to(A.pk_pos[i], ref, cl.s10);
        GroupBox gb = group_box(prel, active, ref, cl.s10);
        const R tx = A.pos[i], ty = A.pos[A.n + i], tz = A.pos[2 * A.n + i], te = A.eps[i];
        const float eps_g = warp_max(active ? (float)te : 0.f);
        R ax = 0, ay = 0, az = 0, ph = 0;

        auto load_node = [&](int nd) {
            GN<R> en;
            en.a.x = A.tcom[nd];
            en.a.y = A.tcom[A.cap + nd];
            en.a.z = A.tcom[2 * A.cap + nd];
            en.a.w = A.tmass[nd];
            if (QUAD) {
                en.b.x = A.tquad[nd];
                en.b.y = A.tquad[A.cap + nd];
                en.b.z = A.tquad[2 * A.cap + nd];
                en.b.w = A.tquad[3 * A.cap + nd];
                en.qyz = A.tquad[4 * A.cap + nd];
            }
            return en;
        };
        auto node_interact = [&](const GN<R> *t, int ne) {
            if (!active) return;
            n_node += ne;
            for (int e = 0; e < ne; ++e) {
                const V4<R> a4 = t[e].a;
                const R dx = tx - a4.x, dy = ty - a4.y, dz = tz - a4.z;
                const R r2 = dx * dx + dy * dy + dz * dz;
                const R rinv = rsq(r2);
                const R rinv2 = rinv * rinv;
                const R M = a4.w;
                const R mr3 = M * rinv * rinv2;
                ax -= mr3 * dx;
                ay -= mr3 * dy;
                az -= mr3 * dz;
                if (PHI) ph -= M * rinv;
                if (QUAD) {
                    const V4<R> b4 = t[e].b;
                    const R qyz = t[e].qyz;
                    const R qzz = -b4.x - b4.w;
                    const R Qx = b4.x * dx + b4.y * dy + b4.z * dz;
                    const R Qy = b4.y * dx + b4.w * dy + qyz * dz;
                    const R Qz = b4.z * dx + qyz * dy + qzz * dz;
                    const R rQr = dx * Qx + dy * Qy + dz * Qz;
                    const R rinv5 = rinv2 * rinv2 * rinv;
                    const R tq = (R)2.5 * rQr * rinv5 * rinv2;
                    ax += Qx * rinv5 - tq * dx;
                    ay += Qy * rinv5 - tq * dy;
                    az += Qz * rinv5 - tq * dz;
                    if (PHI) ph -= (R)0.5 * rQr * rinv5;
                }
            }
        };
        auto flush_nodes = [&](int nq) {
            GN<R> cur;
            bool have = lane < nq;
            if (have) cur = load_node(tile.nodeq[lane]);
            int buf = 0;
            for (int base = 0; base < nq; base += 32) {
                if (have) tile.nd[buf * 32 + lane] = cur;
                __syncwarp();
                have = base + 32 + lane < nq;
                if (have) cur = load_node(tile.nodeq[base + 32 + lane]);
                node_interact(tile.nd + buf * 32, min(32, nq - base));
                buf ^= 1;
            }
            __syncwarp();
        };
        auto load_part = [&](int j) {
            GP<R> en;
            en.p.x = A.pos[j];
            en.p.y = A.pos[A.n + j];
            en.p.z = A.pos[2 * A.n + j];
            en.p.w = A.m[j];
            en.e = A.eps[j];
            return en;
        };
        auto part_interact = [&](const GP<R> *t, int ne) {
            if (!active) return;
            n_part += ne;
            for (int e = 0; e < ne; ++e) {
                const V4<R> p4 = t[e].p;
                const R dx = tx - p4.x, dy = ty - p4.y, dz = tz - p4.z;
                const R r2 = dx * dx + dy * dy + dz * dz;
                if (r2 > (R)0) spline_force<R>(r2, dx, dy, dz, p4.w, (R)0.5 * (te + t[e].e), ax, ay, az, ph);
            }
        };
        auto flush_leaves_fn = [&](int nl) {
            flush_leaves(A.range, wm.leafq, nl, tile.pt, load_part, part_interact);
        };
        unsigned long long visits = 0;
        // one leaf queue: the FP64 pair loop has no separate spline branch to skip
        const int guard = grav_walk<false>(A, wm, tile.nodeq, nullptr, cl, ref, gb, eps_g, flush_nodes,
                                           flush_leaves_fn, flush_leaves_fn, visits);
        if (lane == 0) {  // walk statistics
            atomicAdd(&A.counters[kCntVisitsGravity], visits);
            atomicMax(&A.counters[kCntWalkMaxIter], (unsigned long long)guard);
        }
        if (active) {
            A.acc_g[i] = A.G * ax;
            A.acc_g[A.n + i] = A.G * ay;
            A.acc_g[2 * A.n + i] = A.G * az;
            if (PHI) A.phi[i] = A.G * ph;
        }
    }
    n_node = warp_sum(n_node);
    n_part = warp_sum(n_part);
    if (lane == 0) {
        atomicAdd(&A.counters[0], n_node);
        atomicAdd(&A.counters[1], n_part);
        atomicAdd(&A.counters[kCntGravGroups], n_grp);
    }
}

// ------------------------------------------------------------ FP32 path
// Mixed path with Blackwell's packed FP32 pipe (FFMA2 / FADD2 / FMUL2): each
// lane runs its target against two tile entries per instruction, so the
// issue slots per interaction halve.  Tiles are stored as pairs: one 128-bit
// shared load yields {x0, x1, y0, y1}, i.e. two ready packed operands.
// Every tile slot is written (padding: zero mass at 1e18, which contributes
// exactly zero), so whole pairs run without bounds checks.
//
// Signs: with d = source - target the monopole pulls along +d.  Quadrupoles
// are staged negated (Qn = -Q); with w = d.Qn.d the acceleration is
//   a += (M r^-3 - 2.5 w r^-7) d + (Qn d) r^-5
// and the potential is -P with P = M r^-1 - 0.5 w r^-5, the same terms as
// the FP64 path written for the other sign of d.
//
// Small groups split the warp: a group of <= 16 (<= 8) targets runs 2 (4)
// lanes per target, each lane over every 2nd (4th) entry pair, and the
// copies are summed with shuffles, so fewer lanes idle.
struct GTileF {
    union {  // the node and particle flushes never overlap
        struct {
            float4 na[2][16], nb[2][16], nc[2][16], nd[2][16], ne[2][16];  // node pairs, two buffers
        };
        struct {
            float4 pa[2][16], pb[2][16];  // particle pairs
            float2 pe[2][16];
        };
    };
    int nodeq[kNodeQ];
    int farq[kLeafQ];  // opened leaves outside every softening kernel
};

struct NodeF {
    float x, y, z, m, qxx, qxy, qxz, qyy, qyz;
};

struct PartF {
    float x, y, z, m, e;
};

constexpr float kPadFar = 1e18f;

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ void put2(float4 &dst, int h, float a, float b) {
    float *p = reinterpret_cast<float *>(&dst);
    p[h] = a;
    p[2 + h] = b;
}

// The reference's softened kernel inside its support (r < 2 eps), for both
// halves of a pair at once: the two polynomial pieces (q <= 1 and q <= 2,
// written in Horner form) are evaluated packed and selected per half, so
// lanes never diverge; halves outside the support keep the far values
// (fk = 1/r^3, pk = 1/r), and r2 = 0 (a particle and itself, or coincident
// particles) contributes nothing.  Same pieces as the FP64 path's
// spline_force (sph_code/libsx.py:640-652 force, :609-616 potential).
__device__ __forceinline__ void spline_near2(float2 r2, float2 r, float2 rinv, float2 e, float2 &fk, float2 &pk) {
    const float2 ie = make_float2(__fdividef(1.f, e.x), __fdividef(1.f, e.y));
    const float2 q = __fmul2_rn(r, ie);
    const float2 q2 = __fmul2_rn(q, q);
    const float2 q3 = __fmul2_rn(q2, q);
    const float2 ie3 = __fmul2_rn(__fmul2_rn(ie, ie), ie);
    // q <= 1: fk = ie^3 (4/3 + q^2 (-6/5 + q/2)), pk = ie (7/5 + q^2 (-2/3 + q^2 (3/10 - q/10)))
    float2 t = __ffma2_rn(q, f2(0.5f), f2(-1.2f));
    t = __ffma2_rn(q2, t, f2(4.f / 3.f));
    const float2 fk1 = __fmul2_rn(ie3, t);
    float2 u = __ffma2_rn(q, f2(-0.1f), f2(0.3f));
    u = __ffma2_rn(q2, u, f2(-2.f / 3.f));
    u = __ffma2_rn(q2, u, f2(1.4f));
    const float2 pk1 = __fmul2_rn(ie, u);
    // 1 < q <= 2: fk = r^-3 (-1/15 + q^3 (8/3 + q (-3 + q (6/5 - q/6)))),
    //             pk = -r^-1/15 + ie (8/5 - q^2 (4/3 + q (-1 + q (3/10 - q/30))))
    float2 v = __ffma2_rn(q, f2(-1.f / 6.f), f2(1.2f));
    v = __ffma2_rn(q, v, f2(-3.f));
    v = __ffma2_rn(q, v, f2(8.f / 3.f));
    v = __ffma2_rn(q3, v, f2(-1.f / 15.f));
    const float2 fk2 = __fmul2_rn(fk, v);  // fk holds r^-3 on entry
    float2 w = __ffma2_rn(q, f2(-1.f / 30.f), f2(0.3f));
    w = __ffma2_rn(q, w, f2(-1.f));
    w = __ffma2_rn(q, w, f2(4.f / 3.f));
    const float2 x = __ffma2_rn(__fmul2_rn(q2, f2(-1.f)), w, f2(1.6f));
    const float2 pk2 = __ffma2_rn(ie, x, __fmul2_rn(rinv, f2(-1.f / 15.f)));
    // select per half
    if (!(r.x >= 2.f * e.x)) {
        const bool z = !(r2.x > 0.f);
        fk.x = z ? 0.f : (q.x <= 1.f ? fk1.x : fk2.x);
        pk.x = z ? 0.f : (q.x <= 1.f ? pk1.x : pk2.x);
    }
    if (!(r.y >= 2.f * e.y)) {
        const bool z = !(r2.y > 0.f);
        fk.y = z ? 0.f : (q.y <= 1.f ? fk1.y : fk2.y);
        pk.y = z ? 0.f : (q.y <= 1.f ? pk1.y : pk2.y);
    }
}

// At most 72 registers: 28 resident warps per SM (registers are granted in
// steps of 8 per thread, so 73 would already cost a block of four warps).
// The walk part is latency-bound and wants the residency.
constexpr int kGravMaxRegs = 72;

template <bool QUAD, bool PHI>
__global__ void __maxnreg__(kGravMaxRegs) k_gravity_f32(GArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    WarpMem wm = carve_warp_mem(smem, A.stack_cap, sizeof(GTileF));
    GTileF &tile = *reinterpret_cast<GTileF *>(wm.tile);
    const int lane = lane_id();
    unsigned long long n_node = 0, n_part = 0, n_grp = 0;
    for (int g = next_group(A.work, A.status); g < *A.ngroups_dev; g = next_group(A.work, A.status)) {
        const int2 gr = A.groups[g];
        const Cloud &cl = A.clouds[A.group_cloud[g]];
        const int ref = __float_as_int(A.pk_pos[gr.x].w);
        ++n_grp;
        const int split = gr.y <= 8 ? 4 : (gr.y <= 16 ? 2 : 1);
        const int gw = 32 / split;  // lanes per copy of the group
        const int slot = lane & (gw - 1), cp = lane / gw;
        const bool active = slot < gr.y;
        const bool lead = active && cp == 0;
        const int i = gr.x + (active ? slot : 0);
        const float3 prel = rel_to(A.pk_pos[i], ref, cl.s10);
        GroupBox gb = group_box(prel, active, ref, cl.s10);
        const float te = A.pk_hme[i].z;
        const float eps_g = warp_max(active ? te : 0.f);
        const float2 ntx = f2(-prel.x), nty = f2(-prel.y), ntz = f2(-prel.z), hte = f2(0.5f * te);
        float2 ax = f2(0.f), ay = f2(0.f), az = f2(0.f), pp = f2(0.f);

        // ---- accepted multipoles
        auto load_node = [&](int nd) {
            NodeF en;
            const float3 c = rel_to(A.com_c[nd], ref, cl.s10);
            en.x = c.x;
            en.y = c.y;
            en.z = c.z;
            en.m = A.mono[nd].x;
            if (QUAD) {
                const float4 q = A.quad4[nd];
                en.qxx = q.x;
                en.qxy = q.y;
                en.qxz = q.z;
                en.qyy = q.w;
                en.qyz = A.quad1[nd];
            }
            return en;
        };
        auto store_node = [&](int buf, int s, const NodeF &e, bool have) {
            const int p = s >> 1, h = s & 1;
            put2(tile.na[buf][p], h, have ? e.x : kPadFar, have ? e.y : kPadFar);
            put2(tile.nb[buf][p], h, have ? e.z : kPadFar, have ? e.m : 0.f);
            if (QUAD) {
                put2(tile.nc[buf][p], h, have ? -e.qxx : 0.f, have ? -e.qxy : 0.f);
                put2(tile.nd[buf][p], h, have ? -e.qxz : 0.f, have ? -e.qyy : 0.f);
                put2(tile.ne[buf][p], h, have ? -e.qyz : 0.f, have ? e.qxx + e.qyy : 0.f);  // -qzz
            }
        };
        auto node_interact = [&](int buf, int ne) {
            if (lead) n_node += ne;
            const int np = (ne + 1) >> 1;
            for (int pb = 0; pb < np; pb += split) {
                const int p = pb + cp;  // < 16; pairs past np are padding
                const float4 a4 = tile.na[buf][p], b4 = tile.nb[buf][p];
                const float2 dx = __fadd2_rn(lo2(a4), ntx), dy = __fadd2_rn(hi2(a4), nty),
                             dz = __fadd2_rn(lo2(b4), ntz);
                const float2 M = hi2(b4);
                float2 r2 = __fmul2_rn(dx, dx);
                r2 = __ffma2_rn(dy, dy, r2);
                r2 = __ffma2_rn(dz, dz, r2);
                const float2 rinv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
                const float2 rinv2 = __fmul2_rn(rinv, rinv);
                const float2 rinv3 = __fmul2_rn(rinv2, rinv);
                float2 s = __fmul2_rn(M, rinv3);
                if (PHI) pp = __ffma2_rn(M, rinv, pp);
                if (QUAD) {
                    const float4 c4 = tile.nc[buf][p], d4 = tile.nd[buf][p], e4 = tile.ne[buf][p];
                    float2 qx = __fmul2_rn(lo2(c4), dx);  // Qn d
                    qx = __ffma2_rn(hi2(c4), dy, qx);
                    qx = __ffma2_rn(lo2(d4), dz, qx);
                    float2 qy = __fmul2_rn(hi2(c4), dx);
                    qy = __ffma2_rn(hi2(d4), dy, qy);
                    qy = __ffma2_rn(lo2(e4), dz, qy);
                    float2 qz = __fmul2_rn(lo2(d4), dx);
                    qz = __ffma2_rn(lo2(e4), dy, qz);
                    qz = __ffma2_rn(hi2(e4), dz, qz);
                    float2 w = __fmul2_rn(dx, qx);  // d.Qn.d
                    w = __ffma2_rn(dy, qy, w);
                    w = __ffma2_rn(dz, qz, w);
                    const float2 rinv5 = __fmul2_rn(rinv3, rinv2);
                    const float2 rinv7 = __fmul2_rn(rinv5, rinv2);
                    s = __ffma2_rn(__fmul2_rn(w, f2(-2.5f)), rinv7, s);
                    if (PHI) pp = __ffma2_rn(__fmul2_rn(w, f2(-0.5f)), rinv5, pp);
                    ax = __ffma2_rn(qx, rinv5, ax);
                    ay = __ffma2_rn(qy, rinv5, ay);
                    az = __ffma2_rn(qz, rinv5, az);
                }
                ax = __ffma2_rn(s, dx, ax);
                ay = __ffma2_rn(s, dy, ay);
                az = __ffma2_rn(s, dz, az);
            }
        };
        auto flush_nodes = [&](int nq) {
            NodeF cur{};
            bool have = lane < nq;
            if (have) cur = load_node(tile.nodeq[lane]);
            int buf = 0;
            for (int base = 0; base < nq; base += 32) {
                store_node(buf, lane, cur, have);
                __syncwarp();
                have = base + 32 + lane < nq;
                if (have) cur = load_node(tile.nodeq[base + 32 + lane]);
                node_interact(buf, min(32, nq - base));
                buf ^= 1;
            }
            __syncwarp();
        };

        // ---- opened leaves: particle-particle terms
        auto load_part = [&](int j) {
            PartF en;
            const float3 p = rel_to(A.pk_pos[j], ref, cl.s10);
            const float4 hm = A.pk_hme[j];
            en.x = p.x;
            en.y = p.y;
            en.z = p.z;
            en.m = hm.y;
            en.e = hm.z;
            return en;
        };
        auto store_part = [&](int buf, int s, const PartF &e, bool have) {
            const int p = s >> 1, h = s & 1;
            put2(tile.pa[buf][p], h, have ? e.x : kPadFar, have ? e.y : kPadFar);
            put2(tile.pb[buf][p], h, have ? e.z : kPadFar, have ? e.m : 0.f);
            reinterpret_cast<float *>(&tile.pe[buf][p])[h] = have ? e.e : 1.f;
        };
        auto part_interact = [&](int buf, int ne) {
            if (lead) n_part += ne;
            const int np = (ne + 1) >> 1;
            for (int pb = 0; pb < np; pb += split) {
                const int p = pb + cp;
                const float4 a4 = tile.pa[buf][p], b4 = tile.pb[buf][p];
                const float2 e2 = tile.pe[buf][p];
                const float2 dx = __fadd2_rn(lo2(a4), ntx), dy = __fadd2_rn(hi2(a4), nty),
                             dz = __fadd2_rn(lo2(b4), ntz);
                const float2 m = hi2(b4);
                float2 r2 = __fmul2_rn(dx, dx);
                r2 = __ffma2_rn(dy, dy, r2);
                r2 = __ffma2_rn(dz, dz, r2);
                const float2 rinv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
                const float2 r = __fmul2_rn(r2, rinv);
                const float2 eij = __ffma2_rn(e2, f2(0.5f), hte);
                float2 fk = __fmul2_rn(__fmul2_rn(rinv, rinv), rinv);
                float2 pk = rinv;
                // NaN-safe: r2 = 0 gives r = NaN, which lands in the near branch
                const bool near = active && (!(r.x >= 2.f * eij.x) || !(r.y >= 2.f * eij.y));
                if (__any_sync(kFull, near)) spline_near2(r2, r, rinv, eij, fk, pk);
                const float2 mf = __fmul2_rn(m, fk);
                ax = __ffma2_rn(mf, dx, ax);
                ay = __ffma2_rn(mf, dy, ay);
                az = __ffma2_rn(mf, dz, az);
                if (PHI) pp = __ffma2_rn(m, pk, pp);
            }
        };
        auto flush_leaves_fn = [&](int nl) {
            flush_leaves_st<PartF>(A.range, wm.leafq, nl, load_part, store_part,
                                   part_interact);
        };
        // leaves outside every softening kernel: the plain 1/r^2 law, the
        // same operations as part_interact's far branch (identical results)
        auto part_interact_far = [&](int buf, int ne) {
            if (lead) n_part += ne;
            const int np = (ne + 1) >> 1;
            for (int pb = 0; pb < np; pb += split) {
                const int p = pb + cp;
                const float4 a4 = tile.pa[buf][p], b4 = tile.pb[buf][p];
                const float2 dx = __fadd2_rn(lo2(a4), ntx), dy = __fadd2_rn(hi2(a4), nty),
                             dz = __fadd2_rn(lo2(b4), ntz);
                const float2 m = hi2(b4);
                float2 r2 = __fmul2_rn(dx, dx);
                r2 = __ffma2_rn(dy, dy, r2);
                r2 = __ffma2_rn(dz, dz, r2);
                const float2 rinv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
                const float2 fk = __fmul2_rn(__fmul2_rn(rinv, rinv), rinv);
                const float2 mf = __fmul2_rn(m, fk);
                ax = __ffma2_rn(mf, dx, ax);
                ay = __ffma2_rn(mf, dy, ay);
                az = __ffma2_rn(mf, dz, az);
                if (PHI) pp = __ffma2_rn(m, rinv, pp);
            }
        };
        auto flush_far = [&](int nl) {
            flush_leaves_st<PartF>(A.range, tile.farq, nl, load_part, store_part, part_interact_far);
        };
        unsigned long long visits = 0;
        const int guard = grav_walk<true>(A, wm, tile.nodeq, tile.farq, cl, ref, gb, eps_g, flush_nodes,
                                          flush_leaves_fn, flush_far, visits);
        if (lane == 0) {  // walk statistics
            atomicAdd(&A.counters[kCntVisitsGravity], visits);
            atomicMax(&A.counters[kCntWalkMaxIter], (unsigned long long)guard);
        }
        float fx = ax.x + ax.y, fy = ay.x + ay.y, fz = az.x + az.y, P = pp.x + pp.y;
        for (int off = gw; off < 32; off <<= 1) {
            fx += __shfl_xor_sync(kFull, fx, off);
            fy += __shfl_xor_sync(kFull, fy, off);
            fz += __shfl_xor_sync(kFull, fz, off);
            P += __shfl_xor_sync(kFull, P, off);
        }
        if (lead) {
            A.acc_g[i] = A.G * (double)fx;
            A.acc_g[A.n + i] = A.G * (double)fy;
            A.acc_g[2 * A.n + i] = A.G * (double)fz;
            if (PHI) A.phi[i] = -A.G * (double)P;
        }
    }
    n_node = warp_sum(n_node);
    n_part = warp_sum(n_part);
    if (lane == 0) {
        atomicAdd(&A.counters[0], n_node);
        atomicAdd(&A.counters[1], n_part);
        atomicAdd(&A.counters[kCntGravGroups], n_grp);
    }
}

static void allow_smem_g(const void *kern) {
    static std::mutex mu;
    static std::set<const void *> done;
    std::lock_guard<std::mutex> lk(mu);
    if (done.insert(kern).second)
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

template <bool QUAD, bool PHI>
static void launch_grav_t(const GArgs &A, State &S, const Params &P, cudaStream_t st) {
    // persistent grid: 32 warps' worth of blocks per SM
    const int blocks = S.num_sms * (32 / P.walk_warps), threads = P.walk_warps * 32;
    if (P.precision == SPH3_PREC_FP64) {
        const size_t sm = warp_mem_bytes(P.stack_cap, sizeof(GTile<double>)) * P.walk_warps;
        allow_smem_g((const void *)k_gravity_f64<QUAD, PHI>);
        k_gravity_f64<QUAD, PHI><<<blocks, threads, sm, st>>>(A);
    } else {
        const size_t sm = warp_mem_bytes(P.stack_cap, sizeof(GTileF)) * P.walk_warps;
        allow_smem_g((const void *)k_gravity_f32<QUAD, PHI>);
        k_gravity_f32<QUAD, PHI><<<blocks, threads, sm, st>>>(A);
    }
}

void launch_gravity(State &S, const Params &P, cudaStream_t st, bool with_phi) {
    if (S.n == 0) return;
    GArgs A;
    A.groups = S.groups;
    A.ngroups_dev = S.ngroups_dev;
    A.group_cloud = S.group_cloud;
    A.clouds = S.clouds;
    A.range = S.tree.range;
    A.child = S.tree.child;
    A.com_c = S.tree.com_c;
    A.mono = S.tree.mono;
    A.gw = S.tree.gw;
    A.quad4 = S.tree.quad4;
    A.quad1 = S.tree.quad1;
    A.tcom = S.tree.com;
    A.tmass = S.tree.mass;
    A.tquad = S.tree.quad;
    A.cap = S.tree.cap;
    A.pk_pos = S.pk_pos;
    A.pk_hme = S.pk_hme;
    A.pos = S.pos;
    A.m = S.m;
    A.eps = S.eps;
    A.n = S.n;
    A.G = P.G;
    A.quad = P.quadrupole;
    A.stack_cap = P.stack_cap;
    A.max_depth = S.max_level + 1;
    A.acc_g = S.acc_g;
    A.phi = S.phi;
    A.work = S.work + 5;
    A.status = S.status;
    A.counters = S.counters;
    cudaMemsetAsync(A.work, 0, sizeof(int), st);
    if (P.quadrupole) {
        if (with_phi) launch_grav_t<true, true>(A, S, P, st);
        else launch_grav_t<true, false>(A, S, P, st);
    } else {
        if (with_phi) launch_grav_t<false, true>(A, S, P, st);
        else launch_grav_t<false, false>(A, S, P, st);
    }
}

// ------------------------------------------------------------ FP64 direct sum
// One block per requested row: getAcc_g_smth_mpi's inner loop
// (sph_code/libsx.py:677-703) over the row's own system, in FP64.
__global__ void k_grav_direct(const int64_t *rows, int64_t nrows, const Cloud *clouds, int ncloud,
                              const double *pos, const double *m, const double *eps, int64_t n,
                              double G, double *acc, double *phi) {
    __shared__ double red[4][32];
    for (int64_t r = blockIdx.x; r < nrows; r += gridDim.x) {
        const int64_t i = rows[r];
        int lo = 0, hi = ncloud - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (clouds[mid].begin <= i) lo = mid;
            else hi = mid - 1;
        }
        const Cloud &cl = clouds[lo];
        const double xi = pos[i], yi = pos[n + i], zi = pos[2 * n + i], ei = eps[i];
        double fx = 0, fy = 0, fz = 0, ph = 0;
        for (int64_t j = cl.begin + threadIdx.x; j < cl.end; j += blockDim.x) {
            if (j == i) continue;
            const double dx = xi - pos[j], dy = yi - pos[n + j], dz = zi - pos[2 * n + j];
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > 0.0) spline_force<double>(r2, dx, dy, dz, m[j], 0.5 * (ei + eps[j]), fx, fy, fz, ph);
        }
        fx = warp_sum(fx);
        fy = warp_sum(fy);
        fz = warp_sum(fz);
        ph = warp_sum(ph);
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (lane == 0) {
            red[0][w] = fx;
            red[1][w] = fy;
            red[2][w] = fz;
            red[3][w] = ph;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double s[4] = {0, 0, 0, 0};
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k)
                for (int q = 0; q < 4; ++q) s[q] += red[q][k];
            acc[3 * r + 0] = G * s[0];
            acc[3 * r + 1] = G * s[1];
            acc[3 * r + 2] = G * s[2];
            if (phi) phi[r] = G * s[3];
        }
        __syncthreads();
    }
}

void launch_gravity_direct(State &S, const Params &P, const int64_t *rows_sorted_dev, int64_t nrows,
                           double *acc_dev, double *phi_dev, cudaStream_t st) {
    if (nrows == 0) return;
    int blocks = (int)std::min<int64_t>(nrows, (int64_t)S.num_sms * 16);
    k_grav_direct<<<blocks, 256, 0, st>>>(rows_sorted_dev, nrows, S.clouds, S.ncloud, S.pos, S.m, S.eps,
                                          S.n, P.G, acc_dev, phi_dev);
}

}  // namespace sph3

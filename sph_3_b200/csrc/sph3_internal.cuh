// Internal definitions shared by the CUDA translation units of libsph3.
//
// Data layout in HBM (all arrays indexed by the Morton-sorted position k,
// particles of one cloud contiguous, clouds in input order):
//   FP64 masters, component-major ([3][n] for vectors):  pos, vel, acc,
//     acc_g, acc_sph, u, u_prev, dudt, dudt_prev, m, h, eps, rho, P, c,
//     divV, curlV, bal, phi                                (the state)
//   FP32 packs for the mixed-precision walks:
//     pk_pos   float4 {x - corner, y - corner, z - corner, cell}  where
//              corner is the corner of the particle's level-10 cell of its
//              cloud's root cube and cell = ix | iy << 10 | iz << 20
//     pk_hme   float4 {h, m, eps, 0}
//     pk_vel   float4 {vx, vy, vz, 0}
//     pk_thm   float4 {rho, P / rho^2, c, Balsara f}
//   keys (uint64: cloud id above 3 * max_level Morton bits), orig (int64:
//   the caller's index of the sorted particle).
// Octree (compressed: every internal node has 2..8 children, which are
// stored contiguously; nodes laid out depth by depth):
//   nd_range int2 {first particle, count}, nd_child int2 {first child,
//   nchild | level << 8} (nchild 0 = leaf), FP64 moments and FP32 packs
//   (bbox centre, half size + hmax, centre of mass, mass / opening radii,
//   traceless quadrupole).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/sph3.h"

namespace sph3 {

constexpr int kWarp = 32;
constexpr int kGroup = 32;        // target particles per walk group (one warp)
constexpr int kCellBits = 10;     // level of the FP32 cell-relative frame
constexpr int kWalkWarps = 8;     // largest walk block (warps); the width is a runtime tunable
// resident walk blocks per SM the register budget must allow; capping the
// registers (e.g. 8 -> 64 regs) spilled and measured slower on B200
constexpr int kWalkMinBlocks = 1;
constexpr int kLeafQ = 96;        // queued leaves per warp before a flush
constexpr int kNodeQ = 64;        // queued multipole nodes per warp (gravity)
constexpr unsigned kFull = 0xffffffffu;
constexpr int kBoxChunk = 4096;  // particles per root-cube reduction block

// device counters (sph3_counters): 0..7 as documented in sph3.h, then walk
// statistics
constexpr int kRsOffsetThreads = 1024;  // threads of the one-block radix offset scan
constexpr int kRsTileKeys = 4096;       // keys per radix-sort block (256 threads x 16)
constexpr int kNumCounters = 16;
constexpr int kCntVisitsH = 8;         // nodes popped by the h-search walks
constexpr int kCntVisitsDensity = 9;   // ... density walks
constexpr int kCntVisitsHydro = 10;    // ... hydro walks
constexpr int kCntVisitsGravity = 11;  // ... gravity walks
constexpr int kCntWalkMaxIter = 12;    // longest single walk (loop iterations)
constexpr int kCntWalkMaxWhere = 13;   // iterations << 40 | visit slot << 32 | first particle of that walk
constexpr int kCntGravGroups = 14;     // groups walked by the gravity pass

// ------------------------------------------------------------ per cloud
struct Cloud {
    int64_t begin, end;  // sorted particle range
    double origin[3];    // root cube corner
    double size;         // root cube edge (power of two)
    double inv_cell;     // 2^max_level / size
    float s10;           // size / 1024 (exact power of two)
    int root;            // root node id
};

// ------------------------------------------------------------ tree view
struct Tree {
    int2 *range;        // {first, count}
    int2 *child;        // {first child, nchild | level << 8}
    // FP64 moments
    double *mass;       // [cap]
    double *com;        // [3][cap]
    double *bmin;       // [3][cap]
    double *bmax;       // [3][cap]
    double *hmax;       // [cap]
    double *epsmax;     // [cap]
    double *quad;       // [6][cap] xx xy xz yy yz zz (traceless)
    // FP32 packs for the walks
    float4 *box_c;      // {centre - corner, cell}
    float4 *box_h;      // {half extents, hmax}
    float4 *com_c;      // {com - corner, cell}
    float4 *mono;       // {mass, r_open, r_soft (bmax + epsmax), 0}
    float4 *quad4;      // {xx, xy, xz, yy}
    float *quad1;       // {yz}
    // walk records (one contiguous record per node; child.y = -1 marks an empty node)
    float4 *gw;         // [cap][2] gravity: {com_c}, {r_open, r_soft, first child, nch | level << 8}
    float4 *sw;         // [cap][3] SPH: {box_c}, {box_h}, {first child, nch | level << 8, count, 0}
    int cap;
    int *depth_begin;   // [max_depth + 2] node id where each depth starts
    int *meta;          // [128] depth_begin (first 96) and the scratch counters `total`
    int *parent;        // [cap] parent node (-1 for a root)
    int *arrive;        // [cap] children finished in the bottom-up passes (zero between passes)
    int *total;         // [4] scratch counters
    int *lvl;           // [kLvlEpoch + 1] per-depth tile counters of the level pass, then the build epoch
    unsigned long long *lb;  // [tiles of the largest depth] look-back words of the level pass
};
constexpr int kLvlEpoch = 64;  // index of the build counter in Tree::lvl (tile counters before it)

// ------------------------------------------------------------ state
struct State {
    int64_t n = 0;
    int ncloud = 0;
    int ngroups = 0;          // capacity of the group table (n)
    Cloud *clouds = nullptr;  // device [ncloud]
    int2 *groups = nullptr;   // device [n] {first, count}, rebuilt with the tree
    int *group_cloud = nullptr;
    int *ngroups_dev = nullptr;  // device: number of groups of the current tree
    // root-cube reduction work items: {cloud, begin, end, 0}, at most
    // kBoxChunk particles each, items of a cloud contiguous
    int4 *box_items = nullptr;
    int *box_item_begin = nullptr;  // [ncloud + 1]
    double *box_part = nullptr;     // [nbox_items][6]
    int nbox_items = 0;
    // FP64 masters
    double *pos = nullptr, *vel = nullptr, *acc = nullptr, *acc_g = nullptr, *acc_sph = nullptr;
    double *u = nullptr, *u_prev = nullptr, *dudt = nullptr, *dudt_prev = nullptr;
    double *m = nullptr, *h = nullptr, *eps = nullptr, *rho = nullptr, *P = nullptr, *c = nullptr;
    double *divV = nullptr, *curlV = nullptr, *bal = nullptr, *phi = nullptr;
    double *vsig = nullptr, *dt = nullptr, *dhdt = nullptr;  // signal velocity, time-step estimate
    int *nngb = nullptr;
    int64_t *orig = nullptr;
    // keys / sort
    uint64_t *key = nullptr, *key_alt = nullptr;
    uint32_t *perm = nullptr, *perm_alt = nullptr;
    // FP32 packs
    float4 *pk_pos = nullptr, *pk_hme = nullptr, *pk_vel = nullptr, *pk_thm = nullptr;
    Tree tree{};
    // bookkeeping
    unsigned *status = nullptr;        // device status word
    unsigned long long *counters = nullptr;  // [8]
    int *work = nullptr;               // [8] work-queue counters of the walks
    double *energy_part = nullptr;     // per-block FP64 partial sums [nblk][8]
    double *energy = nullptr;          // [8]
    // scratch for the sort
    uint32_t *sort_hist = nullptr;     // sort scratch (histograms, tile counters, look-back words)
    int sort_blocks = 0;
    int key_bits = 0;
    int max_level = 0;
    int cloud_bits = 0;
    // launch geometry
    int num_sms = 0;
    int walk_blocks = 0;
    int walk_warps = 4;  // warps per walk block (the config's walk_warps)
    // neighbour lists kept by the mixed density walk for the hydro pass
    int *list = nullptr;   // [n][list_cap], slot k of particle i at i * list_cap + k
    int *nlist = nullptr;  // [n] neighbours found (may exceed list_cap: then the hydro pass walks)
    int list_cap = 0;
    bool list_valid = false;  // host flag: lists match the current order, positions and h
    float4 *hrec = nullptr;   // [n][3] hydro source records {pk_pos}, {vx, vy, vz, m}, {rho, P/rho^2, c, h}
    int *ovf = nullptr;       // [1] particles whose lists overflowed in the last density pass
};

struct Params {
    int precision, h_mode, visc, step_order, n_ngb, n_ngb_tol, h_max_iter, n_boot;
    int leaf_size, stack_cap, max_level, gravity, quadrupole;
    int walk_warps;  // warps per walk block (1, 2, 4 or 8)
    int list_cap;    // neighbour-list slots (0: the hydro pass walks)
    int mac;         // SPH3_MAC_*
    int eps_from_h;  // eps = h after every h search
    double gamma, alpha, beta, eta, G, theta, eps;
    double box[3];
    int periodic;
};

// ------------------------------------------------------------ device helpers
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(kFull, v, o);
        v = v > w ? v : w;
    }
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(kFull, v, o);
        v = v < w ? v : w;
    }
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// inclusive scan of ints across the warp
__device__ __forceinline__ int warp_incl_scan(int v) {
    const int lane = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int w = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += w;
    }
    return v;
}

__device__ __forceinline__ void set_status(unsigned *status, unsigned bit) {
    atomicOr(status, bit);
}

// Morton interleave of a 21-bit integer into every third bit
__host__ __device__ __forceinline__ uint64_t spread3(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

// Quantises one coordinate to [0, 2^L) on the cloud's root cube exactly as
// the NumPy restatement does: floor((x - origin) * inv_cell), clamped.
__host__ __device__ __forceinline__ uint32_t quantise(double x, double origin, double inv_cell,
                                                      uint32_t maxq) {
    double t = (x - origin) * inv_cell;
    if (!(t > 0.0)) return 0u;  // also catches NaN
    double f = floor(t);
    if (f >= (double)maxq) return maxq;
    return (uint32_t)f;
}

// level-10 cell of a point in its cloud's root cube, and the FP32 offset from
// that cell's corner
struct CellRel {
    int cell;
    float ox, oy, oz;
};

__device__ __forceinline__ CellRel make_cellrel(double x, double y, double z, const Cloud &cl) {
    const double s = (double)cl.s10;
    const double inv = 1.0 / s;  // power of two: exact
    int ix = (int)floor((x - cl.origin[0]) * inv);
    int iy = (int)floor((y - cl.origin[1]) * inv);
    int iz = (int)floor((z - cl.origin[2]) * inv);
    ix = min(max(ix, 0), 1023);
    iy = min(max(iy, 0), 1023);
    iz = min(max(iz, 0), 1023);
    CellRel r;
    r.cell = ix | (iy << 10) | (iz << 20);
    r.ox = (float)((x - cl.origin[0]) - ix * s);
    r.oy = (float)((y - cl.origin[1]) - iy * s);
    r.oz = (float)((z - cl.origin[2]) - iz * s);
    return r;
}

// position of a packed point relative to the corner of reference cell `ref`
__device__ __forceinline__ float3 rel_to(float4 p, int ref, float s10) {
    const int c = __float_as_int(p.w);
    const int dx = (c & 1023) - (ref & 1023);
    const int dy = ((c >> 10) & 1023) - ((ref >> 10) & 1023);
    const int dz = (c >> 20) - (ref >> 20);
    return make_float3(fmaf((float)dx, s10, p.x), fmaf((float)dy, s10, p.y),
                       fmaf((float)dz, s10, p.z));
}

// ------------------------------------------------------------ launchers
// sort.cu
void launch_cloud_boxes(State &S, const Params &P, cudaStream_t st);
void launch_keys(State &S, const Params &P, cudaStream_t st);
void launch_radix_sort(State &S, cudaStream_t st);  // sorts key/perm in place (ends in key/perm)
void launch_gather(State &S, const double *const *src, double *const *dst, int nfields,
                   const int *ncomp, cudaStream_t st);
void launch_gather_orig(State &S, const int64_t *src, int64_t *dst, cudaStream_t st);
void launch_pack(State &S, const Params &P, unsigned which, cudaStream_t st);
void launch_identity_perm(State &S, cudaStream_t st);
// tree.cu
void launch_tree_build(State &S, const Params &P, cudaStream_t st);
void launch_tree_refit_h(State &S, const Params &P, cudaStream_t st);
void launch_h_guess(State &S, const Params &P, cudaStream_t st);
// walk_sph.cu
void launch_boot_h(State &S, const Params &P, cudaStream_t st);
void launch_h_search(State &S, const Params &P, cudaStream_t st);
void launch_density(State &S, const Params &P, bool divcurl, cudaStream_t st, bool keep_rho = false);
void launch_hydro(State &S, const Params &P, bool want_acc, bool want_dudt, cudaStream_t st);
void launch_eos(State &S, const Params &P, cudaStream_t st);
int launch_neighbours(State &S, const Params &P, const int64_t *rows_sorted_dev, int64_t nrows,
                      int64_t *offsets_dev, int64_t *idx_dev, int64_t cap, cudaStream_t st);
// walk_grav.cu
void launch_gravity(State &S, const Params &P, cudaStream_t st, bool with_phi);
void launch_gravity_direct(State &S, const Params &P, const int64_t *rows_sorted_dev, int64_t nrows,
                           double *acc_dev, double *phi_dev, cudaStream_t st);
// exact.cu (reference-order FP64 sums in the caller's particle order)
void launch_caller_sources(State &S, const int64_t *inv, double *dst, cudaStream_t st);
void launch_grav_pairsum(const double *src, int64_t n, int64_t row0, int64_t row1, int64_t kb, int64_t split,
                         double G, double *out, cudaStream_t st);
void launch_pe_rows(const double *src, int64_t n, double G, double *part, cudaStream_t st);
void launch_kth_dist(const double *q, int64_t mq, const State &S, int64_t kth, double *out, cudaStream_t st);
// integrate.cu
void launch_kick_drift(State &S, const Params &P, double dt, cudaStream_t st);
void launch_kick_update(State &S, const Params &P, double dt, bool update_u, bool second_kick,
                        cudaStream_t st);
void launch_u_update(State &S, const Params &P, double dt, cudaStream_t st);
void launch_first_u(State &S, const Params &P, double dt, cudaStream_t st);
// the second kick of the particles of caller rows [b, e) (sorted index inv[r])
void launch_kick_rows(State &S, double dt, const int64_t *inv, int64_t b, int64_t e, cudaStream_t st);
void launch_sum_acc(State &S, cudaStream_t st);
void launch_energy(State &S, const Params &P, cudaStream_t st);
void launch_check_finite(State &S, cudaStream_t st);
void launch_timestep(State &S, const Params &P, double c_cfl, bool all_pairs, double *dt_min_dev,
                     cudaStream_t st);

// cooling.cu (table-driven heating/cooling of u, hcoolingZ)
int cool_units_valid(const sph3_cool_table *T, const sph3_cool_units *U);
int cool_table_device(const sph3_cool_table *T);
int cool_table_species(const sph3_cool_table *T);
void launch_cooling_state(const State &S, const sph3_cool_table *T, const sph3_cool_units *U, double dt,
                          float *ionfrac, cudaStream_t st);

// pack selectors for launch_pack
constexpr unsigned kPackPos = 1, kPackHme = 2, kPackVel = 4, kPackThm = 8;

}  // namespace sph3

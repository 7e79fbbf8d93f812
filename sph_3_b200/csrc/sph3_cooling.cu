// Table-driven heating/cooling of the gas (the production runs' step after
// the u update): the reference kernel hcoolingZ
// (Particles_in_BH_Tree_III/Evrard_Collapse_2024/hfvCLibs_v7_hfv_v8.1.h:1433-1623,
// launched right after u_updater at Main_Code/hfvGpuSphBHtree_newCool_v8.cu:1552)
// over a table in the layout of the reference's coolHeatGridJan2024.bin
// (Main_Code/hfvGpuSphBHtree_newCool_v8.cu:40-80).
//
// Per gas particle, in FP32 as the reference computes it:
//   r  = |x| in kpc           -> nearest kpc grid point       (ndx_kpc)
//   nH = rho XH / mH (cgs)    -> nearest nH grid point        (ndx_nH)
//   dt in s                   -> nearest elapsed-time point   (ndx_t)
//   u  (cgs)                  -> first T row whose u(T) >= u  (ndx_u)
//   u_new = linear interpolation in u between rows ndx_u - 1 and ndx_u of the
//           evolved-u table at (kpc, nH, Z, t)  (row 0, or u beyond the last
//           row: no interpolation below, extrapolation above, as the reference)
//   ionFrac[i][k] = table species fractions at (kpc, T = ndx_u, nH, Z, k, t)
//
// "First grid point with x <= g[j]" is the reference's linear scan; here it
// is a binary search when the grid (or, for u, every T column of the table)
// is non-decreasing -- checked once when the table is made -- and the same
// linear scan otherwise, so both give the reference's index for every table.
// Products, sums and quotients are written with explicit round-to-nearest
// intrinsics, so the results do not depend on the compiler's FMA choices;
// the one fused operation is the interpolation, fhi * e2 + (flo * e1) with a
// single rounding, which reproduces the reference kernel's outputs bit for
// bit (tested against them).
//
// A particle's ion fractions are one row of N_M floats.  On the raw arrays a
// warp's rows are one contiguous block: the lanes gather their species into
// shared memory and the warp writes the block with consecutive lanes on
// consecutive addresses, instead of 32 stores strided by N_M floats.
#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "sph3_internal.cuh"

struct sph3_cool_table {
    int device = 0;
    int nkpc = 0, nT = 0, nnH = 0, nZ = 0, nM = 0, nt = 0;
    float *kpc = nullptr, *nH = nullptr, *t = nullptr;  // device grids
    float *uevol = nullptr;                               // [kpc][T][nH][Z][t]
    float *metalz = nullptr;                              // [kpc][T][nH][Z][M][t]
    float *uarr = nullptr;                                // [kpc][T][nH][Z]
    int mono_kpc = 0, mono_nH = 0, mono_t = 0, mono_u = 0;
};

namespace sph3 {

namespace {

constexpr float kMassH = 1.6726e-24f;  // g (the reference's mH)
constexpr float kXH = 0.70f;           // hydrogen mass fraction (the reference's XH)

// First j in [0, n) with x <= g[j * stride], or -1 (x above every entry, or
// NaN).  Binary search when the entries are non-decreasing (the predicate is
// then false...false true...true), the reference's linear scan otherwise.
__device__ __forceinline__ int first_at_or_above(const float *g, int n, int64_t stride, float x, int mono) {
    if (mono) {
        int lo = 0, hi = n;  // answer in [lo, hi]; hi == n: none
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (x <= g[mid * stride]) hi = mid;
            else lo = mid + 1;
        }
        return lo < n ? lo : -1;
    }
    for (int j = 0; j < n; ++j)
        if (x <= g[j * stride]) return j;
    return -1;
}

// The reference's nearest grid point: the first point at or above x, moved
// one down when the point below is strictly closer; the last point when x is
// above the grid (or NaN).
__device__ __forceinline__ int nearest_point(const float *g, int n, float x, int mono) {
    int k = first_at_or_above(g, n, 1, x, mono);
    if (k > 0) {
        const float d1 = fabsf(__fsub_rn(g[k], x));
        const float d2 = fabsf(__fsub_rn(g[k - 1], x));
        if (d2 < d1) k -= 1;
    }
    return k < 0 ? n - 1 : k;
}

struct CoolArgs {
    const float *kpc, *nH, *t, *uevol, *metalz, *uarr;
    int nkpc, nT, nnH, nZ, nM, nt;
    int mono_kpc, mono_nH, mono_t, mono_u;
    int z_index;
    float dt;
    float unit_density, unit_time, unit_u, unit_length, kpc_cm;
};

// The kpc and nH grids a block searches (in shared memory when they fit) and
// the elapsed-time index, which is the same for every particle of a call.
struct GridView {
    const float *kpc, *nH;
    int it;
};

constexpr int kGridSmem = 2048;  // floats of the kpc, nH and t grids staged per block (at most)
constexpr int kCoolThreads = 256;
constexpr int kCoolMinBlocks = 5;  // context kernel: 40 resident warps per SM, registers capped at 48
constexpr int kCoolRawMinBlocks = 4;  // raw kernel (two particles per thread): 32 warps, 64 registers
constexpr int kIonStage = 16;      // species staged per particle (rows of N_M + 1 floats) up to this N_M

// Dynamic shared memory of a cooling launch, in floats: the 1-D grids (when
// they fit) and, for the raw arrays with N_M <= kIonStage, a padded row of
// N_M + 1 floats per particle of a block pass (two per thread).
__host__ __device__ __forceinline__ int grid_floats(int nkpc, int nnH, int nt) {
    return nkpc + nnH + nt <= kGridSmem ? nkpc + nnH + nt : 0;
}
__host__ __device__ __forceinline__ int stage_floats(int nM) {
    return nM <= kIonStage ? 2 * kCoolThreads * (nM + 1) : 0;  // two particles per thread
}
// the largest dynamic shared memory of a launch stays within the 48 KB that
// needs no opt-in
static_assert(sizeof(float) * (kGridSmem + 2 * kCoolThreads * (kIonStage + 1)) <= 48 * 1024,
              "cooling launch above 48 KB of dynamic shared memory");

// Stages the 1-D grids in the block's shared memory (when they fit) and finds
// the elapsed-time point.  Every thread of the block calls it once, before
// its particle loop.
__device__ __forceinline__ GridView stage_grids(const CoolArgs &A, float *sg) {
    const bool fit = grid_floats(A.nkpc, A.nnH, A.nt) > 0;
    if (fit) {
        for (int j = threadIdx.x; j < A.nkpc; j += blockDim.x) sg[j] = A.kpc[j];
        for (int j = threadIdx.x; j < A.nnH; j += blockDim.x) sg[A.nkpc + j] = A.nH[j];
        for (int j = threadIdx.x; j < A.nt; j += blockDim.x) sg[A.nkpc + A.nnH + j] = A.t[j];
    }
    __syncthreads();
    GridView g;
    g.kpc = fit ? sg : A.kpc;
    g.nH = fit ? sg + A.nkpc : A.nH;
    const float *tg = fit ? sg + A.nkpc + A.nnH : A.t;
    g.it = nearest_point(tg, A.nt, __fmul_rn(A.dt, A.unit_time), A.mono_t);
    return g;
}

// First j with x[q] <= col[q][j * stride] for K particles at once, -1 when
// none (or NaN), over columns of n non-decreasing entries: a bisection with
// a fixed number of steps (the largest power of two <= n, halved to 1), so
// the K particles' loads of one step are issued together.  pos counts the
// leading entries with the predicate false.
template <int K>
__device__ __forceinline__ void first_at_or_above_k(const float *const (&col)[K], int n, int64_t stride,
                                                    const float (&x)[K], int (&out)[K]) {
    int pos[K];
#pragma unroll
    for (int q = 0; q < K; ++q) pos[q] = 0;
    int step = 1;
    while (2 * step <= n) step *= 2;
    for (; step > 0; step >>= 1) {
        float g[K];
#pragma unroll
        for (int q = 0; q < K; ++q) g[q] = pos[q] + step <= n ? col[q][(int64_t)(pos[q] + step - 1) * stride] : 0.f;
#pragma unroll
        for (int q = 0; q < K; ++q)
            if (pos[q] + step <= n && !(x[q] <= g[q])) pos[q] += step;
    }
#pragma unroll
    for (int q = 0; q < K; ++q) out[q] = pos[q] < n ? pos[q] : -1;
}

// K particles' table lookups, their dependent loads issued together.  u[q]
// (code units) is replaced by the new u; base[q] is the offset of the
// particle's ion fractions in the species table (species k at base + k N_t).
template <int K>
__device__ __forceinline__ void cool_k(const CoolArgs &A, const GridView &G, const float (&x)[K],
                                       const float (&y)[K], const float (&z)[K], const float (&rho)[K],
                                       float (&u)[K], int64_t (&base)[K], bool (&negative)[K]) {
    const int iz = A.z_index;
    const int it = G.it;
    const int64_t sT0 = (int64_t)A.nnH * A.nZ;  // strides of uArr [kpc][T][nH][Z]
    const int64_t sK0 = (int64_t)A.nT * sT0;
    int ik[K], ih[K], iu[K];
    float ucgs[K];
    const float *col[K];
#pragma unroll
    for (int q = 0; q < K; ++q) {
        // distance from the origin in kpc
        float r = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x[q], x[q]), __fmul_rn(y[q], y[q])),
                                       __fmul_rn(z[q], z[q])));
        r = __fdiv_rn(__fmul_rn(r, A.unit_length), A.kpc_cm);
        ik[q] = nearest_point(G.kpc, A.nkpc, r, A.mono_kpc);
        // hydrogen number density
        const float rho_cgs = __fmul_rn(rho[q], A.unit_density);
        const float nh = __fdiv_rn(__fmul_rn(rho_cgs, kXH), kMassH);
        ih[q] = nearest_point(G.nH, A.nnH, nh, A.mono_nH);
        // T row from u
        ucgs[q] = __fmul_rn(u[q], A.unit_u);
        col[q] = A.uarr + ik[q] * sK0 + (int64_t)ih[q] * A.nZ + iz;
    }
    if (A.mono_u) {
        first_at_or_above_k<K>(col, A.nT, sT0, ucgs, iu);
    } else {
#pragma unroll
        for (int q = 0; q < K; ++q) iu[q] = first_at_or_above(col[q], A.nT, sT0, ucgs[q], 0);
    }
    // evolved u: strides of uEvol [kpc][T][nH][Z][t]
    const int64_t sZ = A.nt, sH = (int64_t)A.nZ * sZ, sT = (int64_t)A.nnH * sH, sK = (int64_t)A.nT * sT;
    float e1[K], e2[K], lo[K], hi[K];
#pragma unroll
    for (int q = 0; q < K; ++q) {
        if (iu[q] < 0) iu[q] = A.nT - 1;
        const int64_t at = ik[q] * sK + (int64_t)iu[q] * sT + (int64_t)ih[q] * sH + (int64_t)iz * sZ + it;
        const int below = iu[q] > 0 ? 1 : 0;
        e2[q] = A.uevol[at];
        e1[q] = A.uevol[at - below * sT];
        hi[q] = col[q][(int64_t)iu[q] * sT0];
        lo[q] = col[q][(int64_t)(iu[q] - below) * sT0];
    }
    // species fractions: metalz [kpc][T][nH][Z][M][t]
    const int64_t mM = A.nt, mZ = (int64_t)A.nM * mM, mH = (int64_t)A.nZ * mZ, mT = (int64_t)A.nnH * mH,
                  mK = (int64_t)A.nT * mT;
#pragma unroll
    for (int q = 0; q < K; ++q) {
        float uev;
        if (iu[q] > 0) {
            const float fhi = __fdiv_rn(__fsub_rn(ucgs[q], lo[q]), __fsub_rn(hi[q], lo[q]));
            const float flo = __fsub_rn(1.0f, fhi);
            // fused as fhi * e2 + (flo * e1): the form whose results equal the
            // reference kernel's outputs bit for bit on the golden vectors
            uev = __fmaf_rn(fhi, e2[q], __fmul_rn(flo, e1[q]));
        } else {
            uev = e2[q];
        }
        negative[q] = uev < 0.0f;
        base[q] = ik[q] * mK + (int64_t)iu[q] * mT + (int64_t)ih[q] * mH + (int64_t)iz * mZ + it;
        u[q] = __fdiv_rn(uev, A.unit_u);
    }
}

// One particle's N_M species fractions (species k at metalz[base + k N_t]),
// handed to put(k, value): four loads in flight before their stores, so a
// particle waits on about N_M / 4 memory round trips rather than N_M.
template <class Put>
__device__ __forceinline__ void gather_species(const CoolArgs &A, int64_t base, Put put) {
    for (int k0 = 0; k0 < A.nM; k0 += 4) {
        float v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (k0 + j < A.nM) v[j] = A.metalz[base + (int64_t)(k0 + j) * A.nt];
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (k0 + j < A.nM) put(k0 + j, v[j]);
    }
}

// Raw arrays (the reference's float device arrays, Typ[i] == 0 is gas).
// Each lane takes two particles, i0 + lane and i0 + 32 + lane, whose
// dependent table reads are issued together (cool_k<2>), so a warp's 64
// particles own the contiguous rows [i0, i0 + 64) of ionfrac.  With
// N_M <= kIonStage each lane gathers its particles' species into padded
// shared-memory rows (N_M + 1 floats: an odd stride, so the lanes' rows fall
// in different banks) and the warp then writes the whole block of 64 * N_M
// floats with consecutive lanes on consecutive addresses (rows of non-gas
// particles are skipped, so they keep their contents); with more species
// each thread writes its own rows.  Whole warps stay in the loop.  Dynamic
// shared memory: grid_floats + stage_floats floats.
__global__ void __launch_bounds__(kCoolThreads, kCoolRawMinBlocks)
    k_hcooling(CoolArgs A, int64_t n, const int *typ, float *u, const float *rho, const float *x, const float *y,
               const float *z, float *ionfrac, unsigned *status) {
    extern __shared__ float cool_smem[];
    const GridView G = stage_grids(A, cool_smem);
    const int lane = threadIdx.x & 31;
    const bool staged = A.nM <= kIonStage;
    const int rs = A.nM + 1;  // staged row stride
    float *buf = cool_smem + grid_floats(A.nkpc, A.nnH, A.nt) + 2 * (threadIdx.x & ~31) * rs;
    const int64_t stride = 2 * (int64_t)gridDim.x * blockDim.x;
    for (int64_t i0 = 2 * ((int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31)); i0 < n; i0 += stride) {
        int64_t idx[2];
        bool gas[2];
        float xs[2], ys[2], zs[2], rs_[2], us[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            idx[q] = i0 + 32 * q + lane;
            gas[q] = idx[q] < n && (typ == nullptr || typ[idx[q]] == 0);
            // lanes without a gas particle run the lookups on harmless values
            xs[q] = gas[q] ? x[idx[q]] : 0.f;
            ys[q] = gas[q] ? y[idx[q]] : 0.f;
            zs[q] = gas[q] ? z[idx[q]] : 0.f;
            rs_[q] = gas[q] ? rho[idx[q]] : 1.f;
            us[q] = gas[q] ? u[idx[q]] : 1.f;
        }
        int64_t base[2];
        bool neg[2];
        cool_k<2>(A, G, xs, ys, zs, rs_, us, base, neg);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (!gas[q]) continue;
            u[idx[q]] = us[q];
            if (neg[q] && status) atomicOr(status, SPH3_STATUS_COOL_NEGATIVE_U);
        }
        if (!ionfrac) continue;
        if (!staged) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                float *row = ionfrac + idx[q] * A.nM;
                if (gas[q]) gather_species(A, base[q], [&](int k, float v) { row[k] = v; });
            }
            continue;
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            float *row = buf + (32 * q + lane) * rs;
            if (gas[q]) gather_species(A, base[q], [&](int k, float v) { row[k] = v; });
        }
        const unsigned long long gm = (unsigned long long)__ballot_sync(0xffffffffu, gas[0]) |
                                      ((unsigned long long)__ballot_sync(0xffffffffu, gas[1]) << 32);
        __syncwarp();
        const int rows = n - i0 < 64 ? (int)(n - i0) : 64;
        const int total = rows * A.nM;
        float *out = ionfrac + i0 * A.nM;
        // this lane's first element of the warp block (row p, species k), and
        // the row and species steps of 32 elements
        int p = lane / A.nM, k = lane - p * A.nM;
        const int dp = 32 / A.nM, dk = 32 - dp * A.nM;
        for (int e = lane; e < total; e += 32) {
            if ((gm >> p) & 1ull) out[e] = buf[p * rs + k];
            p += dp;
            k += dk;
            if (k >= A.nM) {
                k -= A.nM;
                ++p;
            }
        }
        __syncwarp();
    }
}

// The context's FP64 state (component-major positions, sorted order; every
// particle is gas): the inputs are rounded to FP32 as the reference's arrays
// are, and u is written back from the FP32 result.  Ion fractions go to the
// particle's row in the caller's order (orig: sorted -> caller index), so they
// stay valid whatever the context's order later becomes; those rows are
// scattered, so each thread writes its own.
__global__ void __launch_bounds__(kCoolThreads, kCoolMinBlocks)
    k_hcooling_state(CoolArgs A, int64_t n, const double *pos, const double *rho, double *u, const int64_t *orig,
                     float *ionfrac, unsigned *status) {
    extern __shared__ float cool_smem[];
    const GridView G = stage_grids(A, cool_smem);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        int64_t base[1];
        bool neg[1];
        const float xs[1] = {(float)pos[i]}, ys[1] = {(float)pos[n + i]}, zs[1] = {(float)pos[2 * n + i]};
        const float rs_[1] = {(float)rho[i]};
        float us[1] = {(float)u[i]};
        cool_k<1>(A, G, xs, ys, zs, rs_, us, base, neg);
        u[i] = (double)us[0];
        if (neg[0]) atomicOr(status, SPH3_STATUS_COOL_NEGATIVE_U);
        if (ionfrac) {
            float *row = ionfrac + orig[i] * A.nM;
            gather_species(A, base[0], [&](int k, float v) { row[k] = v; });
        }
    }
}

CoolArgs make_args(const sph3_cool_table *T, const sph3_cool_units *U, float dt) {
    CoolArgs A;
    A.kpc = T->kpc;
    A.nH = T->nH;
    A.t = T->t;
    A.uevol = T->uevol;
    A.metalz = T->metalz;
    A.uarr = T->uarr;
    A.nkpc = T->nkpc;
    A.nT = T->nT;
    A.nnH = T->nnH;
    A.nZ = T->nZ;
    A.nM = T->nM;
    A.nt = T->nt;
    A.mono_kpc = T->mono_kpc;
    A.mono_nH = T->mono_nH;
    A.mono_t = T->mono_t;
    A.mono_u = T->mono_u;
    A.z_index = U->z_index;
    A.dt = dt;
    A.unit_density = U->unit_density_cgs;
    A.unit_time = U->unit_time_s;
    A.unit_u = U->unit_u_cgs;
    A.unit_length = U->unit_length_cm;
    A.kpc_cm = U->kpc_cm;
    return A;
}

// blocks of a raw-array launch: two particles per thread, at most one wave
// of resident blocks (kCoolRawMinBlocks per SM), which then stride
int cool_grid(int64_t n, int dev) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 2 * kCoolThreads - 1) / (2 * kCoolThreads),
                                                       (int64_t)sms * kCoolRawMinBlocks));
}

bool nondecreasing(const float *g, int64_t n, int64_t stride) {
    for (int64_t j = 1; j < n; ++j)
        if (!(g[(j - 1) * stride] <= g[j * stride])) return false;
    return true;
}

template <typename T>
int upload(T **dst, const T *src, size_t count) {
    if (cudaMalloc(dst, sizeof(T) * std::max<size_t>(count, 1)) != cudaSuccess) return SPH3_ERR_OUT_OF_MEMORY;
    if (cudaMemcpy(*dst, src, sizeof(T) * count, cudaMemcpyHostToDevice) != cudaSuccess) return SPH3_ERR_CUDA;
    return SPH3_OK;
}

}  // namespace

int cool_units_valid(const sph3_cool_table *T, const sph3_cool_units *U) {
    if (!T || !U) return 0;
    return U->z_index >= 0 && U->z_index < T->nZ;
}

int cool_table_device(const sph3_cool_table *T) { return T ? T->device : -1; }
int cool_table_species(const sph3_cool_table *T) { return T ? T->nM : 0; }

void launch_cooling_state(const State &S, const sph3_cool_table *T, const sph3_cool_units *U, double dt,
                          float *ionfrac, cudaStream_t st) {
    if (S.n == 0) return;
    const size_t smem = sizeof(float) * grid_floats(T->nkpc, T->nnH, T->nt);
    k_hcooling_state<<<std::min<int64_t>((S.n + kCoolThreads - 1) / kCoolThreads, (int64_t)S.num_sms * kCoolMinBlocks),
                       kCoolThreads, smem, st>>>(
        make_args(T, U, (float)dt), S.n, S.pos, S.rho, S.u, S.orig, ionfrac, S.status);
}

}  // namespace sph3

using namespace sph3;

extern "C" {

int sph3_cool_table_create(int device, const int32_t dims[6], const float *kpc, const float *nh, const float *t,
                           const float *uevol, const float *metalz, const float *uarr, sph3_cool_table **out) {
    if (!out || !dims || !kpc || !nh || !t || !uevol || !metalz || !uarr) return SPH3_ERR_INVALID_ARG;
    *out = nullptr;
    for (int k = 0; k < 6; ++k)
        if (dims[k] <= 0) return SPH3_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return SPH3_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return SPH3_ERR_INVALID_ARG;
    // dims in the order of the file header: N_kpc, N_T, N_nH, N_Z, N_M, N_t
    const int64_t nk = dims[0], nT = dims[1], nh_ = dims[2], nZ = dims[3], nM = dims[4], nt = dims[5];
    const int64_t n_u = nk * nT * nh_ * nZ, n_ev = n_u * nt, n_mz = n_ev * nM;
    if (n_mz > (int64_t(1) << 40)) return SPH3_ERR_INVALID_ARG;
    auto *T = new (std::nothrow) sph3_cool_table;
    if (!T) return SPH3_ERR_OUT_OF_MEMORY;
    T->device = device;
    T->nkpc = (int)nk;
    T->nT = (int)nT;
    T->nnH = (int)nh_;
    T->nZ = (int)nZ;
    T->nM = (int)nM;
    T->nt = (int)nt;
    T->mono_kpc = nondecreasing(kpc, nk, 1);
    T->mono_nH = nondecreasing(nh, nh_, 1);
    T->mono_t = nondecreasing(t, nt, 1);
    bool mono = true;
    for (int64_t c = 0; c < nk && mono; ++c)
        for (int64_t r = 0; r < nh_ * nZ && mono; ++r) mono = nondecreasing(uarr + c * nT * nh_ * nZ + r, nT, nh_ * nZ);
    T->mono_u = mono;
    int prev = 0;
    cudaGetDevice(&prev);
    int rc = cudaSetDevice(device) == cudaSuccess ? SPH3_OK : SPH3_ERR_CUDA;
    if (!rc) rc = upload(&T->kpc, kpc, nk);
    if (!rc) rc = upload(&T->nH, nh, nh_);
    if (!rc) rc = upload(&T->t, t, nt);
    if (!rc) rc = upload(&T->uarr, uarr, n_u);
    if (!rc) rc = upload(&T->uevol, uevol, n_ev);
    if (!rc) rc = upload(&T->metalz, metalz, n_mz);
    cudaSetDevice(prev);
    if (rc) {
        sph3_cool_table_destroy(T);
        return rc;
    }
    *out = T;
    return SPH3_OK;
}

int sph3_cool_table_destroy(sph3_cool_table *T) {
    if (!T) return SPH3_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(T->device);
    for (float *p : {T->kpc, T->nH, T->t, T->uevol, T->metalz, T->uarr})
        if (p) cudaFree(p);
    cudaSetDevice(prev);
    delete T;
    return SPH3_OK;
}

int sph3_cool_table_dims(const sph3_cool_table *T, int32_t dims[6], int32_t monotone[4]) {
    if (!T || !dims) return SPH3_ERR_INVALID_ARG;
    const int32_t d[6] = {T->nkpc, T->nT, T->nnH, T->nZ, T->nM, T->nt};
    for (int k = 0; k < 6; ++k) dims[k] = d[k];
    if (monotone) {
        monotone[0] = T->mono_kpc;
        monotone[1] = T->mono_nH;
        monotone[2] = T->mono_t;
        monotone[3] = T->mono_u;
    }
    return SPH3_OK;
}

int sph3_hcooling(const sph3_cool_table *T, const sph3_cool_units *U, float dt, int64_t n, const int32_t *typ,
                  float *u, const float *rho, const float *x, const float *y, const float *z, float *ionfrac,
                  uint32_t *status, void *stream) {
    if (!T || !U || n < 0) return SPH3_ERR_INVALID_ARG;
    if (!cool_units_valid(T, U)) return SPH3_ERR_INVALID_ARG;
    if (n == 0) return SPH3_OK;
    if (!u || !rho || !x || !y || !z) return SPH3_ERR_INVALID_ARG;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return SPH3_ERR_CUDA;
    if (prev != T->device && cudaSetDevice(T->device) != cudaSuccess) return SPH3_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t smem = sizeof(float) * (grid_floats(T->nkpc, T->nnH, T->nt) + (ionfrac ? stage_floats(T->nM) : 0));
    k_hcooling<<<cool_grid(n, T->device), kCoolThreads, smem, st>>>(make_args(T, U, dt), n, typ, u, rho, x, y, z, ionfrac,
                                                        status);
    const cudaError_t e = cudaGetLastError();
    if (prev != T->device) cudaSetDevice(prev);
    return e == cudaSuccess ? SPH3_OK : SPH3_ERR_CUDA;
}

}  // extern "C"

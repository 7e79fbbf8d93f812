// Root cubes, Morton keys, LSD radix sort and the permutation gather.
//
// All of these are HBM/L2-bound integer and byte moves: coalesced loads,
// grid sizes in multiples of the SM count, no tensor-core reshaping.
#include <cfloat>

#include "sph3_internal.cuh"

namespace sph3 {

// ------------------------------------------------------------ root cubes
// Two kernels.  k_box_partial: one block per work item (a run of at most
// kBoxChunk particles of one cloud; the item table is fixed per particle
// layout) writes the FP64 min/max of its run.  k_cloud_boxes: one block per
// cloud reduces its items and sets a power-of-two cube [origin, origin + size)
// that contains the cloud, origin on the size/2 grid.  Periodic runs use the
// fixed cube [0, 2^ceil(log2 L)).
__global__ void __launch_bounds__(256) k_box_partial(const int4 *items, const double *pos, int64_t n,
                                                     double *part, unsigned *status) {
    const int4 it = items[blockIdx.x];  // {cloud, begin, end, 0}
    __shared__ double smin[3][8], smax[3][8];
    double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, mx[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    int bad = 0;
    for (int64_t k = it.y + threadIdx.x; k < it.z; k += blockDim.x) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double x = pos[d * n + k];
            if (!isfinite(x)) {
                bad = 1;
                continue;
            }
            mn[d] = fmin(mn[d], x);
            mx[d] = fmax(mx[d], x);
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double a = warp_min(mn[d]), b = warp_max(mx[d]);
        if (lane == 0) {
            smin[d][wid] = a;
            smax[d][wid] = b;
        }
    }
    if (__any_sync(kFull, bad) && lane == 0) atomicOr(status, SPH3_STATUS_NAN_INPUT);
    __syncthreads();
    if (threadIdx.x < 3) {
        const int d = threadIdx.x;
        double lo = DBL_MAX, hi = -DBL_MAX;
        for (int w = 0; w < 8; ++w) {
            lo = fmin(lo, smin[d][w]);
            hi = fmax(hi, smax[d][w]);
        }
        part[blockIdx.x * 6 + d] = lo;
        part[blockIdx.x * 6 + 3 + d] = hi;
    }
}

__global__ void k_cloud_boxes(Cloud *clouds, const int *item_begin, const double *part, int max_level,
                              int periodic, double Lx, double Ly, double Lz) {
    Cloud &cl = clouds[blockIdx.x];
    // one warp: lanes stride over the cloud's items, then a warp reduction
    double lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
        lo[d] = DBL_MAX;
        hi[d] = -DBL_MAX;
        for (int it = item_begin[blockIdx.x] + (int)threadIdx.x; it < item_begin[blockIdx.x + 1]; it += 32) {
            lo[d] = fmin(lo[d], part[it * 6 + d]);
            hi[d] = fmax(hi[d], part[it * 6 + 3 + d]);
        }
        lo[d] = warp_min(lo[d]);
        hi[d] = warp_max(hi[d]);
        if (lo[d] > hi[d]) lo[d] = hi[d] = 0.0;  // empty cloud
    }
    if (threadIdx.x == 0) {
        double size;
        double org[3];
        if (periodic) {
            double L = fmax(Lx, fmax(Ly, Lz));
            int e;
            frexp(L, &e);  // L = f * 2^e, f in [0.5, 1)
            size = ldexp(1.0, e);
            if (size * 0.5 >= L) size *= 0.5;
            org[0] = org[1] = org[2] = 0.0;
        } else {
            double ext = fmax(hi[0] - lo[0], fmax(hi[1] - lo[1], hi[2] - lo[2]));
            if (!(ext > 0.0) || !isfinite(ext)) ext = 1.0;
            int e;
            frexp(ext, &e);
            size = ldexp(1.0, e);  // >= ext
            for (int attempt = 0; attempt < 64; ++attempt) {
                double half = 0.5 * size;
                bool ok = true;
                for (int d = 0; d < 3; ++d) {
                    org[d] = floor(lo[d] / half) * half;
                    if (!(org[d] + size > hi[d])) ok = false;
                }
                if (ok) break;
                size *= 2.0;
            }
        }
        for (int d = 0; d < 3; ++d) cl.origin[d] = org[d];
        cl.size = size;
        cl.inv_cell = ldexp(1.0, max_level) / size;
        cl.s10 = (float)(size / 1024.0);
    }
}

void launch_cloud_boxes(State &S, const Params &P, cudaStream_t st) {
    if (S.ncloud == 0) return;
    if (S.nbox_items > 0)
        k_box_partial<<<S.nbox_items, 256, 0, st>>>(S.box_items, S.pos, S.n, S.box_part, S.status);
    k_cloud_boxes<<<S.ncloud, 32, 0, st>>>(S.clouds, S.box_item_begin, S.box_part, S.max_level, P.periodic,
                                           P.box[0], P.box[1], P.box[2]);
}

// ------------------------------------------------------------ keys
__device__ __forceinline__ int cloud_of_sorted(const Cloud *clouds, int ncloud, int64_t k) {
    int lo = 0, hi = ncloud - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (clouds[mid].begin <= k) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void k_keys(const Cloud *clouds, int ncloud, const double *pos, int64_t n,
                       int max_level, uint64_t *key, uint32_t *perm) {
    const uint32_t maxq = (1u << max_level) - 1u;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int c = cloud_of_sorted(clouds, ncloud, k);
        const Cloud &cl = clouds[c];
        uint32_t ix = quantise(pos[k], cl.origin[0], cl.inv_cell, maxq);
        uint32_t iy = quantise(pos[n + k], cl.origin[1], cl.inv_cell, maxq);
        uint32_t iz = quantise(pos[2 * n + k], cl.origin[2], cl.inv_cell, maxq);
        uint64_t mort = spread3(ix) | (spread3(iy) << 1) | (spread3(iz) << 2);
        key[k] = ((uint64_t)c << (3 * max_level)) | mort;
        perm[k] = (uint32_t)k;
    }
}

void launch_keys(State &S, const Params &P, cudaStream_t st) {
    if (S.n == 0) return;
    int blocks = (int)std::min<int64_t>((S.n + 255) / 256, (int64_t)S.num_sms * 8);
    k_keys<<<blocks, 256, 0, st>>>(S.clouds, S.ncloud, S.pos, S.n, S.max_level, S.key, S.perm);
}

__global__ void k_identity(uint32_t *perm, int64_t n) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x)
        perm[k] = (uint32_t)k;
}

void launch_identity_perm(State &S, cudaStream_t st) {
    if (S.n == 0) return;
    int blocks = (int)std::min<int64_t>((S.n + 255) / 256, (int64_t)S.num_sms * 8);
    k_identity<<<blocks, 256, 0, st>>>(S.perm, S.n);
}

// ------------------------------------------------------------ radix sort
// LSD, 8-bit digits, stable.  Per pass: a tile histogram, one scan of the
// digit-major histogram table, and a stable scatter that ranks each key
// within its tile with warp match (order = memory order inside a warp's
// segment, then warp order).
constexpr int kRsThreads = 256;
constexpr int kRsItems = kRsTileKeys / kRsThreads;
constexpr int kRsTile = kRsThreads * kRsItems;
constexpr int kRsWarps = kRsThreads / 32;

__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const uint64_t *key, int64_t n, int shift,
                                                        uint32_t *hist, int nblocks) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kRsTile;
#pragma unroll
    for (int t = 0; t < kRsItems; ++t) {
        int64_t k = base + t * kRsThreads + threadIdx.x;
        if (k < n) atomicAdd(&h[(key[k] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[blockIdx.x * 256 + threadIdx.x] = h[threadIdx.x];  // block-major table
}

// Exclusive prefix of the block-major digit histogram, in place: hist[b][d]
// becomes the number of keys with digit d in blocks before b, and
// hist[nblocks][d] the number of keys with a smaller digit.  One block of
// kRsOffsetThreads threads: 256 digits x kOffQ block ranges; each range is
// summed with kOffU independent loads in flight, the ranges and digits are
// combined in shared memory, and a second pass over the (L2-resident) table
// writes the prefixes.
constexpr int kOffQ = kRsOffsetThreads / 256;
constexpr int kOffU = 16;

__global__ void __launch_bounds__(kRsOffsetThreads) k_rs_offsets(uint32_t *hist, int nblocks) {
    __shared__ uint32_t part[kOffQ][256];
    __shared__ uint32_t tot[256];
    const int d = threadIdx.x & 255, q = threadIdx.x >> 8;
    const int per = (nblocks + kOffQ - 1) / kOffQ;
    const int b0 = min(nblocks, q * per), b1 = min(nblocks, b0 + per);
    uint32_t s = 0;
    int b = b0;
    for (; b + kOffU <= b1; b += kOffU) {
        uint32_t v[kOffU];
#pragma unroll
        for (int k = 0; k < kOffU; ++k) v[k] = hist[(size_t)(b + k) * 256 + d];
#pragma unroll
        for (int k = 0; k < kOffU; ++k) s += v[k];
    }
    for (; b < b1; ++b) s += hist[(size_t)b * 256 + d];
    part[q][d] = s;
    __syncthreads();
    if (q == 0) {
        uint32_t run = 0;
#pragma unroll
        for (int k = 0; k < kOffQ; ++k) {
            const uint32_t t = part[k][d];
            part[k][d] = run;
            run += t;
        }
        tot[d] = run;
    }
    __syncthreads();
    const uint32_t own = tot[d];
    for (int o = 1; o < 256; o <<= 1) {
        const uint32_t v = (q == 0 && d >= o) ? tot[d - o] : 0u;
        __syncthreads();
        if (q == 0) tot[d] += v;
        __syncthreads();
    }
    uint32_t run = part[q][d];
    b = b0;
    for (; b + kOffU <= b1; b += kOffU) {
        uint32_t v[kOffU];
#pragma unroll
        for (int k = 0; k < kOffU; ++k) v[k] = hist[(size_t)(b + k) * 256 + d];
#pragma unroll
        for (int k = 0; k < kOffU; ++k) {
            hist[(size_t)(b + k) * 256 + d] = run;
            run += v[k];
        }
    }
    for (; b < b1; ++b) {
        const uint32_t v = hist[(size_t)b * 256 + d];
        hist[(size_t)b * 256 + d] = run;
        run += v;
    }
    if (q == 0) hist[(size_t)nblocks * 256 + d] = tot[d] - own;  // exclusive digit base
}

// Stable scatter of one tile.  Each key's rank inside the tile (digit
// start in the tile + earlier warps' count of the digit + rank inside its
// warp, in memory order) is computed with warp match; the tile is then
// staged in shared memory in digit order, so that every digit's run leaves
// as consecutive addresses (coalesced stores instead of one scattered 8-byte
// store per key).  The output is the same as scattering each key directly.
// offsets(d, count of digit d in this tile) gives the output start of the
// tile's keys of digit d (called by thread d once the counts are known).
template <class Offsets>
__device__ __forceinline__ void rs_scatter_tile(const uint64_t *key_in, const uint32_t *val_in, uint64_t *key_out,
                                                uint32_t *val_out, int64_t n, int shift, int tile_index,
                                                Offsets &offsets) {
    __shared__ uint32_t wcnt[kRsWarps][256];
    __shared__ uint32_t goff[256];  // output start of the tile's keys of digit d
    __shared__ uint32_t toff[256];  // start of digit d inside the tile
    __shared__ uint32_t wsum[kRsWarps];
    __shared__ uint64_t stage[kRsTile];  // keys in tile order, then the values
    __shared__ uint8_t sdig[kRsTile];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kRsWarps * 256; i += kRsThreads) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const int64_t tile = (int64_t)tile_index * kRsTile;
    const int64_t base = tile + (int64_t)w * (kRsItems * 32);
    uint64_t kk[kRsItems];
    uint32_t vv[kRsItems];
    uint32_t rank[kRsItems];
    int dig[kRsItems];
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int t = 0; t < kRsItems; ++t) {
        int64_t k = base + t * 32 + lane;
        bool ok = k < n;
        kk[t] = ok ? key_in[k] : 0ull;
        vv[t] = ok ? val_in[k] : 0u;
        int d = ok ? (int)((kk[t] >> shift) & 255u) : 256;
        dig[t] = d;
        unsigned peers = __match_any_sync(kFull, d);
        uint32_t b = d < 256 ? wcnt[w][d] : 0u;
        __syncwarp();
        if (d < 256 && (peers & lt) == 0) wcnt[w][d] = b + __popc(peers);
        __syncwarp();
        rank[t] = b + __popc(peers & lt);
    }
    __syncthreads();
    // prefix over warps for each digit, and the tile's count of the digit
    uint32_t cnt_d;
    {
        const int d = threadIdx.x;
        uint32_t run = 0;
#pragma unroll
        for (int ww = 0; ww < kRsWarps; ++ww) {
            uint32_t c = wcnt[ww][d];
            wcnt[ww][d] = run;
            run += c;
        }
        cnt_d = run;
    }
    // exclusive scan of the digit counts over the tile (256 threads = 256 digits)
    {
        const uint32_t incl = (uint32_t)warp_incl_scan((int)cnt_d);
        if (lane == 31) wsum[w] = incl;
        __syncthreads();
        uint32_t pre = 0;
#pragma unroll
        for (int ww = 0; ww < kRsWarps; ++ww) pre += ww < w ? wsum[ww] : 0u;
        toff[threadIdx.x] = pre + incl - cnt_d;
    }
    goff[threadIdx.x] = offsets(threadIdx.x, cnt_d);  // output start of the tile's keys of the digit
    __syncthreads();
    uint32_t lpos[kRsItems];
#pragma unroll
    for (int t = 0; t < kRsItems; ++t) {
        const int d = dig[t];
        if (d < 256) {
            lpos[t] = toff[d] + wcnt[w][d] + rank[t];
            stage[lpos[t]] = kk[t];
            sdig[lpos[t]] = (uint8_t)d;
        }
    }
    __syncthreads();
    const int cnt = (int)min((int64_t)kRsTile, n - tile);
    for (int j = threadIdx.x; j < cnt; j += kRsThreads) {
        const int d = sdig[j];
        key_out[goff[d] + (uint32_t)j - toff[d]] = stage[j];
    }
    __syncthreads();
    uint32_t *sval = reinterpret_cast<uint32_t *>(stage);
#pragma unroll
    for (int t = 0; t < kRsItems; ++t)
        if (dig[t] < 256) sval[lpos[t]] = vv[t];
    __syncthreads();
    for (int j = threadIdx.x; j < cnt; j += kRsThreads) {
        const int d = sdig[j];
        val_out[goff[d] + (uint32_t)j - toff[d]] = sval[j];
    }
}

// The tile scatter with offsets from the digit-major table of k_rs_offsets
// (one tile per block, in block order).
__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const uint64_t *key_in,
                                                           const uint32_t *val_in, uint64_t *key_out,
                                                           uint32_t *val_out, int64_t n, int shift,
                                                           const uint32_t *hist, int nblocks) {
    auto offsets = [&](int d, uint32_t) { return hist[nblocks * 256 + d] + hist[blockIdx.x * 256 + d]; };
    rs_scatter_tile(key_in, val_in, key_out, val_out, n, shift, blockIdx.x, offsets);
}

// ---- one sweep per digit pass (the context's sort)
// All passes' digit histograms in one read of the keys (per-warp private
// tables in shared memory, then one atomic per bin and block); the scatter
// of each pass then takes its tiles in order from an atomic counter and finds
// each digit's offset over the earlier tiles by decoupled look-back: a tile
// publishes its count of each digit (AGG), adds up its predecessors' counts
// back to one that knows its inclusive prefix (INCL) and publishes its own.
// One launch per pass instead of histogram + table scan + scatter.  Every
// predecessor tile was taken by a running block, so each wait ends; waits are
// bounded all the same and raise SPH3_STATUS_SORT if one ever ran out.
constexpr int kHaThreads = 128;
constexpr int kMaxPasses = 8;
constexpr uint32_t kOsAgg = 1u << 30, kOsIncl = 2u << 30, kOsMask = (1u << 30) - 1u;
constexpr int kOsMaxSpin = 1 << 22;

__global__ void __launch_bounds__(kHaThreads) k_rs_hist_all(const uint64_t *key, int64_t n, int passes,
                                                            uint32_t *hist_all) {
    __shared__ uint32_t h[kHaThreads / 32][kMaxPasses][256];
    const int w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < (kHaThreads / 32) * kMaxPasses * 256; i += kHaThreads) (&h[0][0][0])[i] = 0;
    __syncthreads();
    for (int64_t k = (int64_t)blockIdx.x * kHaThreads + threadIdx.x; k < n; k += (int64_t)gridDim.x * kHaThreads) {
        const uint64_t kv = key[k];
        for (int p = 0; p < passes; ++p) atomicAdd(&h[w][p][(kv >> (8 * p)) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += kHaThreads) {
        uint32_t t = 0;
#pragma unroll
        for (int q = 0; q < kHaThreads / 32; ++q) t += (&h[q][0][0])[i];
        if (t) atomicAdd(hist_all + i, t);
    }
}

__global__ void __launch_bounds__(kRsThreads) k_rs_onesweep(const uint64_t *key_in, const uint32_t *val_in,
                                                            uint64_t *key_out, uint32_t *val_out, int64_t n,
                                                            int pass, const uint32_t *hist_all, uint32_t *state,
                                                            int *tile_ctr, unsigned *status) {
    __shared__ int s_tile;
    __shared__ uint32_t wtot[kRsWarps];
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr + pass, 1);
    // exclusive scan over digits of this pass's global histogram: digit bases
    const int d0 = threadIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t hd = hist_all[pass * 256 + d0];
    const uint32_t incl = (uint32_t)warp_incl_scan((int)hd);
    if (lane == 31) wtot[w] = incl;
    __syncthreads();
    uint32_t dbase = incl - hd;
#pragma unroll
    for (int q = 0; q < kRsWarps; ++q) dbase += q < w ? wtot[q] : 0u;
    const int tile = s_tile;
    uint32_t *st = state + (size_t)tile * 256;
    auto offsets = [&](int d, uint32_t cnt) -> uint32_t {
        if (tile == 0) {
            atomicExch(st + d, kOsIncl | cnt);
            return dbase;
        }
        atomicExch(st + d, kOsAgg | cnt);
        uint32_t excl = 0;
        int j = tile - 1, spins = 0;
        while (j >= 0) {
            const uint32_t v = atomicAdd(state + (size_t)j * 256 + d, 0u);
            if ((v & ~kOsMask) == 0u) {
                if (++spins > kOsMaxSpin) {
                    atomicOr(status, SPH3_STATUS_SORT);
                    break;
                }
                __nanosleep(32);
                continue;
            }
            excl += v & kOsMask;
            if ((v & ~kOsMask) == kOsIncl) break;
            --j;
        }
        atomicExch(st + d, kOsIncl | (excl + cnt));
        return dbase + excl;
    };
    rs_scatter_tile(key_in, val_in, key_out, val_out, n, 8 * pass, tile, offsets);
}

void launch_radix_sort(State &S, cudaStream_t st) {
    if (S.n <= 1) return;
    const int nb = (int)((S.n + kRsTile - 1) / kRsTile);
    const int passes = (S.key_bits + 7) / 8;
    uint64_t *kin = S.key, *kout = S.key_alt;
    uint32_t *vin = S.perm, *vout = S.perm_alt;
    // scratch: all passes' histograms, the tile counters, the look-back words
    uint32_t *hist_all = S.sort_hist;
    int *tile_ctr = reinterpret_cast<int *>(S.sort_hist + kMaxPasses * 256);
    uint32_t *state = S.sort_hist + kMaxPasses * 256 + 64;
    cudaMemsetAsync(S.sort_hist, 0, sizeof(uint32_t) * ((size_t)kMaxPasses * 256 + 64 + (size_t)passes * nb * 256), st);
    k_rs_hist_all<<<(int)std::min<int64_t>(nb, (int64_t)S.num_sms * 4), kHaThreads, 0, st>>>(kin, S.n, passes,
                                                                                          hist_all);
    for (int p = 0; p < passes; ++p) {
        k_rs_onesweep<<<nb, kRsThreads, 0, st>>>(kin, vin, kout, vout, S.n, p, hist_all, state + (size_t)p * nb * 256,
                                                 tile_ctr, S.status);
        uint64_t *tk = kin;
        kin = kout;
        kout = tk;
        uint32_t *tv = vin;
        vin = vout;
        vout = tv;
    }
    if (kin != S.key) {  // odd pass count: copy back so the result is in key/perm
        cudaMemcpyAsync(S.key, kin, sizeof(uint64_t) * S.n, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(S.perm, vin, sizeof(uint32_t) * S.n, cudaMemcpyDeviceToDevice, st);
    }
}

// ------------------------------------------------------------ gather
constexpr int kMaxGather = 40;
struct GatherArgs {
    const double *src[kMaxGather];
    double *dst[kMaxGather];
    int nf;
};

__global__ void k_gather(const uint32_t *perm, GatherArgs a, int64_t n) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t j = perm[k];
        for (int f = 0; f < a.nf; ++f) a.dst[f][k] = a.src[f][j];
    }
}

void launch_gather(State &S, const double *const *src, double *const *dst, int nfields,
                   const int *ncomp, cudaStream_t st) {
    if (S.n == 0) return;
    GatherArgs a;
    a.nf = 0;
    for (int f = 0; f < nfields; ++f) {
        for (int c = 0; c < ncomp[f]; ++c) {
            if (a.nf == kMaxGather) {
                int blocks = (int)std::min<int64_t>((S.n + 255) / 256, (int64_t)S.num_sms * 8);
                k_gather<<<blocks, 256, 0, st>>>(S.perm, a, S.n);
                a.nf = 0;
            }
            a.src[a.nf] = src[f] + (int64_t)c * S.n;
            a.dst[a.nf] = dst[f] + (int64_t)c * S.n;
            ++a.nf;
        }
    }
    if (a.nf) {
        int blocks = (int)std::min<int64_t>((S.n + 255) / 256, (int64_t)S.num_sms * 8);
        k_gather<<<blocks, 256, 0, st>>>(S.perm, a, S.n);
    }
}

__global__ void k_gather_i64(const uint32_t *perm, const int64_t *src, int64_t *dst, int64_t n) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x)
        dst[k] = src[perm[k]];
}

void launch_gather_orig(State &S, const int64_t *src, int64_t *dst, cudaStream_t st) {
    if (S.n == 0) return;
    int blocks = (int)std::min<int64_t>((S.n + 255) / 256, (int64_t)S.num_sms * 8);
    k_gather_i64<<<blocks, 256, 0, st>>>(S.perm, src, dst, S.n);
}

// ------------------------------------------------------------ packs
__global__ void k_pack(const Cloud *clouds, const uint64_t *key, int max_level, int64_t n,
                       const double *pos, const double *vel, const double *h, const double *m,
                       const double *eps, const double *rho, const double *P, const double *c,
                       const double *bal, float4 *pk_pos, float4 *pk_hme, float4 *pk_vel,
                       float4 *pk_thm, unsigned which) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
        if (which & kPackPos) {
            const Cloud &cl = clouds[(int)(key[k] >> (3 * max_level))];
            CellRel r = make_cellrel(pos[k], pos[n + k], pos[2 * n + k], cl);
            pk_pos[k] = make_float4(r.ox, r.oy, r.oz, __int_as_float(r.cell));
        }
        if (which & kPackHme) pk_hme[k] = make_float4((float)h[k], (float)m[k], (float)eps[k], 0.f);
        if (which & kPackVel)
            pk_vel[k] = make_float4((float)vel[k], (float)vel[n + k], (float)vel[2 * n + k], 0.f);
        if (which & kPackThm) {
            double r = rho[k];
            double pr = r > 0.0 ? P[k] / (r * r) : 0.0;
            pk_thm[k] = make_float4((float)r, (float)pr, (float)c[k], (float)bal[k]);
        }
    }
}

void launch_pack(State &S, const Params &P, unsigned which, cudaStream_t st) {
    if (S.n == 0 || which == 0) return;
    (void)P;
    int blocks = (int)std::min<int64_t>((S.n + 255) / 256, (int64_t)S.num_sms * 8);
    k_pack<<<blocks, 256, 0, st>>>(S.clouds, S.key, S.max_level, S.n, S.pos, S.vel, S.h, S.m,
                                   S.eps, S.rho, S.P, S.c, S.bal, S.pk_pos, S.pk_hme, S.pk_vel,
                                   S.pk_thm, which);
}

}  // namespace sph3

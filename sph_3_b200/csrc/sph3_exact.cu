// Reference-order FP64 passes for the drop-in functions whose results depend
// on the summation order of the reference's serial loops.  They run in the
// caller's particle order and round every operation as the reference's numba
// code does (no contraction into FMA, numba's integer-power expansion), so on
// the same inputs they return the reference's values bit for bit:
//
//   k_grav_pairsum  getAcc_g_smth (sph_code/libsx.py:623-662),
//                   getAcc_g_smth_mpi (:667-705), getAcc_g_smthx (:710-747)
//                   and getAcc_g_smth_mimj_mpi (:908-947)
//   k_pe_rows       the per-row partial sums of getPE (:583-620)
//   k_kth_dist      do_smoothingX (:752-774) for query points that are not
//                   the particles themselves
//
// Why one kernel covers all four gravity forms: every form accumulates, for a
// row r, the terms t(r, k) = ((G fk) (x_k - x_r)) m_k over a set of sources
// k in ascending k.  getAcc_g_smth's j > i loop adds the reactions of the
// rows i < r (outer loop) before r's own j > r terms, i.e. ascending k; the
// row forms subtract G fk (x_r - x_k) m_k, which is the same number with its
// sign flipped exactly (IEEE negation is exact and a - b == a + (-b)); fk
// depends only on |x_r - x_k| and eps_r + eps_k, both symmetric.  The partial
// array of getAcc_g_smth_mimj_mpi(nbeg, nend) gives row r
//   nothing                 for r <  nbeg,
//   k in [nbeg, n), k != r  for nbeg <= r < nend (reactions, then own terms),
//   k in [nbeg, nend)       for r >= nend (reactions only).
#include "sph3_internal.cuh"

namespace sph3 {
namespace {

constexpr int kPsThreads = 128;   // rows per pair-sum block (one thread per row)
constexpr int kKthThreads = 256;  // threads per k-th-distance query

// numba's expansion of x**e for an integer literal e: r = 1; repeat { if the
// low bit of e is set: r = r * v; e >>= 1; if e: v = v * v }
__device__ __forceinline__ double ipow_rn(double x, int e) {
    double r = 1.0, v = x;
    while (e) {
        if (e & 1) r = __dmul_rn(r, v);
        e >>= 1;
        if (e) v = __dmul_rn(v, v);
    }
    return r;
}

// force kernel fk of libsx.py:640-652 with eps_ij = (eps_i + eps_j) / 2
__device__ __forceinline__ double ref_fk(double rr, double epsij) {
    const double q = __ddiv_rn(rr, epsij);
    if (q <= 1.0) {
        const double a = __dsub_rn(4.0 / 3.0, __dmul_rn(6.0 / 5.0, ipow_rn(q, 2)));
        return __dmul_rn(__ddiv_rn(1.0, ipow_rn(epsij, 3)), __dadd_rn(a, __dmul_rn(0.5, ipow_rn(q, 3))));
    }
    const double inv_r3 = __ddiv_rn(1.0, ipow_rn(rr, 3));
    if (q <= 2.0) {
        double s = __dadd_rn(-1.0 / 15.0, __dmul_rn(8.0 / 3.0, ipow_rn(q, 3)));
        s = __dsub_rn(s, __dmul_rn(3.0, ipow_rn(q, 4)));
        s = __dadd_rn(s, __dmul_rn(6.0 / 5.0, ipow_rn(q, 5)));
        s = __dsub_rn(s, __dmul_rn(1.0 / 6.0, ipow_rn(q, 6)));
        return __dmul_rn(inv_r3, s);
    }
    return inv_r3;
}

// m_j times the potential kernel of getPE (libsx.py:598-616); 0 for q = 0
__device__ __forceinline__ double ref_pk(double rr, double epsij, double mj) {
    const double q = __ddiv_rn(rr, epsij);
    double fk = 0.0;
    if (q <= 1.0 && q != 0.0) {
        double s = __dsub_rn(__dmul_rn(1.0 / 3.0, ipow_rn(q, 2)), __dmul_rn(3.0 / 20.0, ipow_rn(q, 4)));
        s = __dadd_rn(s, __dmul_rn(1.0 / 20.0, ipow_rn(q, 5)));
        const double t = __dadd_rn(__dmul_rn(__ddiv_rn(-2.0, epsij), s), __ddiv_rn(7.0 / 5.0, epsij));
        fk = __dmul_rn(mj, t);
    } else if (q > 1.0 && q <= 2.0) {
        const double inv_r = __ddiv_rn(1.0, rr);
        double s = __dsub_rn(__dmul_rn(4.0 / 3.0, ipow_rn(q, 2)), ipow_rn(q, 3));
        s = __dadd_rn(s, __dmul_rn(3.0 / 10.0, ipow_rn(q, 4)));
        s = __dsub_rn(s, __dmul_rn(1.0 / 30.0, ipow_rn(q, 5)));
        double t = __dsub_rn(__dmul_rn(-1.0 / 15.0, inv_r), __dmul_rn(__ddiv_rn(1.0, epsij), s));
        t = __dadd_rn(t, __ddiv_rn(8.0 / 5.0, epsij));
        fk = __dmul_rn(mj, t);
    } else if (q > 2.0) {
        fk = __dmul_rn(mj, __ddiv_rn(1.0, rr));
    }
    return fk;
}

// src: [5][n] x, y, z, m, eps in the caller's order.  Rows [row0, row1);
// row r sums the sources k in [kb, ke(r)), k != r, ascending, where
// ke(r) = n for r < split and split otherwise.  out: (row1 - row0) x 3.
__global__ void __launch_bounds__(kPsThreads) k_grav_pairsum(const double *__restrict__ src, int64_t n,
                                                             int64_t row0, int64_t row1, int64_t kb,
                                                             int64_t split, double G,
                                                             double *__restrict__ out) {
    __shared__ double sx[kPsThreads], sy[kPsThreads], sz[kPsThreads], sm[kPsThreads], se[kPsThreads];
    const int64_t rfirst = row0 + (int64_t)blockIdx.x * kPsThreads;
    const int64_t r = rfirst + threadIdx.x;
    const bool live = r < row1;
    const int64_t ke = !live ? kb : (r < split ? n : split);
    const int64_t blk_ke = rfirst < split ? n : split;  // the block's first row reaches furthest
    double xr = 0, yr = 0, zr = 0, er = 0;
    if (live) {
        xr = src[r];
        yr = src[n + r];
        zr = src[2 * n + r];
        er = src[4 * n + r];
    }
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int64_t t0 = kb; t0 < blk_ke; t0 += kPsThreads) {
        const int64_t k = t0 + threadIdx.x;
        if (k < blk_ke) {
            sx[threadIdx.x] = src[k];
            sy[threadIdx.x] = src[n + k];
            sz[threadIdx.x] = src[2 * n + k];
            sm[threadIdx.x] = src[3 * n + k];
            se[threadIdx.x] = src[4 * n + k];
        }
        __syncthreads();
        const int cnt = (int)(blk_ke - t0 < kPsThreads ? blk_ke - t0 : kPsThreads);
        if (live) {
            for (int t = 0; t < cnt; ++t) {
                const int64_t kk = t0 + t;
                if (kk == r || kk >= ke) continue;
                const double dx = __dsub_rn(sx[t], xr), dy = __dsub_rn(sy[t], yr), dz = __dsub_rn(sz[t], zr);
                const double rr = __dsqrt_rn(
                    __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
                const double fk = ref_fk(rr, __dmul_rn(0.5, __dadd_rn(er, se[t])));
                const double gf = __dmul_rn(G, fk);
                ax = __dadd_rn(ax, __dmul_rn(__dmul_rn(gf, dx), sm[t]));
                ay = __dadd_rn(ay, __dmul_rn(__dmul_rn(gf, dy), sm[t]));
                az = __dadd_rn(az, __dmul_rn(__dmul_rn(gf, dz), sm[t]));
            }
        }
        __syncthreads();
    }
    if (live) {
        out[3 * (r - row0) + 0] = ax;
        out[3 * (r - row0) + 1] = ay;
        out[3 * (r - row0) + 2] = az;
    }
}

// part[i] = sum over j > i, ascending, of -(G m_i) pk_ij m_j (the terms getPE
// subtracts in its row i); src as above
__global__ void __launch_bounds__(kPsThreads) k_pe_rows(const double *__restrict__ src, int64_t n, double G,
                                                        double *__restrict__ part) {
    __shared__ double sx[kPsThreads], sy[kPsThreads], sz[kPsThreads], sm[kPsThreads], se[kPsThreads];
    const int64_t rfirst = (int64_t)blockIdx.x * kPsThreads;
    const int64_t r = rfirst + threadIdx.x;
    const bool live = r < n;
    double xr = 0, yr = 0, zr = 0, er = 0, gm = 0;
    if (live) {
        xr = src[r];
        yr = src[n + r];
        zr = src[2 * n + r];
        er = src[4 * n + r];
        gm = __dmul_rn(G, src[3 * n + r]);
    }
    double pe = 0.0;
    for (int64_t t0 = rfirst + 1; t0 < n; t0 += kPsThreads) {
        const int64_t k = t0 + threadIdx.x;
        if (k < n) {
            sx[threadIdx.x] = src[k];
            sy[threadIdx.x] = src[n + k];
            sz[threadIdx.x] = src[2 * n + k];
            sm[threadIdx.x] = src[3 * n + k];
            se[threadIdx.x] = src[4 * n + k];
        }
        __syncthreads();
        const int cnt = (int)(n - t0 < kPsThreads ? n - t0 : kPsThreads);
        if (live) {
            for (int t = 0; t < cnt; ++t) {
                if (t0 + t <= r) continue;
                const double dx = __dsub_rn(xr, sx[t]), dy = __dsub_rn(yr, sy[t]), dz = __dsub_rn(zr, sz[t]);
                const double rr = __dsqrt_rn(
                    __dadd_rn(__dadd_rn(ipow_rn(dx, 2), ipow_rn(dy, 2)), ipow_rn(dz, 2)));
                const double fk = ref_pk(rr, __dmul_rn(0.5, __dadd_rn(er, se[t])), sm[t]);
                pe = __dsub_rn(pe, __dmul_rn(gm, fk));
            }
        }
        __syncthreads();
    }
    if (live) part[r] = pe;
}

// out[i] = 0.5 * (distance from query i to its (kth+1)-th nearest particle),
// the particle itself included when a query coincides with one: the value at
// index kth of the sorted distances, as np.sort(dist)[kth] in do_smoothingX.
// The squared distances are computed as the reference does and the kth one
// is found exactly by an 8-bit-digit radix select on their bit patterns
// (non-negative doubles order as unsigned integers); sqrt is monotone, so the
// kth distance is the root of the kth squared distance.
__global__ void __launch_bounds__(kKthThreads) k_kth_dist(const double *__restrict__ q, int64_t mq,
                                                          const double *__restrict__ pos, int64_t n, int64_t kth,
                                                          double *__restrict__ out) {
    __shared__ unsigned hist[256];
    __shared__ unsigned long long s_prefix;
    __shared__ long long s_rank;
    const int lane = threadIdx.x & 31;
    for (int64_t qi = blockIdx.x; qi < mq; qi += gridDim.x) {
        const double qx = q[3 * qi], qy = q[3 * qi + 1], qz = q[3 * qi + 2];
        unsigned long long prefix = 0ull;
        long long rank = kth;
        for (int shift = 56; shift >= 0; shift -= 8) {
            for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0u;
            __syncthreads();
            const unsigned long long hmask = shift == 56 ? 0ull : (~0ull << (shift + 8));
            for (int64_t j0 = 0; j0 < n; j0 += blockDim.x) {
                const int64_t j = j0 + threadIdx.x;
                unsigned bin = 256u;  // no bin
                if (j < n) {
                    const double dx = __dsub_rn(pos[j], qx);
                    const double dy = __dsub_rn(pos[n + j], qy);
                    const double dz = __dsub_rn(pos[2 * n + j], qz);
                    const double d2 =
                        __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                    const unsigned long long b = (unsigned long long)__double_as_longlong(d2);
                    if ((b & hmask) == prefix) bin = (unsigned)((b >> shift) & 255ull);
                }
                // one shared atomic per distinct bin of the warp
                const unsigned peers = __match_any_sync(kFull, bin);
                if (bin < 256u && lane == __ffs(peers) - 1) atomicAdd(&hist[bin], (unsigned)__popc(peers));
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                long long below = 0;
                int bin = 0;
                for (; bin < 255; ++bin) {
                    if (below + (long long)hist[bin] > rank) break;
                    below += hist[bin];
                }
                s_prefix = prefix | ((unsigned long long)bin << shift);
                s_rank = rank - below;
            }
            __syncthreads();
            prefix = s_prefix;
            rank = s_rank;
            __syncthreads();
        }
        if (threadIdx.x == 0) out[qi] = __dmul_rn(__dsqrt_rn(__longlong_as_double((long long)prefix)), 0.5);
    }
}

__global__ void k_caller_sources(const double *__restrict__ pos, const double *__restrict__ m,
                                 const double *__restrict__ eps, const int64_t *__restrict__ inv, int64_t n,
                                 double *__restrict__ dst) {
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = inv[r];
        dst[r] = pos[k];
        dst[n + r] = pos[n + k];
        dst[2 * n + r] = pos[2 * n + k];
        dst[3 * n + r] = m[k];
        dst[4 * n + r] = eps[k];
    }
}

}  // namespace

void launch_caller_sources(State &S, const int64_t *inv, double *dst, cudaStream_t st) {
    if (S.n == 0) return;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((S.n + 255) / 256, (int64_t)S.num_sms * 8));
    k_caller_sources<<<blocks, 256, 0, st>>>(S.pos, S.m, S.eps, inv, S.n, dst);
}

void launch_grav_pairsum(const double *src, int64_t n, int64_t row0, int64_t row1, int64_t kb, int64_t split,
                         double G, double *out, cudaStream_t st) {
    if (row1 <= row0) return;
    const int64_t blocks = (row1 - row0 + kPsThreads - 1) / kPsThreads;
    k_grav_pairsum<<<(unsigned)blocks, kPsThreads, 0, st>>>(src, n, row0, row1, kb, split, G, out);
}

void launch_pe_rows(const double *src, int64_t n, double G, double *part, cudaStream_t st) {
    if (n == 0) return;
    const int64_t blocks = (n + kPsThreads - 1) / kPsThreads;
    k_pe_rows<<<(unsigned)blocks, kPsThreads, 0, st>>>(src, n, G, part);
}

void launch_kth_dist(const double *q, int64_t mq, const State &S, int64_t kth, double *out, cudaStream_t st) {
    if (mq == 0) return;
    const int blocks = (int)std::min<int64_t>(mq, (int64_t)S.num_sms * 8);
    k_kth_dist<<<blocks, kKthThreads, 0, st>>>(q, mq, S.pos, S.n, kth, out);
}

}  // namespace sph3

// Leapfrog kick-drift-kick, the trapezoidal u update and the FP64 global sums.
// All FP64 (the time-integration accumulators), all HBM-bound streaming.
//
// Step order of the reference serial driver (sph_code/sph_serial.py:142-193):
//   v += a dt/2; r += v dt                       -> k_kick_drift
//   h, rho, a_g, P, c, du/dt(v_half)             -> walks
//   u = u_prev + dt/2 (ut + ut_prev)             -> k_kick_update (update_u)
//   a_sph; a = a_g + a_sph; v += a dt/2          -> k_kick_update (second_kick)
// The MPI driver (sph_code/sph_mpi4_v4.py:380-427) kicks first and computes
// du/dt with the full-step v; both orders are available.
#include <algorithm>
#include <cmath>

#include "sph3_internal.cuh"

namespace sph3 {

static int grid_for(const State &S, int64_t n) {
    return (int)std::min<int64_t>((n + 255) / 256, (int64_t)S.num_sms * 8);
}

__global__ void k_kick_drift(int64_t n, double dt, double *pos, double *vel, const double *acc,
                             double Lx, double Ly, double Lz) {
    const double L[3] = {Lx, Ly, Lz};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            // v + acc * dt / 2.0 and r + v * dt, rounded as NumPy does (no FMA)
            double v = __dadd_rn(vel[d * n + i], __dmul_rn(__dmul_rn(acc[d * n + i], dt), 0.5));
            double x = __dadd_rn(pos[d * n + i], __dmul_rn(v, dt));
            if (L[d] > 0.0) {
                if (x < 0.0) x += L[d];
                if (x >= L[d]) x -= L[d];
            }
            vel[d * n + i] = v;
            pos[d * n + i] = x;
        }
    }
}

void launch_kick_drift(State &S, const Params &P, double dt, cudaStream_t st) {
    if (S.n == 0) return;
    k_kick_drift<<<grid_for(S, S.n), 256, 0, st>>>(S.n, dt, S.pos, S.vel, S.acc, P.box[0], P.box[1], P.box[2]);
}

// the second kick (v += a dt / 2, a = a_g + a_sph) of sorted particle i
__device__ __forceinline__ void second_kick_one(int64_t n, int64_t i, double dt, double *acc, const double *acc_g,
                                                const double *acc_sph, double *vel, float4 *pk_vel) {
    float v3[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double a = acc_g[d * n + i] + acc_sph[d * n + i];
        acc[d * n + i] = a;
        const double v = __dadd_rn(vel[d * n + i], __dmul_rn(__dmul_rn(a, dt), 0.5));
        vel[d * n + i] = v;
        v3[d] = (float)v;
    }
    pk_vel[i] = make_float4(v3[0], v3[1], v3[2], 0.f);
}

__global__ void k_kick_update(int64_t n, double dt, int update_u, int second_kick, double *u,
                              double *u_prev, const double *dudt, double *dudt_prev, double *acc,
                              const double *acc_g, const double *acc_sph, double *vel, float4 *pk_vel) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (update_u) {
            const double ut = dudt[i];
            const double un = __dadd_rn(u_prev[i], __dmul_rn(__dmul_rn(0.5, dt), __dadd_rn(ut, dudt_prev[i])));
            u[i] = un;
            u_prev[i] = un;
            dudt_prev[i] = ut;
        }
        if (second_kick) second_kick_one(n, i, dt, acc, acc_g, acc_sph, vel, pk_vel);
    }
}

void launch_kick_update(State &S, const Params &P, double dt, bool update_u, bool second_kick,
                        cudaStream_t st) {
    (void)P;
    if (S.n == 0) return;
    k_kick_update<<<grid_for(S, S.n), 256, 0, st>>>(S.n, dt, update_u, second_kick, S.u, S.u_prev, S.dudt,
                                                   S.dudt_prev, S.acc, S.acc_g, S.acc_sph, S.vel, S.pk_vel);
}

// The second kick for the particles of caller rows [b, e) (the same
// arithmetic as k_kick_update's), so that a step can finish its particles
// chunk by chunk and hand each chunk to a copy as soon as it is done.
__global__ void k_kick_rows(int64_t n, double dt, const int64_t *inv, int64_t b, int64_t e, double *acc,
                            const double *acc_g, const double *acc_sph, double *vel, float4 *pk_vel) {
    for (int64_t r = b + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < e; r += (int64_t)gridDim.x * blockDim.x)
        second_kick_one(n, inv[r], dt, acc, acc_g, acc_sph, vel, pk_vel);
}

void launch_kick_rows(State &S, double dt, const int64_t *inv, int64_t b, int64_t e, cudaStream_t st) {
    if (e <= b) return;
    k_kick_rows<<<grid_for(S, e - b), 256, 0, st>>>(S.n, dt, inv, b, e, S.acc, S.acc_g, S.acc_sph, S.vel, S.pk_vel);
}

void launch_u_update(State &S, const Params &P, double dt, cudaStream_t st) {
    launch_kick_update(S, P, dt, true, false, st);
}

// first step (sph_serial.py:123-134): a = a_g + a_sph; u += du/dt dt;
// u_prev = u; dudt_prev = du/dt
__global__ void k_first_u(int64_t n, double dt, double *u, double *u_prev, const double *dudt,
                          double *dudt_prev, double *acc, const double *acc_g, const double *acc_sph) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int d = 0; d < 3; ++d) acc[d * n + i] = acc_g[d * n + i] + acc_sph[d * n + i];
        const double un = __dadd_rn(u[i], __dmul_rn(dudt[i], dt));
        u[i] = un;
        u_prev[i] = un;
        dudt_prev[i] = dudt[i];
    }
}

void launch_first_u(State &S, const Params &P, double dt, cudaStream_t st) {
    (void)P;
    if (S.n == 0) return;
    k_first_u<<<grid_for(S, S.n), 256, 0, st>>>(S.n, dt, S.u, S.u_prev, S.dudt, S.dudt_prev, S.acc, S.acc_g,
                                               S.acc_sph);
}

__global__ void k_sum_acc(int64_t n, double *acc, const double *acc_g, const double *acc_sph) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * n; i += (int64_t)gridDim.x * blockDim.x)
        acc[i] = acc_g[i] + acc_sph[i];
}

void launch_sum_acc(State &S, cudaStream_t st) {
    if (S.n == 0) return;
    k_sum_acc<<<grid_for(S, 3 * S.n), 256, 0, st>>>(S.n, S.acc, S.acc_g, S.acc_sph);
}

// ------------------------------------------------------------ energy
// Deterministic two-stage FP64 reduction: each of kEnergyBlocks blocks sums a
// fixed contiguous chunk, one block adds the partials in order.
constexpr int kEnergyBlocks = 296;

__global__ void __launch_bounds__(256) k_energy_part(int64_t n, const double *vel, const double *m,
                                                     const double *u, const double *phi, double *part) {
    const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const int64_t beg = (int64_t)blockIdx.x * chunk;
    const int64_t end = min(beg + chunk, n);
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
        const double mi = m[i];
        const double vx = vel[i], vy = vel[n + i], vz = vel[2 * n + i];
        s[0] += 0.5 * mi * (vx * vx + vy * vy + vz * vz);
        s[1] += mi * u[i];
        s[2] += 0.5 * mi * phi[i];
        s[4] += mi * vx;
        s[5] += mi * vy;
        s[6] += mi * vz;
        s[7] += mi;
    }
    __shared__ double red[8][8];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        double v = warp_sum(s[q]);
        if (lane == 0) red[q][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        double t = 0;
        for (int k = 0; k < 8; ++k) t += red[threadIdx.x][k];
        part[blockIdx.x * 8 + threadIdx.x] = t;
    }
}

// one warp per sum: lane l adds the partials l, l + 32, ... in order, then a
// fixed butterfly combines the lanes (the same order every call)
__global__ void __launch_bounds__(256) k_energy_final(const double *part, int nb, double *out) {
    __shared__ double tot[8];
    const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double t = 0;
    for (int b = lane; b < nb; b += 32) t += part[b * 8 + q];
    t = warp_sum(t);
    if (lane == 0) tot[q] = t;
    __syncthreads();
    if (threadIdx.x < 8) out[threadIdx.x] = threadIdx.x == 3 ? tot[0] + tot[1] + tot[2] : tot[threadIdx.x];
}

void launch_energy(State &S, const Params &P, cudaStream_t st) {
    (void)P;
    if (S.n == 0) {
        cudaMemsetAsync(S.energy, 0, sizeof(double) * 8, st);
        return;
    }
    k_energy_part<<<kEnergyBlocks, 256, 0, st>>>(S.n, S.vel, S.m, S.u, S.phi, S.energy_part);
    k_energy_final<<<1, 256, 0, st>>>(S.energy_part, kEnergyBlocks, S.energy);
}

// ------------------------------------------------------------ time step
// Per-particle time-step estimate of the reference's dt_array_indiv_dt
// (Particles_in_BH_Tree_III/Evrard_Collapse_2024/hfvCLibs_v7_hfv_v8.1.h:
// 1189-1262), in FP64: dt_i = min(dt_hyd, dt_cour, dt_f, dt_kin, dt_G1, dt_G2)
// with dt_hyd = C h / max_j vsig_ij, dt_cour = C h / (h |divV| + max(c, |v|)
// (1 + 0.6 alpha)), dt_f = sqrt(h / |a_g|), dt_kin = sqrt(h / |a|),
// dt_G1 = 0.4 sqrt(eps / |a|), dt_G2 = 0.4 eps / |v|; dh/dt = h divV / 3.

// signal-velocity maximum over every particle of the same system (the
// reference's all-pairs loop): one block per target row, FP64
__global__ void __launch_bounds__(256) k_vsig_all(const Cloud *clouds, int ncloud, const double *pos,
                                                  const double *vel, const double *c, int64_t n,
                                                  double *vsig) {
    __shared__ double red[8];
    for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
        int lo = 0, hi = ncloud - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (clouds[mid].begin <= i) lo = mid;
            else hi = mid - 1;
        }
        const Cloud &cl = clouds[lo];
        const double xi = pos[i], yi = pos[n + i], zi = pos[2 * n + i];
        const double vxi = vel[i], vyi = vel[n + i], vzi = vel[2 * n + i], ci = c[i];
        double m = 0.0;
        for (int64_t j = cl.begin + threadIdx.x; j < cl.end; j += blockDim.x) {
            const double dx = xi - pos[j], dy = yi - pos[n + j], dz = zi - pos[2 * n + j];
            const double rr = sqrt(dx * dx + dy * dy + dz * dz);
            const double vr = (vxi - vel[j]) * dx + (vyi - vel[n + j]) * dy + (vzi - vel[2 * n + j]) * dz;
            const double sig = ci + c[j] - 3.0 * (vr / (rr + 1e-5));
            m = fmax(m, sig);
        }
        m = warp_max(m);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmax(t, red[w]);
            vsig[i] = t;
        }
        __syncthreads();
    }
}

constexpr int kDtBlocks = 296;

__global__ void __launch_bounds__(256) k_timestep(int64_t n, const double *vel, const double *acc,
                                                  const double *acc_g, const double *h, const double *c,
                                                  const double *divV, const double *eps, const double *vsig,
                                                  double c_cfl, double alpha, double *dt, double *dhdt,
                                                  double *part) {
    double lmin = INFINITY;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double ag = sqrt(acc_g[i] * acc_g[i] + acc_g[n + i] * acc_g[n + i] + acc_g[2 * n + i] * acc_g[2 * n + i]);
        const double at = sqrt(acc[i] * acc[i] + acc[n + i] * acc[n + i] + acc[2 * n + i] * acc[2 * n + i]);
        const double av = sqrt(vel[i] * vel[i] + vel[n + i] * vel[n + i] + vel[2 * n + i] * vel[2 * n + i]);
        const double hi = h[i], ci = c[i], ei = eps[i];
        const double d[6] = {c_cfl * hi / vsig[i],
                             c_cfl * hi / (hi * fabs(divV[i]) + fmax(ci, av) * (1.0 + 0.6 * alpha)),
                             sqrt(hi / ag),
                             sqrt(hi / at),
                             0.4 * sqrt(ei / at),
                             0.4 * ei / av};
        double m = d[0];
#pragma unroll
        for (int k = 0; k < 6; ++k)
            if (d[k] <= m) m = d[k];
        dt[i] = m;
        dhdt[i] = 1.0 / 3.0 * hi * divV[i];
        lmin = fmin(lmin, m);
    }
    __shared__ double red[8];
    lmin = warp_min(lmin);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = lmin;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = INFINITY;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmin(t, red[w]);
        part[blockIdx.x] = t;
    }
}

__global__ void k_min_final(const double *part, int nb, double *out) {
    if (threadIdx.x == 0) {
        double t = INFINITY;
        for (int b = 0; b < nb; ++b) t = fmin(t, part[b]);
        *out = t;
    }
}

void launch_timestep(State &S, const Params &P, double c_cfl, bool all_pairs, double *dt_min_dev,
                     cudaStream_t st) {
    if (S.n == 0) return;
    if (all_pairs) {
        const int blocks = (int)std::min<int64_t>(S.n, (int64_t)S.num_sms * 16);
        k_vsig_all<<<blocks, 256, 0, st>>>(S.clouds, S.ncloud, S.pos, S.vel, S.c, S.n, S.vsig);
    }
    k_timestep<<<kDtBlocks, 256, 0, st>>>(S.n, S.vel, S.acc, S.acc_g, S.h, S.c, S.divV, S.eps, S.vsig, c_cfl,
                                          P.alpha, S.dt, S.dhdt, S.energy_part);
    k_min_final<<<1, 32, 0, st>>>(S.energy_part, kDtBlocks, dt_min_dev);
}

// non-finite velocity, mass, u or h -> SPH3_STATUS_NAN_INPUT (positions are
// checked while the root cubes are computed)
__global__ void k_check_finite(int64_t n, const double *vel, const double *m, const double *u,
                               const double *h, unsigned *status) {
    int bad = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        bad |= !isfinite(vel[i]) | !isfinite(vel[n + i]) | !isfinite(vel[2 * n + i]);
        bad |= !isfinite(m[i]) | !isfinite(u[i]) | !isfinite(h[i]);
    }
    if (__any_sync(kFull, bad) && (threadIdx.x & 31) == 0) atomicOr(status, SPH3_STATUS_NAN_INPUT);
}

void launch_check_finite(State &S, cudaStream_t st) {
    if (S.n == 0) return;
    k_check_finite<<<grid_for(S, S.n), 256, 0, st>>>(S.n, S.vel, S.m, S.u, S.h, S.status);
}

}  // namespace sph3

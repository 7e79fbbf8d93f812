/*
 * CPU oracle for the SPH_3 per-step particle path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C with FP64 arithmetic, the all-pairs numba
 * functions of the reference's CPU library (sph_code/libsx.py and
 * sph_code/shear.py).  It exists so that the tests, the smoke check and the
 * CPU-baseline leg of the benchmark have a checker; nothing in the product
 * (sph_3_b200/) links to it.
 *
 * Faithfulness rules (so that results agree bit-for-bit with the numba
 * originals on the committed golden vectors):
 *   - every row keeps the reference's j = 0..N-1 summation order;
 *   - expressions keep the reference's operation order, and the file is
 *     compiled with -ffp-contract=off (numba/LLVM do not fuse a*b+c);
 *   - integer powers x**n use the same left-to-right binary exponentiation
 *     that numba unrolls for a constant integer exponent (ipow below);
 *   - x**0.5 is the correctly rounded square root.
 * Rows are processed in parallel with OpenMP; each row is independent, so the
 * result does not depend on the thread count.
 *
 * Additions that the reference does not have (each one reduces to the
 * reference when left at its default):
 *   - a `rows` index list instead of the contiguous [nbeg, nend) of the
 *     *_mpi functions (a contiguous list reproduces them);
 *   - a periodic minimum-image displacement when box[k] > 0 (box = 0: none);
 *   - an iteration cap on the h search (the reference loops without bound).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define SIG_M4 (1.0 / 3.141592653589793)

/* numba's unrolled integer power: r = 1; while e: if e&1: r *= v; e >>= 1; v *= v */
static inline double ipow(double x, int e) {
    double r = 1.0, v = x;
    while (e) {
        if (e & 1) r = r * v;
        e >>= 1;
        if (e) v = v * v;
    }
    return r;
}

/* periodic minimum image of one displacement component; no-op for L <= 0 */
static inline double min_image(double d, double L) {
    if (L > 0.0) {
        if (d > 0.5 * L) d -= L;
        else if (d < -0.5 * L) d += L;
    }
    return d;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* M4 gradient factor nW (gradW = nW * (x_i - x_j)); follows
 * sph_code/libsx.py:127-141 (identical in every hydro function). */
static inline double m4_grad_factor(double q, double hij) {
    double nW = 0.0;
    if (q <= 1.0) {
        nW = SIG_M4 / ipow(hij, 5) * (-3.0 + 9.0 / 4.0 * q);
    }
    if ((q > 1.0) && (q <= 2.0)) {
        nW = -3.0 * SIG_M4 / 4.0 / ipow(hij, 5) * ipow(2.0 - q, 2) / (q + 1e-20);
    }
    return nW;
}

/* ---------------------------------------------------------------- density
 * getDensity / getDensity_mpi, sph_code/libsx.py:10-44, 50-86. */
void orc_density(int64_t n, const double *pos, const double *m, const double *h,
                 const int64_t *rows, int64_t nrows, const double *box, double *rho) {
    const double bx = box ? box[0] : 0.0, by = box ? box[1] : 0.0, bz = box ? box[2] : 0.0;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t r = 0; r < nrows; ++r) {
        int64_t i = rows[r];
        double s = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            double dx = min_image(pos[3 * i + 0] - pos[3 * j + 0], bx);
            double dy = min_image(pos[3 * i + 1] - pos[3 * j + 1], by);
            double dz = min_image(pos[3 * i + 2] - pos[3 * j + 2], bz);
            double rr = sqrt(ipow(dx, 2) + ipow(dy, 2) + ipow(dz, 2));
            double hij = 0.5 * (h[i] + h[j]);
            double q = rr / hij;
            double W = 0.0;
            if (q <= 1.0) W = SIG_M4 / ipow(hij, 3) * (1.0 - (3.0 / 2.0) * ipow(q, 2) + (3.0 / 4.0) * ipow(q, 3));
            if ((q > 1.0) && (q <= 2.0)) W = SIG_M4 / ipow(hij, 3) * (1.0 / 4.0) * ipow(2.0 - q, 3);
            s += m[j] * W;
        }
        rho[r] = s;
    }
}

/* Neighbour set of one row: every j with q = |r_ij| / hbar_ij <= 2, the
 * support of all reference hydro kernels (sph_code/libsx.py:34-38).  Writes at
 * most cap indices (ascending j) and returns the full count. */
int64_t orc_neighbours(int64_t n, const double *pos, const double *h, int64_t i,
                       const double *box, int64_t *out, int64_t cap) {
    const double bx = box ? box[0] : 0.0, by = box ? box[1] : 0.0, bz = box ? box[2] : 0.0;
    int64_t k = 0;
    for (int64_t j = 0; j < n; ++j) {
        double dx = min_image(pos[3 * i + 0] - pos[3 * j + 0], bx);
        double dy = min_image(pos[3 * i + 1] - pos[3 * j + 1], by);
        double dz = min_image(pos[3 * i + 2] - pos[3 * j + 2], bz);
        double rr = sqrt(ipow(dx, 2) + ipow(dy, 2) + ipow(dz, 2));
        double hij = 0.5 * (h[i] + h[j]);
        double q = rr / hij;
        if (q <= 2.0) {
            if (k < cap) out[k] = j;
            ++k;
        }
    }
    return k;
}

/* ------------------------------------------------------------- h search
 * h_smooth_fast / h_smooth_fast_mpi, sph_code/libsx.py:804-845, 852-902:
 * count N(dist < 2h) including the particle itself, step h by -/+0.3% until
 * N is in [n_ngb - tol, n_ngb + tol].  The reference fixes n_ngb=50, tol=5 and
 * has no cap; status[r] = number of steps taken, or -1 if max_iter was hit
 * (h is then the value after max_iter steps).
 * The count over all N uses the sorted distance list (same predicate, same
 * result as np.sum(dist < 2h)). */
static int cmp_double(const void *a, const void *b) {
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

static int64_t count_below(const double *sorted, int64_t n, double t) {
    /* number of elements strictly below t */
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (sorted[mid] < t) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

static void select_kth(double *a, int64_t n, int64_t k) {
    int64_t lo = 0, hi = n - 1;
    while (lo < hi) {
        double pivot = a[(lo + hi) >> 1];
        int64_t i = lo, j = hi;
        while (i <= j) {
            while (a[i] < pivot) ++i;
            while (a[j] > pivot) --j;
            if (i <= j) { double t = a[i]; a[i] = a[j]; a[j] = t; ++i; --j; }
        }
        if (k <= j) hi = j;
        else if (k >= i) lo = i;
        else break;
    }
}

/* count of dist[] < t where dist[0..K) holds the K smallest values sorted */
static int64_t count_prefix(const double *dist, int64_t n, int64_t K, double t) {
    if (K == n || (K > 0 && t <= dist[K - 1])) return count_below(dist, K, t);
    int64_t k = 0;
    for (int64_t j = 0; j < n; ++j) k += dist[j] < t;
    return k;
}

void orc_h_smooth(int64_t n, const double *pos, const double *h_in, const int64_t *rows,
                  int64_t nrows, int n_ngb, int tol, int64_t max_iter, const double *box,
                  double *h_out, int64_t *status) {
    const double bx = box ? box[0] : 0.0, by = box ? box[1] : 0.0, bz = box ? box[2] : 0.0;
    const int64_t up = n_ngb + tol, low = n_ngb - tol;
#pragma omp parallel
    {
        double *dist = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
#pragma omp for schedule(dynamic, 4)
        for (int64_t r = 0; r < nrows; ++r) {
            int64_t i = rows[r];
            double hi = h_in[i];
            for (int64_t j = 0; j < n; ++j) {
                double dx = min_image(pos[3 * j + 0] - pos[3 * i + 0], bx);
                double dy = min_image(pos[3 * j + 1] - pos[3 * i + 1], by);
                double dz = min_image(pos[3 * j + 2] - pos[3 * i + 2], bz);
                dist[j] = sqrt(dx * dx + dy * dy + dz * dz);
            }
            /* the first count is one pass over the distances, as the
             * reference's np.sum(dist < 2h); only a row that has to iterate
             * sorts its K smallest distances, so that every further count
             * below t <= dist[K-1] is exact on that prefix (larger t falls
             * back to a full scan) */
            int64_t nn = 0;
            for (int64_t j = 0; j < n; ++j) nn += dist[j] < 2.0 * hi;
            int64_t K = n;
            if ((nn > up) || (nn < low)) {
                K = n < 2048 ? n : 2048;
                if (K < n) select_kth(dist, n, K - 1);
                qsort(dist, (size_t)K, sizeof(double), cmp_double);
            }
            int64_t it = 0;
            while ((nn > up) || (nn < low)) {
                if (it >= max_iter) { it = -1; break; }
                if (nn > up) hi -= 0.003 * hi;
                if (nn < low) hi += 0.003 * hi;
                nn = count_prefix(dist, n, K, 2.0 * hi);
                ++it;
            }
            h_out[r] = hi;
            if (status) status[r] = it;
        }
        free(dist);
    }
}

/* Neighbour count N(dist < 2h) of each row with the row's own h. */
void orc_count_within(int64_t n, const double *pos, const double *h, const int64_t *rows,
                      int64_t nrows, const double *box, int64_t *count) {
    const double bx = box ? box[0] : 0.0, by = box ? box[1] : 0.0, bz = box ? box[2] : 0.0;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t r = 0; r < nrows; ++r) {
        int64_t i = rows[r];
        double t = 2.0 * h[i];
        int64_t k = 0;
        for (int64_t j = 0; j < n; ++j) {
            double dx = min_image(pos[3 * j + 0] - pos[3 * i + 0], bx);
            double dy = min_image(pos[3 * j + 1] - pos[3 * i + 1], by);
            double dz = min_image(pos[3 * j + 2] - pos[3 * i + 2], bz);
            if (sqrt(dx * dx + dy * dy + dz * dz) < t) ++k;
        }
        count[r] = k;
    }
}

/* smoothing_length_mpi / do_smoothingX, sph_code/libsx.py:752-800:
 * h = 0.5 * (k-th smallest distance, self included; the reference uses k=50). */
void orc_smoothing_length(int64_t n, const double *pos, const int64_t *rows, int64_t nrows,
                          int k, const double *box, double *h_out) {
    const double bx = box ? box[0] : 0.0, by = box ? box[1] : 0.0, bz = box ? box[2] : 0.0;
#pragma omp parallel
    {
        double *dist = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
#pragma omp for schedule(dynamic, 4)
        for (int64_t r = 0; r < nrows; ++r) {
            int64_t i = rows[r];
            for (int64_t j = 0; j < n; ++j) {
                double dx = min_image(pos[3 * j + 0] - pos[3 * i + 0], bx);
                double dy = min_image(pos[3 * j + 1] - pos[3 * i + 1], by);
                double dz = min_image(pos[3 * j + 2] - pos[3 * i + 2], bz);
                dist[j] = sqrt(ipow(dx, 2) + ipow(dy, 2) + ipow(dz, 2));
            }
            int64_t kk = k < n ? k : n - 1;
            select_kth(dist, n, kk);
            h_out[r] = dist[kk] * 0.5;
        }
        free(dist);
    }
}

/* -------------------------------------------------------- div / curl v
 * div_curlVel / div_curlVel_mpi, sph_code/shear.py:7-69, 76-142. */
void orc_div_curl(int64_t n, const double *pos, const double *v, const double *rho,
                  const double *m, const double *h, const int64_t *rows, int64_t nrows,
                  const double *box, double *divV, double *curlV) {
    const double bx = box ? box[0] : 0.0, by = box ? box[1] : 0.0, bz = box ? box[2] : 0.0;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t r = 0; r < nrows; ++r) {
        int64_t i = rows[r];
        double s = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            double dx = min_image(pos[3 * i + 0] - pos[3 * j + 0], bx);
            double dy = min_image(pos[3 * i + 1] - pos[3 * j + 1], by);
            double dz = min_image(pos[3 * i + 2] - pos[3 * j + 2], bz);
            double rr = sqrt(ipow(dx, 2) + ipow(dy, 2) + ipow(dz, 2));
            double hij = 0.5 * (h[i] + h[j]);
            double q = rr / hij;
            double nW = m4_grad_factor(q, hij);
            double gWx = 0.0, gWy = 0.0, gWz = 0.0;
            if (q <= 2.0) { gWx = nW * dx; gWy = nW * dy; gWz = nW * dz; }
            double vxji = v[3 * j + 0] - v[3 * i + 0];
            double vyji = v[3 * j + 1] - v[3 * i + 1];
            double vzji = v[3 * j + 2] - v[3 * i + 2];
            s += m[j] / rho[i] * (vxji * gWx + vyji * gWy + vzji * gWz);
            double vxij = v[3 * i + 0] - v[3 * j + 0];
            double vyij = v[3 * i + 1] - v[3 * j + 1];
            double vzij = v[3 * i + 2] - v[3 * j + 2];
            cx += m[j] / rho[i] * (vyij * gWz - vzij * gWy);
            cy += m[j] / rho[i] * (vzij * gWx - vxij * gWz);
            cz += m[j] / rho[i] * (vxij * gWy - vyij * gWx);
        }
        divV[r] = fabs(s);
        curlV[r] = sqrt(cx * cx + cy * cy + cz * cz);
    }
}

/* ------------------------------------------------ hydro accel and du/dt
 * visc = 0: signal-velocity viscosity of getAcc_sph / get_dU
 *           (sph_code/libsx.py:100-177, 268-347, 353-421, 496-564);
 * visc = 1: Monaghan & Gingold (1983) form of getAcc_sph_mpiXXX /
 *           get_dU_mpiXXXX (sph_code/libsx.py:183-262, 427-491);
 * visc = 2: signal form times the Balsara factor of getAcc_sph_shear /
 *           get_dU_shear (sph_code/shear.py:149-235, 332-406).
 * acc (3 per row) and/or dudt may be NULL. */
/* One row of getAcc_sph / get_dU; want_acc and want_dudt are constants at
 * every call site, so each specialisation computes only the terms of the
 * outputs it keeps (as the reference's two separate functions do), with the
 * same operations for those. */
static inline __attribute__((always_inline)) void hydro_row(
    int64_t n, const double *pos, const double *v, const double *rho, const double *P, const double *c,
    const double *h, const double *m, const double *divV, const double *curlV, int visc, double alpha,
    double beta, double eta, int64_t i, double bx, double by, double bz, int want_acc, int want_dudt,
    double *acc_r, double *dudt_r) {
    double axt = 0.0, ayt = 0.0, azt = 0.0, du_t = 0.0;
    for (int64_t j = 0; j < n; ++j) {
        double dx = min_image(pos[3 * i + 0] - pos[3 * j + 0], bx);
        double dy = min_image(pos[3 * i + 1] - pos[3 * j + 1], by);
        double dz = min_image(pos[3 * i + 2] - pos[3 * j + 2], bz);
        double rr = sqrt(ipow(dx, 2) + ipow(dy, 2) + ipow(dz, 2));
        double hij = 0.5 * (h[i] + h[j]);
        double q = rr / hij;
        double nW = m4_grad_factor(q, hij);
        double gWx = 0.0, gWy = 0.0, gWz = 0.0;
        if (q <= 2.0) { gWx = nW * dx; gWy = nW * dy; gWz = nW * dz; }
        double vxij = v[3 * i + 0] - v[3 * j + 0];
        double vyij = v[3 * i + 1] - v[3 * j + 1];
        double vzij = v[3 * i + 2] - v[3 * j + 2];
        double vij_gWij = vxij * gWx + vyij * gWy + vzij * gWz;
        double vij_rij = vxij * dx + vyij * dy + vzij * dz;
        double cij = 0.5 * (c[i] + c[j]);
        double rhoij = 0.5 * (rho[i] + rho[j]);
        double PIij = 0.0;
        if (visc == 1) {
            double muij = hij * vij_rij / (rr * rr + hij * hij * eta * eta);
            if (vij_rij <= 0) PIij = (-alpha * cij * muij + beta * muij * muij) / rhoij;
        } else {
            double wij = vij_rij / (rr + 1e-5);
            double vij_sig = c[i] + c[j] - 3.0 * wij;
            if (vij_rij <= 0) PIij = -0.5 * alpha * vij_sig * wij / rhoij;
            if (visc == 2) {
                double fi = divV[i] / (divV[i] + curlV[i] + 0.0001 * c[i] / h[i]);
                double fj = divV[j] / (divV[j] + curlV[j] + 0.0001 * c[j] / h[j]);
                double fij = 0.5 * (fi + fj);
                PIij = fij * PIij;
            }
        }
        if (want_acc) {
            double pterm = P[i] / ipow(rho[i], 2) + P[j] / ipow(rho[j], 2) + PIij;
            axt -= m[j] * pterm * gWx;
            ayt -= m[j] * pterm * gWy;
            azt -= m[j] * pterm * gWz;
        }
        if (want_dudt) du_t += m[j] * (P[i] / ipow(rho[i], 2) + PIij / 2.) * vij_gWij;
    }
    if (want_acc) { acc_r[0] = axt; acc_r[1] = ayt; acc_r[2] = azt; }
    if (want_dudt) *dudt_r = du_t;
}

void orc_hydro(int64_t n, const double *pos, const double *v, const double *rho,
               const double *P, const double *c, const double *h, const double *m,
               const double *divV, const double *curlV, int visc, double alpha, double beta,
               double eta, const int64_t *rows, int64_t nrows, const double *box,
               double *acc, double *dudt) {
    const double bx = box ? box[0] : 0.0, by = box ? box[1] : 0.0, bz = box ? box[2] : 0.0;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t r = 0; r < nrows; ++r) {
        const int64_t i = rows[r];
        double *ar = acc ? acc + 3 * r : NULL, *dr = dudt ? dudt + r : NULL;
        if (acc && dudt)
            hydro_row(n, pos, v, rho, P, c, h, m, divV, curlV, visc, alpha, beta, eta, i, bx, by, bz, 1, 1, ar, dr);
        else if (acc)
            hydro_row(n, pos, v, rho, P, c, h, m, divV, curlV, visc, alpha, beta, eta, i, bx, by, bz, 1, 0, ar, dr);
        else if (dudt)
            hydro_row(n, pos, v, rho, P, c, h, m, divV, curlV, visc, alpha, beta, eta, i, bx, by, bz, 0, 1, ar, dr);
    }
}

/* --------------------------------------------------------------- gravity
 * Spline-softened direct sum, row form of getAcc_g_smth_mpi / getAcc_g_smthx
 * (sph_code/libsx.py:667-705, 710-747): a_i = -sum_{j != i} G fk (x_i - x_j) m_j
 * with eps_ij = (eps_i + eps_j) / 2.  phi (may be NULL) is the matching
 * potential with getPE's kernel (sph_code/libsx.py:583-620), without G*m_i
 * (a coincident pair adds 0 to phi, as its q = 0 case does in getPE).
 * A coincident pair (r = 0, j != i) contributes nothing, where the reference
 * raises ZeroDivisionError. */
static inline double grav_fk(double rr, double epsij) {
    double q = rr / epsij;
    double fk;
    if (q <= 1.0) {
        fk = (1.0 / ipow(epsij, 3)) * ((4.0 / 3.0) - (6.0 / 5.0) * ipow(q, 2) + (1.0 / 2.0) * ipow(q, 3));
    } else {
        double inv_r3 = 1.0 / ipow(rr, 3);
        if (q <= 2.0)
            fk = inv_r3 * ((-1.0 / 15.0) + (8.0 / 3.0) * ipow(q, 3) - 3.0 * ipow(q, 4) + (6.0 / 5.0) * ipow(q, 5) - (1.0 / 6.0) * ipow(q, 6));
        else
            fk = inv_r3;
    }
    return fk;
}

static inline double grav_pk(double rr, double epsij) {
    /* potential kernel of getPE (positive; phi = -G * sum m_j pk) */
    double q = rr / epsij;
    double inv_r = rr != 0.0 ? 1.0 / rr : 0.0;
    double fk = 0.0;
    if ((q <= 1.0) && (q != 0.0))
        fk = ((-2.0 / epsij) * ((1.0 / 3.0) * ipow(q, 2) - (3.0 / 20.0) * ipow(q, 4) + (1.0 / 20.0) * ipow(q, 5)) + 7.0 / 5.0 / epsij);
    if ((q > 1.) && (q <= 2.))
        fk = ((-1.0 / 15.0) * inv_r - (1.0 / epsij) * ((4.0 / 3.0) * ipow(q, 2) - ipow(q, 3) + (3.0 / 10.0) * ipow(q, 4) - (1.0 / 30.0) * ipow(q, 5)) + 8.0 / 5.0 / epsij);
    if (q > 2.) fk = inv_r;
    return fk;
}

void orc_grav_direct(int64_t n, const double *pos, const double *mass, double G,
                     const double *eps, const int64_t *rows, int64_t nrows, double *acc,
                     double *phi) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t r = 0; r < nrows; ++r) {
        int64_t i = rows[r];
        double fx = 0.0, fy = 0.0, fz = 0.0, ph = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            if (i == j) continue;
            double dx = pos[3 * i + 0] - pos[3 * j + 0];
            double dy = pos[3 * i + 1] - pos[3 * j + 1];
            double dz = pos[3 * i + 2] - pos[3 * j + 2];
            double rr = sqrt(dx * dx + dy * dy + dz * dz);
            double epsij = 0.5 * (eps[i] + eps[j]);
            if (rr > 0.0) {
                double fk = grav_fk(rr, epsij);
                fx -= G * fk * dx * mass[j];
                fy -= G * fk * dy * mass[j];
                fz -= G * fk * dz * mass[j];
            }
            if (phi) {
                ph -= G * mass[j] * grav_pk(rr, epsij);
            }
        }
        acc[3 * r + 0] = fx; acc[3 * r + 1] = fy; acc[3 * r + 2] = fz;
        if (phi) phi[r] = ph;
    }
}

/* Pairwise-symmetric form of getAcc_g_smth (sph_code/libsx.py:623-662): the
 * j > i loop with both updates, serial (its sums depend on the order). */
void orc_grav_sym(int64_t n, const double *pos, const double *mass, double G,
                  const double *eps, double *field) {
    memset(field, 0, sizeof(double) * 3 * (size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t j = i + 1; j < n; ++j) {
            double dx = pos[3 * j + 0] - pos[3 * i + 0];
            double dy = pos[3 * j + 1] - pos[3 * i + 1];
            double dz = pos[3 * j + 2] - pos[3 * i + 2];
            double rr = sqrt(dx * dx + dy * dy + dz * dz);
            double epsij = 0.5 * (eps[i] + eps[j]);
            double q = rr / epsij;
            double fk;
            if (q <= 1.0) {
                fk = (1.0 / ipow(epsij, 3)) * ((4.0 / 3.0) - (6.0 / 5.0) * ipow(q, 2) + (1.0 / 2.0) * ipow(q, 3));
            } else {
                double inv_r3 = 1.0 / ipow(rr, 3);
                if (q <= 2.)
                    fk = inv_r3 * ((-1.0 / 15.0) + (8.0 / 3.0) * ipow(q, 3) - 3.0 * ipow(q, 4) + (6.0 / 5.0) * ipow(q, 5) - (1.0 / 6.0) * ipow(q, 6));
                else
                    fk = inv_r3;
            }
            field[3 * i + 0] += G * fk * dx * mass[j];
            field[3 * j + 0] -= G * fk * dx * mass[i];
            field[3 * i + 1] += G * fk * dy * mass[j];
            field[3 * j + 1] -= G * fk * dy * mass[i];
            field[3 * i + 2] += G * fk * dz * mass[j];
            field[3 * j + 2] -= G * fk * dz * mass[i];
        }
    }
}

/* getAcc_g_smth_mimj_mpi, sph_code/libsx.py:908-947: the (n, 3) partial
 * field of the rows i in [nbeg, nend) (their j > i terms) and the reactions
 * on the rows j > i, serial in the reference's loop order. */
void orc_grav_mimj(int64_t n, const double *pos, const double *mass, double G,
                   const double *eps, int64_t nbeg, int64_t nend, double *field) {
    memset(field, 0, sizeof(double) * 3 * (size_t)n);
    for (int64_t i = nbeg; i < nend; ++i) {
        for (int64_t j = i + 1; j < n; ++j) {
            double dx = pos[3 * j + 0] - pos[3 * i + 0];
            double dy = pos[3 * j + 1] - pos[3 * i + 1];
            double dz = pos[3 * j + 2] - pos[3 * i + 2];
            double rr = sqrt(dx * dx + dy * dy + dz * dz);
            double fk = grav_fk(rr, 0.5 * (eps[i] + eps[j]));
            field[3 * i + 0] += G * fk * dx * mass[j];
            field[3 * j + 0] -= G * fk * dx * mass[i];
            field[3 * i + 1] += G * fk * dy * mass[j];
            field[3 * j + 1] -= G * fk * dy * mass[i];
            field[3 * i + 2] += G * fk * dz * mass[j];
            field[3 * j + 2] -= G * fk * dz * mass[i];
        }
    }
}

/* do_smoothingX((pos, subpos)), sph_code/libsx.py:752-774: for each of the m
 * query points, 0.5 * (the k-th smallest distance to the n points of pos,
 * 0-based; the reference uses k = 50). */
void orc_smoothing_points(int64_t n, const double *pos, int64_t m, const double *q, int k,
                          double *h_out) {
#pragma omp parallel
    {
        double *dist = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
#pragma omp for schedule(dynamic, 4)
        for (int64_t r = 0; r < m; ++r) {
            for (int64_t j = 0; j < n; ++j) {
                double dx = pos[3 * j + 0] - q[3 * r + 0];
                double dy = pos[3 * j + 1] - q[3 * r + 1];
                double dz = pos[3 * j + 2] - q[3 * r + 2];
                dist[j] = sqrt(ipow(dx, 2) + ipow(dy, 2) + ipow(dz, 2));
            }
            int64_t kk = k < n ? k : n - 1;
            select_kth(dist, n, kk);
            h_out[r] = dist[kk] * 0.5;
        }
        free(dist);
    }
}

/* getPE, sph_code/libsx.py:583-620 (serial j > i double loop). */
double orc_pe(int64_t n, const double *pos, const double *m, double G, const double *eps) {
    double PE = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t j = i + 1; j < n; ++j) {
            double dx = pos[3 * i + 0] - pos[3 * j + 0];
            double dy = pos[3 * i + 1] - pos[3 * j + 1];
            double dz = pos[3 * i + 2] - pos[3 * j + 2];
            double rr = sqrt(ipow(dx, 2) + ipow(dy, 2) + ipow(dz, 2));
            double epsij = 0.5 * (eps[i] + eps[j]);
            double fk = 0.0;
            double q = rr / epsij;
            double inv_r = rr != 0.0 ? 1.0 / rr : 0.0;
            if ((q <= 1.0) && (q != 0.0))
                fk = m[j] * ((-2.0 / epsij) * ((1.0 / 3.0) * ipow(q, 2) - (3.0 / 20.0) * ipow(q, 4) + (1.0 / 20.0) * ipow(q, 5)) + 7.0 / 5.0 / epsij);
            if ((q > 1.) && (q <= 2.))
                fk = m[j] * ((-1.0 / 15.0) * inv_r - (1.0 / epsij) * ((4.0 / 3.0) * ipow(q, 2) - ipow(q, 3) + (3.0 / 10.0) * ipow(q, 4) - (1.0 / 30.0) * ipow(q, 5)) + 8.0 / 5.0 / epsij);
            if (q > 2.) fk = m[j] * inv_r;
            PE -= G * m[i] * fk;
        }
    }
    return PE;
}

/* getKE, sph_code/libsx.py:569-579. */
double orc_ke(int64_t n, const double *v, const double *m) {
    double KE = 0.0;
    for (int64_t i = 0; i < n; ++i)
        KE += 0.5 * m[i] * (ipow(v[3 * i + 0], 2) + ipow(v[3 * i + 1], 2) + ipow(v[3 * i + 2], 2));
    return KE;
}

/* Per-particle time step, restating dt_array_indiv_dt
 * (Particles_in_BH_Tree_III/Evrard_Collapse_2024/hfvCLibs_v7_hfv_v8.1.h:
 * 1189-1262) in FP64:
 *   vsig_ij  = c_i + c_j - 3 w_ij,  w_ij = (v_ij . r_ij) / (|r_ij| + 1e-5)
 *   dt_hyd   = C h_i / max_j vsig_ij            (max starts at 0)
 *   dt_cour  = C h_i / (h_i |divV_i| + max(c_i, |v_i|) (1 + 0.6 alpha))
 *   dt_G1    = 0.4 sqrt(eps_i / |a_tot,i|),  dt_G2 = 0.4 eps_i / |v_i|
 *   dt_f     = sqrt(h_i / |a_g,i|),          dt_kin = sqrt(h_i / |a_tot,i|)
 *   dt_i     = min of the six;  dh/dt_i = h_i divV_i / 3.
 * The reference takes the signal-velocity maximum over every particle
 * (neighbours = 0); neighbours = 1 restricts it to |r_ij| <= h_i + h_j (the
 * support of the hydro pairs, as in the criterion's source, Springel 2005
 * eq. 16).  j = i contributes c_i + c_i (w = 0), as in the reference loop. */
void orc_timestep(int64_t n, const double *pos, const double *v, const double *acc_tot,
                  const double *acc_g, const double *h, const double *c, const double *divV,
                  const double *eps, double c_cfl, double alpha, int neighbours,
                  const int64_t *rows, int64_t nrows, double *dt, double *dhdt) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t r = 0; r < nrows; ++r) {
        const int64_t i = rows[r];
        double vmax = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            const double dx = pos[3 * i + 0] - pos[3 * j + 0];
            const double dy = pos[3 * i + 1] - pos[3 * j + 1];
            const double dz = pos[3 * i + 2] - pos[3 * j + 2];
            const double rr = sqrt(dx * dx + dy * dy + dz * dz);
            if (neighbours && !(rr <= h[i] + h[j])) continue;
            const double vx = v[3 * i + 0] - v[3 * j + 0];
            const double vy = v[3 * i + 1] - v[3 * j + 1];
            const double vz = v[3 * i + 2] - v[3 * j + 2];
            const double w = (vx * dx + vy * dy + vz * dz) / (rr + 1e-5);
            const double s = c[i] + c[j] - 3.0 * w;
            if (s > vmax) vmax = s;
        }
        const double ag = sqrt(acc_g[3 * i] * acc_g[3 * i] + acc_g[3 * i + 1] * acc_g[3 * i + 1] +
                               acc_g[3 * i + 2] * acc_g[3 * i + 2]);
        const double at = sqrt(acc_tot[3 * i] * acc_tot[3 * i] + acc_tot[3 * i + 1] * acc_tot[3 * i + 1] +
                               acc_tot[3 * i + 2] * acc_tot[3 * i + 2]);
        const double av = sqrt(v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
        const double d[6] = {
            c_cfl * h[i] / vmax,
            c_cfl * h[i] / (h[i] * fabs(divV[i]) + fmax(c[i], av) * (1.0 + 0.6 * alpha)),
            sqrt(h[i] / ag),
            sqrt(h[i] / at),
            0.4 * sqrt(eps[i] / at),
            0.4 * eps[i] / av,
        };
        double m = d[0];
        for (int k = 0; k < 6; ++k)
            if (d[k] <= m) m = d[k];
        dt[r] = m;
        dhdt[r] = 1.0 / 3.0 * h[i] * divV[i];
    }
}

/* ------------------------------------------------------------------------
 * Table-driven heating/cooling: hcoolingZ
 * (Particles_in_BH_Tree_III/Evrard_Collapse_2024/hfvCLibs_v7_hfv_v8.1.h:1433-1623),
 * restated in FP32 with the reference's linear scans and nearest-point rule.
 * Table layout of coolHeatGridJan2024.bin (Main_Code/hfvGpuSphBHtree_newCool_v8.cu:40-80):
 * uevol [kpc][T][nH][Z][t], metalz [kpc][T][nH][Z][M][t], uarr [kpc][T][nH][Z].
 * dims: N_kpc, N_T, N_nH, N_Z, N_M, N_t.  units: unit density (cgs), unit time
 * (s), unit u (cgs), unit length (cm), kpc (cm).  Particles with typ != 0 are
 * left alone (typ NULL: all gas).  No contraction (-ffp-contract=off) except
 * the explicit fmaf of the interpolation. */
static int orc_nearest(const float *g, int n, float x) {
    int k = -1;
    for (int j = 0; j < n; ++j)
        if (k == -1 && x <= g[j]) k = j;
    if (k > 0) {
        const float d1 = fabsf(g[k] - x);
        const float d2 = fabsf(g[k - 1] - x);
        if (d2 < d1) k -= 1;
    }
    if (k == -1) k = n - 1;
    return k;
}

void orc_hcooling(int64_t n, const int32_t *typ, float *u, const float *rho, const float *x, const float *y,
                  const float *z, float *ionfrac, float dt, const int32_t *dims, const float *kpc, const float *nhg,
                  const float *tg, const float *uevol, const float *metalz, const float *uarr, const float *units,
                  int32_t z_index) {
    const int NK = dims[0], NT = dims[1], NH = dims[2], NZ = dims[3], NM = dims[4], Nt = dims[5];
    const float ud = units[0], ut = units[1], uu = units[2], ul = units[3], kpc_cm = units[4];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        if (typ && typ[i] != 0) continue;
        const float dt_sec = dt * ut;
        float r = sqrtf(x[i] * x[i] + y[i] * y[i] + z[i] * z[i]);
        r = r * ul / kpc_cm;
        const int ik = orc_nearest(kpc, NK, r);
        const float mH = 1.6726e-24f, XH = 0.70f;
        const float rho_cgs = rho[i] * ud;
        const float nH = rho_cgs * XH / mH;
        const int ih = orc_nearest(nhg, NH, nH);
        const int iz = z_index;
        const int it = orc_nearest(tg, Nt, dt_sec);
        /* uarr strides */
        const int64_t sZ0 = 1, sH0 = NZ * sZ0, sT0 = (int64_t)NH * sH0, sK0 = (int64_t)NT * sT0;
        const float u_i = u[i] * uu;
        int iu = -1;
        for (int j = 0; j < NT; ++j) {
            const int64_t idx = ik * sK0 + j * sT0 + ih * sH0 + iz;
            if (iu == -1 && u_i <= uarr[idx]) iu = j;
        }
        if (iu == -1) iu = NT - 1;
        /* uevol strides */
        const int64_t st = 1, sZ = Nt * st, sH = NZ * sZ, sT = (int64_t)NH * sH, sK = (int64_t)NT * sT;
        const int64_t ndx = ik * sK + iu * sT + ih * sH + iz * sZ + it;
        float uEv;
        if (iu > 0) {
            const float e1 = uevol[ndx - sT], e2 = uevol[ndx];
            const int64_t iU = ik * sK0 + iu * sT0 + ih * sH0 + iz;
            const int64_t iUm = ik * sK0 + (iu - 1) * sT0 + ih * sH0 + iz;
            const float diff = uarr[iU] - uarr[iUm];
            const float fhi = (u_i - uarr[iUm]) / diff;
            const float flow = 1.0f - fhi;
            /* one fused multiply-add: the reference kernel's compiled form
               (its outputs on the golden vectors equal this bit for bit) */
            uEv = fmaf(fhi, e2, flow * e1);
        } else {
            uEv = uevol[ndx];
        }
        u[i] = uEv / uu;
        if (ionfrac) {
            const int64_t mt = 1, mM = Nt * mt, mZ = (int64_t)NM * mM, mH = (int64_t)NZ * mZ, mT = (int64_t)NH * mH,
                          mK = (int64_t)NT * mT;
            for (int k = 0; k < NM; ++k)
                ionfrac[i * NM + k] = metalz[ik * mK + iu * mT + ih * mH + iz * mZ + k * mM + it];
        }
    }
}

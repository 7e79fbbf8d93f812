/* A plain C99 consumer of the C ABI (include/sph3.h, libsph3.so): what a
 * non-Python host program binds.  It builds a uniform sphere of N particles
 * (equal masses, u = 0.05, at rest), runs the first step and two KDK steps on
 * GPU 0 and checks the density and the energy sums.  Without a GPU it checks
 * that the library says so (SPH3_ERR_NO_DEVICE) and exits 0.
 * Output: one line, "no device" or "ok ...".  Exit status 0 on success. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "sph3.h"

#define N 4096

static uint64_t lcg = 88172645463325252ull;
static double urand(void) {
    lcg = lcg * 6364136223846793005ull + 1442695040888963407ull;
    return (double)(lcg >> 11) * (1.0 / 9007199254740992.0);
}

static int fail(const char *what, int rc) {
    printf("error %s: %d (%s)\n", what, rc, sph3_error_string(rc));
    return 1;
}

int main(void) {
    if (sph3_version() <= 0) return fail("version", sph3_version());
    sph3_config cfg;
    sph3_default_config(&cfg);
    sph3_ctx *ctx = NULL;
    int rc = sph3_ctx_create(&cfg, 0, &ctx);
    if (rc == SPH3_ERR_NO_DEVICE) {
        printf("no device\n");
        return 0;
    }
    if (rc) return fail("ctx_create", rc);

    /* positions and velocities (N, 3) row-major, as the header says */
    double *pos = malloc(sizeof(double) * 3 * N), *vel = calloc(3 * N, sizeof(double));
    double *m = malloc(sizeof(double) * N), *u = malloc(sizeof(double) * N);
    double *h = calloc(N, sizeof(double)), *rho = malloc(sizeof(double) * N);
    if (!pos || !vel || !m || !u || !h || !rho) return fail("malloc", -1);
    for (int i = 0; i < N; ++i) {
        double x, y, z;
        do {
            x = 2.0 * urand() - 1.0;
            y = 2.0 * urand() - 1.0;
            z = 2.0 * urand() - 1.0;
        } while (x * x + y * y + z * z > 1.0);
        pos[3 * i] = x;
        pos[3 * i + 1] = y;
        pos[3 * i + 2] = z;
        m[i] = 1.0 / N;
        u[i] = 0.05;
    }
    /* h = 0 everywhere: the first step starts the h search from its own guess */
    if ((rc = sph3_set_particles(ctx, N, pos, vel, m, u, h, NULL, 0, NULL))) return fail("set_particles", rc);
    if ((rc = sph3_first_step(ctx, 1e-3, NULL))) return fail("first_step", rc);
    if ((rc = sph3_step(ctx, 1e-3, 2, NULL))) return fail("step", rc);
    if ((rc = sph3_get_field(ctx, SPH3_FIELD_RHO, rho, 0, N, 0, NULL))) return fail("get_field", rc);
    double e[8];
    if ((rc = sph3_energy(ctx, e, NULL))) return fail("energy", rc);
    uint32_t status = 0;
    if ((rc = sph3_status(ctx, &status, 0))) return fail("status", rc);
    double rmin = rho[0], rmax = rho[0], rsum = 0.0;
    for (int i = 0; i < N; ++i) {
        if (!(rho[i] > 0.0) || !isfinite(rho[i])) return fail("density not positive and finite", i);
        rmin = rho[i] < rmin ? rho[i] : rmin;
        rmax = rho[i] > rmax ? rho[i] : rmax;
        rsum += rho[i];
    }
    /* a uniform unit sphere of unit mass has mean density 3 / (4 pi) = 0.239 */
    const double mean = rsum / N;
    if (status != 0 || mean < 0.1 || mean > 0.4) return fail("density or status out of range", (int)status);
    if (fabs(e[7] - 1.0) > 1e-12) return fail("mass sum", 0);
    printf("ok rho mean %.4f min %.4f max %.4f, KE %.6e, thermal %.6e, PE %.6e\n", mean, rmin, rmax, e[0], e[1],
           e[2]);
    sph3_ctx_destroy(ctx);
    free(pos);
    free(vel);
    free(m);
    free(u);
    free(h);
    free(rho);
    return 0;
}

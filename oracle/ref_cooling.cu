// Test infrastructure, not part of the library: runs the reference's
// heating/cooling kernel hcoolingZ
// (Particles_in_BH_Tree_III/Evrard_Collapse_2024/hfvCLibs_v7_hfv_v8.1.h:1433-1623)
// unchanged, compiled from the reference's own header by oracle/build_ref.sh,
// on an input file written by tests/golden/make_cooling.py, so that the
// oracle's restatement (orc_hcooling) is pinned to the reference's outputs.
//
//   ref_cooling IN.bin OUT.bin
//   IN:  int32 N; float32 dt, unit density (cgs), unit time (s), unit u (cgs),
//        unit length (cm), kpc (cm); int32 dims[6] = N_kpc N_T N_nH N_Z N_M N_t;
//        float32 kpc[N_kpc] nH[N_nH] t[N_t] uEvol[kpc][T][nH][Z][t]
//        metalz[kpc][T][nH][Z][M][t] uArr[kpc][T][nH][Z];
//        int32 typ[N]; float32 u[N] rho[N] x[N] y[N] z[N]
//   OUT: int32 N, int32 N_M, float32 u[N], float32 ionFrac[N][N_M] (zero for typ != 0)
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "hfvCLibs_v7_hfv_v8.1.h"

static int fail(const char *what) {
    std::fprintf(stderr, "ref_cooling: %s\n", what);
    return 1;
}

template <typename T>
static bool rd(std::FILE *f, std::vector<T> &v, size_t n) {
    v.resize(n);
    return std::fread(v.data(), sizeof(T), n, f) == n;
}

template <typename T>
static T *dev(const std::vector<T> &h) {
    T *p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * (h.size() ? h.size() : 1)) != cudaSuccess) return nullptr;
    if (!h.empty() && cudaMemcpy(p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return nullptr;
    return p;
}

int main(int argc, char **argv) {
    if (argc != 3) return fail("usage: ref_cooling IN.bin OUT.bin");
    std::FILE *fi = std::fopen(argv[1], "rb");
    if (!fi) return fail("cannot open input");
    int n = 0;
    std::vector<float> par;
    std::vector<int> dims;
    if (std::fread(&n, sizeof(int), 1, fi) != 1 || n <= 0 || n > (1 << 22)) return fail("bad N");
    if (!rd(fi, par, 6) || !rd(fi, dims, 6)) return fail("bad header");
    for (int d : dims)
        if (d <= 0 || d > 4096) return fail("bad dims");
    const int NK = dims[0], NT = dims[1], NH = dims[2], NZ = dims[3], NM = dims[4], Nt = dims[5];
    if (NZ < 2) return fail("the kernel reads metallicity row 1: N_Z must be >= 2");
    const size_t nu = (size_t)NK * NT * NH * NZ, nev = nu * Nt, nmz = nev * NM;
    std::vector<float> kpc, nh, tg, uev, mz, ua, u, rho, x, y, z;
    std::vector<int> typ;
    if (!rd(fi, kpc, NK) || !rd(fi, nh, NH) || !rd(fi, tg, Nt) || !rd(fi, uev, nev) || !rd(fi, mz, nmz) ||
        !rd(fi, ua, nu) || !rd(fi, typ, n) || !rd(fi, u, n) || !rd(fi, rho, n) || !rd(fi, x, n) || !rd(fi, y, n) ||
        !rd(fi, z, n))
        return fail("short input");
    std::fclose(fi);
    // arrays the kernel takes but does not read: Z grid, mu, log T
    std::vector<float> zgrid(NZ, 0.f), mu(nev, 0.f), logT(NT, 0.f), ion((size_t)n * NM, 0.f);
    int *d_typ = dev(typ);
    float *d_u = dev(u), *d_rho = dev(rho), *d_x = dev(x), *d_y = dev(y), *d_z = dev(z);
    float *d_kpc = dev(kpc), *d_nh = dev(nh), *d_t = dev(tg), *d_uev = dev(uev), *d_mz = dev(mz), *d_ua = dev(ua);
    float *d_zg = dev(zgrid), *d_mu = dev(mu), *d_lt = dev(logT), *d_ion = dev(ion);
    if (!d_typ || !d_u || !d_rho || !d_x || !d_y || !d_z || !d_kpc || !d_nh || !d_t || !d_uev || !d_mz || !d_ua ||
        !d_zg || !d_mu || !d_lt || !d_ion)
        return fail("device copies");
    const float dt = par[0], Zmetal = 0.1f, gm1 = 2.0f / 3.0f;
    hcoolingZ<<<(n + 255) / 256, 256>>>(d_typ, d_u, d_ua, d_rho, d_mz, Zmetal, dt, d_nh, d_zg, d_uev, d_ion, d_x,
                                        d_y, d_z, d_mu, d_lt, d_kpc, par[1], par[2], par[3], par[4], par[5], gm1,
                                        d_t, NK, NH, NZ, NT, NM, Nt, n);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return fail("kernel");
    if (cudaMemcpy(u.data(), d_u, sizeof(float) * n, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(ion.data(), d_ion, sizeof(float) * ion.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail("cudaMemcpy out");
    std::FILE *fo = std::fopen(argv[2], "wb");
    if (!fo) return fail("cannot open output");
    std::fwrite(&n, sizeof(int), 1, fo);
    std::fwrite(&NM, sizeof(int), 1, fo);
    std::fwrite(u.data(), sizeof(float), n, fo);
    std::fwrite(ion.data(), sizeof(float), ion.size(), fo);
    std::fclose(fo);
    std::printf("ref_cooling: %d particles, %d species\n", n, NM);
    return 0;
}

// Test infrastructure, not part of the library: runs the reference GPU
// driver's per-particle time-step kernel dt_array_indiv_dt
// (Particles_in_BH_Tree_III/Evrard_Collapse_2024/hfvCLibs_v7_hfv_v8.1.h:1189-1262)
// unchanged, compiled from the reference's own header by oracle/build_ref.sh,
// on an input file written by tests/golden/make_timestep.py, so that the
// oracle's restatement of that criterion (orc_timestep) can be pinned to the
// reference's own outputs.
//
//   ref_timestep IN.bin OUT.bin
//   IN:  int32 N, float32 C_CFL, float32 alpha, then N float32 each of
//        x y z vx vy vz ax ay az (gravity) atx aty atz (total) h c divV eps
//   OUT: int32 N, then N float32 each of dt, dh_dt, |a_g|, |a_tot|
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
    std::fprintf(stderr, "ref_timestep: %s\n", what);
    return 1;
}

int main(int argc, char **argv) {
    if (argc != 3) return fail("usage: ref_timestep IN.bin OUT.bin");
    std::FILE *fi = std::fopen(argv[1], "rb");
    if (!fi) return fail("cannot open input");
    int n = 0;
    float c_cfl = 0.f, alpha = 0.f;
    if (std::fread(&n, sizeof(int), 1, fi) != 1 || std::fread(&c_cfl, sizeof(float), 1, fi) != 1 ||
        std::fread(&alpha, sizeof(float), 1, fi) != 1 || n <= 0 || n > (1 << 22))
        return fail("bad header");
    const int nin = 16;  // x y z vx vy vz ax ay az atx aty atz h c divV eps
    std::vector<float> host((size_t)nin * n);
    if (std::fread(host.data(), sizeof(float), host.size(), fi) != host.size()) return fail("short input");
    std::fclose(fi);
    // device copies of the inputs, the particle types (all gas) and the outputs
    std::vector<float *> d(nin + 4, nullptr);
    for (auto &p : d)
        if (cudaMalloc(&p, sizeof(float) * n) != cudaSuccess) return fail("cudaMalloc");
    int *typ = nullptr;
    if (cudaMalloc(&typ, sizeof(int) * n) != cudaSuccess || cudaMemset(typ, 0, sizeof(int) * n) != cudaSuccess)
        return fail("cudaMalloc typ");
    for (int k = 0; k < nin; ++k)
        if (cudaMemcpy(d[k], host.data() + (size_t)k * n, sizeof(float) * n, cudaMemcpyHostToDevice) != cudaSuccess)
            return fail("cudaMemcpy in");
    float *dt = d[nin], *dhdt = d[nin + 1], *ag = d[nin + 2], *at = d[nin + 3];
    dt_array_indiv_dt<<<(n + 255) / 256, 256>>>(typ, d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7], d[8], d[9],
                                               d[10], d[11], d[12], d[13], dt, ag, at, d[14], dhdt, c_cfl, alpha,
                                               d[15], n);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return fail("kernel");
    std::vector<float> out((size_t)4 * n);
    const float *src[4] = {dt, dhdt, ag, at};
    for (int k = 0; k < 4; ++k)
        if (cudaMemcpy(out.data() + (size_t)k * n, src[k], sizeof(float) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
            return fail("cudaMemcpy out");
    std::FILE *fo = std::fopen(argv[2], "wb");
    if (!fo) return fail("cannot open output");
    std::fwrite(&n, sizeof(int), 1, fo);
    std::fwrite(out.data(), sizeof(float), out.size(), fo);
    std::fclose(fo);
    for (auto p : d) cudaFree(p);
    cudaFree(typ);
    std::printf("ref_timestep: %d particles\n", n);
    return 0;
}

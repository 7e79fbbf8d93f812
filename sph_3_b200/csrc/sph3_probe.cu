// Measured FP32 issue rate of this GPU, the denominator of the walk kernels'
// roofline (the walks are bound by the FP32 pipe, not by HBM or the tensor
// cores).  Every thread runs 8 independent chains of packed FP32 FMAs
// (FFMA2, two multiply-adds per instruction), then 16 chains of scalar FMAs;
// the rate is the larger of the two, flops of the whole grid over its
// CUDA-event time.  No waits, fixed trip counts.
#include "sph3_internal.cuh"

namespace sph3 {

constexpr int kProbeChains = 8;

__global__ void __launch_bounds__(256) k_fp32_rate(float *sink, int iters) {
    float2 a[kProbeChains];
#pragma unroll
    for (int u = 0; u < kProbeChains; ++u) a[u] = make_float2(1e-3f * (threadIdx.x + u), 1e-3f * u);
    const float2 m = make_float2(0.9999999f, 0.9999998f), c = make_float2(1e-7f, 2e-7f);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < kProbeChains; ++u) a[u] = __ffma2_rn(a[u], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int u = 0; u < kProbeChains; ++u) s += a[u].x + a[u].y;
    if (s == 1234.5f) sink[0] = s;  // never true in practice; keeps the chains live
}

// the same with scalar FMAs (16 chains): the rate is the larger of the two
__global__ void __launch_bounds__(256) k_fp32_rate_scalar(float *sink, int iters) {
    float a[2 * kProbeChains];
#pragma unroll
    for (int u = 0; u < 2 * kProbeChains; ++u) a[u] = 1e-3f * (threadIdx.x + u);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 2 * kProbeChains; ++u) a[u] = fmaf(a[u], 0.9999999f, 1e-7f);
    }
    float s = 0.f;
#pragma unroll
    for (int u = 0; u < 2 * kProbeChains; ++u) s += a[u];
    if (s == 1234.5f) sink[0] = s;
}

}  // namespace sph3

using namespace sph3;

extern "C" int sph3_probe_fp32_rate(int device, double *tflops, void *stream) {
    if (!tflops) return SPH3_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return SPH3_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return SPH3_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return SPH3_ERR_CUDA;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * 8, threads = 256, iters = 1 << 16;
    float *sink = nullptr;
    if (cudaMalloc(&sink, sizeof(float)) != cudaSuccess) return SPH3_ERR_OUT_OF_MEMORY;
    cudaEvent_t e[4];
    for (auto &x : e) cudaEventCreate(&x);
    // each form launched twice, the second timed (the first brings the clocks up)
    k_fp32_rate<<<blocks, threads, 0, st>>>(sink, iters / 4);
    cudaEventRecord(e[0], st);
    k_fp32_rate<<<blocks, threads, 0, st>>>(sink, iters);
    cudaEventRecord(e[1], st);
    k_fp32_rate_scalar<<<blocks, threads, 0, st>>>(sink, iters / 4);
    cudaEventRecord(e[2], st);
    k_fp32_rate_scalar<<<blocks, threads, 0, st>>>(sink, iters);
    cudaEventRecord(e[3], st);
    cudaError_t err = cudaEventSynchronize(e[3]);
    float ms2 = 0.f, ms1 = 0.f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms2, e[0], e[1]);
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms1, e[2], e[3]);
    for (auto &x : e) cudaEventDestroy(x);
    cudaFree(sink);
    if (err != cudaSuccess || !(ms2 > 0.f) || !(ms1 > 0.f)) return SPH3_ERR_CUDA;
    // flops: FFMA2 = 2 multiply-adds = 4 flops; FFMA = 2 flops (16 chains)
    const double f2 = (double)blocks * threads * iters * kProbeChains * 4.0;
    const double f1 = (double)blocks * threads * iters * (2 * kProbeChains) * 2.0;
    *tflops = fmax(f2 / (ms2 * 1e-3), f1 / (ms1 * 1e-3)) / 1e12;
    return SPH3_OK;
}

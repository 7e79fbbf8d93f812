// Morton sort that allocates nothing: sph3_morton_sort_noalloc.
//
// Who needs it: code that runs where device allocation is not allowed or not
// possible -- inside a caller-owned memory pool or arena that forbids
// cudaMalloc, in a process whose allocator is owned by a host framework
// (e.g. an embedding application that routes every allocation through its
// own pool), or in a tight loop where the latency and implicit
// synchronisation of cudaMalloc/cudaFree are unacceptable.  Such a caller
// passes device buffers for the input and the outputs only; every
// intermediate lives in one file-scope __device__ array below.
//
// The array is g_sort_scratch: kNoAllocMaxN = 65536 particles, about 3 MB.
// It exists once per GPU that loads the library and stays until the process
// exits.  In host code its name is only a host-side stand-in, not a device
// address, so the entry point resolves the real address with
// cudaGetSymbolAddress once per device and CUDA context (the first call on a
// device does this, and again the first call after cudaDeviceReset; make
// that first call before any stream capture).  Every call on a device shares
// the array and it keeps the last call's contents: calls that overlap on the
// GPU (different streams without ordering) race on it.
//
// Device-side conditions (non-finite coordinates) are collected in a status
// word inside the scratch, cleared at the start of every call and copied at
// its end into the caller's optional device word `status`.
//
// The work is the same as the context path's sort (sph3_sort.cu): root cube
// of the particles, 3 * max_level-bit Morton keys, stable 8-bit LSD radix
// sort of (key, index); the kernels are shared, only the buffers differ.
#include <mutex>

#include "sph3_internal.cuh"

namespace sph3 {

// kernels of sph3_sort.cu
__global__ void __launch_bounds__(256) k_box_partial(const int4 *items, const double *pos, int64_t n,
                                                     double *part, unsigned *status);
__global__ void k_cloud_boxes(Cloud *clouds, const int *item_begin, const double *part, int max_level,
                              int periodic, double Lx, double Ly, double Lz);
__global__ void k_keys(const Cloud *clouds, int ncloud, const double *pos, int64_t n, int max_level,
                       uint64_t *key, uint32_t *perm);
__global__ void __launch_bounds__(256) k_rs_hist(const uint64_t *key, int64_t n, int shift, uint32_t *hist,
                                                 int nblocks);
__global__ void __launch_bounds__(kRsOffsetThreads) k_rs_offsets(uint32_t *hist, int nblocks);
__global__ void __launch_bounds__(256) k_rs_scatter(const uint64_t *key_in, const uint32_t *val_in,
                                                    uint64_t *key_out, uint32_t *val_out, int64_t n, int shift,
                                                    const uint32_t *hist, int nblocks);

namespace {

constexpr int64_t kNoAllocMaxN = 65536;
constexpr int kSortTile = kRsTileKeys;  // keys per radix-sort block
constexpr int64_t kMaxSortBlocks = kNoAllocMaxN / kSortTile;
constexpr int64_t kMaxItems = (kNoAllocMaxN + kBoxChunk - 1) / kBoxChunk;

constexpr size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

// byte layout of the scratch array
constexpr size_t kOffPos = 0;                                                    // double [3][N]
constexpr size_t kOffKeyA = kOffPos + al256(sizeof(double) * 3 * kNoAllocMaxN);  // uint64 [N]
constexpr size_t kOffKeyB = kOffKeyA + al256(sizeof(uint64_t) * kNoAllocMaxN);
constexpr size_t kOffValA = kOffKeyB + al256(sizeof(uint64_t) * kNoAllocMaxN);   // uint32 [N]
constexpr size_t kOffValB = kOffValA + al256(sizeof(uint32_t) * kNoAllocMaxN);
constexpr size_t kOffHist = kOffValB + al256(sizeof(uint32_t) * kNoAllocMaxN);   // uint32 [256][blocks+1]
constexpr size_t kOffPart = kOffHist + al256(sizeof(uint32_t) * 256 * (kMaxSortBlocks + 1));
constexpr size_t kOffItems = kOffPart + al256(sizeof(double) * 6 * kMaxItems);
constexpr size_t kOffItemBeg = kOffItems + al256(sizeof(int4) * kMaxItems);
constexpr size_t kOffCloud = kOffItemBeg + al256(sizeof(int) * 2);
constexpr size_t kOffStatus = kOffCloud + al256(sizeof(Cloud));
constexpr size_t kScratchBytes = kOffStatus + al256(sizeof(unsigned));

static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_dev_ptr[kMaxDevices] = {};
void *g_dev_ctx[kMaxDevices] = {};  // the CUDA context the cached address belongs to

// The current CUDA context (driver handle), looked up through the runtime's
// driver entry point so the library needs no link against libcuda.
using CtxGetCurrentFn = int (*)(void **);
void *current_context() {
    static CtxGetCurrentFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(f);
        tried = true;
    }
    void *ctx = nullptr;
    if (fn && fn(&ctx) != 0) ctx = nullptr;
    return ctx;
}

// device address of g_sort_scratch on the current device, looked up once per
// device and context (a cudaDeviceReset makes a new context, in which the
// module and its array are loaded again, possibly elsewhere)
int scratch_for_current_device(unsigned char **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return SPH3_ERR_NO_DEVICE;
    if (dev < 0 || dev >= kMaxDevices) return SPH3_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_mu);
    void *ctx = current_context();
    if (!g_dev_ptr[dev] || ctx == nullptr || ctx != g_dev_ctx[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return SPH3_ERR_CUDA;
        }
        g_dev_ptr[dev] = static_cast<unsigned char *>(p);
        g_dev_ctx[dev] = current_context();
    }
    *out = g_dev_ptr[dev];
    return SPH3_OK;
}

// (n, 3) row-major positions -> component-major copy; one cloud covering all
// particles and its root-cube reduction items; status cleared
__global__ void k_na_setup(const double *pos_rm, int64_t n, double *pos_cm, int4 *items, int *item_begin,
                           Cloud *cloud, unsigned *status) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        pos_cm[k] = pos_rm[3 * k + 0];
        pos_cm[n + k] = pos_rm[3 * k + 1];
        pos_cm[2 * n + k] = pos_rm[3 * k + 2];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        int ni = 0;
        for (int64_t b = 0; b < n; b += kBoxChunk, ++ni)
            items[ni] = make_int4(0, (int)b, (int)(b + kBoxChunk < n ? b + kBoxChunk : n), 0);
        item_begin[0] = 0;
        item_begin[1] = ni;
        cloud->begin = 0;
        cloud->end = n;
        cloud->root = 0;
        *status = 0u;
    }
}

__global__ void k_na_output(const uint64_t *key, const uint32_t *val, int64_t n, int64_t *order,
                            uint64_t *keys_out, const unsigned *status, unsigned *status_out) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        if (order) order[k] = (int64_t)val[k];
        if (keys_out) keys_out[k] = key[k];
    }
    if (status_out && blockIdx.x == 0 && threadIdx.x == 0) *status_out = *status;
}

}  // namespace
}  // namespace sph3

using namespace sph3;

extern "C" int sph3_morton_sort_noalloc(const double *pos, int64_t n, int32_t max_level, int64_t *order,
                                        uint64_t *keys, unsigned *status_out, void *stream) {
    if (n < 0 || (n > 0 && !pos) || (!order && !keys) || max_level < 4 || max_level > 21)
        return SPH3_ERR_INVALID_ARG;
    if (n > kNoAllocMaxN) return SPH3_ERR_TOO_LARGE;
    if (n == 0) return status_out ? (cudaMemsetAsync(status_out, 0, sizeof(unsigned), (cudaStream_t)stream) ==
                                             cudaSuccess ? SPH3_OK : SPH3_ERR_CUDA)
                                  : SPH3_OK;
    // an error left pending by the caller's own work is not this call's: leave
    // it for the caller to read and do nothing
    if (cudaPeekAtLastError() != cudaSuccess) return SPH3_ERR_CUDA;
    unsigned char *s = nullptr;
    int rc = scratch_for_current_device(&s);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    double *pos_cm = reinterpret_cast<double *>(s + kOffPos);
    uint64_t *kA = reinterpret_cast<uint64_t *>(s + kOffKeyA);
    uint64_t *kB = reinterpret_cast<uint64_t *>(s + kOffKeyB);
    uint32_t *vA = reinterpret_cast<uint32_t *>(s + kOffValA);
    uint32_t *vB = reinterpret_cast<uint32_t *>(s + kOffValB);
    uint32_t *hist = reinterpret_cast<uint32_t *>(s + kOffHist);
    double *part = reinterpret_cast<double *>(s + kOffPart);
    int4 *items = reinterpret_cast<int4 *>(s + kOffItems);
    int *item_begin = reinterpret_cast<int *>(s + kOffItemBeg);
    Cloud *cloud = reinterpret_cast<Cloud *>(s + kOffCloud);
    unsigned *status = reinterpret_cast<unsigned *>(s + kOffStatus);

    const int blocks = (int)((n + 255) / 256);
    k_na_setup<<<blocks, 256, 0, st>>>(pos, n, pos_cm, items, item_begin, cloud, status);
    const int nitems = (int)((n + kBoxChunk - 1) / kBoxChunk);
    k_box_partial<<<nitems, 256, 0, st>>>(items, pos_cm, n, part, status);
    k_cloud_boxes<<<1, 32, 0, st>>>(cloud, item_begin, part, max_level, 0, 0.0, 0.0, 0.0);
    k_keys<<<blocks, 256, 0, st>>>(cloud, 1, pos_cm, n, max_level, kA, vA);
    if (cudaGetLastError() != cudaSuccess) return SPH3_ERR_CUDA;
    const int nb = (int)((n + kSortTile - 1) / kSortTile);
    const int passes = (3 * max_level + 7) / 8;
    uint64_t *kin = kA, *kout = kB;
    uint32_t *vin = vA, *vout = vB;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        k_rs_hist<<<nb, 256, 0, st>>>(kin, n, shift, hist, nb);
        k_rs_offsets<<<1, kRsOffsetThreads, 0, st>>>(hist, nb);
        k_rs_scatter<<<nb, 256, 0, st>>>(kin, vin, kout, vout, n, shift, hist, nb);
        uint64_t *tk = kin;
        kin = kout;
        kout = tk;
        uint32_t *tv = vin;
        vin = vout;
        vout = tv;
    }
    if (cudaGetLastError() != cudaSuccess) return SPH3_ERR_CUDA;
    k_na_output<<<blocks, 256, 0, st>>>(kin, vin, n, order, keys, status, status_out);
    return cudaGetLastError() == cudaSuccess ? SPH3_OK : SPH3_ERR_CUDA;
}

// C ABI of libsph3: context lifetime, host/device transfers in the caller's
// particle order, the compute passes and the captured timestep.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <new>
#include <vector>

#include "sph3_internal.cuh"

using namespace sph3;

namespace sph3 {
void launch_balsara(State &S, cudaStream_t st);
}

// ------------------------------------------------------------ context
// row chunks of the host-buffer step's first inputs and last outputs
constexpr int kIoChunks = 8;

struct sph3_ctx {
    sph3_config cfg{};
    Params P{};
    State S{};
    int device = 0;
    cudaStream_t stream = nullptr;
    // carried fields (permuted with the particles every step), two blocks
    double *carried[2] = {nullptr, nullptr};
    int64_t *orig_blk[2] = {nullptr, nullptr};
    int cur = 0;
    // fields recomputed every step (permuted only on an explicit re-sort)
    double *fixed = nullptr;
    double *tmp = nullptr;       // 9 n scratch for permuting fixed fields
    double *staging = nullptr;   // 3 n, transfers in the caller's order
    int64_t *inv = nullptr;      // caller index -> sorted index
    bool inv_valid = false;
    int64_t cap_n = -1;
    int cap_nodes = 0;
    int cap_groups = 0;
    int cap_clouds = 0;
    int cap_sortblk = 0;
    std::vector<int64_t> cloud_counts;  // layout for the next set_particles
    std::vector<int64_t> cur_counts;
    bool have = false;
    unsigned pack_dirty = 0;
    bool bal_dirty = false;
    bool tree_dirty = true;
    bool h_dirty_tree = false;  // node hmax stale
    bool order_dirty = false;   // positions changed since the last sort
    bool phi_valid = false;     // the potential matches the current positions, masses and eps
    // graphs (one per carried-block parity)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    double graph_dt[2] = {0, 0};
    int64_t graph_kernels[2] = {0, 0};  // kernel nodes of each captured step graph
    int warm_steps = 0;
    // timing
    cudaEvent_t ev[12] = {};
    double phase_ms[9] = {};
    // host-buffer step (sph3_step_io): input / output staging in the caller's
    // order, a copy stream per direction, events between them and the step
    double *io_in = nullptr, *io_out = nullptr;
    int64_t io_in_cap = 0, io_out_cap = 0;  // doubles
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t io_ev[10] = {};
    // row chunks of the position/velocity/acceleration inputs and of the
    // end-of-step outputs, so that copies and kernels overlap chunk by chunk
    cudaEvent_t io_chunk_ev[2][kIoChunks] = {};
    // the host-buffer step captured as a graph per carried-block parity, with
    // the call it was captured for (buffers, fields, dt, steps)
    cudaGraphExec_t io_graph[2] = {nullptr, nullptr};
    std::vector<uint64_t> io_key[2];
    // row-restricted compute (sph3_compute_rows): the groups holding the
    // requested rows, and a per-particle mark
    int2 *sub_groups = nullptr;
    int *sub_cloud = nullptr, *sub_n = nullptr;
    unsigned char *row_flag = nullptr;
    int64_t sub_cap = 0;
    // heating / cooling after the u update (sph3_set_cooling): the caller's
    // table and units, and the last cooled step's ion fractions, (n, N_M)
    // float in the caller's particle order
    const sph3_cool_table *cool = nullptr;
    sph3_cool_units cool_units{};
    float *ionfrac = nullptr;
    int64_t ionfrac_cap = 0;  // floats
    bool ionfrac_valid = false;
};

namespace {

int cuda_err(cudaError_t e) { return e == cudaSuccess ? SPH3_OK : SPH3_ERR_CUDA; }

// number of kernel launches recorded in a captured graph
int64_t count_kernel_nodes(cudaGraph_t g) {
    size_t nn = 0;
    if (cudaGraphGetNodes(g, nullptr, &nn) != cudaSuccess || nn == 0) return 0;
    std::vector<cudaGraphNode_t> nodes(nn);
    if (cudaGraphGetNodes(g, nodes.data(), &nn) != cudaSuccess) return 0;
    int64_t k = 0;
    for (size_t i = 0; i < nn; ++i) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
    }
    return k;
}

#define CK(x)                                            \
    do {                                                 \
        cudaError_t _e = (x);                            \
        if (_e != cudaSuccess) return SPH3_ERR_CUDA;     \
    } while (0)

int check_launch() { return cuda_err(cudaGetLastError()); }

constexpr int kCarried = 12;  // pos(3) vel(3) u u_prev dudt_prev m h eps
constexpr int kFixed = 20;    // acc(3) acc_g(3) acc_sph(3) dudt rho P c divV curlV bal phi vsig dt dhdt

void point_carried(sph3_ctx *c) {
    State &S = c->S;
    const int64_t n = std::max<int64_t>(c->cap_n, 1);
    double *b = c->carried[c->cur];
    S.pos = b;
    S.vel = b + 3 * n;
    S.u = b + 6 * n;
    S.u_prev = b + 7 * n;
    S.dudt_prev = b + 8 * n;
    S.m = b + 9 * n;
    S.h = b + 10 * n;
    S.eps = b + 11 * n;
    S.orig = c->orig_blk[c->cur];
}

void point_fixed(sph3_ctx *c) {
    State &S = c->S;
    const int64_t n = std::max<int64_t>(c->cap_n, 1);
    double *b = c->fixed;
    S.acc = b;
    S.acc_g = b + 3 * n;
    S.acc_sph = b + 6 * n;
    S.dudt = b + 9 * n;
    S.rho = b + 10 * n;
    S.P = b + 11 * n;
    S.c = b + 12 * n;
    S.divV = b + 13 * n;
    S.curlV = b + 14 * n;
    S.bal = b + 15 * n;
    S.phi = b + 16 * n;
    S.vsig = b + 17 * n;
    S.dt = b + 18 * n;
    S.dhdt = b + 19 * n;
}

void params_from(const sph3_config &cfg, Params &P) {
    P.precision = cfg.precision;
    P.h_mode = cfg.h_mode;
    P.visc = cfg.visc;
    P.step_order = cfg.step_order;
    P.n_ngb = cfg.n_ngb;
    P.n_ngb_tol = cfg.n_ngb_tol;
    P.h_max_iter = cfg.h_max_iter;
    P.n_boot = cfg.n_boot;
    P.leaf_size = cfg.leaf_size;
    P.stack_cap = cfg.stack_cap;
    P.max_level = cfg.max_level;
    P.gravity = cfg.gravity;
    P.quadrupole = cfg.quadrupole;
    P.walk_warps = cfg.walk_warps;
    P.list_cap = cfg.list_cap;
    P.mac = cfg.mac;
    P.eps_from_h = cfg.eps_from_h;
    P.gamma = cfg.gamma;
    P.alpha = cfg.alpha;
    P.beta = cfg.beta;
    P.eta = cfg.eta;
    P.G = cfg.G;
    P.theta = cfg.theta;
    P.eps = cfg.eps;
    P.periodic = 0;
    for (int d = 0; d < 3; ++d) {
        P.box[d] = cfg.box[d];
        if (cfg.box[d] > 0) P.periodic = 1;
    }
}

int validate(const sph3_config *c) {
    if (!c) return SPH3_ERR_INVALID_ARG;
    if (c->precision != SPH3_PREC_MIXED && c->precision != SPH3_PREC_FP64) return SPH3_ERR_INVALID_ARG;
    if (c->h_mode != SPH3_H_NEWTON && c->h_mode != SPH3_H_REFSTEP) return SPH3_ERR_INVALID_ARG;
    if (c->visc < 0 || c->visc > 2) return SPH3_ERR_INVALID_ARG;
    if (c->step_order != SPH3_ORDER_SERIAL && c->step_order != SPH3_ORDER_MPI4) return SPH3_ERR_INVALID_ARG;
    if (c->n_ngb < 1 || c->n_ngb_tol < 0 || c->n_ngb_tol >= c->n_ngb) return SPH3_ERR_INVALID_ARG;
    if (c->h_max_iter < 1 || c->n_boot < 0) return SPH3_ERR_INVALID_ARG;
    if (c->leaf_size < 1 || c->leaf_size > 64) return SPH3_ERR_INVALID_ARG;
    if (c->walk_warps != 1 && c->walk_warps != 2 && c->walk_warps != 4 && c->walk_warps != 8)
        return SPH3_ERR_INVALID_ARG;
    if (c->max_level < 4 || c->max_level > 21) return SPH3_ERR_INVALID_ARG;
    if (c->list_cap < 0 || c->list_cap > 1024 || c->list_cap % 8) return SPH3_ERR_INVALID_ARG;
    if (c->mac != SPH3_MAC_BH && c->mac != SPH3_MAC_BH_OFFSET) return SPH3_ERR_INVALID_ARG;
    if (c->eps_from_h != 0 && c->eps_from_h != 1) return SPH3_ERR_INVALID_ARG;
    if (c->step_potential != 0 && c->step_potential != 1) return SPH3_ERR_INVALID_ARG;
    if (c->stack_cap < 7 * (c->max_level + 2) + 32 || c->stack_cap > 4096) return SPH3_ERR_INVALID_ARG;
    if (!(c->theta >= 0.0) || !(c->eps > 0.0) || !(c->gamma >= 1.0)) return SPH3_ERR_INVALID_ARG;
    for (int d = 0; d < 3; ++d)
        if (!(c->box[d] >= 0.0) || !std::isfinite(c->box[d])) return SPH3_ERR_INVALID_ARG;
    if ((c->box[0] > 0 || c->box[1] > 0 || c->box[2] > 0) && c->gravity) return SPH3_ERR_UNSUPPORTED;
    return SPH3_OK;
}

void free_buffers(sph3_ctx *c) {
    State &S = c->S;
    void *ptrs[] = {c->carried[0], c->carried[1], c->orig_blk[0], c->orig_blk[1], c->fixed, c->tmp,
                    c->staging, c->inv, S.nngb, S.key, S.key_alt, S.perm, S.perm_alt, S.pk_pos, S.pk_hme,
                    S.pk_vel, S.pk_thm, S.sort_hist, S.tree.range, S.tree.child, S.tree.mass, S.tree.com,
                    S.tree.bmin, S.tree.bmax, S.tree.hmax, S.tree.epsmax, S.tree.quad, S.tree.box_c,
                    S.tree.box_h, S.tree.com_c, S.tree.mono, S.tree.quad4, S.tree.quad1,
                    S.tree.meta, S.tree.parent, S.tree.arrive, S.tree.lvl, S.tree.lb, S.tree.gw, S.tree.sw, S.list, S.nlist, S.hrec, S.ovf, S.groups, S.group_cloud, S.ngroups_dev, S.clouds, S.box_items,
                    S.box_item_begin, S.box_part, c->sub_groups, c->sub_cloud, c->sub_n, c->row_flag};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    c->sub_groups = nullptr;
    c->sub_cloud = nullptr;
    c->sub_n = nullptr;
    c->row_flag = nullptr;
    c->sub_cap = 0;
    c->carried[0] = c->carried[1] = nullptr;
    c->orig_blk[0] = c->orig_blk[1] = nullptr;
    c->fixed = c->tmp = c->staging = nullptr;
    c->inv = nullptr;
    S.nngb = nullptr;
    S.key = S.key_alt = nullptr;
    S.perm = S.perm_alt = nullptr;
    S.pk_pos = S.pk_hme = S.pk_vel = S.pk_thm = nullptr;
    S.sort_hist = nullptr;
    S.list = S.nlist = nullptr;
    S.hrec = nullptr;
    S.ovf = nullptr;
    S.list_cap = 0;
    S.list_valid = false;
    S.tree = Tree{};
    S.groups = nullptr;
    S.group_cloud = nullptr;
    S.ngroups_dev = nullptr;
    S.box_items = nullptr;
    S.box_item_begin = nullptr;
    S.box_part = nullptr;
    S.nbox_items = 0;
    S.clouds = nullptr;
    c->cap_n = -1;
    c->cap_nodes = c->cap_groups = c->cap_clouds = c->cap_sortblk = 0;
}

void drop_graphs(sph3_ctx *c) {
    for (int k = 0; k < 2; ++k) {
        if (c->graph[k]) cudaGraphExecDestroy(c->graph[k]);
        c->graph[k] = nullptr;
        if (c->io_graph[k]) cudaGraphExecDestroy(c->io_graph[k]);
        c->io_graph[k] = nullptr;
        c->io_key[k].clear();
    }
    c->warm_steps = 0;
}

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
    return cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(count, 1));
}

// the ion-fraction buffer of a context with cooling, (n, N_M) floats; any
// earlier fractions become invalid
int ensure_ionfrac(sph3_ctx *c) {
    c->ionfrac_valid = false;
    if (!c->cool) return SPH3_OK;
    const int64_t want = std::max<int64_t>(c->S.n, 1) * cool_table_species(c->cool);
    if (want > c->ionfrac_cap) {
        if (c->ionfrac) cudaFree(c->ionfrac);
        c->ionfrac = nullptr;
        c->ionfrac_cap = 0;
        if (dalloc(&c->ionfrac, (size_t)want) != cudaSuccess) return SPH3_ERR_OUT_OF_MEMORY;
        c->ionfrac_cap = want;
    }
    return SPH3_OK;
}

// a temporary device buffer freed on every return path
template <typename T>
struct DevTmp {
    T *p = nullptr;
    cudaError_t alloc(size_t count) { return dalloc(&p, count); }
    ~DevTmp() {
        if (p) cudaFree(p);
    }
};

// neighbour lists of the mixed path: list_cap slots per particle (particle-major,
// slot k of particle i at i * list_cap + k) and the count per particle
int ensure_lists(sph3_ctx *c, int64_t nn) {
    State &S = c->S;
    const int want = c->P.list_cap;
    S.list_valid = false;
    if (want == S.list_cap && (want == 0 || S.list)) return SPH3_OK;
    if (S.list) cudaFree(S.list);
    if (S.nlist) cudaFree(S.nlist);
    if (S.hrec) cudaFree(S.hrec);
    if (S.ovf) cudaFree(S.ovf);
    S.list = S.nlist = nullptr;
    S.hrec = nullptr;
    S.ovf = nullptr;
    S.list_cap = 0;
    if (want == 0) return SPH3_OK;
    CK(dalloc(&S.list, (size_t)want * nn));
    CK(dalloc(&S.nlist, nn));
    CK(dalloc(&S.hrec, 3 * (size_t)nn));
    CK(dalloc(&S.ovf, 1));
    CK(cudaMemset(S.ovf, 0, sizeof(int)));
    S.list_cap = want;
    return SPH3_OK;
}

int alloc_for(sph3_ctx *c, int64_t n, int ncloud, int ngroups) {
    if (n == c->cap_n && ncloud <= c->cap_clouds && ngroups <= c->cap_groups) return SPH3_OK;
    drop_graphs(c);
    free_buffers(c);
    State &S = c->S;
    const int64_t nn = std::max<int64_t>(n, 1);
    c->cap_n = n;
    CK(dalloc(&c->carried[0], kCarried * nn));
    CK(dalloc(&c->carried[1], kCarried * nn));
    CK(dalloc(&c->orig_blk[0], nn));
    CK(dalloc(&c->orig_blk[1], nn));
    CK(dalloc(&c->fixed, kFixed * nn));
    CK(dalloc(&c->tmp, 9 * nn));
    CK(dalloc(&c->staging, 3 * nn));
    CK(dalloc(&c->inv, nn));
    CK(cudaMemset(c->carried[0], 0, sizeof(double) * kCarried * nn));
    CK(cudaMemset(c->carried[1], 0, sizeof(double) * kCarried * nn));
    CK(cudaMemset(c->fixed, 0, sizeof(double) * kFixed * nn));
    CK(dalloc(&S.nngb, nn));
    CK(cudaMemset(S.nngb, 0, sizeof(int) * nn));
    CK(dalloc(&S.key, nn));
    CK(dalloc(&S.key_alt, nn));
    CK(dalloc(&S.perm, nn));
    CK(dalloc(&S.perm_alt, nn));
    CK(dalloc(&S.pk_pos, nn));
    CK(dalloc(&S.pk_hme, nn));
    CK(dalloc(&S.pk_vel, nn));
    CK(dalloc(&S.pk_thm, nn));
    CK(cudaMemset(S.pk_thm, 0, sizeof(float4) * nn));
    c->cap_sortblk = (int)((nn + kRsTileKeys - 1) / kRsTileKeys);
    // the one-sweep sort's scratch: 8 passes' histograms, tile counters, and a
    // look-back word per (pass, tile, digit); at least the table of the
    // three-kernel pass (256 x (tiles + 1))
    CK(dalloc(&S.sort_hist, (size_t)8 * 256 + 64 + (size_t)8 * 256 * (c->cap_sortblk + 1)));
    const int cap = (int)std::min<int64_t>(2 * nn + ncloud + 64, (int64_t)INT32_MAX - 1);
    c->cap_nodes = cap;
    Tree &T = S.tree;
    T.cap = cap;
    CK(dalloc(&T.range, cap));
    CK(dalloc(&T.child, cap));
    CK(dalloc(&T.mass, cap));
    CK(dalloc(&T.com, 3 * (size_t)cap));
    CK(dalloc(&T.bmin, 3 * (size_t)cap));
    CK(dalloc(&T.bmax, 3 * (size_t)cap));
    CK(dalloc(&T.hmax, cap));
    CK(dalloc(&T.epsmax, cap));
    CK(dalloc(&T.quad, 6 * (size_t)cap));
    CK(dalloc(&T.box_c, cap));
    CK(dalloc(&T.box_h, cap));
    CK(dalloc(&T.com_c, cap));
    CK(dalloc(&T.mono, cap));
    CK(dalloc(&T.quad4, cap));
    CK(dalloc(&T.quad1, cap));
    CK(dalloc(&T.gw, 2 * (size_t)cap));
    CK(dalloc(&T.sw, 3 * (size_t)cap));
    CK(dalloc(&T.parent, cap));
    CK(dalloc(&T.arrive, cap));
    CK(cudaMemset(T.arrive, 0, sizeof(int) * (size_t)cap));
    // a depth holds at most one node per particle
    CK(dalloc(&T.meta, 128));
    T.depth_begin = T.meta;
    T.total = T.meta + 96;
    CK(dalloc(&T.lvl, kLvlEpoch + 1));
    CK(cudaMemset(T.lvl, 0, sizeof(int) * (kLvlEpoch + 1)));
    // a depth holds at most n + clouds + 64 nodes: tiles of at least 8 nodes of the level pass
    const size_t ntiles = (size_t)(nn + ncloud + 64) / 8 + 2;
    CK(dalloc(&T.lb, ntiles));
    CK(cudaMemset(T.lb, 0, sizeof(unsigned long long) * ntiles));
    c->cap_groups = std::max(ngroups, 1);
    CK(dalloc(&S.groups, c->cap_groups));
    CK(dalloc(&S.group_cloud, c->cap_groups));
    CK(dalloc(&S.ngroups_dev, 1));
    CK(cudaMemset(S.ngroups_dev, 0, sizeof(int)));
    c->cap_clouds = std::max(ncloud, 1);
    CK(dalloc(&S.clouds, c->cap_clouds));
    c->cur = 0;
    point_carried(c);
    point_fixed(c);
    return ensure_lists(c, nn);
}

cudaStream_t pick(sph3_ctx *c, void *stream) { return stream ? (cudaStream_t)stream : c->stream; }

// ------------------------------------------------------------ small kernels
// row-major (n, ncomp) caller-order array -> component-major sorted field
__global__ void k_scatter_in(const double *src, double *dst, const int64_t *orig, int64_t n, int ncomp) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = orig[k];
        for (int c = 0; c < ncomp; ++c) dst[c * n + k] = src[o * ncomp + c];
    }
}

// rows [b, e) of a row-major (n, ncomp) caller-order array -> component-major
// sorted field (sorted index inv[r])
__global__ void k_scatter_rows(const double *src, double *dst, const int64_t *inv, int64_t n, int ncomp, int64_t b,
                               int64_t e) {
    for (int64_t r = b + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < e; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = inv[r];
        for (int c = 0; c < ncomp; ++c) dst[c * n + k] = src[r * ncomp + c];
    }
}

// rows [b, e) of a component-major sorted field -> row-major caller order
__global__ void k_gather_out(const double *src, double *dst, const int64_t *inv, int64_t n, int ncomp,
                             int64_t b, int64_t e) {
    for (int64_t r = b + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < e; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = inv[r];
        for (int c = 0; c < ncomp; ++c) dst[(r - b) * ncomp + c] = src[c * n + k];
    }
}

__global__ void k_gather_out_int(const int *src, double *dst, const int64_t *inv, int64_t b, int64_t e) {
    for (int64_t r = b + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < e; r += (int64_t)gridDim.x * blockDim.x)
        dst[r - b] = (double)src[inv[r]];
}

// mark the particles of caller rows [b, e) (sorted index inv[r])
__global__ void k_mark_rows(const int64_t *inv, int64_t b, int64_t e, unsigned char *flag) {
    for (int64_t r = b + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < e; r += (int64_t)gridDim.x * blockDim.x)
        flag[inv[r]] = 1;
}

// the walk groups holding at least one marked particle (order does not
// matter: a group's results depend only on the group)
__global__ void k_select_groups(const int2 *groups, const int *gcl, const int *ng, const unsigned char *flag,
                                int2 *gsub, int *csub, int *nsub) {
    const int n = *ng;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        const int2 gr = groups[g];
        bool any = false;
        for (int k = gr.x; k < gr.x + gr.y && !any; ++k) any = flag[k] != 0;
        if (any) {
            const int s = atomicAdd(nsub, 1);
            gsub[s] = gr;
            csub[s] = gcl[g];
        }
    }
}

__global__ void k_invert(const int64_t *orig, int64_t *inv, int64_t n) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        inv[orig[k]] = k;
}

__global__ void k_iota64(int64_t *a, int64_t n) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        a[k] = k;
}

__global__ void k_fill(double *a, int64_t n, double v) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        a[k] = v;
}

__global__ void k_copy(const double *s, double *d, int64_t n) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        d[k] = s[k];
}

int blocks_for(const sph3_ctx *c, int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)c->S.num_sms * 8));
}

// field id -> (pointer, components)
double *field_ptr(sph3_ctx *c, int f, int *ncomp) {
    State &S = c->S;
    *ncomp = 1;
    switch (f) {
        case SPH3_FIELD_POS: *ncomp = 3; return S.pos;
        case SPH3_FIELD_VEL: *ncomp = 3; return S.vel;
        case SPH3_FIELD_MASS: return S.m;
        case SPH3_FIELD_U: return S.u;
        case SPH3_FIELD_H: return S.h;
        case SPH3_FIELD_EPS: return S.eps;
        case SPH3_FIELD_RHO: return S.rho;
        case SPH3_FIELD_P: return S.P;
        case SPH3_FIELD_C: return S.c;
        case SPH3_FIELD_DIVV: return S.divV;
        case SPH3_FIELD_CURLV: return S.curlV;
        case SPH3_FIELD_ACC: *ncomp = 3; return S.acc;
        case SPH3_FIELD_ACC_G: *ncomp = 3; return S.acc_g;
        case SPH3_FIELD_ACC_SPH: *ncomp = 3; return S.acc_sph;
        case SPH3_FIELD_DUDT: return S.dudt;
        case SPH3_FIELD_DUDT_PREV: return S.dudt_prev;
        case SPH3_FIELD_PHI: return S.phi;
        case SPH3_FIELD_BALSARA: return S.bal;
        case SPH3_FIELD_U_PREV: return S.u_prev;
        case SPH3_FIELD_VSIG: return S.vsig;
        case SPH3_FIELD_DT: return S.dt;
        case SPH3_FIELD_DHDT: return S.dhdt;
        default: return nullptr;
    }
}

// sort the current particles (positions changed) and permute every field
int resort_all(sph3_ctx *c, cudaStream_t st) {
    State &S = c->S;
    if (S.n == 0) return SPH3_OK;
    launch_cloud_boxes(S, c->P, st);
    launch_keys(S, c->P, st);
    launch_radix_sort(S, st);
    // carried block -> other block
    const int other = c->cur ^ 1;
    double *src = c->carried[c->cur], *dst = c->carried[other];
    const int64_t n = c->cap_n;
    const double *srcs[kCarried];
    double *dsts[kCarried];
    int nc[kCarried];
    for (int k = 0; k < kCarried; ++k) {
        srcs[k] = src + k * n;
        dsts[k] = dst + k * n;
        nc[k] = 1;
    }
    launch_gather(S, srcs, dsts, kCarried, nc, st);
    launch_gather_orig(S, c->orig_blk[c->cur], c->orig_blk[other], st);
    // fixed fields: through tmp, 9 at a time
    for (int k0 = 0; k0 < kFixed; k0 += 9) {
        const int cnt = std::min(9, kFixed - k0);
        const double *s2[9];
        double *d2[9];
        int n2[9];
        for (int k = 0; k < cnt; ++k) {
            s2[k] = c->fixed + (k0 + k) * n;
            d2[k] = c->tmp + k * n;
            n2[k] = 1;
        }
        launch_gather(S, s2, d2, cnt, n2, st);
        k_copy<<<blocks_for(c, cnt * n), 256, 0, st>>>(c->tmp, c->fixed + k0 * n, cnt * n);
    }
    // nngb is not permuted (an h-search output); clear it
    cudaMemsetAsync(S.nngb, 0, sizeof(int) * n, st);
    c->cur = other;
    point_carried(c);
    c->inv_valid = false;
    launch_pack(S, c->P, kPackPos | kPackHme | kPackVel | kPackThm, st);
    c->pack_dirty = 0;
    launch_tree_build(S, c->P, st);
    c->tree_dirty = false;
    c->h_dirty_tree = false;
    return check_launch();
}

int ensure_inv(sph3_ctx *c, cudaStream_t st) {
    if (c->inv_valid || c->S.n == 0) return SPH3_OK;
    k_invert<<<blocks_for(c, c->S.n), 256, 0, st>>>(c->S.orig, c->inv, c->S.n);
    c->inv_valid = true;
    return check_launch();
}

// Brings the FP32 packs, Balsara factors and the tree up to date with the
// FP64 fields.  A timestep rebuilds all of them itself (after its own sort),
// so for_step only drops the pending work.
int sync_packs(sph3_ctx *c, cudaStream_t st, bool for_step = false) {
    if (for_step) {
        c->order_dirty = false;
        c->pack_dirty = 0;
        c->bal_dirty = false;
        c->tree_dirty = false;
        c->h_dirty_tree = false;
        return SPH3_OK;
    }
    if (c->order_dirty) {
        const int rc = resort_all(c, st);
        if (rc) return rc;
        c->order_dirty = false;
    }
    if (c->pack_dirty) {
        launch_pack(c->S, c->P, c->pack_dirty, st);
        c->pack_dirty = 0;
    }
    if (c->bal_dirty) {
        launch_balsara(c->S, st);
        c->bal_dirty = false;
    }
    if (c->tree_dirty) {
        launch_tree_build(c->S, c->P, st);
        c->tree_dirty = false;
        c->h_dirty_tree = false;
    }
    if (c->h_dirty_tree) {
        launch_tree_refit_h(c->S, c->P, st);
        c->h_dirty_tree = false;
    }
    return check_launch();
}

void record(sph3_ctx *c, int k, cudaStream_t st) {
    if (c->cfg.timing) cudaEventRecord(c->ev[k], st);
}

// Points inside one step where the host-buffer step moves its inputs in and
// its outputs out, each called on the compute stream: after the gather that
// follows the sort (new order in place, packs not yet built), after the h
// search, before the kick that updates u, and at the end.  second_kick, if
// set, may run the serial order's closing kick itself (returning true), e.g.
// chunk by chunk with each chunk's outputs handed to a copy.
struct StepHooks {
    std::function<void(cudaStream_t)> after_gather, after_h, before_kick, after_u, at_end;
    std::function<bool(cudaStream_t)> second_kick;
};

// One timestep, enqueued on st.  Switches the carried block half way (the
// gather after the sort writes the other block).
void enqueue_step(sph3_ctx *c, double dt, cudaStream_t st, const StepHooks *hk = nullptr) {
    State &S = c->S;
    const Params &P = c->P;
    record(c, 0, st);
    launch_kick_drift(S, P, dt, st);
    launch_cloud_boxes(S, P, st);
    launch_keys(S, P, st);
    record(c, 1, st);
    launch_radix_sort(S, st);
    record(c, 2, st);
    {
        const int other = c->cur ^ 1;
        const int64_t n = c->cap_n;
        const double *srcs[kCarried];
        double *dsts[kCarried];
        int nc[kCarried];
        for (int k = 0; k < kCarried; ++k) {
            srcs[k] = c->carried[c->cur] + k * n;
            dsts[k] = c->carried[other] + k * n;
            nc[k] = 1;
        }
        launch_gather(S, srcs, dsts, kCarried, nc, st);
        launch_gather_orig(S, c->orig_blk[c->cur], c->orig_blk[other], st);
        c->cur = other;
        point_carried(c);
        if (hk && hk->after_gather) hk->after_gather(st);
        launch_pack(S, P, kPackPos | kPackHme | kPackVel, st);
    }
    record(c, 3, st);
    launch_tree_build(S, P, st);
    record(c, 4, st);
    launch_h_search(S, P, st);
    launch_tree_refit_h(S, P, st);
    if (hk && hk->after_h) hk->after_h(st);
    record(c, 5, st);
    launch_density(S, P, P.visc == SPH3_VISC_BALSARA, st);
    record(c, 6, st);
    const bool serial = P.step_order == SPH3_ORDER_SERIAL;
    const bool phi = c->cfg.step_potential != 0;
    if (serial) {
        // the serial driver's order, with the hydro pass and the u update
        // (which need no gravity) before the gravity walk, so that u and the
        // hydro results are final while gravity runs
        launch_hydro(S, P, true, true, st);
        record(c, 7, st);
        if (hk && hk->before_kick) hk->before_kick(st);
        launch_kick_update(S, P, dt, true, false, st);
        if (c->cool) launch_cooling_state(S, c->cool, &c->cool_units, dt, c->ionfrac, st);
        if (hk && hk->after_u) hk->after_u(st);
        record(c, 8, st);
        if (P.gravity) launch_gravity(S, P, st, phi);
        record(c, 9, st);
        if (!(hk && hk->second_kick && hk->second_kick(st))) launch_kick_update(S, P, dt, false, true, st);
    } else {
        if (P.gravity) launch_gravity(S, P, st, phi);
        record(c, 7, st);
        launch_hydro(S, P, true, false, st);
        record(c, 8, st);
        if (hk && hk->before_kick) hk->before_kick(st);
        launch_kick_update(S, P, dt, false, true, st);
        record(c, 9, st);
        launch_hydro(S, P, false, true, st);
        record(c, 10, st);
        launch_u_update(S, P, dt, st);
        if (c->cool) launch_cooling_state(S, c->cool, &c->cool_units, dt, c->ionfrac, st);
        if (hk && hk->after_u) hk->after_u(st);
    }
    // (no energy sums here: the reference's loop takes none per step, and
    // sph3_energy computes them when asked)
    if (hk && hk->at_end) hk->at_end(st);
    record(c, 11, st);
    c->inv_valid = false;
    c->phi_valid = !P.gravity || c->cfg.step_potential != 0;
}

// staging and copy streams of sph3_step_io, made on first use
int ensure_io(sph3_ctx *c, int64_t in_tot, int64_t out_tot) {
    if (!c->h2d) {
        CK(cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking));
        for (auto &e : c->io_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        for (auto &row : c->io_chunk_ev)
            for (auto &e : row) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    if (in_tot > c->io_in_cap) {
        if (c->io_in) cudaFree(c->io_in);
        c->io_in = nullptr;
        c->io_in_cap = 0;
        CK(dalloc(&c->io_in, (size_t)in_tot));
        c->io_in_cap = in_tot;
    }
    if (out_tot > c->io_out_cap) {
        if (c->io_out) cudaFree(c->io_out);
        c->io_out = nullptr;
        c->io_out_cap = 0;
        CK(dalloc(&c->io_out, (size_t)out_tot));
        c->io_out_cap = out_tot;
    }
    return SPH3_OK;
}

// when an input of the host-buffer step is scattered into the state: 0 before
// the first kick, 1 after the gather (h: before the packs and the tree), 2
// after the h search (u: before the EOS), 3 before the kick that updates u
int io_stage_in(int f) {
    switch (f) {
        case SPH3_FIELD_H: return 1;
        case SPH3_FIELD_U: return 2;
        case SPH3_FIELD_U_PREV:
        case SPH3_FIELD_DUDT_PREV: return 3;
        default: return 0;
    }
}

// when an output is final: 0 after the gather (positions), 1 after the h
// search (h, neighbour counts), 2 after the u update (u, its history, the
// density-pass and hydro results), 3 at the end of the step
int io_stage_out(int f) {
    switch (f) {
        case SPH3_FIELD_POS: return 0;
        case SPH3_FIELD_H:
        case SPH3_FIELD_NNGB: return 1;
        case SPH3_FIELD_U:
        case SPH3_FIELD_U_PREV:
        case SPH3_FIELD_DUDT:
        case SPH3_FIELD_DUDT_PREV:
        case SPH3_FIELD_RHO:
        case SPH3_FIELD_P:
        case SPH3_FIELD_C:
        case SPH3_FIELD_ACC_SPH:
        case SPH3_FIELD_VSIG: return 2;
        default: return 3;
    }
}

void accumulate_times(sph3_ctx *c, bool serial) {
    float ms;
    auto add = [&](int slot, int a, int b) {
        if (cudaEventElapsedTime(&ms, c->ev[a], c->ev[b]) == cudaSuccess) c->phase_ms[slot] += ms;
    };
    add(0, 0, 1);
    add(1, 1, 2);
    add(2, 2, 3);
    add(3, 3, 4);
    add(4, 4, 5);
    add(5, 5, 6);
    if (serial) {  // hydro, u update, gravity, second kick (see enqueue_step)
        add(7, 6, 7);
        add(8, 7, 8);
        add(6, 8, 9);
        add(8, 9, 11);
    } else {
        add(6, 6, 7);
        add(7, 7, 8);
        add(8, 8, 9);
        add(7, 9, 10);
        add(8, 10, 11);
    }
}

}  // namespace

// ================================================================== ABI
extern "C" {

int sph3_version(void) { return 10000; }

void sph3_default_config(sph3_config *cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->precision = SPH3_PREC_MIXED;
    cfg->h_mode = SPH3_H_NEWTON;
    cfg->visc = SPH3_VISC_SIGNAL;
    cfg->step_order = SPH3_ORDER_SERIAL;
    cfg->n_ngb = 64;
    cfg->n_ngb_tol = 5;
    cfg->h_max_iter = 64;
    cfg->n_boot = 50;
    cfg->leaf_size = 16;
    cfg->stack_cap = 768;
    cfg->max_level = 16;
    cfg->gravity = 1;
    cfg->quadrupole = 1;
    cfg->walk_warps = 4;
    cfg->list_cap = 128;
    cfg->mac = SPH3_MAC_BH;
    cfg->use_graph = 1;
    cfg->timing = 0;
    cfg->gamma = 5.0 / 3.0;
    cfg->alpha = 1.0;
    cfg->beta = 2.0;
    cfg->eta = 0.1;
    cfg->G = 1.0;
    cfg->theta = 0.5;
    cfg->eps = 0.01;
}

const char *sph3_error_string(int code) {
    switch (code) {
        case SPH3_OK: return "ok";
        case SPH3_ERR_INVALID_ARG: return "invalid argument";
        case SPH3_ERR_CUDA: return "CUDA error";
        case SPH3_ERR_NO_DEVICE: return "no CUDA device";
        case SPH3_ERR_STATE: return "call out of order (no particles loaded?)";
        case SPH3_ERR_UNSUPPORTED: return "unsupported combination (e.g. gravity with a periodic box)";
        case SPH3_ERR_OUT_OF_MEMORY: return "out of device memory";
        case SPH3_ERR_DEVICE_STATUS: return "device status bit set";
        case SPH3_ERR_TOO_LARGE: return "size above the fixed maximum of the no-allocation entry point (65536)";
        default: return "unknown error";
    }
}

int sph3_ctx_create(const sph3_config *cfg, int device, sph3_ctx **out) {
    if (!out) return SPH3_ERR_INVALID_ARG;
    *out = nullptr;
    sph3_config def;
    sph3_default_config(&def);
    if (!cfg) cfg = &def;
    int rc = validate(cfg);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return SPH3_ERR_NO_DEVICE;
    }
    if (device < 0) CK(cudaGetDevice(&device));
    if (device >= ndev) return SPH3_ERR_INVALID_ARG;
    CK(cudaSetDevice(device));
    sph3_ctx *c = new (std::nothrow) sph3_ctx();
    if (!c) return SPH3_ERR_OUT_OF_MEMORY;
    c->cfg = *cfg;
    c->device = device;
    params_from(*cfg, c->P);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        delete c;
        return SPH3_ERR_CUDA;
    }
    c->S.num_sms = prop.multiProcessorCount;
    c->S.walk_blocks = prop.multiProcessorCount * 8;
    c->S.walk_warps = cfg->walk_warps;
    c->S.max_level = cfg->max_level;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return SPH3_ERR_CUDA;
    }
    for (auto &e : c->ev) cudaEventCreate(&e);
    if (cudaMalloc(&c->S.status, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&c->S.counters, sizeof(unsigned long long) * kNumCounters) != cudaSuccess ||
        cudaMalloc(&c->S.work, sizeof(int) * 8) != cudaSuccess ||
        cudaMalloc(&c->S.energy_part, sizeof(double) * 8 * 512) != cudaSuccess ||
        cudaMalloc(&c->S.energy, sizeof(double) * 8) != cudaSuccess) {
        sph3_ctx_destroy(c);
        return SPH3_ERR_OUT_OF_MEMORY;
    }
    cudaMemset(c->S.status, 0, sizeof(unsigned));
    cudaMemset(c->S.counters, 0, sizeof(unsigned long long) * kNumCounters);
    cudaMemset(c->S.energy, 0, sizeof(double) * 8);
    *out = c;
    return SPH3_OK;
}

int sph3_ctx_destroy(sph3_ctx *c) {
    if (!c) return SPH3_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graphs(c);
    free_buffers(c);
    State &S = c->S;
    if (S.status) cudaFree(S.status);
    if (S.counters) cudaFree(S.counters);
    if (S.work) cudaFree(S.work);
    if (S.energy_part) cudaFree(S.energy_part);
    if (S.energy) cudaFree(S.energy);
    for (auto &e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->h2d) cudaStreamSynchronize(c->h2d);
    if (c->d2h) cudaStreamSynchronize(c->d2h);
    for (auto &e : c->io_ev)
        if (e) cudaEventDestroy(e);
    for (auto &row : c->io_chunk_ev)
        for (auto &e : row)
            if (e) cudaEventDestroy(e);
    if (c->io_in) cudaFree(c->io_in);
    if (c->io_out) cudaFree(c->io_out);
    if (c->ionfrac) cudaFree(c->ionfrac);
    if (c->h2d) cudaStreamDestroy(c->h2d);
    if (c->d2h) cudaStreamDestroy(c->d2h);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return SPH3_OK;
}

int sph3_set_config(sph3_ctx *c, const sph3_config *cfg) {
    if (!c) return SPH3_ERR_INVALID_ARG;
    int rc = validate(cfg);
    if (rc) return rc;
    const bool relevel = cfg->max_level != c->cfg.max_level || cfg->leaf_size != c->cfg.leaf_size ||
                         cfg->theta != c->cfg.theta || cfg->quadrupole != c->cfg.quadrupole ||
                         cfg->mac != c->cfg.mac;
    if (cfg->max_level != c->cfg.max_level && c->have) {
        int cb = 0;
        while ((1ll << cb) < (int64_t)c->S.ncloud) ++cb;
        if (3 * cfg->max_level + cb > 63) return SPH3_ERR_INVALID_ARG;
    }
    c->cfg = *cfg;
    params_from(*cfg, c->P);
    c->S.walk_warps = cfg->walk_warps;
    drop_graphs(c);
    if (c->cap_n > 0) {
        cudaSetDevice(c->device);
        rc = ensure_lists(c, std::max<int64_t>(c->cap_n, 1));
        if (rc) return rc;
    }
    if (relevel && c->have) {
        cudaSetDevice(c->device);
        c->S.max_level = cfg->max_level;
        int cb = 0;
        while ((1ll << cb) < (int64_t)c->S.ncloud) ++cb;
        c->S.cloud_bits = cb;
        c->S.key_bits = 3 * cfg->max_level + cb;
        return resort_all(c, c->stream) ? SPH3_ERR_CUDA : cuda_err(cudaStreamSynchronize(c->stream));
    }
    c->S.max_level = cfg->max_level;
    return SPH3_OK;
}

int sph3_get_config(const sph3_ctx *c, sph3_config *cfg) {
    if (!c || !cfg) return SPH3_ERR_INVALID_ARG;
    *cfg = c->cfg;
    return SPH3_OK;
}

int sph3_set_clouds(sph3_ctx *c, const int64_t *counts, int32_t ncloud) {
    if (!c || ncloud < 1 || !counts) return SPH3_ERR_INVALID_ARG;
    for (int k = 0; k < ncloud; ++k)
        if (counts[k] < 0) return SPH3_ERR_INVALID_ARG;
    c->cloud_counts.assign(counts, counts + ncloud);
    return SPH3_OK;
}

int64_t sph3_num_particles(const sph3_ctx *c) { return c ? c->S.n : -1; }

int sph3_set_particles(sph3_ctx *c, int64_t n, const double *pos, const double *vel, const double *mass,
                       const double *u, const double *h, const double *eps, int on_device, void *stream) {
    if (!c || n < 0 || (n > 0 && (!pos || !mass))) return SPH3_ERR_INVALID_ARG;
    if (n > (int64_t)INT32_MAX / 2 - 1024) return SPH3_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    // cloud layout
    std::vector<int64_t> counts = c->cloud_counts;
    if (counts.empty()) counts.push_back(n);
    int64_t tot = 0;
    for (auto k : counts) tot += k;
    if (tot != n) return SPH3_ERR_INVALID_ARG;
    const int ncloud = (int)counts.size();
    int cb = 0;
    while ((1ll << cb) < (int64_t)ncloud) ++cb;
    if (3 * c->cfg.max_level + cb > 63) return SPH3_ERR_INVALID_ARG;
    std::vector<Cloud> cl(ncloud);
    int64_t at = 0;
    for (int k = 0; k < ncloud; ++k) {
        std::memset(&cl[k], 0, sizeof(Cloud));
        cl[k].begin = at;
        cl[k].end = at + counts[k];
        at += counts[k];
    }
    drop_graphs(c);
    // walk groups are rebuilt with every tree; at most one per particle
    int rc = alloc_for(c, n, ncloud, (int)std::max<int64_t>(n, 1));
    if (rc) return rc;
    State &S = c->S;
    S.n = n;
    S.ncloud = ncloud;
    S.ngroups = (int)n;
    S.cloud_bits = cb;
    S.max_level = c->cfg.max_level;
    S.key_bits = 3 * c->cfg.max_level + cb;
    c->cur_counts = counts;
    CK(cudaMemcpyAsync(S.clouds, cl.data(), sizeof(Cloud) * ncloud, cudaMemcpyHostToDevice, st));
    {
        // root-cube reduction items: runs of <= kBoxChunk particles per cloud
        std::vector<int4> items;
        std::vector<int> ibeg(ncloud + 1, 0);
        for (int k = 0; k < ncloud; ++k) {
            ibeg[k] = (int)items.size();
            for (int64_t b = cl[k].begin; b < cl[k].end; b += kBoxChunk)
                items.push_back(make_int4(k, (int)b, (int)std::min<int64_t>(b + kBoxChunk, cl[k].end), 0));
        }
        ibeg[ncloud] = (int)items.size();
        if (S.box_items) cudaFree(S.box_items);
        if (S.box_item_begin) cudaFree(S.box_item_begin);
        if (S.box_part) cudaFree(S.box_part);
        S.box_items = nullptr;
        S.box_item_begin = nullptr;
        S.box_part = nullptr;
        S.nbox_items = (int)items.size();
        CK(dalloc(&S.box_items, items.size()));
        CK(dalloc(&S.box_item_begin, ibeg.size()));
        CK(dalloc(&S.box_part, 6 * items.size()));
        if (!items.empty())
            CK(cudaMemcpyAsync(S.box_items, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S.box_item_begin, ibeg.data(), sizeof(int) * ibeg.size(), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));  // the host vectors go out of scope
    }
    CK(cudaMemsetAsync(S.status, 0, sizeof(unsigned), st));
    CK(cudaMemsetAsync(c->fixed, 0, sizeof(double) * kFixed * std::max<int64_t>(n, 1), st));
    CK(cudaMemsetAsync(c->carried[c->cur], 0, sizeof(double) * kCarried * std::max<int64_t>(n, 1), st));
    if (n > 0) {
        k_iota64<<<blocks_for(c, n), 256, 0, st>>>(S.orig, n);
        const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        auto put = [&](const double *src, double *dst, int ncomp) -> int {
            CK(cudaMemcpyAsync(c->staging, src, sizeof(double) * n * ncomp, kind, st));
            k_scatter_in<<<blocks_for(c, n), 256, 0, st>>>(c->staging, dst, S.orig, n, ncomp);
            return check_launch();
        };
        if ((rc = put(pos, S.pos, 3))) return rc;
        if ((rc = put(mass, S.m, 1))) return rc;
        if (vel && (rc = put(vel, S.vel, 3))) return rc;
        if (u && (rc = put(u, S.u, 1))) return rc;
        if (u) CK(cudaMemcpyAsync(S.u_prev, S.u, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        if (h && (rc = put(h, S.h, 1))) return rc;
        if (eps) {
            if ((rc = put(eps, S.eps, 1))) return rc;
        } else {
            k_fill<<<blocks_for(c, n), 256, 0, st>>>(S.eps, n, c->cfg.eps);
        }
        launch_check_finite(S, st);
    }
    c->have = true;
    c->phi_valid = false;
    rc = ensure_ionfrac(c);
    if (rc) return rc;
    rc = resort_all(c, st);
    if (rc) return rc;
    CK(cudaStreamSynchronize(st));
    return SPH3_OK;
}

int sph3_set_field(sph3_ctx *c, int field, const double *src, int on_device, void *stream) {
    if (!c || !src) return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    int ncomp;
    double *dst = field_ptr(c, field, &ncomp);
    if (!dst) return SPH3_ERR_INVALID_ARG;
    const int64_t n = c->S.n;
    if (n == 0) return SPH3_OK;
    // the captured step graphs stay valid: buffers do not move
    CK(cudaMemcpyAsync(c->staging, src, sizeof(double) * n * ncomp,
                       on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    k_scatter_in<<<blocks_for(c, n), 256, 0, st>>>(c->staging, dst, c->S.orig, n, ncomp);
    int rc = check_launch();
    if (rc) return rc;
    switch (field) {
        case SPH3_FIELD_POS:
            // re-sorted lazily: by the next pass that needs the tree, or by
            // the next step, which sorts anyway
            c->order_dirty = true;
            c->S.list_valid = false;
            c->phi_valid = false;
            break;
        case SPH3_FIELD_VEL: c->pack_dirty |= kPackVel; break;
        case SPH3_FIELD_MASS:
        case SPH3_FIELD_EPS:
            c->pack_dirty |= kPackHme;
            c->tree_dirty = true;
            c->phi_valid = false;
            break;
        case SPH3_FIELD_H:
            c->pack_dirty |= kPackHme;
            c->h_dirty_tree = true;
            c->bal_dirty = true;
            c->S.list_valid = false;
            break;
        case SPH3_FIELD_RHO:
        case SPH3_FIELD_P: c->pack_dirty |= kPackThm; break;
        case SPH3_FIELD_C:
        case SPH3_FIELD_DIVV:
        case SPH3_FIELD_CURLV: c->pack_dirty |= kPackThm; c->bal_dirty = true; break;
        case SPH3_FIELD_BALSARA: c->pack_dirty |= kPackThm; break;
        default: break;
    }
    CK(cudaStreamSynchronize(st));
    return SPH3_OK;
}

int sph3_get_field(sph3_ctx *c, int field, double *dst, int64_t row_begin, int64_t row_end, int on_device,
                   void *stream) {
    if (!c || (!dst && row_end > row_begin)) return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    const int64_t n = c->S.n;
    if (row_begin < 0 || row_end > n || row_begin > row_end) return SPH3_ERR_INVALID_ARG;
    if (row_end == row_begin) return SPH3_OK;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    int rc = ensure_inv(c, st);
    if (rc) return rc;
    const int64_t cnt = row_end - row_begin;
    int ncomp = 1;
    if (field == SPH3_FIELD_NNGB) {
        k_gather_out_int<<<blocks_for(c, cnt), 256, 0, st>>>(c->S.nngb, c->staging, c->inv, row_begin, row_end);
    } else {
        double *src = field_ptr(c, field, &ncomp);
        if (!src) return SPH3_ERR_INVALID_ARG;
        k_gather_out<<<blocks_for(c, cnt), 256, 0, st>>>(src, c->staging, c->inv, n, ncomp, row_begin, row_end);
    }
    rc = check_launch();
    if (rc) return rc;
    CK(cudaMemcpyAsync(dst, c->staging, sizeof(double) * cnt * ncomp,
                       on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    if (!on_device) CK(cudaStreamSynchronize(st));
    return SPH3_OK;
}

namespace {
// the body of sph3_compute over whatever group table S holds
int compute_impl(sph3_ctx *c, uint32_t what, cudaStream_t st) {
    State &S = c->S;
    const Params &P = c->P;
    int rc = sync_packs(c, st);
    if (rc) return rc;
    if (what & SPH3_DO_BOOT_H) {
        launch_boot_h(S, P, st);
        c->h_dirty_tree = true;
        c->bal_dirty = true;
    }
    if (what & SPH3_DO_H) {
        launch_h_search(S, P, st);
        c->h_dirty_tree = true;
        c->bal_dirty = true;
        if (P.eps_from_h) c->phi_valid = false;  // eps follows h
    }
    if ((rc = sync_packs(c, st))) return rc;
    if (what & SPH3_DO_DENSITY) {
        launch_density(S, P, (what & SPH3_DO_DIVCURL) != 0, st);
        c->bal_dirty = false;
    } else if (what & SPH3_DO_DIVCURL) {
        // div/curl alone (div_curlVel): keep the stored rho, P, c
        launch_density(S, P, true, st, true);
        c->bal_dirty = false;
    }
    if (what & SPH3_DO_EOS) {
        launch_eos(S, P, st);
        c->bal_dirty = false;
    }
    if ((rc = sync_packs(c, st))) return rc;
    if (what & SPH3_DO_GRAVITY) {
        launch_gravity(S, P, st, true);
        c->phi_valid = true;
    }
    if (what & (SPH3_DO_ACC_SPH | SPH3_DO_DUDT))
        launch_hydro(S, P, (what & SPH3_DO_ACC_SPH) != 0, (what & SPH3_DO_DUDT) != 0, st);
    return check_launch();
}
}  // namespace

int sph3_compute(sph3_ctx *c, uint32_t what, void *stream) {
    if (!c) return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    if (c->S.n == 0) return SPH3_OK;
    if ((what & SPH3_DO_GRAVITY) && c->P.periodic) return SPH3_ERR_UNSUPPORTED;
    const int rc = compute_impl(c, what, st);
    if (rc) return rc;
    CK(cudaStreamSynchronize(st));
    return SPH3_OK;
}

int sph3_compute_rows(sph3_ctx *c, uint32_t what, int64_t row_begin, int64_t row_end, void *stream) {
    if (!c) return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    State &S = c->S;
    if (row_begin < 0 || row_end > S.n || row_begin > row_end) return SPH3_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    if (S.n == 0 || row_begin == row_end) return SPH3_OK;
    if ((what & SPH3_DO_GRAVITY) && c->P.periodic) return SPH3_ERR_UNSUPPORTED;
    int rc = sync_packs(c, st);  // order, tree and groups as the full call would see them
    if (rc) return rc;
    if (c->sub_cap < (int64_t)c->cap_groups || !c->row_flag) {
        if (c->sub_groups) cudaFree(c->sub_groups);
        if (c->sub_cloud) cudaFree(c->sub_cloud);
        if (c->sub_n) cudaFree(c->sub_n);
        if (c->row_flag) cudaFree(c->row_flag);
        c->sub_groups = nullptr;
        c->sub_cloud = nullptr;
        c->sub_n = nullptr;
        c->row_flag = nullptr;
        c->sub_cap = 0;
        CK(dalloc(&c->sub_groups, c->cap_groups));
        CK(dalloc(&c->sub_cloud, c->cap_groups));
        CK(dalloc(&c->sub_n, 1));
        CK(dalloc(&c->row_flag, c->cap_n));
        c->sub_cap = c->cap_groups;
    }
    const int64_t n = S.n;
    k_invert<<<blocks_for(c, n), 256, 0, st>>>(S.orig, c->inv, n);
    CK(cudaMemsetAsync(c->row_flag, 0, (size_t)n, st));
    CK(cudaMemsetAsync(c->sub_n, 0, sizeof(int), st));
    k_mark_rows<<<blocks_for(c, row_end - row_begin), 256, 0, st>>>(c->inv, row_begin, row_end, c->row_flag);
    k_select_groups<<<c->S.num_sms * 4, 256, 0, st>>>(S.groups, S.group_cloud, S.ngroups_dev, c->row_flag,
                                                      c->sub_groups, c->sub_cloud, c->sub_n);
    // the walks run over the selected groups only
    std::swap(S.groups, c->sub_groups);
    std::swap(S.group_cloud, c->sub_cloud);
    std::swap(S.ngroups_dev, c->sub_n);
    rc = compute_impl(c, what, st);
    std::swap(S.groups, c->sub_groups);
    std::swap(S.group_cloud, c->sub_cloud);
    std::swap(S.ngroups_dev, c->sub_n);
    // lists, potentials and div/curl exist for these rows only
    S.list_valid = false;
    c->phi_valid = false;
    c->inv_valid = true;
    if (rc) return rc;
    CK(cudaStreamSynchronize(st));
    return SPH3_OK;
}

int sph3_first_step(sph3_ctx *c, double dt, void *stream) {
    if (!c) return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    State &S = c->S;
    const Params &P = c->P;
    if (S.n == 0) return SPH3_OK;
    int rc = sync_packs(c, st);
    if (rc) return rc;
    // bootstrap h where none was given (h <= 0 everywhere is the signal)
    std::vector<double> h0(1);
    CK(cudaMemcpyAsync(h0.data(), S.h, sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (!(h0[0] > 0.0)) {
        // the reference rule starts from its exact bootstrap; Newton needs only a start
        if (P.h_mode == SPH3_H_REFSTEP) launch_boot_h(S, P, st);
        else launch_h_guess(S, P, st);
    }
    launch_h_search(S, P, st);
    launch_tree_refit_h(S, P, st);
    launch_density(S, P, P.visc == SPH3_VISC_BALSARA, st);
    if (P.gravity) launch_gravity(S, P, st, true);
    else cudaMemsetAsync(S.acc_g, 0, sizeof(double) * 3 * c->cap_n, st);
    c->phi_valid = true;
    launch_hydro(S, P, true, true, st);
    launch_first_u(S, P, dt, st);
    launch_energy(S, P, st);
    c->h_dirty_tree = false;
    c->bal_dirty = false;
    rc = check_launch();
    if (rc) return rc;
    CK(cudaStreamSynchronize(st));
    return SPH3_OK;
}

int sph3_step(sph3_ctx *c, double dt, int32_t nsteps, void *stream) {
    if (!c || nsteps < 0) return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    State &S = c->S;
    if (S.n == 0) return SPH3_OK;
    int rc = sync_packs(c, st, true);
    if (rc) return rc;
    if (!c->P.gravity) cudaMemsetAsync(S.acc_g, 0, sizeof(double) * 3 * c->cap_n, st);
    const bool serial = c->P.step_order == SPH3_ORDER_SERIAL;
    for (int s = 0; s < nsteps; ++s) {
        const bool graph_ok = c->cfg.use_graph && !c->cfg.timing && c->warm_steps >= 2;
        if (!graph_ok) {
            enqueue_step(c, dt, st);
            rc = check_launch();
            if (rc) return rc;
            if (c->cfg.timing) {
                CK(cudaEventSynchronize(c->ev[11]));
                accumulate_times(c, serial);
            }
            ++c->warm_steps;
            continue;
        }
        const int par = c->cur;
        // capture the graphs of both carried-block parities together, so that
        // later steps only replay (no capture inside a timed sequence)
        for (int q = 0; q < 2; ++q) {
            const int pq = par ^ q;
            if (c->graph[pq] && c->graph_dt[pq] != dt) {
                cudaGraphExecDestroy(c->graph[pq]);
                c->graph[pq] = nullptr;
            }
            if (c->graph[pq]) continue;
            c->cur = pq;
            point_carried(c);
            cudaGraph_t g;
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            enqueue_step(c, dt, st);
            cudaError_t e = cudaStreamEndCapture(st, &g);
            if (e != cudaSuccess) return SPH3_ERR_CUDA;
            c->graph_kernels[pq] = count_kernel_nodes(g);
            e = cudaGraphInstantiate(&c->graph[pq], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return SPH3_ERR_CUDA;
            c->graph_dt[pq] = dt;
        }
        // capture switched the carried block without running: restore it
        c->cur = par;
        point_carried(c);
        CK(cudaGraphLaunch(c->graph[par], st));
        c->cur = par ^ 1;
        point_carried(c);
        c->inv_valid = false;
    }
    if (c->cool && nsteps > 0) c->ionfrac_valid = true;
    return SPH3_OK;
}

int sph3_step_io(sph3_ctx *c, double dt, int32_t nsteps, int32_t nin, const int32_t *in_fields,
                 const double *const *in, int32_t nout, const int32_t *out_fields, double *const *out,
                 void *stream) {
    if (!c || nsteps < 1 || nin < 0 || nout < 0 || (nin > 0 && (!in_fields || !in)) ||
        (nout > 0 && (!out_fields || !out)))
        return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    State &S = c->S;
    const int64_t n = S.n;
    std::vector<int64_t> in_off(nin), out_off(nout);
    std::vector<int> in_nc(nin), out_nc(nout);
    int64_t in_tot = 0, out_tot = 0;
    bool has_u = false, has_uprev = false;
    for (int k = 0; k < nin; ++k) {
        int nc = 1;
        if (!in[k] || !field_ptr(c, in_fields[k], &nc)) return SPH3_ERR_INVALID_ARG;
        has_u |= in_fields[k] == SPH3_FIELD_U;
        has_uprev |= in_fields[k] == SPH3_FIELD_U_PREV;
        in_off[k] = in_tot;
        in_nc[k] = nc;
        in_tot += nc * n;
    }
    for (int k = 0; k < nout; ++k) {
        int nc = 1;
        if (!out[k] || (out_fields[k] != SPH3_FIELD_NNGB && !field_ptr(c, out_fields[k], &nc)))
            return SPH3_ERR_INVALID_ARG;
        out_off[k] = out_tot;
        out_nc[k] = nc;
        out_tot += nc * n;
    }
    if (n == 0) return SPH3_OK;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    int rc = ensure_io(c, std::max<int64_t>(in_tot, 1), std::max<int64_t>(out_tot, 1));
    if (rc) return rc;
    if ((rc = sync_packs(c, st, true))) return rc;
    if (!c->P.gravity) CK(cudaMemsetAsync(S.acc_g, 0, sizeof(double) * 3 * c->cap_n, st));
    // everything below, up to the join of the copy streams, is one enqueue:
    // run directly or captured once and replayed as a graph
    auto enqueue_io = [&]() -> int {
        // Inputs: host -> staging on the copy stream, ordered by when the step
        // needs them.  The first group (positions, velocities, accelerations:
        // everything the opening kick reads) goes in row chunks, each scattered
        // into the state as soon as it has landed, so the scatter kernels overlap
        // the rest of the copy.
        const int nchunk = n >= (int64_t)kIoChunks * 8192 ? kIoChunks : 1;
        auto chunk_rows = [&](int ch, int64_t &b, int64_t &e) {
            b = n * ch / nchunk;
            e = n * (ch + 1) / nchunk;
        };
        CK(cudaEventRecord(c->io_ev[9], st));
        CK(cudaStreamWaitEvent(c->h2d, c->io_ev[9], 0));
        for (int ch = 0; ch < nchunk; ++ch) {
            int64_t b, e;
            chunk_rows(ch, b, e);
            for (int k = 0; k < nin; ++k)
                if (io_stage_in(in_fields[k]) == 0)
                    CK(cudaMemcpyAsync(c->io_in + in_off[k] + b * in_nc[k], in[k] + b * in_nc[k],
                                       sizeof(double) * in_nc[k] * (e - b), cudaMemcpyHostToDevice, c->h2d));
            CK(cudaEventRecord(c->io_chunk_ev[0][ch], c->h2d));
        }
        for (int stage = 1; stage < 4; ++stage) {
            for (int k = 0; k < nin; ++k)
                if (io_stage_in(in_fields[k]) == stage)
                    CK(cudaMemcpyAsync(c->io_in + in_off[k], in[k], sizeof(double) * in_nc[k] * n,
                                       cudaMemcpyHostToDevice, c->h2d));
            CK(cudaEventRecord(c->io_ev[stage], c->h2d));
        }
        // staging -> state in the current order (field pointers looked up when the
        // hook runs: the carried block switches inside the step)
        auto scatter = [&](int stage, cudaStream_t s) {
            cudaStreamWaitEvent(s, c->io_ev[stage], 0);
            for (int k = 0; k < nin; ++k) {
                if (io_stage_in(in_fields[k]) != stage) continue;
                int nc = 1;
                double *dst = field_ptr(c, in_fields[k], &nc);
                k_scatter_in<<<blocks_for(c, n), 256, 0, s>>>(c->io_in + in_off[k], dst, S.orig, n, nc);
            }
            // the reference's loop keeps u_previous = u between iterations
            // (sph_serial.py:181-182): an input u alone sets both
            if (stage == 3 && has_u && !has_uprev)
                cudaMemcpyAsync(S.u_prev, S.u, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
        };
        // outputs: state -> staging in the caller's order as soon as each is final
        auto gather = [&](int stage, cudaStream_t s) {
            for (int k = 0; k < nout; ++k) {
                if (io_stage_out(out_fields[k]) != stage) continue;
                if (out_fields[k] == SPH3_FIELD_NNGB) {
                    k_gather_out_int<<<blocks_for(c, n), 256, 0, s>>>(S.nngb, c->io_out + out_off[k], c->inv, 0, n);
                } else {
                    int nc = 1;
                    const double *src = field_ptr(c, out_fields[k], &nc);
                    k_gather_out<<<blocks_for(c, n), 256, 0, s>>>(src, c->io_out + out_off[k], c->inv, n, nc, 0, n);
                }
            }
            cudaEventRecord(c->io_ev[4 + stage], s);
        };
        // the first group by rows, through the inverse of the current order
        k_invert<<<blocks_for(c, n), 256, 0, st>>>(S.orig, c->inv, n);
        for (int ch = 0; ch < nchunk; ++ch) {
            int64_t b, e;
            chunk_rows(ch, b, e);
            CK(cudaStreamWaitEvent(st, c->io_chunk_ev[0][ch], 0));
            for (int k = 0; k < nin; ++k) {
                if (io_stage_in(in_fields[k]) != 0) continue;
                int nc = 1;
                double *dst = field_ptr(c, in_fields[k], &nc);
                k_scatter_rows<<<blocks_for(c, e - b), 256, 0, st>>>(c->io_in + in_off[k], dst, c->inv, n, nc, b, e);
            }
        }
        // The closing outputs (velocities, accelerations and whatever else is
        // final only at the end) by rows as well: in the serial order the closing
        // kick runs chunk by chunk in caller order, each chunk gathered into the
        // staging and copied out while the next is kicked.
        bool tail_chunked = false;
        for (int k = 0; k < nout; ++k) tail_chunked |= io_stage_out(out_fields[k]) == 3;
        tail_chunked &= c->P.step_order == SPH3_ORDER_SERIAL;
        auto gather_rows = [&](int64_t b, int64_t e, cudaStream_t s) {
            for (int k = 0; k < nout; ++k) {
                if (io_stage_out(out_fields[k]) != 3) continue;
                int nc = 1;
                const double *src = field_ptr(c, out_fields[k], &nc);
                k_gather_out<<<blocks_for(c, e - b), 256, 0, s>>>(src, c->io_out + out_off[k] + b * nc, c->inv, n, nc,
                                                                  b, e);
            }
        };
        for (int step = 0; step < nsteps; ++step) {
            const bool first = step == 0, last = step == nsteps - 1;
            StepHooks hk;
            hk.after_gather = [&](cudaStream_t s) {
                if (first) scatter(1, s);
                if (last) {
                    k_invert<<<blocks_for(c, n), 256, 0, s>>>(S.orig, c->inv, n);
                    gather(0, s);
                }
            };
            hk.after_h = [&](cudaStream_t s) {
                if (first) scatter(2, s);
                if (last) gather(1, s);
            };
            hk.before_kick = [&](cudaStream_t s) {
                if (first) scatter(3, s);
            };
            hk.after_u = [&](cudaStream_t s) {
                if (last) gather(2, s);
            };
            hk.at_end = [&](cudaStream_t s) {
                if (last && !tail_chunked) gather(3, s);
            };
            if (last && tail_chunked)
                hk.second_kick = [&](cudaStream_t s) {
                    for (int ch = 0; ch < nchunk; ++ch) {
                        int64_t b, e;
                        chunk_rows(ch, b, e);
                        launch_kick_rows(S, dt, c->inv, b, e, s);
                        gather_rows(b, e, s);
                        cudaEventRecord(c->io_chunk_ev[1][ch], s);
                    }
                    return true;
                };
            enqueue_step(c, dt, st, &hk);
            if ((rc = check_launch())) return rc;
        }
        // staging -> host on the other copy stream, each group as soon as it is
        // final (the closing group chunk by chunk when the kick ran by rows)
        for (int stage = 0; stage < 4; ++stage) {
            if (stage == 3 && tail_chunked) {
                for (int ch = 0; ch < nchunk; ++ch) {
                    int64_t b, e;
                    chunk_rows(ch, b, e);
                    CK(cudaStreamWaitEvent(c->d2h, c->io_chunk_ev[1][ch], 0));
                    for (int k = 0; k < nout; ++k)
                        if (io_stage_out(out_fields[k]) == 3)
                            CK(cudaMemcpyAsync(out[k] + b * out_nc[k], c->io_out + out_off[k] + b * out_nc[k],
                                               sizeof(double) * out_nc[k] * (e - b), cudaMemcpyDeviceToHost, c->d2h));
                }
                continue;
            }
            CK(cudaStreamWaitEvent(c->d2h, c->io_ev[4 + stage], 0));
            for (int k = 0; k < nout; ++k)
                if (io_stage_out(out_fields[k]) == stage)
                    CK(cudaMemcpyAsync(out[k], c->io_out + out_off[k], sizeof(double) * out_nc[k] * n,
                                       cudaMemcpyDeviceToHost, c->d2h));
        }
        // the copy-out stream joins the step's stream
        CK(cudaEventRecord(c->io_ev[8], c->d2h));
        CK(cudaStreamWaitEvent(st, c->io_ev[8], 0));
        return SPH3_OK;
    };
    // Replay a graph when this call repeats an earlier one (same buffers,
    // fields, dt and step count, every host buffer page-locked: a captured copy
    // from pageable memory is not allowed); the first such call captures it.
    bool pinned = true;
    auto is_pinned = [](const void *ptr) {
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return at.type == cudaMemoryTypeHost;
    };
    for (int k = 0; k < nin; ++k) pinned = pinned && is_pinned(in[k]);
    for (int k = 0; k < nout; ++k) pinned = pinned && is_pinned(out[k]);
    const bool graph_ok = pinned && c->cfg.use_graph && !c->cfg.timing && c->warm_steps >= 2;
    if (!graph_ok) {
        if ((rc = enqueue_io())) return rc;
        c->warm_steps += nsteps;
    } else {
        std::vector<uint64_t> key;
        uint64_t dtb;
        std::memcpy(&dtb, &dt, sizeof(dtb));
        key.push_back(dtb);
        key.push_back((uint64_t)nsteps);
        key.push_back((uint64_t)n);
        key.push_back((uint64_t)nin);
        for (int k = 0; k < nin; ++k) {
            key.push_back((uint64_t)in_fields[k]);
            key.push_back((uint64_t)(uintptr_t)in[k]);
        }
        key.push_back((uint64_t)nout);
        for (int k = 0; k < nout; ++k) {
            key.push_back((uint64_t)out_fields[k]);
            key.push_back((uint64_t)(uintptr_t)out[k]);
        }
        const int par = c->cur;
        if (!c->io_graph[par] || c->io_key[par] != key) {
            if (c->io_graph[par]) cudaGraphExecDestroy(c->io_graph[par]);
            c->io_graph[par] = nullptr;
            cudaGraph_t g;
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            rc = enqueue_io();
            cudaError_t e = cudaStreamEndCapture(st, &g);
            // capture switched the carried block without running: restore it
            c->cur = par;
            point_carried(c);
            if (rc) return rc;
            if (e != cudaSuccess) return SPH3_ERR_CUDA;
            e = cudaGraphInstantiate(&c->io_graph[par], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return SPH3_ERR_CUDA;
            c->io_key[par] = key;
        }
        CK(cudaGraphLaunch(c->io_graph[par], st));
        c->cur = par ^ (nsteps & 1);
        point_carried(c);
    }
    CK(cudaStreamSynchronize(st));
    c->inv_valid = true;
    if (c->cool) c->ionfrac_valid = true;
    return SPH3_OK;
}

int sph3_timestep(sph3_ctx *c, double c_cfl, int all_pairs, double *dt_min, void *stream) {
    if (!c || !dt_min || !(c_cfl > 0.0)) return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    State &S = c->S;
    if (S.n == 0) {
        *dt_min = INFINITY;
        return SPH3_OK;
    }
    int rc = sync_packs(c, st);
    if (rc) return rc;
    // div v at the current positions and velocities (rho, P, c kept)
    launch_density(S, c->P, true, st, true);
    c->bal_dirty = false;
    launch_timestep(S, c->P, c_cfl, all_pairs != 0, c->staging, st);
    rc = check_launch();
    if (rc) return rc;
    CK(cudaMemcpyAsync(dt_min, c->staging, sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return SPH3_OK;
}

int sph3_kernels_per_step(sph3_ctx *c, int64_t *out) {
    if (!c || !out) return SPH3_ERR_INVALID_ARG;
    const int64_t k = c->graph_kernels[c->cur];
    *out = k > 0 ? k : -1;
    return SPH3_OK;
}

int sph3_energy(sph3_ctx *c, double out[8], void *stream) {
    if (!c || !out) return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    if (!c->phi_valid && c->S.n > 0) {
        // the steps ran without the potential: one gravity walk with it
        int rc = sync_packs(c, st);
        if (rc) return rc;
        if (c->P.gravity && !c->P.periodic) launch_gravity(c->S, c->P, st, true);
        else CK(cudaMemsetAsync(c->S.phi, 0, sizeof(double) * c->S.n, st));
        rc = check_launch();
        if (rc) return rc;
        c->phi_valid = true;
    }
    launch_energy(c->S, c->P, st);
    CK(cudaMemcpyAsync(out, c->S.energy, sizeof(double) * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return SPH3_OK;
}

int sph3_status(sph3_ctx *c, uint32_t *status, int clear) {
    if (!c || !status) return SPH3_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaDeviceSynchronize());
    unsigned v = 0;
    CK(cudaMemcpy(&v, c->S.status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (clear) CK(cudaMemset(c->S.status, 0, sizeof(unsigned)));
    *status = v;
    return SPH3_OK;
}

static int rows_to_sorted(sph3_ctx *c, const int64_t *rows, int64_t nrows, std::vector<int64_t> &sorted) {
    cudaStream_t st = c->stream;
    int rc = ensure_inv(c, st);
    if (rc) return rc;
    std::vector<int64_t> inv(c->S.n);
    CK(cudaMemcpyAsync(inv.data(), c->inv, sizeof(int64_t) * c->S.n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    sorted.resize(nrows);
    for (int64_t r = 0; r < nrows; ++r) {
        if (rows[r] < 0 || rows[r] >= c->S.n) return SPH3_ERR_INVALID_ARG;
        sorted[r] = inv[rows[r]];
    }
    return SPH3_OK;
}

int sph3_gravity_direct_rows(sph3_ctx *c, const int64_t *rows, int64_t nrows, double *acc, double *phi) {
    if (!c || nrows < 0 || (nrows > 0 && (!rows || !acc))) return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    if (nrows == 0) return SPH3_OK;
    CK(cudaSetDevice(c->device));
    std::vector<int64_t> srt;
    int rc = rows_to_sorted(c, rows, nrows, srt);
    if (rc) return rc;
    cudaStream_t st = c->stream;
    DevTmp<int64_t> drows;
    DevTmp<double> dacc, dphi;
    CK(drows.alloc(nrows));
    CK(dacc.alloc(3 * nrows));
    CK(dphi.alloc(nrows));
    CK(cudaMemcpyAsync(drows.p, srt.data(), sizeof(int64_t) * nrows, cudaMemcpyHostToDevice, st));
    launch_gravity_direct(c->S, c->P, drows.p, nrows, dacc.p, dphi.p, st);
    rc = check_launch();
    if (!rc) {
        CK(cudaMemcpyAsync(acc, dacc.p, sizeof(double) * 3 * nrows, cudaMemcpyDeviceToHost, st));
        if (phi) CK(cudaMemcpyAsync(phi, dphi.p, sizeof(double) * nrows, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    return rc;
}

int sph3_neighbours(sph3_ctx *c, const int64_t *rows, int64_t nrows, int64_t *offsets, int64_t *idx, int64_t cap) {
    if (!c || nrows < 0 || !offsets || (nrows > 0 && !rows) || cap < 0 || (cap > 0 && !idx))
        return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    offsets[0] = 0;
    if (nrows == 0) return SPH3_OK;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    int rc = sync_packs(c, st);
    if (rc) return rc;
    std::vector<int64_t> srt;
    rc = rows_to_sorted(c, rows, nrows, srt);
    if (rc) return rc;
    DevTmp<int64_t> drows, doff, didx;
    CK(drows.alloc(nrows));
    CK(doff.alloc(nrows + 1));
    CK(didx.alloc(std::max<int64_t>(cap, 1)));
    CK(cudaMemcpyAsync(drows.p, srt.data(), sizeof(int64_t) * nrows, cudaMemcpyHostToDevice, st));
    launch_neighbours(c->S, c->P, drows.p, nrows, doff.p, didx.p, cap, st);
    rc = check_launch();
    if (!rc) {
        CK(cudaMemcpyAsync(offsets, doff.p, sizeof(int64_t) * (nrows + 1), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        const int64_t tot = std::min(offsets[nrows], cap);
        if (tot > 0) CK(cudaMemcpy(idx, didx.p, sizeof(int64_t) * tot, cudaMemcpyDeviceToHost));
        for (int64_t r = 0; r < nrows; ++r) {
            const int64_t b = std::min(offsets[r], cap), e = std::min(offsets[r + 1], cap);
            std::sort(idx + b, idx + e);
        }
    }
    return rc;
}

int sph3_pair_lists(sph3_ctx *c, const int64_t *rows, int64_t nrows, int64_t *offsets, int64_t *idx, int64_t cap) {
    if (!c || nrows < 0 || !offsets || (nrows > 0 && !rows) || cap < 0 || (cap > 0 && !idx))
        return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    offsets[0] = 0;
    if (nrows == 0) return SPH3_OK;
    State &S = c->S;
    if (!S.list_valid || S.list_cap == 0) return SPH3_ERR_STATE;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    std::vector<int64_t> srt;
    int rc = rows_to_sorted(c, rows, nrows, srt);
    if (rc) return rc;
    std::vector<int64_t> orig(S.n);
    CK(cudaMemcpyAsync(orig.data(), S.orig, sizeof(int64_t) * S.n, cudaMemcpyDeviceToHost, st));
    std::vector<int> cnt(nrows), row(S.list_cap);
    for (int64_t r = 0; r < nrows; ++r)
        CK(cudaMemcpyAsync(&cnt[r], S.nlist + srt[r], sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    int64_t pos = 0;
    for (int64_t r = 0; r < nrows; ++r) {
        const int k = std::min(cnt[r], S.list_cap);
        CK(cudaMemcpy(row.data(), S.list + (size_t)srt[r] * S.list_cap, sizeof(int) * k, cudaMemcpyDeviceToHost));
        const int64_t b = pos;
        for (int s = 0; s < k; ++s, ++pos)
            if (pos < cap) idx[pos] = orig[row[s]];
        std::sort(idx + std::min(b, cap), idx + std::min(pos, cap));
        offsets[r + 1] = pos;
    }
    return SPH3_OK;
}

int sph3_morton_order(sph3_ctx *c, int64_t *order, uint64_t *keys) {
    if (!c) return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    if (c->S.n == 0) return SPH3_OK;
    CK(cudaSetDevice(c->device));
    const int rc = sync_packs(c, c->stream);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    if (order) CK(cudaMemcpy(order, c->S.orig, sizeof(int64_t) * c->S.n, cudaMemcpyDeviceToHost));
    if (keys) CK(cudaMemcpy(keys, c->S.key, sizeof(uint64_t) * c->S.n, cudaMemcpyDeviceToHost));
    return SPH3_OK;
}

int sph3_counters(sph3_ctx *c, int64_t out[16], int clear) {
    if (!c || !out) return SPH3_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    unsigned long long v[kNumCounters];
    CK(cudaMemcpy(v, c->S.counters, sizeof(v), cudaMemcpyDeviceToHost));
    for (int k = 0; k < kNumCounters; ++k) out[k] = (int64_t)v[k];
    if (clear) CK(cudaMemset(c->S.counters, 0, sizeof(v)));
    return SPH3_OK;
}

int sph3_phase_times(sph3_ctx *c, double out[9], int clear) {
    if (!c || !out) return SPH3_ERR_INVALID_ARG;
    for (int k = 0; k < 9; ++k) out[k] = c->phase_ms[k];
    if (clear)
        for (double &v : c->phase_ms) v = 0;
    return SPH3_OK;
}

// ------------------------------------------------------------ reference-order sums
int sph3_gravity_pairsum(sph3_ctx *c, int form, int64_t nbeg, int64_t nend, double *out, int on_device,
                         void *stream) {
    if (!c || (form != SPH3_GSUM_ROWS && form != SPH3_GSUM_MIMJ)) return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    const int64_t n = c->S.n;
    if (nbeg < 0 || nend > n || nbeg > nend) return SPH3_ERR_INVALID_ARG;
    const int64_t rows = form == SPH3_GSUM_ROWS ? nend - nbeg : n;
    if (rows == 0) return SPH3_OK;
    if (!out) return SPH3_ERR_INVALID_ARG;
    if (c->S.ncloud > 1 || c->P.periodic) return SPH3_ERR_UNSUPPORTED;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    int rc = ensure_inv(c, st);
    if (rc) return rc;
    double *src = c->tmp;  // [5][n] caller order
    launch_caller_sources(c->S, c->inv, src, st);
    double *dst = on_device ? out : c->staging;
    if (form == SPH3_GSUM_ROWS) {
        launch_grav_pairsum(src, n, nbeg, nend, 0, n, c->P.G, dst, st);
    } else {
        // rows below nbeg receive nothing
        if (nbeg > 0) CK(cudaMemsetAsync(dst, 0, sizeof(double) * 3 * nbeg, st));
        launch_grav_pairsum(src, n, nbeg, n, nbeg, nend, c->P.G, dst + 3 * nbeg, st);
    }
    rc = check_launch();
    if (rc) return rc;
    if (!on_device) {
        CK(cudaMemcpyAsync(out, c->staging, sizeof(double) * 3 * rows, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    return SPH3_OK;
}

int sph3_potential_pairsum(sph3_ctx *c, double *pe, void *stream) {
    if (!c || !pe) return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    const int64_t n = c->S.n;
    *pe = 0.0;
    if (n == 0) return SPH3_OK;
    if (c->S.ncloud > 1 || c->P.periodic) return SPH3_ERR_UNSUPPORTED;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    int rc = ensure_inv(c, st);
    if (rc) return rc;
    launch_caller_sources(c->S, c->inv, c->tmp, st);
    launch_pe_rows(c->tmp, n, c->P.G, c->staging, st);
    rc = check_launch();
    if (rc) return rc;
    std::vector<double> part(n);
    CK(cudaMemcpyAsync(part.data(), c->staging, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += part[i];
    *pe = s;
    return SPH3_OK;
}

int sph3_kth_distance(sph3_ctx *c, const double *qpos, int64_t m, int32_t k, double *out, int on_device,
                      void *stream) {
    if (!c || m < 0 || k < 0 || (m > 0 && (!qpos || !out))) return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    if (m == 0) return SPH3_OK;
    if ((int64_t)k >= c->S.n) return SPH3_ERR_INVALID_ARG;
    if (c->P.periodic) return SPH3_ERR_UNSUPPORTED;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    int rc = SPH3_OK;
    if (on_device) {
        launch_kth_dist(qpos, m, c->S, k, out, st);
        return check_launch();
    }
    DevTmp<double> dq, dout;
    CK(dq.alloc(3 * m));
    CK(dout.alloc(m));
    CK(cudaMemcpyAsync(dq.p, qpos, sizeof(double) * 3 * m, cudaMemcpyHostToDevice, st));
    launch_kth_dist(dq.p, m, c->S, k, dout.p, st);
    rc = check_launch();
    if (rc) return rc;
    CK(cudaMemcpyAsync(out, dout.p, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return SPH3_OK;
}

int sph3_set_cooling(sph3_ctx *c, const sph3_cool_table *table, const sph3_cool_units *units) {
    if (!c) return SPH3_ERR_INVALID_ARG;
    if (table) {
        if (!units || !cool_units_valid(table, units)) return SPH3_ERR_INVALID_ARG;
        if (cool_table_device(table) != c->device) return SPH3_ERR_INVALID_ARG;
    }
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    drop_graphs(c);  // the step graphs change
    c->cool = table;
    if (table) c->cool_units = *units;
    const int rc = ensure_ionfrac(c);
    if (rc) c->cool = nullptr;  // no buffer for the ion fractions: cooling stays off
    return rc;
}

int sph3_cool_now(sph3_ctx *c, double dt, void *stream) {
    if (!c) return SPH3_ERR_INVALID_ARG;
    if (!c->have) return SPH3_ERR_STATE;
    if (!c->cool) return SPH3_ERR_STATE;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    launch_cooling_state(c->S, c->cool, &c->cool_units, dt, c->ionfrac, st);
    int rc = check_launch();
    if (rc) return rc;
    CK(cudaStreamSynchronize(st));
    c->ionfrac_valid = true;
    return SPH3_OK;
}

int sph3_get_ionfrac(sph3_ctx *c, float *out, int64_t n_species) {
    if (!c || !out) return SPH3_ERR_INVALID_ARG;
    if (!c->cool || !c->ionfrac_valid) return SPH3_ERR_STATE;
    if (n_species != cool_table_species(c->cool)) return SPH3_ERR_INVALID_ARG;
    if (c->S.n == 0) return SPH3_OK;
    CK(cudaSetDevice(c->device));
    CK(cudaDeviceSynchronize());  // the last step may have run on any stream of the caller's
    CK(cudaMemcpy(out, c->ionfrac, sizeof(float) * c->S.n * n_species, cudaMemcpyDeviceToHost));
    return SPH3_OK;
}

}  // extern "C"


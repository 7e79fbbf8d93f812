/*
 * sph3.h -- C ABI of the B200 (sm_100a) SPH + Barnes-Hut particle step.
 *
 * One shared library (sph_3_b200/lib/libsph3.so).  Plain pointers and sizes,
 * int status returns, no C++ or torch types.  A context (sph3_ctx) owns the
 * device copy of one particle set -- or of a batch of independent particle
 * systems ("clouds") -- in Morton order, its octree and all scratch buffers,
 * so a step allocates nothing.
 *
 * Which reference interface each entry point replaces (paths are within the
 * reference project hassanfv/SPH_3):
 *
 *   sph3_set_particles / sph3_set_field   the NumPy arrays handed to every
 *        libsx function (sph_code/sph_serial.py:37-97 builds them)
 *   sph3_compute(SPH3_DO_BOOT_H)          smoothing_length_mpi / do_smoothingX
 *        (sph_code/libsx.py:752-800)
 *   sph3_compute(SPH3_DO_H)               h_smooth_fast(_mpi) (libsx.py:804-902);
 *        GPU: smoothing_h_ngb + ngbDB_new_v3
 *        (Particles_in_BH_Tree_III/Evrard_Collapse_2024/hfvCLibs_v7_hfv_v8.1.h:485-579,
 *         .../ngb_v5.1.h:125-264)
 *   sph3_compute(SPH3_DO_DENSITY)         getDensity(_mpi) (libsx.py:10-86),
 *        getPressure (libsx.py:91-96) and c = sqrt(gamma (gamma-1) u)
 *        (sph_serial.py:116); with SPH3_DO_DIVCURL also div_curlVel(_mpi)
 *        (sph_code/shear.py:7-142)
 *   sph3_compute(SPH3_DO_ACC_SPH | SPH3_DO_DUDT)  getAcc_sph(_mpi), get_dU(_mpi)
 *        (libsx.py:100-177, 268-347, 353-421, 496-564), their Monaghan-Gingold
 *        forms (libsx.py:183-262, 427-491) and the Balsara forms
 *        getAcc_sph_shear(_mpi), get_dU_shear(_mpi) (shear.py:149-485)
 *   sph3_compute(SPH3_DO_GRAVITY)         getAcc_g_smth* (libsx.py:623-747, 908-947)
 *        as a Barnes-Hut walk; GPU: bh_tree_iteration_v2.h:29-588
 *   sph3_gravity_direct_rows              getAcc_g_smth_mpi (libsx.py:667-705), FP64
 *   sph3_gravity_pairsum                  getAcc_g_smth, getAcc_g_smth_mpi, getAcc_g_smthx,
 *        getAcc_g_smth_mimj_mpi (libsx.py:623-747, 908-947) in the reference's
 *        summation order (bit for bit)
 *   sph3_potential_pairsum                getPE (libsx.py:583-620) as FP64 pair sums
 *   sph3_kth_distance                     do_smoothingX((pos, subpos)) for query points
 *        (libsx.py:752-774)
 *   sph3_first_step                       sph_serial.py:85-134
 *   sph3_step                             one loop body of sph_serial.py:142-196
 *        (or sph_mpi4_v4.py:278-430 with step_order = SPH3_ORDER_MPI4);
 *        GPU: hfvGpuSphBHtree_newCool_v8_KH.cu:985-1582
 *   sph3_step_io                          the same loop body with its arrays in host
 *        memory (sph_serial.py:142-193 keeps r, v, acc, h, u, ut_previous as NumPy arrays)
 *   sph3_energy                           getKE / getPE (libsx.py:569-620)
 *   sph3_cool_table_create                the cooling table read from coolHeatGridJan2024.bin
 *        (Main_Code/hfvGpuSphBHtree_newCool_v8.cu:40-80, 122-199)
 *   sph3_hcooling / sph3_set_cooling      hcoolingZ after u_updater
 *        (Evrard_Collapse_2024/hfvCLibs_v7_hfv_v8.1.h:1433-1623; launched at
 *         Main_Code/hfvGpuSphBHtree_newCool_v8.cu:1552)
 *
 * Buffers: every pointer argument names memory of the kind its `on_device`
 * flag says (0: host memory, pageable or pinned; 1: device memory of the
 * context's GPU).  Host pointers are copied with cudaMemcpyAsync on `stream`
 * and the call synchronises that stream before it returns; device pointers
 * are used in stream order without synchronisation.  `stream` is a
 * cudaStream_t (NULL: the context's own stream).
 *
 * Threads: a context is not thread-safe; use one context per host thread or
 * lock around it.  Errors: every call returns SPH3_OK (0) or an SPH3_ERR_*
 * code; sph3_error_string() names it.  Device-side conditions (an h search
 * that did not converge, non-finite input, ...) set bits in a status word that
 * sph3_status() returns; kernels never trap and every loop in them is bounded.
 */
#ifndef SPH3_H
#define SPH3_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------- return codes */
#define SPH3_OK 0
#define SPH3_ERR_INVALID_ARG 1
#define SPH3_ERR_CUDA 2
#define SPH3_ERR_NO_DEVICE 3
#define SPH3_ERR_STATE 4
#define SPH3_ERR_UNSUPPORTED 5
#define SPH3_ERR_OUT_OF_MEMORY 6
#define SPH3_ERR_DEVICE_STATUS 7 /* a device status bit is set, see sph3_status */
#define SPH3_ERR_TOO_LARGE 8     /* size above the fixed maximum of sph3_morton_sort_noalloc */

/* ----------------------------------------------- device status word bits */
#define SPH3_STATUS_H_NOT_CONVERGED 0x1u  /* h search hit its iteration cap */
#define SPH3_STATUS_STACK_OVERFLOW 0x2u   /* walk stack full (cannot happen with stack_cap >= 7*(max_level+2)+32) */
#define SPH3_STATUS_NAN_INPUT 0x4u        /* non-finite position, velocity, mass or h */
#define SPH3_STATUS_TREE_CAPACITY 0x8u    /* node array too small */
#define SPH3_STATUS_ZERO_DENSITY 0x10u    /* rho <= 0 where a division by rho follows */
#define SPH3_STATUS_LIST_OVERFLOW 0x20u   /* neighbour export capacity exceeded */
#define SPH3_STATUS_SORT 0x40u            /* radix-sort bookkeeping mismatch */
#define SPH3_STATUS_BOX_TOO_SMALL 0x80u   /* 2h above half a periodic box length: no unique minimum image */
#define SPH3_STATUS_COOL_NEGATIVE_U 0x100u /* the cooling table gave a negative u (the reference prints it) */

/* ----------------------------------------------------------------- enums */
#define SPH3_PREC_MIXED 0 /* FP32 cell-relative pair arithmetic, FP64 state/accumulators/sums */
#define SPH3_PREC_FP64 1  /* FP64 everywhere */

#define SPH3_H_NEWTON 0  /* Newton iteration on ln N(h) to the window, bounded */
#define SPH3_H_REFSTEP 1 /* the reference rule: h -/+= 0.003 h until N in the window */

#define SPH3_VISC_SIGNAL 0  /* getAcc_sph / get_dU (libsx.py:151-160) */
#define SPH3_VISC_MG83 1    /* getAcc_sph_mpiXXX / get_dU_mpiXXXX (libsx.py:236-246) */
#define SPH3_VISC_BALSARA 2 /* getAcc_sph_shear / get_dU_shear (shear.py:193-215) */

#define SPH3_MAC_BH 0        /* Barnes-Hut: accept a node when d(com, group box) > s / theta */
#define SPH3_MAC_BH_OFFSET 1 /* ... when d > s / theta + the offset of the com from the node's box centre */

#define SPH3_ORDER_SERIAL 0 /* du/dt with the half-step v, before the 2nd kick (sph_serial.py) */
#define SPH3_ORDER_MPI4 1   /* du/dt with the full-step v, after the 2nd kick (sph_mpi4_v4.py) */

/* compute flags for sph3_compute */
#define SPH3_DO_TREE 0x1u      /* Morton sort + octree (implied by every walk) */
#define SPH3_DO_BOOT_H 0x2u    /* h = 0.5 * distance to the n_boot-th nearest particle */
#define SPH3_DO_H 0x4u         /* h search to n_ngb +- n_ngb_tol */
#define SPH3_DO_DENSITY 0x8u   /* rho, P, c (EOS from u) */
#define SPH3_DO_DIVCURL 0x10u  /* div v, |curl v|, Balsara factor (needs rho: fused with DENSITY) */
#define SPH3_DO_ACC_SPH 0x20u  /* hydro acceleration from the stored rho, P, c */
#define SPH3_DO_DUDT 0x40u     /* du/dt from the stored rho, P, c */
#define SPH3_DO_GRAVITY 0x80u  /* Barnes-Hut acceleration and potential (theta = 0: exact) */
#define SPH3_DO_EOS 0x100u     /* P, c from the stored rho and u only */

/* field ids for sph3_set_field / sph3_get_field (components per particle) */
#define SPH3_FIELD_POS 0       /* 3 */
#define SPH3_FIELD_VEL 1       /* 3 */
#define SPH3_FIELD_MASS 2      /* 1 */
#define SPH3_FIELD_U 3         /* 1 */
#define SPH3_FIELD_H 4         /* 1 */
#define SPH3_FIELD_EPS 5       /* 1 */
#define SPH3_FIELD_RHO 6       /* 1 */
#define SPH3_FIELD_P 7         /* 1 */
#define SPH3_FIELD_C 8         /* 1 */
#define SPH3_FIELD_DIVV 9      /* 1 */
#define SPH3_FIELD_CURLV 10    /* 1 */
#define SPH3_FIELD_ACC 11      /* 3, total acceleration of the last step */
#define SPH3_FIELD_ACC_G 12    /* 3 */
#define SPH3_FIELD_ACC_SPH 13  /* 3 */
#define SPH3_FIELD_DUDT 14     /* 1 */
#define SPH3_FIELD_DUDT_PREV 15 /* 1 */
#define SPH3_FIELD_PHI 16      /* 1, gravitational potential (G included) */
#define SPH3_FIELD_NNGB 17     /* 1, neighbour count N(r < 2h) of the last h search */
#define SPH3_FIELD_BALSARA 18  /* 1 */
#define SPH3_FIELD_U_PREV 19   /* 1 */
#define SPH3_FIELD_VSIG 20     /* 1, max signal velocity c_i + c_j - 3 w_ij over the last hydro pass's pairs */
#define SPH3_FIELD_DT 21       /* 1, per-particle time step of the last sph3_timestep */
#define SPH3_FIELD_DHDT 22     /* 1, h divV / 3 of the last sph3_timestep */
#define SPH3_NUM_FIELDS 23

/* ---------------------------------------------------------------- config */
typedef struct sph3_config {
    int32_t precision;   /* SPH3_PREC_* */
    int32_t h_mode;      /* SPH3_H_* */
    int32_t visc;        /* SPH3_VISC_* */
    int32_t step_order;  /* SPH3_ORDER_* */
    int32_t n_ngb;       /* target neighbour count N(r < 2h) (reference CPU: 50, GPU: 64) */
    int32_t n_ngb_tol;   /* accepted window n_ngb +- tol (reference: 5) */
    int32_t h_max_iter;  /* cap on h iterations (SPH3_STATUS_H_NOT_CONVERGED past it) */
    int32_t n_boot;      /* k of the bootstrap h (reference: 50, 0-based sorted index) */
    int32_t leaf_size;   /* octree leaf capacity (1..64) */
    int32_t stack_cap;   /* walk-stack entries per warp (default 768; >= 7 (max_level + 2) + 32, <= 4096).
                          * Wide pops need room: once the stack nears its capacity the walk pops one
                          * node per iteration, which is exact but slow. */
    int32_t max_level;   /* octree levels (3 key bits each), 4..21 */
    int32_t gravity;     /* 0: hydro only */
    int32_t quadrupole;  /* 1: monopole + quadrupole nodes, 0: monopole only */
    int32_t use_graph;   /* 1: sph3_step replays a captured CUDA graph */
    int32_t timing;      /* 1: record per-phase CUDA events (no graph) */
    int32_t walk_warps;  /* warps per walk block: 1, 2, 4 (default) or 8; each warp walks one group of <= 32 particles */
    int32_t list_cap;    /* neighbour-list slots per particle that the density walk keeps for the hydro
                          * pass (default 128; 0 = the hydro pass walks the tree).  The lists hold exactly
                          * the pairs inside the support (|r| <= h_i + h_j, tested in the precision of the
                          * path); a particle with more neighbours than list_cap is handled by a walk.  In
                          * FP64 the list pass runs the walk's arithmetic in the walk's pair order, so its
                          * results equal the walk's.  4 * list_cap bytes per particle; a multiple of 8 in
                          * 0..1024. */
    int32_t mac;         /* multipole acceptance: SPH3_MAC_BH (d > s/theta, the default) or
                          * SPH3_MAC_BH_OFFSET (d > s/theta + |com - box centre|, more conservative) */
    int32_t eps_from_h;  /* 1: gravitational softening eps = h after every h search, as the reference GPU
                          * driver's set_eps_of_gas_to_h (Evrard_Collapse_2024/hfvCLibs_v7_hfv_v8.1.h:584-593);
                          * 0 (default): eps stays as set (the benchmark fixes eps = 0.01) */
    int32_t step_potential; /* 1: every step's gravity walk also computes the potential; 0 (default): the
                          * steps compute accelerations only (the reference's loop computes no energies)
                          * and sph3_energy runs the walk with the potential when it needs a fresh one */
    double gamma;        /* adiabatic index (5/3) */
    double alpha;        /* artificial viscosity alpha (1) */
    double beta;         /* beta of the MG83 form (2) */
    double eta;          /* eta of the MG83 form (0.1) */
    double G;            /* gravitational constant (1) */
    double theta;        /* opening angle; 0 = exact direct sum through the tree */
    double eps;          /* softening length used when no eps field is set (0.01) */
    double box[3];       /* periodic box lengths, 0 = open boundary in that axis */
    double reserved_d[4];
} sph3_config;

typedef struct sph3_ctx sph3_ctx;

/* Library version (major * 10000 + minor * 100 + patch). */
int sph3_version(void);

/* Fills cfg with the defaults listed in the struct comments. */
void sph3_default_config(sph3_config *cfg);

/* Names an SPH3_ERR_* code; a static string. */
const char *sph3_error_string(int code);

/* Creates a context on CUDA device `device` (-1: the current device). */
int sph3_ctx_create(const sph3_config *cfg, int device, sph3_ctx **out);
int sph3_ctx_destroy(sph3_ctx *ctx);

/* Replaces the physics / numerics parameters (sizes of existing buffers stay). */
int sph3_set_config(sph3_ctx *ctx, const sph3_config *cfg);
int sph3_get_config(const sph3_ctx *ctx, sph3_config *cfg);

/* Splits the next particle set into `ncloud` independent systems of
 * counts[0..ncloud) consecutive particles (a batched ensemble).  Default: one
 * system.  Call before sph3_set_particles. */
int sph3_set_clouds(sph3_ctx *ctx, const int64_t *counts, int32_t ncloud);

/* Loads n particles (arrays in the caller's order, pos/vel as (n,3) row-major
 * FP64).  pos and mass are required; vel, u, h, eps may be NULL (0, 0, 0 and
 * cfg.eps).  Sorts them into Morton order and builds the octree. */
int sph3_set_particles(sph3_ctx *ctx, int64_t n, const double *pos, const double *vel,
                       const double *mass, const double *u, const double *h,
                       const double *eps, int on_device, void *stream);

/* Number of particles currently loaded. */
int64_t sph3_num_particles(const sph3_ctx *ctx);

/* Overwrites one field from an array in the caller's particle order.
 * Writing SPH3_FIELD_POS re-sorts and rebuilds the tree. */
int sph3_set_field(sph3_ctx *ctx, int field, const double *src, int on_device, void *stream);

/* Copies rows [row_begin, row_end) of a field, in the caller's particle order,
 * to dst ((row_end-row_begin) x components, FP64). */
int sph3_get_field(sph3_ctx *ctx, int field, double *dst, int64_t row_begin, int64_t row_end,
                   int on_device, void *stream);

/* Runs the passes named by `what` (SPH3_DO_* bits) on the loaded state. */
int sph3_compute(sph3_ctx *ctx, uint32_t what, void *stream);

/* As sph3_compute, but the walks run only for the particles of caller rows
 * [row_begin, row_end) (the walk groups that hold them): the *_mpi forms of
 * sph_code/libsx.py (getDensity_mpi :50-86, h_smooth_fast_mpi :852-902,
 * getAcc_sph_mpi / get_dU_mpi, getAcc_g_smth_mpi), where each rank of
 * sph_mpi4_v4.py asks for its own slice.  The rows' results equal those of
 * sph3_compute bit for bit (a group's results depend only on the group);
 * other rows' pair results are left undefined, and the neighbour lists and
 * the potential are marked stale. */
int sph3_compute_rows(sph3_ctx *ctx, uint32_t what, int64_t row_begin, int64_t row_end, void *stream);

/* The reference's start-up: h (bootstrap if h is all zero, then the h search),
 * rho, gravity, P, c, hydro acceleration, du/dt, then u += du/dt * dt,
 * u_prev = u, dudt_prev = du/dt (sph_serial.py:85-134). */
int sph3_first_step(sph3_ctx *ctx, double dt, void *stream);

/* nsteps leapfrog kick-drift-kick steps of length dt. */
int sph3_step(sph3_ctx *ctx, double dt, int32_t nsteps, void *stream);

/* nsteps steps of length dt with the state moved in from and out to HOST
 * buffers in the same call: the loop body of sph_code/sph_serial.py:142-193
 * as the reference runs it, its arrays (r, v, acc, h, u, ut_previous) living
 * in host memory.  in[k] holds field in_fields[k] ((n x components)
 * row-major FP64, caller's order) and is written into the state before the
 * steps; out[k] receives field out_fields[k] after them (SPH3_FIELD_NNGB
 * too, as doubles).  Transfers overlap the step: each input is copied on a
 * copy stream and scattered just before the step first needs it (h after
 * the sort, u before the EOS, u_prev and dudt_prev before the kick that
 * updates u; all others before the first kick), and each output leaves on a
 * second copy stream as soon as it is final (positions after the sort, h
 * after the h search, u, u_prev, dudt_prev, dudt, rho, P, c, acc_sph and
 * vsig after the u update -- which the serial order runs before the gravity
 * walk -- the rest at the end).  An input u without u_prev also
 * sets u_prev (the reference's loop keeps u_previous = u between
 * iterations).  The positions, velocities and accelerations (what the
 * opening kick reads) move in row chunks, each scattered as soon as it lands;
 * in the serial order the closing kick runs by row chunks too, each chunk's
 * outputs copied out while the next is kicked.  Page-locked host buffers are
 * needed for the overlap (pageable ones work, serialised).  With page-locked
 * buffers (and use_graph, timing off, after two warm-up steps) the whole call
 * -- copies, scatters, steps, gathers -- is captured as a CUDA graph and
 * replayed by later calls with the same buffers, fields, dt and nsteps (a
 * different call captures again).  The call synchronises before it returns. */
int sph3_step_io(sph3_ctx *ctx, double dt, int32_t nsteps, int32_t nin, const int32_t *in_fields,
                 const double *const *in, int32_t nout, const int32_t *out_fields, double *const *out,
                 void *stream);

/* Global sums in FP64 of the current state: out[0] KE, out[1] thermal energy
 * sum m u, out[2] PE = 1/2 sum m phi, out[3] total, out[4..6] momentum,
 * out[7] mass.  When the potential is older than the positions (steps run
 * with step_potential = 0), it first runs the gravity walk with the potential.
 * Synchronises `stream`. */
int sph3_energy(sph3_ctx *ctx, double out[8], void *stream);

/* Device status word (SPH3_STATUS_* bits) accumulated since the last clear.
 * Synchronises the context's streams. */
int sph3_status(sph3_ctx *ctx, uint32_t *status, int clear);

/* FP64 spline-softened direct sum for the listed rows (caller's order) against
 * every particle of the same system: acc (nrows x 3) and, if phi != NULL,
 * the potential.  Host output buffers. */
int sph3_gravity_direct_rows(sph3_ctx *ctx, const int64_t *rows, int64_t nrows, double *acc,
                             double *phi);

/* The pairs the mixed path's hydro pass runs for the listed rows: the
 * neighbour lists the last density pass kept (|r_ij| <= h_i + h_j tested in
 * FP32 on cell-relative positions), as caller's indices in ascending order,
 * laid out as in sph3_neighbours.  A row with more pairs than list_cap gives
 * its first list_cap (its hydro terms come from a walk).  SPH3_ERR_STATE when
 * no valid lists exist (FP64 precision, list_cap = 0, or no density pass since
 * positions or h changed).  No reference counterpart: it states how the
 * mixed-precision pair sets differ from the exact ones. */
int sph3_pair_lists(sph3_ctx *ctx, const int64_t *rows, int64_t nrows, int64_t *offsets, int64_t *idx,
                    int64_t cap);

/* Neighbour sets {j : |r_ij| <= h_i + h_j} (the q <= 2 support of the
 * reference kernels, sph_code/libsx.py:34-38) of the listed rows, as caller's
 * indices in ascending order: row k's set is idx[offsets[k] .. offsets[k+1]).
 * offsets has nrows+1 entries; at most cap indices are written
 * (SPH3_STATUS_LIST_OVERFLOW past it).  Host buffers. */
int sph3_neighbours(sph3_ctx *ctx, const int64_t *rows, int64_t nrows, int64_t *offsets,
                    int64_t *idx, int64_t cap);

/* Spline-softened gravity of the loaded particles (one system, open
 * boundaries) as the reference's FP64 direct sums, in the reference's
 * summation order, so the results equal the reference's bit for bit on the
 * same inputs (a coincident pair adds 0, where the reference raises
 * ZeroDivisionError).  G comes from the config, eps from the eps field.
 *   form SPH3_GSUM_ROWS: rows [nbeg, nend) of a_i = sum_{j != i} ... in the
 *     caller's order, out (nend - nbeg) x 3 -- getAcc_g_smth
 *     (sph_code/libsx.py:623-662), getAcc_g_smth_mpi (:667-705) and
 *     getAcc_g_smthx (:710-747), which agree bit for bit;
 *   form SPH3_GSUM_MIMJ: the n x 3 partial array of
 *     getAcc_g_smth_mimj_mpi(nbeg, nend, ...) (:908-947): the j > i terms of
 *     rows i in [nbeg, nend) and their reactions on rows j > i; summed over a
 *     row partition it is the full field.
 * out is host (on_device = 0; the call synchronises) or device memory.
 * O(n * rows) work: a checker and drop-in, not the step's gravity. */
#define SPH3_GSUM_ROWS 0
#define SPH3_GSUM_MIMJ 1
int sph3_gravity_pairsum(sph3_ctx *ctx, int form, int64_t nbeg, int64_t nend, double *out, int on_device,
                         void *stream);

/* Softened potential energy of getPE (sph_code/libsx.py:583-620): the
 * reference's j > i terms in its order per row i, the row sums added in row
 * order (the reference chains all pairs into one sum, so the result can
 * differ from it in the last bits).  One system, open boundaries. */
int sph3_potential_pairsum(sph3_ctx *ctx, double *pe, void *stream);

/* do_smoothingX((pos, subpos)) (sph_code/libsx.py:752-774) for query points:
 * out[i] = 0.5 * (the value at 0-based index k of the sorted distances from
 * query i to every loaded particle), the reference's h with k = 50.  The
 * k-th squared distance is found exactly (radix select on its bits).  qpos
 * (m x 3 row-major FP64) and out are host (on_device = 0) or device memory.
 * SPH3_ERR_INVALID_ARG when k >= the particle count (the reference raises
 * IndexError); open boundaries only. */
int sph3_kth_distance(sph3_ctx *ctx, const double *qpos, int64_t m, int32_t k, double *out, int on_device,
                      void *stream);

/* Current Morton order: order[k] = caller's index of the k-th sorted particle,
 * keys[k] its 64-bit key (either pointer may be NULL).  Host buffers. */
int sph3_morton_order(sph3_ctx *ctx, int64_t *order, uint64_t *keys);

/* Work counters accumulated since the last clear: [0] gravity node
 * interactions, [1] gravity particle interactions, [2] SPH candidate pairs of
 * the density pass, [3] of the hydro pass, [4] h-search candidate pairs,
 * [5] h passes, [6] tree nodes (of the last build), [7] tree leaves,
 * [8..11] tree nodes visited by the h-search / density / hydro / gravity
 * walks, [12] the longest single walk (loop iterations), [13] where it
 * happened (iterations << 40 | walk kind << 32 | first particle), [14]
 * particle groups walked by the gravity pass, [15] reserved.
 * Clears them if `clear`. */
int sph3_counters(sph3_ctx *ctx, int64_t out[16], int clear);

/* Per-phase device times in ms accumulated while cfg.timing = 1:
 * [0] kick+drift+keys, [1] sort, [2] gather, [3] tree, [4] h search,
 * [5] density, [6] gravity, [7] hydro, [8] kick+u.  Clears if `clear`. */
int sph3_phase_times(sph3_ctx *ctx, double out[9], int clear);

/* Per-particle time step, the reference's dt_array_indiv_dt
 * (Particles_in_BH_Tree_III/Evrard_Collapse_2024/hfvCLibs_v7_hfv_v8.1.h:1189-1262;
 * present but switched off in its driver, hfvGpuSphBHtree_newCool_v8_KH.cu:1540):
 *   dt_i = min(C h/max_j vsig_ij, C h/(h|divV| + max(c,|v|)(1 + 0.6 alpha)),
 *              sqrt(h/|a_g|), sqrt(h/|a|), 0.4 sqrt(eps/|a|), 0.4 eps/|v|),
 * vsig_ij = c_i + c_j - 3 (v_ij . r_ij)/(|r_ij| + 1e-5), in FP64, into the
 * SPH3_FIELD_DT field (and h divV / 3 into SPH3_FIELD_DHDT); *dt_min gets the
 * minimum over all particles.  all_pairs = 1 takes max_j over every particle
 * of the system, as the reference does (O(N^2)); 0 takes it over the pairs of
 * the last hydro pass (|r_ij| <= h_i + h_j), which that pass recorded in
 * SPH3_FIELD_VSIG.  Uses the accelerations of the last step or compute call;
 * div v is recomputed at the current positions and velocities. */
int sph3_timestep(sph3_ctx *ctx, double c_cfl, int all_pairs, double *dt_min, void *stream);

/* Kernel launches one sph3_step makes once its CUDA graph is captured (the
 * kernel nodes of the graph; memsets are not counted), or -1 before the
 * first graph capture.  No reference counterpart: it backs the launch count
 * that benchmarks report. */
int sph3_kernels_per_step(sph3_ctx *ctx, int64_t *out);

/* Measured FP32 rate of GPU `device` in TFLOP/s: a grid of 8 blocks of 256
 * threads per SM running independent FMA chains, packed (FFMA2) and scalar,
 * each timed with CUDA events (about 20 ms in all); the larger rate.  No reference counterpart: it is the
 * denominator benchmarks use for the walk kernels, which are bound by the FP32
 * pipe rather than by HBM or the tensor cores. */
int sph3_probe_fp32_rate(int device, double *tflops, void *stream);

/* Morton sort that allocates no device memory -- it has no counterpart in the
 * reference.  For callers that cannot call cudaMalloc: code running inside a
 * caller-owned pool or arena, or under a host framework that owns the
 * device allocator, or a loop that cannot afford cudaMalloc's latency and
 * implicit synchronisation.  They pass device buffers only: pos ((n,3)
 * row-major FP64, read), order (n int64: caller index of the k-th sorted
 * particle) and keys (n uint64 Morton keys); either output may be NULL, not
 * both.  status (one device word, may be NULL) receives the SPH3_STATUS_*
 * bits this call raised (SPH3_STATUS_NAN_INPUT: a non-finite coordinate,
 * which is quantised to cell 0), written in stream order at the end of the
 * call.  The result equals sph3_set_particles + sph3_morton_order for one
 * system with the same max_level (4..21).
 * Limit: n <= 65536 (SPH3_ERR_TOO_LARGE above it).  The scratch is a fixed
 * static device array (about 3 MB) that every GPU loading the library holds
 * until the process exits; the first call on a device (and the first after a
 * cudaDeviceReset) looks up its address, so make that first call before any
 * stream capture.  All calls share the array: calls that overlap on the GPU
 * race.  Stream-ordered on `stream`; does not synchronise.  Returns
 * SPH3_ERR_CUDA without doing anything when a CUDA error is already pending
 * on entry (the caller's own; it is left unread). */
int sph3_morton_sort_noalloc(const double *pos, int64_t n, int32_t max_level, int64_t *order,
                             uint64_t *keys, unsigned *status, void *stream);


/* ------------------------------------------------------ heating / cooling */
/* A heating/cooling table in the layout of the reference's
 * coolHeatGridJan2024.bin (Particles_in_BH_Tree_III/Main_Code/
 * hfvGpuSphBHtree_newCool_v8.cu:40-80 reads it; :122-199 uploads it).  dims
 * in the file header's order: N_kpc, N_T, N_nH, N_Z, N_M, N_t.  Host float
 * arrays: kpc[N_kpc], nh[N_nH], t[N_t] (elapsed seconds), uevol (u after t,
 * cgs) [N_kpc][N_T][N_nH][N_Z][N_t], metalz (species fractions)
 * [N_kpc][N_T][N_nH][N_Z][N_M][N_t], uarr (u at t = 0) [N_kpc][N_T][N_nH][N_Z].
 * The file's Z, T and mu arrays are not used by the step.  Copied to device
 * `device`; the caller's arrays may be freed after the call. */
typedef struct sph3_cool_table sph3_cool_table;
int sph3_cool_table_create(int device, const int32_t dims[6], const float *kpc, const float *nh, const float *t,
                           const float *uevol, const float *metalz, const float *uarr, sph3_cool_table **out);
int sph3_cool_table_destroy(sph3_cool_table *table);
/* dims as given to create; monotone (may be NULL): whether the kpc, nH and t
 * grids and every T column of uarr are non-decreasing (searched by bisection;
 * otherwise by the reference's linear scan -- the same index either way). */
int sph3_cool_table_dims(const sph3_cool_table *table, int32_t dims[6], int32_t monotone[4]);

/* Unit conversions of the reference's params.txt (readParams,
 * Evrard_Collapse_2024/hfvCLibs_v7_hfv_v8.1.h:24-53), in float as there. */
typedef struct sph3_cool_units {
    float unit_density_cgs; /* UnitDensity_in_cgs */
    float unit_time_s;      /* unitTime_in_s */
    float unit_u_cgs;       /* Unit_u_in_cgs */
    float unit_length_cm;   /* unitLength_in_cm */
    float kpc_cm;           /* kpc_in_cm (the reference: 3.086e21) */
    int32_t z_index;        /* metallicity row of the table (the reference fixes 1: [Z/H] = -1) */
} sph3_cool_units;

/* hcoolingZ (Particles_in_BH_Tree_III/Evrard_Collapse_2024/
 * hfvCLibs_v7_hfv_v8.1.h:1433-1623) on the reference's float device arrays:
 * for every particle with typ[i] == 0 (typ NULL: all), u[i] (code units) is
 * replaced by the table's evolved u after dt at the nearest kpc, nH and t grid
 * points, interpolated linearly in u along T, and ionfrac[i * N_M + k] (may be
 * NULL) receives the species fractions.  FP32 as the reference, with the
 * reference kernel's results bit for bit.  status (one device word, may be NULL): SPH3_STATUS_COOL_NEGATIVE_U
 * when a particle's new u is negative.  Device pointers on the table's GPU;
 * stream-ordered, does not synchronise. */
int sph3_hcooling(const sph3_cool_table *table, const sph3_cool_units *units, float dt, int64_t n,
                  const int32_t *typ, float *u, const float *rho, const float *x, const float *y, const float *z,
                  float *ionfrac, uint32_t *status, void *stream);

/* Makes every sph3_step / sph3_step_io of the context apply the table to u
 * right after the u update, as the production driver calls hcoolingZ after
 * u_updater (Main_Code/hfvGpuSphBHtree_newCool_v8.cu:1546-1556); every
 * particle is gas.  sph3_first_step does not cool, as the driver's first
 * step before its loop does not (:1033).  The state is rounded to float for the lookups and u is
 * written back from the float result.  The table must live on the context's
 * GPU and outlive the setting; table NULL turns cooling off.  The context
 * keeps the ion fractions of the last step (sph3_get_ionfrac). */
int sph3_set_cooling(sph3_ctx *ctx, const sph3_cool_table *table, const sph3_cool_units *units);

/* Applies the context's cooling table once to the current state (dt in code
 * units), outside a step. */
int sph3_cool_now(sph3_ctx *ctx, double dt, void *stream);

/* Ion fractions of the last cooled step, (n, N_M) float in the caller's
 * particle order, into a host buffer (synchronises the device first).
 * SPH3_ERR_STATE when none exist; SPH3_ERR_INVALID_ARG when n_species is not
 * the table's N_M. */
int sph3_get_ionfrac(sph3_ctx *ctx, float *out, int64_t n_species);

#ifdef __cplusplus
}
#endif

#endif /* SPH3_H */

/*
 * fmm_b200.h -- C ABI of the B200 (sm_100a) fast multipole library.
 *
 * The library replaces the evaluation hot path of FastMultipole.jl
 * (byuflowlab/FastMultipole, v1.0.0): octree construction, dual-tree
 * interaction lists, P2M / M2M / M2L / L2L / L2P and the P2P near field for
 * Laplace point sources and vortex particles.  A host binding (Julia ccall,
 * Python ctypes, ...) gathers bodies through the reference's per-system
 * interface (source_system_to_buffer!, get_position) into the plain buffers
 * below, calls one entry point, and scatters the result through
 * buffer_to_target_system!.
 *
 * Conventions
 *  - All functions return an fmm_status; 0 is success.  Nothing aborts or
 *    exits; the message of the last failure is fmm_ctx_last_error().
 *  - Indices are 0-based.  Buffers are body-major ("column-major d x N" in the
 *    reference's Julia layout): body i occupies buffer[i*stride ... ].
 *  - Source buffer rows (src/compatibility.jl:10-16): x y z radius strength...
 *    (strength is 1 value for a point source, 3 for a vortex particle).
 *  - Target buffer rows (src/compatibility.jl:159-161): x y z phi grad(3)
 *    hessian(9, column-major SMatrix order).  The library writes all 16 rows
 *    in the caller's body order (rows 1..3 = the target positions).
 *  - Calls on one context are serialised; use one context per host thread.
 */
#ifndef FMM_B200_H
#define FMM_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FMM_API __attribute__((visibility("default")))
#else
#define FMM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  FMM_OK = 0,
  FMM_ERR_ARGUMENT = 1,    /* invalid argument (sizes, kinds, options)             */
  FMM_ERR_CUDA = 2,        /* a CUDA runtime call failed                            */
  FMM_ERR_NO_DEVICE = 3,   /* no usable sm_100 device                               */
  FMM_ERR_TREE_DEPTH = 4,  /* bodies too clustered for the 21-level octant key     */
  FMM_ERR_MEMORY = 5,      /* the request exceeds the context's HBM budget          */
  FMM_ERR_STATE = 6,       /* export requested before any solve / server not running */
  FMM_PENDING = 7          /* fmm_serve_poll: the request has not finished yet       */
} fmm_status;

/* body_to_multipole!(system, ...) = body_to_multipole!(Point{Source|Vortex}, ...)
 * (src/bodytomultipole.jl:403-489); the value is the strength dimension. */
typedef enum { FMM_POINT_SOURCE = 1, FMM_POINT_VORTEX = 3 } fmm_kind;

/* InteractionListMethod (src/containers.jl:108-123) */
typedef enum {
  FMM_LIST_SELF_TUNING_TREE_STOP = 0, /* default of fmm! (src/fmm.jl:868) */
  FMM_LIST_BARBA = 1,
  FMM_LIST_SELF_TUNING = 2
} fmm_list_method;

/* error_tolerance (src/containers.jl:84-104); NONE is the plain fixed-order method */
typedef enum {
  FMM_ERROR_NONE = 0,
  FMM_POWER_ABSOLUTE_GRADIENT = 1,
  FMM_POWER_RELATIVE_GRADIENT = 2,
  FMM_ROTATED_COEFFICIENTS_ABSOLUTE_GRADIENT = 3,
  FMM_ROTATED_COEFFICIENTS_RELATIVE_GRADIENT = 4,
  FMM_POWER_ABSOLUTE_POTENTIAL = 5, /* src/translate.jl:831-972 */
  FMM_POWER_RELATIVE_POTENTIAL = 6  /* src/translate.jl:974-1122; influence = scalar potential */
} fmm_error_method;

/* Arithmetic of the evaluation passes. F64 is the drop-in (reference
 * arithmetic); MIXED runs P2P and the translation passes in FP32 with FP64
 * tree geometry and FP64 rotation coefficients. */
typedef enum { FMM_PRECISION_F64 = 0, FMM_PRECISION_MIXED = 1 } fmm_precision;

typedef enum { FMM_MEMORY_HOST = 0, FMM_MEMORY_DEVICE = 1 } fmm_memory;

typedef struct {
  int kind;             /* fmm_kind                                             */
  int64_t n_bodies;     /* get_n_bodies(system)                                 */
  int data_per_body;    /* data_per_body(system) >= 4 + kind                    */
  const double* buffer; /* data_per_body * n_bodies, body-major                 */
  int memory;           /* fmm_memory of `buffer`                               */
} fmm_source_system;

typedef struct {
  int64_t n_bodies;
  const double* positions; /* positions[i*stride + 0..2] = get_position(system, i);
                              NULL in fmm_solve: the targets are the source bodies
                              (fmm!(system), src/fmm.jl:807)                         */
  int64_t stride;          /* >= 3 (use data_per_body to read a source buffer)     */
  double* out;             /* 16 * n_bodies, body-major: rows 1..3 receive the
                              positions, rows 4..16 phi, gradient, hessian          */
  int memory;              /* fmm_memory of `positions` and `out`                  */
} fmm_target_system;

/* Keyword arguments of fmm! (src/fmm.jl:862-923). */
typedef struct {
  int expansion_order;         /* 5                                              */
  int leaf_size_source;        /* 20                                             */
  int leaf_size_target;        /* <= 0: leaf_size_source (src/fmm.jl:874)       */
  double multipole_acceptance; /* 0.4                                            */
  int error_method;            /* fmm_error_method, default NONE                 */
  double error_tolerance;      /* epsilon of the error method                    */
  int bonus_expansion;         /* BE parameter of the error methods, default 1   */
  int shrink_recenter;         /* 1                                              */
  int list_method;             /* fmm_list_method                                */
  int farfield, nearfield, self_induced;             /* 1, 1, 1                   */
  int upward_pass, horizontal_pass, downward_pass;   /* 1, 1, 1                   */
  int scalar_potential, gradient, hessian;           /* 0, 1, 0                   */
  int precision;               /* fmm_precision, default F64                     */
} fmm_options;

typedef struct {
  int p_max;           /* largest expansion order used by M2L (+1 on failure) */
  int error_success;   /* every error-controlled M2L met its tolerance       */
  int64_t n_target_branches, n_source_branches, n_target_leaves, n_source_leaves;
  int64_t n_m2l, n_direct;
  int64_t n_p2p_pairs; /* sum over the direct list of n_target * n_source     */
  int64_t m2l_flops;   /* algorithmic M2L flops at the orders actually used  */
  /* stage times on the device stream [ms]; zero unless timing was requested */
  double t_total_ms, t_tree_ms, t_lists_ms, t_nearfield_ms, t_upward_ms, t_horizontal_ms, t_downward_ms;
  int64_t n_kernel_launches; /* kernels of this library launched by the solve (CUB sort/scan
                                passes not included)                                       */
  double t_influence_ms;       /* influence estimate of the relative error methods [ms]    */
} fmm_result;

typedef struct fmm_ctx fmm_ctx;

/* ---- context ------------------------------------------------------------- */
FMM_API int fmm_ctx_create(fmm_ctx** ctx, int device);
FMM_API int fmm_ctx_destroy(fmm_ctx* ctx);
/* Launch everything on this cudaStream_t (NULL = the legacy default stream). */
FMM_API int fmm_ctx_set_stream(fmm_ctx* ctx, void* cuda_stream);
/* Record per-stage CUDA events into fmm_result (adds small overhead). */
FMM_API int fmm_ctx_set_timing(fmm_ctx* ctx, int enabled);
/* Upper bound on the context's device allocations (0 = unlimited). */
FMM_API int fmm_ctx_set_hbm_budget(fmm_ctx* ctx, size_t bytes);
FMM_API size_t fmm_ctx_device_bytes(const fmm_ctx* ctx);
FMM_API const char* fmm_ctx_last_error(const fmm_ctx* ctx);
FMM_API void fmm_default_options(fmm_options* opt);

/* ---- fmm! ------------------------------------------------------------------
 * fmm!(target_systems, source_systems; kwargs...) with automatic trees
 * (src/fmm.jl:807-884 -> :886-912 -> :914-1176).  target->positions == NULL
 * means fmm!(system): the source bodies are also the targets and target->out
 * holds 16 * source->n_bodies doubles.  Results are accumulated into a zeroed
 * 16-row buffer exactly as the reference's target buffer is, then written in
 * the caller's body order.  Rows of quantities that were not requested are
 * zero, except the point-source gradient, which the reference's near-field
 * kernel always evaluates. */
FMM_API int fmm_solve(fmm_ctx* ctx, const fmm_target_system* target, const fmm_source_system* source,
              const fmm_options* opt, fmm_result* result);

/* ---- direct! ---------------------------------------------------------------
 * direct!(targets, sources) all pairs with the same P2P kernels
 * (src/direct.jl:43-75); target->positions == NULL: the sources are the targets. */
FMM_API int fmm_direct(fmm_ctx* ctx, const fmm_target_system* target, const fmm_source_system* source,
               int scalar_potential, int gradient, int hessian, int precision);

/* ---- several source systems -----------------------------------------------------
 * fmm!(targets, (system_1, system_2, ...)) with systems of different kernels (point
 * sources and vortex particles, src/fmm.jl:807-884 with tuples of systems): one octree
 * over the bodies of all systems, as Tree(systems::Tuple, ...) (src/tree.jl:3-122)
 * builds it, with per branch one body range per system; body_to_multipole! and direct!
 * run per system, the translations once, with the Lamb-Helmholtz form when any system
 * is a vortex system (src/fmm.jl:927; the reference warns that the scalar potential is
 * then not meaningful).  Splits follow the total body count (the TreeStop and
 * SelfTuning rules with one leaf size); the Barba rule, which splits on per-system
 * counts, is rejected (FMM_ERR_ARGUMENT).  At most 8 systems; target->positions must
 * be given when n_sources > 1; n_sources == 1 is fmm_solve.  fmm_get_tree / _lists
 * export the shared trees and lists of the last call. */
FMM_API int fmm_solve_multi(fmm_ctx* ctx, const fmm_target_system* target, const fmm_source_system* sources,
                            int n_sources, const fmm_options* options, fmm_result* result);

/* ---- adjoint (vector-Jacobian product) ----------------------------------------
 * Gradients of a scalar loss L through fmm!: given the cotangents d_out = dL/d(target
 * buffer) (16 x n_t, body-major, the layout of target->out), returns dL/dstrength,
 * dL/d(source position) and, for a separate target system, dL/d(target position).
 * The reference provides this through automatic differentiation of fmm! (README.md:19;
 * no reference test pins it).  Here it is two solves with the same options: the
 * forward solve (written to target->out, as fmm_solve) and the adjoint solve, whose
 * sources sit at the targets with the cotangents as strengths and whose targets are
 * the sources:
 *   point sources (kind 1): reads row 4 (phi) of d_out, w_t = dL/dphi_t;
 *     dL/dq_s = psi(x_s), dL/dx_s = -q_s g_psi(x_s) [- w_s g(x_s) when the sources are
 *     the targets], dL/dy_t = -w_t g(y_t), with psi, g_psi the adjoint solve's potential
 *     and gradient rows and g the forward gradient rows;
 *   vortex particles (kind 3): reads rows 5..7 (u) of d_out, w_t = dL/du_t;
 *     dL/dGamma_s = u_w(x_s), (dL/dx_s)_i = sum_c Gamma_sc du_w,c/dx_i [+ sum_c w_sc
 *     du_c/dx_i when the sources are the targets], (dL/dy_t)_i = sum_c w_tc du_c/dx_i(y_t).
 * Cotangents on rows 1..3 (the target positions echoed into the buffer) pass through
 * to dL/dy (or dL/dx when the sources are the targets).  A non-zero cotangent on any
 * other row (the gradient and Hessian rows of point sources, which would need dipole
 * sources; the potential and velocity-gradient rows of vortex particles) is rejected
 * with FMM_ERR_ARGUMENT before any work.  The result is the exact gradient of the
 * continuous problem evaluated to the FMM's accuracy.  All arrays use source->memory; d_strength holds 1 (kind 1) or 3
 * (kind 3) values per source, the position gradients 3 per body; d_target_position
 * may be NULL and is not written when target->positions == NULL. */
FMM_API int fmm_vjp(fmm_ctx* ctx, const fmm_target_system* target, const fmm_source_system* source,
                    const fmm_options* options, const double* d_out, double* d_strength, double* d_source_position,
                    double* d_target_position, fmm_result* result);

/* ---- serving: concurrent requests on one device -------------------------------
 * The reference reuses a Cache across fmm! calls (src/containers.jl:264-292) and runs
 * one call at a time.  A serving context keeps n_workers solver contexts, each with
 * its own stream and resident buffers, and runs queued requests concurrently: a
 * worker takes the oldest queued request as soon as it finishes one.  n_workers / 2
 * (at least one) express workers besides take only requests of at most 65,536 source
 * plus target bodies, on highest-priority streams, so that small requests do not wait
 * behind large ones.  Device memory is one account of hbm_budget_bytes shared by all
 * workers (0 = unlimited): a request whose estimated footprint fits the budget waits,
 * in arrival order, until the memory held by the other workers' buffers (which they
 * hand back while someone waits) leaves room for it; only a request larger than the
 * whole budget finishes with FMM_ERR_MEMORY.  A request's result does not depend on what else is
 * running (each request runs the deterministic fmm_solve path on its own buffers).
 * The caller keeps every buffer of a request alive until fmm_serve_poll has
 * returned something other than FMM_PENDING for its id; each id is polled to
 * completion once.  fmm_ctx_destroy stops the server. */
typedef struct {
  fmm_target_system target; /* target.out receives the 16-row buffer, as in fmm_solve */
  fmm_source_system source;
  fmm_options options;
} fmm_request;

FMM_API int fmm_serve_start(fmm_ctx* ctx, int n_workers, size_t hbm_budget_bytes);
FMM_API int fmm_serve_submit(fmm_ctx* ctx, const fmm_request* request, uint64_t* id);
/* waits up to timeout_ms (< 0: without limit); returns the request's fmm_solve status,
 * or FMM_PENDING if it has not finished (the request stays queued) */
FMM_API int fmm_serve_poll(fmm_ctx* ctx, uint64_t id, fmm_result* result, int timeout_ms);
/* finishes the queued requests, then stops the workers */
FMM_API int fmm_serve_stop(fmm_ctx* ctx);
/* the device-memory estimate the serving account reserves for a request (bytes) */
FMM_API size_t fmm_request_footprint(const fmm_request* request);

/* ---- direct! without device allocations --------------------------------------
 * No counterpart in the reference: an all-pairs direct! (same kernels as
 * fmm_direct) for callers that cannot allocate device memory -- code running
 * while a CUDA graph is captured, hosts that give the library a fixed
 * device-memory arena, real-time loops that must not touch the allocator.
 * Needs no context and allocates nothing: inputs and output must be device
 * memory (FMM_MEMORY_DEVICE), and the only other memory used is a static
 * 6.6 MB array that every GPU loading the library holds until exit.
 * Limits: at most 32,768 sources and 32,768 targets (FMM_ERR_MEMORY beyond).
 * The work is queued on `cuda_stream` (NULL = legacy default stream) and the
 * call returns without synchronising; target->out is valid in stream order.
 * The first call on a device looks up the array's device address, so make
 * that first call before any stream capture (a failed lookup is retried by the
 * next call).  Calls share the array: calls that overlap on the GPU (other
 * streams or host threads) race on it.  The caller's current device is
 * restored before the call returns. */
FMM_API int fmm_direct_noalloc(int device, void* cuda_stream, const fmm_target_system* target,
                               const fmm_source_system* source, int scalar_potential, int gradient, int hessian,
                               int precision);

/* ---- measurement -----------------------------------------------------------
 * No counterpart in the reference: the FP32 throughput of the device's CUDA cores
 * (TFLOP/s, an FMA counting two), measured by one launch of independent fused
 * multiply-add chains (packed != 0: f32x2 operations, the form of the mixed near
 * field; else scalar) after a warm-up.  The roofline denominator of the near field.
 * Allocates a 1 KB buffer; the caller's current device is restored. */
FMM_API int fmm_measure_fp32_peak(int device, int packed, double* tflops);

/* ---- parity exports of the last fmm_solve (host memory) -------------------- */
typedef struct {
  int64_t n_branches, n_levels, n_leaves, n_bodies;
  /* Branch fields (src/containers.jl:150-164); one entry per branch */
  int64_t* body_start;   /* bodies_index[1] - 1                      */
  int64_t* body_count;
  int64_t* child_start;  /* branch_index[1] - 1                      */
  int64_t* n_children;   /* n_branches                               */
  int64_t* parent;       /* i_parent - 1 (-1 for the root)           */
  int64_t* i_leaf;       /* i_leaf - 1 (-1 for non-leaves)           */
  double* target_center; /* 3 per branch */
  double* source_center; /* 3 per branch */
  double* target_radius;
  double* source_radius;
  double* target_box;    /* 3 per branch */
  double* source_box;    /* 3 per branch */
  double* max_influence;
  int64_t* sort_index;   /* n_bodies: sorted position -> original index (Tree.sort_index_list) */
  int64_t* levels_start; /* n_levels (levels_index) */
  int64_t* levels_end;
  int64_t* leaf_index;   /* n_leaves */
} fmm_tree_view;

/* which: 0 = target tree, 1 = source tree. Call once with all pointers NULL
 * to get the counts, then again with caller-allocated arrays. */
FMM_API int fmm_get_tree(fmm_ctx* ctx, int which, fmm_tree_view* view);
/* m2l_list / direct_list (src/fmm.jl:904-907), (target, source) pairs sorted by
 * target.  Pass NULL arrays to query the counts. */
FMM_API int fmm_get_lists(fmm_ctx* ctx, int32_t* m2l, int64_t* n_m2l, int32_t* direct, int64_t* n_direct);
/* Expansions of the last solve: 4*Nh doubles per branch (Tree.expansions). */
FMM_API int fmm_get_expansions(fmm_ctx* ctx, int which, double* out, int64_t n_doubles);

/* ---- single operators on host arrays (device kernels), batched ------------
 * Expansions use the reference layout e[4*i + 2*set + reim] (i = n(n+1)/2+m,
 * set 0 = phi, 1 = chi), Nh = (p+1)(p+2)/2 coefficients.
 * lh != 0 selects the Lamb-Helmholtz (vortex) form. */
/* body_to_multipole!: bodies buf (d x n) about `center`, accumulate into expansion. */
FMM_API int fmm_op_p2m(fmm_ctx* ctx, int kind, const double* buf, int d, int64_t n, const double* center,
               int p, double* expansion);
/* multipole_to_multipole! (src/translate.jl:144): accumulate n_pairs translations
 * target[k] += M2M(src[k], src_center[k] -> target_center[k]). */
FMM_API int fmm_op_m2m(fmm_ctx* ctx, int64_t n_pairs, double* target, const double* target_center,
               const double* src, const double* src_center, int p, int lh);
/* multipole_to_local! (src/translate.jl:519-1412) with optional error control;
 * target_box/target_radius/max_influence are the target branch geometry used
 * by the error predictors. p_used (n_pairs ints) may be NULL. */
FMM_API int fmm_op_m2l(fmm_ctx* ctx, int64_t n_pairs, double* target, const double* target_center,
               const double* target_box, const double* target_radius, const double* max_influence,
               const double* src, const double* src_center, int p, int lh, int error_method,
               double eps, int bonus_expansion, int* p_used);
/* local_to_local! (src/translate.jl:1896) */
FMM_API int fmm_op_l2l(fmm_ctx* ctx, int64_t n_pairs, double* target, const double* target_center,
               const double* src, const double* src_center, int p, int lh);
/* evaluate_local (src/evaluate_expansions.jl:45): n points dx (3 each) against
 * one local expansion; out 13 per point: phi, grad(3), hessian(9). */
FMM_API int fmm_op_l2p(fmm_ctx* ctx, int64_t n, const double* dx, const double* local, int p, int lh,
               int scalar_potential, int gradient, int hessian, double* out13);

#ifdef __cplusplus
}
#endif
#endif

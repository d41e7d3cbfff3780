/*
 * fmm_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++17 FP64 restatement of FastMultipole's evaluation hot path
 * (tree -> interaction lists -> P2M/M2M/M2L/L2L/L2P + P2P), used as the
 * checker for the CUDA library and as the timed CPU baseline.  Nothing in the
 * product (fastmultipole_b200/) links, loads or calls this code; only tests/,
 * the smoke check and bench.py's CPU-baseline leg do.
 *
 * Every function in fmm_oracle.cpp cites the reference file:line it restates
 * (paths relative to the FastMultipole.jl project root).  Indices exported
 * through this header are 0-based.
 *
 * Layouts (identical to the reference's Julia arrays, column-major):
 *   expansion  : double[4*Nh]   e[4*i + 2*set + reim], set 0 = phi, 1 = chi
 *   source buf : double[d*N]    body-major, d = 5 (point source) or 7 (vortex):
 *                x y z radius strength...
 *   target buf : double[16*N]   x y z phi grad(3) hessian(9, column-major)
 */
#ifndef FMM_ORACLE_H
#define FMM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_POINT_SOURCE = 1, ORACLE_POINT_VORTEX = 3 };
/* kind of a source buffer whose rows are (x, y, z, radius, s0, s1, s2, kind): a tuple of
 * systems concatenated in tuple order, each body carrying its own kind (1 or 3) */
enum { ORACLE_KIND_PER_BODY = -1 };
enum { ORACLE_LIST_SELF_TUNING_TREE_STOP = 0, ORACLE_LIST_BARBA = 1, ORACLE_LIST_SELF_TUNING = 2 };
enum {
  ORACLE_ERR_NONE = 0,
  ORACLE_ERR_POWER_ABSOLUTE_GRADIENT = 1,
  ORACLE_ERR_POWER_RELATIVE_GRADIENT = 2,
  ORACLE_ERR_ROTATED_COEFFICIENTS_ABSOLUTE_GRADIENT = 3,
  ORACLE_ERR_ROTATED_COEFFICIENTS_RELATIVE_GRADIENT = 4,
  ORACLE_ERR_POWER_ABSOLUTE_POTENTIAL = 5,
  ORACLE_ERR_POWER_RELATIVE_POTENTIAL = 6
};

typedef struct {
  int expansion_order;
  int leaf_size_source;
  int leaf_size_target;
  double multipole_acceptance;
  int error_method;        /* ORACLE_ERR_* */
  double error_tolerance;
  int bonus_expansion;     /* BE type parameter of the error methods */
  int shrink_recenter;
  int list_method;         /* ORACLE_LIST_* */
  int farfield, nearfield, self_induced;
  int upward_pass, horizontal_pass, downward_pass;
  int scalar_potential, gradient, hessian;
  int n_threads;           /* <= 0: all OpenMP threads */
} oracle_options;

typedef struct {
  int64_t n_branches, n_levels, n_leaves, n_bodies;
  const int64_t *body_start, *body_count, *child_start, *n_children, *parent, *i_leaf;
  const double *target_center, *source_center, *target_radius, *source_radius;
  const double *target_box, *source_box, *max_influence;
  const int64_t *sort_index;      /* sorted position -> original body index */
  const int64_t *levels_start, *levels_end, *leaf_index;
} oracle_tree_view;

typedef struct oracle_run oracle_run;

/* fmm!(targets, sources; ...) with automatic trees (src/fmm.jl:862-884).
 * target_pos: 3*n_t (body-major); source_buf: d*n_s.  same_system != 0 means
 * fmm!(system) (targets are the source bodies). Returns NULL on bad input. */
oracle_run* oracle_fmm_run(const double* target_pos, int64_t n_t,
                           const double* source_buf, int d, int kind, int64_t n_s,
                           const oracle_options* opt);
int  oracle_run_output(const oracle_run* run, double* out16);          /* original order */
int  oracle_run_target_tree(const oracle_run* run, oracle_tree_view* v);
int  oracle_run_source_tree(const oracle_run* run, oracle_tree_view* v);
int64_t oracle_run_n_m2l(const oracle_run* run);
int64_t oracle_run_n_direct(const oracle_run* run);
int  oracle_run_lists(const oracle_run* run, int32_t* m2l /*2*n*/, int32_t* direct /*2*n*/);
int  oracle_run_pmax(const oracle_run* run, int* pmax, int* error_success);
int  oracle_run_times(const oracle_run* run, double* t6); /* tree, lists, near, up, horiz, down [s] */
void oracle_run_free(oracle_run* run);

/* direct!(targets, sources) all pairs (src/direct.jl:43-75), out16 original order. */
int oracle_direct(const double* target_pos, int64_t n_t, const double* source_buf, int d, int kind,
                  int64_t n_s, int scalar_potential, int gradient, int hessian, int n_threads,
                  double* out16);
/* Same, but only for the targets listed in target_ids (a subsample): out16 is 16*n_ids. */
int oracle_direct_subset(const double* target_pos, int64_t n_t, const int64_t* target_ids,
                         int64_t n_ids, const double* source_buf, int d, int kind, int64_t n_s,
                         int n_threads, double* out16);

/* ---- unit-level restatements (golden-vector pins) ---- */
int  oracle_tables(int p, double* Hs, double* zeta, double* eta, double* Mt, double* Lt);
int64_t oracle_length_Hs(int p);
int64_t oracle_length_Ts(int p);
int  oracle_update_Ts(int p, double beta, double* Ts);
int  oracle_compute_Pnms(int p, double s, double c, double* out);
int  oracle_regular_harmonics(double rho, double theta, double phi, int p, double* h /*4*Nh*/);
int  oracle_irregular_harmonics(double rho, double theta, double phi, int p, double* h);
int  oracle_translate_multipole_z(const double* src, double t, int p, int lh, double* out);
int  oracle_translate_multipole_to_local_z(const double* src, double t, int p, int lh, double* out);
int  oracle_translate_local_z(const double* src, double t, int p, int lh, double* out);
int  oracle_m2m(double* target, const double* target_center, const double* src,
                const double* src_center, int p, int lh);
int  oracle_m2l(double* target, const double* target_center, const double* target_box,
                double target_radius, double max_influence, const double* src,
                const double* src_center, int p, int lh, int error_method, double eps, int be,
                int* p_used, int* success);
int  oracle_l2l(double* target, const double* target_center, const double* src,
                const double* src_center, int p, int lh);
int  oracle_l2p(const double* dx, const double* local, int p, int lh, int ps, int gs, int hs,
                double* phi, double* grad3, double* hess9);
int  oracle_p2m(int kind, const double* buf, int d, int64_t n, const double* center, int p,
                double* expansion);
int  oracle_lh_transform(double* e, double r, int p, int local);
int  oracle_cartesian_to_spherical(double x, double y, double z, double* rtp);

#ifdef __cplusplus
}
#endif
#endif

// internal.h -- TEST INFRASTRUCTURE ONLY (see fmm_oracle.h).
// Shared declarations of the FP64 restatement.  0-based indices throughout;
// harmonic_index(n,m) of the reference (src/harmonics.jl:5-7) minus one.
#pragma once
#include <cstdint>
#include <vector>
#include <cmath>

namespace orc {

inline int64_t hidx(int n, int m) { return (int64_t)n * (n + 1) / 2 + m; }
inline int64_t nh(int p) { return (int64_t)(p + 1) * (p + 2) / 2; }
inline int64_t length_Hs(int p) { return p < 0 ? 0 : (int64_t)(p + 1) * (p + 2) * (p + 3) / 6; }
inline int64_t length_H(int n) { return (int64_t)(n + 1) * (n + 2) / 2; }
inline int64_t H_index(int mp, int m) { return (int64_t)m * (m + 1) / 2 + mp; }
inline int64_t length_Ts(int p) { return p < 0 ? 0 : (int64_t)(p + 1) * (p + 2) * (2 * p + 3) / 6; }
inline int64_t T_index(int mp, int m) { return (int64_t)m * m + mp + m; }

// expansion element access: e[4*i + 2*set + reim]  (src/tree.jl:1334-1339 layout)
inline double& ER(double* e, int set, int64_t i) { return e[4 * i + 2 * set]; }
inline double& EI(double* e, int set, int64_t i) { return e[4 * i + 2 * set + 1]; }
inline double ER(const double* e, int set, int64_t i) { return e[4 * i + 2 * set]; }
inline double EI(const double* e, int set, int64_t i) { return e[4 * i + 2 * set + 1]; }

struct Tables {
  int p = -1;
  std::vector<double> Hs, zeta, eta, Mt, Lt;
};
const Tables& tables(int p);  // grown on demand; call before any parallel region

// ---- harmonics / tables (src/harmonics.jl, src/rotate.jl, src/translate.jl) ----
void compute_Pnms(int p, double s, double c, double* out);
void compute_Hs(double* Hs, double beta, int n_start, int n_end);
void zeta_mag(double* z, int n_end);
void eta_mag(double* e, int n_end);
void power_norms(double* Mt, double* Lt, int n_end);
void regular_harmonics(double* h, double rho, double theta, double phi, int p);
void irregular_harmonics(double* h, double rho, double theta, double phi, int p);
void cartesian_to_spherical(double x, double y, double z, double& r, double& theta, double& phi);
void update_Ts(double* Ts, const double* Hs, double beta, int p);

// ---- operators ----
struct Work {  // per-thread scratch (weights_tmp_1..3, Ts, eimphis, harmonics)
  std::vector<double> t1, t2, t3, Ts, eim, harm, gnm;
  void resize(int p);
};
void p2m_point_source(double* M, double* harm, double dx, double dy, double dz, double q, int p);
void p2m_point_vortex(double* M, double* harm, double dx, double dy, double dz,
                      double vx, double vy, double vz, int p);
void translate_multipole_z(double* out, const double* src, double t, int p, bool lh);
void translate_multipole_to_local_z(double* out, const double* src, double t, int p, bool lh);
void translate_local_z(double* out, const double* src, double t, int p, bool lh);
void lh_multipole(double* M, double r, int P);
void lh_local(double* L, double r, int P);
void m2m(double* target, const double* tc, const double* src, const double* sc, int p, bool lh, Work& w);
void l2l(double* target, const double* tc, const double* src, const double* sc, int p, bool lh, Work& w);
// M2L; target geometry needed by the error-controlled variants.
struct M2LTarget {
  const double* center;
  const double* box;
  double radius;
  double max_influence;
};
int m2l(double* target, const M2LTarget& tg, const double* src, const double* sc, int p, bool lh,
        int error_method, double eps, int be, bool& success, Work& w);
void evaluate_local(const double* dx, const double* local, int p, bool lh, bool ps, bool gs, bool hs,
                    double& phi, double* grad, double* hess, Work& w);

}  // namespace orc

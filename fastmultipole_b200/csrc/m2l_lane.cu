// m2l_lane.cu -- lane-per-pair M2L for point sources, orders 1..kLaneMaxP,
// plain and error-controlled.
//
// One warp owns one target branch and takes its M2L sources 32 at a time, one
// (target, source) pair per lane.  Each lane runs the reference's chain
// (multipole_to_local!, src/translate.jl:519-550 and :555-829, :1124-1412):
// rotate_z -> rotate_y -> [degree-by-degree error control] -> coaxial
// translation -> rotate_y back -> back_rotate_z, and the 32 results of every
// degree are summed across the lanes into the warp's accumulator.
//
// Rotation about y.  The reference builds the Wigner matrix of each degree at
// beta for every pair (update_Ts_n!, src/rotate.jl:363-441),
//   T(m', m) = sum_nu w_nu H(m', nu) H(m, nu) Re(i^(m + |m'|) e^{i nu beta})  (x (-1)^(n+nu) for m' <= 0),
// H the Wigner matrix at pi/2, w_0 = 1, w_nu>0 = 2, and applies it with the
// magnitudes mag(m, a) = A(m) B(a) (src/rotate.jl:660-689, :975-1004) and the
// phases i^(a - m).  Substituting T and splitting the input by the parity of a
// gives, for the multipole (local: e^{+-i nu beta} exchanged),
//   E_nu = sum_{a even >= 2} B(a) H(a, nu) X(a),  O_nu = sum_{a odd} B(a) H(a, nu) X(a),
//   Z_nu = B(0) H(0, nu) X(0),
//   S1 = E - O,  S3 = E + O,  S2 = conj(Z + E + O),  S4 = conj(Z + E - O),  s = (-1)^(n + nu),
//   P_nu = e^{i nu beta} (S1 + s S2),  Q_nu = e^{-i nu beta} (S3 + s S4),
//   out(m) = sum_nu [A(m) H(m, nu) w_nu / 2] (P_nu + (-1)^m Q_nu),
// two products with constant (n+1) x (n+1) matrices per degree instead of a
// per-pair O(n^3) matrix build and an O(n^2) application.  The constant
// matrices B H and A H w / 2 of both magnitude sets live in constant memory
// (warp-uniform reads).  The expansions of one degree sit in registers padded
// to the kernel's maximum order, loops exit at the degree, so a single copy of
// the code serves every degree and stays resident in the instruction cache.
// The rotated multipole of all degrees (needed by the coaxial step) is kept in
// the warp's shared memory, one column per lane.
#include <mutex>

#include "context.cuh"

namespace fmmb {

namespace {

constexpr int kLaneMaxP = 12;
constexpr int kLenT = (kLaneMaxP + 1) * (kLaneMaxP + 2) * (2 * kLaneMaxP + 3) / 6;  // sum_n (n+1)^2
constexpr int kNhMax = (kLaneMaxP + 1) * (kLaneMaxP + 2) / 2;
constexpr unsigned kAll = 0xffffffffu;

// column nu of degree n at [lenT(n-1) + nu (n+1)]: B H over a, (A H w / 2) over m;
// zeta (multipole) and eta (local) magnitude sets.  kLaneMaxP padding entries let
// a sum run to the kernel's maximum order past the degree (its inputs are zero).
constexpr int kLenTPad = kLenT + kLaneMaxP + 1;
__constant__ double c_HBz[kLenTPad], c_HAz[kLenTPad], c_HBe[kLenTPad], c_HAe[kLenTPad];
// single-precision copies for the mixed path: column (n, nu) at float4 4 hi(n, nu), 16 floats
// (entries past n zero), read four entries per constant load; and k! for its scaled coaxial step
constexpr int kNCols = (kLaneMaxP + 1) * (kLaneMaxP + 2) / 2;
constexpr int kColQ = 4;  // float4 per column (kLaneMaxP + 1 <= 16 entries)
__constant__ float4 c_HBzQ[kNCols * kColQ], c_HAzQ[kNCols * kColQ], c_HBeQ[kNCols * kColQ], c_HAeQ[kNCols * kColQ];
constexpr int kFact = 2 * kLaneMaxP + 2;
__constant__ double c_fact[kFact];
__constant__ float c_factF[kFact];
__constant__ double c_Mt[kNhMax], c_Lt[kNhMax];
__constant__ double c_ifact[kMaxP + 1] = {FMM_INV_FACTORIALS};

__host__ __device__ constexpr int hi(int n, int m) { return n * (n + 1) / 2 + m; }
__host__ __device__ constexpr int lenT(int n) { return n < 0 ? 0 : (n + 1) * (n + 2) * (2 * n + 3) / 6; }

std::mutex g_tab_mu;
bool g_tab_done[64];

// B H and A H w / 2 of both magnitude sets, degrees 0..kLaneMaxP, once per device
void ensure_lane_tables(cudaStream_t st) {
  int dev = 0;
  FMM_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_tab_mu);
  if (dev < 64 && g_tab_done[dev]) return;
  HostTables h;
  build_tables(h, kLaneMaxP);
  std::vector<double> hbz(kLenTPad, 0.0), haz(kLenTPad, 0.0), hbe(kLenTPad, 0.0), hae(kLenTPad, 0.0), mt(kNhMax),
      lt(kNhMax);
  for (int n = 0; n <= kLaneMaxP; ++n) {
    const double* H = h.Hs.data() + length_Hs(n - 1);
    const double* z = h.zeta.data() + length_Ts(n - 1);
    const double* e = h.eta.data() + length_Ts(n - 1);
    const int off = lenT(n - 1);
    for (int a = 0; a <= n; ++a)
      for (int nu = 0; nu <= n; ++nu) {
        const double Hv = H[H_index(std::min(a, nu), std::max(a, nu))];
        const double w = nu == 0 ? 0.5 : 1.0;
        hbz[off + nu * (n + 1) + a] = z[a] * Hv;  // B(a): row 0 of the magnitudes
        hbe[off + nu * (n + 1) + a] = e[a] * Hv;
        haz[off + nu * (n + 1) + a] = z[a * (n + 1)] * Hv * w;  // A(m): column 0, m = a
        hae[off + nu * (n + 1) + a] = e[a * (n + 1)] * Hv * w;
      }
  }
  for (int i = 0; i < kNhMax; ++i) {
    mt[i] = h.Mt[i];
    lt[i] = h.Lt[i];
  }
  FMM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_HBz, hbz.data(), kLenTPad * 8, 0, cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_HAz, haz.data(), kLenTPad * 8, 0, cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_HBe, hbe.data(), kLenTPad * 8, 0, cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_HAe, hae.data(), kLenTPad * 8, 0, cudaMemcpyHostToDevice, st));
  // the FP32 tables in padded columns
  std::vector<float> fbz(kNCols * kColQ * 4, 0.f), faz(fbz), fbe(fbz), fae(fbz);
  for (int n = 0; n <= kLaneMaxP; ++n)
    for (int nu = 0; nu <= n; ++nu)
      for (int a = 0; a <= n; ++a) {
        const int src = lenT(n - 1) + nu * (n + 1) + a, dst = hi(n, nu) * kColQ * 4 + a;
        fbz[dst] = (float)hbz[src];
        faz[dst] = (float)haz[src];
        fbe[dst] = (float)hbe[src];
        fae[dst] = (float)hae[src];
      }
  const size_t qb = (size_t)kNCols * kColQ * sizeof(float4);
  FMM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_HBzQ, fbz.data(), qb, 0, cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_HAzQ, faz.data(), qb, 0, cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_HBeQ, fbe.data(), qb, 0, cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_HAeQ, fae.data(), qb, 0, cudaMemcpyHostToDevice, st));
  std::vector<double> fact(kFact);
  std::vector<float> factf(kFact);
  fact[0] = 1.0;
  for (int k = 1; k < kFact; ++k) fact[k] = fact[k - 1] * k;
  for (int k = 0; k < kFact; ++k) factf[k] = (float)fact[k];
  FMM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_fact, fact.data(), kFact * 8, 0, cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_factF, factf.data(), kFact * 4, 0, cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_Mt, mt.data(), kNhMax * 8, 0, cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_Lt, lt.data(), kNhMax * 8, 0, cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaStreamSynchronize(st));
  if (dev < 64) g_tab_done[dev] = true;
}

// rotate_y of degree n (X -> Y) on expansions padded to PMAX + 1 registers
// (entries past n are zero); LOCAL: eta magnitudes and e^{-+i nu beta}.  The nu
// loop runs at run time and fuses both matrix products: column nu of B H gives
// E, O, Z, and P_nu +- Q_nu is accumulated into every output at once through
// column nu of A H w / 2.  Sums run to PMAX from one column base, so the table
// entries are uniform constant reads at fixed offsets and no term is predicated
// (measured: sums that stop at the degree are slower, the fixed trip counts
// schedule better than the skipped terms save).
template <bool LOCAL, class V>
__device__ __forceinline__ V tab_b(int i) {
  return LOCAL ? c_HBe[i] : c_HBz[i];
}
template <bool LOCAL, class V>
__device__ __forceinline__ V tab_a(int i) {
  return LOCAL ? c_HAe[i] : c_HAz[i];
}

// FP32 rotate_y (the mixed path): rot_y below with the tables read as float4 quads of a
// padded column, the same terms in the same order
template <int PMAX, bool LOCAL>
__device__ __forceinline__ void rot_y_q(int n, const float (&Xr)[PMAX + 1], const float (&Xi)[PMAX + 1], float cb,
                                        float sb, float (&Yr)[PMAX + 1], float (&Yi)[PMAX + 1]) {
  constexpr int NQ = PMAX / 4 + 1;  // quads covering entries 0..PMAX
#pragma unroll
  for (int m = 0; m <= PMAX; ++m) Yr[m] = Yi[m] = 0.f;
  float c = 1.f, s = 0.f;  // cos, sin (nu beta) by the reference's recurrence
#pragma unroll 1
  for (int nu = 0; nu <= n; ++nu) {
    if (nu > 0) {
      const float cn = cb * c - sb * s;
      const float sn = sb * c + cb * s;
      c = cn;
      s = sn;
    }
    const int q0 = hi(n, nu) * kColQ;
    float Er = 0, Ei = 0, Or = 0, Oi = 0, h0 = 0;
#pragma unroll
    for (int aq = 0; aq < NQ; ++aq) {
      const float4 h4 = LOCAL ? c_HBeQ[q0 + aq] : c_HBzQ[q0 + aq];
      const float hh[4] = {h4.x, h4.y, h4.z, h4.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int a = 4 * aq + j;
        if (a > PMAX) break;
        if (a == 0) {
          h0 = hh[0];
        } else if (a & 1) {
          Or += hh[j] * Xr[a];
          Oi += hh[j] * Xi[a];
        } else {
          Er += hh[j] * Xr[a];
          Ei += hh[j] * Xi[a];
        }
      }
    }
    const float Zr = h0 * Xr[0], Zi = h0 * Xi[0];
    const float sg = ((n + nu) & 1) ? -1.f : 1.f;
    const float S1r = Er - Or, S1i = Ei - Oi;
    const float S3r = Er + Or, S3i = Ei + Oi;
    const float S2r = Zr + S3r, S2i = -(Zi + S3i);
    const float S4r = Zr + S1r, S4i = -(Zi + S1i);
    const float A1r = S1r + sg * S2r, A1i = S1i + sg * S2i;
    const float A3r = S3r + sg * S4r, A3i = S3i + sg * S4i;
    const float ss = LOCAL ? -s : s;
    const float Pr = c * A1r - ss * A1i, Pi = c * A1i + ss * A1r;
    const float Qr = c * A3r + ss * A3i, Qi = c * A3i - ss * A3r;
    const float Rpr = Pr + Qr, Rpi = Pi + Qi, Rmr = Pr - Qr, Rmi = Pi - Qi;
#pragma unroll
    for (int mq = 0; mq < NQ; ++mq) {
      const float4 h4 = LOCAL ? c_HAeQ[q0 + mq] : c_HAzQ[q0 + mq];
      const float hh[4] = {h4.x, h4.y, h4.z, h4.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int m = 4 * mq + j;
        if (m > PMAX) break;
        Yr[m] += hh[j] * ((m & 1) ? Rmr : Rpr);
        Yi[m] += hh[j] * ((m & 1) ? Rmi : Rpi);
      }
    }
  }
}

template <int PMAX, bool LOCAL, class V = double>
__device__ __forceinline__ void rot_y(int n, const V (&Xr)[PMAX + 1], const V (&Xi)[PMAX + 1], V cb, V sb,
                                      V (&Yr)[PMAX + 1], V (&Yi)[PMAX + 1]) {
  if constexpr (sizeof(V) == 4) {
    rot_y_q<PMAX, LOCAL>(n, Xr, Xi, cb, sb, Yr, Yi);
  } else {
    const int t0 = lenT(n - 1), w = n + 1;
#pragma unroll
    for (int m = 0; m <= PMAX; ++m) Yr[m] = Yi[m] = V(0);
    V c = V(1), s = V(0);  // cos, sin (nu beta) by the reference's recurrence
#pragma unroll 1
    for (int nu = 0; nu <= n; ++nu) {
      if (nu > 0) {
        const V cn = cb * c - sb * s;
        const V sn = sb * c + cb * s;
        c = cn;
        s = sn;
      }
      const int col = t0 + nu * w;
      V Er = 0, Ei = 0, Or = 0, Oi = 0;
#pragma unroll
      for (int a = 1; a <= PMAX; ++a) {
        const V h = tab_b<LOCAL, V>(col + a);
        if (a & 1) {
          Or += h * Xr[a];
          Oi += h * Xi[a];
        } else {
          Er += h * Xr[a];
          Ei += h * Xi[a];
        }
      }
      const V h0 = tab_b<LOCAL, V>(col);
      const V Zr = h0 * Xr[0], Zi = h0 * Xi[0];
      const V sg = ((n + nu) & 1) ? V(-1) : V(1);
      const V S1r = Er - Or, S1i = Ei - Oi;
      const V S3r = Er + Or, S3i = Ei + Oi;
      const V S2r = Zr + S3r, S2i = -(Zi + S3i);
      const V S4r = Zr + S1r, S4i = -(Zi + S1i);
      const V A1r = S1r + sg * S2r, A1i = S1i + sg * S2i;
      const V A3r = S3r + sg * S4r, A3i = S3i + sg * S4i;
      const V ss = LOCAL ? -s : s;
      const V Pr = c * A1r - ss * A1i, Pi = c * A1i + ss * A1r;
      const V Qr = c * A3r + ss * A3i, Qi = c * A3i - ss * A3r;
      const V Rpr = Pr + Qr, Rpi = Pi + Qi, Rmr = Pr - Qr, Rmi = Pi - Qi;
#pragma unroll
      for (int m = 0; m <= PMAX; ++m) {
        const V h = tab_a<LOCAL, V>(col + m);
        Yr[m] += h * ((m & 1) ? Rmr : Rpr);
        Yi[m] += h * ((m & 1) ? Rmi : Rpi);
      }
    }
  }
}

// per-lane state of one (target, source) pair
struct Pair {
  const double* src;  // multipole of the source branch (interleaved e[4 i + 2 set + reim])
  double cph, sph, cth, sth, r, rinv;
  int P;        // order used
  bool valid;   // lane holds a pair
  bool active;  // still inside the error-control loop
  bool ok;      // tolerance met
  // error control (src/translate.jl:1124-1412, :555-829)
  double thr, r_mp, r_mp_inv, r_mp_inv_np2, r_l, r_l_nm1, nm1_fact_inv, np1_fact, n_fact_t_np1, mp_phi, Mn0;
  double un;  // n! / t^(n+1) of the current degree (coaxial factor of source degree 0)
};

// rotated multipole in shared memory: plane c (re, im) of coefficient i, column lane
__device__ __forceinline__ double& MS(double* Ms, int i, int c, int lane) { return Ms[(2 * i + c) * 32 + lane]; }
__device__ __forceinline__ double MSr(const double* Ms, int i, int c, int lane) { return Ms[(2 * i + c) * 32 + lane]; }

// rotate_z + rotate_y of degree n of the lane's multipole into shared memory;
// returns the multipole power of degree n (rotate_z_n_power!, weight 1 for every m)
template <int PMAX>
__device__ __forceinline__ double fwd_degree(int n, const Pair& q, double* Ms, int lane, double& y0r, double& y1r,
                                             double& y1i) {
  double Xr[PMAX + 1], Xi[PMAX + 1];
  double er = 1.0, ei = 0.0, pw = 0.0;
  const int base = hi(n, 0);
#pragma unroll
  for (int a = 0; a <= PMAX; ++a) {
    Xr[a] = Xi[a] = 0.0;
    if (a > n) continue;
    const double2 u = __ldg(reinterpret_cast<const double2*>(q.src) + 2 * (base + a));
    const double Nt = c_Mt[base + a];
    pw += (u.x * u.x + u.y * u.y) * Nt * Nt;
    Xr[a] = n == 0 ? u.x : u.x * er - u.y * ei;
    Xi[a] = n == 0 ? u.y : u.x * ei + u.y * er;
    const double t = er;
    er = er * q.cph - ei * q.sph;
    ei = t * q.sph + ei * q.cph;
  }
  double Yr[PMAX + 1], Yi[PMAX + 1];
  rot_y<PMAX, false>(n, Xr, Xi, q.cth, q.sth, Yr, Yi);
#pragma unroll
  for (int m = 0; m <= PMAX; ++m) {
    if (m > n) break;
    MS(Ms, base + m, 0, lane) = Yr[m];
    MS(Ms, base + m, 1, lane) = Yi[m];
  }
  y0r = Yr[0];
  y1r = Yr[1 % (PMAX + 1)];
  y1i = Yi[1 % (PMAX + 1)];
  return sqrt(pw);
}

// local error estimate of degree n from the rotated multipole of degrees <= n
// The coaxial factor of source degree n' is the running product n!/t^(n+1) * prod_{j<=n'}
// (n+j)/t in the reference's order whatever the order m, so the sums run source degrees
// outer and orders inner (one degree's loads and FMAs independent; each sum keeps its
// n'-ascending order).
// power: 0 = the RotatedCoefficients methods, 1 = Power*Gradient, 2 = Power*Potential
template <int PMAX>
__device__ __forceinline__ double eps_local(int n, const Pair& q, const double* Ms, int lane, int power) {
  if (power) {
    // degree n of translate_multipole_to_local_z_n! and local_power (src/translate.jl:238-295, :455-502)
    double vr[PMAX + 1], vi[PMAX + 1];
#pragma unroll
    for (int m = 0; m <= PMAX; ++m) vr[m] = vi[m] = 0.0;
    double c = q.un;
#pragma unroll 1
    for (int np = 0; np <= n; ++np) {
      if (np > 0) c *= (n + np) * q.rinv;  // (n + n')! / t^(n+n'+1), the reference's product order
      const int base = hi(np, 0);
#pragma unroll
      for (int m = 0; m <= PMAX; ++m) {
        if (m > np) break;
        vr[m] += c * MSr(Ms, base + m, 0, lane);
        vi[m] += c * MSr(Ms, base + m, 1, lane);
      }
    }
    double a = 0.0;
#pragma unroll
    for (int m = 0; m <= PMAX; ++m) {
      if (m > n) break;
      const double Nt = c_Lt[hi(n, m)];
      a += (vr[m] * vr[m] + vi[m] * vi[m]) * Nt * Nt;
    }
    const double lphi = sqrt(a);
    if (power == 2)  // src/translate.jl:912
      return 1.7320508075688772 * lphi * q.r_l_nm1 * q.r_l * q.nm1_fact_inv / (c_Lt[hi(n, 0)] * n);
    return 1.7320508075688772 * lphi * q.r_l_nm1 * q.nm1_fact_inv / c_Lt[hi(n, 0)];
  }
  // translate_multipole_to_local_z_m01_n (src/translate.jl:302-364)
  double c = q.n_fact_t_np1;
  int n_np = n;
  double a0 = 0;
#pragma unroll 1
  for (int np = 0; np <= n; ++np) {
    a0 += c * MSr(Ms, hi(np, 0), 0, lane);
    n_np += 1;
    c *= n_np * q.rinv;
  }
  c = q.n_fact_t_np1 * ((n + 1) * q.rinv);
  n_np = n + 1;
  double b1r = 0, b1i = 0;
#pragma unroll 1
  for (int np = 1; np <= n; ++np) {
    b1r += c * MSr(Ms, hi(np, 1), 0, lane);
    b1i += c * MSr(Ms, hi(np, 1), 1, lane);
    n_np += 1;
    c *= n_np * q.rinv;
  }
  return (fabs(b1r) + fabs(b1i) + fabs(a0)) * q.r_l_nm1 * q.nm1_fact_inv;
}

// one degree of the reference's error-controlled loop (src/translate.jl:1124-1412,
// :555-829) after degree n of the rotated multipole is in shared memory
template <int PMAX>
__device__ __forceinline__ void err_step(int n, Pair& q, const double* Ms, int lane, int power, int be,
                                         double pn_phi, double y0r, double y1r, double y1i) {
  const double Mn0_next = c_Mt[hi(n, 0)];
  double eps_mp;
  if (power == 2)  // the potential variants read degree n's power (src/translate.jl:893)
    eps_mp = 1.7320508075688772 * pn_phi * q.r_mp_inv_np2 * q.r_mp * q.np1_fact / (q.Mn0 * (n + 1));
  else if (power)
    eps_mp = 1.7320508075688772 * q.mp_phi * q.r_mp_inv_np2 * q.np1_fact / q.Mn0;
  else
    eps_mp = (sqrt(y1r * y1r + y1i * y1i) + fabs(y0r)) * q.np1_fact * q.r_mp_inv_np2;
  if (eps_mp <= q.thr) {
    const double eps_l = eps_local<PMAX>(n, q, Ms, lane, power);
    if (eps_mp + eps_l * 2.0 <= q.thr) {
      q.P = n - 1 + (be ? 1 : 0);
      q.ok = true;
      q.active = false;
      return;
    }
  }
  if (power || n < PMAX) {
    q.n_fact_t_np1 *= (n + 1) * q.rinv;
    q.r_l_nm1 *= q.r_l;
    q.r_mp_inv_np2 *= q.r_mp_inv;
    q.nm1_fact_inv /= n;
    q.np1_fact *= n + 1;
  }
  if (power) {
    q.mp_phi = pn_phi;
    q.Mn0 = Mn0_next;
  }
}

// degree n of the local expansion: coaxial translation of the rotated multipole
// (sources m..P), rotate_y back, back_rotate_z, then the sum over the 32 lanes
// into the warp accumulator (stage: 2 (PMAX+1) rows of 33 doubles)
template <int PMAX>
__device__ __forceinline__ void back_degree(int n, double un, const Pair& q, const double* Ms, double* stage,
                                            double* acc, int lane) {
  const bool on = q.valid && n <= q.P;
  // (n + n')! / t^(n+n'+1) as one running product in the reference's order, common to every
  // order m: source degrees outer, orders inner
  double Xr[PMAX + 1], Xi[PMAX + 1];
#pragma unroll
  for (int m = 0; m <= PMAX; ++m) Xr[m] = Xi[m] = 0.0;
  const int top = on ? q.P : -1;
  double c = un;
#pragma unroll 1
  for (int np = 0; np <= top; ++np) {
    if (np > 0) c *= (n + np) * q.rinv;
    const int base = hi(np, 0);
#pragma unroll
    for (int m = 0; m <= PMAX; ++m) {
      if (m > n || m > np) break;
      Xr[m] += c * MSr(Ms, base + m, 0, lane);
      Xi[m] += c * MSr(Ms, base + m, 1, lane);
    }
  }
  double Yr[PMAX + 1], Yi[PMAX + 1];
  rot_y<PMAX, true>(n, Xr, Xi, q.cth, q.sth, Yr, Yi);
  double er = 1.0, ei = 0.0;
#pragma unroll
  for (int m = 0; m <= PMAX; ++m) {
    if (m > n) break;
    const double cr = er, ci = -ei;
    const double vr = n == 0 ? Yr[m] : Yr[m] * cr - Yi[m] * ci;
    const double vi = n == 0 ? Yi[m] : Yr[m] * ci + Yi[m] * cr;
    stage[(2 * m) * 33 + lane] = on ? vr : 0.0;
    stage[(2 * m + 1) * 33 + lane] = on ? vi : 0.0;
    const double t = er;
    er = er * q.cph - ei * q.sph;
    ei = t * q.sph + ei * q.cph;
  }
  __syncwarp();
  if (lane < 2 * (n + 1)) {
    double v = 0.0;
#pragma unroll 8
    for (int k = 0; k < 32; ++k) v += stage[lane * 33 + k];
    acc[2 * hi(n, 0) + lane] += v;
  }
  __syncwarp();
}

// ---- single precision (the mixed solve).  Degree n of the rotated multipole is
// stored scaled by t^-n (t = |target centre - source centre|), M'(n, m) = M(n, m) / t^n,
// which keeps the FP32 values of order q (sources lie within MAC * t of their centre):
// the coaxial factor (n + n')! / t^(n+n'+1) becomes (n + n')! with t^-(n+1) applied to
// the finished local coefficient in FP64.  The error control reads the same quantities
// unscaled in FP64; accumulation is FP64.
__device__ __forceinline__ float& MSf(float* Ms, int i, int c, int lane) { return Ms[(2 * i + c) * 32 + lane]; }
__device__ __forceinline__ float MSfr(const float* Ms, int i, int c, int lane) { return Ms[(2 * i + c) * 32 + lane]; }

// rotate_z + rotate_y of degree n into shared memory (scaled by sc = t^-n); returns the
// multipole power of degree n; y0r, y1r, y1i: unscaled rotated coefficients (n, 0), (n, 1)
template <int PMAX>
__device__ __forceinline__ double fwd_degree_f(int n, const Pair& q, float* Ms, int lane, double sc, double& y0r,
                                               double& y1r, double& y1i) {
  float Xr[PMAX + 1], Xi[PMAX + 1];
  double er = 1.0, ei = 0.0, pw = 0.0;
  const int base = hi(n, 0);
#pragma unroll
  for (int a = 0; a <= PMAX; ++a) {
    Xr[a] = Xi[a] = 0.0f;
    if (a > n) continue;
    const double2 u = __ldg(reinterpret_cast<const double2*>(q.src) + 2 * (base + a));
    const double Nt = c_Mt[base + a];
    pw += (u.x * u.x + u.y * u.y) * Nt * Nt;
    Xr[a] = (float)((n == 0 ? u.x : u.x * er - u.y * ei) * sc);
    Xi[a] = (float)((n == 0 ? u.y : u.x * ei + u.y * er) * sc);
    const double t = er;
    er = er * q.cph - ei * q.sph;
    ei = t * q.sph + ei * q.cph;
  }
  float Yr[PMAX + 1], Yi[PMAX + 1];
  rot_y<PMAX, false, float>(n, Xr, Xi, (float)q.cth, (float)q.sth, Yr, Yi);
#pragma unroll
  for (int m = 0; m <= PMAX; ++m) {
    if (m > n) break;
    MSf(Ms, base + m, 0, lane) = Yr[m];
    MSf(Ms, base + m, 1, lane) = Yi[m];
  }
  const double us = 1.0 / sc;
  y0r = Yr[0] * us;
  y1r = Yr[1 % (PMAX + 1)] * us;
  y1i = Yi[1 % (PMAX + 1)] * us;
  return sqrt(pw);
}

// local error estimate of degree n (eps_local above) from the scaled rotated multipole;
// tn1 = t^-(n+1)
// (the coaxial sums run source degrees outer, orders inner, so that one degree's loads and
// FMAs are independent; each sum keeps its n'-ascending order)
template <int PMAX>
__device__ __forceinline__ double eps_local_f(int n, const Pair& q, const float* Ms, int lane, int power,
                                              double tn1) {
  if (power) {
    double vr[PMAX + 1], vi[PMAX + 1];
#pragma unroll
    for (int m = 0; m <= PMAX; ++m) vr[m] = vi[m] = 0.0;
#pragma unroll 1
    for (int np = 0; np <= n; ++np) {
      const double c = c_fact[n + np];
      const int base = hi(np, 0);
#pragma unroll
      for (int m = 0; m <= PMAX; ++m) {
        if (m > np) break;
        vr[m] += c * MSfr(Ms, base + m, 0, lane);
        vi[m] += c * MSfr(Ms, base + m, 1, lane);
      }
    }
    double a = 0.0;
#pragma unroll
    for (int m = 0; m <= PMAX; ++m) {
      if (m > n) break;
      const double xr = vr[m] * tn1, xi = vi[m] * tn1;
      const double Nt = c_Lt[hi(n, m)];
      a += (xr * xr + xi * xi) * Nt * Nt;
    }
    const double lphi = sqrt(a);
    if (power == 2)
      return 1.7320508075688772 * lphi * q.r_l_nm1 * q.r_l * q.nm1_fact_inv / (c_Lt[hi(n, 0)] * n);
    return 1.7320508075688772 * lphi * q.r_l_nm1 * q.nm1_fact_inv / c_Lt[hi(n, 0)];
  }
  double a0 = 0, b1r = 0, b1i = 0;
#pragma unroll 1
  for (int np = 0; np <= n; ++np) {
    const double c = c_fact[n + np];
    a0 += c * MSfr(Ms, hi(np, 0), 0, lane);
    if (np >= 1) {
      b1r += c * MSfr(Ms, hi(np, 1), 0, lane);
      b1i += c * MSfr(Ms, hi(np, 1), 1, lane);
    }
  }
  return (fabs(b1r * tn1) + fabs(b1i * tn1) + fabs(a0 * tn1)) * q.r_l_nm1 * q.nm1_fact_inv;
}

template <int PMAX>
__device__ __forceinline__ void err_step_f(int n, Pair& q, const float* Ms, int lane, int power, int be,
                                           double pn_phi, double y0r, double y1r, double y1i, double tn1) {
  const double Mn0_next = c_Mt[hi(n, 0)];
  double eps_mp;
  if (power == 2)
    eps_mp = 1.7320508075688772 * pn_phi * q.r_mp_inv_np2 * q.r_mp * q.np1_fact / (q.Mn0 * (n + 1));
  else if (power)
    eps_mp = 1.7320508075688772 * q.mp_phi * q.r_mp_inv_np2 * q.np1_fact / q.Mn0;
  else
    eps_mp = (sqrt(y1r * y1r + y1i * y1i) + fabs(y0r)) * q.np1_fact * q.r_mp_inv_np2;
  if (eps_mp <= q.thr) {
    const double eps_l = eps_local_f<PMAX>(n, q, Ms, lane, power, tn1);
    if (eps_mp + eps_l * 2.0 <= q.thr) {
      q.P = n - 1 + (be ? 1 : 0);
      q.ok = true;
      q.active = false;
      return;
    }
  }
  if (power || n < PMAX) {
    q.r_l_nm1 *= q.r_l;
    q.r_mp_inv_np2 *= q.r_mp_inv;
    q.nm1_fact_inv /= n;
    q.np1_fact *= n + 1;
  }
  if (power) {
    q.mp_phi = pn_phi;
    q.Mn0 = Mn0_next;
  }
}

// degree n of the local expansion from the scaled rotated multipole: coaxial
// translation with (n + n')!, rotate_y back and back_rotate_z in FP32, then t^-(n+1) and
// the sum over the 32 lanes in FP64 (tn1 = t^-(n+1))
template <int PMAX>
__device__ __forceinline__ void back_degree_f(int n, const Pair& q, const float* Ms, double* stage, double* acc,
                                              int lane, double tn1) {
  const bool on = q.valid && n <= q.P;
  // out(n, m) = sum_{n' >= m} (n + n')! M(n', m): source degrees outer, orders inner, so that
  // one degree's loads and FMAs are independent (each sum keeps its n'-ascending order)
  float Xr[PMAX + 1], Xi[PMAX + 1];
#pragma unroll
  for (int m = 0; m <= PMAX; ++m) Xr[m] = Xi[m] = 0.0f;
  const int top = on ? q.P : -1;
#pragma unroll 1
  for (int np = 0; np <= top; ++np) {
    const float c = c_factF[n + np];
    const int base = hi(np, 0);
#pragma unroll
    for (int m = 0; m <= PMAX; ++m) {
      if (m > n || m > np) break;
      Xr[m] += c * MSfr(Ms, base + m, 0, lane);
      Xi[m] += c * MSfr(Ms, base + m, 1, lane);
    }
  }
  float Yr[PMAX + 1], Yi[PMAX + 1];
  rot_y<PMAX, true, float>(n, Xr, Xi, (float)q.cth, (float)q.sth, Yr, Yi);
  float er = 1.0f, ei = 0.0f;
  const float cph = (float)q.cph, sph = (float)q.sph;
#pragma unroll
  for (int m = 0; m <= PMAX; ++m) {
    if (m > n) break;
    const float cr = er, ci = -ei;
    const float vr = n == 0 ? Yr[m] : Yr[m] * cr - Yi[m] * ci;
    const float vi = n == 0 ? Yi[m] : Yr[m] * ci + Yi[m] * cr;
    stage[(2 * m) * 33 + lane] = on ? vr * tn1 : 0.0;
    stage[(2 * m + 1) * 33 + lane] = on ? vi * tn1 : 0.0;
    const float t = er;
    er = er * cph - ei * sph;
    ei = t * sph + ei * cph;
  }
  __syncwarp();
  if (lane < 2 * (n + 1)) {
    double v = 0.0;
#pragma unroll 8
    for (int k = 0; k < 32; ++k) v += stage[lane * 33 + k];
    acc[2 * hi(n, 0) + lane] += v;
  }
  __syncwarp();
}

__device__ __forceinline__ unsigned long long lane_pair_flops(int P) {
  // the reference's operation count: 4 [2 sum_n (n+1)(2n+1) + sum_n sum_m (P-m+1)]
  // closed forms: sum_n (n+1)(2n+1) = P(P+1)(2P+1)/3 + 3P(P+1)/2 + P+1, sum_m (P-m+1)^2 = (P+1)(P+2)(2P+3)/6
  const unsigned long long p = (unsigned long long)P;
  const unsigned long long rot = p * (p + 1) * (2 * p + 1) / 3 + 3 * p * (p + 1) / 2 + p + 1;
  const unsigned long long coax = (p + 1) * (p + 2) * (2 * p + 3) / 6;
  return 4ull * (2 * rot + coax);
}

// minimum_distance, src/error.jl:5-20
__device__ __forceinline__ double minabs(double x, double y) {
  return x * (fabs(x) <= fabs(y) ? 1.0 : 0.0) + y * (fabs(y) < fabs(x) ? 1.0 : 0.0);
}
__device__ __forceinline__ double min_dist_1d(double dx, double rm, double rp) {
  double right = dx + rp, left = dx + rm;
  double same = (right * left >= 0) ? 1.0 : 0.0;
  return same * minabs(right, left);
}

// bytes: rotated multipole [2 NH][32] (V), stage [2 (PMAX+1)][33] and accumulator [2 NH] (FP64)
template <int PMAX, class V>
__host__ __device__ constexpr size_t lane_smem_bytes() {
  return (size_t)2 * hi(PMAX + 1, 0) * 32 * sizeof(V) +
         ((size_t)2 * (PMAX + 1) * 33 + (size_t)2 * hi(PMAX + 1, 0)) * sizeof(double);
}

// one warp per CTA; warp b owns target tgt_list[b] and its sources src_of[off[b] .. off[b+1])
// W warps per CTA share one target row (pairs strided over the warps), for launches of few
// rows; the warps' accumulators are summed in warp order
template <int PMAX, class V, int W = 1>
__global__ void __launch_bounds__(32 * W) k_m2l_lane(const int* __restrict__ tgt_list, const int* __restrict__ off,
                                                 const int* __restrict__ src_of, double* __restrict__ local,
                                                 const double* __restrict__ multipole,
                                                 const double* __restrict__ tcen, const double* __restrict__ tbox,
                                                 const double* __restrict__ trad, const double* __restrict__ maxinf,
                                                 const double* __restrict__ scen, int em, double eps_in, int be,
                                                 int* __restrict__ p_used, int* __restrict__ st_pmax,
                                                 int* __restrict__ st_fail,
                                                 unsigned long long* __restrict__ st_flops) {
  constexpr int NH = hi(PMAX + 1, 0);
  constexpr bool F32 = sizeof(V) == 4;
  extern __shared__ double lane_smem[];
  constexpr size_t WSM = lane_smem_bytes<PMAX, V>() / sizeof(double);  // one warp's region
  const int w = threadIdx.x >> 5;
  double* stage = lane_smem + (size_t)w * WSM;       // [2 (PMAX+1)][33]
  double* acc = stage + 2 * (PMAX + 1) * 33;         // [2 NH]
  V* MsV = reinterpret_cast<V*>(acc + 2 * NH);       // rotated multipole [2 NH][32]
  double* Ms = reinterpret_cast<double*>(MsV);
  float* Msf = reinterpret_cast<float*>(MsV);
  const int lane = threadIdx.x & 31;
  const int b = blockIdx.x;
  const int t = tgt_list[b];
  const double tc0 = tcen[3 * t], tc1 = tcen[3 * t + 1], tc2 = tcen[3 * t + 2];
  const bool errc = em != FMM_ERROR_NONE;
  const bool relative = (em == FMM_POWER_RELATIVE_GRADIENT || em == FMM_ROTATED_COEFFICIENTS_RELATIVE_GRADIENT ||
                        em == FMM_POWER_RELATIVE_POTENTIAL);
  const int power = (em == FMM_POWER_ABSOLUTE_POTENTIAL || em == FMM_POWER_RELATIVE_POTENTIAL)
                        ? 2
                        : ((em == FMM_POWER_ABSOLUTE_GRADIENT || em == FMM_POWER_RELATIVE_GRADIENT) ? 1 : 0);
  const double eps = relative ? maxinf[t] * eps_in : eps_in;
  const double tb0 = tbox[3 * t], tb1 = tbox[3 * t + 1], tb2 = tbox[3 * t + 2];
  const double r_l = trad[t];
  for (int i = lane; i < 2 * NH; i += 32) acc[i] = 0.0;
  int pmax = 0;
  bool fail = false;
  unsigned long long fl = 0;
  const int l0 = off[b], l1 = off[b + 1];
  for (int lb = l0 + 32 * w; lb < l1; lb += 32 * W) {
    Pair q;
    const int l = lb + lane;
    q.valid = l < l1;
    q.P = PMAX;
    q.ok = true;
    q.active = false;
    q.src = multipole;
    q.cph = 1.0;
    q.sph = 0.0;
    q.cth = 1.0;
    q.sth = 0.0;
    q.r = 1.0;
    q.rinv = 1.0;
    q.un = 1.0;
    if (q.valid) {
      const int s = src_of[l];
      q.src = multipole + (int64_t)4 * NH * s;
      const double x = tc0 - scen[3 * s], y = tc1 - scen[3 * s + 1], z = tc2 - scen[3 * s + 2];
      // cartesian_to_spherical (src/rotate.jl:9-21) in cos/sin form
      const double x2y2 = x * x + y * y;
      const double r2 = x2y2 + z * z;
      q.r = (r2 == 0.0) ? r2 : sqrt(r2);
      if (x2y2 > 0) {
        const double rho = sqrt(x2y2);
        q.cph = x / rho;
        q.sph = y / rho;
        q.cth = z / q.r;
        q.sth = rho / q.r;
      } else {
        q.cth = (q.r > 0 && z < 0) ? -1.0 : 1.0;
      }
      q.rinv = 1 / q.r;
      q.un = q.rinv;
      if (errc) {
        const double mdx = min_dist_1d(x, -tb0, tb0), mdy = min_dist_1d(y, -tb1, tb1), mdz = min_dist_1d(z, -tb2, tb2);
        const double r_mp = sqrt(mdx * mdx + mdy * mdy + mdz * mdz);
        q.r_mp = r_mp;
        q.r_mp_inv = 1.0 / r_mp;
        q.r_mp_inv_np2 = q.r_mp_inv * q.r_mp_inv * q.r_mp_inv;
        q.r_l = r_l;
        q.r_l_nm1 = 1.0;
        q.n_fact_t_np1 = q.rinv * q.rinv;
        q.nm1_fact_inv = 1.0;
        q.np1_fact = 2.0;
        q.Mn0 = c_Mt[0];
        q.mp_phi = sqrt((q.src[0] * q.src[0] + q.src[1] * q.src[1]) * q.Mn0 * q.Mn0);
        q.thr = eps * 4 * kPi;
        q.ok = false;
        q.active = true;
      }
    }
    // degree 0 for every valid lane, then degree by degree while a lane is active
    // (error control) or up to PMAX (plain)
    q.active = q.valid;
    double sc = 1.0;  // t^-n (single precision path)
#pragma unroll 1
    for (int n = 0; n <= PMAX; ++n) {
      if (!__any_sync(kAll, q.active)) break;
      if (!q.active) continue;
      if (n > 0) {
        q.un *= n * q.rinv;
        sc *= q.rinv;
      }
      double y0r, y1r, y1i;
      if constexpr (F32) {
        const double pn_phi = fwd_degree_f<PMAX>(n, q, Msf, lane, sc, y0r, y1r, y1i);
        if (errc && n > 0) err_step_f<PMAX>(n, q, Msf, lane, power, be, pn_phi, y0r, y1r, y1i, sc * q.rinv);
      } else {
        const double pn_phi = fwd_degree<PMAX>(n, q, Ms, lane, y0r, y1r, y1i);
        if (errc && n > 0) err_step<PMAX>(n, q, Ms, lane, power, be, pn_phi, y0r, y1r, y1i);
      }
    }
    q.active = false;  // error control: lanes still active reached PMAX (P = PMAX, tolerance missed)
    int pw = q.valid ? q.P : -1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pw = max(pw, __shfl_xor_sync(kAll, pw, o));
    __syncwarp();
    double un = q.rinv, tn1 = q.rinv;  // n! / t^(n+1) and t^-(n+1)
#pragma unroll 1
    for (int n = 0; n <= pw; ++n) {
      if (n > 0) {
        un *= n * q.rinv;
        tn1 *= q.rinv;
      }
      if constexpr (F32)
        back_degree_f<PMAX>(n, q, Msf, stage, acc, lane, tn1);
      else
        back_degree<PMAX>(n, un, q, Ms, stage, acc, lane);
    }
    if (q.valid) {
      if (p_used) p_used[l] = q.P;
      pmax = max(pmax, q.P);
      fail = fail || !q.ok;
      fl += lane_pair_flops(q.P);
    }
    __syncwarp();
  }
  double* dst = local + (int64_t)4 * NH * t;
  if constexpr (W == 1) {
    for (int i = lane; i < 2 * NH; i += 32) dst[4 * (i >> 1) + (i & 1)] += acc[i];
  } else {
    __syncthreads();
    if (w == 0)
      for (int i = lane; i < 2 * NH; i += 32) {
        double v = acc[i];
        for (int q = 1; q < W; ++q) v += acc[(size_t)q * WSM + i];
        dst[4 * (i >> 1) + (i & 1)] += v;
      }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    pmax = max(pmax, __shfl_xor_sync(kAll, pmax, o));
    fl += __shfl_xor_sync(kAll, fl, o);
  }
  const bool any_fail = __any_sync(kAll, fail);
  if (lane == 0) {
    atomicMax(st_pmax, pmax);
    if (any_fail) atomicExch(st_fail, 1);
    atomicAdd(st_flops, fl);
  }
}

// launches of fewer M2L target rows than kWideM2LRowsPerSM per SM take kWideM2LWarps warps per row
constexpr int kWideM2LWarps = 4;
constexpr int kWideM2LRowsPerSM = 4;

template <int PMAX, class V>
void run_lane_v(DevTree& t, const DevTree& s, const DevLists& L, int em, double eps, int be, int* p_used, int* stats,
                cudaStream_t st) {
  const size_t sm = lane_smem_bytes<PMAX, V>();
  note_launch();
  int dev = 0, n_sm = 0;
  FMM_CUDA_TRY(cudaGetDevice(&dev));
  FMM_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  if (L.n_m2l_targets < (int64_t)kWideM2LRowsPerSM * n_sm) {
    // few target rows (small problems, probe trees): kWideM2LWarps warps share each row
    constexpr int WW = kWideM2LWarps;
    FMM_CUDA_TRY(cudaFuncSetAttribute(k_m2l_lane<PMAX, V, WW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(WW * sm)));
    k_m2l_lane<PMAX, V, WW><<<(int)L.n_m2l_targets, 32 * WW, WW * sm, st>>>(
        L.m2l_tgt.ptr, L.m2l_off.ptr, L.m2l_s.ptr, t.local.ptr, s.multipole.ptr, t.tcenter.ptr, t.tbox.ptr,
        t.tradius.ptr, t.max_influence.ptr, s.scenter.ptr, em, eps, be, p_used, stats, stats + 1,
        reinterpret_cast<unsigned long long*>(stats + 2));
  } else {
    if (sm > 48 * 1024)
      FMM_CUDA_TRY(cudaFuncSetAttribute(k_m2l_lane<PMAX, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_m2l_lane<PMAX, V><<<(int)L.n_m2l_targets, 32, sm, st>>>(
        L.m2l_tgt.ptr, L.m2l_off.ptr, L.m2l_s.ptr, t.local.ptr, s.multipole.ptr, t.tcenter.ptr, t.tbox.ptr,
        t.tradius.ptr, t.max_influence.ptr, s.scenter.ptr, em, eps, be, p_used, stats, stats + 1,
        reinterpret_cast<unsigned long long*>(stats + 2));
  }
  FMM_CUDA_TRY(cudaGetLastError());
}

template <int PMAX>
void run_lane(DevTree& t, const DevTree& s, const DevLists& L, int em, double eps, int be, int* p_used, int* stats,
              int precision, cudaStream_t st) {
  if (precision == FMM_PRECISION_MIXED)
    run_lane_v<PMAX, float>(t, s, L, em, eps, be, p_used, stats, st);
  else
    run_lane_v<PMAX, double>(t, s, L, em, eps, be, p_used, stats, st);
}

// ---------------------------------------------------------------------------
// M2M and L2L with one lane per child (multipole_to_multipole!, src/translate.jl:
// 144-174; local_to_local!, :1896-1926): rotate_z -> rotate_y -> coaxial
// translation (translate_multipole_z!, :6-50; translate_local_z!, :1851-1891) ->
// rotate_y -> back_rotate_z, both rotations with the zeta set for M2M and the
// eta set for L2L, as the reference's chain does.

struct Geo {
  double cph, sph, cth, sth, r;
};
// cartesian_to_spherical (src/rotate.jl:9-21) in cos/sin form
__device__ __forceinline__ Geo geo_of(double x, double y, double z) {
  Geo g{1.0, 0.0, 1.0, 0.0, 0.0};
  const double x2y2 = x * x + y * y;
  const double r2 = x2y2 + z * z;
  g.r = (r2 == 0.0) ? r2 : sqrt(r2);
  if (x2y2 > 0) {
    const double rho = sqrt(x2y2);
    g.cph = x / rho;
    g.sph = y / rho;
    g.cth = z / g.r;
    g.sth = rho / g.r;
  } else {
    g.cth = (g.r > 0 && z < 0) ? -1.0 : 1.0;
  }
  return g;
}

// rotate_z of degree n of an interleaved expansion (set 0) into padded registers
template <int PMAX>
__device__ __forceinline__ void rotz_in(int n, bool on, const double* e, const Geo& g, double (&Xr)[PMAX + 1],
                                        double (&Xi)[PMAX + 1]) {
  double er = 1.0, ei = 0.0;
  const int base = hi(n, 0);
#pragma unroll
  for (int a = 0; a <= PMAX; ++a) {
    Xr[a] = Xi[a] = 0.0;
    if (a > n || !on) continue;
    const double2 u = __ldg(reinterpret_cast<const double2*>(e) + 2 * (base + a));
    Xr[a] = n == 0 ? u.x : u.x * er - u.y * ei;
    Xi[a] = n == 0 ? u.y : u.x * ei + u.y * er;
    const double t = er;
    er = er * g.cph - ei * g.sph;
    ei = t * g.sph + ei * g.cph;
  }
}

// back_rotate_z of degree n in place
template <int PMAX>
__device__ __forceinline__ void rotz_back(int n, const Geo& g, double (&Yr)[PMAX + 1], double (&Yi)[PMAX + 1]) {
  double er = 1.0, ei = 0.0;
#pragma unroll
  for (int m = 0; m <= PMAX; ++m) {
    if (m > n) break;
    const double cr = er, ci = -ei;
    const double vr = n == 0 ? Yr[m] : Yr[m] * cr - Yi[m] * ci;
    const double vi = n == 0 ? Yi[m] : Yr[m] * ci + Yi[m] * cr;
    Yr[m] = vr;
    Yi[m] = vi;
    const double t = er;
    er = er * g.cph - ei * g.sph;
    ei = t * g.sph + ei * g.cph;
  }
}

// M2M of one level: warp w takes parents l0 + 4 w .. + 3; lanes 8 g .. 8 g + 7 carry
// the children of parent l0 + 4 w + g; per degree the eight contributions are summed
// by shuffles and added to the parent by the group's first lane
template <int PMAX>
__global__ void __launch_bounds__(32) k_m2m_lane(int l0, int l1, const int* __restrict__ child_start,
                                                 const int* __restrict__ n_children,
                                                 const double* __restrict__ scen, double* __restrict__ M) {
  constexpr int NH = hi(PMAX + 1, 0);
  extern __shared__ double lane_smem[];
  double* Ms = lane_smem;  // [2 NH][32]
  const int lane = threadIdx.x, j = lane & 7;
  const int k = l0 + blockIdx.x * 4 + (lane >> 3);
  bool on = false;
  int c = 0;
  if (k < l1 && j < n_children[k]) {
    on = true;
    c = child_start[k] + j;
  }
  Geo g{1.0, 0.0, 1.0, 0.0, 0.0};
  if (on) g = geo_of(scen[3 * k] - scen[3 * c], scen[3 * k + 1] - scen[3 * c + 1], scen[3 * k + 2] - scen[3 * c + 2]);
  const double* src = M + (int64_t)4 * NH * c;
  double* dst = M + (int64_t)4 * NH * (k < l1 ? k : l0);
  const double mt = -g.r;
#pragma unroll 1
  for (int n = 0; n <= PMAX; ++n) {
    double Xr[PMAX + 1], Xi[PMAX + 1], Yr[PMAX + 1], Yi[PMAX + 1];
    rotz_in<PMAX>(n, on, src, g, Xr, Xi);
    rot_y<PMAX, false>(n, Xr, Xi, g.cth, g.sth, Yr, Yi);
#pragma unroll
    for (int m = 0; m <= PMAX; ++m) {
      if (m > n) break;
      MS(Ms, hi(n, m), 0, lane) = Yr[m];
      MS(Ms, hi(n, m), 1, lane) = Yi[m];
    }
    // translate_multipole_z!: out(n, m) = sum_{n' = n..m} (-t)^(n-n') / (n-n')! M(n', m); the
    // factor depends on n - n' only: source degrees outer (descending), orders inner
#pragma unroll
    for (int m = 0; m <= PMAX; ++m) Xr[m] = Xi[m] = 0.0;
    {
      double tp = 1.0;
#pragma unroll 1
      for (int np = n; np >= 0; --np) {
        const double cc = tp * c_ifact[n - np];  // (-t)^(n-n') / (n-n')!
        const int base = hi(np, 0);
#pragma unroll
        for (int m = 0; m <= PMAX; ++m) {
          if (m > np) break;
          Xr[m] += cc * MSr(Ms, base + m, 0, lane);
          Xi[m] += cc * MSr(Ms, base + m, 1, lane);
        }
        tp *= mt;
      }
    }
    rot_y<PMAX, false>(n, Xr, Xi, g.cth, g.sth, Yr, Yi);
    rotz_back<PMAX>(n, g, Yr, Yi);
#pragma unroll
    for (int m = 0; m <= PMAX; ++m) {
      if (m > n) break;
      double vr = on ? Yr[m] : 0.0, vi = on ? Yi[m] : 0.0;
      vr += __shfl_xor_sync(kAll, vr, 1);
      vi += __shfl_xor_sync(kAll, vi, 1);
      vr += __shfl_xor_sync(kAll, vr, 2);
      vi += __shfl_xor_sync(kAll, vi, 2);
      vr += __shfl_xor_sync(kAll, vr, 4);
      vi += __shfl_xor_sync(kAll, vi, 4);
      if (j == 0 && k < l1 && n_children[k] > 0) {
        dst[4 * hi(n, m)] += vr;
        dst[4 * hi(n, m) + 1] += vi;
      }
    }
  }
}

// L2L of one level: one lane per child c in [c0, c1), from its parent's local expansion
template <int PMAX>
__global__ void __launch_bounds__(32) k_l2l_lane(int c0, int c1, const int* __restrict__ parent,
                                                 const double* __restrict__ tcen, double* __restrict__ L) {
  constexpr int NH = hi(PMAX + 1, 0);
  extern __shared__ double lane_smem[];
  double* Ls = lane_smem;  // rotated parent local, [2 NH][32]
  const int lane = threadIdx.x;
  const int c = c0 + blockIdx.x * 32 + lane;
  const bool on = c < c1;
  int k = 0;
  Geo g{1.0, 0.0, 1.0, 0.0, 0.0};
  if (on) {
    k = parent[c];
    g = geo_of(tcen[3 * c] - tcen[3 * k], tcen[3 * c + 1] - tcen[3 * k + 1], tcen[3 * c + 2] - tcen[3 * k + 2]);
  }
  const double* src = L + (int64_t)4 * NH * k;
  double* dst = L + (int64_t)4 * NH * (on ? c : c0);
  const double mt = -g.r;
#pragma unroll 1
  for (int n = 0; n <= PMAX; ++n) {
    double Xr[PMAX + 1], Xi[PMAX + 1], Yr[PMAX + 1], Yi[PMAX + 1];
    rotz_in<PMAX>(n, on, src, g, Xr, Xi);
    rot_y<PMAX, true>(n, Xr, Xi, g.cth, g.sth, Yr, Yi);
#pragma unroll
    for (int m = 0; m <= PMAX; ++m) {
      if (m > n) break;
      MS(Ls, hi(n, m), 0, lane) = Yr[m];
      MS(Ls, hi(n, m), 1, lane) = Yi[m];
    }
  }
#pragma unroll 1
  for (int n = 0; n <= PMAX; ++n) {
    // translate_local_z!: out(n, m) = sum_{n' = n..P} (-t)^(n'-n) / (n'-n)! L(n', m); the
    // factor depends on n' - n only: source degrees outer, orders inner
    double Xr[PMAX + 1], Xi[PMAX + 1], Yr[PMAX + 1], Yi[PMAX + 1];
#pragma unroll
    for (int m = 0; m <= PMAX; ++m) Xr[m] = Xi[m] = 0.0;
    {
      double tp = 1.0;
#pragma unroll 1
      for (int np = n; np <= PMAX; ++np) {
        const double cc = tp * c_ifact[np - n];  // (-t)^(n'-n) / (n'-n)!
        const int base = hi(np, 0);
#pragma unroll
        for (int m = 0; m <= PMAX; ++m) {
          if (m > n) break;
          Xr[m] += cc * MSr(Ls, base + m, 0, lane);
          Xi[m] += cc * MSr(Ls, base + m, 1, lane);
        }
        tp *= mt;
      }
    }
    rot_y<PMAX, true>(n, Xr, Xi, g.cth, g.sth, Yr, Yi);
    rotz_back<PMAX>(n, g, Yr, Yi);
    if (on) {
#pragma unroll
      for (int m = 0; m <= PMAX; ++m) {
        if (m > n) break;
        dst[4 * hi(n, m)] += Yr[m];
        dst[4 * hi(n, m) + 1] += Yi[m];
      }
    }
  }
}

// Plain M2L at orders <= 3 (the influence estimate runs at order 3): one warp per
// target, one lane per pair, the whole rotated multipole and the lane's share of
// the target's local expansion in registers (every degree loop unrolled), the 32
// shares summed by shuffles once per target.
template <int P>
__global__ void __launch_bounds__(128) k_m2l_small(const int* __restrict__ tgt_list, const int* __restrict__ off,
                                                   const int* __restrict__ src_of, int n_targets,
                                                   double* __restrict__ local, const double* __restrict__ multipole,
                                                   const double* __restrict__ tcen, const double* __restrict__ scen,
                                                   int* __restrict__ p_used, int* __restrict__ st_pmax,
                                                   unsigned long long* __restrict__ st_flops) {
  constexpr int NH = hi(P + 1, 0);
  const int lane = threadIdx.x & 31;
  const int b = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (b >= n_targets) return;
  const int t = tgt_list[b];
  const double tc0 = tcen[3 * t], tc1 = tcen[3 * t + 1], tc2 = tcen[3 * t + 2];
  double accr[NH], acci[NH];
#pragma unroll
  for (int i = 0; i < NH; ++i) accr[i] = acci[i] = 0.0;
  const int l0 = off[b], l1 = off[b + 1];
  for (int l = l0 + lane; l < l1; l += 32) {
    const int s = src_of[l];
    const double* src = multipole + (int64_t)4 * NH * s;
    const Geo g = geo_of(tc0 - scen[3 * s], tc1 - scen[3 * s + 1], tc2 - scen[3 * s + 2]);
    const double rinv = 1 / g.r;
    double Mr[NH], Mi[NH];
#pragma unroll
    for (int n = 0; n <= P; ++n) {
      double Xr[P + 1], Xi[P + 1], Yr[P + 1], Yi[P + 1];
      rotz_in<P>(n, true, src, g, Xr, Xi);
      rot_y<P, false>(n, Xr, Xi, g.cth, g.sth, Yr, Yi);
#pragma unroll
      for (int m = 0; m <= n; ++m) {
        Mr[hi(n, m)] = Yr[m];
        Mi[hi(n, m)] = Yi[m];
      }
    }
    double un = rinv;  // n! / t^(n+1), the reference's product order
#pragma unroll
    for (int n = 0; n <= P; ++n) {
      if (n > 0) un *= n * rinv;
      double Xr[P + 1], Xi[P + 1], Yr[P + 1], Yi[P + 1];
      double cs = un;
#pragma unroll
      for (int m = 0; m <= P; ++m) {
        Xr[m] = Xi[m] = 0.0;
        if (m > n) continue;
        if (m > 0) cs *= (n + m) * rinv;
        double c = cs, vr = 0.0, vi = 0.0;
        int n_np = n + m;
#pragma unroll
        for (int np = m; np <= P; ++np) {
          vr += c * Mr[hi(np, m)];
          vi += c * Mi[hi(np, m)];
          n_np += 1;
          c *= n_np * rinv;
        }
        Xr[m] = vr;
        Xi[m] = vi;
      }
      rot_y<P, true>(n, Xr, Xi, g.cth, g.sth, Yr, Yi);
      rotz_back<P>(n, g, Yr, Yi);
#pragma unroll
      for (int m = 0; m <= n; ++m) {
        accr[hi(n, m)] += Yr[m];
        acci[hi(n, m)] += Yi[m];
      }
    }
    if (p_used) p_used[l] = P;
  }
#pragma unroll
  for (int i = 0; i < NH; ++i)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      accr[i] += __shfl_xor_sync(kAll, accr[i], o);
      acci[i] += __shfl_xor_sync(kAll, acci[i], o);
    }
  double* dst = local + (int64_t)4 * NH * t;
#pragma unroll
  for (int i = 0; i < NH; ++i)
    if ((i & 31) == lane) {
      dst[4 * i] += accr[i];
      dst[4 * i + 1] += acci[i];
    }
  if (lane == 0) {
    atomicMax(st_pmax, P);
    atomicAdd(st_flops, (unsigned long long)(l1 - l0) * lane_pair_flops(P));
  }
}

// Mixed-precision plain M2L at orders <= 3: the multipole is scaled by t^-n in FP64
// and rotated in FP32; the coaxial translation runs in FP32 with (n + n')!, giving the
// local coefficients times t^(n + 1), which are rotated back and accumulated in FP32
// relative to the separation t0 of the target's first pair, out(n) += Y(n) (t0 / t)^(n + 1)
// (the ratios stay far inside FP32 range); the lane shares are summed by shuffles and
// scaled by t0^-(n + 1) in FP64 once per target.
template <int P>
__global__ void __launch_bounds__(128) k_m2l_small_f(const int* __restrict__ tgt_list, const int* __restrict__ off,
                                                     const int* __restrict__ src_of, int n_targets,
                                                     double* __restrict__ local, const double* __restrict__ multipole,
                                                     const double* __restrict__ tcen, const double* __restrict__ scen,
                                                     int* __restrict__ p_used, int* __restrict__ st_pmax,
                                                     unsigned long long* __restrict__ st_flops) {
  constexpr int NH = hi(P + 1, 0);
  const int lane = threadIdx.x & 31;
  const int b = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (b >= n_targets) return;
  const int t = tgt_list[b];
  const double tc0 = tcen[3 * t], tc1 = tcen[3 * t + 1], tc2 = tcen[3 * t + 2];
  const int l0 = off[b], l1 = off[b + 1];
  double t0;
  {
    const int s = src_of[l0];
    const double x = tc0 - scen[3 * s], y = tc1 - scen[3 * s + 1], z = tc2 - scen[3 * s + 2];
    t0 = sqrt(x * x + y * y + z * z);
  }
  float accr[NH], acci[NH];
#pragma unroll
  for (int i = 0; i < NH; ++i) accr[i] = acci[i] = 0.f;
  for (int l = l0 + lane; l < l1; l += 32) {
    const int s = src_of[l];
    const double* src = multipole + (int64_t)4 * NH * s;
    const double xd = tc0 - scen[3 * s], yd = tc1 - scen[3 * s + 1], zd = tc2 - scen[3 * s + 2];
    const float x = (float)xd, y = (float)yd, z = (float)zd;
    const float rho2 = x * x + y * y, r2 = rho2 + z * z;
    const float rinv = rsqrtf(r2);
    float cph = 1.f, sph = 0.f, cth = z < 0.f ? -1.f : 1.f, sth = 0.f;
    if (rho2 > 0.f) {
      const float irho = rsqrtf(rho2);
      cph = x * irho;
      sph = y * irho;
      cth = z * rinv;
      sth = rho2 * irho * rinv;
    }
    const double tinv = (double)rinv;
    float Mr[NH], Mi[NH];
    double sn = 1.0;  // t^-n
#pragma unroll
    for (int n = 0; n <= P; ++n) {
      if (n > 0) sn *= tinv;
      float Xr[P + 1], Xi[P + 1], Yr[P + 1], Yi[P + 1];
      float er = 1.f, ei = 0.f;
#pragma unroll
      for (int a = 0; a <= P; ++a) {
        Xr[a] = Xi[a] = 0.f;
        if (a > n) continue;
        const double2 u = __ldg(reinterpret_cast<const double2*>(src) + 2 * (hi(n, 0) + a));
        const float ur = (float)(u.x * sn), ui = (float)(u.y * sn);
        Xr[a] = ur * er - ui * ei;
        Xi[a] = ur * ei + ui * er;
        const float tt = er;
        er = er * cph - ei * sph;
        ei = tt * sph + ei * cph;
      }
      rot_y<P, false, float>(n, Xr, Xi, cth, sth, Yr, Yi);
#pragma unroll
      for (int m = 0; m <= n; ++m) {
        Mr[hi(n, m)] = Yr[m];
        Mi[hi(n, m)] = Yi[m];
      }
    }
    const float q = (float)(t0 * tinv);
    float qn = 1.f;  // (t0 / t)^(n + 1)
#pragma unroll
    for (int n = 0; n <= P; ++n) {
      qn *= q;
      float Xr[P + 1], Xi[P + 1], Yr[P + 1], Yi[P + 1];
#pragma unroll
      for (int m = 0; m <= P; ++m) {
        Xr[m] = Xi[m] = 0.f;
        if (m > n) continue;
        float vr = 0.f, vi = 0.f;
#pragma unroll
        for (int np = m; np <= P; ++np) {
          const float c = c_factF[n + np];
          vr += c * Mr[hi(np, m)];
          vi += c * Mi[hi(np, m)];
        }
        Xr[m] = vr;
        Xi[m] = vi;
      }
      rot_y<P, true, float>(n, Xr, Xi, cth, sth, Yr, Yi);
      float er = 1.f, ei = 0.f;
#pragma unroll
      for (int m = 0; m <= n; ++m) {
        const float vr = Yr[m] * er + Yi[m] * ei;  // times e^{-i m phi}
        const float vi = Yi[m] * er - Yr[m] * ei;
        accr[hi(n, m)] += vr * qn;
        acci[hi(n, m)] += vi * qn;
        const float tt = er;
        er = er * cph - ei * sph;
        ei = tt * sph + ei * cph;
      }
    }
    if (p_used) p_used[l] = P;
  }
#pragma unroll
  for (int i = 0; i < NH; ++i)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      accr[i] += __shfl_xor_sync(kAll, accr[i], o);
      acci[i] += __shfl_xor_sync(kAll, acci[i], o);
    }
  double* dst = local + (int64_t)4 * NH * t;
  const double t0inv = 1.0 / t0;
  double sc = t0inv;  // t0^-(n + 1)
#pragma unroll
  for (int n = 0; n <= P; ++n) {
    if (n > 0) sc *= t0inv;
#pragma unroll
    for (int m = 0; m <= n; ++m) {
      const int i = hi(n, m);
      if ((i & 31) == lane) {
        dst[4 * i] += (double)accr[i] * sc;
        dst[4 * i + 1] += (double)acci[i] * sc;
      }
    }
  }
  if (lane == 0) {
    atomicMax(st_pmax, P);
    atomicAdd(st_flops, (unsigned long long)(l1 - l0) * lane_pair_flops(P));
  }
}

template <int P>
void run_m2l_small(DevTree& t, const DevTree& s, const DevLists& L, int* p_used, int* stats, int precision,
                   cudaStream_t st) {
  note_launch();
  const int g = (int)((L.n_m2l_targets + 3) / 4);
  auto* fl = reinterpret_cast<unsigned long long*>(stats + 2);
  if (precision == FMM_PRECISION_MIXED)
    k_m2l_small_f<P><<<g, 128, 0, st>>>(L.m2l_tgt.ptr, L.m2l_off.ptr, L.m2l_s.ptr, (int)L.n_m2l_targets, t.local.ptr,
                                        s.multipole.ptr, t.tcenter.ptr, s.scenter.ptr, p_used, stats, fl);
  else
    k_m2l_small<P><<<g, 128, 0, st>>>(L.m2l_tgt.ptr, L.m2l_off.ptr, L.m2l_s.ptr, (int)L.n_m2l_targets, t.local.ptr,
                                      s.multipole.ptr, t.tcenter.ptr, s.scenter.ptr, p_used, stats, fl);
  FMM_CUDA_TRY(cudaGetLastError());
}

template <int PMAX>
void run_m2m_lane(DevTree& s, cudaStream_t st) {
  const size_t sm = (size_t)2 * hi(PMAX + 1, 0) * 32 * sizeof(double);
  if (sm > 48 * 1024)
    FMM_CUDA_TRY(cudaFuncSetAttribute(k_m2m_lane<PMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  for (int l = s.n_levels - 2; l >= 0; --l) {
    const int l0 = (int)s.levels_start[l], l1 = (int)s.levels_end[l];
    if (l1 <= l0) continue;
    note_launch();
    k_m2m_lane<PMAX><<<(l1 - l0 + 3) / 4, 32, sm, st>>>(l0, l1, s.child_start.ptr, s.n_children.ptr, s.scenter.ptr,
                                                         s.multipole.ptr);
  }
  FMM_CUDA_TRY(cudaGetLastError());
}

template <int PMAX>
void run_l2l_lane(DevTree& t, cudaStream_t st) {
  const size_t sm = (size_t)2 * hi(PMAX + 1, 0) * 32 * sizeof(double);
  if (sm > 48 * 1024)
    FMM_CUDA_TRY(cudaFuncSetAttribute(k_l2l_lane<PMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  for (int l = 1; l < t.n_levels; ++l) {
    const int c0 = (int)t.levels_start[l], c1 = (int)t.levels_end[l];
    if (c1 <= c0) continue;
    note_launch();
    k_l2l_lane<PMAX><<<(c1 - c0 + 31) / 32, 32, sm, st>>>(c0, c1, t.parent.ptr, t.tcenter.ptr, t.local.ptr);
  }
  FMM_CUDA_TRY(cudaGetLastError());
}

template <class F>
void lane_dispatch(int p, F&& f) {
  switch (p) {
    case 1: f.template go<1>(); break;
    case 2: f.template go<2>(); break;
    case 3: f.template go<3>(); break;
    case 4: f.template go<4>(); break;
    case 5: f.template go<5>(); break;
    case 6: f.template go<6>(); break;
    case 7: f.template go<7>(); break;
    case 8: f.template go<8>(); break;
    case 9: f.template go<9>(); break;
    case 10: f.template go<10>(); break;
    case 11: f.template go<11>(); break;
    default: f.template go<12>(); break;
  }
}

struct M2MLaneGo {
  DevTree& s;
  cudaStream_t st;
  template <int P>
  void go() { run_m2m_lane<P>(s, st); }
};
struct L2LLaneGo {
  DevTree& t;
  cudaStream_t st;
  template <int P>
  void go() { run_l2l_lane<P>(t, st); }
};

// ---- Lamb-Helmholtz (vortex particle) plain M2L ---------------------------------
// One warp per target branch, two lanes per (target, source) pair: lanes 0-15 carry set 0
// (phi) and lanes 16-31 set 1 (chi) of the same 16 pairs, so each lane rotates, translates
// and rotates back one set.  Before the rotations (in V: FP32 on the mixed path, FP64 on the
// drop-in path) set 0 of the multipole is scaled by t^-n and set 1 by t^(1-n); the coaxial
// translation with (n+n')! then gives the local sets times t^(n+1) and t^(n+2), on which the
// Lamb-Helmholtz coupling of transform_lamb_helmholtz_local! (src/translate.jl:98-142) needs no
// power of t:
//   phi(n, m) -= i (m / n) chi(n, m),  chi(n, m) -= chi(n + 1, m) / (n + 1).
// The chi lane translates one degree ahead (it needs chi(n + 1)) and keeps chi(n) from the
// step before, which the phi lane reads across the warp (xor 16).  The rotated-back degrees are
// staged in shared memory unscaled (in V) with each lane's t^-(n+1) (phi) or t^-(n+2) (chi),
// and summed over the 16 pairs in FP64, value times power, into the warp's FP64 accumulator.
// One set per lane halves the registers and the shared memory a pair holds on a lane
// (order 12, FP32: 30 KB per warp, 7 warps per SM instead of 4 with a pair per lane).
template <int PMAX, class V>
constexpr size_t lane_lh_smem_bytes() {
  return ((size_t)4 * hi(PMAX + 1, 0) + 32) * sizeof(double) +
         ((size_t)4 * (PMAX + 1) * 17 + (size_t)2 * hi(PMAX + 1, 0) * 32) * sizeof(V);
}

// coaxial translation of the lane's set, degree n, orders m <= mmax, scaled:
// sum_{n'} (n+n')! M(n', m) (source degrees outer, orders inner: one degree's loads and FMAs
// are independent, each sum keeps its n'-ascending order)
template <int PMAX, class V>
__device__ __forceinline__ void coax_lh(int n, int mmax, int P, const V* Ms, int lane, V (&Xr)[PMAX + 1],
                                        V (&Xi)[PMAX + 1]) {
#pragma unroll
  for (int m = 0; m <= PMAX; ++m) Xr[m] = Xi[m] = V(0);
#pragma unroll 2
  for (int np = 0; np <= P; ++np) {
    const V c = sizeof(V) == 4 ? (V)c_factF[n + np] : (V)c_fact[n + np];
    const int base = hi(np, 0);
#pragma unroll
    for (int m = 0; m <= PMAX; ++m) {
      if (m > mmax || m > np) break;
      Xr[m] += c * Ms[(2 * (base + m)) * 32 + lane];
      Xi[m] += c * Ms[(2 * (base + m) + 1) * 32 + lane];
    }
  }
}

template <int PMAX, class V>
__global__ void __launch_bounds__(32) k_m2l_lane_lh(const int* __restrict__ tgt_list, const int* __restrict__ off,
                                                    const int* __restrict__ src_of, double* __restrict__ local,
                                                    const double* __restrict__ multipole,
                                                    const double* __restrict__ tcen, const double* __restrict__ scen,
                                                    int P, int* __restrict__ p_used, int* __restrict__ st_pmax,
                                                    unsigned long long* __restrict__ st_flops) {
  constexpr int NH = hi(PMAX + 1, 0);
  extern __shared__ double lane_smem[];
  double* acc = lane_smem;                    // [4 NH]
  double* tsc = acc + 4 * NH;                 // per pair t^-(n+1) (set 0), t^-(n+2) (set 1): [2][16]
  V* stage = reinterpret_cast<V*>(tsc + 32);  // unscaled rotated-back values [4 (PMAX+1)][17]
  V* Ms = stage + 4 * (PMAX + 1) * 17;        // rotated multipole of the lane's set [2 NH][32]
  const int lane = threadIdx.x;
  const int set = lane >> 4, slot = lane & 15;
  const int b = blockIdx.x;
  const int t = tgt_list[b];
  const double tc0 = tcen[3 * t], tc1 = tcen[3 * t + 1], tc2 = tcen[3 * t + 2];
  for (int i = lane; i < 4 * NH; i += 32) acc[i] = 0.0;
  const int l0 = off[b], l1 = off[b + 1];
  for (int lb = l0; lb < l1; lb += 16) {
    const int l = lb + slot;
    const bool valid = l < l1;
    const double* src = multipole;
    double cph = 1.0, sph = 0.0, cth = 1.0, sth = 0.0, r = 1.0, rinv = 1.0;
    if (valid) {
      const int s = src_of[l];
      src = multipole + (int64_t)4 * NH * s;
      const double x = tc0 - scen[3 * s], y = tc1 - scen[3 * s + 1], z = tc2 - scen[3 * s + 2];
      const double x2y2 = x * x + y * y;
      r = sqrt(x2y2 + z * z);
      if (x2y2 > 0) {
        const double rho = sqrt(x2y2);
        cph = x / rho;
        sph = y / rho;
        cth = z / r;
        sth = rho / r;
      } else {
        cth = z < 0 ? -1.0 : 1.0;
      }
      rinv = 1 / r;
      if (p_used && set == 0) p_used[l] = P;
    }
    const V fcph = (V)cph, fsph = (V)sph, fcth = (V)cth, fsth = (V)sth;
    // forward: the lane's set of every degree, scaled (t^-n, t^(1-n)) and rotated
    double sc = set ? r : 1.0;
#pragma unroll 1
    for (int n = 0; n <= P; ++n) {
      if (n > 0) sc *= rinv;
      V Xr[PMAX + 1], Xi[PMAX + 1];
      double er = 1.0, ei = 0.0;
      const int base = hi(n, 0);
#pragma unroll
      for (int a = 0; a <= PMAX; ++a) {
        Xr[a] = Xi[a] = V(0);
        if (a > n || !valid) continue;
        const double2 u = __ldg(reinterpret_cast<const double2*>(src) + 2 * (base + a) + set);
        Xr[a] = (V)((u.x * er - u.y * ei) * sc);
        Xi[a] = (V)((u.x * ei + u.y * er) * sc);
        const double tt = er;
        er = er * cph - ei * sph;
        ei = tt * sph + ei * cph;
      }
      V Yr[PMAX + 1], Yi[PMAX + 1];
      rot_y<PMAX, false, V>(n, Xr, Xi, fcth, fsth, Yr, Yi);
#pragma unroll
      for (int m = 0; m <= PMAX; ++m) {
        if (m > n) break;
        Ms[(2 * (base + m)) * 32 + lane] = Yr[m];
        Ms[(2 * (base + m) + 1) * 32 + lane] = Yi[m];
      }
    }
    __syncwarp();
    // back: the chi lane carries chi(n) (Cr, Ci) and translates chi(n + 1); the phi lane
    // translates phi(n) and reads chi(n) from its chi lane
    V Cr[PMAX + 1], Ci[PMAX + 1];
    coax_lh<PMAX, V>(0, 0, P, Ms, lane, Cr, Ci);
    double tn1 = rinv;  // t^-(n+1)
#pragma unroll 1
    for (int n = 0; n <= P; ++n) {
      if (n > 0) tn1 *= rinv;
      const int nd = n + set;  // degree the lane translates
      V Nr[PMAX + 1], Ni[PMAX + 1];
      if (nd <= P) {
        coax_lh<PMAX, V>(nd, n + 1, P, Ms, lane, Nr, Ni);
      } else {
#pragma unroll
        for (int m = 0; m <= PMAX; ++m) Nr[m] = Ni[m] = V(0);
      }
      V Xr[PMAX + 1], Xi[PMAX + 1], Yr[PMAX + 1], Yi[PMAX + 1];
      const V inv_n = n > 0 ? V(1) / (V)n : V(0);
      const V inv_n1 = V(1) / (V)(n + 1);
#pragma unroll
      for (int m = 0; m <= PMAX; ++m) {
        Xr[m] = Xi[m] = V(0);
        if (m > n) continue;
        const V pr = __shfl_xor_sync(kAll, Cr[m], 16), pi = __shfl_xor_sync(kAll, Ci[m], 16);
        if (set == 0) {  // phi(n, m) - i (m / n) chi(n, m)
          const V a = (V)m * inv_n;
          Xr[m] = Nr[m] - a * pi;
          Xi[m] = Ni[m] + a * pr;
        } else {  // chi(n, m) - chi(n + 1, m) / (n + 1)
          Xr[m] = Cr[m] - inv_n1 * Nr[m];
          Xi[m] = Ci[m] - inv_n1 * Ni[m];
        }
      }
      if (set) {  // chi(n + 1) is the next step's chi(n)
#pragma unroll
        for (int m = 0; m <= PMAX; ++m) {
          Cr[m] = Nr[m];
          Ci[m] = Ni[m];
        }
      }
      rot_y<PMAX, true, V>(n, Xr, Xi, fcth, fsth, Yr, Yi);
      V er = 1, ei = 0;
#pragma unroll
      for (int m = 0; m <= PMAX; ++m) {
        if (m > n) break;
        const V vr = Yr[m] * er + Yi[m] * ei;  // times e^{-i m phi}
        const V vi = Yi[m] * er - Yr[m] * ei;
        stage[(4 * m + 2 * set) * 17 + slot] = valid ? vr : V(0);
        stage[(4 * m + 2 * set + 1) * 17 + slot] = valid ? vi : V(0);
        const V tt = er;
        er = er * fcph - ei * fsph;
        ei = tt * fsph + ei * fcph;
      }
      tsc[lane] = set ? tn1 * rinv : tn1;
      __syncwarp();
      // 4 (n + 1) staged rows (order m, set, re/im), each value times its pair's power of t
      // in FP64 (set 0: t^-(n+1), set 1: t^-(n+2))
      for (int row = lane; row < 4 * (n + 1); row += 32) {
        const double* ts = tsc + ((row & 2) ? 16 : 0);
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < 16; ++k) v += (double)stage[row * 17 + k] * ts[k];
        acc[4 * hi(n, 0) + row] += v;
      }
      __syncwarp();
    }
    __syncwarp();
  }
  double* dst = local + (int64_t)4 * NH * t;
  for (int i = lane; i < 4 * NH; i += 32) dst[i] += acc[i];
  if (lane == 0) {
    atomicMax(st_pmax, P);
    atomicAdd(st_flops, (unsigned long long)(l1 - l0) * 2ull * lane_pair_flops(P));
  }
}

template <int PMAX, class V>
void run_m2l_lane_lh_v(DevTree& t, const DevTree& s, const DevLists& L, int P, int* p_used, int* stats,
                       cudaStream_t st) {
  constexpr size_t sm = lane_lh_smem_bytes<PMAX, V>();
  if (sm > 48 * 1024)
    FMM_CUDA_TRY(cudaFuncSetAttribute(k_m2l_lane_lh<PMAX, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  note_launch();
  k_m2l_lane_lh<PMAX, V><<<(int)L.n_m2l_targets, 32, sm, st>>>(
      L.m2l_tgt.ptr, L.m2l_off.ptr, L.m2l_s.ptr, t.local.ptr, s.multipole.ptr, t.tcenter.ptr, s.scenter.ptr, P,
      p_used, stats, reinterpret_cast<unsigned long long*>(stats + 2));
  FMM_CUDA_TRY(cudaGetLastError());
}
template <int PMAX>
void run_m2l_lane_lh(DevTree& t, const DevTree& s, const DevLists& L, int P, int* p_used, int* stats, int precision,
                     cudaStream_t st) {
  if (precision == FMM_PRECISION_MIXED)
    run_m2l_lane_lh_v<PMAX, float>(t, s, L, P, p_used, stats, st);
  else
    run_m2l_lane_lh_v<PMAX, double>(t, s, L, P, p_used, stats, st);
}

}  // namespace

bool launch_m2l_lane(DevTree& t, const DevTree& s, const DevLists& L, int p, bool lh, int em, double eps, int be,
                     int* p_used, int* stats, int precision, cudaStream_t st) {
  if (p < 1 || p > kLaneMaxP) return false;
  if (lh) {
    // vortex particles: the plain M2L from order 4 (orders <= 3 take the thread-per-pair
    // kernel, the error-controlled ones the general engine)
    if (em != FMM_ERROR_NONE || p < 4) return false;
    if (L.n_m2l_targets == 0) return true;
    ensure_lane_tables(st);
    switch (p) {
      case 4: run_m2l_lane_lh<4>(t, s, L, p, p_used, stats, precision, st); break;
      case 5: run_m2l_lane_lh<5>(t, s, L, p, p_used, stats, precision, st); break;
      case 6: run_m2l_lane_lh<6>(t, s, L, p, p_used, stats, precision, st); break;
      case 7: run_m2l_lane_lh<7>(t, s, L, p, p_used, stats, precision, st); break;
      case 8: run_m2l_lane_lh<8>(t, s, L, p, p_used, stats, precision, st); break;
      case 9: run_m2l_lane_lh<9>(t, s, L, p, p_used, stats, precision, st); break;
      case 10: run_m2l_lane_lh<10>(t, s, L, p, p_used, stats, precision, st); break;
      case 11: run_m2l_lane_lh<11>(t, s, L, p, p_used, stats, precision, st); break;
      default: run_m2l_lane_lh<12>(t, s, L, p, p_used, stats, precision, st); break;
    }
    return true;
  }
  if (L.n_m2l_targets == 0) return true;
  ensure_lane_tables(st);
  if (em == FMM_ERROR_NONE && p <= 3) {
    if (p == 1)
      run_m2l_small<1>(t, s, L, p_used, stats, precision, st);
    else if (p == 2)
      run_m2l_small<2>(t, s, L, p_used, stats, precision, st);
    else
      run_m2l_small<3>(t, s, L, p_used, stats, precision, st);
    return true;
  }
  switch (p) {
    case 1: run_lane<1>(t, s, L, em, eps, be, p_used, stats, precision, st); break;
    case 2: run_lane<2>(t, s, L, em, eps, be, p_used, stats, precision, st); break;
    case 3: run_lane<3>(t, s, L, em, eps, be, p_used, stats, precision, st); break;
    case 4: run_lane<4>(t, s, L, em, eps, be, p_used, stats, precision, st); break;
    case 5: run_lane<5>(t, s, L, em, eps, be, p_used, stats, precision, st); break;
    case 6: run_lane<6>(t, s, L, em, eps, be, p_used, stats, precision, st); break;
    case 7: run_lane<7>(t, s, L, em, eps, be, p_used, stats, precision, st); break;
    case 8: run_lane<8>(t, s, L, em, eps, be, p_used, stats, precision, st); break;
    case 9: run_lane<9>(t, s, L, em, eps, be, p_used, stats, precision, st); break;
    case 10: run_lane<10>(t, s, L, em, eps, be, p_used, stats, precision, st); break;
    case 11: run_lane<11>(t, s, L, em, eps, be, p_used, stats, precision, st); break;
    default: run_lane<12>(t, s, L, em, eps, be, p_used, stats, precision, st); break;
  }
  return true;
}

}  // namespace fmmb

namespace fmmb {

bool launch_m2m_lane(DevTree& s, int p, bool lh, cudaStream_t st) {
  if (lh || p < 1 || p > kLaneMaxP) return false;
  if (s.n_levels < 2) return true;
  ensure_lane_tables(st);
  lane_dispatch(p, M2MLaneGo{s, st});
  return true;
}

bool launch_l2l_lane(DevTree& t, int p, bool lh, cudaStream_t st) {
  // above order 6 the warp-per-child engine is faster (one rotation pair per child, no reduction)
  if (lh || p < 1 || p > 6) return false;
  if (t.n_levels < 2) return true;
  ensure_lane_tables(st);
  lane_dispatch(p, L2LLaneGo{t, st});
  return true;
}

}  // namespace fmmb

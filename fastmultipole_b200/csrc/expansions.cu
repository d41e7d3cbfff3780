// expansions.cu -- far-field kernels: P2M, M2M, M2L (plain and error-controlled),
// L2L and L2P, FP64, rotation-based ("point-and-shoot") operators.
//
// Every translation follows the reference's operator chain
//   rotate about z (e^{i m phi})  ->  rotate about y (Wigner d at theta, built
//   from the pi/2 table)  ->  coaxial translation along z  ->  [Lamb-Helmholtz
//   re-centring]  ->  rotate back about y  ->  rotate back about z and accumulate
// (src/translate.jl:144-174, 519-550, 1896-1926; src/rotate.jl).  One warp
// owns one output expansion (a target branch for M2L, a parent for M2M, a
// child for L2L), loops over its inputs, keeps the sum in registers (lane l
// holds coefficients l, l+32, ...) and writes once: no atomics.  Intermediate
// expansions, the Wigner matrices and e^{i m phi} live in the warp's slice of
// shared memory; the lanes split each stage over output coefficients
// (n, m), or over (m, m') for the Wigner entries, or over m for the
// column-recursive steps.
//
// Expansion layout: 4*Nh doubles per branch, e[4*i + 2*set + reim], i = n(n+1)/2 + m,
// set 0 = phi, set 1 = chi (Lamb-Helmholtz), as the reference's Tree.expansions.
#include "engine.cuh"
#include "pair_m2l.cuh"

namespace fmmb {

namespace {

constexpr int kWarps = 4;                      // warps per CTA
constexpr int kSlots = (231 + 31) / 32;        // nh(kMaxP) coefficients over 32 lanes
__host__ __device__ constexpr int hi_nm(int n, int m) { return n * (n + 1) / 2 + m; }

using eng::nm_of;
using eng::sph;

// P2M accumulator (lane l holds coefficients l + 32 k of both sets)
__device__ __forceinline__ void acc_zero(double (&acc)[kSlots][4]) {
#pragma unroll
  for (int k = 0; k < kSlots; ++k) acc[k][0] = acc[k][1] = acc[k][2] = acc[k][3] = 0.0;
}

__device__ __forceinline__ void acc_store_add(double* dst, const double (&acc)[kSlots][4], int P, bool lh) {
  int lane = threadIdx.x & 31;
  int NH = (P + 1) * (P + 2) / 2;
#pragma unroll
  for (int k = 0; k < kSlots; ++k) {
    int i = lane + 32 * k;
    if (i < NH) {
      dst[4 * i] += acc[k][0];
      dst[4 * i + 1] += acc[k][1];
      if (lh) {
        dst[4 * i + 2] += acc[k][2];
        dst[4 * i + 3] += acc[k][3];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// translation kernels (templated on SLOTS = ceil(Nh/32) and Lamb-Helmholtz)

using eng::Tab;
using eng::WS;
using eng::ws_doubles;
using eng::ws_of;

struct M2LStats {
  int* pmax;
  int* fail;
  unsigned long long* flops;
};

__device__ __forceinline__ unsigned long long m2l_pair_flops(int P, bool lh) {
  // 4 * [2 * sum_n (n+1)(2n+1) + sum_n sum_m (P-m+1)], x2 with Lamb-Helmholtz
  unsigned long long rot = 0, coax = 0;
  for (int n = 0; n <= P; ++n) {
    rot += (unsigned long long)(n + 1) * (2 * n + 1);
    for (int m = 0; m <= n; ++m) coax += (unsigned long long)(P - m + 1);
  }
  unsigned long long f = 4ull * (2 * rot + coax);
  return lh ? 2 * f : f;
}

template <int SLOTS, bool LH>
__global__ void __launch_bounds__(32 * kWarps) k_m2l(const int* __restrict__ tgt_list, const int* __restrict__ off,
                                                     const int* __restrict__ src_of, int n_targets,
                                                     double* __restrict__ local, const double* __restrict__ multipole,
                                                     const double* __restrict__ tcen, const double* __restrict__ tbox,
                                                     const double* __restrict__ trad,
                                                     const double* __restrict__ maxinf,
                                                     const double* __restrict__ scen, int p, int em, double eps,
                                                     int be, int* __restrict__ p_used, Tab tb, M2LStats stats) {
  extern __shared__ double smem[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.x * kWarps + wid;
  if (b >= n_targets) return;
  WS w = ws_of(smem + wid * ws_doubles(p), p);
  eng::SlotNM<SLOTS> L;
  L.init(w.NH);
  const int t = tgt_list[b];
  const int64_t NH4 = 4 * nh(p);
  eng::M2LGeom g;
  for (int d = 0; d < 3; ++d) {
    g.tc[d] = tcen[3 * t + d];
    g.tbox[d] = tbox[3 * t + d];
  }
  g.trad = trad[t];
  g.maxinf = maxinf[t];
  double acc[SLOTS][LH ? 4 : 2];
  eng::acc_zero<SLOTS, LH>(acc);
  int pmax = 0;
  bool all_ok = true;
  unsigned long long fl = 0;
  for (int l = off[b]; l < off[b + 1]; ++l) {
    int s = src_of[l];
    double sc[3] = {scen[3 * s], scen[3 * s + 1], scen[3 * s + 2]};
    bool ok;
    int P = eng::chain_m2l<SLOTS, LH>(w, acc, multipole + NH4 * s, sc, g, p, em, eps, be, ok, tb, L);
    if (p_used && lane == 0) p_used[l] = P;
    pmax = max(pmax, P);
    all_ok = all_ok && ok;
    fl += m2l_pair_flops(P, LH);
  }
  eng::acc_store_add<SLOTS, LH>(local + NH4 * t, acc, w.NH);
  if (lane == 0) {
    atomicMax(stats.pmax, pmax);
    if (!all_ok) atomicExch(stats.fail, 1);
    atomicAdd(stats.flops, fl);
  }
}

// M2L at orders <= 3 without error control: warp per target, lane per pair
// (thread-per-pair chain of pair_m2l.cuh), lane partials summed by shuffles
template <int P, bool LH>
__global__ void __launch_bounds__(32 * kWarps) k_m2l_pair(const int* __restrict__ tgt_list,
                                                          const int* __restrict__ off, const int* __restrict__ src_of,
                                                          int n_targets, double* __restrict__ local,
                                                          const double* __restrict__ multipole,
                                                          const double* __restrict__ tcen,
                                                          const double* __restrict__ scen, int* __restrict__ p_used,
                                                          Tab tb, M2LStats stats) {
  using K = eng::PairM2L<P, LH>;
  constexpr int NV = K::NH * K::NC;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.x * kWarps + wid;
  if (b >= n_targets) return;
  const int t = tgt_list[b];
  const int64_t NH4 = 4 * K::NH;
  const double tx = tcen[3 * t], ty = tcen[3 * t + 1], tz = tcen[3 * t + 2];
  double acc[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) acc[v] = 0.0;
  const int l0 = off[b], l1 = off[b + 1];
  for (int l = l0 + lane; l < l1; l += 32) {
    const int s = src_of[l];
    K::run(acc, multipole + NH4 * s, tx - scen[3 * s], ty - scen[3 * s + 1], tz - scen[3 * s + 2], tb);
    if (p_used) p_used[l] = P;
  }
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[v] += __shfl_xor_sync(0xffffffffu, acc[v], o);
  double* dst = local + NH4 * t;
#pragma unroll
  for (int v = 0; v < NV; ++v)
    if ((v & 31) == lane) dst[4 * (v / K::NC) + (v % K::NC)] += acc[v];
  if (lane == 0) {
    atomicMax(stats.pmax, P);
    atomicAdd(stats.flops, (unsigned long long)(l1 - l0) * m2l_pair_flops(P, LH));
  }
}

// M2M for one level: warp per parent, loop over its children
template <int SLOTS, bool LH>
__global__ void __launch_bounds__(32 * kWarps) k_m2m(int l0, int l1, const int* __restrict__ child_start,
                                                     const int* __restrict__ n_children,
                                                     const double* __restrict__ scen, double* __restrict__ M, int p,
                                                     Tab tb) {
  extern __shared__ double smem[];
  const int wid = threadIdx.x >> 5;
  const int k = l0 + blockIdx.x * kWarps + wid;
  if (k >= l1) return;
  int nc = n_children[k];
  if (nc == 0) return;
  WS w = ws_of(smem + wid * ws_doubles(p), p);
  eng::SlotNM<SLOTS> L;
  L.init(w.NH);
  const int64_t NH4 = 4 * nh(p);
  double acc[SLOTS][LH ? 4 : 2];
  eng::acc_zero<SLOTS, LH>(acc);
  int c0 = child_start[k];
  for (int c = c0; c < c0 + nc; ++c) {
    double dx = scen[3 * k] - scen[3 * c], dy = scen[3 * k + 1] - scen[3 * c + 1], dz = scen[3 * k + 2] - scen[3 * c + 2];
    eng::chain_mm_ll<SLOTS, LH>(w, acc, M + NH4 * c, dx, dy, dz, p, false, tb, L);
  }
  eng::acc_store_add<SLOTS, LH>(M + NH4 * k, acc, w.NH);
}

// L2L for one level: warp per child of a level-l parent
template <int SLOTS, bool LH>
__global__ void __launch_bounds__(32 * kWarps) k_l2l(int c0, int c1, const int* __restrict__ parent,
                                                     const double* __restrict__ tcen, double* __restrict__ Lx, int p,
                                                     Tab tb) {
  extern __shared__ double smem[];
  const int wid = threadIdx.x >> 5;
  const int c = c0 + blockIdx.x * kWarps + wid;
  if (c >= c1) return;
  WS w = ws_of(smem + wid * ws_doubles(p), p);
  eng::SlotNM<SLOTS> L;
  L.init(w.NH);
  const int64_t NH4 = 4 * nh(p);
  int k = parent[c];
  double acc[SLOTS][LH ? 4 : 2];
  eng::acc_zero<SLOTS, LH>(acc);
  double dx = tcen[3 * c] - tcen[3 * k], dy = tcen[3 * c + 1] - tcen[3 * k + 1], dz = tcen[3 * c + 2] - tcen[3 * k + 2];
  eng::chain_mm_ll<SLOTS, LH>(w, acc, Lx + NH4 * k, dx, dy, dz, p, true, tb, L);
  eng::acc_store_add<SLOTS, LH>(Lx + NH4 * c, acc, w.NH);
}

// unit operator: explicit pairs (target k <- source k)
template <int SLOTS, bool LH>
__global__ void __launch_bounds__(32 * kWarps) k_op_pairs(int64_t n, double* __restrict__ tgt,
                                                          const double* __restrict__ tc, const double* __restrict__ src,
                                                          const double* __restrict__ sc, int p, int local, Tab tb) {
  extern __shared__ double smem[];
  const int wid = threadIdx.x >> 5;
  const int64_t k = (int64_t)blockIdx.x * kWarps + wid;
  if (k >= n) return;
  WS w = ws_of(smem + wid * ws_doubles(p), p);
  eng::SlotNM<SLOTS> L;
  L.init(w.NH);
  const int64_t NH4 = 4 * nh(p);
  double acc[SLOTS][LH ? 4 : 2];
  eng::acc_zero<SLOTS, LH>(acc);
  eng::chain_mm_ll<SLOTS, LH>(w, acc, src + NH4 * k, tc[3 * k] - sc[3 * k], tc[3 * k + 1] - sc[3 * k + 1],
                              tc[3 * k + 2] - sc[3 * k + 2], p, local != 0, tb, L);
  eng::acc_store_add<SLOTS, LH>(tgt + NH4 * k, acc, w.NH);
}

template <int SLOTS, bool LH>
__global__ void __launch_bounds__(32 * kWarps) k_op_m2l(int64_t n, double* __restrict__ tgt,
                                                        const double* __restrict__ tc, const double* __restrict__ tbox,
                                                        const double* __restrict__ trad,
                                                        const double* __restrict__ maxinf,
                                                        const double* __restrict__ src, const double* __restrict__ sc,
                                                        int p, int em, double eps, int be, int* p_used, Tab tb) {
  extern __shared__ double smem[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t k = (int64_t)blockIdx.x * kWarps + wid;
  if (k >= n) return;
  WS w = ws_of(smem + wid * ws_doubles(p), p);
  eng::SlotNM<SLOTS> L;
  L.init(w.NH);
  const int64_t NH4 = 4 * nh(p);
  eng::M2LGeom g;
  for (int d = 0; d < 3; ++d) {
    g.tc[d] = tc[3 * k + d];
    g.tbox[d] = tbox ? tbox[3 * k + d] : 0.0;
  }
  g.trad = trad ? trad[k] : 0.0;
  g.maxinf = maxinf ? maxinf[k] : 0.0;
  double acc[SLOTS][LH ? 4 : 2];
  eng::acc_zero<SLOTS, LH>(acc);
  double s[3] = {sc[3 * k], sc[3 * k + 1], sc[3 * k + 2]};
  bool ok;
  int P = eng::chain_m2l<SLOTS, LH>(w, acc, src + NH4 * k, s, g, p, em, eps, be, ok, tb, L);
  if (p_used && lane == 0) p_used[k] = ok ? P : -P - 1;
  eng::acc_store_add<SLOTS, LH>(tgt + NH4 * k, acc, w.NH);
}

// call f.template go<SLOTS, LH>() for the instantiation matching (p, lh)
template <class F>
void dispatch_slots(int p, bool lh, F& f) {
  int slots = (int)((nh(p) + 31) / 32);
  switch (slots * 2 + (lh ? 1 : 0)) {
#define FMM_CASE(S)                 \
  case 2 * S:                       \
    f.template go<S, false>();      \
    break;                          \
  case 2 * S + 1:                   \
    f.template go<S, true>();       \
    break;
    FMM_CASE(1)
    FMM_CASE(2)
    FMM_CASE(3)
    FMM_CASE(4)
    FMM_CASE(5)
    FMM_CASE(6)
    FMM_CASE(7)
    FMM_CASE(8)
#undef FMM_CASE
    default:
      throw Error{FMM_ERR_ARGUMENT, "expansion order out of range"};
  }
}

// ---------------------------------------------------------------------------
// P2M: body_to_multipole! of Point{Source} / Point{Vortex}
// (src/bodytomultipole.jl:112-139, 283-334, 387-489).  The unit operator below
// uses one warp per expansion, lanes over m for the harmonics recursion and over
// (n, m) for the accumulation; the tree pass uses k_p2m_lane (lane per body).
__device__ __forceinline__ void q_nm1(const double* h, int n, int m, double _1_m, double* o) {
  int i = (n - 1) * n / 2 + m;  // index of (n-1, m)
  if (m > 0) {
    o[0] = h[2 * (i - 1)];
    o[1] = h[2 * (i - 1) + 1];
  } else if (n > 1) {
    o[0] = -_1_m * h[2 * (i + 1)];
    o[1] = _1_m * h[2 * (i + 1) + 1];
  } else {
    o[0] = o[1] = 0;
  }
  if (m < n) {
    o[2] = h[2 * i];
    o[3] = h[2 * i + 1];
  } else {
    o[2] = o[3] = 0;
  }
  if (m + 1 < n) {
    o[4] = h[2 * (i + 1)];
    o[5] = h[2 * (i + 1) + 1];
  } else {
    o[4] = o[5] = 0;
  }
}

__device__ __forceinline__ void q_n(const double* h, int n, int m, double _1_m, double* o) {
  int i = n * (n + 1) / 2 + m;
  if (m > 0) {
    o[0] = h[2 * (i - 1)];
    o[1] = h[2 * (i - 1) + 1];
  } else if (n == 0) {
    o[0] = o[1] = 0;
  } else {
    o[0] = -_1_m * h[2 * (i + 1)];
    o[1] = _1_m * h[2 * (i + 1) + 1];
  }
  o[2] = h[2 * i];
  o[3] = h[2 * i + 1];
  if (m < n) {
    o[4] = h[2 * (i + 1)];
    o[5] = h[2 * (i + 1) + 1];
  } else {
    o[4] = o[5] = 0;
  }
}

// calculate_q! with lanes over m; h holds 2 doubles per coefficient
__device__ __forceinline__ void calc_q(double* h, double xr, double xi, double er, double ei, double z, int P) {
  int lane = threadIdx.x & 31;
  if (lane == 0) {
    h[0] = 1.0;
    h[1] = 0.0;
  }
  __syncwarp();
  for (int n = 1; n <= P; ++n) {
    for (int m = lane; m <= n; m += 32) {
      double q[6];
      double _1_m = (m & 1) ? -1.0 : 1.0;
      q_nm1(h, n, m, _1_m, q);
      int i = n * (n + 1) / 2 + m;
      h[2 * i] = (-(xr * q[1] + xi * q[0]) - (er * q[5] + ei * q[4]) - z * q[2]) / n;
      h[2 * i + 1] = ((xr * q[0] - xi * q[1]) + (er * q[4] - ei * q[5]) - z * q[3]) / n;
    }
    __syncwarp();
  }
}

__device__ __forceinline__ void p2m_body(double (&acc)[kSlots][4], double* h, int kind, double dx, double dy, double dz,
                                         double4 s, int P) {
  const int lane = threadIdx.x & 31;
  const int NH = (P + 1) * (P + 2) / 2;
  if (kind == FMM_POINT_SOURCE) {
    calc_q(h, dx * 0.5, dy * 0.5, dx * 0.5, -(dy * 0.5), dz, P);
    double strength = -s.x;
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      int i = lane + 32 * k;
      if (i < NH) {
        int n, m;
        nm_of(i, n, m);
        double sg = ((n + m) & 1) ? -1.0 : 1.0;
        acc[k][0] += h[2 * i] * sg * strength;
        acc[k][1] -= h[2 * i + 1] * sg * strength;
      }
    }
  } else {
    double xr = -dx * 0.5, xi = -dy * 0.5;
    calc_q(h, xr, xi, xr, -xi, -dz, P);
    double vx = s.x, vy = s.y, vz = s.z;
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      int i = lane + 32 * k;
      if (i < NH) {
        int n, m;
        nm_of(i, n, m);
        double _1_m = (m & 1) ? -1.0 : 1.0;
        double q[6];
        q_n(h, n, m, _1_m, q);
        double a = (double)(n - m + 1) * 0.5, b = (double)(n + m + 1) * 0.5, _1_np1 = 1.0 / (n + 1);
        acc[k][0] += _1_m * ((-vx * q[0] + vy * q[1]) * a + (vx * q[4] + vy * q[5]) * b - vz * m * q[3]) * _1_np1;
        acc[k][1] += _1_m * ((vx * q[1] + vy * q[0]) * a + (-vx * q[5] + vy * q[4]) * b - vz * m * q[2]) * _1_np1;
        if (n >= 1) {
          double r[6];
          q_nm1(h, n, m, _1_m, r);
          double _1_over_n = 1.0 / n;
          acc[k][2] -= _1_m * _1_over_n * (0.5 * (-vy * r[0] - vx * r[1] + vy * r[4] - vx * r[5]) - vz * r[2]);
          acc[k][3] -= _1_m * _1_over_n * (0.5 * (vy * r[1] - vx * r[0] - vy * r[5] - vx * r[4]) + vz * r[3]);
        }
      }
    }
  }
  __syncwarp();
}

// P2M, one group of G lanes per leaf and one lane per body (G bodies at a time):
// each lane runs the regular-harmonic recurrence of calculate_q!
// (src/bodytomultipole.jl:112-139) for its body, degree n from degree n-1 in
// registers, forms the degree-n contributions of body_to_multipole! (source:
// :283-334, vortex: :387-489), and the group's contributions are summed into the
// leaf's multipole (the group owns the leaf: no atomics) -- column by column
// through shared memory for G = 32, by shuffles for G = 8 (leaves of a few bodies).
template <int PMAX, bool VORTEX, int G>
__global__ void __launch_bounds__(32 * kWarps) k_p2m_lane(const int* __restrict__ leaf_index, int n_leaves,
                                                          const int* __restrict__ body_start,
                                                          const int* __restrict__ body_count,
                                                          const double* __restrict__ scen,
                                                          const double4* __restrict__ pos,
                                                          const double4* __restrict__ str, double* __restrict__ M) {
  constexpr int NC = VORTEX ? 4 : 2;  // doubles per coefficient written
  constexpr int ROWS = NC * (PMAX + 1);
  extern __shared__ double smem[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31, gl = lane % G;
  const int w = (blockIdx.x * kWarps + wid) * (32 / G) + lane / G;
  if ((blockIdx.x * kWarps + wid) * (32 / G) >= n_leaves) return;  // the whole warp is past the end
  double* stage = smem + wid * ROWS * 33;
  const bool has = w < n_leaves;
  const int b = has ? leaf_index[w] : 0;
  const int s0 = has ? body_start[b] : 0, cnt = has ? body_count[b] : 0;
  const double cx = scen[3 * b], cy = scen[3 * b + 1], cz = scen[3 * b + 2];
  double* Mb = M + (int64_t)4 * ((PMAX + 1) * (PMAX + 2) / 2) * b;
  int cmax = cnt;  // every lane runs the same number of batches (the reductions are warp-wide)
  for (int o = 16; o > 0; o >>= 1) cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
  for (int j0 = 0; j0 < cmax; j0 += G) {
    const int j = j0 + gl;
    const bool valid = j < cnt;
    double dx = 0, dy = 0, dz = 0;
    double4 sv = make_double4(0, 0, 0, 0);
    if (valid) {
      const double4 x = pos[s0 + j];
      dx = x.x - cx;
      dy = x.y - cy;
      dz = x.z - cz;
      sv = str[s0 + j];
    }
    // calculate_q! arguments: source (dx/2, dy/2, dx/2, -dy/2, dz), vortex (-dx/2, -dy/2, -dx/2, dy/2, -dz)
    const double xr = VORTEX ? -dx * 0.5 : dx * 0.5, xi = VORTEX ? -dy * 0.5 : dy * 0.5;
    const double er = xr, ei = -xi, z = VORTEX ? -dz : dz;
    double Hr[PMAX + 1], Hi[PMAX + 1], Pr[PMAX + 1], Pi[PMAX + 1];
#pragma unroll
    for (int m = 0; m <= PMAX; ++m) Hr[m] = Hi[m] = Pr[m] = Pi[m] = 0.0;
    Hr[0] = 1.0;
#pragma unroll 1
    for (int n = 0; n <= PMAX; ++n) {
      if (n > 0) {
#pragma unroll
        for (int m = 0; m <= PMAX; ++m) {
          Pr[m] = Hr[m];
          Pi[m] = Hi[m];
        }
        // q_nm1: (n-1, m-1) [m = 0: -conj-mirror of (n-1, 1)], (n-1, m), (n-1, m+1); the
        // reference's division by n as a product with 1/n (one division per degree, not per
        // coefficient; within an ulp of the quotient)
        const double inv_n = 1.0 / n;
#pragma unroll
        for (int m = 0; m <= PMAX; ++m) {
          if (m > n) continue;
          double q0, q1;
          if (m > 0) {
            q0 = Pr[m > 0 ? m - 1 : 0];
            q1 = Pi[m > 0 ? m - 1 : 0];
          } else {
            q0 = n > 1 ? -Pr[1 % (PMAX + 1)] : 0.0;
            q1 = n > 1 ? Pi[1 % (PMAX + 1)] : 0.0;
          }
          const double q2 = m < n ? Pr[m] : 0.0, q3 = m < n ? Pi[m] : 0.0;
          const double q4 = (m + 1 <= PMAX && m + 1 < n) ? Pr[(m + 1) % (PMAX + 1)] : 0.0;
          const double q5 = (m + 1 <= PMAX && m + 1 < n) ? Pi[(m + 1) % (PMAX + 1)] : 0.0;
          Hr[m] = (-(xr * q1 + xi * q0) - (er * q5 + ei * q4) - z * q2) * inv_n;
          Hi[m] = ((xr * q0 - xi * q1) + (er * q4 - ei * q5) - z * q3) * inv_n;
        }
      }
      // degree-n contributions of this lane's body
#pragma unroll
      for (int m = 0; m <= PMAX; ++m) {
        if (m > n) continue;
        double v0, v1, v2 = 0, v3 = 0;
        const double _1_m = (m & 1) ? -1.0 : 1.0;
        if (!VORTEX) {
          const double sg = ((n + m) & 1) ? -1.0 : 1.0, strength = -sv.x;
          v0 = Hr[m] * sg * strength;
          v1 = -(Hi[m] * sg * strength);
        } else {
          // q_n: (n, m-1) [m = 0: mirror of (n, 1)], (n, m), (n, m+1)
          double q0, q1;
          if (m > 0) {
            q0 = Hr[m > 0 ? m - 1 : 0];
            q1 = Hi[m > 0 ? m - 1 : 0];
          } else {
            q0 = n > 0 ? -_1_m * Hr[1 % (PMAX + 1)] : 0.0;
            q1 = n > 0 ? _1_m * Hi[1 % (PMAX + 1)] : 0.0;
          }
          const double q2 = Hr[m], q3 = Hi[m];
          const double q4 = (m + 1 <= PMAX && m < n) ? Hr[(m + 1) % (PMAX + 1)] : 0.0;
          const double q5 = (m + 1 <= PMAX && m < n) ? Hi[(m + 1) % (PMAX + 1)] : 0.0;
          const double vx = sv.x, vy = sv.y, vz = sv.z;
          const double a = (double)(n - m + 1) * 0.5, bb = (double)(n + m + 1) * 0.5, _1_np1 = 1.0 / (n + 1);
          v0 = _1_m * ((-vx * q0 + vy * q1) * a + (vx * q4 + vy * q5) * bb - vz * m * q3) * _1_np1;
          v1 = _1_m * ((vx * q1 + vy * q0) * a + (-vx * q5 + vy * q4) * bb - vz * m * q2) * _1_np1;
          if (n >= 1) {
            double r0, r1;
            if (m > 0) {
              r0 = Pr[m > 0 ? m - 1 : 0];
              r1 = Pi[m > 0 ? m - 1 : 0];
            } else {
              r0 = n > 1 ? -_1_m * Pr[1 % (PMAX + 1)] : 0.0;
              r1 = n > 1 ? _1_m * Pi[1 % (PMAX + 1)] : 0.0;
            }
            const double r2 = m < n ? Pr[m] : 0.0, r3 = m < n ? Pi[m] : 0.0;
            const double r4 = (m + 1 <= PMAX && m + 1 < n) ? Pr[(m + 1) % (PMAX + 1)] : 0.0;
            const double r5 = (m + 1 <= PMAX && m + 1 < n) ? Pi[(m + 1) % (PMAX + 1)] : 0.0;
            const double _1_over_n = 1.0 / n;
            v2 = -(_1_m * _1_over_n * (0.5 * (-vy * r0 - vx * r1 + vy * r4 - vx * r5) - vz * r2));
            v3 = -(_1_m * _1_over_n * (0.5 * (vy * r1 - vx * r0 - vy * r5 - vx * r4) + vz * r3));
          }
        }
        if constexpr (G == 32) {
          stage[(NC * m) * 33 + lane] = valid ? v0 : 0.0;
          stage[(NC * m + 1) * 33 + lane] = valid ? v1 : 0.0;
          if (VORTEX) {
            stage[((NC * m + 2) % ROWS) * 33 + lane] = valid ? v2 : 0.0;
            stage[((NC * m + 3) % ROWS) * 33 + lane] = valid ? v3 : 0.0;
          }
        } else {
          double u[4] = {valid ? v0 : 0.0, valid ? v1 : 0.0, valid ? v2 : 0.0, valid ? v3 : 0.0};
#pragma unroll
          for (int c = 0; c < NC; ++c) {
#pragma unroll
            for (int o = 1; o < G; o <<= 1) u[c] += __shfl_xor_sync(0xffffffffu, u[c], o);
            if (gl == 0 && has) Mb[4 * hi_nm(n, m) + c] += u[c];
          }
        }
      }
      if constexpr (G == 32) {
        __syncwarp();
        const int hn = n * (n + 1) / 2;
        for (int v = lane; v < NC * (n + 1); v += 32) {
          double t = 0.0;
#pragma unroll 8
          for (int k = 0; k < 32; ++k) t += stage[v * 33 + k];
          Mb[4 * (hn + v / NC) + v % NC] += t;
        }
        __syncwarp();
      }
    }
  }
}

template <bool VORTEX>
struct P2MLaneLaunch {
  DevTree& s;
  cudaStream_t st;
  template <int PMAX, int G>
  void run() {
    constexpr size_t sm = G == 32 ? (size_t)kWarps * (VORTEX ? 4 : 2) * (PMAX + 1) * 33 * sizeof(double) : 0;
    if (sm > 48 * 1024)
      FMM_CUDA_TRY(cudaFuncSetAttribute(k_p2m_lane<PMAX, VORTEX, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sm));
    const int64_t per_cta = (int64_t)kWarps * (32 / G);
    int g = (int)((s.n_leaves + per_cta - 1) / per_cta);
    note_launch();
    k_p2m_lane<PMAX, VORTEX, G><<<g, 32 * kWarps, sm, st>>>(s.leaf_index.ptr, (int)s.n_leaves, s.body_start.ptr,
                                                              s.body_count.ptr, s.scenter.ptr, s.pos.ptr, s.str.ptr,
                                                              s.multipole.ptr);
    FMM_CUDA_TRY(cudaGetLastError());
  }
  template <int PMAX>
  void go() {
    // leaves of a few bodies (on average <= 8) take groups of 8 lanes, four leaves per warp
    if (s.n_bodies <= 8 * s.n_leaves)
      run<PMAX, 8>();
    else
      run<PMAX, 32>();
  }
};

template <class F>
void dispatch_order(int p, F& f) {
  switch (p) {
#define FMM_P(PP) \
  case PP:        \
    f.template go<PP>(); \
    break;
    FMM_P(0) FMM_P(1) FMM_P(2) FMM_P(3) FMM_P(4) FMM_P(5) FMM_P(6) FMM_P(7) FMM_P(8) FMM_P(9) FMM_P(10)
    FMM_P(11) FMM_P(12) FMM_P(13) FMM_P(14) FMM_P(15) FMM_P(16) FMM_P(17) FMM_P(18) FMM_P(19) FMM_P(20)
#undef FMM_P
    default:
      throw Error{FMM_ERR_ARGUMENT, "expansion order out of range"};
  }
}

__global__ void __launch_bounds__(32) k_op_p2m(const double4* __restrict__ pos, const double4* __restrict__ str,
                                               int64_t n, double cx, double cy, double cz, double* __restrict__ M,
                                               int p, int kind) {
  extern __shared__ double smem[];
  double acc[kSlots][4];
  acc_zero(acc);
  for (int64_t j = 0; j < n; ++j) {
    double4 x = pos[j];
    p2m_body(acc, smem, kind, x.x - cx, x.y - cy, x.z - cz, str[j], p);
  }
  acc_store_add(M, acc, p, kind == FMM_POINT_VORTEX);
}

// ---------------------------------------------------------------------------
// L2P: evaluate_local (src/evaluate_expansions.jl:45-399).  The coefficient
// combinations the reference forms per body (potential, the three velocity
// components and the nine gradient entries) depend only on the local
// expansion, so a CTA forms them once per leaf in shared memory; each thread
// then runs the regular-harmonic recursion (regular_harmonics!,
// src/harmonics.jl:13-58) for its body and contracts.
constexpr int kL2PThreads = 128;
constexpr int kCh = 13;  // channels: u, vx, vy, vz, h_xx..h_zz (column-major order)

// threads tid of nthr (the CTA, or a group of lanes of one warp when !cta) fill C
__device__ void l2p_coefficients(double* C, const double* __restrict__ L, int p, bool lh, bool ps, bool gs, bool hs,
                                 int tid, int nthr, bool cta) {
  // C[(ch * NH + i) * 2 + reim]
  const int NH = (p + 1) * (p + 2) / 2;
  for (int i = tid; i < NH; i += nthr) {
    int n, m;
    nm_of(i, n, m);
    double* c = C;
    // potential
    double ur = 0, ui = 0;
    if (ps && (n == 0 || !lh)) {
      ur = L[4 * i];
      ui = L[4 * i + 1];
    }
    c[(0 * NH + i) * 2] = ur;
    c[(0 * NH + i) * 2 + 1] = ui;
    double vxr = 0, vxi = 0, vyr = 0, vyi = 0, vzr = 0, vzi = 0;
    if (gs || hs) {
      if (m == 0) {
        if (n == 0 || n < p) {
          int a = i + n + 1, b2 = i + n + 2;
          vxr -= L[4 * b2 + 1];
          vyr -= L[4 * b2];
          vzr -= L[4 * a];
          vzi -= L[4 * a + 1];
        }
        if (lh && n > 0) {
          vxr += n * L[4 * (i + 1) + 2];
          vyr -= n * L[4 * (i + 1) + 3];
        }
      } else {
        if (n < p) {
          int am = i + n, a0 = i + n + 1, ap = i + n + 2;
          vxr -= (L[4 * am + 1] + L[4 * ap + 1]) * 0.5;
          vxi += (L[4 * am] + L[4 * ap]) * 0.5;
          vyr += (L[4 * am] - L[4 * ap]) * 0.5;
          vyi += (L[4 * am + 1] - L[4 * ap + 1]) * 0.5;
          vzr -= L[4 * a0];
          vzi -= L[4 * a0 + 1];
        }
        if (lh) {
          double cmr = L[4 * (i - 1) + 2], cmi = L[4 * (i - 1) + 3];
          vxr -= (n + m) * cmr * 0.5;
          vxi -= (n + m) * cmi * 0.5;
          vyr -= (n + m) * cmi * 0.5;
          vyi += (n + m) * cmr * 0.5;
          if (m < n) {
            double cpr = L[4 * (i + 1) + 2], cpi = L[4 * (i + 1) + 3];
            vxr += (n - m) * cpr * 0.5;
            vxi += (n - m) * cpi * 0.5;
            vyr -= (n - m) * cpi * 0.5;
            vyi += (n - m) * cpr * 0.5;
          }
          vzr += m * L[4 * i + 3];
          vzi -= m * L[4 * i + 2];
        }
      }
    }
    double V[6] = {vxr, vxi, vyr, vyi, vzr, vzi};
    for (int d = 0; d < 3; ++d) {
      c[((1 + d) * NH + i) * 2] = gs ? V[2 * d] : 0.0;
      c[((1 + d) * NH + i) * 2 + 1] = gs ? V[2 * d + 1] : 0.0;
    }
  }
  if (cta)
    __syncthreads();
  else
    __syncwarp();
  // hessian channels from the velocity coefficients ("gradient_n_m"), n <= p-1
  for (int i = tid; i < NH; i += nthr) {
    int n, m;
    nm_of(i, n, m);
    double h[9][2];
    for (int a = 0; a < 9; ++a) h[a][0] = h[a][1] = 0.0;
    if (hs && n <= p - 1) {
      // G(comp, idx): velocity coefficient comp of entry idx (stored in channels 1..3 when gs;
      // recomputed here from L when the gradient itself is not requested)
      auto G = [&](int comp, int idx, int reim) -> double {
        int nn, mm;
        nm_of(idx, nn, mm);
        double vr = 0, vi = 0;
        // same formulas as above for entry idx, component comp
        if (mm == 0) {
          if (nn == 0 || nn < p) {
            int a = idx + nn + 1, b2 = idx + nn + 2;
            if (comp == 0) vr -= L[4 * b2 + 1];
            if (comp == 1) vr -= L[4 * b2];
            if (comp == 2) {
              vr -= L[4 * a];
              vi -= L[4 * a + 1];
            }
          }
          if (lh && nn > 0) {
            if (comp == 0) vr += nn * L[4 * (idx + 1) + 2];
            if (comp == 1) vr -= nn * L[4 * (idx + 1) + 3];
          }
        } else {
          if (nn < p) {
            int am = idx + nn, a0 = idx + nn + 1, ap = idx + nn + 2;
            if (comp == 0) {
              vr -= (L[4 * am + 1] + L[4 * ap + 1]) * 0.5;
              vi += (L[4 * am] + L[4 * ap]) * 0.5;
            } else if (comp == 1) {
              vr += (L[4 * am] - L[4 * ap]) * 0.5;
              vi += (L[4 * am + 1] - L[4 * ap + 1]) * 0.5;
            } else {
              vr -= L[4 * a0];
              vi -= L[4 * a0 + 1];
            }
          }
          if (lh) {
            double cmr = L[4 * (idx - 1) + 2], cmi = L[4 * (idx - 1) + 3];
            if (comp == 0) {
              vr -= (nn + mm) * cmr * 0.5;
              vi -= (nn + mm) * cmi * 0.5;
            } else if (comp == 1) {
              vr -= (nn + mm) * cmi * 0.5;
              vi += (nn + mm) * cmr * 0.5;
            }
            if (mm < nn) {
              double cpr = L[4 * (idx + 1) + 2], cpi = L[4 * (idx + 1) + 3];
              if (comp == 0) {
                vr += (nn - mm) * cpr * 0.5;
                vi += (nn - mm) * cpi * 0.5;
              } else if (comp == 1) {
                vr -= (nn - mm) * cpi * 0.5;
                vi += (nn - mm) * cpr * 0.5;
              }
            }
            if (comp == 2) {
              vr += mm * L[4 * idx + 3];
              vi -= mm * L[4 * idx + 2];
            }
          }
        }
        return reim ? vi : vr;
      };
      for (int col = 0; col < 3; ++col) {
        if (m == 0) {
          int ap = i + n + 2, a0 = i + n + 1;
          h[3 * col + 0][0] = -G(col, ap, 1);
          h[3 * col + 1][0] = -G(col, ap, 0);
          h[3 * col + 2][0] = -G(col, a0, 0);
          h[3 * col + 2][1] = -G(col, a0, 1);
        } else {
          int am = i + n, a0 = i + n + 1, ap = i + n + 2;
          h[3 * col + 0][0] = -(G(col, am, 1) + G(col, ap, 1)) * 0.5;
          h[3 * col + 0][1] = (G(col, am, 0) + G(col, ap, 0)) * 0.5;
          h[3 * col + 1][0] = (G(col, am, 0) - G(col, ap, 0)) * 0.5;
          h[3 * col + 1][1] = (G(col, am, 1) - G(col, ap, 1)) * 0.5;
          h[3 * col + 2][0] = -G(col, a0, 0);
          h[3 * col + 2][1] = -G(col, a0, 1);
        }
      }
    }
    // channel 4 + (row + 3*col) for the SMatrix(vxx, vxy, vxz, vyx, ...) order:
    // entry (row r = x|y|z of velocity, col c = derivative direction): vrc at 4 + 3*r + c
    for (int col = 0; col < 3; ++col)
      for (int row = 0; row < 3; ++row) {
        int ch = 4 + 3 * row + col;
        C[(ch * NH + i) * 2] = h[3 * col + row][0];
        C[(ch * NH + i) * 2 + 1] = h[3 * col + row][1];
      }
  }
  if (cta)
    __syncthreads();
  else
    __syncwarp();
}

// 1/k for the body-wise recursions (k <= 2 kMaxP + 1): a product with 1/k in place of the
// division by k in the hot loops (within an ulp of the quotient)
__constant__ double c_rcp[42] = {
    0.0, 1.0 / 1, 1.0 / 2, 1.0 / 3, 1.0 / 4, 1.0 / 5, 1.0 / 6, 1.0 / 7, 1.0 / 8, 1.0 / 9, 1.0 / 10, 1.0 / 11,
    1.0 / 12, 1.0 / 13, 1.0 / 14, 1.0 / 15, 1.0 / 16, 1.0 / 17, 1.0 / 18, 1.0 / 19, 1.0 / 20, 1.0 / 21,
    1.0 / 22, 1.0 / 23, 1.0 / 24, 1.0 / 25, 1.0 / 26, 1.0 / 27, 1.0 / 28, 1.0 / 29, 1.0 / 30, 1.0 / 31,
    1.0 / 32, 1.0 / 33, 1.0 / 34, 1.0 / 35, 1.0 / 36, 1.0 / 37, 1.0 / 38, 1.0 / 39, 1.0 / 40, 1.0 / 41};

// contract one body: regular harmonics by the reference's column recursion
__device__ void l2p_body(const double* C, int p, double x, double y, double z, bool ps, bool gs, bool hs, double* out) {
  const int NH = (p + 1) * (p + 2) / 2;
  // cos and sin of the polar angle and e^{i (phi + pi/2)} of cartesian_to_spherical
  // (src/rotate.jl:9-21) straight from the offsets, without forming the angles (the same
  // values up to rounding; on the z axis exact 0 where the trigonometric route leaves ~1e-16)
  const double x2y2 = x * x + y * y;
  const double r2 = x2y2 + z * z;
  const double r = (r2 == 0.0) ? r2 : sqrt(r2);
  double cx = 1.0, sy = 0.0, iei_r = 0.0, iei_i = 1.0;
  if (r > 0) {
    if (x2y2 > 0) {
      const double rho = sqrt(x2y2);
      cx = z / r;
      sy = rho / r;
      iei_r = -y / rho;
      iei_i = x / rho;
    } else {
      cx = z < 0 ? -1.0 : 1.0;
    }
  }
  double fact = 1.0, pn = 1.0, rhom = 1.0;
  double er = 1.0, ei = 0.0;
  double a[kCh];
  for (int c = 0; c < kCh; ++c) a[c] = 0.0;
  const int nch = hs ? kCh : 4;
  for (int m = 0; m <= p; ++m) {
    double pl = pn;
    double rhon = rhom;
    double p1 = pl, p2 = 0;
    double wgt = (m == 0) ? 1.0 : 2.0;
    for (int n = m; n <= p; ++n) {
      double R;
      if (n == m) {
        R = rhom * pl;
      } else {
        rhon *= -c_rcp[n + m];
        R = rhon * pl;
      }
      double Rr = R * er, Ri = R * ei;
      int i = n * (n + 1) / 2 + m;
      for (int c = 0; c < nch; ++c) {
        double cr = C[(c * NH + i) * 2], ci = C[(c * NH + i) * 2 + 1];
        a[c] += wgt * (Rr * cr - Ri * ci);
      }
      // Legendre recursion
      if (n == m) {
        p1 = pl;
        pl = cx * (2 * m + 1) * p1;
        rhom *= r;
        rhon = rhom;
      } else {
        p2 = p1;
        p1 = pl;
        pl = (cx * (2 * n + 1) * p1 - (n + m) * p2) * c_rcp[n - m + 1];
        rhon *= r;
      }
    }
    rhom /= -(2 * m + 2) * (2 * m + 1);
    pn = -pn * fact * sy;
    fact += 2;
    double tr = er, ti = ei;
    er = tr * iei_r - ti * iei_i;
    ei = tr * iei_i + ti * iei_r;
  }
  if (ps) out[0] += -a[0] * kOneOver4Pi;
  if (gs) {
    out[1] += a[1] * kOneOver4Pi;
    out[2] += a[2] * kOneOver4Pi;
    out[3] += a[3] * kOneOver4Pi;
  }
  if (hs)
    for (int c = 4; c < kCh; ++c) out[c] += a[c] * kOneOver4Pi;
}

__global__ void __launch_bounds__(kL2PThreads) k_l2p(const int* __restrict__ leaf_index,
                                                     const int* __restrict__ body_start,
                                                     const int* __restrict__ body_count,
                                                     const double* __restrict__ tcen, const double4* __restrict__ pos,
                                                     const double* __restrict__ L, int p, int lh, int ps, int gs, int hs,
                                                     double* __restrict__ acc13) {
  extern __shared__ double C[];
  const int b = leaf_index[blockIdx.x];
  l2p_coefficients(C, L + 4 * nh(p) * b, p, lh != 0, ps != 0, gs != 0, hs != 0, threadIdx.x, blockDim.x, true);
  const int s0 = body_start[b], cnt = body_count[b];
  const double cx = tcen[3 * b], cy = tcen[3 * b + 1], cz = tcen[3 * b + 2];
  for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
    double4 x = pos[s0 + j];
    l2p_body(C, p, x.x - cx, x.y - cy, x.z - cz, ps != 0, gs != 0, hs != 0, acc13 + 13 * (int64_t)(s0 + j));
  }
}

// leaves of a few bodies: a group of 8 lanes per leaf, 16 leaves per CTA of 128 threads,
// each group with its own coefficients in shared memory
constexpr int kL2PGroup = 8, kL2PGroupThreads = 128;
__global__ void __launch_bounds__(kL2PGroupThreads) k_l2p_group(const int* __restrict__ leaf_index, int n_leaves,
                                                               const int* __restrict__ body_start,
                                                               const int* __restrict__ body_count,
                                                               const double* __restrict__ tcen,
                                                               const double4* __restrict__ pos,
                                                               const double* __restrict__ L, int p, int lh, int ps,
                                                               int gs, int hs, double* __restrict__ acc13) {
  extern __shared__ double Cg[];
  const int g = threadIdx.x / kL2PGroup, lane = threadIdx.x % kL2PGroup;
  const int leaf = blockIdx.x * (kL2PGroupThreads / kL2PGroup) + g;
  const bool valid = leaf < n_leaves;  // groups past the end repeat the last leaf and write nothing
  const int b = leaf_index[valid ? leaf : n_leaves - 1];
  double* C = Cg + (size_t)g * kCh * 2 * nh(p);
  l2p_coefficients(C, L + 4 * nh(p) * b, p, lh != 0, ps != 0, gs != 0, hs != 0, lane, kL2PGroup, false);
  if (!valid) return;
  const int s0 = body_start[b], cnt = body_count[b];
  const double cx = tcen[3 * b], cy = tcen[3 * b + 1], cz = tcen[3 * b + 2];
  for (int j = lane; j < cnt; j += kL2PGroup) {
    double4 x = pos[s0 + j];
    l2p_body(C, p, x.x - cx, x.y - cy, x.z - cz, ps != 0, gs != 0, hs != 0, acc13 + 13 * (int64_t)(s0 + j));
  }
}

__global__ void __launch_bounds__(kL2PThreads) k_op_l2p(int64_t n, const double* __restrict__ dx,
                                                        const double* __restrict__ L, int p, int lh, int ps, int gs,
                                                        int hs, double* __restrict__ out13) {
  extern __shared__ double C[];
  l2p_coefficients(C, L, p, lh != 0, ps != 0, gs != 0, hs != 0, threadIdx.x, blockDim.x, true);
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    l2p_body(C, p, dx[3 * j], dx[3 * j + 1], dx[3 * j + 2], ps != 0, gs != 0, hs != 0, out13 + 13 * j);
}

inline size_t pair_smem(int p) { return (size_t)kWarps * ws_doubles(p) * sizeof(double); }
inline size_t l2p_smem(int p) { return (size_t)kCh * 2 * nh(p) * sizeof(double); }

template <class K>
void allow_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) FMM_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

Tab tab_of(const DevTables& t) { return Tab{t.Hs.ptr, t.zeta.ptr, t.eta.ptr, t.Mt.ptr, t.Lt.ptr}; }

}  // namespace

void upload_tables(DevTables& dt, int p, cudaStream_t st) {
  if (dt.p >= p && dt.p >= kMaxP) return;
  HostTables h;
  build_tables(h, p);
  dt.Hs.grow(h.Hs.size());
  dt.zeta.grow(h.zeta.size());
  dt.eta.grow(h.eta.size());
  dt.Mt.grow(h.Mt.size());
  dt.Lt.grow(h.Lt.size());
  FMM_CUDA_TRY(cudaMemcpyAsync(dt.Hs.ptr, h.Hs.data(), h.Hs.size() * 8, cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaMemcpyAsync(dt.zeta.ptr, h.zeta.data(), h.zeta.size() * 8, cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaMemcpyAsync(dt.eta.ptr, h.eta.data(), h.eta.size() * 8, cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaMemcpyAsync(dt.Mt.ptr, h.Mt.data(), h.Mt.size() * 8, cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaMemcpyAsync(dt.Lt.ptr, h.Lt.data(), h.Lt.size() * 8, cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaStreamSynchronize(st));
  dt.p = h.p;
}

void launch_p2m(DevTree& s, int p, int kind, const DevTables&, cudaStream_t st) {
  if (s.n_leaves == 0) return;
  if (kind == FMM_POINT_VORTEX) {
    P2MLaneLaunch<true> f{s, st};
    dispatch_order(p, f);
  } else {
    P2MLaneLaunch<false> f{s, st};
    dispatch_order(p, f);
  }
}

namespace {
struct M2MLaunch {
  DevTree& s;
  int p;
  Tab tb;
  cudaStream_t st;
  template <int S, bool LH>
  void go() {
    size_t sm = pair_smem(p);
    allow_smem(k_m2m<S, LH>, sm);
    for (int l = s.n_levels - 2; l >= 0; --l) {
      int l0 = (int)s.levels_start[l], l1 = (int)s.levels_end[l];
      int g = (l1 - l0 + kWarps - 1) / kWarps;
      note_launch();
      k_m2m<S, LH><<<g, 32 * kWarps, sm, st>>>(l0, l1, s.child_start.ptr, s.n_children.ptr, s.scenter.ptr,
                                               s.multipole.ptr, p, tb);
    }
    FMM_CUDA_TRY(cudaGetLastError());
  }
};

struct M2LLaunch {
  DevTree& t;
  const DevTree& s;
  const DevLists& L;
  int p, em, be;
  double eps;
  int* p_used;
  M2LStats S;
  Tab tb;
  cudaStream_t st;
  template <int SL, bool LH>
  void go() {
    size_t sm = pair_smem(p);
    allow_smem(k_m2l<SL, LH>, sm);
    int g = (int)((L.n_m2l_targets + kWarps - 1) / kWarps);
    note_launch();
    k_m2l<SL, LH><<<g, 32 * kWarps, sm, st>>>(L.m2l_tgt.ptr, L.m2l_off.ptr, L.m2l_s.ptr, (int)L.n_m2l_targets,
                                              t.local.ptr, s.multipole.ptr, t.tcenter.ptr, t.tbox.ptr, t.tradius.ptr,
                                              t.max_influence.ptr, s.scenter.ptr, p, em, eps, be, p_used, tb, S);
    FMM_CUDA_TRY(cudaGetLastError());
  }
};

struct L2LLaunch {
  DevTree& t;
  int p;
  Tab tb;
  cudaStream_t st;
  template <int S, bool LH>
  void go() {
    size_t sm = pair_smem(p);
    allow_smem(k_l2l<S, LH>, sm);
    for (int l = 1; l < t.n_levels; ++l) {
      int c0 = (int)t.levels_start[l], c1 = (int)t.levels_end[l];
      int g = (c1 - c0 + kWarps - 1) / kWarps;
      note_launch();
      k_l2l<S, LH><<<g, 32 * kWarps, sm, st>>>(c0, c1, t.parent.ptr, t.tcenter.ptr, t.local.ptr, p, tb);
    }
    FMM_CUDA_TRY(cudaGetLastError());
  }
};

struct OpPairsLaunch {
  int64_t n;
  double* target;
  const double *tc, *src, *sc;
  int p;
  bool local;
  Tab tb;
  cudaStream_t st;
  template <int S, bool LH>
  void go() {
    size_t sm = pair_smem(p);
    allow_smem(k_op_pairs<S, LH>, sm);
    note_launch();
    k_op_pairs<S, LH><<<(int)((n + kWarps - 1) / kWarps), 32 * kWarps, sm, st>>>(n, target, tc, src, sc, p,
                                                                                 local ? 1 : 0, tb);
    FMM_CUDA_TRY(cudaGetLastError());
  }
};

struct OpM2LLaunch {
  int64_t n;
  double* target;
  const double *tc, *tbox, *trad, *maxinf, *src, *sc;
  int p, em, be;
  double eps;
  int* p_used;
  Tab tb;
  cudaStream_t st;
  template <int S, bool LH>
  void go() {
    size_t sm = pair_smem(p);
    allow_smem(k_op_m2l<S, LH>, sm);
    note_launch();
    k_op_m2l<S, LH><<<(int)((n + kWarps - 1) / kWarps), 32 * kWarps, sm, st>>>(n, target, tc, tbox, trad, maxinf,
                                                                               src, sc, p, em, eps, be, p_used, tb);
    FMM_CUDA_TRY(cudaGetLastError());
  }
};
}  // namespace

void launch_m2m(DevTree& s, int p, bool lh, const DevTables& tb, cudaStream_t st) {
  if (launch_m2m_lane(s, p, lh, st)) return;
  M2MLaunch f{s, p, tab_of(tb), st};
  dispatch_slots(p, lh, f);
}

void launch_m2l(DevTree& t, const DevTree& s, const DevLists& L, int p, bool lh, int em, double eps, int be,
                int* p_used, int* stats, const DevTables& tb, int precision, cudaStream_t st) {
  if (L.n_m2l_targets == 0) return;
  // stats: [0] = max order used, [1] = any tolerance missed, [2..3] = flop count (u64)
  M2LStats S{stats, stats + 1, reinterpret_cast<unsigned long long*>(stats + 2)};
  if (lh && em == FMM_ERROR_NONE && p >= 1 && p <= 3) {
    int g = (int)((L.n_m2l_targets + kWarps - 1) / kWarps);
    Tab T = tab_of(tb);
    note_launch();
#define FMM_M2L_PAIR(PP, LL)                                                                                   \
  k_m2l_pair<PP, LL><<<g, 32 * kWarps, 0, st>>>(L.m2l_tgt.ptr, L.m2l_off.ptr, L.m2l_s.ptr, (int)L.n_m2l_targets, \
                                                t.local.ptr, s.multipole.ptr, t.tcenter.ptr, s.scenter.ptr, p_used, T, S)
    if (lh) {
      if (p == 1) FMM_M2L_PAIR(1, true);
      else if (p == 2) FMM_M2L_PAIR(2, true);
      else FMM_M2L_PAIR(3, true);
    } else {
      if (p == 1) FMM_M2L_PAIR(1, false);
      else if (p == 2) FMM_M2L_PAIR(2, false);
      else FMM_M2L_PAIR(3, false);
    }
#undef FMM_M2L_PAIR
    FMM_CUDA_TRY(cudaGetLastError());
    return;
  }
  if (launch_m2l_lane(t, s, L, p, lh, em, eps, be, p_used, stats, precision, st)) return;
  M2LLaunch f{t, s, L, p, em, be, eps, p_used, S, tab_of(tb), st};
  dispatch_slots(p, lh, f);
}

void launch_l2l(DevTree& t, int p, bool lh, const DevTables& tb, cudaStream_t st) {
  if (launch_l2l_lane(t, p, lh, st)) return;
  L2LLaunch f{t, p, tab_of(tb), st};
  dispatch_slots(p, lh, f);
}

void launch_l2p(DevTree& t, int p, bool lh, bool ps, bool gs, bool hs, double* acc13, cudaStream_t st) {
  if (t.n_leaves == 0) return;
  size_t sm = l2p_smem(p);
  note_launch();
  const bool small = t.n_bodies <= 8 * t.n_leaves;
  const size_t smg = (kL2PGroupThreads / kL2PGroup) * sm;
  if (small && smg <= 96 * 1024) {
    // leaves of a few bodies (on average <= 8), low orders: 8 lanes each, 16 per CTA
    allow_smem(k_l2p_group, smg);
    const int per = kL2PGroupThreads / kL2PGroup;
    k_l2p_group<<<(int)((t.n_leaves + per - 1) / per), kL2PGroupThreads, smg, st>>>(
        t.leaf_index.ptr, (int)t.n_leaves, t.body_start.ptr, t.body_count.ptr, t.tcenter.ptr, t.pos.ptr, t.local.ptr,
        p, lh ? 1 : 0, ps ? 1 : 0, gs ? 1 : 0, hs ? 1 : 0, acc13);
  } else {
    allow_smem(k_l2p, sm);
    k_l2p<<<(int)t.n_leaves, small ? 32 : kL2PThreads, sm, st>>>(t.leaf_index.ptr, t.body_start.ptr, t.body_count.ptr,
                                                     t.tcenter.ptr, t.pos.ptr, t.local.ptr, p, lh ? 1 : 0, ps ? 1 : 0,
                                                     gs ? 1 : 0, hs ? 1 : 0, acc13);
  }
  FMM_CUDA_TRY(cudaGetLastError());
}

void launch_op_m2m(int64_t n, double* target, const double* tc, const double* src, const double* sc, int p, bool lh,
                   bool local, const DevTables& tb, cudaStream_t st) {
  if (n == 0) return;
  OpPairsLaunch f{n, target, tc, src, sc, p, local, tab_of(tb), st};
  dispatch_slots(p, lh, f);
}

void launch_op_m2l(int64_t n, double* target, const double* tc, const double* tbox, const double* trad,
                   const double* maxinf, const double* src, const double* sc, int p, bool lh, int em, double eps,
                   int be, int* p_used, const DevTables& tb, cudaStream_t st) {
  if (n == 0) return;
  OpM2LLaunch f{n, target, tc, tbox, trad, maxinf, src, sc, p, em, be, eps, p_used, tab_of(tb), st};
  dispatch_slots(p, lh, f);
}

void launch_op_p2m(int kind, const double4* pos, const double4* str, int64_t n, const double* center, int p,
                   double* expansion, cudaStream_t st) {
  size_t sm = 2 * nh(p) * sizeof(double);
  note_launch();
  k_op_p2m<<<1, 32, sm, st>>>(pos, str, n, center[0], center[1], center[2], expansion, p, kind);
  FMM_CUDA_TRY(cudaGetLastError());
}

void launch_op_l2p(int64_t n, const double* dx, const double* local, int p, bool lh, bool ps, bool gs, bool hs,
                   double* out13, cudaStream_t st) {
  if (n == 0) return;
  size_t sm = l2p_smem(p);
  allow_smem(k_op_l2p, sm);
  int g = (int)std::min<int64_t>((n + kL2PThreads - 1) / kL2PThreads, 1024);
  note_launch();
  k_op_l2p<<<g, kL2PThreads, sm, st>>>(n, dx, local, p, lh ? 1 : 0, ps ? 1 : 0, gs ? 1 : 0, hs ? 1 : 0, out13);
  FMM_CUDA_TRY(cudaGetLastError());
}

}  // namespace fmmb

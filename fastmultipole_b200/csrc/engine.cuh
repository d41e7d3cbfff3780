// engine.cuh -- warp-level rotation-based translation operators (point-and-shoot).
//
// One warp applies the reference's chain
//   rotate_z -> rotate_y (Wigner d at theta from the pi/2 table) -> coaxial
//   translation -> [Lamb-Helmholtz re-centring] -> rotate_y back -> rotate_z back
// (src/translate.jl:144-174, 519-550, 1896-1926; src/rotate.jl) to one pair at a
// time and accumulates the result into registers owned by the lanes: lane l
// holds coefficients i = l + 32 k, k < SLOTS.  Intermediate expansions live in
// the warp's slice of shared memory as planes (phi.re, phi.im, chi.re, chi.im),
// each a contiguous array over the coefficient index, so the lane-per-coefficient
// stages read and write consecutive doubles (no bank conflicts).  The degree of
// coefficient i and its order are computed once per lane (SlotNM).
//
// SLOTS = ceil(Nh / 32) and LH (Lamb-Helmholtz, vortex sources) are template
// parameters, so the accumulator holds exactly the live coefficients.
#pragma once
#include "context.cuh"

namespace fmmb {
namespace eng {

__constant__ double c_ifact[kMaxP + 1] = {FMM_INV_FACTORIALS};

constexpr unsigned kFull = 0xffffffffu;

struct Tab {
  const double* Hs;
  const double* zeta;
  const double* eta;
  const double* Mt;
  const double* Lt;
};

__device__ __forceinline__ void nm_of(int i, int& n, int& m) {
  n = (int)((sqrtf(8.0f * (float)i + 1.0f) - 1.0f) * 0.5f);
  while ((n + 1) * (n + 2) / 2 <= i) ++n;
  while (n * (n + 1) / 2 > i) --n;
  m = i - n * (n + 1) / 2;
}

template <int SLOTS>
struct SlotNM {
  int n[SLOTS], m[SLOTS];
  __device__ __forceinline__ void init(int NH) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < SLOTS; ++k) {
      int i = lane + 32 * k;
      if (i < NH) {
        nm_of(i, n[k], m[k]);
      } else {
        n[k] = -1;
        m[k] = 0;
      }
    }
  }
};

// per-warp shared-memory workspace (doubles)
struct WS {
  int NH;        // coefficients of the workspace (order p)
  double* a;     // 4 planes x NH
  double* b;     // 4 planes x NH
  double* ts;    // Wigner matrices, length_Ts(p)
  double* eim;   // e^{i m phi}, 2 (p+1)
  double* cs;    // cos, sin (nu beta), 2 (p+1)
  double* w3;    // one degree, 4 planes x (p+1)
};

__host__ __device__ inline int64_t ws_doubles(int p) {
  return 8 * nh(p) + length_Ts(p) + 2 * (p + 1) + 2 * (p + 1) + 4 * (p + 1) + 8;
}

__device__ __forceinline__ WS ws_of(double* base, int p) {
  WS w;
  w.NH = (int)nh(p);
  w.a = base;
  w.b = w.a + 4 * w.NH;
  w.ts = w.b + 4 * w.NH;
  w.eim = w.ts + length_Ts(p);
  w.cs = w.eim + 2 * (p + 1);
  w.w3 = w.cs + 2 * (p + 1);
  return w;
}

// plane accessors: plane 0 = phi.re, 1 = phi.im, 2 = chi.re, 3 = chi.im
#define PL(arr, plane, i, NH) (arr)[(plane) * (NH) + (i)]

// cartesian_to_spherical, src/rotate.jl:9-21
__device__ __forceinline__ void sph(double x, double y, double z, double& r, double& th, double& ph) {
  double x2y2 = x * x + y * y;
  double r2 = x2y2 + z * z;
  r = (r2 == 0.0) ? r2 : sqrt(r2);
  double z_r = z / r;
  if (r > 0)
    th = x2y2 > 0 ? acos(z_r) : kPi * (z < 0 ? 1.0 : 0.0);
  else
    th = 0.0;
  ph = (x2y2 == 0.0) ? 0.0 : atan2(y, x);
}

// e^{i m phi} (update_eimphis!, src/rotate.jl:25-37) and cos/sin(nu beta)
// (update_Ts!, src/rotate.jl:296-298) by the reference's recurrences, lane 0
__device__ __forceinline__ void angles(const WS& w, double ph, double beta, int P) {
  if ((threadIdx.x & 31) == 0) {
    double ei = sin(ph), er = cos(ph);
    double cr = 1.0, ci = 0.0;
    for (int m = 0; m <= P; ++m) {
      w.eim[2 * m] = cr;
      w.eim[2 * m + 1] = ci;
      double t = cr;
      cr = cr * er - ci * ei;
      ci = t * ei + ci * er;
    }
    double sb = sin(beta), cb = cos(beta);
    double c = 1.0, s = 0.0;
    w.cs[0] = 1.0;
    w.cs[1] = 0.0;
    for (int nu = 1; nu <= P; ++nu) {
      double cn = cb * c - sb * s;
      double sn = sb * c + cb * s;
      w.cs[2 * nu] = cn;
      w.cs[2 * nu + 1] = sn;
      c = cn;
      s = sn;
    }
  }
}

__device__ __forceinline__ double get_scalar(int m_mp) {
  if (m_mp & 1) m_mp += 1;
  return ((m_mp >> 1) & 1) == 0 ? 1.0 : -1.0;
}

// Wigner matrix of degree n at beta from the pi/2 table (update_Ts_n!,
// src/rotate.jl:363-441); lanes over (m, m') with 0 <= m' <= m <= n
__device__ __forceinline__ void ts_degree(double* Ts, const double* __restrict__ Hs, const double* cs, int n) {
  const int lane = threadIdx.x & 31;
  const double* H = Hs + length_Hs(n - 1);
  double* T = Ts + length_Ts(n - 1);
  const double _1_n = (n & 1) ? -1.0 : 1.0;
  const int cnt = (n + 1) * (n + 2) / 2;
  for (int j = lane; j < cnt; j += 32) {
    int m, mp;
    nm_of(j, m, mp);
    double H_m_0 = __ldg(H + H_index(0, m));
    double H_mp_0 = __ldg(H + H_index(0, mp));
    double _1_mp_odd = (mp & 1) ? -1.0 : 1.0;
    double _1_n_mp = (mp & 1) ? -_1_n : _1_n;
    int m_mp = m + mp;
    bool even = (m_mp & 1) == 0;
    double scalar = get_scalar(m_mp);
    double vp = 0, vn = 0;
    double _1_n_mp_nu = -_1_n_mp;
    for (int nu = 1; nu <= n; ++nu) {
      double sc = even ? scalar * cs[2 * nu] : scalar * cs[2 * nu + 1];
      double H_mp_nu = __ldg(H + H_index(min(mp, nu), max(mp, nu)));
      double H_m_nu = __ldg(H + H_index(min(m, nu), max(m, nu)));
      double val = H_mp_nu * H_m_nu * sc;
      vp += val;
      vn += val * _1_n_mp_nu * _1_mp_odd;
      _1_n_mp_nu = -_1_n_mp_nu;
    }
    vp *= 2.0;
    vn *= 2.0;
    double s0 = even ? scalar : 0.0;
    double val = H_m_0 * H_mp_0 * s0;
    vp += val;
    vn += val * _1_n_mp * _1_mp_odd;
    T[T_index(mp, m)] = vp;
    T[T_index(-mp, m)] = vn;
  }
}

__device__ __forceinline__ void ts_all(const WS& w, const double* __restrict__ Hs, int P) {
  if ((threadIdx.x & 31) == 0) w.ts[0] = 1.0;
  for (int n = 1; n <= P; ++n) ts_degree(w.ts, Hs, w.cs, n);
}

__device__ __forceinline__ void quarter(double mag, int k, double& re, double& im) {
  k %= 4;
  if (k < 0) k += 4;
  re = (k == 0) ? mag : ((k == 2) ? -mag : 0.0);
  im = (k == 1) ? mag : ((k == 3) ? -mag : 0.0);
}


// ---------------------------------------------------------------------------
// stages.  "all" variants: lanes over the slots, degrees 0..P; "deg" variants:
// one degree n, lane = m (n < 32).

// rotate_z! (src/rotate.jl:448-483): planar dst <- interleaved src (global)
template <bool LH>
__device__ __forceinline__ void rot_z_one(const WS& w, double* dst, const double2* __restrict__ s2, int i, int n, int m) {
  const int NH = w.NH;
  double er = w.eim[2 * m], ei = w.eim[2 * m + 1];
  double2 x = s2[2 * i];
  if (n == 0) {
    dst[i] = x.x;
    dst[NH + i] = x.y;
  } else {
    dst[i] = x.x * er - x.y * ei;
    dst[NH + i] = x.x * ei + x.y * er;
  }
  if (LH) {
    double2 y = s2[2 * i + 1];
    if (n == 0) {
      dst[2 * NH + i] = y.x;
      dst[3 * NH + i] = y.y;
    } else {
      dst[2 * NH + i] = y.x * er - y.y * ei;
      dst[3 * NH + i] = y.x * ei + y.y * er;
    }
  }
}

template <int SLOTS, bool LH>
__device__ __forceinline__ void rot_z_all(const WS& w, double* dst, const double* __restrict__ src,
                                          const SlotNM<SLOTS>& L, int P) {
  const int lane = threadIdx.x & 31, NHP = (P + 1) * (P + 2) / 2;
  const double2* s2 = reinterpret_cast<const double2*>(src);
#pragma unroll
  for (int k = 0; k < SLOTS; ++k) {
    int i = lane + 32 * k;
    if (i < NHP) rot_z_one<LH>(w, dst, s2, i, L.n[k], L.m[k]);
  }
}

template <bool LH>
__device__ __forceinline__ void rot_z_deg(const WS& w, double* dst, const double* __restrict__ src, int n) {
  const int m = threadIdx.x & 31;
  if (m <= n) rot_z_one<LH>(w, dst, reinterpret_cast<const double2*>(src), n * (n + 1) / 2 + m, n, m);
}

// _rotate_multipole_y! (local=false, src/rotate.jl:699-803) / _rotate_local_y!
// (local=true, src/rotate.jl:1014-1113) for output coefficient (n, m)
template <bool LH>
__device__ __forceinline__ void rot_y_one(const WS& w, double* dst, const double* src, const double* __restrict__ mags,
                                          bool local, int n, int m) {
  const int NH = w.NH;
  const int iT = (int)length_Ts(n - 1), base = n * (n + 1) / 2;
  double v1r = 0, v1i = 0, v2r = 0, v2i = 0;
  for (int mp = -n; mp <= n; ++mp) {
    int amp = mp < 0 ? -mp : mp;
    double T = (mp <= 0) ? w.ts[iT + T_index(-min(amp, m), max(amp, m))] : w.ts[iT + T_index(min(mp, m), max(mp, m))];
    double mag = __ldg(mags + iT + m * (n + 1) + amp) * T;
    double zr, zi;
    quarter(mag, local ? (m - amp) : (amp - m), zr, zi);
    int iw = base + amp;
    double Mr = src[iw], Mi = src[NH + iw];
    if (mp <= 0) {
      Mi = -Mi;
      if (mp & 1) {
        Mr = -Mr;
        Mi = -Mi;
      }
    }
    v1r += Mr * zr - Mi * zi;
    v1i += Mr * zi + Mi * zr;
    if (LH) {
      double Cr = src[2 * NH + iw], Ci = src[3 * NH + iw];
      if (mp <= 0) {
        Ci = -Ci;
        if (mp & 1) {
          Cr = -Cr;
          Ci = -Ci;
        }
      }
      v2r += Cr * zr - Ci * zi;
      v2i += Cr * zi + Ci * zr;
    }
  }
  int i = base + m;
  dst[i] = v1r;
  dst[NH + i] = v1i;
  if (LH) {
    dst[2 * NH + i] = v2r;
    dst[3 * NH + i] = v2i;
  }
}

template <int SLOTS, bool LH>
__device__ __forceinline__ void rot_y_all(const WS& w, double* dst, const double* src, const double* __restrict__ mags,
                                          bool local, const SlotNM<SLOTS>& L, int P) {
  const int lane = threadIdx.x & 31, NHP = (P + 1) * (P + 2) / 2;
#pragma unroll
  for (int k = 0; k < SLOTS; ++k) {
    int i = lane + 32 * k;
    if (i < NHP) rot_y_one<LH>(w, dst, src, mags, local, L.n[k], L.m[k]);
  }
}

template <bool LH>
__device__ __forceinline__ void rot_y_deg(const WS& w, double* dst, const double* src, const double* __restrict__ mags,
                                          bool local, int n) {
  const int m = threadIdx.x & 31;
  if (m <= n) rot_y_one<LH>(w, dst, src, mags, local, n, m);
}

// (n+m)!/t^(n+m+1) by the reference's recurrence (src/translate.jl:184-225)
__device__ __forceinline__ double m2l_coef0(int n, int m, double one_over_t) {
  double c = one_over_t;
  for (int k = 0; k < n; ++k) c *= (k + 1) * one_over_t;
  int nm = n;
  for (int j = 0; j < m; ++j) {
    nm += 1;
    c *= nm * one_over_t;
  }
  return c;
}

// translate_multipole_to_local_z! (src/translate.jl:181-232) for output (n, m),
// source degrees m..Psrc; result to dst[plane * stride + o]
template <bool LH>
__device__ __forceinline__ void m2l_z_one(const WS& w, double* dst, int stride, int o, const double* src, double t,
                                          int Psrc, int n, int m) {
  const int NH = w.NH;
  double one_over_t = 1 / t;
  double c = m2l_coef0(n, m, one_over_t);
  int n_np = n + m;
  double v1r = 0, v1i = 0, v2r = 0, v2i = 0;
  for (int np = m; np <= Psrc; ++np) {
    int iw = np * (np + 1) / 2 + m;
    v1r += c * src[iw];
    v1i += c * src[NH + iw];
    if (LH) {
      v2r += c * src[2 * NH + iw];
      v2i += c * src[3 * NH + iw];
    }
    n_np += 1;
    c *= n_np * one_over_t;
  }
  dst[o] = v1r;
  dst[stride + o] = v1i;
  if (LH) {
    dst[2 * stride + o] = v2r;
    dst[3 * stride + o] = v2i;
  }
}

template <int SLOTS, bool LH>
__device__ __forceinline__ void m2l_z_all(const WS& w, double* dst, const double* src, double t,
                                          const SlotNM<SLOTS>& L, int P) {
  const int lane = threadIdx.x & 31, NHP = (P + 1) * (P + 2) / 2;
#pragma unroll
  for (int k = 0; k < SLOTS; ++k) {
    int i = lane + 32 * k;
    if (i < NHP) m2l_z_one<LH>(w, dst, w.NH, i, src, t, P, L.n[k], L.m[k]);
  }
}

// translate_multipole_z! (src/translate.jl:6-50)
template <int SLOTS, bool LH>
__device__ __forceinline__ void m2m_z_all(const WS& w, double* dst, const double* src, double t,
                                          const SlotNM<SLOTS>& L, int P) {
  const int lane = threadIdx.x & 31, NHP = (P + 1) * (P + 2) / 2, NH = w.NH;
  const double _t = -t;
#pragma unroll
  for (int k = 0; k < SLOTS; ++k) {
    int i = lane + 32 * k;
    if (i >= NHP) continue;
    int n = L.n[k], m = L.m[k];
    double v1r = 0, v1i = 0, v2r = 0, v2i = 0, tp = 1.0;
    for (int np = n; np >= m; --np) {
      double c = tp * c_ifact[n - np];  // (-t)^(n-n') / (n-n')!
      int iw = np * (np + 1) / 2 + m;
      v1r += c * src[iw];
      v1i += c * src[NH + iw];
      if (LH) {
        v2r += c * src[2 * NH + iw];
        v2i += c * src[3 * NH + iw];
      }
      tp *= _t;
    }
    dst[i] = v1r;
    dst[NH + i] = v1i;
    if (LH) {
      dst[2 * NH + i] = v2r;
      dst[3 * NH + i] = v2i;
    }
  }
}

// translate_local_z! (src/translate.jl:1851-1891)
template <int SLOTS, bool LH>
__device__ __forceinline__ void l2l_z_all(const WS& w, double* dst, const double* src, double t,
                                          const SlotNM<SLOTS>& L, int P) {
  const int lane = threadIdx.x & 31, NHP = (P + 1) * (P + 2) / 2, NH = w.NH;
  const double _t = -t;
#pragma unroll
  for (int k = 0; k < SLOTS; ++k) {
    int i = lane + 32 * k;
    if (i >= NHP) continue;
    int n = L.n[k], m = L.m[k];
    double v1r = 0, v1i = 0, v2r = 0, v2i = 0, tp = 1.0;
    for (int np = n; np <= P; ++np) {
      const double c = tp * c_ifact[np - n];  // (-t)^(n'-n) / (n'-n)!
      int iw = np * (np + 1) / 2 + m;
      v1r += c * src[iw];
      v1i += c * src[NH + iw];
      if (LH) {
        v2r += c * src[2 * NH + iw];
        v2i += c * src[3 * NH + iw];
      }
      tp *= _t;
    }
    dst[i] = v1r;
    dst[NH + i] = v1i;
    if (LH) {
      dst[2 * NH + i] = v2r;
      dst[3 * NH + i] = v2i;
    }
  }
}

// transform_lamb_helmholtz_multipole! (src/translate.jl:52-96), lane = m
__device__ __forceinline__ void lh_multipole(const WS& w, double* M, double r, int P) {
  const int NH = w.NH;
  for (int m = threadIdx.x & 31; m <= P; m += 32) {
    int i = P * (P + 1) / 2 + m;
    double cr = M[2 * NH + i], ci = M[3 * NH + i];
    for (int n = P; n >= max(m, 1); --n) {
      double pr = M[i], pi = M[NH + i];
      double xr = cr, xi = ci;
      double a = r * m / (n + 1);
      M[i] = pr + a * xi;
      M[NH + i] = pi - a * xr;
      if (m < n) {
        cr = M[2 * NH + i - n];
        ci = M[3 * NH + i - n];
      } else {
        cr = 0;
        ci = 0;
      }
      double b = r / n;
      M[2 * NH + i] = xr + b * cr;
      M[3 * NH + i] = xi + b * ci;
      i -= n;
    }
  }
}

// transform_lamb_helmholtz_local! (src/translate.jl:98-142), lane = m
__device__ __forceinline__ void lh_local(const WS& w, double* Lx, double r, int P) {
  const int NH = w.NH;
  for (int m = threadIdx.x & 31; m <= P; m += 32) {
    int i = m * (m + 1) / 2 + m;
    double cr = Lx[2 * NH + i], ci = Lx[3 * NH + i];
    for (int n = m; n <= P; ++n) {
      double xr = cr, xi = ci;
      if (n > 0) {
        double pr = Lx[i], pi = Lx[NH + i];
        double a = r * m / n;
        Lx[i] = pr - a * xi;
        Lx[NH + i] = pi + a * xr;
      }
      if (n < P) {
        cr = Lx[2 * NH + i + n + 1];
        ci = Lx[3 * NH + i + n + 1];
        double b = r / (n + 1);
        Lx[2 * NH + i] = xr - b * cr;
        Lx[3 * NH + i] = xi - b * ci;
      }
      i += n + 1;
    }
  }
}

// back_rotate_z! (src/rotate.jl:584-616) into the lane-owned accumulator
template <int SLOTS, bool LH>
__device__ __forceinline__ void back_z_acc(double (&acc)[SLOTS][LH ? 4 : 2], const WS& w, const double* src,
                                           const SlotNM<SLOTS>& L, int P) {
  const int lane = threadIdx.x & 31, NHP = (P + 1) * (P + 2) / 2, NH = w.NH;
#pragma unroll
  for (int k = 0; k < SLOTS; ++k) {
    int i = lane + 32 * k;
    if (i >= NHP) continue;
    int n = L.n[k], m = L.m[k];
    double er = w.eim[2 * m], ei = -w.eim[2 * m + 1];
    double xr = src[i], xi = src[NH + i];
    if (n == 0) {
      acc[k][0] += xr;
      acc[k][1] += xi;
    } else {
      acc[k][0] += xr * er - xi * ei;
      acc[k][1] += xr * ei + xi * er;
    }
    if (LH) {
      double yr = src[2 * NH + i], yi = src[3 * NH + i];
      if (n == 0) {
        acc[k][2 % (LH ? 4 : 2)] += yr;
        acc[k][3 % (LH ? 4 : 2)] += yi;
      } else {
        acc[k][2 % (LH ? 4 : 2)] += yr * er - yi * ei;
        acc[k][3 % (LH ? 4 : 2)] += yr * ei + yi * er;
      }
    }
  }
}

template <int SLOTS, bool LH>
__device__ __forceinline__ void acc_zero(double (&acc)[SLOTS][LH ? 4 : 2]) {
#pragma unroll
  for (int k = 0; k < SLOTS; ++k)
#pragma unroll
    for (int c = 0; c < (LH ? 4 : 2); ++c) acc[k][c] = 0.0;
}

// accumulate into an interleaved expansion in global memory (e[4 i + 2 set + reim])
template <int SLOTS, bool LH>
__device__ __forceinline__ void acc_store_add(double* dst, const double (&acc)[SLOTS][LH ? 4 : 2], int NH) {
  const int lane = threadIdx.x & 31;
  double2* d2 = reinterpret_cast<double2*>(dst);
#pragma unroll
  for (int k = 0; k < SLOTS; ++k) {
    int i = lane + 32 * k;
    if (i < NH) {
      double2 v = d2[2 * i];
      v.x += acc[k][0];
      v.y += acc[k][1];
      d2[2 * i] = v;
      if (LH) {
        double2 u = d2[2 * i + 1];
        u.x += acc[k][2 % (LH ? 4 : 2)];
        u.y += acc[k][3 % (LH ? 4 : 2)];
        d2[2 * i + 1] = u;
      }
    }
  }
}


// ---------------------------------------------------------------------------
// chains

// multipole_to_multipole! (local=false, src/translate.jl:144-174) / local_to_local!
// (local=true, src/translate.jl:1896-1926) of one source expansion (global,
// interleaved) translated by (dx, dy, dz) = target centre - source centre
template <int SLOTS, bool LH>
__device__ __forceinline__ void chain_mm_ll(const WS& w, double (&acc)[SLOTS][LH ? 4 : 2],
                                            const double* __restrict__ src, double dx, double dy, double dz, int p,
                                            bool local, const Tab& tb, const SlotNM<SLOTS>& L) {
  double r, th, ph;
  sph(dx, dy, dz, r, th, ph);
  angles(w, ph, th, p);
  __syncwarp();
  rot_z_all<SLOTS, LH>(w, w.a, src, L, p);
  ts_all(w, tb.Hs, p);
  __syncwarp();
  const double* mags = local ? tb.eta : tb.zeta;
  rot_y_all<SLOTS, LH>(w, w.b, w.a, mags, local, L, p);
  __syncwarp();
  if (local)
    l2l_z_all<SLOTS, LH>(w, w.a, w.b, r, L, p);
  else
    m2m_z_all<SLOTS, LH>(w, w.a, w.b, r, L, p);
  __syncwarp();
  if (LH) {
    if (local)
      lh_local(w, w.a, r, p);
    else
      lh_multipole(w, w.a, r, p);
    __syncwarp();
  }
  rot_y_all<SLOTS, LH>(w, w.b, w.a, mags, local, L, p);
  __syncwarp();
  back_z_acc<SLOTS, LH>(acc, w, w.b, L, p);
  __syncwarp();
}

__device__ __forceinline__ double warp_sum_bcast(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return __shfl_sync(kFull, v, 0);
}

__device__ __forceinline__ double minabs(double x, double y) {
  return x * (fabs(x) <= fabs(y) ? 1.0 : 0.0) + y * (fabs(y) < fabs(x) ? 1.0 : 0.0);
}
// minimum_distance, src/error.jl:5-20
__device__ __forceinline__ double min_dist_1d(double dx, double rm, double rp) {
  double right = dx + rp, left = dx + rm;
  double same = (right * left >= 0) ? 1.0 : 0.0;
  return same * minabs(right, left);
}

struct M2LGeom {
  double tc[3];
  double tbox[3];
  double trad;
  double maxinf;
};

// multipole_to_local!: plain (src/translate.jl:519-550) and the error-controlled
// Power{Absolute,Relative}Gradient (:1124-1412) and RotatedCoefficients{Absolute,
// Relative}Gradient (:555-829).  Returns the order used; ok = tolerance met.
template <int SLOTS, bool LH>
__device__ __forceinline__ int chain_m2l(const WS& w, double (&acc)[SLOTS][LH ? 4 : 2],
                                         const double* __restrict__ src, const double* sc, const M2LGeom& g, int p,
                                         int em, double eps_in, int be, bool& ok, const Tab& tb,
                                         const SlotNM<SLOTS>& L) {
  const int lane = threadIdx.x & 31;
  const int NH = w.NH, S3 = p + 1;
  double r, th, ph;
  sph(g.tc[0] - sc[0], g.tc[1] - sc[1], g.tc[2] - sc[2], r, th, ph);
  angles(w, ph, th, p);
  __syncwarp();
  int P = p;
  ok = true;
  if (em == FMM_ERROR_NONE) {
    rot_z_all<SLOTS, LH>(w, w.a, src, L, p);
    ts_all(w, tb.Hs, p);
    __syncwarp();
    rot_y_all<SLOTS, LH>(w, w.b, w.a, tb.zeta, false, L, p);
    __syncwarp();
  } else {
    const bool relative = (em == FMM_POWER_RELATIVE_GRADIENT || em == FMM_ROTATED_COEFFICIENTS_RELATIVE_GRADIENT ||
                           em == FMM_POWER_RELATIVE_POTENTIAL);
    // Power{Absolute,Relative}Potential (src/translate.jl:831-1122): the power family with
    // the potential's error formulas
    const bool potential = (em == FMM_POWER_ABSOLUTE_POTENTIAL || em == FMM_POWER_RELATIVE_POTENTIAL);
    const bool power = (em == FMM_POWER_ABSOLUTE_GRADIENT || em == FMM_POWER_RELATIVE_GRADIENT || potential);
    const double eps = relative ? g.maxinf * eps_in : eps_in;
    double mdx = min_dist_1d(g.tc[0] - sc[0], -g.tbox[0], g.tbox[0]);
    double mdy = min_dist_1d(g.tc[1] - sc[1], -g.tbox[1], g.tbox[1]);
    double mdz = min_dist_1d(g.tc[2] - sc[2], -g.tbox[2], g.tbox[2]);
    double r_mp = sqrt(mdx * mdx + mdy * mdy + mdz * mdz);
    double r_l = g.trad;
    double rinv = 1.0 / r, r_mp_inv = 1.0 / r_mp;
    double r_mp_inv_np2 = r_mp_inv * r_mp_inv * r_mp_inv;
    double r_l_nm1 = 1.0;
    rot_z_deg<LH>(w, w.a, src, 0);
    if (lane == 0) w.ts[0] = 1.0;
    __syncwarp();
    rot_y_deg<LH>(w, w.b, w.a, tb.zeta, false, 0);
    double n_fact_t_np1 = rinv * rinv, nm1_fact_inv = 1.0, np1_fact = 2.0;
    double Mn0 = tb.Mt[0];
    double mp_phi = sqrt((src[0] * src[0] + src[1] * src[1]) * Mn0 * Mn0);
    const double four_pi_eps = eps * 4 * kPi;
    ok = false;
    for (int n = 1; n <= p; ++n) {
      double pn_phi = 0, pn_chi = 0, Mn0_next = tb.Mt[n * (n + 1) / 2];
      if (power) {
        // multipole power of degree n (rotate_z_n_power!, src/rotate.jl:528-576);
        // the reference's `(1 + m>0)` weight evaluates to 1
        double a = 0, b = 0;
        if (lane <= n) {
          int i = n * (n + 1) / 2 + lane;
          double Nt = tb.Mt[i];
          a = (src[4 * i] * src[4 * i] + src[4 * i + 1] * src[4 * i + 1]) * Nt * Nt;
          if (LH) b = (src[4 * i + 2] * src[4 * i + 2] + src[4 * i + 3] * src[4 * i + 3]) * Nt * Nt;
        }
        pn_phi = sqrt(warp_sum_bcast(a));
        pn_chi = sqrt(warp_sum_bcast(b));
      }
      rot_z_deg<LH>(w, w.a, src, n);
      ts_degree(w.ts, tb.Hs, w.cs, n);
      __syncwarp();
      rot_y_deg<LH>(w, w.b, w.a, tb.zeta, false, n);
      __syncwarp();
      double eps_mp;
      const int in0 = n * (n + 1) / 2;
      if (potential) {
        eps_mp = 1.7320508075688772 * pn_phi * r_mp_inv_np2 * r_mp * np1_fact / (Mn0 * (n + 1));
        if (LH) eps_mp += 1.7320508075688772 * n * pn_chi * r_mp_inv_np2 * r_mp * np1_fact / (Mn0_next * (n + 1));
      } else if (power) {
        eps_mp = 1.7320508075688772 * mp_phi * r_mp_inv_np2 * np1_fact / Mn0;
        if (LH) eps_mp += 1.7320508075688772 * n * pn_chi * r_mp_inv_np2 * np1_fact / Mn0_next;
      } else {
        double p0 = w.b[in0];
        double p1r = w.b[in0 + 1], p1i = w.b[NH + in0 + 1];
        eps_mp = (sqrt(p1r * p1r + p1i * p1i) + fabs(p0)) * np1_fact * r_mp_inv_np2;
        if (LH) {
          double c1r = w.b[2 * NH + in0 + 1], c1i = w.b[3 * NH + in0 + 1];
          eps_mp += sqrt(c1r * c1r + c1i * c1i) * np1_fact * r_mp_inv_np2 * r_mp;
        }
      }
      if (eps_mp <= four_pi_eps) {
        double eps_l;
        if (power) {
          // degree n of translate_multipole_to_local_z_n! (src/translate.jl:238-295)
          // and local_power (:455-502)
          if (lane <= n) m2l_z_one<LH>(w, w.w3, S3, lane, w.b, r, n, n, lane);
          __syncwarp();
          double a = 0, b = 0;
          if (lane <= n) {
            int m = lane;
            double Nt = tb.Lt[in0 + m];
            double pr = w.w3[m], pi = w.w3[S3 + m];
            if (LH) {
              double cro = w.w3[2 * S3 + m], cio = w.w3[3 * S3 + m];
              double crn = (m < n) ? w.w3[2 * S3 + m + 1] : 0.0;
              double cin = (m < n) ? w.w3[3 * S3 + m + 1] : 0.0;
              pr = pr - cio * r * m / n;
              pi = pi + cro * r * m / n;
              double cr = cro - crn * r / (n + 1);
              double ci = cio - cin * r / (n + 1);
              b = (cr * cr + ci * ci) * Nt * Nt;
            }
            a = (pr * pr + pi * pi) * Nt * Nt;
          }
          double lphi = sqrt(warp_sum_bcast(a));
          double lchi = sqrt(warp_sum_bcast(b));
          double Ln0 = tb.Lt[in0];
          if (potential)
            eps_l = 1.7320508075688772 * lphi * r_l_nm1 * r_l * nm1_fact_inv / (Ln0 * n);
          else
            eps_l = 1.7320508075688772 * lphi * r_l_nm1 * nm1_fact_inv / Ln0;
          if (LH) eps_l += 1.7320508075688772 * n * lchi * r_l_nm1 * r_l * nm1_fact_inv / (Ln0 * n);
          __syncwarp();
        } else {
          // translate_multipole_to_local_z_m01_n, src/translate.jl:302-364 (all lanes alike)
          double one_over_t = rinv;
          double c = n_fact_t_np1;
          int n_np = n;
          double a0 = 0;
          for (int np = 0; np <= n; ++np) {
            a0 += c * w.b[np * (np + 1) / 2];
            n_np += 1;
            c *= n_np * one_over_t;
          }
          c = n_fact_t_np1 * ((n + 1) * one_over_t);
          n_np = n + 1;
          double b1r = 0, b1i = 0, x1r = 0, x1i = 0;
          for (int np = 1; np <= n; ++np) {
            int iw = np * (np + 1) / 2 + 1;
            b1r += c * w.b[iw];
            b1i += c * w.b[NH + iw];
            if (LH) {
              x1r += c * w.b[2 * NH + iw];
              x1i += c * w.b[3 * NH + iw];
            }
            n_np += 1;
            c *= n_np * one_over_t;
          }
          if (LH) {
            double t_over_n = r / n;
            b1r -= t_over_n * x1i;
            b1i += t_over_n * x1r;
          }
          eps_l = (fabs(b1r) + fabs(b1i) + fabs(a0)) * r_l_nm1 * nm1_fact_inv;
          if (LH) eps_l += sqrt(x1r * x1r + x1i * x1i) * r_l_nm1 * r_l * nm1_fact_inv;
        }
        if (eps_mp + eps_l * 2.0 <= four_pi_eps) {
          P = n - 1 + (be ? 1 : 0);
          ok = true;
          break;
        }
      }
      if (power || n < p) {
        n_fact_t_np1 *= (n + 1) * rinv;
        r_l_nm1 *= r_l;
        r_mp_inv_np2 *= r_mp_inv;
        nm1_fact_inv /= n;
        np1_fact *= n + 1;
      }
      if (power) {
        mp_phi = pn_phi;
        Mn0 = Mn0_next;
      }
    }
  }
  m2l_z_all<SLOTS, LH>(w, w.a, w.b, r, L, P);
  __syncwarp();
  if (LH) {
    lh_local(w, w.a, r, P);
    __syncwarp();
  }
  rot_y_all<SLOTS, LH>(w, w.b, w.a, tb.eta, true, L, P);
  __syncwarp();
  back_z_acc<SLOTS, LH>(acc, w, w.b, L, P);
  __syncwarp();
  return P;
}

}  // namespace eng
}  // namespace fmmb

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
#include "context.cuh"

namespace fmmb {

namespace {

constexpr int kWarps = 4;                      // warps per CTA
constexpr int kSlots = (231 + 31) / 32;        // nh(kMaxP) coefficients over 32 lanes
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

// per-warp shared-memory workspace (doubles)
struct WS {
  double* w1;   // 4*Nh
  double* w2;   // 4*Nh
  double* ts;   // length_Ts(p)
  double* eim;  // 2*(p+1)
  double* cs;   // 2*(p+1): cos(nu beta), sin(nu beta)
  double* w3;   // 4*(p+1): one degree (error prediction)
};

__host__ __device__ inline int64_t ws_doubles(int p) {
  return 8 * nh(p) + length_Ts(p) + 4 * (p + 1) + 4 * (p + 1) + 8;
}

__device__ __forceinline__ WS ws_of(double* base, int p) {
  WS w;
  w.w1 = base;
  w.w2 = w.w1 + 4 * nh(p);
  w.ts = w.w2 + 4 * nh(p);
  w.eim = w.ts + length_Ts(p);
  w.cs = w.eim + 2 * (p + 1);
  w.w3 = w.cs + 2 * (p + 1);
  return w;
}

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

// e^{i m phi} (update_eimphis!, src/rotate.jl:25-37) and cos/sin(nu beta) of
// update_Ts! (src/rotate.jl:296-298), by the reference's recurrences, in lane 0
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

// rotate_z! restricted to degrees [n0, n1] (src/rotate.jl:448-483)
__device__ __forceinline__ void rot_z(double* dst, const double* __restrict__ src, const double* eim, int n0, int n1,
                                      bool lh) {
  int lane = threadIdx.x & 31;
  int i0 = n0 * (n0 + 1) / 2, i1 = (n1 + 1) * (n1 + 2) / 2;
  for (int i = i0 + lane; i < i1; i += 32) {
    int n, m;
    nm_of(i, n, m);
    double er = eim[2 * m], ei = eim[2 * m + 1];
    for (int s = 0; s <= (lh ? 1 : 0); ++s) {
      double xr = src[4 * i + 2 * s], xi = src[4 * i + 2 * s + 1];
      if (n == 0) {
        dst[4 * i + 2 * s] = xr;
        dst[4 * i + 2 * s + 1] = xi;
      } else {
        dst[4 * i + 2 * s] = xr * er - xi * ei;
        dst[4 * i + 2 * s + 1] = xr * ei + xi * er;
      }
    }
  }
}

__device__ __forceinline__ double get_scalar(int m_mp) {
  if (m_mp & 1) m_mp += 1;
  return ((m_mp >> 1) & 1) == 0 ? 1.0 : -1.0;
}

// Wigner matrix of degree n at beta from the pi/2 table (update_Ts_n!, src/rotate.jl:363-441);
// lanes over (m, m') with 0 <= m' <= m <= n
__device__ __forceinline__ void ts_degree(double* Ts, const double* __restrict__ Hs, const double* cs, int n) {
  int lane = threadIdx.x & 31;
  const double* H = Hs + length_Hs(n - 1);
  double* T = Ts + length_Ts(n - 1);
  const double _1_n = (n & 1) ? -1.0 : 1.0;
  int cnt = (n + 1) * (n + 2) / 2;
  for (int j = lane; j < cnt; j += 32) {
    int m, mp;
    nm_of(j, m, mp);
    double H_m_0 = H[H_index(0, m)];
    double H_mp_0 = H[H_index(0, mp)];
    double _1_mp_odd = (mp & 1) ? -1.0 : 1.0;
    double _1_n_mp = (mp & 1) ? -_1_n : _1_n;
    int m_mp = m + mp;
    bool even = (m_mp & 1) == 0;
    double scalar = get_scalar(m_mp);
    double vp = 0, vn = 0;
    double _1_n_mp_nu = -_1_n_mp;
    for (int nu = 1; nu <= n; ++nu) {
      double sc = even ? scalar * cs[2 * nu] : scalar * cs[2 * nu + 1];
      double H_mp_nu = H[H_index(min(mp, nu), max(mp, nu))];
      double H_m_nu = H[H_index(min(m, nu), max(m, nu))];
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

__device__ __forceinline__ void quarter(double mag, int k, double& re, double& im) {
  k %= 4;
  if (k < 0) k += 4;
  re = (k == 0) ? mag : ((k == 2) ? -mag : 0.0);
  im = (k == 1) ? mag : ((k == 3) ? -mag : 0.0);
}

// _rotate_multipole_y! (local=false, src/rotate.jl:699-803) / _rotate_local_y!
// (local=true, src/rotate.jl:1014-1113) for degrees [n0, n1]; lanes over (n, m)
__device__ __forceinline__ void rot_y(double* dst, const double* src, const double* Ts, const double* __restrict__ mags,
                                      int n0, int n1, bool lh, bool local) {
  int lane = threadIdx.x & 31;
  int i0 = n0 * (n0 + 1) / 2, i1 = (n1 + 1) * (n1 + 2) / 2;
  for (int i = i0 + lane; i < i1; i += 32) {
    int n, m;
    nm_of(i, n, m);
    int iT = (int)length_Ts(n - 1);
    double v1r = 0, v1i = 0, v2r = 0, v2i = 0;
    for (int mp = -n; mp <= n; ++mp) {
      int amp = mp < 0 ? -mp : mp;
      double T;
      if (mp <= 0)
        T = Ts[iT + T_index(-min(amp, m), max(amp, m))];
      else
        T = Ts[iT + T_index(min(mp, m), max(mp, m))];
      double mag = mags[iT + m * (n + 1) + amp] * T;
      double zr, zi;
      quarter(mag, local ? (m - amp) : (amp - m), zr, zi);
      int iw = n * (n + 1) / 2 + amp;
      {
        double Mr = src[4 * iw], Mi = src[4 * iw + 1];
        if (mp <= 0) {
          Mi = -Mi;
          if (mp & 1) {
            Mr = -Mr;
            Mi = -Mi;
          }
        }
        v1r += Mr * zr - Mi * zi;
        v1i += Mr * zi + Mi * zr;
      }
      if (lh) {
        double Mr = src[4 * iw + 2], Mi = src[4 * iw + 3];
        if (mp <= 0) {
          Mi = -Mi;
          if (mp & 1) {
            Mr = -Mr;
            Mi = -Mi;
          }
        }
        v2r += Mr * zr - Mi * zi;
        v2i += Mr * zi + Mi * zr;
      }
    }
    dst[4 * i] = v1r;
    dst[4 * i + 1] = v1i;
    if (lh) {
      dst[4 * i + 2] = v2r;
      dst[4 * i + 3] = v2i;
    }
  }
}

// translate_multipole_z!, src/translate.jl:6-50
__device__ __forceinline__ void m2m_z(double* dst, const double* src, double t, int P, bool lh) {
  int lane = threadIdx.x & 31;
  double _t = -t;
  for (int i = lane; i < (P + 1) * (P + 2) / 2; i += 32) {
    int n, m;
    nm_of(i, n, m);
    double v1r = 0, v1i = 0, v2r = 0, v2i = 0, f = 1.0, tp = 1.0;
    int k = 1;
    for (int np = n; np >= m; --np) {
      double c = tp / f;
      int iw = np * (np + 1) / 2 + m;
      v1r += c * src[4 * iw];
      v1i += c * src[4 * iw + 1];
      if (lh) {
        v2r += c * src[4 * iw + 2];
        v2i += c * src[4 * iw + 3];
      }
      tp *= _t;
      f *= k;
      k += 1;
    }
    dst[4 * i] = v1r;
    dst[4 * i + 1] = v1i;
    if (lh) {
      dst[4 * i + 2] = v2r;
      dst[4 * i + 3] = v2i;
    }
  }
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

// translate_multipole_to_local_z!, src/translate.jl:181-232 (degrees [n0,n1] of the output,
// source degrees up to Psrc)
__device__ __forceinline__ void m2l_z(double* dst, const double* src, double t, int n0, int n1, int Psrc, bool lh,
                                      int dst_offset_degree = -1) {
  int lane = threadIdx.x & 31;
  double one_over_t = 1 / t;
  int i0 = n0 * (n0 + 1) / 2, i1 = (n1 + 1) * (n1 + 2) / 2;
  for (int i = i0 + lane; i < i1; i += 32) {
    int n, m;
    nm_of(i, n, m);
    double c = m2l_coef0(n, m, one_over_t);
    int n_np = n + m;
    double v1r = 0, v1i = 0, v2r = 0, v2i = 0;
    for (int np = m; np <= Psrc; ++np) {
      int iw = np * (np + 1) / 2 + m;
      v1r += c * src[4 * iw];
      v1i += c * src[4 * iw + 1];
      if (lh) {
        v2r += c * src[4 * iw + 2];
        v2i += c * src[4 * iw + 3];
      }
      n_np += 1;
      c *= n_np * one_over_t;
    }
    int o = (dst_offset_degree >= 0) ? m : i;  // degree-local destination (error prediction)
    dst[4 * o] = v1r;
    dst[4 * o + 1] = v1i;
    if (lh) {
      dst[4 * o + 2] = v2r;
      dst[4 * o + 3] = v2i;
    }
  }
}

// translate_local_z!, src/translate.jl:1851-1891
__device__ __forceinline__ void l2l_z(double* dst, const double* src, double t, int P, bool lh) {
  int lane = threadIdx.x & 31;
  double _t = -t;
  for (int i = lane; i < (P + 1) * (P + 2) / 2; i += 32) {
    int n, m;
    nm_of(i, n, m);
    double v1r = 0, v1i = 0, v2r = 0, v2i = 0, c = 1.0;
    int k = 1;
    for (int np = n; np <= P; ++np) {
      int iw = np * (np + 1) / 2 + m;
      v1r += c * src[4 * iw];
      v1i += c * src[4 * iw + 1];
      if (lh) {
        v2r += c * src[4 * iw + 2];
        v2i += c * src[4 * iw + 3];
      }
      c *= _t / k;
      k += 1;
    }
    dst[4 * i] = v1r;
    dst[4 * i + 1] = v1i;
    if (lh) {
      dst[4 * i + 2] = v2r;
      dst[4 * i + 3] = v2i;
    }
  }
}

// transform_lamb_helmholtz_multipole!, src/translate.jl:52-96 (lane = m)
__device__ __forceinline__ void lh_multipole(double* M, double r, int P) {
  int lane = threadIdx.x & 31;
  for (int m = lane; m <= P; m += 32) {
    int i = P * (P + 1) / 2 + m;
    double cr = M[4 * i + 2], ci = M[4 * i + 3];
    for (int n = P; n >= max(m, 1); --n) {
      double pr = M[4 * i], pi = M[4 * i + 1];
      double xr = cr, xi = ci;
      double a = r * m / (n + 1);
      M[4 * i] = pr + a * xi;
      M[4 * i + 1] = pi - a * xr;
      if (m < n) {
        cr = M[4 * (i - n) + 2];
        ci = M[4 * (i - n) + 3];
      } else {
        cr = 0;
        ci = 0;
      }
      double b = r / n;
      M[4 * i + 2] = xr + b * cr;
      M[4 * i + 3] = xi + b * ci;
      i -= n;
    }
  }
}

// transform_lamb_helmholtz_local!, src/translate.jl:98-142 (lane = m)
__device__ __forceinline__ void lh_local(double* L, double r, int P) {
  int lane = threadIdx.x & 31;
  for (int m = lane; m <= P; m += 32) {
    int i = m * (m + 1) / 2 + m;
    double cr = L[4 * i + 2], ci = L[4 * i + 3];
    for (int n = m; n <= P; ++n) {
      double xr = cr, xi = ci;
      if (n > 0) {
        double pr = L[4 * i], pi = L[4 * i + 1];
        double a = r * m / n;
        L[4 * i] = pr - a * xi;
        L[4 * i + 1] = pi + a * xr;
      }
      if (n < P) {
        cr = L[4 * (i + n + 1) + 2];
        ci = L[4 * (i + n + 1) + 3];
        double b = r / (n + 1);
        L[4 * i + 2] = xr - b * cr;
        L[4 * i + 3] = xi - b * ci;
      }
      i += n + 1;
    }
  }
}

// back_rotate_z! (src/rotate.jl:584-616) into the lane-owned accumulator
__device__ __forceinline__ void back_z_acc(double (&acc)[kSlots][4], const double* src, const double* eim, int P,
                                           bool lh) {
  int lane = threadIdx.x & 31;
  int NH = (P + 1) * (P + 2) / 2;
#pragma unroll
  for (int k = 0; k < kSlots; ++k) {
    int i = lane + 32 * k;
    if (i < NH) {
      int n, m;
      nm_of(i, n, m);
      double er = eim[2 * m], ei = -eim[2 * m + 1];
      for (int s = 0; s <= (lh ? 1 : 0); ++s) {
        double xr = src[4 * i + 2 * s], xi = src[4 * i + 2 * s + 1];
        if (n == 0) {
          acc[k][2 * s] += xr;
          acc[k][2 * s + 1] += xi;
        } else {
          acc[k][2 * s] += xr * er - xi * ei;
          acc[k][2 * s + 1] += xr * ei + xi * er;
        }
      }
    }
  }
}

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

// full operator chain of multipole_to_multipole! (kind 0) / local_to_local! (kind 2)
// for one (source expansion, target centre) pair, accumulated into acc
__device__ __forceinline__ void chain_mm_ll(const WS& w, double (&acc)[kSlots][4], const double* __restrict__ src, double dx, double dy,
                            double dz, int P, bool lh, bool local, const Tab& tb) {
  double r, th, ph;
  sph(dx, dy, dz, r, th, ph);
  angles(w, ph, th, P);
  __syncwarp();
  rot_z(w.w1, src, w.eim, 0, P, lh);
  if ((threadIdx.x & 31) == 0) w.ts[0] = 1.0;
  for (int n = 1; n <= P; ++n) ts_degree(w.ts, tb.Hs, w.cs, n);
  __syncwarp();
  const double* mags = local ? tb.eta : tb.zeta;
  rot_y(w.w2, w.w1, w.ts, mags, 0, P, lh, local);
  __syncwarp();
  if (local)
    l2l_z(w.w1, w.w2, r, P, lh);
  else
    m2m_z(w.w1, w.w2, r, P, lh);
  __syncwarp();
  if (lh) {
    if (local)
      lh_local(w.w1, r, P);
    else
      lh_multipole(w.w1, r, P);
    __syncwarp();
  }
  rot_y(w.w2, w.w1, w.ts, mags, 0, P, lh, local);
  __syncwarp();
  back_z_acc(acc, w.w2, w.eim, P, lh);
  __syncwarp();
}

__device__ __forceinline__ double warp_sum_bcast(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return __shfl_sync(kFull, v, 0);
}

__device__ __forceinline__ double minabs(double x, double y) {
  return x * (fabs(x) <= fabs(y) ? 1.0 : 0.0) + y * (fabs(y) < fabs(x) ? 1.0 : 0.0);
}
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
// Relative}Gradient (:555-829) variants.  Returns the order used; ok = tolerance met.
__device__ __forceinline__ int chain_m2l(const WS& w, double (&acc)[kSlots][4], const double* __restrict__ src, const double* sc,
                         const M2LGeom& g, int p, bool lh, int em, double eps_in, int be, bool& ok, const Tab& tb) {
  const int lane = threadIdx.x & 31;
  double r, th, ph;
  sph(g.tc[0] - sc[0], g.tc[1] - sc[1], g.tc[2] - sc[2], r, th, ph);
  angles(w, ph, th, p);
  __syncwarp();
  int P = p;
  ok = true;
  if (em == FMM_ERROR_NONE) {
    rot_z(w.w1, src, w.eim, 0, p, lh);
    if (lane == 0) w.ts[0] = 1.0;
    for (int n = 1; n <= p; ++n) ts_degree(w.ts, tb.Hs, w.cs, n);
    __syncwarp();
    rot_y(w.w2, w.w1, w.ts, tb.zeta, 0, p, lh, false);
    __syncwarp();
  } else {
    const bool relative = (em == FMM_POWER_RELATIVE_GRADIENT || em == FMM_ROTATED_COEFFICIENTS_RELATIVE_GRADIENT);
    const bool power = (em == FMM_POWER_ABSOLUTE_GRADIENT || em == FMM_POWER_RELATIVE_GRADIENT);
    const double eps = relative ? g.maxinf * eps_in : eps_in;
    double mdx = min_dist_1d(g.tc[0] - sc[0], -g.tbox[0], g.tbox[0]);
    double mdy = min_dist_1d(g.tc[1] - sc[1], -g.tbox[1], g.tbox[1]);
    double mdz = min_dist_1d(g.tc[2] - sc[2], -g.tbox[2], g.tbox[2]);
    double r_mp = sqrt(mdx * mdx + mdy * mdy + mdz * mdz);
    double r_l = g.trad;
    double rinv = 1.0 / r, r_mp_inv = 1.0 / r_mp;
    double r_mp_inv_np2 = r_mp_inv * r_mp_inv * r_mp_inv;
    double r_l_nm1 = 1.0;
    rot_z(w.w1, src, w.eim, 0, 0, lh);
    if (lane == 0) w.ts[0] = 1.0;
    __syncwarp();
    rot_y(w.w2, w.w1, w.ts, tb.zeta, 0, 0, lh, false);
    double n_fact_t_np1 = rinv * rinv, nm1_fact_inv = 1.0, np1_fact = 2.0;
    double Mn0 = tb.Mt[0];
    double mp_phi = sqrt((src[0] * src[0] + src[1] * src[1]) * Mn0 * Mn0);
    const double four_pi_eps = eps * 4 * kPi;
    ok = false;
    for (int n = 1; n <= p; ++n) {
      double pn_phi = 0, pn_chi = 0, Mn0_next = tb.Mt[n * (n + 1) / 2];
      if (power) {
        // multipole power of degree n (rotate_z_n_power!, src/rotate.jl:528-576); weight 1 per m
        double a = 0, b = 0;
        if (lane <= n) {
          int i = n * (n + 1) / 2 + lane;
          double Nt = tb.Mt[i];
          a = (src[4 * i] * src[4 * i] + src[4 * i + 1] * src[4 * i + 1]) * Nt * Nt;
          if (lh) b = (src[4 * i + 2] * src[4 * i + 2] + src[4 * i + 3] * src[4 * i + 3]) * Nt * Nt;
        }
        pn_phi = sqrt(warp_sum_bcast(a));
        pn_chi = sqrt(warp_sum_bcast(b));
      }
      rot_z(w.w1, src, w.eim, n, n, lh);
      ts_degree(w.ts, tb.Hs, w.cs, n);
      __syncwarp();
      rot_y(w.w2, w.w1, w.ts, tb.zeta, n, n, lh, false);
      __syncwarp();
      double eps_mp;
      int in0 = n * (n + 1) / 2;
      if (power) {
        eps_mp = 1.7320508075688772 * mp_phi * r_mp_inv_np2 * np1_fact / Mn0;
        if (lh) eps_mp += 1.7320508075688772 * n * pn_chi * r_mp_inv_np2 * np1_fact / Mn0_next;
      } else {
        double p0 = w.w2[4 * in0];
        double p1r = w.w2[4 * (in0 + 1)], p1i = w.w2[4 * (in0 + 1) + 1];
        eps_mp = (sqrt(p1r * p1r + p1i * p1i) + fabs(p0)) * np1_fact * r_mp_inv_np2;
        if (lh) {
          double c1r = w.w2[4 * (in0 + 1) + 2], c1i = w.w2[4 * (in0 + 1) + 3];
          eps_mp += sqrt(c1r * c1r + c1i * c1i) * np1_fact * r_mp_inv_np2 * r_mp;
        }
      }
      if (eps_mp <= four_pi_eps) {
        double eps_l;
        if (power) {
          // degree n of translate_multipole_to_local_z_n! (src/translate.jl:238-295) + local_power (:455-502)
          m2l_z(w.w3, w.w2, r, n, n, n, lh, n);
          __syncwarp();
          double a = 0, b = 0, Nt = 0;
          if (lane <= n) {
            int m = lane;
            Nt = tb.Lt[in0 + m];
            double pr = w.w3[4 * m], pi = w.w3[4 * m + 1];
            if (lh) {
              double cro = w.w3[4 * m + 2], cio = w.w3[4 * m + 3];
              double crn = (m < n) ? w.w3[4 * (m + 1) + 2] : 0.0;
              double cin = (m < n) ? w.w3[4 * (m + 1) + 3] : 0.0;
              // the reference recurses m downward with chi_{n+1}^m taken from the
              // previous (m+1) entry of the same degree
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
          eps_l = 1.7320508075688772 * lphi * r_l_nm1 * nm1_fact_inv / Ln0;
          if (lh) eps_l += 1.7320508075688772 * n * lchi * r_l_nm1 * r_l * nm1_fact_inv / (Ln0 * n);
          __syncwarp();
        } else {
          // translate_multipole_to_local_z_m01_n, src/translate.jl:302-364 (all lanes, identical)
          double one_over_t = rinv;
          double c = n_fact_t_np1;
          int n_np = n;
          double a0 = 0;
          for (int np = 0; np <= n; ++np) {
            a0 += c * w.w2[4 * (np * (np + 1) / 2)];
            n_np += 1;
            c *= n_np * one_over_t;
          }
          c = n_fact_t_np1 * ((n + 1) * one_over_t);
          n_np = n + 1;
          double b1r = 0, b1i = 0, x1r = 0, x1i = 0;
          for (int np = 1; np <= n; ++np) {
            int iw = np * (np + 1) / 2 + 1;
            b1r += c * w.w2[4 * iw];
            b1i += c * w.w2[4 * iw + 1];
            if (lh) {
              x1r += c * w.w2[4 * iw + 2];
              x1i += c * w.w2[4 * iw + 3];
            }
            n_np += 1;
            c *= n_np * one_over_t;
          }
          if (lh) {
            double t_over_n = r / n;
            b1r -= t_over_n * x1i;
            b1i += t_over_n * x1r;
          }
          eps_l = (fabs(b1r) + fabs(b1i) + fabs(a0)) * r_l_nm1 * nm1_fact_inv;
          if (lh) eps_l += sqrt(x1r * x1r + x1i * x1i) * r_l_nm1 * r_l * nm1_fact_inv;
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
  m2l_z(w.w1, w.w2, r, 0, P, P, lh);
  __syncwarp();
  if (lh) {
    lh_local(w.w1, r, P);
    __syncwarp();
  }
  rot_y(w.w2, w.w1, w.ts, tb.eta, 0, P, lh, true);
  __syncwarp();
  back_z_acc(acc, w.w2, w.eim, P, lh);
  __syncwarp();
  return P;
}

// ---------------------------------------------------------------------------
// kernels

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

__global__ void __launch_bounds__(32 * kWarps) k_m2l(const int* __restrict__ tgt_list, const int* __restrict__ off,
                                                     const int* __restrict__ src_of, int n_targets,
                                                     double* __restrict__ local, const double* __restrict__ multipole,
                                                     const double* __restrict__ tcen, const double* __restrict__ tbox,
                                                     const double* __restrict__ trad,
                                                     const double* __restrict__ maxinf,
                                                     const double* __restrict__ scen, int p, int lh, int em,
                                                     double eps, int be, int* __restrict__ p_used, Tab tb,
                                                     M2LStats stats) {
  extern __shared__ double smem[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.x * kWarps + wid;
  if (b >= n_targets) return;
  WS w = ws_of(smem + wid * ws_doubles(p), p);
  const int t = tgt_list[b];
  const int64_t NH4 = 4 * nh(p);
  M2LGeom g;
  for (int d = 0; d < 3; ++d) {
    g.tc[d] = tcen[3 * t + d];
    g.tbox[d] = tbox[3 * t + d];
  }
  g.trad = trad[t];
  g.maxinf = maxinf[t];
  double acc[kSlots][4];
  acc_zero(acc);
  int pmax = 0;
  bool all_ok = true;
  unsigned long long fl = 0;
  for (int l = off[b]; l < off[b + 1]; ++l) {
    int s = src_of[l];
    double sc[3] = {scen[3 * s], scen[3 * s + 1], scen[3 * s + 2]};
    bool ok;
    int P = chain_m2l(w, acc, multipole + NH4 * s, sc, g, p, lh != 0, em, eps, be, ok, tb);
    if (p_used && lane == 0) p_used[l] = P;
    pmax = max(pmax, P);
    all_ok = all_ok && ok;
    fl += m2l_pair_flops(P, lh != 0);
  }
  acc_store_add(local + NH4 * t, acc, p, lh != 0);
  if (lane == 0) {
    atomicMax(stats.pmax, pmax);
    if (!all_ok) atomicExch(stats.fail, 1);
    atomicAdd(stats.flops, fl);
  }
}

// M2M for one level: warp per parent, loop over its children
__global__ void __launch_bounds__(32 * kWarps) k_m2m(int l0, int l1, const int* __restrict__ child_start,
                                                     const int* __restrict__ n_children,
                                                     const double* __restrict__ scen, double* __restrict__ M, int p,
                                                     int lh, Tab tb) {
  extern __shared__ double smem[];
  const int wid = threadIdx.x >> 5;
  const int k = l0 + blockIdx.x * kWarps + wid;
  if (k >= l1) return;
  int nc = n_children[k];
  if (nc == 0) return;
  WS w = ws_of(smem + wid * ws_doubles(p), p);
  const int64_t NH4 = 4 * nh(p);
  double acc[kSlots][4];
  acc_zero(acc);
  int c0 = child_start[k];
  for (int c = c0; c < c0 + nc; ++c) {
    double dx = scen[3 * k] - scen[3 * c], dy = scen[3 * k + 1] - scen[3 * c + 1], dz = scen[3 * k + 2] - scen[3 * c + 2];
    chain_mm_ll(w, acc, M + NH4 * c, dx, dy, dz, p, lh != 0, false, tb);
  }
  acc_store_add(M + NH4 * k, acc, p, lh != 0);
}

// L2L for one level: warp per child of a level-l parent
__global__ void __launch_bounds__(32 * kWarps) k_l2l(int c0, int c1, const int* __restrict__ parent,
                                                     const double* __restrict__ tcen, double* __restrict__ L, int p,
                                                     int lh, Tab tb) {
  extern __shared__ double smem[];
  const int wid = threadIdx.x >> 5;
  const int c = c0 + blockIdx.x * kWarps + wid;
  if (c >= c1) return;
  WS w = ws_of(smem + wid * ws_doubles(p), p);
  const int64_t NH4 = 4 * nh(p);
  int k = parent[c];
  double acc[kSlots][4];
  acc_zero(acc);
  double dx = tcen[3 * c] - tcen[3 * k], dy = tcen[3 * c + 1] - tcen[3 * k + 1], dz = tcen[3 * c + 2] - tcen[3 * k + 2];
  chain_mm_ll(w, acc, L + NH4 * k, dx, dy, dz, p, lh != 0, true, tb);
  acc_store_add(L + NH4 * c, acc, p, lh != 0);
}

// unit operator: explicit pairs (target k <- source k)
__global__ void __launch_bounds__(32 * kWarps) k_op_pairs(int64_t n, double* __restrict__ tgt,
                                                          const double* __restrict__ tc, const double* __restrict__ src,
                                                          const double* __restrict__ sc, int p, int lh, int local,
                                                          Tab tb) {
  extern __shared__ double smem[];
  const int wid = threadIdx.x >> 5;
  const int64_t k = (int64_t)blockIdx.x * kWarps + wid;
  if (k >= n) return;
  WS w = ws_of(smem + wid * ws_doubles(p), p);
  const int64_t NH4 = 4 * nh(p);
  double acc[kSlots][4];
  acc_zero(acc);
  chain_mm_ll(w, acc, src + NH4 * k, tc[3 * k] - sc[3 * k], tc[3 * k + 1] - sc[3 * k + 1], tc[3 * k + 2] - sc[3 * k + 2],
              p, lh != 0, local != 0, tb);
  acc_store_add(tgt + NH4 * k, acc, p, lh != 0);
}

__global__ void __launch_bounds__(32 * kWarps) k_op_m2l(int64_t n, double* __restrict__ tgt,
                                                        const double* __restrict__ tc, const double* __restrict__ tbox,
                                                        const double* __restrict__ trad,
                                                        const double* __restrict__ maxinf,
                                                        const double* __restrict__ src, const double* __restrict__ sc,
                                                        int p, int lh, int em, double eps, int be, int* p_used, Tab tb) {
  extern __shared__ double smem[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t k = (int64_t)blockIdx.x * kWarps + wid;
  if (k >= n) return;
  WS w = ws_of(smem + wid * ws_doubles(p), p);
  const int64_t NH4 = 4 * nh(p);
  M2LGeom g;
  for (int d = 0; d < 3; ++d) {
    g.tc[d] = tc[3 * k + d];
    g.tbox[d] = tbox ? tbox[3 * k + d] : 0.0;
  }
  g.trad = trad ? trad[k] : 0.0;
  g.maxinf = maxinf ? maxinf[k] : 0.0;
  double acc[kSlots][4];
  acc_zero(acc);
  double s[3] = {sc[3 * k], sc[3 * k + 1], sc[3 * k + 2]};
  bool ok;
  int P = chain_m2l(w, acc, src + NH4 * k, s, g, p, lh != 0, em, eps, be, ok, tb);
  if (p_used && lane == 0) p_used[k] = ok ? P : -P - 1;
  acc_store_add(tgt + NH4 * k, acc, p, lh != 0);
}

// ---------------------------------------------------------------------------
// P2M: body_to_multipole! of Point{Source} / Point{Vortex}
// (src/bodytomultipole.jl:112-139, 283-334, 387-489); warp per leaf, lanes over m
// for the harmonics recursion, lanes over (n, m) for the accumulation.
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

__global__ void __launch_bounds__(32 * kWarps) k_p2m(const int* __restrict__ leaf_index, int n_leaves,
                                                     const int* __restrict__ body_start,
                                                     const int* __restrict__ body_count,
                                                     const double* __restrict__ scen, const double4* __restrict__ pos,
                                                     const double4* __restrict__ str, double* __restrict__ M, int p,
                                                     int kind) {
  extern __shared__ double smem[];
  const int wid = threadIdx.x >> 5;
  const int w = blockIdx.x * kWarps + wid;
  if (w >= n_leaves) return;
  double* h = smem + wid * 2 * nh(p);
  const int b = leaf_index[w];
  const int s0 = body_start[b], cnt = body_count[b];
  double c[3] = {scen[3 * b], scen[3 * b + 1], scen[3 * b + 2]};
  double acc[kSlots][4];
  acc_zero(acc);
  for (int j = 0; j < cnt; ++j) {
    double4 x = pos[s0 + j];
    p2m_body(acc, h, kind, x.x - c[0], x.y - c[1], x.z - c[2], str[s0 + j], p);
  }
  acc_store_add(M + 4 * nh(p) * b, acc, p, kind == FMM_POINT_VORTEX);
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

__device__ void l2p_coefficients(double* C, const double* __restrict__ L, int p, bool lh, bool ps, bool gs, bool hs) {
  // C[(ch * NH + i) * 2 + reim]
  const int NH = (p + 1) * (p + 2) / 2;
  for (int i = threadIdx.x; i < NH; i += blockDim.x) {
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
  __syncthreads();
  // hessian channels from the velocity coefficients ("gradient_n_m"), n <= p-1
  for (int i = threadIdx.x; i < NH; i += blockDim.x) {
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
  __syncthreads();
}

// contract one body: regular harmonics by the reference's column recursion
__device__ void l2p_body(const double* C, int p, double x, double y, double z, bool ps, bool gs, bool hs, double* out) {
  const int NH = (p + 1) * (p + 2) / 2;
  double r, th, ph;
  sph(x, y, z, r, th, ph);
  double sy = sin(th), cx = cos(th);
  double fact = 1.0, pn = 1.0, rhom = 1.0;
  double iei_i = sin(ph + kPi / 2), iei_r = cos(ph + kPi / 2);
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
        rhon /= -(n + m);
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
        pl = (cx * (2 * n + 1) * p1 - (n + m) * p2) / (n - m + 1);
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
  l2p_coefficients(C, L + 4 * nh(p) * b, p, lh != 0, ps != 0, gs != 0, hs != 0);
  const int s0 = body_start[b], cnt = body_count[b];
  const double cx = tcen[3 * b], cy = tcen[3 * b + 1], cz = tcen[3 * b + 2];
  for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
    double4 x = pos[s0 + j];
    l2p_body(C, p, x.x - cx, x.y - cy, x.z - cz, ps != 0, gs != 0, hs != 0, acc13 + 13 * (int64_t)(s0 + j));
  }
}

__global__ void __launch_bounds__(kL2PThreads) k_op_l2p(int64_t n, const double* __restrict__ dx,
                                                        const double* __restrict__ L, int p, int lh, int ps, int gs,
                                                        int hs, double* __restrict__ out13) {
  extern __shared__ double C[];
  l2p_coefficients(C, L, p, lh != 0, ps != 0, gs != 0, hs != 0);
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
  size_t sm = (size_t)kWarps * 2 * nh(p) * sizeof(double);
  allow_smem(k_p2m, sm);
  int g = (int)((s.n_leaves + kWarps - 1) / kWarps);
  note_launch();
  k_p2m<<<g, 32 * kWarps, sm, st>>>(s.leaf_index.ptr, (int)s.n_leaves, s.body_start.ptr, s.body_count.ptr,
                                    s.scenter.ptr, s.pos.ptr, s.str.ptr, s.multipole.ptr, p, kind);
  FMM_CUDA_TRY(cudaGetLastError());
}

void launch_m2m(DevTree& s, int p, bool lh, const DevTables& tb, cudaStream_t st) {
  size_t sm = pair_smem(p);
  allow_smem(k_m2m, sm);
  for (int l = s.n_levels - 2; l >= 0; --l) {
    int l0 = (int)s.levels_start[l], l1 = (int)s.levels_end[l];
    int g = (l1 - l0 + kWarps - 1) / kWarps;
    note_launch();
    k_m2m<<<g, 32 * kWarps, sm, st>>>(l0, l1, s.child_start.ptr, s.n_children.ptr, s.scenter.ptr, s.multipole.ptr, p,
                                      lh ? 1 : 0, tab_of(tb));
  }
  FMM_CUDA_TRY(cudaGetLastError());
}

void launch_m2l(DevTree& t, const DevTree& s, const DevLists& L, int p, bool lh, int em, double eps, int be,
                int* p_used, int* stats, const DevTables& tb, cudaStream_t st) {
  if (L.n_m2l_targets == 0) return;
  size_t sm = pair_smem(p);
  allow_smem(k_m2l, sm);
  int g = (int)((L.n_m2l_targets + kWarps - 1) / kWarps);
  // stats: [0] = max order used, [1] = any tolerance missed, [2..3] = flop count (u64)
  M2LStats S{stats, stats + 1, reinterpret_cast<unsigned long long*>(stats + 2)};
  note_launch();
  k_m2l<<<g, 32 * kWarps, sm, st>>>(L.m2l_tgt.ptr, L.m2l_off.ptr, L.m2l_s.ptr, (int)L.n_m2l_targets, t.local.ptr,
                                    s.multipole.ptr, t.tcenter.ptr, t.tbox.ptr, t.tradius.ptr, t.max_influence.ptr,
                                    s.scenter.ptr, p, lh ? 1 : 0, em, eps, be, p_used, tab_of(tb), S);
  FMM_CUDA_TRY(cudaGetLastError());
}

void launch_l2l(DevTree& t, int p, bool lh, const DevTables& tb, cudaStream_t st) {
  size_t sm = pair_smem(p);
  allow_smem(k_l2l, sm);
  for (int l = 1; l < t.n_levels; ++l) {
    int c0 = (int)t.levels_start[l], c1 = (int)t.levels_end[l];
    int g = (c1 - c0 + kWarps - 1) / kWarps;
    note_launch();
    k_l2l<<<g, 32 * kWarps, sm, st>>>(c0, c1, t.parent.ptr, t.tcenter.ptr, t.local.ptr, p, lh ? 1 : 0,
                                      tab_of(tb));
  }
  FMM_CUDA_TRY(cudaGetLastError());
}

void launch_l2p(DevTree& t, int p, bool lh, bool ps, bool gs, bool hs, double* acc13, cudaStream_t st) {
  if (t.n_leaves == 0) return;
  size_t sm = l2p_smem(p);
  allow_smem(k_l2p, sm);
  note_launch();
  k_l2p<<<(int)t.n_leaves, kL2PThreads, sm, st>>>(t.leaf_index.ptr, t.body_start.ptr, t.body_count.ptr,
                                                   t.tcenter.ptr, t.pos.ptr, t.local.ptr, p, lh ? 1 : 0,
                                                   ps ? 1 : 0, gs ? 1 : 0, hs ? 1 : 0, acc13);
  FMM_CUDA_TRY(cudaGetLastError());
}

void launch_op_m2m(int64_t n, double* target, const double* tc, const double* src, const double* sc, int p, bool lh,
                   bool local, const DevTables& tb, cudaStream_t st) {
  if (n == 0) return;
  size_t sm = pair_smem(p);
  allow_smem(k_op_pairs, sm);
  note_launch();
  k_op_pairs<<<(int)((n + kWarps - 1) / kWarps), 32 * kWarps, sm, st>>>(n, target, tc, src, sc, p, lh ? 1 : 0,
                                                                        local ? 1 : 0, tab_of(tb));
  FMM_CUDA_TRY(cudaGetLastError());
}

void launch_op_m2l(int64_t n, double* target, const double* tc, const double* tbox, const double* trad,
                   const double* maxinf, const double* src, const double* sc, int p, bool lh, int em, double eps,
                   int be, int* p_used, const DevTables& tb, cudaStream_t st) {
  if (n == 0) return;
  size_t sm = pair_smem(p);
  allow_smem(k_op_m2l, sm);
  note_launch();
  k_op_m2l<<<(int)((n + kWarps - 1) / kWarps), 32 * kWarps, sm, st>>>(n, target, tc, tbox, trad, maxinf, src, sc, p,
                                                                      lh ? 1 : 0, em, eps, be, p_used, tab_of(tb));
  FMM_CUDA_TRY(cudaGetLastError());
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

// pair_m2l.cuh -- thread-per-pair M2L for low expansion orders.
//
// At orders P <= 3 an expansion holds at most 10 coefficients, so a warp
// spread over one pair's coefficients would idle most lanes.  Here one thread
// carries one (target, source) pair through the reference's point-and-shoot
// chain (src/translate.jl:519-550):
//   rotate_z (src/rotate.jl:448-483) -> Wigner matrices at beta from the pi/2
//   table (update_Ts_n!, src/rotate.jl:363-441) -> rotate_y with the zeta
//   magnitudes (src/rotate.jl:699-803) -> coaxial translation
//   (translate_multipole_to_local_z!, src/translate.jl:181-232) -> [Lamb-
//   Helmholtz re-centring, src/translate.jl:98-142] -> rotate_y back with the
//   eta magnitudes (src/rotate.jl:1014-1113) -> back_rotate_z
//   (src/rotate.jl:584-616)
// with P a template parameter, so every loop unrolls, every table offset is a
// constant (the table reads are warp-uniform broadcasts) and the expansions
// live in registers.
//
// The angles come from the translation vector directly (cos phi = x / rho,
// sin theta = rho / r, ...) instead of atan2/acos followed by cos/sin; the two
// agree to rounding.  The e^{i m phi} and cos/sin(nu beta) recurrences are the
// reference's.
#pragma once
#include "context.cuh"

namespace fmmb {
namespace eng {

template <int P, bool LH>
struct PairM2L {
  static constexpr int NH = (P + 1) * (P + 2) / 2;
  static constexpr int NC = LH ? 4 : 2;  // doubles per coefficient: phi (re, im) [, chi (re, im)]
  static constexpr int NT = (P + 1) * (P + 2) * (2 * P + 3) / 6;

  static __device__ __forceinline__ constexpr int hi(int n, int m) { return n * (n + 1) / 2 + m; }
  static __device__ __forceinline__ constexpr int lenH(int n) { return n < 0 ? 0 : (n + 1) * (n + 2) * (n + 3) / 6; }
  static __device__ __forceinline__ constexpr int lenT(int n) {
    return n < 0 ? 0 : (n + 1) * (n + 2) * (2 * n + 3) / 6;
  }
  static __device__ __forceinline__ constexpr int Hix(int a, int b) { return b * (b + 1) / 2 + a; }
  static __device__ __forceinline__ constexpr int Tix(int a, int b) { return b * b + a + b; }
  static __device__ __forceinline__ constexpr int imin(int a, int b) { return a < b ? a : b; }
  static __device__ __forceinline__ constexpr int imax(int a, int b) { return a < b ? b : a; }

  // i^k * mag
  static __device__ __forceinline__ void quarter(double mag, int k, double& re, double& im) {
    k %= 4;
    if (k < 0) k += 4;
    re = (k == 0) ? mag : ((k == 2) ? -mag : 0.0);
    im = (k == 1) ? mag : ((k == 3) ? -mag : 0.0);
  }

  // Wigner matrices of degrees 0..P at beta (cs = cos, sin of nu beta), layout of update_Ts!
  static __device__ __forceinline__ void wigner(double (&T)[NT], const double* __restrict__ Hs,
                                                const double (&cb)[P + 1], const double (&sb)[P + 1]) {
    T[0] = 1.0;
#pragma unroll
    for (int n = 1; n <= P; ++n) {
      const double* H = Hs + lenH(n - 1);
      const double _1_n = (n & 1) ? -1.0 : 1.0;
#pragma unroll
      for (int m = 0; m <= n; ++m) {
#pragma unroll
        for (int mp = 0; mp <= m; ++mp) {
          const double H_m_0 = __ldg(H + Hix(0, m));
          const double H_mp_0 = __ldg(H + Hix(0, mp));
          const double _1_mp_odd = (mp & 1) ? -1.0 : 1.0;
          const double _1_n_mp = (mp & 1) ? -_1_n : _1_n;
          const int m_mp = m + mp;
          const bool even = (m_mp & 1) == 0;
          const int mm = (m_mp & 1) ? m_mp + 1 : m_mp;
          const double scalar = ((mm >> 1) & 1) == 0 ? 1.0 : -1.0;
          double vp = 0, vn = 0;
          double _1_n_mp_nu = -_1_n_mp;
#pragma unroll
          for (int nu = 1; nu <= n; ++nu) {
            const double sc = even ? scalar * cb[nu] : scalar * sb[nu];
            const double val = __ldg(H + Hix(imin(mp, nu), imax(mp, nu))) * __ldg(H + Hix(imin(m, nu), imax(m, nu))) * sc;
            vp += val;
            vn += val * _1_n_mp_nu * _1_mp_odd;
            _1_n_mp_nu = -_1_n_mp_nu;
          }
          vp *= 2.0;
          vn *= 2.0;
          const double s0 = even ? scalar : 0.0;
          const double val = H_m_0 * H_mp_0 * s0;
          vp += val;
          vn += val * _1_n_mp * _1_mp_odd;
          T[lenT(n - 1) + Tix(mp, m)] = vp;
          T[lenT(n - 1) + Tix(-mp, m)] = vn;
        }
      }
    }
  }

  // rotate_y of every degree: out(n, m) = sum over m' of T * mag * i^k * in(n, m')
  // (in(n, -a) = (-1)^a conj(in(n, a))); local selects eta and the sign of k
  static __device__ __forceinline__ void rot_y(double (&out)[NH * NC], const double (&in)[NH * NC],
                                               const double (&T)[NT], const double* __restrict__ mags, bool local) {
#pragma unroll
    for (int n = 0; n <= P; ++n) {
      const int iT = lenT(n - 1);
#pragma unroll
      for (int m = 0; m <= n; ++m) {
        double v1r = 0, v1i = 0, v2r = 0, v2i = 0;
#pragma unroll
        for (int mp = -n; mp <= n; ++mp) {
          const int amp = mp < 0 ? -mp : mp;
          const double t = (mp <= 0) ? T[iT + Tix(-imin(amp, m), imax(amp, m))] : T[iT + Tix(imin(mp, m), imax(mp, m))];
          const double mag = __ldg(mags + iT + m * (n + 1) + amp) * t;
          double zr, zi;
          quarter(mag, local ? (m - amp) : (amp - m), zr, zi);
          const int iw = hi(n, amp);
          double Mr = in[NC * iw], Mi = in[NC * iw + 1];
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
            double Cr = in[(NC * iw + 2) % (NH * NC)], Ci = in[(NC * iw + 3) % (NH * NC)];
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
        const int i = hi(n, m);
        out[NC * i] = v1r;
        out[NC * i + 1] = v1i;
        if (LH) {
          out[(NC * i + 2) % (NH * NC)] = v2r;
          out[(NC * i + 3) % (NH * NC)] = v2i;
        }
      }
    }
  }

  // one pair: acc += M2L(src multipole at sc -> target centre tc)
  static __device__ __forceinline__ void run(double (&acc)[NH * NC], const double* __restrict__ src, double x,
                                             double y, double z, const Tab& tb) {
    // geometry (cartesian_to_spherical, src/rotate.jl:9-21, in cos/sin form)
    const double x2y2 = x * x + y * y;
    const double r2 = x2y2 + z * z;
    const double r = (r2 == 0.0) ? r2 : sqrt(r2);
    double cph = 1.0, sph = 0.0, cth, sth;
    if (x2y2 > 0) {
      const double rho = sqrt(x2y2);
      cph = x / rho;
      sph = y / rho;
      cth = z / r;
      sth = rho / r;
    } else {
      cth = (r > 0 && z < 0) ? -1.0 : 1.0;
      sth = 0.0;
    }
    double er[P + 1], ei[P + 1], cb[P + 1], sb[P + 1];
    {
      double cr = 1.0, ci = 0.0;
#pragma unroll
      for (int m = 0; m <= P; ++m) {
        er[m] = cr;
        ei[m] = ci;
        const double t = cr;
        cr = cr * cph - ci * sph;
        ci = t * sph + ci * cph;
      }
      double c = 1.0, s = 0.0;
      cb[0] = 1.0;
      sb[0] = 0.0;
#pragma unroll
      for (int nu = 1; nu <= P; ++nu) {
        const double cn = cth * c - sth * s;
        const double sn = sth * c + cth * s;
        cb[nu] = cn;
        sb[nu] = sn;
        c = cn;
        s = sn;
      }
    }
    // rotate_z (multipole): a = M e^{i m phi}
    double a[NH * NC];
#pragma unroll
    for (int n = 0; n <= P; ++n)
#pragma unroll
      for (int m = 0; m <= n; ++m) {
        const int i = hi(n, m);
        const double2 u = __ldg(reinterpret_cast<const double2*>(src) + 2 * i);
        a[NC * i] = n == 0 ? u.x : u.x * er[m] - u.y * ei[m];
        a[NC * i + 1] = n == 0 ? u.y : u.x * ei[m] + u.y * er[m];
        if (LH) {
          const double2 v = __ldg(reinterpret_cast<const double2*>(src) + 2 * i + 1);
          a[(NC * i + 2) % (NH * NC)] = n == 0 ? v.x : v.x * er[m] - v.y * ei[m];
          a[(NC * i + 3) % (NH * NC)] = n == 0 ? v.y : v.x * ei[m] + v.y * er[m];
        }
      }
    double T[NT];
    wigner(T, tb.Hs, cb, sb);
    double b[NH * NC];
    rot_y(b, a, T, tb.zeta, false);
    // coaxial multipole -> local: c(n, m) = sum_{n' >= m} (n + n')! / t^(n + n' + 1) b(n', m)
    const double one_over_t = 1 / r;
#pragma unroll
    for (int n = 0; n <= P; ++n)
#pragma unroll
      for (int m = 0; m <= n; ++m) {
        double c = one_over_t;
#pragma unroll
        for (int k = 0; k < n; ++k) c *= (k + 1) * one_over_t;
        int nm = n;
#pragma unroll
        for (int j = 0; j < m; ++j) {
          nm += 1;
          c *= nm * one_over_t;
        }
        int n_np = n + m;
        double v1r = 0, v1i = 0, v2r = 0, v2i = 0;
#pragma unroll
        for (int np = m; np <= P; ++np) {
          const int iw = hi(np, m);
          v1r += c * b[NC * iw];
          v1i += c * b[NC * iw + 1];
          if (LH) {
            v2r += c * b[(NC * iw + 2) % (NH * NC)];
            v2i += c * b[(NC * iw + 3) % (NH * NC)];
          }
          n_np += 1;
          c *= n_np * one_over_t;
        }
        const int i = hi(n, m);
        a[NC * i] = v1r;
        a[NC * i + 1] = v1i;
        if (LH) {
          a[(NC * i + 2) % (NH * NC)] = v2r;
          a[(NC * i + 3) % (NH * NC)] = v2i;
        }
      }
    if (LH) {
      // transform_lamb_helmholtz_local! (src/translate.jl:98-142)
#pragma unroll
      for (int m = 0; m <= P; ++m) {
        int i = hi(m, m);
        double cr = a[(NC * i + 2) % (NH * NC)], ci = a[(NC * i + 3) % (NH * NC)];
#pragma unroll
        for (int n = m; n <= P; ++n) {
          const double xr = cr, xi = ci;
          if (n > 0) {
            const double pr = a[NC * i], pi = a[NC * i + 1];
            const double f = r * m / n;
            a[NC * i] = pr - f * xi;
            a[NC * i + 1] = pi + f * xr;
          }
          if (n < P) {
            cr = a[(NC * (i + n + 1) + 2) % (NH * NC)];
            ci = a[(NC * (i + n + 1) + 3) % (NH * NC)];
            const double f = r / (n + 1);
            a[(NC * i + 2) % (NH * NC)] = xr - f * cr;
            a[(NC * i + 3) % (NH * NC)] = xi - f * ci;
          }
          i += n + 1;
        }
      }
    }
    rot_y(b, a, T, tb.eta, true);
    // back_rotate_z into the accumulator
#pragma unroll
    for (int n = 0; n <= P; ++n)
#pragma unroll
      for (int m = 0; m <= n; ++m) {
        const int i = hi(n, m);
        const double cr = er[m], ci = -ei[m];
        const double xr = b[NC * i], xi = b[NC * i + 1];
        acc[NC * i] += n == 0 ? xr : xr * cr - xi * ci;
        acc[NC * i + 1] += n == 0 ? xi : xr * ci + xi * cr;
        if (LH) {
          const double yr = b[(NC * i + 2) % (NH * NC)], yi = b[(NC * i + 3) % (NH * NC)];
          acc[(NC * i + 2) % (NH * NC)] += n == 0 ? yr : yr * cr - yi * ci;
          acc[(NC * i + 3) % (NH * NC)] += n == 0 ? yi : yr * ci + yi * cr;
        }
      }
  }
};

}  // namespace eng
}  // namespace fmmb

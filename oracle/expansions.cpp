// expansions.cpp -- TEST INFRASTRUCTURE ONLY (see fmm_oracle.h).
// FP64 restatement of the reference's expansion math: constant tables, solid
// harmonics, P2M, rotations, coaxial translations, Lamb-Helmholtz transforms,
// M2M / M2L (plain and error-controlled) / L2L and L2P.
#include "internal.h"
#include <algorithm>
#include <cstring>
#include <mutex>

namespace orc {

static const double PI = 3.141592653589793;
static const double ONE_OVER_4PI = 1.0 / (4.0 * 3.141592653589793);  // src/FastMultipole.jl:13
static const double SQRT3 = 1.7320508075688772;                    // src/FastMultipole.jl:17
static const double LOCAL_ERROR_SAFETY = 2.0;                        // src/FastMultipole.jl:18

// ---------------------------------------------------------------------------
// exact factorial -> nearest double (Float64(factorial(big(k))), src/translate.jl:396)
static double factorial_to_double(int k) {
  std::vector<uint32_t> limb(1, 1u);
  for (int f = 2; f <= k; ++f) {
    uint64_t carry = 0;
    for (auto& l : limb) {
      uint64_t v = (uint64_t)l * (uint64_t)f + carry;
      l = (uint32_t)v;
      carry = v >> 32;
    }
    if (carry) limb.push_back((uint32_t)carry);
  }
  int top = (int)limb.size() - 1;
  int nbits = top * 32 + (32 - __builtin_clz(limb[top]));
  if (nbits <= 53) {
    double v = 0;
    for (int i = top; i >= 0; --i) v = v * 4294967296.0 + limb[i];
    return v;
  }
  int shift = nbits - 64;  // take the top 64 bits
  auto bit = [&](int b) -> uint64_t { return (limb[b / 32] >> (b % 32)) & 1u; };
  uint64_t topbits = 0;
  for (int b = nbits - 1; b >= shift; --b) topbits = (topbits << 1) | bit(b);
  bool sticky = false;
  for (int b = 0; b < shift; ++b) sticky |= bit(b) != 0;
  uint64_t low = topbits & 0x7FF, mant = topbits >> 11;
  if (low > 0x400 || (low == 0x400 && (sticky || (mant & 1)))) mant++;
  return std::ldexp((double)mant, shift + 11);
}

// compute_Pnms, src/rotate.jl:99-117
void compute_Pnms(int p, double s, double c, double* P) {
  double Pn0 = 1.0, fact = 1.0;
  for (int m = 0; m <= p; ++m) {
    double Pnm = Pn0;
    P[hidx(m, m)] = Pnm;
    double tmp1 = Pnm;
    Pnm = c * (2 * m + 1) * tmp1;
    for (int n = m + 1; n <= p; ++n) {
      P[hidx(n, m)] = Pnm;
      double tmp2 = tmp1;
      tmp1 = Pnm;
      Pnm = (c * (2 * n + 1) * tmp1 - (n + m) * tmp2) / (n - m + 1);
    }
    Pn0 = -Pn0 * fact * s;
    fact += 2;
  }
}

// compute_Hs!, src/rotate.jl:119-203 (Wigner d at beta, normalized; H_index layout)
void compute_Hs(double* Hs, double beta, int n_start, int n_end) {
  double sb = std::sin(beta), cb = std::cos(beta);
  std::vector<double> P(nh(n_end + 1));
  compute_Pnms(n_end + 1, sb, cb, P.data());
  std::vector<double> H_np1(n_end + 2), bnms(2 * (n_end + 1) + 1), dnms(n_end + 1);
  int64_t i_start = length_Hs(n_start - 1);
  for (int n = n_start; n <= n_end; ++n) {
    double* H = Hs + i_start;
    {  // H_n_0m
      double sgn = 1, fact = 1;
      for (int m = 0; m <= n; ++m) {
        H[H_index(0, m)] = sgn * fact * P[hidx(n, m)];
        sgn = -sgn;
        fact /= std::sqrt((double)((n + m + 1) * (n - m)));
      }
    }
    {  // H_np1_0m
      double sgn = 1, fact = 1;
      for (int m = 0; m <= n + 1; ++m) {
        H_np1[m] = sgn * fact * P[hidx(n + 1, m)];
        sgn = -sgn;
        fact /= std::sqrt((double)((n + 1 - m) * (n + m + 2)));
      }
    }
    int b_n = n + 1;  // b_np1_m, stored at bnms[b_n + m]
    for (int m = -b_n; m <= b_n; ++m) {
      double v = std::sqrt((double)(b_n - m - 1) / (double)(2 * b_n - 1) * (double)(b_n - m) /
                           (double)(2 * b_n + 1));
      bnms[b_n + m] = m < 0 ? -v : v;
    }
    double one_m_cb_2 = (1.0 - cb) / 2, one_p_cb_2 = (1.0 + cb) / 2;
    for (int m = 1; m <= n; ++m) {  // H_n_1m
      double b_np1__mm1 = bnms[b_n - m - 1];
      double b_np1_mm1 = bnms[b_n + m - 1];
      double b_np1_0 = bnms[b_n];
      double a_n_m = std::sqrt((double)(n + 1 + m) / (double)(2 * n + 1) * (double)(n + 1 - m) /
                               (double)(2 * n + 3));
      H[H_index(1, m)] = (b_np1__mm1 * one_m_cb_2 * H_np1[m + 1] - b_np1_mm1 * one_p_cb_2 * H_np1[m - 1] -
                          a_n_m * sb * H_np1[m]) / b_np1_0;
    }
    for (int m = 0; m <= n; ++m) dnms[m] = std::sqrt((double)((n - m) * (n + m + 1))) / 2;
    for (int mp = 1; mp <= n - 1; ++mp) {  // H_n_mp+1_m
      for (int m = mp + 1; m <= n - 1; ++m) {
        double val = dnms[mp - 1] * H[H_index(mp - 1, m)] - dnms[m - 1] * H[H_index(mp, m - 1)] +
                     dnms[m] * H[H_index(mp, m + 1)];
        H[H_index(mp + 1, m)] = val / dnms[mp];
      }
      int m = n;
      double val = dnms[mp - 1] * H[H_index(mp - 1, m)] - dnms[m - 1] * H[H_index(mp, m - 1)];
      H[H_index(mp + 1, m)] = val / dnms[mp];
    }
    i_start += length_H(n);
  }
}

// update_zeta_s_mag!, src/rotate.jl:660-689
void zeta_mag(double* z, int n_end) {
  z[0] = 1.0;
  for (int n = 1; n <= n_end; ++n) {
    double* zn = z + length_Ts(n - 1);
    int64_t i = 0;
    double mag_m = 1.0;
    for (int m = 0; m <= n; ++m) {
      double mag_mp = mag_m;
      for (int mp = 0; mp <= n; ++mp) {
        zn[i++] = mag_mp;
        double num = n + mp + 1, den = (mp + 1 < n) ? n - mp : 1;
        mag_mp *= std::sqrt(num / den);
      }
      double num = (m < n - 1) ? n - m : 1, den = n + m + 1;
      mag_m *= std::sqrt(num / den);
    }
  }
}

// update_eta_s_mag!, src/rotate.jl:975-1004
void eta_mag(double* e, int n_end) {
  e[0] = 1.0;
  for (int n = 1; n <= n_end; ++n) {
    double* en = e + length_Ts(n - 1);
    int64_t i = 0;
    double mag_m = 1.0;
    for (int m = 0; m <= n; ++m) {
      double mag_mp = mag_m;
      for (int mp = 0; mp <= n; ++mp) {
        en[i++] = mag_mp;
        double num = (mp + 1 < n) ? n - mp : 1, den = n + mp + 1;
        mag_mp *= std::sqrt(num / den);
      }
      double num = n + m + 1, den = (m < n - 1) ? n - m : 1;
      mag_m *= std::sqrt(num / den);
    }
  }
}

// update_M~! / update_L~!, src/translate.jl:386-448
void power_norms(double* Mt, double* Lt, int n_end) {
  int64_t i = 0;
  for (int n = 0; n <= n_end; ++n)
    for (int m = 0; m <= n; ++m, ++i) {
      double a = factorial_to_double(n + m), b = factorial_to_double(n - m);
      Mt[i] = (n == 0) ? 1.0 : std::sqrt(a * b / (2 * n + 1));
      Lt[i] = (n == 0) ? 1.0 : std::sqrt(1 / (a * b * (2 * n + 1)));
    }
}

static std::mutex g_tab_mutex;
static Tables g_tab;

const Tables& tables(int p) {
  std::lock_guard<std::mutex> lock(g_tab_mutex);
  int want = std::max(p, 21);  // module load precomputes to 20th order (src/FastMultipole.jl:137-148)
  if (g_tab.p < want) {
    g_tab.p = want;
    g_tab.Hs.assign(length_Hs(want), 0.0);
    g_tab.Hs[0] = 1.0;
    compute_Hs(g_tab.Hs.data(), PI / 2, 1, want);
    g_tab.zeta.assign(length_Ts(want), 0.0);
    zeta_mag(g_tab.zeta.data(), want);
    g_tab.eta.assign(length_Ts(want), 0.0);
    eta_mag(g_tab.eta.data(), want);
    g_tab.Mt.assign(nh(want), 0.0);
    g_tab.Lt.assign(nh(want), 0.0);
    power_norms(g_tab.Mt.data(), g_tab.Lt.data(), want);
  }
  return g_tab;
}

// ---------------------------------------------------------------------------
// regular_harmonics!, src/harmonics.jl:13-58
void regular_harmonics(double* h, double rho, double theta, double phi, int p) {
  double y = std::sin(theta), x = std::cos(theta);
  double fact = 1.0, pn = 1.0, rhom = 1.0;
  double i_ei_imag = std::sin(phi + PI / 2), i_ei_real = std::cos(phi + PI / 2);
  double er = 1.0, ei = 0.0;
  for (int m = 0; m <= p; ++m) {
    double pl = pn;
    int64_t i = hidx(m, m);
    double rhom_p = rhom * pl;
    h[4 * i] = rhom_p * er;
    h[4 * i + 1] = rhom_p * ei;
    double p1 = pl;
    pl = x * (2 * m + 1) * p1;
    rhom *= rho;
    double rhon = rhom;
    for (int n = m + 1; n <= p; ++n) {
      i = hidx(n, m);
      rhon /= -(n + m);
      double rhon_p = rhon * pl;
      h[4 * i] = rhon_p * er;
      h[4 * i + 1] = rhon_p * ei;
      double p2 = p1;
      p1 = pl;
      pl = (x * (2 * n + 1) * p1 - (n + m) * p2) / (n - m + 1);
      rhon *= rho;
    }
    rhom /= -(2 * m + 2) * (2 * m + 1);
    pn = -pn * fact * y;
    fact += 2;
    double tr = er, ti = ei;
    er = tr * i_ei_real - ti * i_ei_imag;
    ei = tr * i_ei_imag + ti * i_ei_real;
  }
}

// irregular_harmonics!, src/harmonics.jl:64-104
void irregular_harmonics(double* h, double rho, double theta, double phi, int p) {
  double y = std::sin(theta), x = std::cos(theta);
  double fact = 1.0, pn = 1.0;
  double one_over_rho = 1.0 / rho, rhom = one_over_rho;
  double i_ei_imag = std::sin(phi + PI / 2), i_ei_real = std::cos(phi + PI / 2);
  double er = 1.0, ei = 0.0;
  for (int m = 0; m <= p; ++m) {
    double pl = pn;
    int64_t i = hidx(m, m);
    double rhom_p = rhom * pl;
    h[4 * i] = rhom_p * er;
    h[4 * i + 1] = rhom_p * ei;
    double p1 = pl;
    pl = x * (2 * m + 1) * p1;
    rhom *= -one_over_rho;
    double rhon = -rhom;
    for (int n = m + 1; n <= p; ++n) {
      i = hidx(n, m);
      double rhon_p = rhon * pl;
      h[4 * i] = rhon_p * er;
      h[4 * i + 1] = rhon_p * ei;
      double p2 = p1;
      p1 = pl;
      pl = (x * (2 * n + 1) * p1 - (n + m) * p2) / (n - m + 1);
      rhon *= one_over_rho * (n - m + 1);
    }
    pn *= -fact * y;
    fact += 2;
    double tr = er, ti = ei;
    er = tr * i_ei_real - ti * i_ei_imag;
    ei = tr * i_ei_imag + ti * i_ei_real;
  }
}

// cartesian_to_spherical, src/rotate.jl:9-21
void cartesian_to_spherical(double x, double y, double z, double& r, double& theta, double& phi) {
  double x2y2 = x * x + y * y;
  double r2 = x2y2 + z * z;
  r = (r2 == 0.0) ? r2 : std::sqrt(r2);
  double z_r = z / r;
  if (r > 0)
    theta = x2y2 > 0 ? std::acos(z_r) : PI * (z < 0 ? 1.0 : 0.0);
  else
    theta = 0.0;
  phi = (x2y2 == 0.0) ? 0.0 : std::atan2(y, x);
}

// ---------------------------------------------------------------------------
// Wigner matrices at angle beta from H(pi/2): update_Ts_n!, src/rotate.jl:363-441
static double get_scalar(int m_mp) {  // src/rotate.jl:235-242
  if (m_mp & 1) m_mp += 1;
  return ((m_mp >> 1) % 2 == 0) ? 1.0 : -1.0;
}

static double ts_degree(double* T, const double* H, double sb, double cb, double _1_n, int n) {
  for (int m = 0; m <= n; ++m) {
    double H_m_0 = H[H_index(0, m)];
    double _1_mp_odd = 1.0;
    int m_mp = m;
    double _1_n_mp = _1_n;
    for (int mp = 0; mp <= m; ++mp) {
      double H_mp_0 = H[H_index(0, mp)];
      double vp = 0, vn = 0, s_prev = 0.0, c_prev = 1.0;
      bool even = (m_mp % 2) == 0;
      double scalar = get_scalar(m_mp);
      double _1_n_mp_nu = -_1_n_mp;
      for (int nu = 1; nu <= n; ++nu) {
        double c = cb * c_prev - sb * s_prev;
        double s = sb * c_prev + cb * s_prev;
        double sc = even ? scalar * c : scalar * s;
        double H_mp_nu = H[H_index(std::min(mp, nu), std::max(mp, nu))];
        double H_m_nu = H[H_index(std::min(m, nu), std::max(m, nu))];
        double val = H_mp_nu * H_m_nu * sc;
        vp += val;
        vn += val * _1_n_mp_nu * _1_mp_odd;
        c_prev = c;
        s_prev = s;
        _1_n_mp_nu = -_1_n_mp_nu;
      }
      vp *= 2.0;
      vn *= 2.0;
      scalar = even ? scalar : 0.0;
      double val = H_m_0 * H_mp_0 * scalar;
      vp += val;
      vn += val * _1_n_mp * _1_mp_odd;
      T[T_index(mp, m)] = vp;
      T[T_index(-mp, m)] = vn;
      _1_n_mp = -_1_n_mp;
      _1_mp_odd = -_1_mp_odd;
      m_mp += 1;
    }
  }
  return -_1_n;
}

// update_Ts!, src/rotate.jl:260-346
void update_Ts(double* Ts, const double* Hs, double beta, int p) {
  double sb = std::sin(beta), cb = std::cos(beta);
  double _1_n = -1.0;
  Ts[0] = 1.0;
  for (int n = 1; n <= p; ++n) _1_n = ts_degree(Ts + length_Ts(n - 1), Hs + length_Hs(n - 1), sb, cb, _1_n, n);
}

// z rotation: update_eimphis! + rotate_z!, src/rotate.jl:25-37, 448-483
static void update_eim(double* eim, double phi, int P) {
  double ei = std::sin(phi), er = std::cos(phi);
  double cr = 1.0, ci = 0.0;
  for (int m = 0; m <= P; ++m) {
    eim[2 * m] = cr;
    eim[2 * m + 1] = ci;
    double t = cr;
    cr = cr * er - ci * ei;
    ci = t * ei + ci * er;
  }
}

static void rotate_z_degree(double* rot, const double* src, const double* eim, int n, bool lh) {
  for (int m = 0; m <= n; ++m) {
    int64_t i = hidx(n, m);
    double er = eim[2 * m], ei = eim[2 * m + 1];
    for (int set = 0; set <= (lh ? 1 : 0); ++set) {
      double xr = ER(src, set, i), xi = EI(src, set, i);
      if (n == 0) {
        ER(rot, set, i) = xr;
        EI(rot, set, i) = xi;
      } else {
        ER(rot, set, i) = xr * er - xi * ei;
        EI(rot, set, i) = xr * ei + xi * er;
      }
    }
  }
}

// back_rotate_z!, src/rotate.jl:584-616 (accumulates)
static void back_rotate_z(double* target, const double* src, const double* eim, int P, bool lh) {
  for (int n = 0; n <= P; ++n)
    for (int m = 0; m <= n; ++m) {
      int64_t i = hidx(n, m);
      double er = eim[2 * m], ei = -eim[2 * m + 1];
      for (int set = 0; set <= (lh ? 1 : 0); ++set) {
        double xr = ER(src, set, i), xi = EI(src, set, i);
        if (n == 0) {
          ER(target, set, i) += xr;
          EI(target, set, i) += xi;
        } else {
          ER(target, set, i) += xr * er - xi * ei;
          EI(target, set, i) += xr * ei + xi * er;
        }
      }
    }
}

// sign patterns zeta_sign / eta_sign, src/rotate.jl:643-655, 958-970
static inline void quarter_sign(double mag, int k, double& re, double& im) {
  k %= 4;
  if (k < 0) k += 4;
  switch (k) {
    case 0: re = mag; im = 0.0; break;
    case 1: re = 0.0; im = mag; break;
    case 2: re = -mag; im = 0.0; break;
    default: re = 0.0; im = -mag; break;
  }
}

// one degree of _rotate_multipole_y! (local=false, src/rotate.jl:699-803) or
// _rotate_local_y! (local=true, src/rotate.jl:1014-1113)
static void rotate_y_degree(double* rot, const double* src, const double* Ts, const double* mags, int n,
                            bool lh, bool local) {
  int64_t iT = length_Ts(n - 1);
  for (int m = 0; m <= n; ++m) {
    double v1r = 0, v1i = 0, v2r = 0, v2i = 0;
    for (int mp = -n; mp <= n; ++mp) {
      double T;
      if (mp <= 0) {
        int i1 = std::min(-mp, m), i2 = std::max(-mp, m);
        T = Ts[iT + T_index(-i1, i2)];
      } else {
        int i1 = std::min(mp, m), i2 = std::max(mp, m);
        T = Ts[iT + T_index(i1, i2)];
      }
      int amp = mp < 0 ? -mp : mp;
      double mag = mags[iT + (int64_t)m * (n + 1) + amp] * T;
      double zr, zi;
      quarter_sign(mag, local ? (m - amp) : (amp - m), zr, zi);
      int64_t iw = hidx(n, amp);
      for (int set = 0; set <= (lh ? 1 : 0); ++set) {
        double Mr = ER(src, set, iw), Mi = EI(src, set, iw);
        if (mp <= 0) {
          Mi = -Mi;
          if (mp & 1) {
            Mr = -Mr;
            Mi = -Mi;
          }
        }
        double ar = Mr * zr - Mi * zi, ai = Mr * zi + Mi * zr;
        if (set == 0) {
          v1r += ar;
          v1i += ai;
        } else {
          v2r += ar;
          v2i += ai;
        }
      }
    }
    int64_t i = hidx(n, m);
    ER(rot, 0, i) = v1r;
    EI(rot, 0, i) = v1i;
    if (lh) {
      ER(rot, 1, i) = v2r;
      EI(rot, 1, i) = v2i;
    }
  }
}

static void rotate_y(double* rot, const double* src, const double* Ts, const double* mags, int P, bool lh,
                     bool local) {
  for (int n = 0; n <= P; ++n) rotate_y_degree(rot, src, Ts, mags, n, lh, local);
}

// ---------------------------------------------------------------------------
// translate_multipole_z!, src/translate.jl:6-50
void translate_multipole_z(double* out, const double* src, double t, int p, bool lh) {
  double _t = -t;
  int64_t i = 0;
  for (int n = 0; n <= p; ++n)
    for (int m = 0; m <= n; ++m, ++i) {
      double v1r = 0, v1i = 0, v2r = 0, v2i = 0;
      double n_np_f = 1.0, _t_n_np = 1.0;
      int n_np = 1;
      for (int np = n; np >= m; --np) {
        double tmp = _t_n_np / n_np_f;
        int64_t iw = hidx(np, m);
        v1r += tmp * ER(src, 0, iw);
        v1i += tmp * EI(src, 0, iw);
        if (lh) {
          v2r += tmp * ER(src, 1, iw);
          v2i += tmp * EI(src, 1, iw);
        }
        _t_n_np *= _t;
        n_np_f *= n_np;
        n_np += 1;
      }
      ER(out, 0, i) = v1r;
      EI(out, 0, i) = v1i;
      if (lh) {
        ER(out, 1, i) = v2r;
        EI(out, 1, i) = v2i;
      }
    }
}

// translate_multipole_to_local_z!, src/translate.jl:181-232
void translate_multipole_to_local_z(double* out, const double* src, double t, int p, bool lh) {
  double one_over_t = 1 / t;
  double n_fact_t_np1 = one_over_t;
  int64_t i = 0;
  for (int n = 0; n <= p; ++n) {
    double n_m_fact = n_fact_t_np1;
    int n_m = n;
    for (int m = 0; m <= n; ++m, ++i) {
      double v1r = 0, v1i = 0, v2r = 0, v2i = 0;
      double c = n_m_fact;
      int n_np = n_m;
      for (int np = m; np <= p; ++np) {
        int64_t iw = hidx(np, m);
        v1r += c * ER(src, 0, iw);
        v1i += c * EI(src, 0, iw);
        if (lh) {
          v2r += c * ER(src, 1, iw);
          v2i += c * EI(src, 1, iw);
        }
        n_np += 1;
        c *= n_np * one_over_t;
      }
      ER(out, 0, i) = v1r;
      EI(out, 0, i) = v1i;
      if (lh) {
        ER(out, 1, i) = v2r;
        EI(out, 1, i) = v2i;
      }
      n_m += 1;
      n_m_fact *= n_m * one_over_t;
    }
    n_fact_t_np1 *= (n + 1) * one_over_t;
  }
}

// translate_multipole_to_local_z_n!, src/translate.jl:238-295 (degree n only)
static double translate_multipole_to_local_z_n(double* out, const double* src, double one_over_t,
                                               double n_fact_t_np1, int n, bool lh) {
  int64_t i = hidx(n, 0);
  double n_m_fact = n_fact_t_np1;
  int n_m = n;
  for (int m = 0; m <= n; ++m, ++i) {
    double v1r = 0, v1i = 0, v2r = 0, v2i = 0;
    double c = n_m_fact;
    int n_np = n_m;
    for (int np = m; np <= n; ++np) {
      int64_t iw = hidx(np, m);
      v1r += c * ER(src, 0, iw);
      v1i += c * EI(src, 0, iw);
      if (lh) {
        v2r += c * ER(src, 1, iw);
        v2i += c * EI(src, 1, iw);
      }
      n_np += 1;
      c *= n_np * one_over_t;
    }
    ER(out, 0, i) = v1r;
    EI(out, 0, i) = v1i;
    if (lh) {
      ER(out, 1, i) = v2r;
      EI(out, 1, i) = v2i;
    }
    n_m += 1;
    n_m_fact *= n_m * one_over_t;
  }
  return n_fact_t_np1 * ((n + 1) * one_over_t);
}

// translate_multipole_to_local_z_m01_n, src/translate.jl:302-364
static void translate_m2l_z_m01_n(const double* src, double t, double one_over_t, bool lh,
                                  double n_fact_t_np1, int n, double& phi_n0_re, double& phi_n1_re,
                                  double& phi_n1_im, double& chi_n1_re, double& chi_n1_im) {
  double n_m_fact = n_fact_t_np1;
  int n_m = n;
  phi_n0_re = 0;
  double c = n_m_fact;
  int n_np = n_m;
  for (int np = 0; np <= n; ++np) {
    phi_n0_re += c * ER(src, 0, hidx(np, 0));
    n_np += 1;
    c *= n_np * one_over_t;
  }
  n_m += 1;
  n_m_fact *= n_m * one_over_t;
  phi_n1_re = phi_n1_im = chi_n1_re = chi_n1_im = 0;
  c = n_m_fact;
  n_np = n_m;
  for (int np = 1; np <= n; ++np) {
    int64_t iw = hidx(np, 1);
    phi_n1_re += c * ER(src, 0, iw);
    phi_n1_im += c * EI(src, 0, iw);
    if (lh) {
      chi_n1_re += c * ER(src, 1, iw);
      chi_n1_im += c * EI(src, 1, iw);
    }
    n_np += 1;
    c *= n_np * one_over_t;
  }
  if (lh) {
    double t_over_n = t / n;
    phi_n1_re -= t_over_n * chi_n1_im;
    phi_n1_im += t_over_n * chi_n1_re;
  }
}

// translate_local_z!, src/translate.jl:1851-1891
void translate_local_z(double* out, const double* src, double t, int p, bool lh) {
  double _t = -t;
  int64_t i = 0;
  for (int n = 0; n <= p; ++n)
    for (int m = 0; m <= n; ++m, ++i) {
      double v1r = 0, v1i = 0, v2r = 0, v2i = 0;
      int n_np = 1;
      double c = 1.0;
      for (int np = n; np <= p; ++np) {
        int64_t iw = hidx(np, m);
        v1r += c * ER(src, 0, iw);
        v1i += c * EI(src, 0, iw);
        if (lh) {
          v2r += c * ER(src, 1, iw);
          v2i += c * EI(src, 1, iw);
        }
        c *= _t / n_np;
        n_np += 1;
      }
      ER(out, 0, i) = v1r;
      EI(out, 0, i) = v1i;
      if (lh) {
        ER(out, 1, i) = v2r;
        EI(out, 1, i) = v2i;
      }
    }
}

// transform_lamb_helmholtz_multipole!, src/translate.jl:52-96
void lh_multipole(double* M, double r, int P) {
  for (int m = 0; m <= P; ++m) {
    int64_t i = hidx(P, m);
    double cr = ER(M, 1, i), ci = EI(M, 1, i);
    for (int n = P; n >= std::max(m, 1); --n) {
      double pr = ER(M, 0, i), pi = EI(M, 0, i);
      double xr = cr, xi = ci;
      double r_m_np1 = r * m / (n + 1);
      ER(M, 0, i) = pr + r_m_np1 * xi;
      EI(M, 0, i) = pi - r_m_np1 * xr;
      if (m < n) {
        cr = ER(M, 1, i - n);
        ci = EI(M, 1, i - n);
      } else {
        cr = 0;
        ci = 0;
      }
      double r_n = r / n;
      ER(M, 1, i) = xr + r_n * cr;
      EI(M, 1, i) = xi + r_n * ci;
      i -= n;
    }
  }
}

// transform_lamb_helmholtz_local!, src/translate.jl:98-142
void lh_local(double* L, double r, int P) {
  for (int m = 0; m <= P; ++m) {
    int64_t i = hidx(m, m);
    double cr = ER(L, 1, i), ci = EI(L, 1, i);
    for (int n = m; n <= P; ++n) {
      double xr = cr, xi = ci;
      if (n > 0) {
        double pr = ER(L, 0, i), pi = EI(L, 0, i);
        double r_m_n = r * m / n;
        ER(L, 0, i) = pr - r_m_n * xi;
        EI(L, 0, i) = pi + r_m_n * xr;
      }
      if (n < P) {
        cr = ER(L, 1, i + n + 1);
        ci = EI(L, 1, i + n + 1);
        double r_np1 = r / (n + 1);
        ER(L, 1, i) = xr - r_np1 * cr;
        EI(L, 1, i) = xi - r_np1 * ci;
      }
      i += n + 1;
    }
  }
}

// local_power, src/translate.jl:455-502
static void local_power(const double* w, double r, int n, const double* Lt, bool lh, double& pphi,
                        double& pchi, double& Nt) {
  pphi = 0;
  pchi = 0;
  Nt = 0;
  double chr_np1 = 0, chi_np1 = 0;
  int64_t i = hidx(n, 0);
  for (int m = n; m >= 0; --m) {
    Nt = Lt[i + m];
    double pr = ER(w, 0, i + m), pi = EI(w, 0, i + m);
    // the reference writes `(1 + m>0)`, which Julia parses as `(1 + m) > 0 == true`: a weight of 1
    const double mult = 1.0;
    if (lh) {
      double cro = ER(w, 1, i + m), cio = EI(w, 1, i + m);
      pr = pr - cio * r * m / n;
      pi = pi + cro * r * m / n;
      double cr = cro - chr_np1 * r / (n + 1);
      double ci = cio - chi_np1 * r / (n + 1);
      chr_np1 = cro;
      chi_np1 = cio;
      pchi += (cr * cr + ci * ci) * Nt * Nt * mult;
    }
    pphi += (pr * pr + pi * pi) * Nt * Nt * mult;
  }
  pphi = std::sqrt(pphi);
  if (lh) pchi = std::sqrt(pchi);
}

// ---------------------------------------------------------------------------
void Work::resize(int p) {
  int64_t N = nh(p + 2);
  t1.assign(4 * N, 0.0);
  t2.assign(4 * N, 0.0);
  t3.assign(4 * N, 0.0);
  Ts.assign(length_Ts(p + 1), 0.0);
  eim.assign(2 * (p + 3), 0.0);
  harm.assign(4 * N, 0.0);
  gnm.assign(6 * N, 0.0);
}

// multipole_to_multipole!, src/translate.jl:144-174
void m2m(double* target, const double* tc, const double* src, const double* sc, int p, bool lh, Work& w) {
  const Tables& tb = tables(p);
  double r, th, ph;
  cartesian_to_spherical(tc[0] - sc[0], tc[1] - sc[1], tc[2] - sc[2], r, th, ph);
  update_eim(w.eim.data(), ph, p);
  for (int n = 0; n <= p; ++n) rotate_z_degree(w.t1.data(), src, w.eim.data(), n, lh);
  update_Ts(w.Ts.data(), tb.Hs.data(), th, p);
  rotate_y(w.t2.data(), w.t1.data(), w.Ts.data(), tb.zeta.data(), p, lh, false);
  translate_multipole_z(w.t1.data(), w.t2.data(), r, p, lh);
  if (lh) lh_multipole(w.t1.data(), r, p);
  rotate_y(w.t2.data(), w.t1.data(), w.Ts.data(), tb.zeta.data(), p, lh, false);
  back_rotate_z(target, w.t2.data(), w.eim.data(), p, lh);
}

// local_to_local!, src/translate.jl:1896-1926
void l2l(double* target, const double* tc, const double* src, const double* sc, int p, bool lh, Work& w) {
  const Tables& tb = tables(p);
  double r, th, ph;
  cartesian_to_spherical(tc[0] - sc[0], tc[1] - sc[1], tc[2] - sc[2], r, th, ph);
  update_eim(w.eim.data(), ph, p);
  for (int n = 0; n <= p; ++n) rotate_z_degree(w.t1.data(), src, w.eim.data(), n, lh);
  update_Ts(w.Ts.data(), tb.Hs.data(), th, p);
  rotate_y(w.t2.data(), w.t1.data(), w.Ts.data(), tb.eta.data(), p, lh, true);
  translate_local_z(w.t1.data(), w.t2.data(), r, p, lh);
  if (lh) lh_local(w.t1.data(), r, p);
  rotate_y(w.t2.data(), w.t1.data(), w.Ts.data(), tb.eta.data(), p, lh, true);
  back_rotate_z(target, w.t2.data(), w.eim.data(), p, lh);
}

// minimum_distance, src/error.jl:3-20
static inline double minabs(double x, double y) {
  return x * (std::fabs(x) <= std::fabs(y) ? 1.0 : 0.0) + y * (std::fabs(y) < std::fabs(x) ? 1.0 : 0.0);
}
static inline double min_dist_1d(double dx, double rm, double rp) {
  double right = dx + rp, left = dx + rm;
  double same = (right * left >= 0) ? 1.0 : 0.0;
  return same * minabs(right, left);
}

// multipole_to_local! plain (src/translate.jl:519-550) and the error-controlled
// variants RotatedCoefficients{Absolute,Relative}Gradient (:555-829),
// Power{Absolute,Relative}Potential (:831-1122) and Power{Absolute,Relative}Gradient
// (:1124-1412).  Returns the expansion order used.
int m2l(double* target, const M2LTarget& tg, const double* src, const double* sc, int p, bool lh,
        int error_method, double eps_in, int be, bool& success, Work& w) {
  const Tables& tb = tables(p);
  double r, th, ph;
  cartesian_to_spherical(tg.center[0] - sc[0], tg.center[1] - sc[1], tg.center[2] - sc[2], r, th, ph);
  int P = p;
  success = true;
  if (error_method == 0) {
    update_eim(w.eim.data(), ph, p);
    for (int n = 0; n <= p; ++n) rotate_z_degree(w.t1.data(), src, w.eim.data(), n, lh);
    update_Ts(w.Ts.data(), tb.Hs.data(), th, p);
    rotate_y(w.t2.data(), w.t1.data(), w.Ts.data(), tb.zeta.data(), p, lh, false);
  } else {
    bool relative = (error_method == 2 || error_method == 4 || error_method == 6);
    bool potential = (error_method == 5 || error_method == 6);
    bool power = (error_method == 1 || error_method == 2 || potential);
    double eps = relative ? tg.max_influence * eps_in : eps_in;
    double mdx = min_dist_1d(tg.center[0] - sc[0], -tg.box[0], tg.box[0]);
    double mdy = min_dist_1d(tg.center[1] - sc[1], -tg.box[1], tg.box[1]);
    double mdz = min_dist_1d(tg.center[2] - sc[2], -tg.box[2], tg.box[2]);
    double r_mp = std::sqrt(mdx * mdx + mdy * mdy + mdz * mdz);
    double r_l = tg.radius;
    double rinv = 1.0 / r, r_mp_inv = 1.0 / r_mp;
    double r_mp_inv_np2 = r_mp_inv * r_mp_inv * r_mp_inv;
    double r_l_nm1 = 1.0;
    update_eim(w.eim.data(), ph, p);
    rotate_z_degree(w.t1.data(), src, w.eim.data(), 0, lh);
    double sb = std::sin(th), cb = std::cos(th), _1_n = -1.0;
    w.Ts[0] = 1.0;
    rotate_y_degree(w.t2.data(), w.t1.data(), w.Ts.data(), tb.zeta.data(), 0, lh, false);
    double n_fact_t_np1 = rinv * rinv, nm1_fact_inv = 1.0, np1_fact = 2.0;
    double Mn0 = tb.Mt[0];
    double mp_phi = std::sqrt((ER(src, 0, 0) * ER(src, 0, 0) + EI(src, 0, 0) * EI(src, 0, 0)) * Mn0 * Mn0);
    // the reference also tracks the chi power of degree n-1, but its error formula only reads degree n's
    success = false;
    const double four_pi_eps = eps * 4 * PI;
    for (int n = 1; n <= p; ++n) {
      // z rotation of degree n (+ multipole power for the Power* methods)
      double pn_phi = 0, pn_chi = 0, Mn0_next = tb.Mt[hidx(n, 0)];
      for (int m = 0; m <= n; ++m) {
        int64_t i = hidx(n, m);
        if (power) {
          // `(1 + m>0)` in rotate_z_n_power! (src/rotate.jl:549) evaluates to true, i.e. a weight of 1
          double Nt = tb.Mt[i], mult = 1.0;
          pn_phi += (ER(src, 0, i) * ER(src, 0, i) + EI(src, 0, i) * EI(src, 0, i)) * Nt * Nt * mult;
          if (lh) pn_chi += (ER(src, 1, i) * ER(src, 1, i) + EI(src, 1, i) * EI(src, 1, i)) * Nt * Nt * mult;
        }
      }
      pn_phi = std::sqrt(pn_phi);
      pn_chi = std::sqrt(pn_chi);
      rotate_z_degree(w.t1.data(), src, w.eim.data(), n, lh);
      _1_n = ts_degree(w.Ts.data() + length_Ts(n - 1), tb.Hs.data() + length_Hs(n - 1), sb, cb, _1_n, n);
      rotate_y_degree(w.t2.data(), w.t1.data(), w.Ts.data(), tb.zeta.data(), n, lh, false);
      double eps_mp;
      if (potential) {
        // the potential variants read degree n's multipole power (src/translate.jl:893-896)
        eps_mp = SQRT3 * pn_phi * r_mp_inv_np2 * r_mp * np1_fact / (Mn0 * (n + 1));
        if (lh) eps_mp += SQRT3 * n * pn_chi * r_mp_inv_np2 * r_mp * np1_fact / (Mn0_next * (n + 1));
      } else if (power) {
        eps_mp = SQRT3 * mp_phi * r_mp_inv_np2 * np1_fact / Mn0;
        if (lh) eps_mp += SQRT3 * n * pn_chi * r_mp_inv_np2 * np1_fact / Mn0_next;
      } else {
        int64_t in0 = hidx(n, 0);
        double p0 = ER(w.t2.data(), 0, in0);
        double p1r = ER(w.t2.data(), 0, in0 + 1), p1i = EI(w.t2.data(), 0, in0 + 1);
        eps_mp = (std::sqrt(p1r * p1r + p1i * p1i) + std::fabs(p0)) * np1_fact * r_mp_inv_np2;
        if (lh) {
          double c1r = ER(w.t2.data(), 1, in0 + 1), c1i = EI(w.t2.data(), 1, in0 + 1);
          eps_mp += std::sqrt(c1r * c1r + c1i * c1i) * np1_fact * r_mp_inv_np2 * r_mp;
        }
      }
      if (eps_mp <= four_pi_eps) {
        double eps_l;
        if (power) {
          translate_multipole_to_local_z_n(w.t3.data(), w.t2.data(), rinv, n_fact_t_np1, n, lh);
          double lphi, lchi, Ln0;
          local_power(w.t3.data(), r, n, tb.Lt.data(), lh, lphi, lchi, Ln0);
          if (potential)  // src/translate.jl:912-915
            eps_l = SQRT3 * lphi * r_l_nm1 * r_l * nm1_fact_inv / (Ln0 * n);
          else
            eps_l = SQRT3 * lphi * r_l_nm1 * nm1_fact_inv / Ln0;
          if (lh) eps_l += SQRT3 * n * lchi * r_l_nm1 * r_l * nm1_fact_inv / (Ln0 * n);
        } else {
          double a, b, c, d, e;
          translate_m2l_z_m01_n(w.t2.data(), r, rinv, lh, n_fact_t_np1, n, a, b, c, d, e);
          eps_l = (std::fabs(b) + std::fabs(c) + std::fabs(a)) * r_l_nm1 * nm1_fact_inv;
          if (lh) eps_l += std::sqrt(d * d + e * e) * r_l_nm1 * r_l * nm1_fact_inv;
        }
        if (eps_mp + eps_l * LOCAL_ERROR_SAFETY <= four_pi_eps) {
          P = n - 1 + (be ? 1 : 0);
          success = true;
          break;
        }
      }
      if (power || n < p) {  // the RotatedCoefficients variants guard the recursion with n < P
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
  translate_multipole_to_local_z(w.t1.data(), w.t2.data(), r, P, lh);
  if (lh) lh_local(w.t1.data(), r, P);
  rotate_y(w.t2.data(), w.t1.data(), w.Ts.data(), tb.eta.data(), P, lh, true);
  back_rotate_z(target, w.t2.data(), w.eim.data(), P, lh);
  return P;
}

// ---------------------------------------------------------------------------
// P2M helpers: get_n / get_nm1 / calculate_q!, src/bodytomultipole.jl:39-139
static inline void get_nm1(const double* h, int n, int m, int64_t i_nm1_m, double _1_m, double* o) {
  // o = {mm1_re, mm1_im, m_re, m_im, mp1_re, mp1_im}; harmonics set index 0
  if (m > 0) {
    o[0] = h[4 * (i_nm1_m - 1)];
    o[1] = h[4 * (i_nm1_m - 1) + 1];
  } else if (n > 1) {
    o[0] = -_1_m * h[4 * (i_nm1_m + 1)];
    o[1] = _1_m * h[4 * (i_nm1_m + 1) + 1];
  } else {
    o[0] = o[1] = 0;
  }
  if (m < n) {
    o[2] = h[4 * i_nm1_m];
    o[3] = h[4 * i_nm1_m + 1];
  } else {
    o[2] = o[3] = 0;
  }
  if (m + 1 < n) {
    o[4] = h[4 * (i_nm1_m + 1)];
    o[5] = h[4 * (i_nm1_m + 1) + 1];
  } else {
    o[4] = o[5] = 0;
  }
}

static inline void get_n(const double* h, int n, int m, int64_t i, double _1_m, double* o) {
  if (m > 0) {
    o[0] = h[4 * (i - 1)];
    o[1] = h[4 * (i - 1) + 1];
  } else if (n == 0) {
    o[0] = o[1] = 0;
  } else {
    o[0] = -_1_m * h[4 * (i + 1)];
    o[1] = _1_m * h[4 * (i + 1) + 1];
  }
  o[2] = h[4 * i];
  o[3] = h[4 * i + 1];
  if (m < n) {
    o[4] = h[4 * (i + 1)];
    o[5] = h[4 * (i + 1) + 1];
  } else {
    o[4] = o[5] = 0;
  }
}

static void calculate_q(double* h, double xr, double xi, double er, double ei, double z, int p) {
  h[0] = 1.0;
  h[1] = 0.0;
  int64_t i = 1;
  for (int n = 1; n <= p; ++n) {
    int64_t i_nm1_m = i - n;
    double _1_m = 1.0;
    for (int m = 0; m <= n; ++m) {
      double q[6];
      get_nm1(h, n, m, i_nm1_m, _1_m, q);
      h[4 * i] = (-(xr * q[1] + xi * q[0]) - (er * q[5] + ei * q[4]) - z * q[2]) / n;
      h[4 * i + 1] = ((xr * q[0] - xi * q[1]) + (er * q[4] - ei * q[5]) - z * q[3]) / n;
      i++;
      i_nm1_m++;
      _1_m = -_1_m;
    }
  }
}

// body_to_multipole_point!(Point{Source}), src/bodytomultipole.jl:403-429
void p2m_point_source(double* M, double* h, double dx, double dy, double dz, double q, int p) {
  double xr = dx * 0.5, xi = dy * 0.5, er = xr, ei = -xi, z = dz;
  double strength = -q;
  calculate_q(h, xr, xi, er, ei, z, p);
  double _1_n = 1.0;
  int64_t i = 0;
  for (int n = 0; n <= p; ++n) {
    double _1_n_m = _1_n;
    for (int m = 0; m <= n; ++m, ++i) {
      ER(M, 0, i) += h[4 * i] * _1_n_m * strength;
      EI(M, 0, i) -= h[4 * i + 1] * _1_n_m * strength;
      _1_n_m = -_1_n_m;
    }
    _1_n = -_1_n;
  }
}

// body_to_multipole_point!(Point{Vortex}) + mirrored_source_to_vortex!,
// src/bodytomultipole.jl:465-489, 283-334
void p2m_point_vortex(double* M, double* h, double dx, double dy, double dz, double vx, double vy,
                      double vz, int p) {
  double xr = -dx * 0.5, xi = -dy * 0.5, er = xr, ei = -xi, z = -dz;
  calculate_q(h, xr, xi, er, ei, z, p);
  const double mult = 1.0;
  int64_t i = 0;
  for (int n = 0; n <= p; ++n) {
    double _1_m = 1.0, _1_np1 = 1.0 / (n + 1);
    for (int m = 0; m <= n; ++m, ++i) {
      double q[6];
      get_n(h, n, m, i, _1_m, q);
      double a = (double)(n - m + 1) * 0.5, b = (double)(n + m + 1) * 0.5;
      ER(M, 0, i) += mult * _1_m * ((-vx * q[0] + vy * q[1]) * a + (vx * q[4] + vy * q[5]) * b - vz * m * q[3]) * _1_np1;
      EI(M, 0, i) += mult * _1_m * ((vx * q[1] + vy * q[0]) * a + (-vx * q[5] + vy * q[4]) * b - vz * m * q[2]) * _1_np1;
      _1_m = -_1_m;
    }
  }
  i = 1;
  for (int n = 1; n <= p; ++n) {
    int64_t i_nm1_m = i - n;
    double _1_m = 1.0, _1_over_n = 1.0 / n;
    for (int m = 0; m <= n; ++m) {
      double q[6];
      get_nm1(h, n, m, i_nm1_m, _1_m, q);
      ER(M, 1, i) -= mult * _1_m * _1_over_n * (0.5 * (-vy * q[0] - vx * q[1] + vy * q[4] - vx * q[5]) - vz * q[2]);
      EI(M, 1, i) -= mult * _1_m * _1_over_n * (0.5 * (vy * q[1] - vx * q[0] - vy * q[5] - vx * q[4]) + vz * q[3]);
      i++;
      i_nm1_m++;
      _1_m = -_1_m;
    }
  }
}

// ---------------------------------------------------------------------------
// evaluate_local, src/evaluate_expansions.jl:45-399
void evaluate_local(const double* dx, const double* L, int p, bool lh, bool ps, bool gs, bool hs,
                    double& phi_out, double* grad, double* hess, Work& w) {
  double r, th, ph;
  cartesian_to_spherical(dx[0], dx[1], dx[2], r, th, ph);
  double* R = w.harm.data();
  regular_harmonics(R, r, th, ph, p);
  double* g = w.gnm.data();  // gradient_n_m[reim, comp, i] at g[6*i + 2*comp + reim]
  if (hs) std::fill(g, g + 6 * nh(p), 0.0);
  double u = 0, vx = 0, vy = 0, vz = 0;
  double vxx = 0, vxy = 0, vxz = 0, vyx = 0, vyy = 0, vyz = 0, vzx = 0, vzy = 0, vzz = 0;
  int64_t i = 0;
  {  // n = 0, m = 0
    int n = 0;
    double Rr = R[0], Ri = R[1];
    if (ps) u += Rr * ER(L, 0, i) - Ri * EI(L, 0, i);
    if (gs || hs) {
      double vxr = 0, vyr = 0, vzr = 0, vzi = 0;
      vxr -= EI(L, 0, i + n + 2);
      vyr -= ER(L, 0, i + n + 2);
      vzr -= ER(L, 0, i + n + 1);
      vzi -= EI(L, 0, i + n + 1);
      if (gs) {
        vx += vxr * Rr;
        vy += vyr * Rr;
        vz += vzr * Rr - vzi * Ri;
      }
      if (hs) {
        g[6 * i + 0] = vxr;
        g[6 * i + 2] = vyr;
        g[6 * i + 4] = vzr;
        g[6 * i + 5] = vzi;
      }
    }
  }
  for (int n = 1; n <= p; ++n) {
    ++i;  // m = 0
    {
      double Rr = R[4 * i], Ri = R[4 * i + 1];
      if (ps && !lh) u += Rr * ER(L, 0, i) - Ri * EI(L, 0, i);
      if (gs || hs) {
        double vxr = 0, vyr = 0, vzr = 0, vzi = 0;
        if (n < p) {
          vxr -= EI(L, 0, i + n + 2);
          vyr -= ER(L, 0, i + n + 2);
          vzr -= ER(L, 0, i + n + 1);
          vzi -= EI(L, 0, i + n + 1);
        }
        if (lh) {
          vxr += n * ER(L, 1, i + 1);
          vyr -= n * EI(L, 1, i + 1);
        }
        if (gs) {
          vx += vxr * Rr;
          vy += vyr * Rr;
          vz += vzr * Rr - vzi * Ri;
        }
        if (hs) {
          g[6 * i + 0] = vxr;
          g[6 * i + 2] = vyr;
          g[6 * i + 4] = vzr;
          g[6 * i + 5] = vzi;
        }
      }
    }
    for (int m = 1; m <= n; ++m) {
      ++i;
      double Rr = R[4 * i], Ri = R[4 * i + 1];
      if (ps && !lh) u += 2 * (Rr * ER(L, 0, i) - Ri * EI(L, 0, i));
      if (gs || hs) {
        double vxr = 0, vxi = 0, vyr = 0, vyi = 0, vzr = 0, vzi = 0;
        if (n < p) {
          double amr = ER(L, 0, i + n), ami = EI(L, 0, i + n);
          double a0r = ER(L, 0, i + n + 1), a0i = EI(L, 0, i + n + 1);
          double apr = ER(L, 0, i + n + 2), api = EI(L, 0, i + n + 2);
          vxr -= (ami + api) * 0.5;
          vxi += (amr + apr) * 0.5;
          vyr += (amr - apr) * 0.5;
          vyi += (ami - api) * 0.5;
          vzr -= a0r;
          vzi -= a0i;
        }
        if (lh) {
          double cmr = ER(L, 1, i - 1), cmi = EI(L, 1, i - 1);
          vxr -= (n + m) * cmr * 0.5;
          vxi -= (n + m) * cmi * 0.5;
          vyr -= (n + m) * cmi * 0.5;
          vyi += (n + m) * cmr * 0.5;
          if (m < n) {
            double cpr = ER(L, 1, i + 1), cpi = EI(L, 1, i + 1);
            vxr += (n - m) * cpr * 0.5;
            vxi += (n - m) * cpi * 0.5;
            vyr -= (n - m) * cpi * 0.5;
            vyi += (n - m) * cpr * 0.5;
          }
          double c0r = ER(L, 1, i), c0i = EI(L, 1, i);
          vzr += m * c0i;
          vzi -= m * c0r;
        }
        vx += 2 * (vxr * Rr - vxi * Ri);
        vy += 2 * (vyr * Rr - vyi * Ri);
        vz += 2 * (vzr * Rr - vzi * Ri);
        if (hs) {
          g[6 * i + 0] = vxr;
          g[6 * i + 1] = vxi;
          g[6 * i + 2] = vyr;
          g[6 * i + 3] = vyi;
          g[6 * i + 4] = vzr;
          g[6 * i + 5] = vzi;
        }
      }
    }
  }
  if (hs) {
    auto G = [&](int reim, int comp, int64_t k) { return g[6 * k + 2 * comp + reim]; };
    int64_t k = -1;
    for (int n = 0; n <= p - 1; ++n) {
      ++k;  // m = 0
      double Rr = R[4 * k], Ri = R[4 * k + 1];
      vxx += -G(1, 0, k + n + 2) * Rr;
      vyx += -G(0, 0, k + n + 2) * Rr;
      vzx += -G(0, 0, k + n + 1) * Rr - (-G(1, 0, k + n + 1)) * Ri;
      vxy += -G(1, 1, k + n + 2) * Rr;
      vyy += -G(0, 1, k + n + 2) * Rr;
      vzy += -G(0, 1, k + n + 1) * Rr - (-G(1, 1, k + n + 1)) * Ri;
      vxz += -G(1, 2, k + n + 2) * Rr;
      vyz += -G(0, 2, k + n + 2) * Rr;
      vzz += -G(0, 2, k + n + 1) * Rr - (-G(1, 2, k + n + 1)) * Ri;
      for (int m = 1; m <= n; ++m) {
        ++k;
        Rr = R[4 * k];
        Ri = R[4 * k + 1];
        for (int c = 0; c < 3; ++c) {
          double xr = -(G(1, c, k + n) + G(1, c, k + n + 2)) * 0.5;
          double xi = (G(0, c, k + n) + G(0, c, k + n + 2)) * 0.5;
          double yr = (G(0, c, k + n) - G(0, c, k + n + 2)) * 0.5;
          double yi = (G(1, c, k + n) - G(1, c, k + n + 2)) * 0.5;
          double zr = -G(0, c, k + n + 1);
          double zi = -G(1, c, k + n + 1);
          double ax = 2 * (xr * Rr - xi * Ri), ay = 2 * (yr * Rr - yi * Ri), az = 2 * (zr * Rr - zi * Ri);
          if (c == 0) {
            vxx += ax;
            vyx += ay;
            vzx += az;
          } else if (c == 1) {
            vxy += ax;
            vyy += ay;
            vzy += az;
          } else {
            vxz += ax;
            vyz += ay;
            vzz += az;
          }
        }
      }
    }
  }
  phi_out = -u * ONE_OVER_4PI;
  grad[0] = vx * ONE_OVER_4PI;
  grad[1] = vy * ONE_OVER_4PI;
  grad[2] = vz * ONE_OVER_4PI;
  // SMatrix{3,3}(vxx, vxy, vxz, vyx, vyy, vyz, vzx, vzy, vzz): column-major storage order
  double Hm[9] = {vxx, vxy, vxz, vyx, vyy, vyz, vzx, vzy, vzz};
  for (int c = 0; c < 9; ++c) hess[c] = Hm[c] * ONE_OVER_4PI;
}

}  // namespace orc

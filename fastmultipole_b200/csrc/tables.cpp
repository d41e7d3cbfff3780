// tables.cpp -- FP64 constant tables of the rotation-based translation operators.
//
// Generated once per context on the host and uploaded to HBM:
//   Hs    : Wigner small-d matrices at beta = pi/2 (compute_Hs!, src/rotate.jl:119-203)
//   zeta  : multipole rotation normalisation magnitudes (src/rotate.jl:660-689)
//   eta   : local rotation normalisation magnitudes (src/rotate.jl:975-1004)
//   Mt/Lt : multipole / local power normalisations (src/translate.jl:386-448)
// The recurrences are the reference's; they are evaluated in the same order so
// that the tables agree with the reference's to the last bit.
#include <algorithm>
#include <cmath>
#include <cstdint>

#include "common.cuh"

namespace fmmb {

// nearest double to k! from the exact integer (Float64(factorial(big(k))))
static double factorial_double(int k) {
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
  auto bit = [&](int b) -> uint64_t { return (limb[b / 32] >> (b % 32)) & 1u; };
  if (nbits <= 53) {
    double v = 0;
    for (int i = top; i >= 0; --i) v = v * 4294967296.0 + limb[i];
    return v;
  }
  int shift = nbits - 64;
  uint64_t hi = 0;
  for (int b = nbits - 1; b >= shift; --b) hi = (hi << 1) | bit(b);
  bool sticky = false;
  for (int b = 0; b < shift; ++b) sticky |= bit(b) != 0;
  uint64_t low = hi & 0x7FF, mant = hi >> 11;
  if (low > 0x400 || (low == 0x400 && (sticky || (mant & 1)))) mant++;
  return std::ldexp((double)mant, shift + 11);
}

static void legendre(int p, double s, double c, std::vector<double>& P) {
  P.assign(nh(p), 0.0);
  double Pn0 = 1.0, fact = 1.0;
  for (int m = 0; m <= p; ++m) {
    double Pnm = Pn0;
    P[hidx(m, m)] = Pnm;
    double t1 = Pnm;
    Pnm = c * (2 * m + 1) * t1;
    for (int n = m + 1; n <= p; ++n) {
      P[hidx(n, m)] = Pnm;
      double t2 = t1;
      t1 = Pnm;
      Pnm = (c * (2 * n + 1) * t1 - (n + m) * t2) / (n - m + 1);
    }
    Pn0 = -Pn0 * fact * s;
    fact += 2;
  }
}

static void wigner_pi2(std::vector<double>& Hs, int p) {
  const double beta = kPi / 2;
  double sb = std::sin(beta), cb = std::cos(beta);
  std::vector<double> P;
  legendre(p + 1, sb, cb, P);
  Hs.assign(length_Hs(p), 0.0);
  Hs[0] = 1.0;
  std::vector<double> Hn1(p + 2), b(2 * (p + 1) + 1), dn(p + 1);
  for (int n = 1; n <= p; ++n) {
    double* H = Hs.data() + length_Hs(n - 1);
    double sg = 1, f = 1;
    for (int m = 0; m <= n; ++m) {
      H[H_index(0, m)] = sg * f * P[hidx(n, m)];
      sg = -sg;
      f /= std::sqrt((double)((n + m + 1) * (n - m)));
    }
    sg = 1;
    f = 1;
    for (int m = 0; m <= n + 1; ++m) {
      Hn1[m] = sg * f * P[hidx(n + 1, m)];
      sg = -sg;
      f /= std::sqrt((double)((n + 1 - m) * (n + m + 2)));
    }
    int bn = n + 1;
    for (int m = -bn; m <= bn; ++m) {
      double v = std::sqrt((double)(bn - m - 1) / (double)(2 * bn - 1) * (double)(bn - m) / (double)(2 * bn + 1));
      b[bn + m] = m < 0 ? -v : v;
    }
    double omc = (1.0 - cb) / 2, opc = (1.0 + cb) / 2;
    for (int m = 1; m <= n; ++m) {
      double a = std::sqrt((double)(n + 1 + m) / (double)(2 * n + 1) * (double)(n + 1 - m) / (double)(2 * n + 3));
      H[H_index(1, m)] = (b[bn - m - 1] * omc * Hn1[m + 1] - b[bn + m - 1] * opc * Hn1[m - 1] - a * sb * Hn1[m]) / b[bn];
    }
    for (int m = 0; m <= n; ++m) dn[m] = std::sqrt((double)((n - m) * (n + m + 1))) / 2;
    for (int mp = 1; mp <= n - 1; ++mp) {
      for (int m = mp + 1; m <= n - 1; ++m) {
        double v = dn[mp - 1] * H[H_index(mp - 1, m)] - dn[m - 1] * H[H_index(mp, m - 1)] + dn[m] * H[H_index(mp, m + 1)];
        H[H_index(mp + 1, m)] = v / dn[mp];
      }
      int m = n;
      double v = dn[mp - 1] * H[H_index(mp - 1, m)] - dn[m - 1] * H[H_index(mp, m - 1)];
      H[H_index(mp + 1, m)] = v / dn[mp];
    }
  }
}

static void rotation_magnitudes(std::vector<double>& t, int p, bool local) {
  t.assign(length_Ts(p), 0.0);
  t[0] = 1.0;
  for (int n = 1; n <= p; ++n) {
    double* z = t.data() + length_Ts(n - 1);
    int64_t i = 0;
    double mm = 1.0;
    for (int m = 0; m <= n; ++m) {
      double mag = mm;
      for (int mp = 0; mp <= n; ++mp) {
        z[i++] = mag;
        double a = n + mp + 1, c = (mp + 1 < n) ? n - mp : 1;
        mag *= local ? std::sqrt(c / a) : std::sqrt(a / c);
      }
      double a = (m < n - 1) ? n - m : 1, c = n + m + 1;
      mm *= local ? std::sqrt(c / a) : std::sqrt(a / c);
    }
  }
}

void build_tables(HostTables& t, int p) {
  int want = std::max(p, kMaxP);
  if (t.p >= want) return;
  t.p = want;
  wigner_pi2(t.Hs, want);
  rotation_magnitudes(t.zeta, want, false);
  rotation_magnitudes(t.eta, want, true);
  t.Mt.assign(nh(want), 0.0);
  t.Lt.assign(nh(want), 0.0);
  int64_t i = 0;
  for (int n = 0; n <= want; ++n)
    for (int m = 0; m <= n; ++m, ++i) {
      double a = factorial_double(n + m), b = factorial_double(n - m);
      t.Mt[i] = n == 0 ? 1.0 : std::sqrt(a * b / (2 * n + 1));
      t.Lt[i] = n == 0 ? 1.0 : std::sqrt(1 / (a * b * (2 * n + 1)));
    }
}

}  // namespace fmmb

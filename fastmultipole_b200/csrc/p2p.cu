// p2p.cu -- near-field (P2P) kernels over the target-sorted direct list.
//
// Kernels of the reference's point systems:
//   Laplace point source  (test/gravitational.jl:80-104): phi += q/(4 pi r),
//     grad += q dx/(4 pi r^3), pairs with r^2 = 0 skipped, no hessian;
//   vortex particle       (test/vortex.jl:83-128): u = (dx x Gamma)/(4 pi r^3)
//     and the 9-term velocity gradient.
// k_p2p (direct list): one CTA per target leaf, source bodies gathered into
// warp-private shared-memory batches, lanes split between targets and sources
// by the leaf's size (details at the kernel).  k_direct (all pairs): one CTA
// per block of targets, sources staged through shared memory.  FP64 is the
// drop-in arithmetic; the MIXED variant moves every body relative to a nearby
// centre in FP64, then evaluates the kernel in FP32 (rsqrt on the SFU),
// summing blocks of sources in FP32 and the block partials in FP64.
#include <climits>
#include <vector>
#include <algorithm>

#include "context.cuh"

namespace fmmb {

namespace {

constexpr int kP2PThreads = 128;
// targets per thread held in registers: 4 for point sources (4 accumulators),
// 2 for vortex particles (up to 12 accumulators)
template <int KIND>
__host__ __device__ constexpr int tpt() { return KIND == FMM_POINT_SOURCE ? 4 : 2; }

template <class R>
struct Vec4 {};
template <>
struct Vec4<double> {
  using T = double4;
};
template <>
struct Vec4<float> {
  using T = float4;
};

__device__ __forceinline__ double rsq(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsq(float x) { return rsqrtf(x); }

// one source body on NT targets; acc layout per target: [0]=phi [1..3]=grad [4..12]=hessian
template <class R, int KIND, bool PS, bool GS, bool HS, int TPT>
__device__ __forceinline__ void interact(const R (&tx)[TPT], const R (&ty)[TPT], const R (&tz)[TPT], int nt,
                                         R sx, R sy, R sz, R s0, R s1, R s2, R (&acc)[TPT][13]) {
#pragma unroll
  for (int k = 0; k < TPT; ++k) {
    if (k < nt) {
      R dx = tx[k] - sx, dy = ty[k] - sy, dz = tz[k] - sz;
      R r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > R(0)) {
        R rinv = rsq(r2);
        if (KIND == FMM_POINT_SOURCE) {
          R qr = s0 * rinv;
          if (PS) acc[k][0] += qr;
          R q3 = qr * rinv * rinv;
          acc[k][1] += dx * q3;
          acc[k][2] += dy * q3;
          acc[k][3] += dz * q3;
        } else {
          R rinv2 = rinv * rinv;
          R den = rinv * rinv2;
          // Gamma = (s0, s1, s2)
          if (GS) {
            acc[k][1] += (dz * s1 - dy * s2) * den;
            acc[k][2] += (dx * s2 - dz * s0) * den;
            acc[k][3] += (dy * s0 - dx * s1) * den;
          }
          if (HS) {
            R d5 = den * rinv2;
            R cx = s1 * dz - s2 * dy, cy = s2 * dx - s0 * dz, cz = s0 * dy - s1 * dx;
            acc[k][4] += R(-3) * dx * cx * d5;
            acc[k][5] += (R(-3) * dx * cy + s2 * r2) * d5;
            acc[k][6] += (R(-3) * dx * cz - s1 * r2) * d5;
            acc[k][7] += (R(-3) * dy * cx - s2 * r2) * d5;
            acc[k][8] += R(-3) * dy * cy * d5;
            acc[k][9] += (R(-3) * dy * cz + s0 * r2) * d5;
            acc[k][10] += (R(-3) * dz * cx + s1 * r2) * d5;
            acc[k][11] += (R(-3) * dz * cy - s0 * r2) * d5;
            acc[k][12] += R(-3) * dz * cz * d5;
          }
        }
      }
    }
  }
}

// FP32 sums each source leaf in FP32 and the leaf partials in FP64; FP64 sums directly.
template <class R, int TPT>
struct Acc {
  R part[TPT][13];
  double tot[TPT][13];
  __device__ __forceinline__ void init() {
#pragma unroll
    for (int k = 0; k < TPT; ++k)
#pragma unroll
      for (int a = 0; a < 13; ++a) part[k][a] = R(0), tot[k][a] = 0.0;
  }
  __device__ __forceinline__ void flush() {
#pragma unroll
    for (int k = 0; k < TPT; ++k)
#pragma unroll
      for (int a = 0; a < 13; ++a) tot[k][a] += (double)part[k][a], part[k][a] = R(0);
  }
  __device__ __forceinline__ double get(int k, int a) const { return tot[k][a]; }
};
template <int TPT>
struct Acc<double, TPT> {
  double part[TPT][13];
  __device__ __forceinline__ void init() {
#pragma unroll
    for (int k = 0; k < TPT; ++k)
#pragma unroll
      for (int a = 0; a < 13; ++a) part[k][a] = 0.0;
  }
  __device__ __forceinline__ void flush() {}
  __device__ __forceinline__ double get(int k, int a) const { return part[k][a]; }
};

template <int KIND, bool PS, bool GS, bool HS, class A>
__device__ __forceinline__ void store(double* o, const A& acc, int k) {
  if (PS) o[0] += acc.get(k, 0) * kOneOver4Pi;
  if (GS || KIND == FMM_POINT_SOURCE) {
    o[1] += acc.get(k, 1) * kOneOver4Pi;
    o[2] += acc.get(k, 2) * kOneOver4Pi;
    o[3] += acc.get(k, 3) * kOneOver4Pi;
  }
  if (HS && KIND == FMM_POINT_VORTEX)
#pragma unroll
    for (int a = 4; a < 13; ++a) o[a] += acc.get(k, a) * kOneOver4Pi;
}

// ---------------------------------------------------------------------------
// Direct-list P2P.  One CTA of kWarps warps (kWideWarps when the launch has few rows, so
// that a few long rows still fill the GPU) owns one direct-list row (a target leaf).
// Each warp takes every W-th source leaf of the leaf's direct-list row and
// gathers up to batch_bodies() bodies of consecutive leaves of its share (many
// small leaves, or a piece of a large one) into its own shared-memory batch,
// converted once per body (to FP32 relative to the target leaf centre on the
// mixed path).  Targets sit in registers, kTPT per lane.  A target tile holds
// up to 32 * kTPT targets; the lanes split into TS lanes along the tile times
// 32 / TS slices along the batch, TS the smallest power of two that covers the
// tile, so a leaf of 5 bodies keeps every lane busy as a leaf of 64 does.
// Slices are summed by shuffles, warps through shared memory.  The mixed path
// sums each batch in FP32 and the batches in FP64.  On the packed FP32 path, rows
// of small target leaves (at most 8 bodies on average) take one warp each instead of
// a CTA, so that the per-row setup and the cross-warp sum do not dominate their work.
constexpr int kWarps = 4;
// launches of fewer rows than kWideRowsPerSM per SM take kWideWarps warps per row: a few
// long rows (targets of a dual tree near many sources) would otherwise leave the SMs idle
constexpr int kWideWarps = 16;
constexpr int kWideRowsPerSM = 4;
constexpr int kChunksPerSM = 8;  // chunks of the rows of such a launch, per SM
constexpr double kChunkPairs = 1e8;  // estimated body pairs above which their rows are cut
constexpr int kTPT = 2;
constexpr unsigned kAll = 0xffffffffu;

template <int KIND>
struct Batch {
  static constexpr int n = KIND == FMM_POINT_SOURCE ? 256 : 128;  // bodies per warp batch
  static constexpr int nv = KIND == FMM_POINT_SOURCE ? 4 : 6;     // values per body: x y z + strengths
};

// FP32 point sources evaluate two targets per lane with packed f32x2 arithmetic;
// their batch holds per body {-x, -x, -y, -y}, {-z, -z, q, q} (ready-made pairs)
template <class R, int KIND>
__host__ __device__ constexpr bool packed() { return sizeof(R) == 4 && KIND == FMM_POINT_SOURCE; }
// FP32 vortex particles: two targets per lane as well; batch per body {-x, -x, -y, -y},
// {-z, -z, G0, G0}, {G1, G1, G2, G2}
template <class R, int KIND>
__host__ __device__ constexpr bool packed_vortex() { return sizeof(R) == 4 && KIND == FMM_POINT_VORTEX; }
template <class R, int KIND>
__host__ __device__ constexpr int slots_per_body() {
  return packed<R, KIND>() ? 8 : packed_vortex<R, KIND>() ? 12 : Batch<KIND>::nv;
}
// bodies per warp batch: the packed batch is halved to keep the same shared memory per CTA
template <class R, int KIND>
__host__ __device__ constexpr int batch_bodies() { return packed<R, KIND>() ? 128 : Batch<KIND>::n; }

// 1/sqrt(x) on the SFU, denormal inputs flushed (rsqrt.approx.ftz.f32)
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// accumulated channels: Laplace phi, grad (3); vortex u (3) if GS, grad u (9) if HS
template <int KIND, bool GS, bool HS>
__host__ __device__ constexpr int n_chan() {
  return KIND == FMM_POINT_SOURCE ? 4 : (GS ? 3 : 0) + (HS ? 9 : 0);
}
// acc13 row of channel a
template <int KIND, bool GS>
__device__ __forceinline__ int chan_row(int a) {
  return KIND == FMM_POINT_SOURCE ? a : (GS ? a + 1 : a + 4);
}

// one source body (x, y, z, s0, s1, s2) on one target; same arithmetic as interact()
template <class R, int KIND, bool PS, bool GS, bool HS, int NA>
__device__ __forceinline__ void pair1(R tx, R ty, R tz, R sx, R sy, R sz, R s0, R s1, R s2, R (&a)[NA]) {
  R dx = tx - sx, dy = ty - sy, dz = tz - sz;
  R r2 = dx * dx + dy * dy + dz * dz;
  if (r2 > R(0)) {
    R rinv = rsq(r2);
    if (KIND == FMM_POINT_SOURCE) {
      R qr = s0 * rinv;
      if (PS) a[0] += qr;
      R q3 = qr * rinv * rinv;
      a[1] += dx * q3;
      a[2] += dy * q3;
      a[3] += dz * q3;
    } else {
      R rinv2 = rinv * rinv;
      R den = rinv * rinv2;
      constexpr int h = GS ? 3 : 0;
      if (GS) {
        a[0] += (dz * s1 - dy * s2) * den;
        a[1] += (dx * s2 - dz * s0) * den;
        a[2] += (dy * s0 - dx * s1) * den;
      }
      if (HS) {
        R d5 = den * rinv2;
        R cx = s1 * dz - s2 * dy, cy = s2 * dx - s0 * dz, cz = s0 * dy - s1 * dx;
        a[(h + 0) % NA] += R(-3) * dx * cx * d5;
        a[(h + 1) % NA] += (R(-3) * dx * cy + s2 * r2) * d5;
        a[(h + 2) % NA] += (R(-3) * dx * cz - s1 * r2) * d5;
        a[(h + 3) % NA] += (R(-3) * dy * cx - s2 * r2) * d5;
        a[(h + 4) % NA] += R(-3) * dy * cy * d5;
        a[(h + 5) % NA] += (R(-3) * dy * cz + s0 * r2) * d5;
        a[(h + 6) % NA] += (R(-3) * dz * cx + s1 * r2) * d5;
        a[(h + 7) % NA] += (R(-3) * dz * cy - s0 * r2) * d5;
        a[(h + 8) % NA] += R(-3) * dz * cz * d5;
      }
    }
  }
}

// One lane's slice of a packed batch on its two targets.  GUARD skips pairs with
// r^2 = 0 (coincident bodies); without it such a pair makes the sums non-finite.
template <bool GUARD, bool PS>
__device__ __forceinline__ void packed_batch(const float4* __restrict__ B4, int j0, int nb, int SS, float2 tx2,
                                             float2 ty2, float2 tz2, float2& ph, float2& gx, float2& gy, float2& gz) {
#pragma unroll 4
  for (int j = j0; j < nb; j += SS) {
    const float4 u = B4[2 * j], v = B4[2 * j + 1];
    const float2 dx = __fadd2_rn(tx2, make_float2(u.x, u.y));
    const float2 dy = __fadd2_rn(ty2, make_float2(u.z, u.w));
    const float2 dz = __fadd2_rn(tz2, make_float2(v.x, v.y));
    float2 r2 = __fmul2_rn(dx, dx);
    r2 = __ffma2_rn(dy, dy, r2);
    r2 = __ffma2_rn(dz, dz, r2);
    float2 ri;
    if (GUARD) {
      ri.x = r2.x > 0.f ? rsqrt_ftz(r2.x) : 0.f;
      ri.y = r2.y > 0.f ? rsqrt_ftz(r2.y) : 0.f;
    } else {
      ri = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
    }
    // q / r and q / r^3 = (q / r) (1 / r^2): the two products after the rsqrt are independent
    const float2 qr = __fmul2_rn(make_float2(v.z, v.w), ri);
    const float2 ri2 = __fmul2_rn(ri, ri);
    if (PS) ph = __fadd2_rn(ph, qr);
    const float2 q3 = __fmul2_rn(qr, ri2);
    gx = __ffma2_rn(dx, q3, gx);
    gy = __ffma2_rn(dy, q3, gy);
    gz = __ffma2_rn(dz, q3, gz);
  }
}

// one source body on one target, vortex particles with the velocity gradient (FP64 path):
// velocity into u[0..2] (GS); the gradient as Q_ij += d_i (G x d)_j / r^5 and E_k += G_k / r^3,
// which the caller combines to -3 Q_ij + eps_jki E_k (r^2 / r^5 = 1 / r^3)
template <class R, bool GS>
__device__ __forceinline__ void vortex_pair_qe(R tx, R ty, R tz, R sx, R sy, R sz, R s0, R s1, R s2, R* u,
                                               R (&Q)[9], R (&E)[3]) {
  const R dx = tx - sx, dy = ty - sy, dz = tz - sz;
  const R r2 = dx * dx + dy * dy + dz * dz;
  if (r2 > R(0)) {
    const R rinv = rsq(r2);
    const R rinv2 = rinv * rinv;
    const R den = rinv * rinv2;
    const R cx = s1 * dz - s2 * dy, cy = s2 * dx - s0 * dz, cz = s0 * dy - s1 * dx;
    if (GS) {
      u[0] += cx * den;
      u[1] += cy * den;
      u[2] += cz * den;
    }
    const R d5 = den * rinv2;
    const R px = dx * d5, py = dy * d5, pz = dz * d5;
    Q[0] += px * cx;
    Q[1] += px * cy;
    Q[2] += px * cz;
    Q[3] += py * cx;
    Q[4] += py * cy;
    Q[5] += py * cz;
    Q[6] += pz * cx;
    Q[7] += pz * cy;
    Q[8] += pz * cz;
    E[0] += s0 * den;
    E[1] += s1 * den;
    E[2] += s2 * den;
  }
}

// the gradient channels g[0..8] (column-major d u_j / d x_i at 3 i + j) from Q and E
template <class R>
__device__ __forceinline__ void vortex_grad_from_qe(const R (&Q)[9], const R (&E)[3], R* g) {
  g[0] = R(-3) * Q[0];
  g[1] = R(-3) * Q[1] + E[2];
  g[2] = R(-3) * Q[2] - E[1];
  g[3] = R(-3) * Q[3] - E[2];
  g[4] = R(-3) * Q[4];
  g[5] = R(-3) * Q[5] + E[0];
  g[6] = R(-3) * Q[6] + E[1];
  g[7] = R(-3) * Q[7] - E[0];
  g[8] = R(-3) * Q[8];
}

// f32x2 with both halves negated
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// One lane's slice of a packed vortex batch on its two targets: velocity
// u = (G x d) / r^3 (GS) and its gradient (HS, the SMatrix column-major order of
// test/vortex.jl:83-128).  acc[a] receives channel a of the two targets.  The gradient
// du_j/dx_i = eps_jki G_k / r^3 - 3 d_i (G x d)_j / r^5 is summed as two parts, Q_ij =
// sum d_i (G x d)_j / r^5 and E_k = sum G_k / r^3, combined once per batch (r^2 / r^5 =
// 1 / r^3, so the six eps terms need three sums; the trace of Q vanishes, so Q_zz is not
// summed).  GUARD skips pairs with r^2 = 0
// (coincident bodies); without it such a pair makes the sums non-finite.
template <bool GUARD, bool GS, bool HS, int NA>
__device__ __forceinline__ void packed_vortex_batch(const float4* __restrict__ B4, int j0, int nb, int SS,
                                                    float2 tx2, float2 ty2, float2 tz2, float2 (&acc)[NA]) {
  constexpr int h = GS ? 3 : 0;
  float2 u[3], Q[9], E[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) u[a] = E[a] = make_float2(0.f, 0.f);
#pragma unroll
  for (int a = 0; a < 9; ++a) Q[a] = make_float2(0.f, 0.f);
#pragma unroll 2
  for (int j = j0; j < nb; j += SS) {
    const float4 p = B4[3 * j], v = B4[3 * j + 1], w = B4[3 * j + 2];
    const float2 dx = __fadd2_rn(tx2, make_float2(p.x, p.y));
    const float2 dy = __fadd2_rn(ty2, make_float2(p.z, p.w));
    const float2 dz = __fadd2_rn(tz2, make_float2(v.x, v.y));
    const float2 g0 = make_float2(v.z, v.w), g1 = make_float2(w.x, w.y), g2 = make_float2(w.z, w.w);
    float2 r2 = __fmul2_rn(dx, dx);
    r2 = __ffma2_rn(dy, dy, r2);
    r2 = __ffma2_rn(dz, dz, r2);
    float2 ri;
    if (GUARD) {
      ri.x = r2.x > 0.f ? rsqrt_ftz(r2.x) : 0.f;
      ri.y = r2.y > 0.f ? rsqrt_ftz(r2.y) : 0.f;
    } else {
      ri = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
    }
    const float2 ri2 = __fmul2_rn(ri, ri);
    const float2 den = __fmul2_rn(ri, ri2);
    // c = G x d
    const float2 cx = __ffma2_rn(g1, dz, neg2(__fmul2_rn(g2, dy)));
    const float2 cy = __ffma2_rn(g2, dx, neg2(__fmul2_rn(g0, dz)));
    const float2 cz = __ffma2_rn(g0, dy, neg2(__fmul2_rn(g1, dx)));
    if (GS) {
      u[0] = __ffma2_rn(cx, den, u[0]);
      u[1] = __ffma2_rn(cy, den, u[1]);
      u[2] = __ffma2_rn(cz, den, u[2]);
    }
    if (HS) {
      const float2 d5 = __fmul2_rn(den, ri2);
      const float2 px = __fmul2_rn(dx, d5), py = __fmul2_rn(dy, d5), pz = __fmul2_rn(dz, d5);
      Q[0] = __ffma2_rn(px, cx, Q[0]);
      Q[1] = __ffma2_rn(px, cy, Q[1]);
      Q[2] = __ffma2_rn(px, cz, Q[2]);
      Q[3] = __ffma2_rn(py, cx, Q[3]);
      Q[4] = __ffma2_rn(py, cy, Q[4]);
      Q[5] = __ffma2_rn(py, cz, Q[5]);
      Q[6] = __ffma2_rn(pz, cx, Q[6]);
      Q[7] = __ffma2_rn(pz, cy, Q[7]);
      E[0] = __ffma2_rn(g0, den, E[0]);
      E[1] = __ffma2_rn(g1, den, E[1]);
      E[2] = __ffma2_rn(g2, den, E[2]);
    }
  }
  if (GS) {
    acc[0] = u[0];
    acc[1 % NA] = u[1];
    acc[2 % NA] = u[2];
  }
  if (HS) {
    // the gradient is trace-free: d . (G x d) = 0 for every pair, so Q_zz = -(Q_xx + Q_yy)
    Q[8] = neg2(__fadd2_rn(Q[0], Q[4]));
    const float2 m3 = make_float2(-3.f, -3.f);
    acc[(h + 0) % NA] = __fmul2_rn(m3, Q[0]);
    acc[(h + 1) % NA] = __ffma2_rn(m3, Q[1], E[2]);
    acc[(h + 2) % NA] = __ffma2_rn(m3, Q[2], neg2(E[1]));
    acc[(h + 3) % NA] = __ffma2_rn(m3, Q[3], neg2(E[2]));
    acc[(h + 4) % NA] = __fmul2_rn(m3, Q[4]);
    acc[(h + 5) % NA] = __ffma2_rn(m3, Q[5], E[0]);
    acc[(h + 6) % NA] = __ffma2_rn(m3, Q[6], E[1]);
    acc[(h + 7) % NA] = __ffma2_rn(m3, Q[7], neg2(E[0]));
    acc[(h + 8) % NA] = __fmul2_rn(m3, Q[8]);
  }
}

// The batch holding the target's own leaf on the mixed path runs in FP64: its closest
// pairs are the ones whose FP32 coordinates relative to the leaf centre (absolute error
// about 2^-24 of the leaf size) would give large relative errors, and a few such pairs
// dominate the error of the whole field.  The batch holds per body (x, y, z, q) (point
// sources) or (x, y, z, G0, G1, G2) (vortex particles) relative to the target leaf
// centre, in FP64 (the size of the packed FP32 record); the lane's targets are read again
// in FP64.
// the lane's two targets relative to the leaf centre in FP64
__device__ __forceinline__ void self_targets_f64(const double4* __restrict__ tpos, int first, int nt, int ti, int TS,
                                                 double ox, double oy, double oz, double (&tx)[2], double (&ty)[2],
                                                 double (&tz)[2]) {
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    tx[k] = ty[k] = tz[k] = 0.0;
    const int i = ti + k * TS;
    if (i < nt) {
      const double4 p = tpos[first + i];
      tx[k] = p.x - ox;
      ty[k] = p.y - oy;
      tz[k] = p.z - oz;
    }
  }
}

template <bool PS, int NA>
__device__ __noinline__ void self_batch_f64_source(const double4* __restrict__ Bd, int j0, int nb, int SS,
                                                      const double (&tx)[2], const double (&ty)[2],
                                                      const double (&tz)[2], double (&tot)[2][NA]) {
  for (int j = j0; j < nb; j += SS) {
    const double4 sp = Bd[j];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const double dx = tx[k] - sp.x, dy = ty[k] - sp.y, dz = tz[k] - sp.z;
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > 0.0) {
        const double ri = rsqrt(r2);
        const double qr = sp.w * ri;
        if (PS) tot[k][0] += qr;
        const double q3 = qr * ri * ri;
        tot[k][1 % NA] += dx * q3;
        tot[k][2 % NA] += dy * q3;
        tot[k][3 % NA] += dz * q3;
      }
    }
  }
}

template <bool GS, bool HS, int NA>
__device__ __noinline__ void self_batch_f64_vortex(const double2* __restrict__ Bd, int j0, int nb, int SS,
                                                      const double (&tx)[2], const double (&ty)[2],
                                                      const double (&tz)[2], double (&tot)[2][NA]) {
  constexpr int h = GS ? 3 : 0;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    double u[3] = {0.0, 0.0, 0.0}, Q[9], E[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int a = 0; a < 9; ++a) Q[a] = 0.0;
    for (int j = j0; j < nb; j += SS) {
      const double2 a = Bd[3 * j], b = Bd[3 * j + 1], c = Bd[3 * j + 2];
      vortex_pair_qe<double, GS>(tx[k], ty[k], tz[k], a.x, a.y, b.x, b.y, c.x, c.y, u, Q, E);
    }
    if (GS)
#pragma unroll
      for (int c = 0; c < 3; ++c) tot[k][c % NA] += u[c];
    if (HS) {
      double gr[9];
      vortex_grad_from_qe<double>(Q, E, gr);
#pragma unroll
      for (int a = 0; a < 9; ++a) tot[k][(h + a) % NA] += gr[a];
    }
  }
}

// RW: one warp per row (rows of small leaves, kWarps rows per CTA), the warp adding its
// sums to the targets itself; otherwise one CTA per row, the warps splitting its sources.
// W warps per CTA: kWarps, or kWideWarps for launches of few rows (one long row per CTA).
// resident CTAs of the mixed instances: the registers the packed loop needs (the FP64
// branch of the batch holding the target's own leaf is a call, and must not raise them);
// the FP64 vortex CTA path keeps 128 registers (4 CTAs per SM)
template <class R, int KIND, bool HS, bool RW, int W>
__host__ __device__ constexpr int p2p_min_blocks() {
  constexpr int regs = (KIND == FMM_POINT_VORTEX && HS) ? (RW ? 168 : 128) : (RW ? 72 : 64);
  if (sizeof(R) != 4) return (KIND == FMM_POINT_VORTEX && HS && !RW && W == kWarps) ? 4 : 1;
  return 65536 / (regs * W * 32) > 0 ? 65536 / (regs * W * 32) : 1;
}

template <class R, int KIND, bool PS, bool GS, bool HS, bool RW, int W = kWarps>
__global__ void __launch_bounds__(W * 32, p2p_min_blocks<R, KIND, HS, RW, W>()) k_p2p(const int* __restrict__ tgt_list, const int* __restrict__ off,
                                                     int n_rows, const int* __restrict__ src_of,
                                                     const int* __restrict__ t_start, const int* __restrict__ t_count,
                                                     const double* __restrict__ t_center,
                                                     const int* __restrict__ s_start, const int* __restrict__ s_count,
                                                     const double4* __restrict__ tpos, const double4* __restrict__ spos,
                                                     const double4* __restrict__ sstr, double* __restrict__ acc13,
                                                     const int4* __restrict__ chunks, double* __restrict__ chunk_sums,
                                                     int exact_self) {
  // chunks (CTA path only; may be null): CTA b takes the source leaves [y, z) of row x and stores
  // its sums (unscaled, not atomically) at chunk_sums + w + NA * (target index in the row) + channel
  constexpr int NB = batch_bodies<R, KIND>(), NV = Batch<KIND>::nv, NA = n_chan<KIND, GS, HS>();
  constexpr int NS = slots_per_body<R, KIND>();
  constexpr bool MIXED = sizeof(R) == 4;
  constexpr bool PACK = packed<R, KIND>();
  constexpr bool PACKV = packed_vortex<R, KIND>();
  // unpacked vortex particles with the gradient (the FP64 path) sum it as two parts per target
  constexpr bool QE = !PACKV && KIND == FMM_POINT_VORTEX && HS;
  static_assert(!QE || !MIXED, "the mixed vortex path is the packed one");
  static_assert((!PACK && !PACKV) || kTPT == 2, "packed paths pair two targets per lane");
  extern __shared__ __align__(16) unsigned char p2p_smem[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  R* B = reinterpret_cast<R*>(p2p_smem) + w * NS * NB;  // this warp's batch, plane v at B[v * NB]
  double* red = reinterpret_cast<double*>(p2p_smem + W * NS * NB * sizeof(R));  // [W][32 kTPT][NA]
  constexpr bool CH = !RW && W > kWarps;  // only the wide instances take chunks
  const bool chunked = CH && chunks != nullptr;
  const int4 ck = chunked ? chunks[blockIdx.x] : make_int4(0, 0, 0, 0);
  const int row = RW ? blockIdx.x * W + w : (chunked ? ck.x : (int)blockIdx.x);
  if (RW && row >= n_rows) return;  // whole warps: no block barrier on the RW path
  const int t = tgt_list[row];
  const int l0 = chunked ? ck.y : off[row], l1 = chunked ? ck.z : off[row + 1];
  const int ts = t_start[t], tc = t_count[t];
  // this warp's share of the row.  Vortex particles (CTA path): an equal contiguous range of
  // the row's source bodies (leaves in row order, split inside a leaf where a range ends), so
  // the warps reach the block's reduction together whatever the leaf sizes.  Point sources
  // (CTA path): every W-th leaf (an even split measured no faster there, and its registers
  // spill at the packed loop's 64).  One warp per row takes them all.
  constexpr bool BAL = !RW && KIND == FMM_POINT_VORTEX;
  constexpr int LS = (RW || BAL) ? 1 : W;  // stride of this warp's source leaves along the row
  int lb0 = l0 + ((RW || BAL) ? 0 : w), poff0 = 0, rem0 = INT_MAX;
  if (BAL) {
    long long total = 0;
    for (int i = l0 + lane; i < l1; i += 32) total += s_count[src_of[i]];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(kAll, total, o);
    const int b_lo = (int)(total * w / W), b_hi = (int)(total * (w + 1) / W);
    rem0 = b_hi - b_lo;
    int before = 0;  // bodies of the leaves ahead of the current 32
    for (int i0 = l0; i0 < l1 && rem0 > 0; i0 += 32) {
      const int i = i0 + lane;
      const int c = i < l1 ? s_count[src_of[i]] : 0;
      int incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(kAll, incl, o);
        if (lane >= o) incl += v;
      }
      const unsigned past = __ballot_sync(kAll, i < l1 && before + incl > b_lo);
      if (past) {  // the range starts inside leaf i0 + f
        const int f = __ffs(past) - 1;
        const int ex = __shfl_sync(kAll, incl - c, f);
        lb0 = i0 + f;
        poff0 = b_lo - before - ex;
        break;
      }
      before += __shfl_sync(kAll, incl, 31);
    }
  }
  const double ox = MIXED ? t_center[3 * t] : 0.0;
  const double oy = MIXED ? t_center[3 * t + 1] : 0.0;
  const double oz = MIXED ? t_center[3 * t + 2] : 0.0;
  for (int tile = 0; tile < tc; tile += 32 * kTPT) {
    const int nt = min(tc - tile, 32 * kTPT);
    int TS = 1;
    while (TS * kTPT < nt) TS <<= 1;
    const int ti = lane & (TS - 1), slice = lane / TS, SS = 32 / TS;
    R tx[kTPT], ty[kTPT], tz[kTPT];
#pragma unroll
    for (int k = 0; k < kTPT; ++k) {
      tx[k] = ty[k] = tz[k] = R(0);
      int i = ti + k * TS;
      if (i < nt) {
        double4 p = tpos[ts + tile + i];
        tx[k] = (R)(p.x - ox);
        ty[k] = (R)(p.y - oy);
        tz[k] = (R)(p.z - oz);
      }
    }
    R part[kTPT][NA];
    double tot[kTPT][NA];
#pragma unroll
    for (int k = 0; k < kTPT; ++k)
#pragma unroll
      for (int a = 0; a < NA; ++a) part[k][a] = R(0), tot[k][a] = 0.0;
    R Qs[kTPT][9], Es[kTPT][3];  // FP64 vortex gradient as two sums (QE)
#pragma unroll
    for (int k = 0; k < kTPT; ++k) {
#pragma unroll
      for (int a = 0; a < 9; ++a) Qs[k][a] = R(0);
      Es[k][0] = Es[k][1] = Es[k][2] = R(0);
    }
    // next source leaf of this warp, bodies of it already taken, bodies of the range still to take
    int lb = lb0, poff = poff0, rem = rem0;
    while (lb < l1 && rem > 0) {
      // candidate leaves lb + LS * lane; take the longest prefix that fits the batch and the range
      const int l = lb + LS * lane;
      int cnt = 0, sb = 0, sl = -1;
      if (l < l1) {
        sl = src_of[l];
        sb = s_start[sl];
        cnt = s_count[sl];
      }
      if (lane == 0) {
        sb += poff;
        cnt -= poff;
      }
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(kAll, incl, o);
        if (lane >= o) incl += v;
      }
      const int excl = incl - cnt;
      const int lim = min(NB, rem);
      int nl = __popc(__ballot_sync(kAll, l < l1 && incl <= lim));
      int nb;
      if (nl == 0) {  // the first leaf alone overflows the batch or ends the range: lim bodies of it
        nl = 1;
        nb = lim;
        poff += lim;
      } else {
        nb = __shfl_sync(kAll, incl, nl - 1);
        lb += LS * nl;
        poff = 0;
      }
      rem -= nb;
      // the batch holds the target branch's own bodies (coincident pairs certain)
      const bool self_batch = __any_sync(kAll, lane < nl && sl == t);
      // mixed path: that batch in FP64 (the solve's own near field; the influence estimate, which
      // only needs the magnitude of the field, keeps it in FP32 with the r^2 > 0 guard)
      // (vortex ring 2e6, p = 12: velocity error 8e-8 against 9e-7 with that batch in FP32, at the
      // same speed)
      const bool self_f64 = self_batch && exact_self != 0;
      // gather: body idx of the batch lies in candidate leaf k (largest k < nl with excl_k <= idx)
      for (int i0 = 0; i0 < nb; i0 += 32) {
        const int idx = i0 + lane;
        int k = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          int c = k + step;
          int e = __shfl_sync(kAll, excl, c & 31);
          if (c < nl && e <= idx) k = c;
        }
        const int ek = __shfl_sync(kAll, excl, k);
        const int sk = __shfl_sync(kAll, sb, k);
        if ((PACK || PACKV) && self_f64 && idx < nb) {
          // FP64 (x, y, z, q) / (x, y, z, G0), (G1, G2, -, -) relative to the target leaf centre
          const int body = sk + idx - ek;
          const double4 p = spos[body];
          const double4 g = sstr[body];
          if (PACK) {
            reinterpret_cast<double4*>(B)[idx] = make_double4(p.x - ox, p.y - oy, p.z - oz, g.x);
          } else {  // 48 bytes per body, the size of the packed FP32 record
            double2* Bd = reinterpret_cast<double2*>(B) + 3 * idx;
            Bd[0] = make_double2(p.x - ox, p.y - oy);
            Bd[1] = make_double2(p.z - oz, g.x);
            Bd[2] = make_double2(g.y, g.z);
          }
        } else if (PACK && idx < nb) {
          const int body = sk + idx - ek;
          const double4 p = spos[body];
          const float x = -(float)(p.x - ox), y = -(float)(p.y - oy), z = -(float)(p.z - oz), q = (float)sstr[body].x;
          float4* B4 = reinterpret_cast<float4*>(B);
          B4[2 * idx] = make_float4(x, x, y, y);
          B4[2 * idx + 1] = make_float4(z, z, q, q);
        } else if (PACKV && idx < nb) {
          const int body = sk + idx - ek;
          const double4 p = spos[body];
          const double4 g = sstr[body];
          const float x = -(float)(p.x - ox), y = -(float)(p.y - oy), z = -(float)(p.z - oz);
          const float g0 = (float)g.x, g1 = (float)g.y, g2 = (float)g.z;
          float4* B4 = reinterpret_cast<float4*>(B);
          B4[3 * idx] = make_float4(x, x, y, y);
          B4[3 * idx + 1] = make_float4(z, z, g0, g0);
          B4[3 * idx + 2] = make_float4(g1, g1, g2, g2);
        } else if (idx < nb) {
          const int body = sk + idx - ek;
          double4 p = spos[body];
          double4 q = sstr[body];
          B[idx] = (R)(p.x - ox);
          B[NB + idx] = (R)(p.y - oy);
          B[2 * NB + idx] = (R)(p.z - oz);
          B[3 * NB + idx] = (R)q.x;
          if (NV == 6) {
            B[(4 % NV) * NB + idx] = (R)q.y;
            B[(5 % NV) * NB + idx] = (R)q.z;
          }
        }
      }
      __syncwarp();
      if constexpr (PACK) {
        // targets 0 and 1 of the lane in the two halves of every f32x2 operation
        const float4* B4 = reinterpret_cast<const float4*>(B);
        const float2 tx2 = make_float2((float)tx[0], (float)tx[1]);
        const float2 ty2 = make_float2((float)ty[0], (float)ty[1]);
        const float2 tz2 = make_float2((float)tz[0], (float)tz[1]);
        float2 ph = make_float2(0.f, 0.f), gx = ph, gy = ph, gz = ph;
        // the batch holding the target's own leaf runs in FP64 and skips coincident bodies;
        // the others run unguarded and, in the rare case that their sums come out non-finite
        // (bodies that coincide in FP32), repeat the batch with the r^2 > 0 guard
        if (self_f64) {
          double txd[2], tyd[2], tzd[2];
          self_targets_f64(tpos, ts + tile, nt, ti, TS, ox, oy, oz, txd, tyd, tzd);
          self_batch_f64_source<PS, NA>(reinterpret_cast<const double4*>(B), slice, nb, SS, txd, tyd, tzd, tot);
        } else if (self_batch) {
          packed_batch<true, PS>(B4, slice, nb, SS, tx2, ty2, tz2, ph, gx, gy, gz);
        } else {
          packed_batch<false, PS>(B4, slice, nb, SS, tx2, ty2, tz2, ph, gx, gy, gz);
          if (!isfinite(ph.x + ph.y + gx.x + gx.y + gy.x + gy.y + gz.x + gz.y)) {
            ph = gx = gy = gz = make_float2(0.f, 0.f);
            packed_batch<true, PS>(B4, slice, nb, SS, tx2, ty2, tz2, ph, gx, gy, gz);
          }
        }
        part[0][0] += (R)ph.x;
        part[1][0] += (R)ph.y;
        part[0][1 % NA] += (R)gx.x;
        part[1][1 % NA] += (R)gx.y;
        part[0][2 % NA] += (R)gy.x;
        part[1][2 % NA] += (R)gy.y;
        part[0][3 % NA] += (R)gz.x;
        part[1][3 % NA] += (R)gz.y;
      } else if constexpr (PACKV) {
        const float2 tx2 = make_float2((float)tx[0], (float)tx[1]);
        const float2 ty2 = make_float2((float)ty[0], (float)ty[1]);
        const float2 tz2 = make_float2((float)tz[0], (float)tz[1]);
        const float4* B4 = reinterpret_cast<const float4*>(B);
        float2 acc[NA];
        // as on the point-source path: the batch holding the target's own leaf runs in FP64
        if (self_f64) {
#pragma unroll
          for (int a = 0; a < NA; ++a) acc[a] = make_float2(0.f, 0.f);
          double txd[2], tyd[2], tzd[2];
          self_targets_f64(tpos, ts + tile, nt, ti, TS, ox, oy, oz, txd, tyd, tzd);
          self_batch_f64_vortex<GS, HS, NA>(reinterpret_cast<const double2*>(B), slice, nb, SS, txd, tyd, tzd, tot);
        } else if (self_batch) {
          packed_vortex_batch<true, GS, HS, NA>(B4, slice, nb, SS, tx2, ty2, tz2, acc);
        } else {
          packed_vortex_batch<false, GS, HS, NA>(B4, slice, nb, SS, tx2, ty2, tz2, acc);
          float sum = 0.f;
#pragma unroll
          for (int a = 0; a < NA; ++a) sum += acc[a].x + acc[a].y;
          if (!isfinite(sum)) packed_vortex_batch<true, GS, HS, NA>(B4, slice, nb, SS, tx2, ty2, tz2, acc);
        }
#pragma unroll
        for (int a = 0; a < NA; ++a) {
          part[0][a] += (R)acc[a].x;
          part[1][a] += (R)acc[a].y;
        }
      } else if constexpr (QE) {
        for (int j = slice; j < nb; j += SS) {
          const R sx = B[j], sy = B[NB + j], sz = B[2 * NB + j], s0 = B[3 * NB + j];
          const R s1 = B[(4 % NV) * NB + j], s2 = B[(5 % NV) * NB + j];
#pragma unroll
          for (int k = 0; k < kTPT; ++k)
            vortex_pair_qe<R, GS>(tx[k], ty[k], tz[k], sx, sy, sz, s0, s1, s2, part[k], Qs[k], Es[k]);
        }
      } else {
        for (int j = slice; j < nb; j += SS) {
          const R sx = B[j], sy = B[NB + j], sz = B[2 * NB + j], s0 = B[3 * NB + j];
          const R s1 = NV == 6 ? B[(4 % NV) * NB + j] : R(0);
          const R s2 = NV == 6 ? B[(5 % NV) * NB + j] : R(0);
#pragma unroll
          for (int k = 0; k < kTPT; ++k)
            pair1<R, KIND, PS, GS, HS, NA>(tx[k], ty[k], tz[k], sx, sy, sz, s0, s1, s2, part[k]);
        }
      }
      __syncwarp();
      if (MIXED) {
#pragma unroll
        for (int k = 0; k < kTPT; ++k)
#pragma unroll
          for (int a = 0; a < NA; ++a) tot[k][a] += (double)part[k][a], part[k][a] = R(0);
      }
    }
    if constexpr (QE) {
#pragma unroll
      for (int k = 0; k < kTPT; ++k) vortex_grad_from_qe<R>(Qs[k], Es[k], &part[k][(GS ? 3 : 0) % NA]);
    }
    if (!MIXED) {
#pragma unroll
      for (int k = 0; k < kTPT; ++k)
#pragma unroll
        for (int a = 0; a < NA; ++a) tot[k][a] = (double)part[k][a];
    }
    // slices -> lanes ti (< TS), then warps -> shared memory
    for (int o = TS; o < 32; o <<= 1)
#pragma unroll
      for (int k = 0; k < kTPT; ++k)
#pragma unroll
        for (int a = 0; a < NA; ++a) tot[k][a] += __shfl_xor_sync(kAll, tot[k][a], o);
    if constexpr (RW) {
      // one warp owns the row: its sums go to the targets directly
      if (slice == 0) {
#pragma unroll
        for (int k = 0; k < kTPT; ++k) {
          const int i = ti + k * TS;
          if (i < nt)
#pragma unroll
            for (int a = 0; a < NA; ++a) {
              if (KIND == FMM_POINT_SOURCE && a == 0 && !PS) continue;
              atomicAdd(acc13 + 13 * (int64_t)(ts + tile + i) + chan_row<KIND, GS>(a), tot[k][a] * kOneOver4Pi);
            }
        }
      }
      continue;
    }
    if (slice == 0) {
#pragma unroll
      for (int k = 0; k < kTPT; ++k) {
        int i = ti + k * TS;
        if (i < nt)
#pragma unroll
          for (int a = 0; a < NA; ++a) red[(w * 32 * kTPT + i) * NA + a] = tot[k][a];
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nt * NA; e += W * 32) {
      const int i = e / NA, a = e - i * NA;
      double v = 0;
#pragma unroll
      for (int q = 0; q < W; ++q) v += red[(q * 32 * kTPT + i) * NA + a];
      if (chunked) {
        chunk_sums[ck.w + (int64_t)NA * (tile + i) + a] = v;
        continue;
      }
      if (KIND == FMM_POINT_SOURCE && a == 0 && !PS) continue;
      // atomic: under SelfTuning a non-leaf target branch and its own leaves can both own direct-list rows
      atomicAdd(acc13 + 13 * (int64_t)(ts + tile + i) + chan_row<KIND, GS>(a), v * kOneOver4Pi);
    }
    __syncthreads();
  }
}

template <class R, int KIND, bool GS, bool HS, int W = kWarps>
constexpr size_t p2p_smem_bytes() {
  return (size_t)W * slots_per_body<R, KIND>() * batch_bodies<R, KIND>() * sizeof(R) +
         (size_t)W * 32 * kTPT * n_chan<KIND, GS, HS>() * sizeof(double);
}

// all pairs: each CTA owns kP2PThreads*TPT consecutive targets
template <class R, int KIND, bool PS, bool GS, bool HS>
__global__ void __launch_bounds__(kP2PThreads) k_direct(const double4* __restrict__ tpos, int64_t nt_total,
                                                        const double4* __restrict__ spos,
                                                        const double4* __restrict__ sstr, int64_t ns,
                                                        double* __restrict__ acc13) {
  constexpr int TPT = tpt<KIND>();
  __shared__ typename Vec4<R>::T sh_p[kP2PThreads];
  __shared__ typename Vec4<R>::T sh_s[kP2PThreads];
  int64_t base = (int64_t)blockIdx.x * kP2PThreads * TPT;
  double ox = 0, oy = 0, oz = 0;
  if (sizeof(R) == 4 && base < nt_total) {
    double4 p = tpos[base];
    ox = p.x;
    oy = p.y;
    oz = p.z;
  }
  R tx[TPT], ty[TPT], tz[TPT];
  Acc<R, TPT> acc;
  acc.init();
  int nt = 0;
#pragma unroll
  for (int k = 0; k < TPT; ++k) {
    int64_t i = base + threadIdx.x + k * kP2PThreads;
    tx[k] = ty[k] = tz[k] = R(0);
    if (i < nt_total) {
      double4 p = tpos[i];
      tx[k] = (R)(p.x - ox);
      ty[k] = (R)(p.y - oy);
      tz[k] = (R)(p.z - oz);
      nt = k + 1;
    }
  }
  for (int64_t c = 0; c < ns; c += kP2PThreads) {
    int64_t j = c + threadIdx.x;
    if (j < ns) {
      double4 p = spos[j];
      double4 q = sstr[j];
      sh_p[threadIdx.x] = {(R)(p.x - ox), (R)(p.y - oy), (R)(p.z - oz), R(0)};
      sh_s[threadIdx.x] = {(R)q.x, (R)q.y, (R)q.z, R(0)};
    }
    __syncthreads();
    int m = (int)min((int64_t)kP2PThreads, ns - c);
    for (int jj = 0; jj < m; ++jj) {
      auto P = sh_p[jj];
      auto S = sh_s[jj];
      interact<R, KIND, PS, GS, HS, TPT>(tx, ty, tz, nt, P.x, P.y, P.z, S.x, S.y, S.z, acc.part);
    }
    acc.flush();
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < TPT; ++k) {
    int64_t i = base + threadIdx.x + k * kP2PThreads;
    if (i < nt_total) store<KIND, PS, GS, HS>(acc13 + 13 * i, acc, k);
  }
}

// Sums of the chunks of each row (rowtab[r] = first chunk, end) in chunk order, added to the
// row's targets: the near field of launches whose rows were cut into chunks.
template <int KIND, bool PS, bool GS, int NA>
__global__ void k_p2p_chunk_sum(const int4* __restrict__ rowtab, const int4* __restrict__ chunks,
                                const double* __restrict__ part, const int* __restrict__ tgt_list,
                                const int* __restrict__ t_start, const int* __restrict__ t_count,
                                double* __restrict__ acc13) {
  const int r = blockIdx.x;
  const int4 rt = rowtab[r];
  const int t = tgt_list[r];
  const int ts = t_start[t], tc = t_count[t];
  for (int e = threadIdx.x; e < tc * NA; e += blockDim.x) {
    const int i = e / NA, a = e - i * NA;
    if (KIND == FMM_POINT_SOURCE && a == 0 && !PS) continue;
    double v = 0.0;
    for (int c = rt.x; c < rt.y; ++c) v += part[chunks[c].w + (int64_t)e];
    // atomic: under SelfTuning a non-leaf target branch and its own leaves can both own rows
    atomicAdd(acc13 + 13 * (int64_t)(ts + i) + chan_row<KIND, GS>(a), v * kOneOver4Pi);
  }
}

template <class R, int KIND, bool PS, bool GS, bool HS>
void run_p2p(const DevTree& tt, const DevTree& stt, DevLists& L, double* acc13, int exact_self, cudaStream_t st) {
  if (L.n_dir_targets == 0) return;
  constexpr size_t smem = p2p_smem_bytes<R, KIND, GS, HS>();
  const int rows = (int)L.n_dir_targets;
  note_launch();
  // target leaves of a few bodies (on average <= 8), packed FP32 kernel: one warp per row
  // (measured slower for the FP64 kernel, whose rows keep a CTA each)
  if (packed<R, KIND>() && tt.n_bodies <= 8 * tt.n_leaves) {
    if (smem > 48 * 1024)
      FMM_CUDA_TRY(cudaFuncSetAttribute(k_p2p<R, KIND, PS, GS, HS, true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_p2p<R, KIND, PS, GS, HS, true><<<(rows + kWarps - 1) / kWarps, kWarps * 32, smem, st>>>(
        L.dir_tgt.ptr, L.dir_off.ptr, rows, L.dir_s.ptr, tt.body_start.ptr, tt.body_count.ptr, tt.tcenter.ptr,
        stt.body_start.ptr, stt.body_count.ptr, tt.pos.ptr, stt.pos.ptr, stt.str.ptr, acc13, nullptr,
        nullptr, exact_self);
  } else {
    int dev = 0, n_sm = 0;
    FMM_CUDA_TRY(cudaGetDevice(&dev));
    FMM_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    // estimated body pairs of the launch: chunking costs a host round trip and a second kernel,
    // which only pays for launches of much work (and the round trip holds back a serving
    // worker's next launches)
    const double est_pairs = (double)L.n_direct * ((double)stt.n_bodies / std::max<int64_t>(1, stt.n_leaves)) *
                             ((double)tt.n_bodies / std::max<int64_t>(1, tt.n_leaves));
    const bool chunk = est_pairs > kChunkPairs;
    if (rows < kWideRowsPerSM * n_sm && !chunk) {
      constexpr size_t smw = p2p_smem_bytes<R, KIND, GS, HS, kWideWarps>();
      FMM_CUDA_TRY(cudaFuncSetAttribute(k_p2p<R, KIND, PS, GS, HS, false, kWideWarps>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smw));
      k_p2p<R, KIND, PS, GS, HS, false, kWideWarps><<<rows, kWideWarps * 32, smw, st>>>(
          L.dir_tgt.ptr, L.dir_off.ptr, rows, L.dir_s.ptr, tt.body_start.ptr, tt.body_count.ptr, tt.tcenter.ptr,
          stt.body_start.ptr, stt.body_count.ptr, tt.pos.ptr, stt.pos.ptr, stt.str.ptr, acc13, nullptr, nullptr,
          exact_self);
    } else if (rows < kWideRowsPerSM * n_sm) {
      // few rows: cut them into chunks of about the same number of source leaves (some
      // kChunksPerSM per SM over the launch), one wide CTA each; the chunks' partial sums are
      // added in chunk order by k_p2p_chunk_sum
      constexpr int NA = n_chan<KIND, GS, HS>();
      std::vector<int> h_off(rows + 1), h_tgt(rows), h_cnt(tt.n_branches);
      FMM_CUDA_TRY(cudaMemcpyAsync(h_off.data(), L.dir_off.ptr, (rows + 1) * sizeof(int), cudaMemcpyDeviceToHost, st));
      FMM_CUDA_TRY(cudaMemcpyAsync(h_tgt.data(), L.dir_tgt.ptr, rows * sizeof(int), cudaMemcpyDeviceToHost, st));
      FMM_CUDA_TRY(cudaMemcpyAsync(h_cnt.data(), tt.body_count.ptr, tt.n_branches * sizeof(int),
                                   cudaMemcpyDeviceToHost, st));
      FMM_CUDA_TRY(cudaStreamSynchronize(st));
      const int64_t total = (int64_t)h_off[rows] - h_off[0], goal = (int64_t)kChunksPerSM * n_sm;
      const int64_t per = std::max<int64_t>(2 * kWideWarps, (total + goal - 1) / goal);
      std::vector<int4> ch, rt(rows);
      int64_t out = 0;
      for (int r = 0; r < rows; ++r) {
        const int a = h_off[r], nl = h_off[r + 1] - a;
        const int k = (int)std::max<int64_t>(1, (nl + per - 1) / per);
        rt[r] = make_int4((int)ch.size(), (int)ch.size() + k, 0, 0);
        const int64_t nt = h_cnt[h_tgt[r]];
        for (int j = 0; j < k; ++j) {
          ch.push_back(make_int4(r, a + (int)((int64_t)nl * j / k), a + (int)((int64_t)nl * (j + 1) / k), (int)out));
          out += nt * NA;
          FMM_CHECK(out < INT_MAX, FMM_ERR_MEMORY, "near-field chunk sums exceed the index range");
        }
      }
      // floors of a few MB: regrowing frees device memory, which waits for the whole device (and
      // for every other context's work on it)
      L.p2p_chunks.grow(std::max<size_t>(ch.size(), 1 << 16));
      L.p2p_rowtab.grow(std::max<size_t>(rows, 1 << 12));
      L.p2p_part.grow(std::max<size_t>((size_t)out + 1, 1 << 19));
      FMM_CUDA_TRY(cudaMemcpyAsync(L.p2p_chunks.ptr, ch.data(), ch.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
      FMM_CUDA_TRY(cudaMemcpyAsync(L.p2p_rowtab.ptr, rt.data(), rt.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
      constexpr size_t smw = p2p_smem_bytes<R, KIND, GS, HS, kWideWarps>();
      FMM_CUDA_TRY(cudaFuncSetAttribute(k_p2p<R, KIND, PS, GS, HS, false, kWideWarps>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smw));
      k_p2p<R, KIND, PS, GS, HS, false, kWideWarps><<<(int)ch.size(), kWideWarps * 32, smw, st>>>(
          L.dir_tgt.ptr, L.dir_off.ptr, rows, L.dir_s.ptr, tt.body_start.ptr, tt.body_count.ptr, tt.tcenter.ptr,
          stt.body_start.ptr, stt.body_count.ptr, tt.pos.ptr, stt.pos.ptr, stt.str.ptr, acc13, L.p2p_chunks.ptr,
          L.p2p_part.ptr, exact_self);
      FMM_CUDA_TRY(cudaGetLastError());
      note_launch();
      k_p2p_chunk_sum<KIND, PS, GS, NA><<<rows, 256, 0, st>>>(L.p2p_rowtab.ptr, L.p2p_chunks.ptr, L.p2p_part.ptr,
                                                               L.dir_tgt.ptr, tt.body_start.ptr, tt.body_count.ptr,
                                                               acc13);
    } else {
      if (smem > 48 * 1024)
        FMM_CUDA_TRY(cudaFuncSetAttribute(k_p2p<R, KIND, PS, GS, HS, false>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_p2p<R, KIND, PS, GS, HS, false><<<rows, kWarps * 32, smem, st>>>(
          L.dir_tgt.ptr, L.dir_off.ptr, rows, L.dir_s.ptr, tt.body_start.ptr, tt.body_count.ptr, tt.tcenter.ptr,
          stt.body_start.ptr, stt.body_count.ptr, tt.pos.ptr, stt.pos.ptr, stt.str.ptr, acc13, nullptr,
        nullptr, exact_self);
    }
  }
  FMM_CUDA_TRY(cudaGetLastError());
}

template <class R, int KIND, bool PS, bool GS, bool HS>
void run_direct(const double4* tpos, int64_t nt, const double4* spos, const double4* sstr, int64_t ns, double* acc13,
                cudaStream_t st) {
  constexpr int T = tpt<KIND>();
  int64_t blocks = (nt + kP2PThreads * T - 1) / (kP2PThreads * T);
  if (blocks == 0) return;
  note_launch();
  k_direct<R, KIND, PS, GS, HS><<<(int)blocks, kP2PThreads, 0, st>>>(tpos, nt, spos, sstr, ns, acc13);
  FMM_CUDA_TRY(cudaGetLastError());
}

template <class R, class F>
void dispatch(int kind, bool ps, bool gs, bool hs, F& f) {
  // Laplace: phi optional, gradient always (the reference's kernel ignores the switch)
  if (kind == FMM_POINT_SOURCE) {
    if (ps)
      f.template go<R, FMM_POINT_SOURCE, true, true, false>();
    else
      f.template go<R, FMM_POINT_SOURCE, false, true, false>();
  } else {
    if (gs && hs)
      f.template go<R, FMM_POINT_VORTEX, false, true, true>();
    else if (hs)
      f.template go<R, FMM_POINT_VORTEX, false, false, true>();
    else
      f.template go<R, FMM_POINT_VORTEX, false, true, false>();
  }
}

struct P2PLaunch {
  const DevTree& tt;
  const DevTree& stt;
  DevLists& L;
  double* acc13;
  int exact_self;
  cudaStream_t st;
  template <class R, int K, bool PS, bool GS, bool HS>
  void go() {
    run_p2p<R, K, PS, GS, HS>(tt, stt, L, acc13, exact_self, st);
  }
};

struct DirectLaunch {
  const double4* tpos;
  int64_t nt;
  const double4* spos;
  const double4* sstr;
  int64_t ns;
  double* acc13;
  cudaStream_t st;
  template <class R, int K, bool PS, bool GS, bool HS>
  void go() {
    run_direct<R, K, PS, GS, HS>(tpos, nt, spos, sstr, ns, acc13, st);
  }
};

__global__ void k_pair_count(const int* __restrict__ dt, const int* __restrict__ ds, int64_t n,
                             const int* __restrict__ tcount, const int* __restrict__ scount,
                             unsigned long long* __restrict__ out) {
  unsigned long long v = 0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    v += (unsigned long long)tcount[dt[k]] * (unsigned long long)scount[ds[k]];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, v);
}

}  // namespace

void count_p2p_pairs(const DevTree& tt, const DevTree& stt, const DevLists& L, unsigned long long* out,
                     cudaStream_t st) {
  if (L.n_direct == 0) return;
  int g = (int)std::min<int64_t>((L.n_direct + 255) / 256, 148 * 8);
  note_launch();
  k_pair_count<<<g, 256, 0, st>>>(L.dir_t.ptr, L.dir_s.ptr, L.n_direct, tt.body_count.ptr, stt.body_count.ptr, out);
  FMM_CUDA_TRY(cudaGetLastError());
}

void launch_p2p(const DevTree& tt, const DevTree& stt, DevLists& L, double* acc13, int kind, bool ps, bool gs,
                bool hs, int precision, cudaStream_t st, bool exact_self) {
  P2PLaunch f{tt, stt, L, acc13, exact_self ? 1 : 0, st};
  if (precision == FMM_PRECISION_MIXED)
    dispatch<float>(kind, ps, gs, hs, f);
  else
    dispatch<double>(kind, ps, gs, hs, f);
}

void launch_direct(const double4* tpos, int64_t nt, const double4* spos, const double4* sstr, int64_t ns, double* acc13,
                   int kind, bool gs, bool hs, int precision, cudaStream_t st) {
  DirectLaunch f{tpos, nt, spos, sstr, ns, acc13, st};
  // direct! always evaluates the potential of point sources (src/direct.jl:66-70 + test/gravitational.jl:92)
  if (precision == FMM_PRECISION_MIXED)
    dispatch<float>(kind, true, gs, hs, f);
  else
    dispatch<double>(kind, true, gs, hs, f);
}

}  // namespace fmmb

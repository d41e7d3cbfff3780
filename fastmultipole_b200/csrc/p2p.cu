// p2p.cu -- near-field (P2P) kernels over the target-sorted direct list.
//
// Kernels of the reference's point systems:
//   Laplace point source  (test/gravitational.jl:80-104): phi += q/(4 pi r),
//     grad += q dx/(4 pi r^3), pairs with r^2 = 0 skipped, no hessian;
//   vortex particle       (test/vortex.jl:83-128): u = (dx x Gamma)/(4 pi r^3)
//     and the 9-term velocity gradient.
// One CTA owns one target leaf (so no atomics): its targets sit in registers,
// the bodies of each source leaf of its direct-list row are staged through
// shared memory and broadcast to all threads.  FP64 is the drop-in arithmetic;
// the MIXED variant moves every body relative to the target leaf centre in
// FP64, then evaluates the kernel in FP32 (rsqrt on the SFU), summing each
// source leaf in FP32 and the leaf partials in FP64.
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

template <class R, int KIND, bool PS, bool GS, bool HS>
__global__ void __launch_bounds__(kP2PThreads) k_p2p(const int* __restrict__ tgt_list, const int* __restrict__ off,
                                                     const int* __restrict__ src_of, const int* __restrict__ t_start,
                                                     const int* __restrict__ t_count, const double* __restrict__ t_center,
                                                     const int* __restrict__ s_start, const int* __restrict__ s_count,
                                                     const double4* __restrict__ tpos, const double4* __restrict__ spos,
                                                     const double4* __restrict__ sstr, double* __restrict__ acc13) {
  constexpr int TPT = tpt<KIND>();
  __shared__ typename Vec4<R>::T sh_p[kP2PThreads];
  __shared__ typename Vec4<R>::T sh_s[kP2PThreads];
  const int b = blockIdx.x;
  const int t = tgt_list[b];
  const int l0 = off[b], l1 = off[b + 1];
  const int ts = t_start[t], tc = t_count[t];
  // FP32 evaluates relative to the target leaf centre; FP64 uses absolute coordinates
  const double ox = (sizeof(R) == 4) ? t_center[3 * t] : 0.0;
  const double oy = (sizeof(R) == 4) ? t_center[3 * t + 1] : 0.0;
  const double oz = (sizeof(R) == 4) ? t_center[3 * t + 2] : 0.0;
  for (int tile = 0; tile < tc; tile += kP2PThreads * TPT) {
    R tx[TPT], ty[TPT], tz[TPT];
    Acc<R, TPT> acc;
    acc.init();
    int nt = 0;
#pragma unroll
    for (int k = 0; k < TPT; ++k) {
      int i = tile + threadIdx.x + k * kP2PThreads;
      tx[k] = ty[k] = tz[k] = R(0);
      if (i < tc) {
        double4 p = tpos[ts + i];
        tx[k] = (R)(p.x - ox);
        ty[k] = (R)(p.y - oy);
        tz[k] = (R)(p.z - oz);
        nt = k + 1;
      }
    }
    for (int l = l0; l < l1; ++l) {
      const int s = src_of[l];
      const int ss = s_start[s], scnt = s_count[s];
      for (int c = 0; c < scnt; c += kP2PThreads) {
        int j = c + threadIdx.x;
        if (j < scnt) {
          double4 p = spos[ss + j];
          double4 q = sstr[ss + j];
          sh_p[threadIdx.x] = {(R)(p.x - ox), (R)(p.y - oy), (R)(p.z - oz), R(0)};
          sh_s[threadIdx.x] = {(R)q.x, (R)q.y, (R)q.z, R(0)};
        }
        __syncthreads();
        int m = min(kP2PThreads, scnt - c);
        for (int jj = 0; jj < m; ++jj) {
          auto P = sh_p[jj];
          auto S = sh_s[jj];
          interact<R, KIND, PS, GS, HS, TPT>(tx, ty, tz, nt, P.x, P.y, P.z, S.x, S.y, S.z, acc.part);
        }
        __syncthreads();
      }
      acc.flush();
    }
#pragma unroll
    for (int k = 0; k < TPT; ++k) {
      int i = tile + threadIdx.x + k * kP2PThreads;
      if (i < tc) store<KIND, PS, GS, HS>(acc13 + 13 * (int64_t)(ts + i), acc, k);
    }
  }
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

template <class R, int KIND, bool PS, bool GS, bool HS>
void run_p2p(const DevTree& tt, const DevTree& stt, const DevLists& L, double* acc13, cudaStream_t st) {
  if (L.n_dir_targets == 0) return;
  note_launch();
  k_p2p<R, KIND, PS, GS, HS><<<(int)L.n_dir_targets, kP2PThreads, 0, st>>>(
      L.dir_tgt.ptr, L.dir_off.ptr, L.dir_s.ptr, tt.body_start.ptr, tt.body_count.ptr, tt.tcenter.ptr,
      stt.body_start.ptr, stt.body_count.ptr, tt.pos.ptr, stt.pos.ptr, stt.str.ptr, acc13);
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
  const DevLists& L;
  double* acc13;
  cudaStream_t st;
  template <class R, int K, bool PS, bool GS, bool HS>
  void go() {
    run_p2p<R, K, PS, GS, HS>(tt, stt, L, acc13, st);
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

void launch_p2p(const DevTree& tt, const DevTree& stt, const DevLists& L, double* acc13, int kind, bool ps, bool gs,
                bool hs, int precision, cudaStream_t st) {
  P2PLaunch f{tt, stt, L, acc13, st};
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

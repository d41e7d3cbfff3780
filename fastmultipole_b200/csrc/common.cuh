// common.cuh -- shared definitions of the B200 FMM library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/fmm_b200.h"

namespace fmmb {

constexpr int kMaxP = 20;         // highest expansion order the kernels are instantiated for
// 1/k! for k = 0..kMaxP, correctly rounded: the coaxial translations multiply by these in place
// of dividing by k! (within an ulp of the quotient)
#define FMM_INV_FACTORIALS \
    1.0, 1.0, 0.5, 0.16666666666666666, 0.041666666666666664, 0.008333333333333333, 0.001388888888888889, \
    0.0001984126984126984, 2.48015873015873e-05, 2.7557319223985893e-06, 2.755731922398589e-07, \
    2.505210838544172e-08, 2.08767569878681e-09, 1.6059043836821613e-10, 1.1470745597729725e-11, \
    7.647163731819816e-13, 4.779477332387385e-14, 2.8114572543455206e-15, 1.5619206968586225e-16, \
    8.22063524662433e-18, 4.110317623312165e-19
constexpr int kMaxDepth = 21;     // octree levels representable by a 63-bit octant path key
constexpr double kOneOver4Pi = 1.0 / (4.0 * 3.141592653589793);
constexpr double kPi = 3.141592653589793;

__host__ __device__ inline int64_t nh(int p) { return (int64_t)(p + 1) * (p + 2) / 2; }
__host__ __device__ inline int hidx(int n, int m) { return n * (n + 1) / 2 + m; }
__host__ __device__ inline int64_t length_Hs(int p) { return p < 0 ? 0 : (int64_t)(p + 1) * (p + 2) * (p + 3) / 6; }
__host__ __device__ inline int64_t length_Ts(int p) { return p < 0 ? 0 : (int64_t)(p + 1) * (p + 2) * (2 * p + 3) / 6; }
__host__ __device__ inline int H_index(int mp, int m) { return m * (m + 1) / 2 + mp; }
__host__ __device__ inline int T_index(int mp, int m) { return m * m + mp + m; }

// Kernel launches issued by this host thread (reported per solve in fmm_result).
inline thread_local int64_t g_launches = 0;
inline void note_launch() { ++g_launches; }

// Status plumbing: every entry point returns an fmm_status and never aborts.
struct Error {
  int code;
  std::string msg;
};

#define FMM_CUDA_TRY(expr)                                                         \
  do {                                                                             \
    cudaError_t e_ = (expr);                                                       \
    if (e_ != cudaSuccess)                                                         \
      throw ::fmmb::Error{FMM_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)}; \
  } while (0)

#define FMM_CHECK(cond, code, msg)                            \
  do {                                                        \
    if (!(cond)) throw ::fmmb::Error{(code), std::string(msg)}; \
  } while (0)

// A growable device allocation owned by a context.  grow() keeps nothing.
template <class T>
struct DevBuf {
  T* ptr = nullptr;
  size_t cap = 0;
  void grow(size_t n) {
    if (n <= cap) return;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    size_t want = n + n / 4 + 64;
    FMM_CUDA_TRY(cudaMalloc((void**)&ptr, want * sizeof(T)));
    cap = want;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
  }
};

// Constant tables of the rotation-based operators (host generated, FP64).
struct HostTables {
  int p = -1;
  std::vector<double> Hs, zeta, eta, Mt, Lt;
};
void build_tables(HostTables& t, int p);

}  // namespace fmmb

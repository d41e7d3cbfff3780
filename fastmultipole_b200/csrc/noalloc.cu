// noalloc.cu -- fmm_direct_noalloc: all-pairs direct! that allocates nothing.
//
// Some callers cannot call cudaMalloc: code running while a CUDA graph is being
// captured (an allocation would break or be baked into the capture), hosts that
// hand the library a fixed device-memory arena and forbid further allocations,
// and real-time loops that must not touch the allocator.  This entry point
// serves them: the caller passes device-resident inputs and output, and the
// only device memory the call uses besides them is the static array below.
//
// The array is a file-scope __device__ object of fixed size, so every GPU that
// loads the library holds it (6.6 MB) until the process exits.  Every call on
// a device shares it and it keeps the last call's contents: the accumulators
// are cleared by each call, and two calls that overlap on the GPU (different
// streams, or different host threads) race on it.
#include <mutex>

#include "context.cuh"

namespace fmmb {

namespace {

// 32,768 sources and 32,768 targets: unpacked source position+radius and strength,
// target positions and the 13 accumulators per target, all double.
constexpr int64_t kNoAllocMaxBodies = 32768;
constexpr int64_t kNoAllocDoubles = kNoAllocMaxBodies * (4 + 4 + 4 + 13);

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// In host code `g_noalloc_scratch` names a host-side stand-in, not device memory;
// its device address is looked up with that device current.  Only a successful
// lookup is kept, so a failed first attempt (a pending error, a call made during
// a capture) is retried by the next call instead of disabling the device.
std::mutex g_addr_mutex;
double* g_addr[64] = {};

double* scratch_for(int device, cudaError_t& err) {
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  err = cudaSuccess;
  if (!g_addr[device]) {
    double* ptr = nullptr;
    err = cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch);
    if (err != cudaSuccess) return nullptr;
    g_addr[device] = ptr;
  }
  return g_addr[device];
}

// The caller's current device is restored on every return.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

__global__ void k_unpack_na(const double* __restrict__ buf, int64_t n, int64_t stride, int ns, int has_r,
                            double4* __restrict__ pos, double4* __restrict__ str) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double* b = buf + i * stride;
    pos[i] = make_double4(b[0], b[1], b[2], has_r ? b[3] : 0.0);
    double4 s = make_double4(0, 0, 0, 0);
    if (ns >= 1) s.x = b[4];
    if (ns >= 3) {
      s.y = b[5];
      s.z = b[6];
    }
    if (str) str[i] = s;
  }
}

__global__ void k_write_na(const double* __restrict__ acc13, const double4* __restrict__ pos, int64_t n,
                           double* __restrict__ out16) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double4 p = pos[i];
    double* d = out16 + 16 * i;
    d[0] = p.x;
    d[1] = p.y;
    d[2] = p.z;
    for (int k = 0; k < 13; ++k) d[3 + k] = acc13[13 * i + k];
  }
}

int grid_na(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 1184)); }

}  // namespace

}  // namespace fmmb

using namespace fmmb;

extern "C" FMM_API int fmm_direct_noalloc(int device, void* cuda_stream, const fmm_target_system* target,
                                          const fmm_source_system* source, int scalar_potential, int gradient,
                                          int hessian, int precision) {
  if (!target || !source) return FMM_ERR_ARGUMENT;
  if (source->kind != FMM_POINT_SOURCE && source->kind != FMM_POINT_VORTEX) return FMM_ERR_ARGUMENT;
  if (source->data_per_body < 4 + source->kind || source->n_bodies < 0) return FMM_ERR_ARGUMENT;
  if (precision != FMM_PRECISION_F64 && precision != FMM_PRECISION_MIXED) return FMM_ERR_ARGUMENT;
  const bool self = target->positions == nullptr;
  if (!self && target->n_bodies < 0) return FMM_ERR_ARGUMENT;
  const int64_t nt = self ? source->n_bodies : target->n_bodies;
  const int64_t ns = source->n_bodies;
  // device-resident inputs and output only: staging host memory would need device memory
  if (source->memory != FMM_MEMORY_DEVICE || target->memory != FMM_MEMORY_DEVICE) return FMM_ERR_ARGUMENT;
  if (!self && target->stride < 3) return FMM_ERR_ARGUMENT;
  if ((ns > 0 && !source->buffer) || (nt > 0 && !target->out)) return FMM_ERR_ARGUMENT;
  if (ns > kNoAllocMaxBodies || nt > kNoAllocMaxBodies) return FMM_ERR_MEMORY;  // beyond the static scratch
  if (device < 0 || device >= 64) return FMM_ERR_ARGUMENT;
  DeviceGuard restore;
  if (cudaSetDevice(device) != cudaSuccess) return FMM_ERR_NO_DEVICE;
  if (nt == 0) return FMM_OK;
  cudaError_t err;
  double* base = scratch_for(device, err);
  if (!base) return FMM_ERR_CUDA;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(cuda_stream);
  double4* spos = reinterpret_cast<double4*>(base);
  double4* sstr = spos + kNoAllocMaxBodies;
  double4* tpos = sstr + kNoAllocMaxBodies;
  double* acc = reinterpret_cast<double*>(tpos + kNoAllocMaxBodies);
  try {
    if (ns > 0)
      k_unpack_na<<<grid_na(ns), 256, 0, st>>>(source->buffer, ns, source->data_per_body, source->kind, 1, spos, sstr);
    const double* tp = self ? source->buffer : target->positions;
    k_unpack_na<<<grid_na(nt), 256, 0, st>>>(tp, nt, self ? source->data_per_body : target->stride, 0, 0, tpos,
                                            nullptr);
    // the scratch keeps the previous call's sums: clear the accumulators
    FMM_CUDA_TRY(cudaMemsetAsync(acc, 0, 13 * nt * sizeof(double), st));
    (void)scalar_potential;
    launch_direct(tpos, nt, spos, sstr, ns, acc, source->kind, gradient != 0, hessian != 0, precision, st);
    k_write_na<<<grid_na(nt), 256, 0, st>>>(acc, tpos, nt, target->out);
    FMM_CUDA_TRY(cudaGetLastError());
  } catch (const Error& e) {
    return e.code;
  }
  return FMM_OK;
}

// peak.cu -- measured CUDA-core FP32 throughput, the denominator of the near-field
// roofline (the pairwise kernels are FP32 FMA work on the CUDA cores, not tensor-core
// or memory work, so neither a copy bandwidth nor a GEMM peak bounds them).
//
// Every thread runs 8 independent fused multiply-add chains (packed f32x2 operations,
// the form the mixed near field issues, or scalar ones) for a fixed number of
// iterations; the grid holds many resident warps per SM, so the FMA pipes, not
// latency, set the rate.  Timed with CUDA events around one launch after a warm-up.
#include "context.cuh"

namespace fmmb {
namespace {

constexpr int kPeakChains = 8;
constexpr int kPeakIters = 16384;
constexpr int kPeakThreads = 256;

template <bool PACKED>
__global__ void __launch_bounds__(kPeakThreads) k_fma_peak(float seed, float* __restrict__ sink) {
  const float b0 = seed * 0.999f, c0 = seed * 1e-3f;
  if constexpr (PACKED) {
    float2 a[kPeakChains];
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k) a[k] = make_float2(seed + k, seed - k);
    const float2 b = make_float2(b0, b0), c = make_float2(c0, -c0);
#pragma unroll 4
    for (int it = 0; it < kPeakIters; ++it)
#pragma unroll
      for (int k = 0; k < kPeakChains; ++k) a[k] = __ffma2_rn(a[k], b, c);
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k) s += a[k].x + a[k].y;
    if (s == 12345.678f) sink[threadIdx.x] = s;  // keeps the chains live
  } else {
    float a[kPeakChains];
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k) a[k] = seed + k;
#pragma unroll 4
    for (int it = 0; it < kPeakIters; ++it)
#pragma unroll
      for (int k = 0; k < kPeakChains; ++k) a[k] = fmaf(a[k], b0, c0);
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k) s += a[k];
    if (s == 12345.678f) sink[threadIdx.x] = s;
  }
}

}  // namespace
}  // namespace fmmb

using namespace fmmb;

extern "C" FMM_API int fmm_measure_fp32_peak(int device, int packed, double* tflops) {
  if (!tflops) return FMM_ERR_ARGUMENT;
  *tflops = 0.0;
  int prev = -1;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return FMM_ERR_NO_DEVICE;
  int rc = FMM_OK;
  float* sink = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  try {
    int n_sm = 0;
    FMM_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device));
    FMM_CUDA_TRY(cudaMalloc(&sink, kPeakThreads * sizeof(float)));
    FMM_CUDA_TRY(cudaEventCreate(&e0));
    FMM_CUDA_TRY(cudaEventCreate(&e1));
    const int blocks = n_sm * 8;
    float ms = 0.0f;
    for (int rep = 0; rep < 2; ++rep) {  // the first launch warms up
      FMM_CUDA_TRY(cudaEventRecord(e0, 0));
      if (packed)
        k_fma_peak<true><<<blocks, kPeakThreads>>>(1.0001f, sink);
      else
        k_fma_peak<false><<<blocks, kPeakThreads>>>(1.0001f, sink);
      FMM_CUDA_TRY(cudaGetLastError());
      FMM_CUDA_TRY(cudaEventRecord(e1, 0));
      FMM_CUDA_TRY(cudaEventSynchronize(e1));
      FMM_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    }
    // flops: one FMA = 2, packed operations carry two FMAs
    const double fmas = (double)blocks * kPeakThreads * kPeakIters * kPeakChains * (packed ? 2 : 1);
    *tflops = 2.0 * fmas / (ms * 1e-3) / 1e12;
  } catch (const Error& e) {
    rc = e.code;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (sink) cudaFree(sink);
  if (prev >= 0) cudaSetDevice(prev);
  return rc;
}

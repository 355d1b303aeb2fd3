// peaks.cu -- the FP64 / FP32 FMA throughput of this GPU, measured.
//
// The compute-bound shape kernels are reported against the arithmetic peak of
// the GPU they run on.  That peak is measured here, not taken from a data
// sheet: every thread runs kChains independent FMA chains (enough independent
// work to cover the FMA latency), the grid is a whole number of waves of
// resident blocks on every SM, and the launch is timed with CUDA events on the
// caller's stream.  One FMA counts two flops.  The chains stay finite
// (acc = acc * a + b with |a| < 1 converges), and their sum is kept in a
// __device__ word so the compiler cannot drop them.
#include <cuda_runtime.h>

#include "geometry.h"

namespace vgb {
namespace {

constexpr int kChains = 8;
constexpr int kBlock = 256;

__device__ double g_peak_sink64;
__device__ float g_peak_sink32;

template <class T>
__device__ __forceinline__ T fma_t(T a, T b, T c);
template <>
__device__ __forceinline__ double fma_t<double>(double a, double b, double c) {
  return __fma_rn(a, b, c);
}
template <>
__device__ __forceinline__ float fma_t<float>(float a, float b, float c) {
  return __fmaf_rn(a, b, c);
}

template <class T>
__global__ void __launch_bounds__(kBlock) k_fma_peak(int iters, T a, T b) {
  T acc[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) acc[c] = (T)(threadIdx.x + c) * (T)1e-3;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) acc[c] = fma_t<T>(acc[c], a, b);
  }
  T s = 0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += acc[c];
  // practically never true; the store keeps every chain alive
  if (s == (T)-1.2345) {
    if (sizeof(T) == 8)
      g_peak_sink64 = (double)s;
    else
      g_peak_sink32 = (float)s;
  }
}

template <class T>
vgb_status run_peak(int32_t iters, cudaStream_t s, double *flops, float *ms) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fma_peak<T>, kBlock, 0);
  if (e != cudaSuccess) return cuda_error(e, "vgb_measure_fma_peak: device query");
  const int grid = sms * (per_sm > 0 ? per_sm : 1);
  cudaEvent_t e0, e1;
  e = cudaEventCreate(&e0);
  if (e != cudaSuccess) return cuda_error(e, "vgb_measure_fma_peak: event");
  e = cudaEventCreate(&e1);
  if (e != cudaSuccess) {
    cudaEventDestroy(e0);
    return cuda_error(e, "vgb_measure_fma_peak: event");
  }
  const T a = (T)0.999, b = (T)1e-3;
  cudaEventRecord(e0, s);
  k_fma_peak<T><<<grid, kBlock, 0, s>>>(iters, a, b);
  cudaEventRecord(e1, s);
  count_launch(1);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float t = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_error(e, "vgb_measure_fma_peak: launch");
  *ms = t;
  *flops = 2.0 * kChains * (double)iters * (double)grid * kBlock;
  return VGB_OK;
}

}  // namespace
}  // namespace vgb

extern "C" vgb_status vgb_measure_fma_peak(int32_t fp32, int32_t iters, void *stream,
                                           double *flops, float *ms) {
  if (iters <= 0 || !flops || !ms)
    return vgb::set_error(VGB_EINVAL, "vgb_measure_fma_peak: iters must be > 0, outputs non-NULL");
  cudaStream_t s = (cudaStream_t)stream;
  return fp32 ? vgb::run_peak<float>(iters, s, flops, ms)
              : vgb::run_peak<double>(iters, s, flops, ms);
}

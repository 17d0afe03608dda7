// sapb_peak.cu -- a probe of the FP64 (and FP32) fused multiply-add rate of
// the current GPU, the denominator of the contact solve's FP64-pipe fraction.
//
// Every thread runs eight independent FMA chains (enough instruction-level
// parallelism to keep the pipe busy) over a grid of 2048 threads per SM; the
// rate is 2 * chains * iterations * threads / the launch's duration (CUDA
// events on the caller's stream, after one warm-up launch).
#include <cuda_runtime.h>

#include <cstdint>

#include "sapb_internal.h"

namespace {

__device__ double g_fma_sink;  // written only if a chain lands on an impossible value

template <typename T>
__global__ void __launch_bounds__(256) fma_chains_kernel(int iters, T b, T c) {
  T a0 = T(threadIdx.x) * T(1e-3), a1 = a0 + T(1), a2 = a0 + T(2), a3 = a0 + T(3);
  T a4 = a0 + T(4), a5 = a0 + T(5), a6 = a0 + T(6), a7 = a0 + T(7);
#pragma unroll 4
  for (int i = 0; i < iters; ++i) {
    a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
    a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
  }
  const T s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
  // the chains stay positive (they converge to c / (1 - b) = 0.1): never
  // true, but it keeps them live
  if (s == T(-12345)) g_fma_sink = double(s);
}

template <typename T>
int32_t measure(int32_t iters, double* flops_per_s, cudaStream_t stream) {
  int dev = 0, sms = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (err != cudaSuccess) {
    sapb::set_last_error("fma rate probe: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  const int threads = 256, blocks = sms * 8;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  err = cudaEventCreate(&e0);
  if (err == cudaSuccess) err = cudaEventCreate(&e1);
  float ms = 0.0f;
  if (err == cudaSuccess) {
    fma_chains_kernel<T><<<blocks, threads, 0, stream>>>(iters, T(0.999999), T(1e-7));
    err = cudaEventRecord(e0, stream);
  }
  if (err == cudaSuccess) {
    fma_chains_kernel<T><<<blocks, threads, 0, stream>>>(iters, T(0.999999), T(1e-7));
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) err = cudaEventRecord(e1, stream);
  if (err == cudaSuccess) err = cudaEventSynchronize(e1);
  if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (err != cudaSuccess || ms <= 0.0f) {
    sapb::set_last_error("fma rate probe: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  *flops_per_s = 2.0 * 8.0 * (double)iters * (double)threads * (double)blocks / (ms * 1.0e-3);
  return SAPB_OK;
}

}  // namespace

extern "C" int32_t sapb_measure_fma_rate(int32_t precision, int32_t iters, double* flops_per_s, void* stream) {
  if (!flops_per_s || iters <= 0 || (precision != SAPB_FP64 && precision != SAPB_FP32)) {
    sapb::set_last_error("sapb_measure_fma_rate: invalid argument");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  return precision == SAPB_FP64 ? measure<double>(iters, flops_per_s, s) : measure<float>(iters, flops_per_s, s);
}

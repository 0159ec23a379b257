// Throughput probes for the roofline denominators of the FP32/SFU/FP64-bound kernels:
// independent FFMA chains (FP32 pipe), __sinf chains (SFU/MUFU pipe) and DFMA chains (FP64
// pipe), timed with CUDA events on the context's stream.
#include <cuda_runtime.h>

#include "hgx_internal.cuh"

namespace hgx {

constexpr int PROBE_CHAINS = 8;

__global__ void __launch_bounds__(256) fma_probe_kernel(float* out, int iters, float b, float c) {
  float a[PROBE_CHAINS];
#pragma unroll
  for (int k = 0; k < PROBE_CHAINS; ++k) a[k] = threadIdx.x * 1e-3f + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u)
#pragma unroll
      for (int k = 0; k < PROBE_CHAINS; ++k) a[k] = fmaf(a[k], b, c);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < PROBE_CHAINS; ++k) s += a[k];
  if (s == 12345.678f) out[threadIdx.x] = s;  // keeps the chains live
}

__global__ void __launch_bounds__(256) sfu_probe_kernel(float* out, int iters) {
  float a[PROBE_CHAINS];
#pragma unroll
  for (int k = 0; k < PROBE_CHAINS; ++k) a[k] = threadIdx.x * 1e-3f + 0.1f * k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 8; ++u)
#pragma unroll
      for (int k = 0; k < PROBE_CHAINS; ++k) a[k] = __sinf(a[k]);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < PROBE_CHAINS; ++k) s += a[k];
  if (s == 12345.678f) out[threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) dfma_probe_kernel(double* out, int iters, double b, double c) {
  double a[PROBE_CHAINS];
#pragma unroll
  for (int k = 0; k < PROBE_CHAINS; ++k) a[k] = threadIdx.x * 1e-3 + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u)
#pragma unroll
      for (int k = 0; k < PROBE_CHAINS; ++k) a[k] = fma(a[k], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < PROBE_CHAINS; ++k) s += a[k];
  if (s == 12345.678) out[threadIdx.x] = s;  // keeps the chains live
}

}  // namespace hgx

using namespace hgx;

extern "C" int hgx_measure_peak_fp64(hgx_ctx c, double* fp64_tflops) {
  if (!c || !fp64_tflops) return fail(HGX_ERR_INVALID_ARG, "hgx_measure_peak_fp64: null argument");
  HGX_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  HGX_TRY(c->scratch.reserve(4096));
  double* out = reinterpret_cast<double*>(c->scratch.p);
  cudaEvent_t e0, e1;
  HGX_CUDA(cudaEventCreate(&e0));
  HGX_CUDA(cudaEventCreate(&e1));
  const int blocks = c->sm_count * 8, threads = 256, iters = 1024;
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    float ms = 0.f;
    cudaEventRecord(e0, st);
    dfma_probe_kernel<<<blocks, threads, 0, st>>>(out, iters, 0.999, 1e-4);
    cudaEventRecord(e1, st);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return cuda_fail(e, "hgx_measure_peak_fp64");
    }
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  HGX_CUDA(cudaGetLastError());
  *fp64_tflops = (double)blocks * threads * iters * 16.0 * PROBE_CHAINS * 2.0 / (best * 1e-3) / 1e12;
  return HGX_OK;
}

extern "C" int hgx_measure_peaks(hgx_ctx c, int sustained_ms, double* fp32_tflops,
                                 double* sfu_gops) {
  if (!c) return fail(HGX_ERR_INVALID_ARG, "hgx_measure_peaks: ctx is NULL");
  HGX_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  HGX_TRY(c->scratch.reserve(4096));
  float* out = reinterpret_cast<float*>(c->scratch.p);
  cudaEvent_t e0, e1;
  HGX_CUDA(cudaEventCreate(&e0));
  HGX_CUDA(cudaEventCreate(&e1));
  const int blocks = c->sm_count * 8, threads = 256;
  float best_fma = 1e30f, best_sfu = 1e30f;
  const int fma_iters = 4096, sfu_iters = 512;
  // sustained mode: keep the FP32 pipe busy for about sustained_ms first, so the clocks
  // settle where a long kernel runs them (power cap), then time as below
  if (sustained_ms > 0) {
    float ms = 0.f, total = 0.f;
    while (total < (float)sustained_ms) {
      cudaEventRecord(e0, st);
      for (int k = 0; k < 16; ++k) fma_probe_kernel<<<blocks, threads, 0, st>>>(out, fma_iters, 0.999f, 1e-4f);
      cudaEventRecord(e1, st);
      HGX_CUDA(cudaEventSynchronize(e1));
      cudaEventElapsedTime(&ms, e0, e1);
      total += ms;
    }
  }
  for (int rep = 0; rep < 4; ++rep) {
    float ms = 0.f;
    cudaEventRecord(e0, st);
    fma_probe_kernel<<<blocks, threads, 0, st>>>(out, fma_iters, 0.999f, 1e-4f);
    cudaEventRecord(e1, st);
    HGX_CUDA(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best_fma) best_fma = ms;
    cudaEventRecord(e0, st);
    sfu_probe_kernel<<<blocks, threads, 0, st>>>(out, sfu_iters);
    cudaEventRecord(e1, st);
    HGX_CUDA(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best_sfu) best_sfu = ms;
  }
  HGX_CUDA(cudaGetLastError());
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  double n = (double)blocks * threads;
  if (fp32_tflops) *fp32_tflops = n * fma_iters * 16.0 * PROBE_CHAINS * 2.0 / (best_fma * 1e-3) / 1e12;
  if (sfu_gops) *sfu_gops = n * sfu_iters * 8.0 * PROBE_CHAINS / (best_sfu * 1e-3) / 1e9;
  return HGX_OK;
}

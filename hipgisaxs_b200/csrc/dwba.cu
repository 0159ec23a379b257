// The four-term DWBA combination (src/sim/hipgisaxs_main.cpp:1086-1100), its SAXS branch
// (:1102-1105), and the distance measures of the fitting front end
// (include/analyzer/distance_functions.hpp:89-143) with a deterministic FP64 reduction.
#include <cuda_runtime.h>

#include "cplx.cuh"
#include "hgx_internal.cuh"

namespace hgx {

template <typename FF>
__device__ __forceinline__ zd load_c(const void* p, long i);
template <>
__device__ __forceinline__ zd load_c<double2>(const void* p, long i) {
  return zd(reinterpret_cast<const double2*>(p)[i]);
}
template <>
__device__ __forceinline__ zd load_c<float2>(const void* p, long i) {
  float2 v = reinterpret_cast<const float2*>(p)[i];
  return zd((double)v.x, (double)v.y);
}

// I[i] += |w * sum_k fc_k sf_k ff_k|^2 ; sf may be NULL (= 1); fc NULL selects SAXS
// (I[i] = |w sf ff|^2 over one block).
template <typename FF>
__global__ void dwba_combine_kernel(long n, const double2* __restrict__ fc,
                                    const double2* __restrict__ sf, const void* __restrict__ ff,
                                    double w, double* __restrict__ inten) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (fc) {
    zd t(0, 0);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      long j = k * n + i;
      zd s = sf ? zd(sf[j]) : zd(1.0, 0.0);
      t += zd(fc[j]) * s * load_c<FF>(ff, j);
    }
    t = w * t;
    inten[i] += t.x * t.x + t.y * t.y;
  } else {
    zd s = sf ? zd(sf[i]) : zd(1.0, 0.0);
    zd t = (w * s) * load_c<FF>(ff, i);
    inten[i] = t.x * t.x + t.y * t.y;
  }
}

// ------------------------------------------------------------- reductions ----
constexpr int RED_BLOCKS = 1184;  // fixed, so the summation order never changes
constexpr int RED_THREADS = 256;

enum DistKind { DIST_ABS_DIFF_SQUARE = 0, DIST_CHI2 = 1 };

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double s[RED_THREADS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < RED_THREADS / 32 ? s[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  }
  return t;  // valid in thread 0
}

__global__ void __launch_bounds__(RED_THREADS)
distance_partial_kernel(int kind, long n, const double* __restrict__ ref,
                        const double* __restrict__ data, const unsigned* __restrict__ mask,
                        double scale, double* __restrict__ partial) {
  double acc = 0.0;
  for (long i = (long)blockIdx.x * RED_THREADS + threadIdx.x; i < n;
       i += (long)RED_BLOCKS * RED_THREADS) {
    double m = mask ? (double)mask[i] : 1.0;
    if (kind == DIST_ABS_DIFF_SQUARE) {
      double t = m * fabs(ref[i] - data[i]);
      acc += t * t;
    } else {  // Poisson chi^2: data = model, ref = counts
      if (m != 0.0) {
        double d = scale * data[i] - ref[i];
        double cw = ref[i] > 1.0 ? ref[i] : 1.0;
        acc += d * d / cw;
      }
    }
  }
  double s = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void __launch_bounds__(RED_THREADS) final_sum_kernel(const double* __restrict__ partial,
                                                               int m, double* __restrict__ out) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < m; i += RED_THREADS) acc += partial[i];
  double s = block_sum(acc);
  if (threadIdx.x == 0) *out = s;
}

__global__ void residual_kernel(long n, const double* __restrict__ ref,
                                const double* __restrict__ data, const unsigned* __restrict__ mask,
                                double* __restrict__ out) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (mask ? (double)mask[i] : 1.0) * (ref[i] - data[i]);
}

// Deterministic FP64 sum of a distance over n pixels into `result_dev` (device).
int distance_device(hgx_ctx c, int kind, long n, const double* ref, const double* data,
                    const unsigned* mask, double scale, double* result_dev) {
  HGX_TRY(c->scratch.reserve(sizeof(double) * RED_BLOCKS));
  double* partial = reinterpret_cast<double*>(c->scratch.p);
  distance_partial_kernel<<<RED_BLOCKS, RED_THREADS, 0, c->stream>>>(kind, n, ref, data, mask, scale,
                                                                     partial);
  final_sum_kernel<<<1, RED_THREADS, 0, c->stream>>>(partial, RED_BLOCKS, result_dev);
  HGX_CUDA(cudaGetLastError());
  return HGX_OK;
}

static int distance_entry(hgx_ctx c, int kind, long n, const double* ref, const double* data,
                          const unsigned* mask, double scale, double* out) {
  if (!c || !ref || !data || !out) return fail(HGX_ERR_INVALID_ARG, "distance: null argument");
  if (n < 1) return fail(HGX_ERR_INVALID_ARG, "distance: empty input");
  HGX_CUDA(cudaSetDevice(c->device));
  DevBuf br, bd, bm;
  const void *dr, *dd, *dm = nullptr;
  HGX_TRY(stage_in(c, ref, sizeof(double) * n, br, &dr));
  HGX_TRY(stage_in(c, data, sizeof(double) * n, bd, &dd));
  HGX_TRY(stage_in(c, mask, sizeof(unsigned) * n, bm, &dm));
  // a host result goes through the context's scratch, after the reduction's partial sums
  HGX_TRY(c->scratch.reserve(sizeof(double) * (RED_BLOCKS + 1)));
  void* dout = is_device_ptr(out) ? (void*)out : (void*)(reinterpret_cast<double*>(c->scratch.p) + RED_BLOCKS);
  HGX_TRY(distance_device(c, kind, n, (const double*)dr, (const double*)dd, (const unsigned*)dm,
                          scale, (double*)dout));
  HGX_TRY(finish_out(c, out, sizeof(double), dout));
  return br.p || bd.p || bm.p ? hgx_synchronize(c) : HGX_OK;
}

}  // namespace hgx

using namespace hgx;

extern "C" {

int hgx_dwba_combine(hgx_ctx c, long n, const double* fc, const double* sf, const void* ff,
                     int ff_type, double weight, double* intensity) {
  if (!c || !ff || !intensity || n < 1)
    return fail(HGX_ERR_INVALID_ARG, "hgx_dwba_combine: null argument or empty input");
  if (ff_type != HGX_C128 && ff_type != HGX_C64)
    return fail(HGX_ERR_INVALID_ARG, "hgx_dwba_combine: unknown ff type");
  HGX_CUDA(cudaSetDevice(c->device));
  const long nb = fc ? 4 * n : n;
  const size_t fsz = ff_type == HGX_C64 ? sizeof(float2) : sizeof(double2);
  DevBuf bfc, bsf, bff, bI;
  const void *dfc = nullptr, *dsf = nullptr, *dff = nullptr;
  HGX_TRY(stage_in(c, fc, sizeof(double2) * nb, bfc, &dfc));
  HGX_TRY(stage_in(c, sf, sizeof(double2) * nb, bsf, &dsf));
  HGX_TRY(stage_in(c, ff, fsz * nb, bff, &dff));
  void* dI = nullptr;
  HGX_TRY(stage_out(c, intensity, sizeof(double) * n, bI, &dI));
  if (dI != intensity)  // the DWBA branch accumulates into the caller's values
    HGX_CUDA(cudaMemcpyAsync(dI, intensity, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  dim3 grid((unsigned)((n + 255) / 256));
  if (ff_type == HGX_C64)
    dwba_combine_kernel<float2><<<grid, 256, 0, c->stream>>>(n, (const double2*)dfc, (const double2*)dsf,
                                                             dff, weight, (double*)dI);
  else
    dwba_combine_kernel<double2><<<grid, 256, 0, c->stream>>>(n, (const double2*)dfc, (const double2*)dsf,
                                                              dff, weight, (double*)dI);
  HGX_CUDA(cudaGetLastError());
  HGX_TRY(finish_out(c, intensity, sizeof(double) * n, dI));
  return (bfc.p || bsf.p || bff.p) ? hgx_synchronize(c) : HGX_OK;
}

int hgx_abs_diff_square(hgx_ctx c, long n, const double* ref, const double* data,
                        const unsigned* mask, double* out) {
  if (!mask) return fail(HGX_ERR_INVALID_ARG, "hgx_abs_diff_square: mask is required (as in the reference)");
  return distance_entry(c, DIST_ABS_DIFF_SQUARE, n, ref, data, mask, 1.0, out);
}

int hgx_chi2(hgx_ctx c, long n, const double* model, const double* counts, const unsigned* mask,
             double scale, double* out) {
  return distance_entry(c, DIST_CHI2, n, counts, model, mask, scale, out);
}

int hgx_residual_vector(hgx_ctx c, long n, const double* ref, const double* data,
                        const unsigned* mask, double* out) {
  if (!c || !ref || !data || !out || n < 1)
    return fail(HGX_ERR_INVALID_ARG, "hgx_residual_vector: null argument or empty input");
  HGX_CUDA(cudaSetDevice(c->device));
  DevBuf br, bd, bm, bo;
  const void *dr, *dd, *dm = nullptr;
  HGX_TRY(stage_in(c, ref, sizeof(double) * n, br, &dr));
  HGX_TRY(stage_in(c, data, sizeof(double) * n, bd, &dd));
  HGX_TRY(stage_in(c, mask, sizeof(unsigned) * n, bm, &dm));
  void* dout = nullptr;
  HGX_TRY(stage_out(c, out, sizeof(double) * n, bo, &dout));
  residual_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
      n, (const double*)dr, (const double*)dd, (const unsigned*)dm, (double*)dout);
  HGX_CUDA(cudaGetLastError());
  HGX_TRY(finish_out(c, out, sizeof(double) * n, dout));
  return (br.p || bd.p || bm.p) ? hgx_synchronize(c) : HGX_OK;
}

}  // extern "C"

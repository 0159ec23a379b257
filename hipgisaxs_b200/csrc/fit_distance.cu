// The distance measures of the reference's HiG-driven fitter (the metrics its fitting block
// names; src/analyzer/hipgisaxs_fit_main.cpp:82-104), from include/analyzer/distance_functions.hpp:
//   SqrtUnitVectorNormL2DistanceSquare      (:423-456)   sqrt_unit_l2
//   SqrtCNormL2DistanceSquare               (:460-499)   sqrt_c_l2
//   CbrtUnitVectorNormL2DistanceSquare      (:543-575)   cbrt_unit_l2
//   CbrtCNormL2DistanceSquare               (:579-616)   cbrt_c_l2
//   SqrtUnitVectorNormL2DistanceSquareResidualVector (:769-801)   sqrt_unit_l2_residual
//   SqrtCNormL2DistanceSquareResidualVector (:807-844)   sqrt_c_l2_residual
//   SqrtUnitVectorNormL1Distance            (:387-419)   sqrt_unit_l1
//   CbrtUnitVectorNormL1Distance            (:507-539)   cbrt_unit_l1
// Each transforms both images (square or cube root), normalises them (by their masked L1/L2
// norms, or the model by c = <d, r> / |d|^2) and sums the masked squared (or absolute)
// differences; the residual forms return the per-pixel terms.  The NaN and non-finite guards
// are the reference's, metric by metric.  FP64; the sums run in a fixed order (a fixed grid
// of blocks, then one block), so a result does not change from run to run.
#include <cuda_runtime.h>
#include <math.h>

#include "hgx_internal.cuh"

namespace hgx {

namespace {

constexpr int FD_BLOCKS = 1184;  // 8 x 148 SMs
constexpr int FD_THREADS = 256;

enum Metric {
  M_SQRT_UNIT_L2 = 0, M_SQRT_C_L2 = 1, M_CBRT_UNIT_L2 = 2, M_CBRT_C_L2 = 3,
  M_SQRT_UNIT_L2_RES = 4, M_SQRT_C_L2_RES = 5, M_SQRT_UNIT_L1 = 6, M_CBRT_UNIT_L1 = 7
};

__device__ __forceinline__ bool is_cbrt(int m) { return m == M_CBRT_UNIT_L2 || m == M_CBRT_C_L2 || m == M_CBRT_UNIT_L1; }
__device__ __forceinline__ bool is_l1(int m) { return m == M_SQRT_UNIT_L1 || m == M_CBRT_UNIT_L1; }
__device__ __forceinline__ double transform(int m, double x) { return is_cbrt(m) ? cbrt(x) : sqrt(x); }

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double s[FD_THREADS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < FD_THREADS / 32 ? s[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  }
  __syncthreads();  // s is reused by the next call
  return t;         // valid in thread 0
}

// pass 1: the norms of the transformed images and their dot product, per block
// (norm_l1 / norm_l2 / vec_dot of DistanceMeasure, distance_functions.hpp:31-55)
__global__ void __launch_bounds__(FD_THREADS) fit_norms_kernel(int metric, long n, const double* __restrict__ ref,
                                                               const double* __restrict__ dat,
                                                               const unsigned* __restrict__ mask,
                                                               double* __restrict__ part) {
  double a = 0.0, b = 0.0, c = 0.0;
  for (long i = (long)blockIdx.x * FD_THREADS + threadIdx.x; i < n; i += (long)FD_BLOCKS * FD_THREADS) {
    const double m = mask ? (double)mask[i] : 1.0;
    const double tr = transform(metric, ref[i]), td = transform(metric, dat[i]);
    if (is_l1(metric)) {
      a += m * fabs(tr);
      b += m * fabs(td);
    } else {
      const double rr = tr * tr, dd = td * td, rd = fabs(td * tr);
      a += m * (isnan(rr) ? 0 : rr);
      b += m * (isnan(dd) ? 0 : dd);
      c += m * (isnan(rd) ? 0 : rd);
    }
  }
  a = block_sum(a);
  b = block_sum(b);
  c = block_sum(c);
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = a;
    part[3 * blockIdx.x + 1] = b;
    part[3 * blockIdx.x + 2] = c;
  }
}

__global__ void __launch_bounds__(FD_THREADS) fit_sums_kernel(const double* __restrict__ part, int nb, int stride,
                                                              int k, double* __restrict__ out) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < nb; i += FD_THREADS) acc += part[stride * i + k];
  acc = block_sum(acc);
  if (threadIdx.x == 0) out[k] = acc;
}

struct Norms {
  double ref_norm, dat_norm, c;
};

// the per-pixel term of each measure
__device__ __forceinline__ double fit_term(int metric, double m, double r, double d, const Norms& nm) {
  const double tr = transform(metric, r), td = transform(metric, d);
  switch (metric) {
    case M_SQRT_UNIT_L2: {
      const double nd = td / nm.dat_norm, nr = tr / nm.ref_norm;
      double t = m * fabs(nr - nd);
      t = isfinite(t) ? t : 0.0;
      return t * t;
    }
    case M_SQRT_C_L2: {
      const double nd = nm.c * td, nr = tr;
      double t = m * fabs(nr - nd);
      t = isfinite(t) ? t : 0.0;
      return t * t;
    }
    case M_CBRT_UNIT_L2: {
      const double nd = td / nm.dat_norm, nr = tr / nm.ref_norm;
      const double t = m * (nd - nr);
      return t * t;
    }
    case M_CBRT_C_L2: {
      const double nd = nm.c * td, nr = tr;
      const double t = m * fabs(nr - nd);
      return t * t;
    }
    case M_SQRT_UNIT_L2_RES: {
      const double nd = td / nm.dat_norm, nr = tr / nm.ref_norm;
      const double t = m * fabs(nd - nr);
      return t * t;
    }
    case M_SQRT_C_L2_RES: {
      const double nd = nm.c * td, nr = tr;
      const double t = m * fabs(nr - nd);
      return t * t;
    }
    default: {  // the L1 forms
      const double nd = td / nm.dat_norm, nr = tr / nm.ref_norm;
      return m * fabs(nd - nr);
    }
  }
}

__global__ void __launch_bounds__(FD_THREADS) fit_terms_kernel(int metric, long n, const double* __restrict__ ref,
                                                               const double* __restrict__ dat,
                                                               const unsigned* __restrict__ mask, Norms nm,
                                                               double* __restrict__ part,
                                                               double* __restrict__ residual) {
  double acc = 0.0;
  for (long i = (long)blockIdx.x * FD_THREADS + threadIdx.x; i < n; i += (long)FD_BLOCKS * FD_THREADS) {
    const double t = fit_term(metric, mask ? (double)mask[i] : 1.0, ref[i], dat[i], nm);
    if (residual) residual[i] = t;
    else acc += t;
  }
  if (!residual) {
    acc = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
  }
}

// A population of images (candidate = blockIdx.y, images npop x n): the same passes as one
// distance, each candidate's partial sums in its own slice, the norms formed on the device
// from the pass-1 sums exactly as the host forms them for one distance.
__global__ void __launch_bounds__(FD_THREADS) fit_norms_pop_kernel(int metric, long n, const double* __restrict__ ref,
                                                                   const double* __restrict__ imgs,
                                                                   const unsigned* __restrict__ mask,
                                                                   double* __restrict__ part) {
  const double* dat = imgs + (long)blockIdx.y * n;
  double* pp = part + (long)blockIdx.y * 3 * FD_BLOCKS;
  double a = 0.0, b = 0.0, c = 0.0;
  for (long i = (long)blockIdx.x * FD_THREADS + threadIdx.x; i < n; i += (long)FD_BLOCKS * FD_THREADS) {
    const double m = mask ? (double)mask[i] : 1.0;
    const double tr = transform(metric, ref[i]), td = transform(metric, dat[i]);
    if (is_l1(metric)) {
      a += m * fabs(tr);
      b += m * fabs(td);
    } else {
      const double rr = tr * tr, dd = td * td, rd = fabs(td * tr);
      a += m * (isnan(rr) ? 0 : rr);
      b += m * (isnan(dd) ? 0 : dd);
      c += m * (isnan(rd) ? 0 : rd);
    }
  }
  a = block_sum(a);
  b = block_sum(b);
  c = block_sum(c);
  if (threadIdx.x == 0) {
    pp[3 * blockIdx.x] = a;
    pp[3 * blockIdx.x + 1] = b;
    pp[3 * blockIdx.x + 2] = c;
  }
}

// one block per candidate: the three pass-1 sums (each in the order of fit_sums_kernel)
__global__ void __launch_bounds__(FD_THREADS) fit_sums3_pop_kernel(const double* __restrict__ part,
                                                                   double* __restrict__ sums) {
  const double* pp = part + (long)blockIdx.x * 3 * FD_BLOCKS;
  for (int k = 0; k < 3; ++k) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < FD_BLOCKS; i += FD_THREADS) acc += pp[3 * i + k];
    acc = block_sum(acc);
    if (threadIdx.x == 0) sums[4 * blockIdx.x + k] = acc;
  }
}

__global__ void __launch_bounds__(FD_THREADS) fit_terms_pop_kernel(int metric, long n, const double* __restrict__ ref,
                                                                   const double* __restrict__ imgs,
                                                                   const unsigned* __restrict__ mask,
                                                                   const double* __restrict__ sums,
                                                                   double* __restrict__ part) {
  const double* h = sums + 4 * (long)blockIdx.y;
  Norms nm;
  const bool l1 = is_l1(metric);
  nm.ref_norm = l1 ? h[0] : sqrt(h[0]);
  nm.dat_norm = l1 ? h[1] : sqrt(h[1]);
  nm.c = h[2] / (nm.dat_norm * nm.dat_norm);
  const double* dat = imgs + (long)blockIdx.y * n;
  double acc = 0.0;
  for (long i = (long)blockIdx.x * FD_THREADS + threadIdx.x; i < n; i += (long)FD_BLOCKS * FD_THREADS)
    acc += fit_term(metric, mask ? (double)mask[i] : 1.0, ref[i], dat[i], nm);
  acc = block_sum(acc);
  if (threadIdx.x == 0) part[(long)blockIdx.y * FD_BLOCKS + blockIdx.x] = acc;
}

__global__ void __launch_bounds__(FD_THREADS) fit_final_pop_kernel(const double* __restrict__ part,
                                                                   double* __restrict__ out) {
  const double* pp = part + (long)blockIdx.x * FD_BLOCKS;
  double acc = 0.0;
  for (int i = threadIdx.x; i < FD_BLOCKS; i += FD_THREADS) acc += pp[i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) out[blockIdx.x] = acc;
}

// d(distance)/d(data) of the scalar measures.  With t = T(data) (square or cube root),
// r = T(ref), masks m in {0, 1}:
//   unit L2:  sum m (t/N - r/R)^2, N = |t|_m:   (2m/N) ((t/N - r/R) - (t/N) K),
//             K = sum m (t/N - r/R) (t/N)
//   c L2:     sum m (r - c t)^2, c = <t, r>_m / |t|_m^2 (the least-squares scale, so its own
//             change drops out):   -2 m c (r - c t)
//   unit L1:  sum m |t/N - r/R|, N = sum m |t|:   (m/N) (sgn(t/N - r/R) - K),
//             K = sum m sgn(t/N - r/R) (t/N)
// each times T'(data); 0 where data <= 0 (the root's derivative is unbounded there).
__global__ void __launch_bounds__(FD_THREADS) fit_kterm_kernel(int metric, long n, const double* __restrict__ ref,
                                                               const double* __restrict__ dat,
                                                               const unsigned* __restrict__ mask, Norms nm,
                                                               double* __restrict__ part) {
  double acc = 0.0;
  for (long i = (long)blockIdx.x * FD_THREADS + threadIdx.x; i < n; i += (long)FD_BLOCKS * FD_THREADS) {
    const double m = mask ? (double)mask[i] : 1.0;
    const double nd = transform(metric, dat[i]) / nm.dat_norm, nr = transform(metric, ref[i]) / nm.ref_norm;
    double k = is_l1(metric) ? m * ((nd > nr) - (nd < nr)) * nd : m * (nd - nr) * nd;
    acc += isfinite(k) ? k : 0.0;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(FD_THREADS) fit_lambda_kernel(int metric, long n, const double* __restrict__ ref,
                                                                const double* __restrict__ dat,
                                                                const unsigned* __restrict__ mask, Norms nm,
                                                                const double* __restrict__ K,
                                                                double* __restrict__ lambda) {
  for (long i = (long)blockIdx.x * FD_THREADS + threadIdx.x; i < n; i += (long)FD_BLOCKS * FD_THREADS) {
    const double m = mask ? (double)mask[i] : 1.0;
    const double d = dat[i];
    const double td = transform(metric, d), tr = transform(metric, ref[i]);
    double g;
    if (metric == M_SQRT_C_L2 || metric == M_CBRT_C_L2) {
      g = -2.0 * m * nm.c * (tr - nm.c * td);
    } else {
      const double nd = td / nm.dat_norm, nr = tr / nm.ref_norm;
      if (is_l1(metric)) g = m / nm.dat_norm * ((double)((nd > nr) - (nd < nr)) - K[0]);
      else g = 2.0 * m / nm.dat_norm * ((nd - nr) - nd * K[0]);
    }
    const double dT = is_cbrt(metric) ? 1.0 / (3.0 * td * td) : 0.5 / td;
    const double v = g * dT;
    lambda[i] = (d > 0.0 && isfinite(v)) ? v : 0.0;
  }
}

__global__ void __launch_bounds__(FD_THREADS) dot_partial_kernel(long n, const double* __restrict__ a,
                                                                 const double* __restrict__ b,
                                                                 double* __restrict__ part) {
  double acc = 0.0;
  for (long i = (long)blockIdx.x * FD_THREADS + threadIdx.x; i < n; i += (long)FD_BLOCKS * FD_THREADS)
    acc += a[i] * b[i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

}  // namespace

// The norms of pass 1 (host copies), shared by the distance and its gradient.
static int fit_norms(hgx_ctx c, int metric, long n, const double* dr, const double* dd, const unsigned* dm,
                     Norms* nm) {
  cudaStream_t st = c->stream;
  HGX_TRY(c->scratch.reserve(sizeof(double) * (3 * FD_BLOCKS + 4)));
  double* part = reinterpret_cast<double*>(c->scratch.p);
  double* sums = part + 3 * FD_BLOCKS;
  fit_norms_kernel<<<FD_BLOCKS, FD_THREADS, 0, st>>>(metric, n, dr, dd, dm, part);
  for (int k = 0; k < 3; ++k) fit_sums_kernel<<<1, FD_THREADS, 0, st>>>(part, FD_BLOCKS, 3, k, sums);
  HGX_CUDA(cudaGetLastError());
  double h[3];
  HGX_CUDA(cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, st));
  HGX_CUDA(cudaStreamSynchronize(st));
  const bool l1 = metric == M_SQRT_UNIT_L1 || metric == M_CBRT_UNIT_L1;
  nm->ref_norm = l1 ? h[0] : sqrt(h[0]);
  nm->dat_norm = l1 ? h[1] : sqrt(h[1]);
  nm->c = h[2] / (nm->dat_norm * nm->dat_norm);
  return HGX_OK;
}

// d(distance)/d(data) of a scalar measure (not the residual-vector forms), device arrays.
int fit_distance_gradient(hgx_ctx c, int metric, long n, const double* ref, const double* data,
                          const unsigned* mask, double* lambda) {
  if (metric < 0 || metric > M_CBRT_UNIT_L1 || metric == M_SQRT_UNIT_L2_RES || metric == M_SQRT_C_L2_RES)
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_objective_grad: the gradient is defined for the scalar "
                                     "distance measures (not the residual vectors)");
  Norms nm;
  HGX_TRY(fit_norms(c, metric, n, ref, data, mask, &nm));
  cudaStream_t st = c->stream;
  double* part = reinterpret_cast<double*>(c->scratch.p);
  double* sums = part + 3 * FD_BLOCKS;
  fit_kterm_kernel<<<FD_BLOCKS, FD_THREADS, 0, st>>>(metric, n, ref, data, mask, nm, part);
  fit_sums_kernel<<<1, FD_THREADS, 0, st>>>(part, FD_BLOCKS, 1, 0, sums + 3);
  fit_lambda_kernel<<<FD_BLOCKS, FD_THREADS, 0, st>>>(metric, n, ref, data, mask, nm, sums + 3, lambda);
  HGX_CUDA(cudaGetLastError());
  return HGX_OK;
}

long fit_population_scratch(int npop) { return (long)npop * (4L * FD_BLOCKS + 4); }

int fit_distance_population(cudaStream_t st, int metric, long n, const double* ref, const double* imgs,
                            const unsigned* mask, int npop, double* scratch, double* dist) {
  if (metric < 0 || metric > M_CBRT_UNIT_L1 || metric == M_SQRT_UNIT_L2_RES || metric == M_SQRT_C_L2_RES)
    return fail(HGX_ERR_INVALID_ARG, "fit_distance_population: a scalar distance measure is needed");
  double* part3 = scratch;
  double* part1 = part3 + 3L * FD_BLOCKS * npop;
  double* sums = part1 + (long)FD_BLOCKS * npop;
  fit_norms_pop_kernel<<<dim3(FD_BLOCKS, npop), FD_THREADS, 0, st>>>(metric, n, ref, imgs, mask, part3);
  fit_sums3_pop_kernel<<<npop, FD_THREADS, 0, st>>>(part3, sums);
  fit_terms_pop_kernel<<<dim3(FD_BLOCKS, npop), FD_THREADS, 0, st>>>(metric, n, ref, imgs, mask, sums, part1);
  fit_final_pop_kernel<<<npop, FD_THREADS, 0, st>>>(part1, dist);
  HGX_CUDA(cudaGetLastError());
  return HGX_OK;
}

int device_dot(hgx_ctx c, long n, const double* a, const double* b, double* out) {
  cudaStream_t st = c->stream;
  HGX_TRY(c->scratch.reserve(sizeof(double) * (FD_BLOCKS + 4)));
  double* part = reinterpret_cast<double*>(c->scratch.p);
  dot_partial_kernel<<<FD_BLOCKS, FD_THREADS, 0, st>>>(n, a, b, part);
  fit_sums_kernel<<<1, FD_THREADS, 0, st>>>(part, FD_BLOCKS, 1, 0, part + FD_BLOCKS);
  HGX_CUDA(cudaGetLastError());
  HGX_CUDA(cudaMemcpyAsync(out, part + FD_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost, st));
  HGX_CUDA(cudaStreamSynchronize(st));
  return HGX_OK;
}

}  // namespace hgx

using namespace hgx;

extern "C" {

int hgx_fit_distance(hgx_ctx c, int metric, long n, const double* ref, const double* data,
                     const unsigned* mask, double* out) {
  if (!c || !ref || !data || !out) return fail(HGX_ERR_INVALID_ARG, "hgx_fit_distance: null argument");
  if (n < 1) return fail(HGX_ERR_INVALID_ARG, "hgx_fit_distance: empty input");
  if (metric < 0 || metric > M_CBRT_UNIT_L1) return fail(HGX_ERR_INVALID_ARG, "hgx_fit_distance: unknown metric");
  HGX_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  DevBuf br, bd, bm, bo;
  const void *dr, *dd, *dm = nullptr;
  HGX_TRY(stage_in(c, ref, sizeof(double) * n, br, &dr));
  HGX_TRY(stage_in(c, data, sizeof(double) * n, bd, &dd));
  HGX_TRY(stage_in(c, mask, sizeof(unsigned) * n, bm, &dm));
  // scratch: 3 partials per block, then 3 sums
  HGX_TRY(c->scratch.reserve(sizeof(double) * (3 * FD_BLOCKS + 4)));
  double* part = reinterpret_cast<double*>(c->scratch.p);
  double* sums = part + 3 * FD_BLOCKS;
  fit_norms_kernel<<<FD_BLOCKS, FD_THREADS, 0, st>>>(metric, n, (const double*)dr, (const double*)dd,
                                                    (const unsigned*)dm, part);
  for (int k = 0; k < 3; ++k) fit_sums_kernel<<<1, FD_THREADS, 0, st>>>(part, FD_BLOCKS, 3, k, sums);
  HGX_CUDA(cudaGetLastError());
  double h[3];
  HGX_CUDA(cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, st));
  HGX_CUDA(cudaStreamSynchronize(st));
  Norms nm;
  const bool l1 = metric == M_SQRT_UNIT_L1 || metric == M_CBRT_UNIT_L1;
  nm.ref_norm = l1 ? h[0] : sqrt(h[0]);
  nm.dat_norm = l1 ? h[1] : sqrt(h[1]);
  nm.c = h[2] / (nm.dat_norm * nm.dat_norm);
  const bool residual = metric == M_SQRT_UNIT_L2_RES || metric == M_SQRT_C_L2_RES;
  if (residual) {
    void* dout = nullptr;
    HGX_TRY(stage_out(c, out, sizeof(double) * n, bo, &dout));
    fit_terms_kernel<<<FD_BLOCKS, FD_THREADS, 0, st>>>(metric, n, (const double*)dr, (const double*)dd,
                                                      (const unsigned*)dm, nm, nullptr, (double*)dout);
    HGX_CUDA(cudaGetLastError());
    return finish_out(c, out, sizeof(double) * n, dout);
  }
  fit_terms_kernel<<<FD_BLOCKS, FD_THREADS, 0, st>>>(metric, n, (const double*)dr, (const double*)dd,
                                                    (const unsigned*)dm, nm, part, nullptr);
  fit_sums_kernel<<<1, FD_THREADS, 0, st>>>(part, FD_BLOCKS, 1, 0, sums + 3);
  HGX_CUDA(cudaGetLastError());
  HGX_CUDA(cudaMemcpyAsync(out, sums + 3, sizeof(double), is_device_ptr(out) ? cudaMemcpyDeviceToDevice
                                                                               : cudaMemcpyDeviceToHost, st));
  return hgx_synchronize(c);
}

}  // extern "C"

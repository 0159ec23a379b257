// Post-processing of the detector image, on the device:
//  * Gaussian smearing: Convolutions::convolution_gaussian_2d as HipGISAXS::gaussian_smearing
//    calls it (include/numerics/convolutions.hpp:127-174, src/sim/hipgisaxs_helpers.cpp:25-27):
//    a horizontal then a vertical pass, each output the weighted mean of the window
//    [i - r, i + r) with r = ceil(6 sigma) (the right end excluded) and the weights indexed from
//    the window's start — so at the left and top borders, where the window is clipped, the
//    weights are those of an unclipped window shifted to the border.  Both as the reference.
//  * normalize: HipGISAXS::normalize (src/sim/hipgisaxs_main.cpp:1439-1450), (x - min) /
//    (max - min) over every element except the first, which the reference leaves unscaled.
//  * save: HipGISAXS::save_gisaxs (src/sim/hipgisaxs_main.cpp:2250-2260), the ".out" text
//    image: each value in the default stream format followed by a tab, one row per line.
// FP64, compiled without fused multiply-adds (hipgisaxs_b200/build.py) so that every sum
// rounds as the reference's does; both passes are bound by memory bandwidth.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>

#include <algorithm>
#include <fstream>
#include <vector>

#include "hgx_internal.cuh"

namespace hgx {

constexpr int PP_THREADS = 256;
constexpr int SMEAR_MAX_TAPS = 8193;  // 2 ceil(6 sigma) + 1: sigma up to about 682 pixels

// one pass along rows (dir 0: out[j][i] from in[j][k]) or columns (dir 1: out[j][i] from in[l][i])
template <int DIR>
__global__ void __launch_bounds__(PP_THREADS) smear_pass_kernel(const double* __restrict__ in,
                                                                double* __restrict__ out, int nx,
                                                                int ny, int r,
                                                                const double* __restrict__ gmap) {
  const int i = blockIdx.x * PP_THREADS + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= nx || j >= ny) return;
  double sum = 0.0, norm = 0.0;
  if (DIR == 0) {
    const int b = max(0, i - r), e = min(nx, i + r);
    const double* row = in + (size_t)j * nx;
    for (int k = b; k < e; ++k) {
      sum += row[k] * gmap[k - b];
      norm += gmap[k - b];
    }
  } else {
    const int b = max(0, j - r), e = min(ny, j + r);
    for (int l = b; l < e; ++l) {
      sum += in[(size_t)l * nx + i] * gmap[l - b];
      norm += gmap[l - b];
    }
  }
  out[(size_t)j * nx + i] = norm > DBL_MIN ? sum / norm : 0.0;
}

constexpr int MM_BLOCKS = 1184;  // 8 x 148 SMs, fixed for a deterministic reduction

__global__ void __launch_bounds__(PP_THREADS) minmax_partial_kernel(const double* __restrict__ d,
                                                                    long n, double2* __restrict__ part) {
  __shared__ double smn[PP_THREADS], smx[PP_THREADS];
  double mn = d[0], mx = d[0];
  for (long i = (long)blockIdx.x * PP_THREADS + threadIdx.x; i < n; i += (long)gridDim.x * PP_THREADS) {
    mn = fmin(mn, d[i]);
    mx = fmax(mx, d[i]);
  }
  smn[threadIdx.x] = mn;
  smx[threadIdx.x] = mx;
  __syncthreads();
  for (int s = PP_THREADS / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      smn[threadIdx.x] = fmin(smn[threadIdx.x], smn[threadIdx.x + s]);
      smx[threadIdx.x] = fmax(smx[threadIdx.x], smx[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = make_double2(smn[0], smx[0]);
}

__global__ void normalize_kernel(double* __restrict__ d, long n, double mn, double dd) {
  const long i = (long)blockIdx.x * PP_THREADS + threadIdx.x;
  if (i >= 1 && i < n) d[i] = (d[i] - mn) / dd;
}

}  // namespace hgx

using namespace hgx;

extern "C" {

int hgx_gaussian_smearing(hgx_ctx c, double* image, int ncol, int nrow, double sigma) {
  if (!c || !image) return fail(HGX_ERR_INVALID_ARG, "hgx_gaussian_smearing: null argument");
  if (ncol < 1 || nrow < 1 || nrow > 65535)
    return fail(HGX_ERR_INVALID_ARG, "hgx_gaussian_smearing: image size out of range");
  if (!(sigma > 0.0)) return fail(HGX_ERR_INVALID_ARG, "hgx_gaussian_smearing: sigma must be > 0");
  const int r = (int)ceil(6 * sigma);
  const int gn = 2 * r + 1;
  if (gn > SMEAR_MAX_TAPS)
    return fail(HGX_ERR_INVALID_ARG, "hgx_gaussian_smearing: sigma too large (at most 8193 taps)");
  HGX_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  // the weights, as Convolutions::gaussian computes them (convolutions.hpp:122-124, 133-135)
  std::vector<double> gmap(gn);
  const double pi = 3.141592653589793;  // PI_, include/common/constants.hpp
  for (int i = 0; i < gn; ++i) {
    const int x = i - r;
    gmap[i] = 1.0 / (sigma * sqrt(2 * pi) * exp((x * x) / (2 * sigma * sigma)));
  }
  const size_t bytes = sizeof(double) * (size_t)ncol * nrow;
  DevBuf bg, bimg, bconv;
  HGX_TRY(bg.reserve(sizeof(double) * gn));
  HGX_CUDA(cudaMemcpyAsync(bg.p, gmap.data(), sizeof(double) * gn, cudaMemcpyHostToDevice, st));
  const bool host = !is_device_ptr(image);
  double* dimg = image;
  if (host) {
    HGX_TRY(bimg.reserve(bytes));
    dimg = (double*)bimg.p;
    HGX_CUDA(cudaMemcpyAsync(dimg, image, bytes, cudaMemcpyHostToDevice, st));
  }
  HGX_TRY(bconv.reserve(bytes));
  dim3 grid((ncol + PP_THREADS - 1) / PP_THREADS, nrow);
  smear_pass_kernel<0><<<grid, PP_THREADS, 0, st>>>(dimg, (double*)bconv.p, ncol, nrow, r,
                                                    (const double*)bg.p);
  smear_pass_kernel<1><<<grid, PP_THREADS, 0, st>>>((const double*)bconv.p, dimg, ncol, nrow, r,
                                                    (const double*)bg.p);
  HGX_CUDA(cudaGetLastError());
  if (host) HGX_CUDA(cudaMemcpyAsync(image, dimg, bytes, cudaMemcpyDeviceToHost, st));
  return hgx_synchronize(c);
}

int hgx_normalize(hgx_ctx c, double* data, long n, int* normalized) {
  if (!c || !data || n < 1) return fail(HGX_ERR_INVALID_ARG, "hgx_normalize: null argument or empty input");
  HGX_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  const bool host = !is_device_ptr(data);
  DevBuf bd, bp;
  double* d = data;
  if (host) {
    HGX_TRY(bd.reserve(sizeof(double) * n));
    d = (double*)bd.p;
    HGX_CUDA(cudaMemcpyAsync(d, data, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  }
  const int blocks = (int)std::min<long>(MM_BLOCKS, (n + PP_THREADS - 1) / PP_THREADS);
  HGX_TRY(bp.reserve(sizeof(double2) * blocks));
  minmax_partial_kernel<<<blocks, PP_THREADS, 0, st>>>(d, n, (double2*)bp.p);
  HGX_CUDA(cudaGetLastError());
  std::vector<double2> part(blocks);
  HGX_CUDA(cudaMemcpyAsync(part.data(), bp.p, sizeof(double2) * blocks, cudaMemcpyDeviceToHost, st));
  HGX_CUDA(cudaStreamSynchronize(st));
  double mn = part[0].x, mx = part[0].y;
  for (int b = 1; b < blocks; ++b) {
    mn = std::min(mn, part[b].x);
    mx = std::max(mx, part[b].y);
  }
  const double dd = mx - mn;
  const int ok = dd < 1e-30 ? 0 : 1;  // a flat image is left as it is, as the reference does
  if (ok) {
    normalize_kernel<<<(unsigned)((n + PP_THREADS - 1) / PP_THREADS), PP_THREADS, 0, st>>>(d, n, mn, dd);
    HGX_CUDA(cudaGetLastError());
    if (host) HGX_CUDA(cudaMemcpyAsync(data, d, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  }
  if (normalized) *normalized = ok;
  return hgx_synchronize(c);
}

int hgx_save_gisaxs(hgx_ctx c, const double* image, int nrow, int ncol, const char* path) {
  if (!image || !path || nrow < 1 || ncol < 1)
    return fail(HGX_ERR_INVALID_ARG, "hgx_save_gisaxs: null argument or empty image");
  const size_t n = (size_t)nrow * ncol;
  std::vector<double> h;
  const double* src = image;
  if (is_device_ptr(image)) {
    if (!c) return fail(HGX_ERR_INVALID_ARG, "hgx_save_gisaxs: a device image needs a context");
    HGX_CUDA(cudaSetDevice(c->device));
    h.resize(n);
    HGX_CUDA(cudaMemcpyAsync(h.data(), image, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    HGX_TRY(hgx_synchronize(c));
    src = h.data();
  }
  std::ofstream f(path);
  if (!f.is_open()) return fail(HGX_ERR_INVALID_ARG, std::string("hgx_save_gisaxs: cannot open ") + path);
  for (int z = 0; z < nrow; ++z) {
    for (int y = 0; y < ncol; ++y) f << src[(size_t)ncol * z + y] << "\t";
    f << std::endl;
  }
  if (!f.good()) return fail(HGX_ERR_INVALID_ARG, std::string("hgx_save_gisaxs: write failed: ") + path);
  return HGX_OK;
}

}  // extern "C"

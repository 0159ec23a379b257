// Device-side q-grid: QGrid::create (src/model/qgrid.cpp:30-99) and
// QGrid::create_qz_extended (src/model/qgrid.cpp:102-127), FP64.
//
// Layout as the reference builds it: exit angles alpha_f per row, computed from the
// q-space rows and then reversed so that row 0 is the top of the detector; 2theta per
// column computed with cos(alpha_f) of the FIRST (unreversed) row for every row, as the
// reference does; flattened qx, qy, qz per pixel; the 4 DWBA blocks
// [kzf - kzi, -kzf - kzi, kzf + kzi, -kzf + kzi].  Built without fused multiply-adds (the
// build passes -fmad=false for this file): 2theta = acos(t) with t just below 1 near qy = 0
// turns a one-ulp change of t into up to ~1e-9 relative in qy, so t is rounded as the
// reference rounds it.
#include <cuda_runtime.h>
#include <math.h>

#include "hgx_internal.cuh"

namespace hgx {

struct QgridArgs {
  int ncol, nrow;
  double qmin_y, qmin_z, qmax_y, qmax_z, alpha_i, k0, dn2_re, dn2_im;
};

// alpha_f per row (already reversed) and 2theta per column.
__global__ void qgrid_angles_kernel(QgridArgs a, double* __restrict__ alpha,
                                    double* __restrict__ theta) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double sin_ai = sin(a.alpha_i);
  if (i < a.nrow) {
    double dq = (a.qmax_z - a.qmin_z) / (a.nrow - 1);
    int src = a.nrow - 1 - i;  // std::reverse
    double qpt = a.qmin_z + src * dq;
    alpha[i] = asin(qpt / a.k0 - sin_ai);
  }
  if (i < a.ncol) {
    double al0 = asin(a.qmin_z / a.k0 - sin_ai);  // alpha_[0] before the reversal
    double dq = (a.qmax_y - a.qmin_y) / (a.ncol - 1);
    double qpt = a.qmin_y + i * dq;
    double cos_ai = cos(a.alpha_i), cos_af = cos(al0);
    double kf2 = (qpt / a.k0) * (qpt / a.k0);
    double tmp = (cos_af * cos_af + cos_ai * cos_ai - kf2) / (2 * cos_af * cos_ai);
    if (tmp > 1.0) tmp = 1.0;
    theta[i] = (qpt < 0 ? -1.0 : 1.0) * acos(tmp);
  }
}

__device__ __forceinline__ double2 csqrt_d(double re, double im) {
  // principal square root (branch cut on the negative real axis), as csqrt
  if (re == 0.0 && im == 0.0) return make_double2(0.0, im);
  double m = hypot(re, im);
  double t = sqrt(0.5 * (m + fabs(re)));
  if (re >= 0.0) return make_double2(t, im / (2.0 * t));
  return make_double2(fabs(im) / (2.0 * t), copysign(t, im));
}

// the four DWBA blocks of pixel p (create_qz_extended, src/model/qgrid.cpp:102-127)
__device__ __forceinline__ void qz_extend_point(double qzp, double k0, double sin_ai, double dn2_re,
                                                double dn2_im, long p, long n, double2* __restrict__ qz_ext) {
  double kzi0 = -1 * k0 * sin_ai;
  double2 r = csqrt_d(sin_ai * sin_ai - dn2_re, -dn2_im);
  double2 kzi = make_double2(-k0 * r.x, -k0 * r.y);
  double kzf0 = qzp + kzi0;
  double2 s = csqrt_d(kzf0 * kzf0 - k0 * k0 * dn2_re, -(k0 * k0 * dn2_im));
  double sg = kzf0 < 0 ? -1.0 : 1.0;
  double2 kzf = make_double2(sg * s.x, sg * s.y);
  qz_ext[p] = make_double2(kzf.x - kzi.x, kzf.y - kzi.y);
  qz_ext[n + p] = make_double2(-kzf.x - kzi.x, -kzf.y - kzi.y);
  qz_ext[2 * n + p] = make_double2(kzf.x + kzi.x, kzf.y + kzi.y);
  qz_ext[3 * n + p] = make_double2(-kzf.x + kzi.x, -kzf.y + kzi.y);
}

__global__ void qgrid_pixels_kernel(QgridArgs a, const double* __restrict__ alpha,
                                    const double* __restrict__ theta, double* __restrict__ qx,
                                    double* __restrict__ qy, double* __restrict__ qz,
                                    double2* __restrict__ qz_ext) {
  long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long n = (long)a.nrow * a.ncol;
  if (p >= n) return;
  int i = (int)(p / a.ncol), j = (int)(p - (long)i * a.ncol);
  double tth = theta[j], alf = alpha[i];
  double cos_ai = cos(a.alpha_i), sin_ai = sin(a.alpha_i);
  qx[p] = a.k0 * (cos(alf) * cos(tth) - cos_ai);
  qy[p] = a.k0 * (cos(alf) * sin(tth));
  double qzp = a.k0 * (sin(alf) + sin_ai);
  qz[p] = qzp;
  qz_extend_point(qzp, a.k0, sin_ai, a.dn2_re, a.dn2_im, p, n, qz_ext);
}

// create_qz_extended alone, for another incidence angle over the same detector grid (the
// reference keeps the grid of its first alpha_i and extends qz for each angle of a scan)
__global__ void qgrid_reextend_kernel(const double* __restrict__ qz, long n, double k0, double alpha_i,
                                      double dn2_re, double dn2_im, double2* __restrict__ qz_ext) {
  long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  qz_extend_point(qz[p], k0, sin(alpha_i), dn2_re, dn2_im, p, n, qz_ext);
}

int qgrid_reextend(hgx_qgrid g, double alpha_i, double k0, double dn2_re, double dn2_im) {
  if (!g || !g->qz_det) return fail(HGX_ERR_INVALID_ARG, "qgrid_reextend: not a grid made by hgx_qgrid_create");
  const long n = (long)g->nqy;
  cudaStream_t st = g->ctx->stream;
  qgrid_reextend_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g->qz_det, n, k0, alpha_i, dn2_re, dn2_im,
                                                                     g->qz);
  HGX_CUDA(cudaGetLastError());
  return qgrid_finalize(g);
}

}  // namespace hgx

using namespace hgx;

extern "C" int hgx_qgrid_create(hgx_ctx c, int ncol, int nrow, double qmin_y, double qmin_z,
                                double qmax_y, double qmax_z, double alpha_i, double k0,
                                double dn2_re, double dn2_im, hgx_qgrid* out) {
  if (!c || !out) return fail(HGX_ERR_INVALID_ARG, "hgx_qgrid_create: null argument");
  *out = nullptr;
  if (ncol < 2 || nrow < 2)
    return fail(HGX_ERR_INVALID_ARG, "hgx_qgrid_create: need at least 2 x 2 pixels");
  if (!(k0 > 0)) return fail(HGX_ERR_INVALID_ARG, "hgx_qgrid_create: k0 must be > 0");
  HGX_CUDA(cudaSetDevice(c->device));
  hgx_qgrid g = new (std::nothrow) hgx_qgrid_s();
  if (!g) return fail(HGX_ERR_NO_MEMORY, "hgx_qgrid_create: host allocation");
  g->ctx = c;
  const long n = (long)ncol * nrow;
  if (n > (long)(1 << 30)) {
    delete g;
    return fail(HGX_ERR_INVALID_ARG, "hgx_qgrid_create: grid too large");
  }
  g->nqy = (int)n;
  g->nqz = (int)(4 * n);
  g->nk = 4;
  g->ncol = ncol;
  g->nrow = nrow;
  double* theta = nullptr;
  cudaError_t e = cudaSuccess;
  if ((e = cudaMalloc(&g->qx, sizeof(double) * n)) != cudaSuccess ||
      (e = cudaMalloc(&g->qy, sizeof(double) * n)) != cudaSuccess ||
      (e = cudaMalloc(&g->qz_det, sizeof(double) * n)) != cudaSuccess ||
      (e = cudaMalloc(&g->qz, sizeof(double2) * 4 * n)) != cudaSuccess ||
      (e = cudaMalloc(&g->alpha, sizeof(double) * nrow)) != cudaSuccess ||
      (e = cudaMalloc(&theta, sizeof(double) * ncol)) != cudaSuccess) {
    hgx_qgrid_destroy(g);
    return cuda_fail(e, "hgx_qgrid_create: cudaMalloc");
  }
  QgridArgs a{ncol, nrow, qmin_y, qmin_z, qmax_y, qmax_z, alpha_i, k0, dn2_re, dn2_im};
  cudaStream_t st = c->stream;
  int m = ncol > nrow ? ncol : nrow;
  qgrid_angles_kernel<<<(m + 127) / 128, 128, 0, st>>>(a, g->alpha, theta);
  qgrid_pixels_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, g->alpha, theta, g->qx, g->qy,
                                                                  g->qz_det, g->qz);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(theta);
  if (e != cudaSuccess) {
    hgx_qgrid_destroy(g);
    return cuda_fail(e, "hgx_qgrid_create: kernels");
  }
  int s = qgrid_finalize(g);
  if (s != HGX_OK) {
    hgx_qgrid_destroy(g);
    return s;
  }
  *out = g;
  return HGX_OK;
}

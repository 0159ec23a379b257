// Paracrystal and Percus-Yevick structure factors (StructureFactor::paracrystal1d,
// paracrystal2d_cubic, paracrystal2d_hex, PYFcn and percus_yevik, src/sf/liquid.cpp:29-165),
// selected as compute_structure_factor selects them (src/sf/sf.cpp:116-161).  FP64, one thread
// per q-point (q-point i uses qx/qy[i % nqy]), the reference's arithmetic including its
// quirks: the 1-D paracrystal uses qy only; the 2-D cubic one uses |q_par| on both axes; the
// 3-D Percus-Yevick result is a fourth root (sqrt of 1/sqrt(...)) while its |q| < 1e-6 value
// alpha/3 + beta/4 + gamma is taken without a root.
//
// Compiled without fused multiply-adds (-fmad=false, hipgisaxs_b200/build.py): PYFcn's terms
// cancel at small q d, and the kernels are bound by memory, not arithmetic.
#include <cuda_runtime.h>
#include <math.h>

#include "cplx.cuh"
#include "hgx_internal.cuh"

namespace hgx {

constexpr int LQ_THREADS = 256;

struct ParaArgs {
  int dims, lattice;
  double dx, dy, sx, sy;
  double exp_v1x, exp_v1y;
  const double* qx;
  const double* qy;
  int nqy;
  long nqz;
  void* out;
};

template <typename OUT>
__device__ __forceinline__ void store_real(OUT* out, long i, double v);
template <>
__device__ __forceinline__ void store_real<float2>(float2* out, long i, double v) {
  out[i] = make_float2((float)v, 0.f);
}
template <>
__device__ __forceinline__ void store_real<double2>(double2* out, long i, double v) {
  out[i] = make_double2(v, 0.0);
}

template <typename OUT>
__global__ void __launch_bounds__(LQ_THREADS) paracrystal_kernel(ParaArgs a) {
  const long i = (long)blockIdx.x * LQ_THREADS + threadIdx.x;
  if (i >= a.nqz) return;
  const int j = (int)(i % a.nqy);
  double v;
  if (a.dims == 1) {
    const double q = a.qy[j];
    const double qysy = a.sy * q;
    const double exp_v2 = exp(-1.0 * qysy * qysy);
    const double exp_v3 = exp(-0.5 * qysy * qysy);
    const double tmp = (1. - exp_v2 * a.exp_v1y) /
                       (1. - 2. * exp_v3 * a.exp_v1y * cos(q * a.dy) + exp_v2 * a.exp_v1y);
    v = sqrt(tmp);
  } else {
    const double x = a.qx[j], y = a.qy[j];
    const double qpar = sqrt(x * x + y * y);
    double s1, s2;
    if (a.lattice == 3) {  // cubic
      const double cos_vx = cos(qpar * a.dx);
      const double cos_vy = cos(qpar * a.dy);
      const double qxsx = qpar * a.sx;
      const double exp_v2x = exp(-1. * qxsx * qxsx);
      const double exp_v3x = exp(-0.5 * qxsx * qxsx);
      const double qysy = qpar * a.sy;
      const double exp_v2y = exp(-1. * qysy * qysy);
      const double exp_v3y = exp(-0.5 * qysy * qysy);
      s1 = (1. - exp_v2x * a.exp_v1x) / (1. - 2. * exp_v3x * a.exp_v1x * cos_vx + exp_v2x * a.exp_v1x);
      s2 = (1. - exp_v2y * a.exp_v1y) / (1. - 2. * exp_v3y * a.exp_v1y * cos_vy + exp_v2y * a.exp_v1y);
    } else {  // hex
      const double C1 = 0.5 * sqrt(3.);
      const double qpsx = qpar * a.sx;
      const double qpsy = qpar * a.sy;
      const double phi_x = cos(C1 * x * a.dx + 0.5 * y * a.dy);
      const double phi_y = cos(y * a.dy);
      const double exp_v2x = exp(-1. * qpsx * qpsx);
      const double exp_v2y = exp(-1. * qpsy * qpsy);
      const double exp_v3x = exp(-0.5 * qpsx * qpsx);
      const double exp_v3y = exp(-0.5 * qpsy * qpsy);
      s1 = (1. - exp_v2x * a.exp_v1x) / (1. - 2. * exp_v3x * a.exp_v1x * phi_x + exp_v2x * a.exp_v1x);
      s2 = (1. - exp_v2y * a.exp_v1y) / (1. - 2. * exp_v3y * a.exp_v1y * phi_y + exp_v2y * a.exp_v1y);
    }
    v = sqrt(fabs(s1 * s2));
  }
  store_real<OUT>(reinterpret_cast<OUT*>(a.out), i, v);
}

struct PYArgs {
  int dims;
  double dia, volf, alpha, beta, gamma;
  const double* qx;
  const double* qy;
  const double2* qz;
  int nqy;
  long nqz;
  void* out;
};

// StructureFactor::PYFcn (src/sf/liquid.cpp:112-125)
__device__ __forceinline__ double py_fcn(double alpha, double beta, double gamma, double x) {
  double sinx, cosx;
  sincos(x, &sinx, &cosx);
  const double x2 = x * x;
  const double x3 = x2 * x;
  const double x4 = x3 * x;
  const double x5 = x4 * x;
  const double t1 = alpha * (sinx - x * cosx) / x2;
  const double t2 = beta * (2 * x * sinx + (2 - x2) * cosx - 2) / x3;
  const double t3 = gamma * (-x4 * cosx + 4 * ((3 * x2 - 6) * cosx + (x3 - 6 * x) * sinx + 6)) / x5;
  return (t1 + t2 + t3);
}

template <typename OUT>
__global__ void __launch_bounds__(LQ_THREADS) percus_yevick_kernel(PYArgs a) {
  const long i = (long)blockIdx.x * LQ_THREADS + threadIdx.x;
  if (i >= a.nqz) return;
  const int j = (int)(i % a.nqy);
  const double x0 = a.qx[j], y0 = a.qy[j];
  double qval;
  if (a.dims == 2) {
    qval = sqrt(x0 * x0 + y0 * y0);
  } else {
    const double2 z = a.qz[i];
    qval = sqrt(x0 * x0 + y0 * y0 + (z.x * z.x + z.y * z.y));
  }
  double v;
  if (qval < 1.0E-06) {
    v = a.alpha / 3. + a.beta / 4. + a.gamma;
  } else {
    const double x = qval * a.dia;
    const double p = py_fcn(a.alpha, a.beta, a.gamma, x);
    const double t = a.dims == 2 ? 1. / (1 + 24 * a.volf * p / x) : 1. / sqrt(1 + 24 * a.volf * p / x);
    v = sqrt(t);
  }
  store_real<OUT>(reinterpret_cast<OUT*>(a.out), i, v);
}

static int out_size(int sf_type, size_t* esz) {
  if (sf_type != HGX_C128 && sf_type != HGX_C64) return fail(HGX_ERR_INVALID_ARG, "unknown output type");
  *esz = sf_type == HGX_C64 ? sizeof(float2) : sizeof(double2);
  return HGX_OK;
}

}  // namespace hgx

using namespace hgx;

extern "C" {

int hgx_sf_paracrystal(hgx_ctx c, hgx_qgrid g, int dims, int lattice, double dist_x, double dist_y,
                       double sdev_x, double sdev_y, double domain, void* sf, int sf_type) {
  if (!c || !g || !sf) return fail(HGX_ERR_INVALID_ARG, "hgx_sf_paracrystal: null argument");
  if (g->ctx != c) return fail(HGX_ERR_INVALID_ARG, "hgx_sf_paracrystal: grid of another context");
  if (dims != 1 && dims != 2)
    return fail(HGX_ERR_INVALID_ARG, "hgx_sf_paracrystal: dims must be 1 or 2");
  if (dims == 2 && lattice != 3 && lattice != 7)
    return fail(HGX_ERR_INVALID_ARG, "hgx_sf_paracrystal: a 2-D paracrystal is defined for the "
                                     "cubic (3) and hex (7) lattices only");
  size_t esz = 0;
  HGX_TRY(out_size(sf_type, &esz));
  HGX_CUDA(cudaSetDevice(c->device));
  DevBuf ob;
  void* dout = nullptr;
  HGX_TRY(stage_out(c, sf, esz * (size_t)g->nqz, ob, &dout));
  ParaArgs a{dims, lattice, dist_x, dist_y, sdev_x, sdev_y, exp(-2. * dist_x / domain),
             exp(-2. * dist_y / domain), g->qx, g->qy, g->nqy, (long)g->nqz, dout};
  const unsigned blocks = (unsigned)((g->nqz + LQ_THREADS - 1) / LQ_THREADS);
  if (sf_type == HGX_C64) paracrystal_kernel<float2><<<blocks, LQ_THREADS, 0, c->stream>>>(a);
  else paracrystal_kernel<double2><<<blocks, LQ_THREADS, 0, c->stream>>>(a);
  HGX_CUDA(cudaGetLastError());
  return finish_out(c, sf, esz * (size_t)g->nqz, dout);
}

int hgx_sf_percus_yevick(hgx_ctx c, hgx_qgrid g, double diameter, double volfract, int dims,
                         void* sf, int sf_type) {
  if (!c || !g || !sf) return fail(HGX_ERR_INVALID_ARG, "hgx_sf_percus_yevick: null argument");
  if (g->ctx != c) return fail(HGX_ERR_INVALID_ARG, "hgx_sf_percus_yevick: grid of another context");
  if (dims != 2 && dims != 3) return fail(HGX_ERR_INVALID_ARG, "hgx_sf_percus_yevick: dims must be 2 or 3");
  size_t esz = 0;
  HGX_TRY(out_size(sf_type, &esz));
  HGX_CUDA(cudaSetDevice(c->device));
  DevBuf ob;
  void* dout = nullptr;
  HGX_TRY(stage_out(c, sf, esz * (size_t)g->nqz, ob, &dout));
  // src/sf/liquid.cpp:128-131
  const double tmp = pow(1 - volfract, 4);
  const double alpha = pow(1 + 2 * volfract, 2) / tmp;
  const double beta = -6 * volfract * pow(1 + 0.5 * volfract, 2) / tmp;
  const double gamma = 0.5 * volfract * alpha;
  PYArgs a{dims, diameter, volfract, alpha, beta, gamma, g->qx, g->qy, g->qz, g->nqy, (long)g->nqz, dout};
  const unsigned blocks = (unsigned)((g->nqz + LQ_THREADS - 1) / LQ_THREADS);
  if (sf_type == HGX_C64) percus_yevick_kernel<float2><<<blocks, LQ_THREADS, 0, c->stream>>>(a);
  else percus_yevick_kernel<double2><<<blocks, LQ_THREADS, 0, c->stream>>>(a);
  HGX_CUDA(cudaGetLastError());
  return finish_out(c, sf, esz * (size_t)g->nqz, dout);
}

}  // extern "C"

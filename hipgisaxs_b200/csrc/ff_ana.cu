// Analytic form factors: box, cube, cylinder, sphere, prism3, prism6, pyramid — the shapes
// the reference implements (AnalyticFormFactor::compute, src/ff/ff_ana.cpp:61-161; CPU
// formulas in src/ff/ff_ana_{box,cube,cylinder,sphere,prism,prism6,pyramid}.cpp; GPU class
// AnalyticFormFactorG, include/ff/gpu/ff_ana_gpu.cuh:28-96).  FP64, one thread per q-point.
//
// Where the reference's nested loops over the size distributions multiply factors that each
// depend on one dimension only (cylinder r x h, box x y z, prism3/prism6 edge x height), the
// kernel sums each dimension once and multiplies the sums: the same value, n_r + n_h work
// instead of n_r * n_h.  The cylinder sums its samples unweighted, as the reference does
// (ff_ana_cylinder.cpp:107-111); the other shapes use the distribution weights.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <cmath>

#include <string>
#include <vector>

#include "ana_sf.cuh"
#include "ana_sf_f32.cuh"
#include "cplx.cuh"
#include "hgx_internal.cuh"

namespace hgx {

template <typename OUT>
__device__ __forceinline__ void put(void* out, long i, zd v);
template <>
__device__ __forceinline__ void put<double2>(void* out, long i, zd v) {
  reinterpret_cast<double2*>(out)[i] = v.d2();
}
template <>
__device__ __forceinline__ void put<float2>(void* out, long i, zd v) {
  reinterpret_cast<float2*>(out)[i] = make_float2((float)v.x, (float)v.y);
}

struct AnaArgs {
  AnaShape s;
  double tv[3];
  Rot9d R;
  const double* qx;
  const double* qy;
  const double2* qz;
  int nqy, nqz;
  void* out;
  int out_c64;
};

template <typename OUT>
__global__ void __launch_bounds__(128) ff_analytic_kernel(const AnaArgs* __restrict__ ap) {
  const AnaArgs& a = *ap;
  long iz = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (iz >= a.nqz) return;
  long iy = iz % a.nqy;
  zd m[3];
  rotate_q(a.R, a.qx[iy], a.qy[iy], zd(a.qz[iz]), m);
  put<OUT>(a.out, iz, ff_analytic_eval(a.s, m, a.tv));
}

// FP32C for a grid with real qz: the rotated q is real, the body is ana_sf_f32.cuh's (FP64
// phase reduction, FP32 transcendentals and sums).  SHAPE: cylinder, sphere or box.
template <int SHAPE, typename OUT>
__global__ void __launch_bounds__(128) ff_analytic_f32c_kernel(const AnaArgs* __restrict__ ap) {
  const AnaArgs& a = *ap;
  long iz = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (iz >= a.nqz) return;
  long iy = iz % a.nqy;
  const double qx = a.qx[iy], qy = a.qy[iy], qz = a.qz[iz].x;
  double m[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) m[j] = a.R.r[3 * j] * qx + a.R.r[3 * j + 1] * qy + a.R.r[3 * j + 2] * qz;
  const cf v = ff_analytic_f32c<SHAPE>(a.s, m, a.tv);
  put<OUT>(a.out, iz, zd((double)v.x, (double)v.y));
}

// ------------------------------------------------------------------- host side ----

// AnalyticFormFactor::param_distribution, src/ff/ff_ana.cpp:235-284.
// stat: StatisticType (include/common/enums.hpp:74-84): 0 null, 2 none, 4 gaussian, 8 uniform.
int param_distribution_host(int stat, double pmin, double pmax, double mean, double dev,
                            int nvalues, std::vector<double>& dim, std::vector<double>& w) {
  if (nvalues < 1) return fail(HGX_ERR_INVALID_ARG, "param_distribution: nvalues < 1");
  double maxv = pmax;
  if (pmax < pmin) pmax = pmin;
  size_t first = dim.size();
  if (nvalues > 1) {
    double step = fabs(pmax - pmin) / (nvalues - 1);
    double curr = pmin;
    do {
      dim.push_back(curr);
      curr += step;
      if (dim.size() - first > (size_t)4 * nvalues + 8)
        return fail(HGX_ERR_INVALID_ARG, "param_distribution: min/max/nvalues inconsistent");
    } while (curr < maxv);
  } else {
    dim.push_back(pmin);
  }
  size_t n = dim.size() - first;
  if (stat == 2 || stat == 0) {
    // the reference pushes a single weight; only single-valued parameters are meaningful
    for (size_t i = 0; i < n; ++i) w.push_back(i == 0 ? 1.0 : 0.0);
  } else if (stat == 8) {
    for (size_t i = 0; i < n; ++i) w.push_back(1.0);
  } else if (stat == 4) {
    if (!std::isfinite(mean)) mean = (dim[first] + dim[first + n - 1]) / 2;
    for (size_t i = 0; i < n; ++i)
      w.push_back(exp(-1.0 * pow((dim[first + i] - mean), 2) / (2 * pow(dev, 2))) /
                  (sqrt(2 * PI_REF) * dev));
  } else {
    return fail(HGX_ERR_INVALID_ARG, "param_distribution: unsupported statistic");
  }
  return HGX_OK;
}

static int fill_dist(Dist& d, int n, const double* v, const double* w, const char* what) {
  if (n < 0 || n > ANA_MAXV)
    return fail(HGX_ERR_INVALID_ARG, std::string("hgx_ff_analytic: ") + what +
                                         ": between 0 and 64 samples per dimension");
  if (n > 0 && !v) return fail(HGX_ERR_INVALID_ARG, std::string("hgx_ff_analytic: ") + what + " values NULL");
  d.n = n;
  for (int i = 0; i < n; ++i) {
    d.v[i] = v[i];
    d.w[i] = w ? w[i] : 1.0;
  }
  // evenly stepped samples (the FP32C cylinder sums their height exponentials in closed form)
  d.prog = 0;
  if (n >= 3) {
    const double step = (v[n - 1] - v[0]) / (n - 1);
    double big = 0.0;
    for (int i = 0; i < n; ++i) big = std::max(big, std::fabs(v[i]));
    bool prog = step != 0.0;
    for (int i = 0; i < n && prog; ++i) prog = std::fabs(v[i] - (v[0] + i * step)) <= 1e-12 * big;
    d.prog = prog ? 1 : 0;
  }
  return HGX_OK;
}

static int check_dims(const AnaShape& a) {
  const int n1 = a.d[0].n, n2 = a.d[1].n, n3 = a.d[2].n;
  switch (a.shape) {
    case SH_BOX:
      if (!n1 || !n2 || !n3) return fail(HGX_ERR_INVALID_ARG, "box needs x, y and height");
      break;
    case SH_CUBE:
    case SH_SPHERE:
      if (!n1) return fail(HGX_ERR_INVALID_ARG, "cube/sphere need dimension 1");
      break;
    case SH_CYLINDER:
    case SH_PRISM3:
      if (!n1 || !n3) return fail(HGX_ERR_INVALID_ARG, "cylinder/prism3 need dimensions 1 and 3");
      break;
    case SH_PRISM6:
    case SH_PYRAMID:
      break;
    default:
      return fail(HGX_ERR_INVALID_ARG, "hgx_ff_analytic: shape not implemented by the reference");
  }
  return HGX_OK;
}

// The reference's parameter routing (the compute_* switch statements of
// src/ff/ff_ana_*.cpp) plus param_distribution: HiG-style parameters (7 doubles each:
// ShapeParamType, StatisticType, min, max, mean, deviation, nvalues) -> the sampled dimensions
// of an AnaShape, checked as hgx_ff_analytic checks them.
int ana_shape_from_params(int shape, int nparam, const double* params, double tau, double eta,
                          AnaShape& out) {
  if (nparam < 0 || (nparam > 0 && !params))
    return fail(HGX_ERR_INVALID_ARG, "analytic shape: bad parameter list");
  enum { P_RADIUS = 2, P_XSIZE = 3, P_YSIZE = 4, P_HEIGHT = 5, P_EDGE = 6, P_BASEANGLE = 7 };
  std::vector<double> v[4], w[4];
  for (int i = 0; i < nparam; ++i) {
    const double* p = params + 7 * i;
    int type = (int)p[0];
    std::vector<int> dims;
    switch (shape) {
      case SH_BOX:
        if (type == P_EDGE) dims = {0, 1, 2};
        else if (type == P_XSIZE) dims = {0};
        else if (type == P_YSIZE) dims = {1};
        else if (type == P_HEIGHT) dims = {2};
        break;
      case SH_CUBE:
        if (type == P_HEIGHT) dims = {0};
        break;
      case SH_CYLINDER:
        if (type == P_RADIUS) dims = {0};
        else if (type == P_HEIGHT) dims = {2};
        break;
      case SH_SPHERE:
        if (type == P_RADIUS) dims = {0};
        else if (type == P_EDGE || type == P_XSIZE || type == P_YSIZE || type == P_HEIGHT)
          dims = {2};
        break;
      case SH_PRISM3:
      case SH_PRISM6:
        if (type == P_EDGE) dims = {0};
        else if (type == P_HEIGHT) dims = {2};
        break;
      case SH_PYRAMID:
        if (type == P_XSIZE) dims = {0};
        else if (type == P_YSIZE) dims = {1};
        else if (type == P_HEIGHT) dims = {2};
        else if (type == P_BASEANGLE) dims = {3};
        break;
      default:
        return fail(HGX_ERR_INVALID_ARG, "analytic shape: shape not implemented by the reference");
    }
    for (int d : dims)
      HGX_TRY(param_distribution_host((int)p[1], p[2], p[3], p[4], p[5], (int)p[6], v[d], w[d]));
  }
  out.shape = shape;
  for (int k = 0; k < 4; ++k)
    HGX_TRY(fill_dist(out.d[k], (int)v[k].size(), v[k].empty() ? nullptr : v[k].data(),
                      w[k].empty() ? nullptr : w[k].data(), "a parameter distribution"));
  out.tau = tau;
  out.eta = eta;
  return check_dims(out);
}

int ff_analytic_launch(hgx_ctx c, hgx_qgrid g, const AnaArgs& host_args, void* out, int ff_type,
                       int precision) {
  // the argument block (about 4 KB) goes to device scratch so the kernel can index it freely
  AnaArgs a = host_args;
  a.qx = g->qx;
  a.qy = g->qy;
  a.qz = g->qz;
  a.nqy = g->nqy;
  a.nqz = g->nqz;
  a.out = out;
  a.out_c64 = ff_type == HGX_C64;
  HGX_TRY(c->scratch.reserve(sizeof(AnaArgs)));
  AnaArgs* d_args = reinterpret_cast<AnaArgs*>(c->scratch.p);
  HGX_CUDA(cudaMemcpyAsync(d_args, &a, sizeof(AnaArgs), cudaMemcpyHostToDevice, c->stream));
  dim3 grid((g->nqz + 127) / 128);
  const int sh = a.s.shape;
  if (precision == HGX_F32C && g->mode == 1 && (sh == SH_CYLINDER || sh == SH_SPHERE || sh == SH_BOX)) {
    cudaStream_t st = c->stream;
    if (sh == SH_CYLINDER) {
      if (a.out_c64) ff_analytic_f32c_kernel<SH_CYLINDER, float2><<<grid, 128, 0, st>>>(d_args);
      else ff_analytic_f32c_kernel<SH_CYLINDER, double2><<<grid, 128, 0, st>>>(d_args);
    } else if (sh == SH_SPHERE) {
      if (a.out_c64) ff_analytic_f32c_kernel<SH_SPHERE, float2><<<grid, 128, 0, st>>>(d_args);
      else ff_analytic_f32c_kernel<SH_SPHERE, double2><<<grid, 128, 0, st>>>(d_args);
    } else {
      if (a.out_c64) ff_analytic_f32c_kernel<SH_BOX, float2><<<grid, 128, 0, st>>>(d_args);
      else ff_analytic_f32c_kernel<SH_BOX, double2><<<grid, 128, 0, st>>>(d_args);
    }
    HGX_CUDA(cudaGetLastError());
    return HGX_OK;
  }
  if (a.out_c64) ff_analytic_kernel<float2><<<grid, 128, 0, c->stream>>>(d_args);
  else ff_analytic_kernel<double2><<<grid, 128, 0, c->stream>>>(d_args);
  HGX_CUDA(cudaGetLastError());
  return HGX_OK;  // a pageable-source cudaMemcpyAsync has consumed `a` when it returns
}

}  // namespace hgx

using namespace hgx;

extern "C" {

int hgx_param_distribution(int stat, double pmin, double pmax, double mean, double dev,
                           int nvalues, double* values, double* weights, int cap, int* count) {
  if (!values || !weights || !count || cap < 1)
    return fail(HGX_ERR_INVALID_ARG, "hgx_param_distribution: null argument");
  std::vector<double> d, w;
  HGX_TRY(param_distribution_host(stat, pmin, pmax, mean, dev, nvalues, d, w));
  if ((int)d.size() > cap) return fail(HGX_ERR_INVALID_ARG, "hgx_param_distribution: cap too small");
  for (size_t i = 0; i < d.size(); ++i) {
    values[i] = d[i];
    weights[i] = w[i];
  }
  *count = (int)d.size();
  return HGX_OK;
}

int hgx_ff_analytic_ex(hgx_ctx c, hgx_qgrid g, int shape, int n1, const double* v1,
                       const double* w1, int n2, const double* v2, const double* w2, int n3,
                       const double* v3, const double* w3, int n4, const double* v4,
                       const double* w4, double tau, double eta, const double* transvec,
                       const double* rot9, void* ff, int ff_type, int precision) {
  if (precision != HGX_F64 && precision != HGX_F32C)
    return fail(HGX_ERR_INVALID_ARG, "hgx_ff_analytic: unknown precision");
  if (!c || !g || !ff) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_analytic: null argument");
  if (g->ctx != c) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_analytic: grid of another context");
  if (ff_type != HGX_C128 && ff_type != HGX_C64)
    return fail(HGX_ERR_INVALID_ARG, "hgx_ff_analytic: unknown output type");
  AnaArgs a;  // about 4 KB; filled here, copied to device scratch by ff_analytic_launch
  a.s.shape = shape;
  HGX_TRY(fill_dist(a.s.d[0], n1, v1, w1, "dimension 1"));
  HGX_TRY(fill_dist(a.s.d[1], n2, v2, w2, "dimension 2"));
  HGX_TRY(fill_dist(a.s.d[2], n3, v3, w3, "dimension 3"));
  HGX_TRY(fill_dist(a.s.d[3], n4, v4, w4, "dimension 4"));
  HGX_TRY(check_dims(a.s));
  a.s.tau = tau;
  a.s.eta = eta;
  for (int i = 0; i < 3; ++i) a.tv[i] = transvec ? transvec[i] : 0.0;
  static const double eye[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int i = 0; i < 9; ++i) a.R.r[i] = rot9 ? rot9[i] : eye[i];
  HGX_CUDA(cudaSetDevice(c->device));
  const size_t esz = ff_type == HGX_C64 ? sizeof(float2) : sizeof(double2);
  const bool host_out = !is_device_ptr(ff);
  DevBuf tmp;
  void* dout = ff;
  if (host_out) {
    HGX_TRY(tmp.reserve(esz * (size_t)g->nqz));
    dout = tmp.p;
  }
  HGX_TRY(ff_analytic_launch(c, g, a, dout, ff_type, precision));
  if (host_out) {
    HGX_CUDA(cudaMemcpyAsync(ff, dout, esz * (size_t)g->nqz, cudaMemcpyDeviceToHost, c->stream));
    return hgx_synchronize(c);
  }
  return HGX_OK;
}

int hgx_ff_analytic(hgx_ctx c, hgx_qgrid g, int shape, int n1, const double* v1,
                    const double* w1, int n2, const double* v2, const double* w2, int n3,
                    const double* v3, const double* w3, int n4, const double* v4,
                    const double* w4, double tau, double eta, const double* transvec,
                    const double* rot9, void* ff, int ff_type) {
  return hgx_ff_analytic_ex(c, g, shape, n1, v1, w1, n2, v2, w2, n3, v3, w3, n4, v4, w4, tau, eta,
                            transvec, rot9, ff, ff_type, HGX_F64);
}

// The reference's parameter routing (the compute_* switch statements of
// src/ff/ff_ana_*.cpp) plus param_distribution, then hgx_ff_analytic.
// params: 7 doubles per parameter (ShapeParamType, StatisticType, min, max, mean,
// deviation, nvalues).
int hgx_ff_analytic_params_ex(hgx_ctx c, hgx_qgrid g, int shape, int nparam, const double* params,
                              double tau, double eta, const double* transvec, const double* rot9,
                              void* ff, int ff_type, int precision) {
  AnaShape s;
  HGX_TRY(ana_shape_from_params(shape, nparam, params, tau, eta, s));
  std::vector<double> v[4], w[4];
  for (int k = 0; k < 4; ++k) {
    v[k].assign(s.d[k].v, s.d[k].v + s.d[k].n);
    w[k].assign(s.d[k].w, s.d[k].w + s.d[k].n);
  }
  auto ptr = [](std::vector<double>& x) { return x.empty() ? nullptr : x.data(); };
  return hgx_ff_analytic_ex(c, g, shape, (int)v[0].size(), ptr(v[0]), ptr(w[0]), (int)v[1].size(),
                            ptr(v[1]), ptr(w[1]), (int)v[2].size(), ptr(v[2]), ptr(w[2]),
                            (int)v[3].size(), ptr(v[3]), ptr(w[3]), tau, eta, transvec, rot9, ff,
                            ff_type, precision);
}

int hgx_ff_analytic_params(hgx_ctx c, hgx_qgrid g, int shape, int nparam, const double* params,
                           double tau, double eta, const double* transvec, const double* rot9,
                           void* ff, int ff_type) {
  return hgx_ff_analytic_params_ex(c, g, shape, nparam, params, tau, eta, transvec, rot9, ff, ff_type,
                                   HGX_F64);
}

}  // extern "C"

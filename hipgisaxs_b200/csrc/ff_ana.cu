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

#include <string>
#include <vector>

#include "cplx.cuh"
#include "hgx_internal.cuh"

namespace hgx {

constexpr double PI_REF = 3.141592653589793;  // PI_, include/common/constants.hpp
constexpr double CUTINY_REF = 1.0e-13;
constexpr int ANA_MAXV = 64;  // samples per dimension

// ShapeName values (include/common/enums.hpp:24-43)
enum { SH_BOX = 2, SH_CUBE = 3, SH_CYLINDER = 4, SH_SPHERE = 5, SH_PRISM3 = 8, SH_PRISM6 = 9,
       SH_PYRAMID = 14 };

struct Dist {
  int n;
  double v[ANA_MAXV];
  double w[ANA_MAXV];
};

struct AnaArgs {
  int shape;
  Dist d[4];
  double tau, eta, tv[3];
  Rot9d R;
  const double* qx;
  const double* qy;
  const double2* qz;
  int nqy, nqz;
  void* out;
  int out_c64;
};

// hig::sinc, include/numerics/numeric_utils.hpp:54-63 (free function)
__device__ __forceinline__ zd sinc_free(zd x) {
  if (cabs_(x) > 1.0E-14) return csin_(x) / x;
  zd x2 = x * x;
  return (1.0 - x2 / 6.0) + (x2 * x * x) / 120.0;
}
// AnalyticFormFactor::sinc, src/ff/ff_ana.cpp:222-227 (member)
__device__ __forceinline__ zd sinc_member(zd v) {
  if (fabs(v.x) <= 1e-14 && fabs(v.y) <= 1e-14) return zd(1.0, 0.0);
  return csin_(v) / v;
}
// AnalyticFormFactor::fq_inv, src/ff/ff_ana.cpp:190-196
__device__ __forceinline__ zd fq_inv(zd value, double y) {
  zd t = (cexp_((zd(0, 1) * value) * y / 2.0) * 2.0) * csin_(value * y / 2.0) / value;
  if (cabs_(t) <= 1e-14) t = zd(y, 0);
  return t;
}
__device__ __forceinline__ zd trans_phase(const zd* m, const double* tv) {
  zd t = m[0] * tv[0] + m[1] * tv[1] + m[2] * tv[2];
  return cexp_(zd(-t.y, t.x));
}

// ff_ana_sphere.cpp:33-45
__device__ zd ff_sphere_one(zd qx, zd qy, zd qz, double radius) {
  zd qval = csqrt_(qx * qx + qy * qy + qz * qz);
  if (cabs_(qval) < 2.2250738585072014e-308) return zd(0, 0);
  zd qR = qval * radius;
  zd qR3 = qR * qR * qR;
  zd t1 = conj(qR3) / norm2(qR3);
  zd c0 = (csin_(qR) - qR * ccos_(qR)) * t1;
  zd c1 = cexp_((zd(0, 1) * qz) * radius);
  double f0 = 4 * PI_REF * radius * radius * radius;
  return (c0 * f0) * c1;
}

// ff_ana_pyramid.cpp:35-78 (angle in degrees)
__device__ zd ff_pyramid_one(zd qx, zd qy, zd qz, double L, double W, double H, double angle) {
  double a = angle * PI_REF / 180.;
  double tan_a = tan(a);
  if ((2 * H / L >= tan_a) || (2 * H / W >= tan_a)) return zd(0, 0);
  zd tmp = qx * qy;
  if (cabs_(tmp) < 1.0E-20) return zd(0, 0);
  const zd PJ(0, 1), NJ(0, -1);
  zd q1 = ((qx - qy) / tan_a + qz) * 0.5;
  zd q2 = ((qx - qy) / tan_a - qz) * 0.5;
  zd q3 = ((qx + qy) / tan_a + qz) * 0.5;
  zd q4 = ((qx + qy) / tan_a - qz) * 0.5;
  zd s1 = sinc_free(q1 * H) * cexp_((NJ * q1) * H), s2 = sinc_free(q2 * H) * cexp_((PJ * q2) * H);
  zd s3 = sinc_free(q3 * H) * cexp_((NJ * q3) * H), s4 = sinc_free(q4 * H) * cexp_((PJ * q4) * H);
  zd k1 = s1 + s2, k2 = s1 * NJ + s2 * PJ, k3 = s3 + s4, k4 = s3 * NJ + s4 * PJ;
  zd am = (qx * L - qy * W) * 0.5, ap = (qx * L + qy * W) * 0.5;
  zd t1 = k1 * ccos_(am), t2 = k2 * csin_(am), t3 = k3 * ccos_(ap), t4 = k4 * csin_(ap);
  return (H / tmp) * (t1 + t2 - t3 - t4);
}

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

template <typename OUT>
__global__ void __launch_bounds__(128) ff_analytic_kernel(const AnaArgs* __restrict__ ap) {
  const AnaArgs& a = *ap;
  long iz = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (iz >= a.nqz) return;
  long iy = iz % a.nqy;
  zd m[3];
  rotate_q(a.R, a.qx[iy], a.qy[iy], zd(a.qz[iz]), m);
  zd out(0, 0);
  const Dist& X = a.d[0];
  const Dist& Y = a.d[1];
  const Dist& Z = a.d[2];
  const Dist& B = a.d[3];
  switch (a.shape) {
    case SH_CYLINDER: {  // ff_ana_cylinder.cpp:34-42,100-117
      zd qpar = csqrt_(m[0] * m[0] + m[1] * m[1]);
      zd fr(0, 0), gh(0, 0);
      for (int i = 0; i < X.n; ++i) {
        double r = X.v[i];
        zd t1 = qpar * r;
        if (norm2(t1) > CUTINY_REF) fr += (zd(j1(t1.x), 0.0) * conj(t1) / norm2(t1)) * (2. * PI_REF * r * r);
      }
      for (int i = 0; i < Z.n; ++i) {
        double h = Z.v[i];
        gh += (sinc_free((m[2] * 0.5) * h) * h) * cexp_(((zd(0, 0.5)) * m[2]) * h);
      }
      out = fr * gh * trans_phase(m, a.tv);
      break;
    }
    case SH_SPHERE: {  // ff_ana_sphere.cpp:95-107
      zd acc(0, 0);
      for (int i = 0; i < X.n; ++i) acc += ff_sphere_one(m[0], m[1], m[2], X.v[i]) * X.w[i];
      out = acc * trans_phase(m, a.tv);
      break;
    }
    case SH_BOX: {  // ff_ana_box.cpp:35-42,96-125
      zd sx(0, 0), sy(0, 0), sz(0, 0);
      for (int i = 0; i < X.n; ++i) sx += sinc_free((m[0] * 0.5) * X.v[i]) * (X.v[i] * X.w[i]);
      for (int i = 0; i < Y.n; ++i) sy += sinc_free((m[1] * 0.5) * Y.v[i]) * (Y.v[i] * Y.w[i]);
      for (int i = 0; i < Z.n; ++i)
        sz += (cexp_((zd(0, 0.5) * m[2]) * Z.v[i]) * sinc_free((m[2] * 0.5) * Z.v[i])) *
              (Z.v[i] * Z.w[i]);
      out = sx * sy * sz * trans_phase(m, a.tv);
      break;
    }
    case SH_CUBE: {  // ff_ana_cube.cpp:35-42,87-107
      zd acc(0, 0);
      for (int i = 0; i < X.n; ++i) {
        double L = X.v[i];
        zd e = cexp_((zd(0, 0.5) * m[2]) * L);
        zd s = sinc_free((m[0] * 0.5) * L) * sinc_free((m[1] * 0.5) * L) * sinc_free((m[2] * 0.5) * L);
        acc += ((e * (L * L * L)) * s) * X.w[i];
      }
      out = acc * trans_phase(m, a.tv);
      break;
    }
    case SH_PRISM3: {  // ff_ana_prism.cpp:82-108 (unweighted)
      const double sqrt3 = sqrt(3.0);
      zd t1 = m[0] * (m[0] * m[0] - (m[1] * 3.0) * m[1]);
      zd t2 = m[2] + (m[0] * sin(a.eta) + m[1] * cos(a.eta)) * tan(a.tau);
      zd sl(0, 0), sh(0, 0);
      for (int i = 0; i < X.n; ++i) {
        double L = X.v[i];
        zd t4 = m[0] * cexp_(((zd(0, 1) * m[1]) * L) * sqrt3);
        zd t5 = m[0] * ccos_(m[0] * L);
        zd t6 = (zd(0, sqrt3) * m[1]) * csin_(m[0] * L);
        zd t3 = (m[1] * L) / sqrt3;
        zd t9 = cexp_(zd(t3.y, -t3.x)) * (2.0 * sqrt3);
        sl += (t9 / t1) * (t4 - t5 - t6);
      }
      for (int i = 0; i < Z.n; ++i) sh += fq_inv(t2, Z.v[i]);
      out = sl * sh * trans_phase(m, a.tv);
      break;
    }
    case SH_PRISM6: {  // ff_ana_prism6.cpp:80-98 (unweighted)
      const double sqrt3 = sqrt(3.0);
      zd qm = (m[0] * sin(a.eta) + m[1] * cos(a.eta)) * tan(a.tau);
      zd t1 = (4.0 * sqrt3) / ((m[1] * 3.0) * m[1] - m[0] * m[0]);
      zd sl(0, 0), sh(0, 0);
      for (int i = 0; i < X.n; ++i) {
        double L = X.v[i];
        zd rmqx = (m[0] * L) / sqrt3, rmqy = m[1] * L;
        zd t2 = rmqy * rmqy * sinc_member(rmqx) * sinc_member(rmqy);
        zd t3 = ccos_(rmqx * 2.0);
        zd t4 = ccos_(rmqy) * ccos_(rmqx);
        sl += t2 + t3 - t4;
      }
      for (int i = 0; i < Z.n; ++i) sh += fq_inv(m[2] + qm, Z.v[i]);
      out = t1 * sl * sh * trans_phase(m, a.tv);
      break;
    }
    case SH_PYRAMID: {  // ff_ana_pyramid.cpp:118-139
      zd acc(0, 0);
      for (int i = 0; i < X.n; ++i)
        for (int j = 0; j < Y.n; ++j)
          for (int h = 0; h < Z.n; ++h)
            for (int b = 0; b < B.n; ++b) {
              double prob = X.w[i] * Y.w[j] * Z.w[h] * B.w[b];
              acc += ff_pyramid_one(m[0], m[1], m[2], X.v[i], Y.v[j], Z.v[h], B.v[b]) * prob;
            }
      zd t1 = m[0] * a.tv[0] + m[1] * a.tv[1] + m[2] * a.tv[2];
      out = acc * cexp_(zd(0, 1) * t1);
      break;
    }
    default:
      break;
  }
  put<OUT>(a.out, iz, out);
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
  return HGX_OK;
}

int ff_analytic_launch(hgx_ctx c, hgx_qgrid g, const AnaArgs& host_args, void* out, int ff_type) {
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

int hgx_ff_analytic(hgx_ctx c, hgx_qgrid g, int shape, int n1, const double* v1,
                    const double* w1, int n2, const double* v2, const double* w2, int n3,
                    const double* v3, const double* w3, int n4, const double* v4,
                    const double* w4, double tau, double eta, const double* transvec,
                    const double* rot9, void* ff, int ff_type) {
  if (!c || !g || !ff) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_analytic: null argument");
  if (g->ctx != c) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_analytic: grid of another context");
  if (ff_type != HGX_C128 && ff_type != HGX_C64)
    return fail(HGX_ERR_INVALID_ARG, "hgx_ff_analytic: unknown output type");
  AnaArgs a;  // about 4 KB; filled here, copied to device scratch by ff_analytic_launch
  a.shape = shape;
  HGX_TRY(fill_dist(a.d[0], n1, v1, w1, "dimension 1"));
  HGX_TRY(fill_dist(a.d[1], n2, v2, w2, "dimension 2"));
  HGX_TRY(fill_dist(a.d[2], n3, v3, w3, "dimension 3"));
  HGX_TRY(fill_dist(a.d[3], n4, v4, w4, "dimension 4"));
  switch (shape) {
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
  a.tau = tau;
  a.eta = eta;
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
  HGX_TRY(ff_analytic_launch(c, g, a, dout, ff_type));
  if (host_out) {
    HGX_CUDA(cudaMemcpyAsync(ff, dout, esz * (size_t)g->nqz, cudaMemcpyDeviceToHost, c->stream));
    return hgx_synchronize(c);
  }
  return HGX_OK;
}

// The reference's parameter routing (the compute_* switch statements of
// src/ff/ff_ana_*.cpp) plus param_distribution, then hgx_ff_analytic.
// params: 7 doubles per parameter (ShapeParamType, StatisticType, min, max, mean,
// deviation, nvalues).
int hgx_ff_analytic_params(hgx_ctx c, hgx_qgrid g, int shape, int nparam, const double* params,
                           double tau, double eta, const double* transvec, const double* rot9,
                           void* ff, int ff_type) {
  if (nparam < 0 || (nparam > 0 && !params))
    return fail(HGX_ERR_INVALID_ARG, "hgx_ff_analytic_params: bad parameter list");
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
        return fail(HGX_ERR_INVALID_ARG, "hgx_ff_analytic_params: shape not implemented by the reference");
    }
    for (int d : dims)
      HGX_TRY(param_distribution_host((int)p[1], p[2], p[3], p[4], p[5], (int)p[6], v[d], w[d]));
  }
  auto ptr = [](std::vector<double>& x) { return x.empty() ? nullptr : x.data(); };
  return hgx_ff_analytic(c, g, shape, (int)v[0].size(), ptr(v[0]), ptr(w[0]), (int)v[1].size(),
                         ptr(v[1]), ptr(w[1]), (int)v[2].size(), ptr(v[2]), ptr(w[2]),
                         (int)v[3].size(), ptr(v[3]), ptr(w[3]), tau, eta, transvec, rot9, ff,
                         ff_type);
}

}  // extern "C"

// Device math shared by the analytic form-factor kernel (ff_ana.cu), the lattice
// structure-factor kernel (sf.cu) and the fused grain kernel (hig_fused.cu): the per-q-point
// bodies, so that every kernel evaluates the reference's formulas with the same code.
#pragma once

#include <cuda_runtime.h>
#include <float.h>
#include <math.h>

#include "cplx.cuh"

namespace hgx {

constexpr double PI_REF = 3.141592653589793;  // PI_, include/common/constants.hpp
constexpr double CUTINY_REF = 1.0e-13;
constexpr int ANA_MAXV = 64;  // samples per dimension

// ShapeName values (include/common/enums.hpp:24-43)
enum { SH_BOX = 2, SH_CUBE = 3, SH_CYLINDER = 4, SH_SPHERE = 5, SH_PRISM3 = 8, SH_PRISM6 = 9,
       SH_PYRAMID = 14 };

struct Dist {
  int n;
  int prog;  // the values form an arithmetic progression (n >= 3, within 1e-12 relative)
  double v[ANA_MAXV];
  double w[ANA_MAXV];
};

// one analytic shape: its kind, up to four sampled dimensions and the prism tilt angles
struct AnaShape {
  int shape;
  Dist d[4];
  double tau, eta;
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
// v * trans_phase(m, tv); at the origin the phase is exactly (1, +-0), whose product leaves a
// finite v as it is (up to the sign of a zero), so it is not evaluated there; a non-finite v
// still takes the product (inf * 0 makes the NaN the reference's product makes)
__device__ __forceinline__ zd with_phase(zd v, const zd* m, const double* tv) {
  if (tv[0] == 0.0 && tv[1] == 0.0 && tv[2] == 0.0 && isfinite(v.x) && isfinite(v.y)) return v;
  return v * trans_phase(m, tv);
}

// ff_ana_sphere.cpp:33-45
static __device__ zd ff_sphere_one(zd qx, zd qy, zd qz, double radius) {
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
static __device__ zd ff_pyramid_one(zd qx, zd qy, zd qz, double L, double W, double H, double angle) {
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

// The analytic form factor of shape `a` at the rotated q (m) translated by tv: the per-q-point
// body of the analytic form-factor kernel, shared with the fused grain kernel (hig_fused.cu).
// SHAPE != 0 compiles the one case (the caller guarantees a.shape == SHAPE).
template <int SHAPE = 0>
__device__ __forceinline__ zd ff_analytic_eval(const AnaShape& a, const zd* m, const double* tv) {
  zd out(0, 0);
  const Dist& X = a.d[0];
  const Dist& Y = a.d[1];
  const Dist& Z = a.d[2];
  const Dist& B = a.d[3];
  switch (SHAPE ? SHAPE : a.shape) {
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
      out = with_phase(fr * gh, m, tv);
      break;
    }
    case SH_SPHERE: {  // ff_ana_sphere.cpp:95-107
      zd acc(0, 0);
      for (int i = 0; i < X.n; ++i) acc += ff_sphere_one(m[0], m[1], m[2], X.v[i]) * X.w[i];
      out = with_phase(acc, m, tv);
      break;
    }
    case SH_BOX: {  // ff_ana_box.cpp:35-42,96-125
      zd sx(0, 0), sy(0, 0), sz(0, 0);
      for (int i = 0; i < X.n; ++i) sx += sinc_free((m[0] * 0.5) * X.v[i]) * (X.v[i] * X.w[i]);
      for (int i = 0; i < Y.n; ++i) sy += sinc_free((m[1] * 0.5) * Y.v[i]) * (Y.v[i] * Y.w[i]);
      for (int i = 0; i < Z.n; ++i)
        sz += (cexp_((zd(0, 0.5) * m[2]) * Z.v[i]) * sinc_free((m[2] * 0.5) * Z.v[i])) *
              (Z.v[i] * Z.w[i]);
      out = with_phase(sx * sy * sz, m, tv);
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
      out = with_phase(acc, m, tv);
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
      out = with_phase(sl * sh, m, tv);
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
      out = with_phase(t1 * sl * sh, m, tv);
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
      zd t1 = m[0] * tv[0] + m[1] * tv[1] + m[2] * tv[2];
      out = acc * cexp_(zd(0, 1) * t1);
      break;
    }
    default:
      break;
  }
  return out;
}

// The quad of four lanes (one per DWBA block) of the fused grain kernel: v summed over the
// quad, the same bits in every lane (an xor butterfly of commutative adds).
__device__ __forceinline__ zd quad_sum_zd(zd v) {
  v.x += __shfl_xor_sync(0xffffffffu, v.x, 1);
  v.y += __shfl_xor_sync(0xffffffffu, v.y, 1);
  v.x += __shfl_xor_sync(0xffffffffu, v.x, 2);
  v.y += __shfl_xor_sync(0xffffffffu, v.y, 2);
  return v;
}

// ff_analytic_eval for a quad whose rotated in-plane q (m[0], m[1]) is the same in its four
// lanes (the element's rotation keeps qz out of them): the cylinder's radial sum and the box's
// x and y sums, which depend on the in-plane q only, are split among the lanes (lane k takes
// the samples k, k + 4, ...) and closed by quad_sum_zd; the rest is per lane, as in
// ff_analytic_eval.  Every lane of the warp calls it (shuffles).
template <int SHAPE>
__device__ __forceinline__ zd ff_analytic_eval_quad(const AnaShape& a, const zd* m, const double* tv, int k) {
  const Dist& X = a.d[0];
  const Dist& Y = a.d[1];
  const Dist& Z = a.d[2];
  if (SHAPE == SH_CYLINDER) {
    zd qpar = csqrt_(m[0] * m[0] + m[1] * m[1]);
    zd fr(0, 0), gh(0, 0);
    for (int i = k; i < X.n; i += 4) {
      double r = X.v[i];
      zd t1 = qpar * r;
      if (norm2(t1) > CUTINY_REF) fr += (zd(j1(t1.x), 0.0) * conj(t1) / norm2(t1)) * (2. * PI_REF * r * r);
    }
    fr = quad_sum_zd(fr);
    for (int i = 0; i < Z.n; ++i) {
      double h = Z.v[i];
      gh += (sinc_free((m[2] * 0.5) * h) * h) * cexp_(((zd(0, 0.5)) * m[2]) * h);
    }
    return with_phase(fr * gh, m, tv);
  }
  if (SHAPE == SH_BOX) {
    zd sx(0, 0), sy(0, 0), sz(0, 0);
    for (int i = k; i < X.n; i += 4) sx += sinc_free((m[0] * 0.5) * X.v[i]) * (X.v[i] * X.w[i]);
    for (int i = k; i < Y.n; i += 4) sy += sinc_free((m[1] * 0.5) * Y.v[i]) * (Y.v[i] * Y.w[i]);
    sx = quad_sum_zd(sx);
    sy = quad_sum_zd(sy);
    for (int i = 0; i < Z.n; ++i)
      sz += (cexp_((zd(0, 0.5) * m[2]) * Z.v[i]) * sinc_free((m[2] * 0.5) * Z.v[i])) * (Z.v[i] * Z.w[i]);
    return with_phase(sx * sy * sz, m, tv);
  }
  return ff_analytic_eval<SHAPE>(a, m, tv);
}

// The lattice structure factor at the rotated q (m): the per-q-point body of the lattice
// structure-factor kernel (sf.cu), shared with the fused grain kernel.  la/lb/lc are the
// scaled lattice vectors.
struct SfLat {
  double la[3], lb[3], lc[3];
  double rep[3];
  double center[3];
};

// Host side (ff_ana.cu): an AnaShape from HiG-style parameters, 7 doubles each (ShapeParamType,
// StatisticType, min, max, mean, deviation, nvalues), routed and sampled as the reference's
// AnalyticFormFactor::compute does.
int ana_shape_from_params(int shape, int nparam, const double* params, double tau, double eta,
                          AnaShape& out);

// One out-of-line copy of each, called from the structure factor: the fused grain kernel
// evaluates it for every grain, and a single copy keeps the kernel within the instruction cache.
static __device__ __noinline__ zd cpow_call(zd x, double y) { return cpow_std(x, y); }
static __device__ __noinline__ zd cexp_call(zd a) { return cexp_(a); }

__device__ __forceinline__ zd times_i(zd s) { return zd(-s.y, s.x); }  // (0,1) * s

__device__ __forceinline__ zd sf_lattice_eval(const SfLat& a, const zd* m) {
  const double eps = DBL_EPSILON;
  const zd one(1.0, 0.0);

  zd e_iqa = cexp_call(times_i(m[0] * a.la[0] + m[1] * a.la[1] + m[2] * a.la[2]));
  zd Xa = one - cpow_call(e_iqa, a.rep[0]);
  zd Ya = one - e_iqa;
  zd sa = (fabs(Ya.y) > eps || fabs(Ya.x) > eps) ? Xa / Ya : zd(a.rep[0], 0.0);
  sa = cpow_call(e_iqa, (1.0 - a.rep[0]) / 2.0) * sa;

  zd iqb = times_i(m[0] * a.lb[0] + m[1] * a.lb[1] + a.lb[2] * a.lb[2]);
  zd iqNb = iqb * a.rep[1];
  zd e_iqb = cexp_call(iqb);
  zd Xb = one - cexp_call(iqNb);
  zd Yb = one - e_iqb;
  zd sb = (fabs(Yb.y) > eps || fabs(Yb.x) > eps) ? Xb / Yb : zd(a.rep[1], 0.0);
  sb = cpow_call(e_iqb, (1.0 - a.rep[1]) / 2.0) * sb;

  zd e_iqc = cexp_call(times_i(m[0] * a.lc[0] + m[1] * a.lc[1] + m[2] * a.lc[2]));
  zd Xc = one - cpow_call(e_iqc, a.rep[2]);
  zd Yc = one - e_iqc;
  zd sc = (fabs(Yc.y) > eps || fabs(Yc.x) > eps) ? Xc / Yc : zd(a.rep[2], 0.0);
  sc = cpow_call(e_iqc, (1.0 - a.rep[2]) / 2.0) * sc;

  zd t3 = m[0] * a.center[0] + m[1] * a.center[1] + m[2] * a.center[2];
  t3 = cexp_call(zd(-t3.y, t3.x));
  return t3 * sa * sb * sc;
}

// sf_lattice_eval for a quad of lanes that hold the four DWBA blocks of one q-point, when the
// a- and b-direction factors do not depend on the block: m[0] and m[1] free of qz (the
// rotation's first two rows have no z entry) and a.la[2] == 0 (the b factor squares lb[2]
// instead of using qz, as the reference does).  Even lanes evaluate the a factor, odd lanes
// the b factor, on one code path: 1 - cpow(e, N) and 1 - cexp(i q.b N) are both
// 1 - exp(A) (cos B, sin B), with (A, B) = N log e (cpow_std's polar form; a positive real e
// takes its real pow) or i q.b N.  The lane pair then swaps factors, and every lane forms
// t3 * sa * sb * sc in the reference's order, so each value is the one sf_lattice_eval
// gives.  All 32 lanes of the warp must call it together.
__device__ __forceinline__ zd sf_lattice_eval_paired(const SfLat& a, const zd* m, bool odd) {
  const double eps = DBL_EPSILON;
  const zd one(1.0, 0.0);
  const double N = odd ? a.rep[1] : a.rep[0];
  const zd iq = odd ? times_i(m[0] * a.lb[0] + m[1] * a.lb[1] + a.lb[2] * a.lb[2])
                    : times_i(m[0] * a.la[0] + m[1] * a.la[1] + m[2] * a.la[2]);
  const zd e = cexp_call(iq);
  zd X;
  if (!odd && e.y == 0.0 && e.x > 0.0) {
    X = one - zd(pow(e.x, N), 0.0);
  } else {
    zd arg;
    if (odd) {
      arg = iq * N;
    } else {
      const zd t = clog_(e);
      arg = zd(N * t.x, N * t.y);
    }
    const double r = exp(arg.x);
    double s, c;
    sincos(arg.y, &s, &c);
    X = one - zd(r * c, r * s);
  }
  const zd Y = one - e;
  zd f = (fabs(Y.y) > eps || fabs(Y.x) > eps) ? X / Y : zd(N, 0.0);
  f = cpow_call(e, (1.0 - N) / 2.0) * f;
  const zd g(__shfl_xor_sync(0xffffffffu, f.x, 1), __shfl_xor_sync(0xffffffffu, f.y, 1));
  const zd sa = odd ? g : f, sb = odd ? f : g;

  zd e_iqc = cexp_call(times_i(m[0] * a.lc[0] + m[1] * a.lc[1] + m[2] * a.lc[2]));
  zd Xc = one - cpow_call(e_iqc, a.rep[2]);
  zd Yc = one - e_iqc;
  zd sc = (fabs(Yc.y) > eps || fabs(Yc.x) > eps) ? Xc / Yc : zd(a.rep[2], 0.0);
  sc = cpow_call(e_iqc, (1.0 - a.rep[2]) / 2.0) * sc;

  zd t3 = m[0] * a.center[0] + m[1] * a.center[1] + m[2] * a.center[2];
  t3 = cexp_call(zd(-t3.y, t3.x));
  return t3 * sa * sb * sc;
}

}  // namespace hgx

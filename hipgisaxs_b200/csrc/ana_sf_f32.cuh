// FP32-compensated bodies of the fused grain kernel (hig_sim.cu) for a real rotated q (grids
// whose DWBA qz blocks are real: a vacuum particle layer): the cylinder, sphere and box form
// factors and the lattice structure factor of the reference's formulas, with every phase
// formed and range-reduced in FP64 and only the transcendental of the reduced argument (and
// the sums) in FP32.  Grids with complex qz keep the FP64 bodies of ana_sf.cuh.
//
// Lattice structure factor (src/sf/sf.cpp:164-246): for a real angle theta the reference's
// principal-branch expression
//   pow(e, (1 - N)/2) (1 - pow(e, N)) / (1 - e),  e = e^{i theta}
// equals sin(N theta_r / 2) / sin(theta_r / 2) with theta_r the principal angle of e in
// (-pi, pi]; on the b axis the numerator takes exp(i N theta) with the unreduced theta,
// which for a non-integer N adds the phase e^{i pi k (N - 1)}, theta = theta_r + 2 pi k.
// N is returned where the reference's guard |1 - e| <= eps takes N.
#pragma once

#include "ana_sf.cuh"
#include "turns.cuh"

namespace hgx {

constexpr double INV_2PI_A = 0.15915494309189533576888376337251;

struct cf {
  float x, y;
};
__device__ __forceinline__ cf cmul(cf a, cf b) { return cf{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__device__ __forceinline__ cf cscale(cf a, float s) { return cf{a.x * s, a.y * s}; }
__device__ __forceinline__ cf cadd(cf a, cf b) { return cf{a.x + b.x, a.y + b.y}; }

// e^{2 pi i u} of a phase in turns (FP64), reduced exactly (FP64 add pipe) before the FP32
// sincospi (FMA pipe)
__device__ __forceinline__ cf expi_turns(double u) {
  u -= round_fp64(u);
  float s, c;
  sincospi_f32((float)(2.0 * u), &s, &c);
  return cf{c, s};
}
// e^{i ph}, ph in radians (FP64)
__device__ __forceinline__ cf expi_f(double ph) { return expi_turns(ph * INV_2PI_A); }

// sin(x)/x (hig::sinc) given sin x from expi_f; the Taylor form near 0
__device__ __forceinline__ float sinc_from(double x, float sinx) {
  if (fabs(x) > 1e-2) return sinx / (float)x;
  const float x2 = (float)(x * x);
  return 1.f - x2 * (1.f / 6.f - x2 * (1.f / 120.f));
}

// with_phase of ana_sf.cuh: v e^{i m.tv}, not evaluated at the origin
__device__ __forceinline__ cf with_phase_f(cf v, const double* m, const double* tv) {
  if (tv[0] == 0.0 && tv[1] == 0.0 && tv[2] == 0.0) return v;
  return cmul(v, expi_f(m[0] * tv[0] + m[1] * tv[1] + m[2] * tv[2]));
}

// an integer-valued k (|k| < 2^51) is odd
__device__ __forceinline__ bool odd_integer(double k) { return 0.5 * k != round_fp64(0.5 * k); }

__device__ __forceinline__ float sinpi_f32(float x) {  // |x| <= 1
  float s, c;
  sincospi_f32(x, &s, &c);
  return s;
}

// sin(pi n u) / sin(pi u) for an integer n >= 1 at an unreduced u (FP64): the sum of
// e^{2 pi i u (j - (n-1)/2)} over j = 0 .. n-1.  u = k + t with |t| <= 1/2 exactly (FP64); the
// value is (-1)^(k(n-1)) times the same at t; near t = 0 (|pi n t| < 1/2) the series
// n [1 - (n^2-1) x^2/6 + (n^2-1)(3n^2-7) x^4/360 - (n^2-1)(3n^4-18n^2+31) x^6/15120], x = pi t
// (the next term is below 1e-8 of n), elsewhere the two sines with n t reduced modulo 2 in FP64.
__device__ __forceinline__ float dirichlet_sum_f32(double u, int n) {
  const double k = round_fp64(u), t = u - k;
  const bool flip = ((n - 1) & 1) && odd_integer(k);
  const float nf = (float)n, x = 3.14159265358979f * (float)t;
  float r;
  if (fabsf(nf * x) < 0.5f) {
    const float n2 = nf * nf, x2 = x * x, a = n2 - 1.0f;
    r = nf * (1.0f - x2 * (a * (1.0f / 6.0f) -
                           x2 * (a * (3.0f * n2 - 7.0f) * (1.0f / 360.0f) -
                                 x2 * a * ((3.0f * n2 - 18.0f) * n2 + 31.0f) * (1.0f / 15120.0f))));
  } else {
    const double v = (double)n * t;
    r = sinpi_f32((float)(v - 2.0 * round_fp64(0.5 * v))) / sinpi_f32((float)t);
  }
  return flip ? -r : r;
}

// The height sum of the cylinder, sum_j h_j sinc(qz h_j/2) e^{i qz h_j/2} over its samples
// (unweighted, as the reference sums them).  Each term is (e^{i qz h_j} - 1)/(i qz); when the
// samples are evenly stepped, h_j = h_0 + j d (the reference's distributions), the
// exponentials sum to e^{i qz h_mid} sin(n qz d/2)/sin(qz d/2), so the sum costs one complex
// exponential, two sines and a division instead of n of each.  Where |qz| h_max < 1/2 the
// difference from n would cancel: there, and for other samples, the per-sample sum.
__device__ __forceinline__ cf cyl_height_sum_f32(const Dist& Z, double qz) {
  const int n = Z.n;
  if (Z.prog && fabs(qz) * fmax(fabs(Z.v[0]), fabs(Z.v[n - 1])) >= 0.5) {
    const double d = (Z.v[n - 1] - Z.v[0]) / (n - 1);
    const float D = dirichlet_sum_f32(qz * d * INV_2PI_A, n);
    const cf e = expi_f(qz * 0.5 * (Z.v[0] + Z.v[n - 1]));
    const float re = e.x * D - (float)n, im = e.y * D, iq = (float)(1.0 / qz);
    return cf{im * iq, -re * iq};
  }
  cf gh{0.f, 0.f};
  for (int i = 0; i < n; ++i) {
    const double h = Z.v[i], x = qz * 0.5 * h;
    const cf e = expi_f(x);
    gh = cadd(gh, cscale(e, sinc_from(x, e.y) * (float)h));
  }
  return gh;
}

// (sin x - x cos x) / x^3 of the sphere, by its series below x = 0.5 (where the difference
// cancels in FP32)
__device__ __forceinline__ float sphere_kernel_f(double x) {
  if (x < 0.5) {
    const float x2 = (float)(x * x);
    return 1.f / 3.f - x2 * (1.f / 30.f - x2 * (1.f / 840.f - x2 * (1.f / 45360.f - x2 * (1.f / 3991680.f))));
  }
  const cf e = expi_f(x);
  return (e.y - (float)x * e.x) / (float)(x * x * x);
}

// The analytic form factor of shape `a` (SHAPE: cylinder, sphere or box) at the real rotated
// q (m) translated by tv: ff_analytic_eval of ana_sf.cuh in FP32C.
template <int SHAPE>
__device__ __forceinline__ cf ff_analytic_f32c(const AnaShape& a, const double* m, const double* tv) {
  const Dist& X = a.d[0];
  const Dist& Y = a.d[1];
  const Dist& Z = a.d[2];
  cf out{0.f, 0.f};
  if (SHAPE == SH_CYLINDER) {  // ff_ana_cylinder.cpp:34-42,100-117 (unweighted)
    const double qpar = sqrt(m[0] * m[0] + m[1] * m[1]);
    float fr = 0.f;
    for (int i = 0; i < X.n; ++i) {
      const double r = X.v[i], x = qpar * r;
      if (x * x > CUTINY_REF) fr += (float)(2. * PI_REF * r * r) * (j1f((float)x) / (float)x);
    }
    const cf gh = cyl_height_sum_f32(Z, m[2]);
    out = with_phase_f(cscale(gh, fr), m, tv);
  } else if (SHAPE == SH_SPHERE) {  // ff_ana_sphere.cpp:33-45,95-107 (weighted)
    const double q = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    cf acc{0.f, 0.f};
    if (q >= 2.2250738585072014e-308)
      for (int i = 0; i < X.n; ++i) {
        const double R = X.v[i];
        const float c0 = sphere_kernel_f(q * R) * (float)(4. * PI_REF * R * R * R * X.w[i]);
        acc = cadd(acc, cscale(expi_f(m[2] * R), c0));
      }
    out = with_phase_f(acc, m, tv);
  } else if (SHAPE == SH_BOX) {  // ff_ana_box.cpp:35-42,96-125 (weighted)
    float sx = 0.f, sy = 0.f;
    cf sz{0.f, 0.f};
    for (int i = 0; i < X.n; ++i) {
      const double x = m[0] * 0.5 * X.v[i];
      sx += sinc_from(x, expi_f(x).y) * (float)(X.v[i] * X.w[i]);
    }
    for (int i = 0; i < Y.n; ++i) {
      const double x = m[1] * 0.5 * Y.v[i];
      sy += sinc_from(x, expi_f(x).y) * (float)(Y.v[i] * Y.w[i]);
    }
    for (int i = 0; i < Z.n; ++i) {
      const double x = m[2] * 0.5 * Z.v[i];
      const cf e = expi_f(x);
      sz = cadd(sz, cscale(e, sinc_from(x, e.y) * (float)(Z.v[i] * Z.w[i])));
    }
    out = with_phase_f(cscale(sz, sx * sy), m, tv);
  }
  return out;
}

// The quad of four lanes (one per DWBA block) of the fused grain kernel: the sum of v over the
// quad, the same bits in every lane (an xor butterfly of commutative adds).
__device__ __forceinline__ float quad_sum(float v) {
  v += __shfl_xor_sync(0xffffffffu, v, 1);
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  return v;
}

// ff_analytic_f32c for a quad whose rotated in-plane q (m[0], m[1]) is the same in its four
// lanes (the element's rotation keeps qz out of them): what depends on the in-plane q only - the
// cylinder's radial sum, the box's x and y sums - is split among the lanes (lane k takes the
// samples k, k + 4, ...) and summed by quad_sum; the qz parts stay per lane.  Every lane of the
// warp calls it (shuffles); the sphere, whose |q| involves qz, keeps ff_analytic_f32c.
template <int SHAPE>
__device__ __forceinline__ cf ff_analytic_f32c_quad(const AnaShape& a, const double* m, const double* tv, int k) {
  const Dist& X = a.d[0];
  const Dist& Y = a.d[1];
  const Dist& Z = a.d[2];
  if (SHAPE == SH_CYLINDER) {
    const double qpar = sqrt(m[0] * m[0] + m[1] * m[1]);
    float fr = 0.f;
    for (int i = k; i < X.n; i += 4) {
      const double r = X.v[i], x = qpar * r;
      if (x * x > CUTINY_REF) fr += (float)(2. * PI_REF * r * r) * (j1f((float)x) / (float)x);
    }
    fr = quad_sum(fr);
    const cf gh = cyl_height_sum_f32(Z, m[2]);
    return with_phase_f(cscale(gh, fr), m, tv);
  } else if (SHAPE == SH_BOX) {
    float sx = 0.f, sy = 0.f;
    for (int i = k; i < X.n; i += 4) {
      const double x = m[0] * 0.5 * X.v[i];
      sx += sinc_from(x, expi_f(x).y) * (float)(X.v[i] * X.w[i]);
    }
    for (int i = k; i < Y.n; i += 4) {
      const double x = m[1] * 0.5 * Y.v[i];
      sy += sinc_from(x, expi_f(x).y) * (float)(Y.v[i] * Y.w[i]);
    }
    sx = quad_sum(sx);
    sy = quad_sum(sy);
    cf sz{0.f, 0.f};
    for (int i = 0; i < Z.n; ++i) {
      const double x = m[2] * 0.5 * Z.v[i];
      const cf e = expi_f(x);
      sz = cadd(sz, cscale(e, sinc_from(x, e.y) * (float)(Z.v[i] * Z.w[i])));
    }
    return with_phase_f(cscale(sz, sx * sy), m, tv);
  }
  return ff_analytic_f32c<SHAPE>(a, m, tv);
}

// sin(N theta_r / 2) / sin(theta_r / 2) on the principal angle theta_r of e^{i theta}
__device__ __forceinline__ float dirichlet_principal(double theta, double N) {
  if (N == 1.0) return 1.f;
  double t = theta * INV_2PI_A;
  t -= round_fp64(t);
  if (t == 0.0) return (float)N;
  double v = N * t;
  const double k = round_fp64(v);
  v -= k;
  const float num = odd_integer(k) ? -sinpi_f32((float)v) : sinpi_f32((float)v);
  return num / sinpi_f32((float)t);
}

// the b-axis factor: e^{i pi k (N - 1)} sin(N theta / 2) / sin(theta / 2)
__device__ __forceinline__ cf dirichlet_b(double theta, double N) {
  if (N == round_fp64(N)) return cf{dirichlet_principal(theta, N), 0.f};
  const double u = theta * INV_2PI_A;
  const double k = round_fp64(u), t = u - k;
  if (t == 0.0) return cf{(float)N, 0.f};
  double v = N * u;
  const double kv = round_fp64(v);
  v -= kv;
  const float num = odd_integer(kv) ? -sinpi_f32((float)v) : sinpi_f32((float)v);
  const float den = odd_integer(k) ? -sinpi_f32((float)t) : sinpi_f32((float)t);
  return cscale(expi_turns(k * (N - 1.0) * 0.5), num / den);
}

// sf_lattice_eval of ana_sf.cuh for a real rotated q, FP32C.  The b angle keeps the
// reference's lb[2] * lb[2] term (src/sf/sf.cpp:212).
__device__ __forceinline__ cf sf_lattice_f32c(const SfLat& L, const double* m) {
  const double ta = m[0] * L.la[0] + m[1] * L.la[1] + m[2] * L.la[2];
  const double tb = m[0] * L.lb[0] + m[1] * L.lb[1] + L.lb[2] * L.lb[2];
  const double tc = m[0] * L.lc[0] + m[1] * L.lc[1] + m[2] * L.lc[2];
  const float sa = dirichlet_principal(ta, L.rep[0]);
  const cf sb = dirichlet_b(tb, L.rep[1]);
  const float sc = dirichlet_principal(tc, L.rep[2]);
  const cf t3 = expi_f(m[0] * L.center[0] + m[1] * L.center[1] + m[2] * L.center[2]);
  return cmul(t3, cscale(sb, sa * sc));
}

// sf_lattice_f32c for a quad whose rotated in-plane q is the same in its four lanes, with an
// in-plane a vector and an integer b repetition: the a- and b-axis factors do not depend on
// the block, so the even lanes evaluate the a factor and the odd lanes the b factor (the same
// code on other arguments) and a shuffle exchanges them; the c factor and the centre phase
// stay per lane.  Every lane of the warp calls it.
__device__ __forceinline__ cf sf_lattice_f32c_paired(const SfLat& L, const double* m, int k) {
  const bool odd = (k & 1) != 0;
  const double th = odd ? m[0] * L.lb[0] + m[1] * L.lb[1] + L.lb[2] * L.lb[2]
                        : m[0] * L.la[0] + m[1] * L.la[1] + m[2] * L.la[2];
  const float own = dirichlet_principal(th, odd ? L.rep[1] : L.rep[0]);
  const float other = __shfl_xor_sync(0xffffffffu, own, 1);
  const float sa = odd ? other : own, sb = odd ? own : other;
  const double tc = m[0] * L.lc[0] + m[1] * L.lc[1] + m[2] * L.lc[2];
  const float sc = dirichlet_principal(tc, L.rep[2]);
  const cf t3 = expi_f(m[0] * L.center[0] + m[1] * L.center[1] + m[2] * L.center[2]);
  return cscale(t3, sb * sa * sc);
}

}  // namespace hgx

// Tangents (directional derivatives) of the analytic form factors of cylinders, spheres and
// boxes and of the lattice structure factor, for a real rotated q (grids whose qz blocks are
// real): given the change dm of the rotated q vector and the changes of the shape's sampled
// dimensions and weights, of the element's location, of the lattice vectors and of the
// grain's centre, each returns the change of the value that ana_sf.cuh evaluates.  They are
// the derivatives of the reference's formulas (cited at each function), written out by hand:
//   cylinder  F = sum_r 2 pi r^2 J1(q r)/(q r) * sum_h sinc(qz h/2) h e^{i qz h/2} * e^{i m.t}
//             d/dr: 2 pi r J0(q r);  d/dq: -2 pi r^3 J2(q r)/(q r);  d/dh: e^{i qz h}
//   sphere    F = sum_R w 4 pi R^3 Phi(q R) e^{i qz R} e^{i m.t},  Phi(x) = (sin x - x cos x)/x^3,
//             Phi'(x) = sin x / x^2 - 3 Phi(x) / x
//   box       F = sx sy sz e^{i m.t},  sx = sum w L sinc(mx L/2),  sz = sum w L sinc(x) e^{i x}
//   lattice   S = e^{i m.c} S_a S_b S_c,  S_N(theta) = sin(N theta_r/2)/sin(theta_r/2) (the
//             reference's principal-branch value for an integer N), dS/dtheta closed form with
//             a series near theta_r = 0.
#pragma once

#include "ana_sf.cuh"

namespace hgx {

// d/dx (sin x / x)
__device__ __forceinline__ double dsinc_dx(double x) {
  if (fabs(x) < 1e-3) return x * (-1.0 / 3.0 + x * x / 30.0);
  double s, c;
  sincos(x, &s, &c);
  return (x * c - s) / (x * x);
}
__device__ __forceinline__ double sinc_real(double x) {
  if (fabs(x) < 1e-3) return 1.0 - x * x / 6.0 + x * x * x * x / 120.0;
  return sin(x) / x;
}

// Phi(x) = (sin x - x cos x)/x^3 and Phi'(x), series below x = 0.05
__device__ __forceinline__ void sphere_phi(double x, double* phi, double* dphi) {
  if (x < 0.05) {
    const double x2 = x * x;
    *phi = 1.0 / 3.0 - x2 * (1.0 / 30.0 - x2 * (1.0 / 840.0 - x2 / 45360.0));
    *dphi = x * (-1.0 / 15.0 + x2 * (1.0 / 210.0 - x2 / 7560.0));
    return;
  }
  double s, c;
  sincos(x, &s, &c);
  *phi = (s - x * c) / (x * x * x);
  *dphi = s / (x * x) - 3.0 * (*phi) / x;
}

// S_N(theta) and dS/dtheta on the principal angle (N = 1: 1 and 0)
__device__ __forceinline__ void dirichlet_tangent(double theta, double N, double* S, double* dS) {
  if (N == 1.0) {
    *S = 1.0;
    *dS = 0.0;
    return;
  }
  double t = theta * (1.0 / (2.0 * PI_REF));
  t -= rint(t);
  const double th = 2.0 * PI_REF * t;
  if (fabs(th) * N < 0.1) {  // series of sum_j cos(th c_j), c_j = j - (N - 1)/2
    const double n2 = N * N;
    const double s2 = N * (n2 - 1.0) / 12.0;
    const double s4 = N * (n2 - 1.0) * (3.0 * n2 - 7.0) / 240.0;
    const double s6 = N * (n2 - 1.0) * (3.0 * n2 * n2 - 18.0 * n2 + 31.0) / 1344.0;
    const double x2 = th * th;
    *S = N - x2 * s2 / 2.0 + x2 * x2 * s4 / 24.0 - x2 * x2 * x2 * s6 / 720.0;
    *dS = -th * s2 + th * x2 * s4 / 6.0 - th * x2 * x2 * s6 / 120.0;
    return;
  }
  double sn, cn, s1, c1;
  sincospi(N * t, &sn, &cn);
  sincospi(t, &s1, &c1);
  *S = sn / s1;
  *dS = (N * cn * s1 - sn * c1) / (2.0 * s1 * s1);
}

// d(value * e^{i m.tv}) = e^{i m.tv} (dvalue + i (dm.tv + m.dtv) value); the phase is not
// evaluated at the origin (as with_phase)
__device__ __forceinline__ zd phase_tangent(zd v, zd dv, const double* m, const double* dm,
                                            const double* tv, const double* dtv) {
  const double dph = dm[0] * tv[0] + dm[1] * tv[1] + dm[2] * tv[2] + m[0] * dtv[0] + m[1] * dtv[1] +
                     m[2] * dtv[2];
  const zd t = dv + zd(-v.y * dph, v.x * dph);
  if (tv[0] == 0.0 && tv[1] == 0.0 && tv[2] == 0.0) return t;
  return t * expi(m[0] * tv[0] + m[1] * tv[1] + m[2] * tv[2]);
}

// The change of ff_analytic_eval<SHAPE>(a, m, tv) for real m (SHAPE: cylinder, sphere, box);
// da: the changes of a's sampled values and weights (same counts).
template <int SHAPE>
__device__ __forceinline__ zd ff_analytic_tangent(const AnaShape& a, const AnaShape& da, const double* m,
                                                  const double* dm, const double* tv, const double* dtv) {
  const Dist& X = a.d[0];
  const Dist& Y = a.d[1];
  const Dist& Z = a.d[2];
  if (SHAPE == SH_CYLINDER) {  // ff_ana_cylinder.cpp:34-42,100-117 (unweighted)
    const double q = sqrt(m[0] * m[0] + m[1] * m[1]);
    const double dq = q > 0.0 ? (m[0] * dm[0] + m[1] * dm[1]) / q : 0.0;
    double fr = 0.0, dfr = 0.0;
    for (int i = 0; i < X.n; ++i) {
      const double r = X.v[i], x = q * r;
      if (x * x > CUTINY_REF) {
        const double J1 = j1(x), J0 = j0(x), J2 = 2.0 * J1 / x - J0;
        fr += 2.0 * PI_REF * r * r * J1 / x;
        dfr += 2.0 * PI_REF * r * J0 * da.d[0].v[i] - 2.0 * PI_REF * r * r * r * J2 / x * dq;
      }
    }
    zd gh(0, 0), dgh(0, 0);
    for (int i = 0; i < Z.n; ++i) {
      const double h = Z.v[i], x = m[2] * 0.5 * h;
      const zd e = expi(x);
      const double s = sinc_real(x);
      gh += e * (s * h);
      dgh += expi(2.0 * x) * da.d[2].v[i] + (e * zd(dsinc_dx(x), s)) * (0.5 * h * h * dm[2]);
    }
    const zd v = gh * fr;
    const zd dv = gh * dfr + dgh * fr;
    return phase_tangent(v, dv, m, dm, tv, dtv);
  } else if (SHAPE == SH_SPHERE) {  // ff_ana_sphere.cpp:33-45,95-107 (weighted)
    const double q = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    zd v(0, 0), dv(0, 0);
    if (q >= 2.2250738585072014e-308) {
      const double dq = (m[0] * dm[0] + m[1] * dm[1] + m[2] * dm[2]) / q;
      for (int i = 0; i < X.n; ++i) {
        const double R = X.v[i], w = X.w[i], dR = da.d[0].v[i], dw = da.d[0].w[i];
        double phi, dphi;
        sphere_phi(q * R, &phi, &dphi);
        const double f0 = 4.0 * PI_REF * R * R * R;
        const zd e = expi(m[2] * R);
        const double amp = w * f0 * phi;
        const double damp = dw * f0 * phi + w * (12.0 * PI_REF * R * R * phi + f0 * dphi * q) * dR +
                            w * f0 * dphi * R * dq;
        const double dphase = R * dm[2] + m[2] * dR;
        v += e * amp;
        dv += e * zd(damp, amp * dphase);
      }
    }
    return phase_tangent(v, dv, m, dm, tv, dtv);
  } else {  // SH_BOX, ff_ana_box.cpp:35-42,96-125 (weighted)
    double sx = 0.0, dsx = 0.0, sy = 0.0, dsy = 0.0;
    for (int i = 0; i < X.n; ++i) {
      const double L = X.v[i], w = X.w[i], x = m[0] * 0.5 * L;
      const double s = sinc_real(x), ds = dsinc_dx(x);
      sx += w * L * s;
      dsx += da.d[0].w[i] * L * s + w * (s + x * ds) * da.d[0].v[i] + w * L * ds * 0.5 * L * dm[0];
    }
    for (int i = 0; i < Y.n; ++i) {
      const double L = Y.v[i], w = Y.w[i], x = m[1] * 0.5 * L;
      const double s = sinc_real(x), ds = dsinc_dx(x);
      sy += w * L * s;
      dsy += da.d[1].w[i] * L * s + w * (s + x * ds) * da.d[1].v[i] + w * L * ds * 0.5 * L * dm[1];
    }
    zd sz(0, 0), dsz(0, 0);
    for (int i = 0; i < Z.n; ++i) {
      const double L = Z.v[i], w = Z.w[i], x = m[2] * 0.5 * L;
      const zd e = expi(x);
      const double s = sinc_real(x);
      sz += e * (w * L * s);
      dsz += e * (da.d[2].w[i] * L * s) + expi(2.0 * x) * (w * da.d[2].v[i]) +
             (e * zd(dsinc_dx(x), s)) * (w * 0.5 * L * L * dm[2]);
    }
    const zd v = sz * (sx * sy);
    const zd dv = dsz * (sx * sy) + sz * (dsx * sy + sx * dsy);
    return phase_tangent(v, dv, m, dm, tv, dtv);
  }
}

// The change of sf_lattice_eval(L, m) for real m and integer repetitions; dL: the changes of
// the scaled lattice vectors and of the centre (dL.rep unused).
__device__ __forceinline__ zd sf_lattice_tangent(const SfLat& L, const SfLat& dL, const double* m,
                                                 const double* dm) {
  const double ta = m[0] * L.la[0] + m[1] * L.la[1] + m[2] * L.la[2];
  const double tb = m[0] * L.lb[0] + m[1] * L.lb[1] + L.lb[2] * L.lb[2];  // sf.cpp:212
  const double tc = m[0] * L.lc[0] + m[1] * L.lc[1] + m[2] * L.lc[2];
  const double dta = dm[0] * L.la[0] + dm[1] * L.la[1] + dm[2] * L.la[2] + m[0] * dL.la[0] +
                     m[1] * dL.la[1] + m[2] * dL.la[2];
  const double dtb = dm[0] * L.lb[0] + dm[1] * L.lb[1] + m[0] * dL.lb[0] + m[1] * dL.lb[1] +
                     2.0 * L.lb[2] * dL.lb[2];
  const double dtc = dm[0] * L.lc[0] + dm[1] * L.lc[1] + dm[2] * L.lc[2] + m[0] * dL.lc[0] +
                     m[1] * dL.lc[1] + m[2] * dL.lc[2];
  double Sa, dSa, Sb, dSb, Sc, dSc;
  dirichlet_tangent(ta, L.rep[0], &Sa, &dSa);
  dirichlet_tangent(tb, L.rep[1], &Sb, &dSb);
  dirichlet_tangent(tc, L.rep[2], &Sc, &dSc);
  const double ph = m[0] * L.center[0] + m[1] * L.center[1] + m[2] * L.center[2];
  const double dph = dm[0] * L.center[0] + dm[1] * L.center[1] + dm[2] * L.center[2] +
                     m[0] * dL.center[0] + m[1] * dL.center[1] + m[2] * dL.center[2];
  const zd t3 = expi(ph);
  const double S = Sa * Sb * Sc;
  const double dS = dSa * dta * Sb * Sc + Sa * dSb * dtb * Sc + Sa * Sb * dSc * dtc;
  return t3 * zd(dS, S * dph);
}

}  // namespace hgx

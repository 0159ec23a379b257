/*
 * TEST INFRASTRUCTURE — the CPU oracle (see hgx_oracle.h).  Never part of the product.
 *
 * FP64 restatement of the reference's CPU hot path.  Each function names the reference
 * lines it follows; the evaluation order mirrors the reference so that the compiled
 * reference (oracle/_ref) and this file agree to rounding.  C99 complex arithmetic is
 * used with the same operation order as the reference's std::complex<double> code:
 *   - complex * real scales both parts (the reference's hig::operator*, utilities.cpp:215-221);
 *   - std::pow(complex, real) follows libstdc++: a positive real base takes the real pow,
 *     otherwise polar(exp(y*log|x|), y*arg(x)) — the principal branch.
 */
#define _GNU_SOURCE
#include "hgx_oracle.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

#define PI_REF 3.141592653589793 /* PI_, include/common/constants.hpp */
#define CUTINY_REF 1.0e-13       /* CUTINY_, include/common/constants.hpp */
#define TINY_REF DBL_MIN         /* TINY_ = numeric_limits<real_t>::min() */

static inline cplx cx(double re, double im) { return CMPLX(re, im); }
static inline cplx ld(const double* p, long i) { return CMPLX(p[2 * i], p[2 * i + 1]); }
static inline void st(double* p, long i, cplx v) {
  p[2 * i] = creal(v);
  p[2 * i + 1] = cimag(v);
}
static inline cplx rs(cplx z, double s) { return CMPLX(creal(z) * s, cimag(z) * s); }
static inline cplx rdiv(cplx z, double s) { return CMPLX(creal(z) / s, cimag(z) / s); }
static inline double cnorm(cplx z) { return creal(z) * creal(z) + cimag(z) * cimag(z); }
/* libstdc++ std::pow(const complex<T>&, const T&) */
static cplx cpow_std(cplx x, double y) {
  if (cimag(x) == 0.0 && creal(x) > 0.0) return CMPLX(pow(creal(x), y), 0.0);
  cplx t = clog(x);
  double rho = exp(y * creal(t)), th = y * cimag(t);
  return CMPLX(rho * cos(th), rho * sin(th));
}
/* hig::sgn, include/utils/utilities.hpp:31-34 (sgn(0) = 1) */
static inline int sgn_ref(double a) { return a < 0 ? -1 : 1; }

int orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

/* ---------------------------------------------------------------- q-grid ---- */

/* src/model/qgrid.cpp:30-99 */
int orc_qgrid_create(int ncol, int nrow, double qmin_y, double qmin_z, double qmax_y,
                     double qmax_z, double alpha_i, double k0, double* qx, double* qy,
                     double* qz, double* alpha) {
  if (ncol < 2 || nrow < 2) return -1;
  double* al = (double*)malloc(sizeof(double) * nrow);
  double* th = (double*)malloc(sizeof(double) * ncol);
  double dq = (qmax_z - qmin_z) / (nrow - 1);
  for (int i = 0; i < nrow; ++i) {
    double qpt = qmin_z + i * dq;
    al[i] = asin(qpt / k0 - sin(alpha_i));
  }
  dq = (qmax_y - qmin_y) / (ncol - 1);
  double cos_ai = cos(alpha_i);
  double cos_af = cos(al[0]); /* first row only, :58-63 */
  for (int i = 0; i < ncol; ++i) {
    double qpt = qmin_y + i * dq;
    double kf2 = pow(qpt / k0, 2);
    double tmp = (cos_af * cos_af + cos_ai * cos_ai - kf2) / (2 * cos_af * cos_ai);
    if (tmp > 1.0) tmp = 1.0;
    th[i] = sgn_ref(qpt) * acos(tmp);
  }
  /* std::reverse(alpha_) then the pixel loop, :75-84 */
  for (int i = 0; i < nrow / 2; ++i) {
    double t = al[i];
    al[i] = al[nrow - 1 - i];
    al[nrow - 1 - i] = t;
  }
  for (int i = 0; i < nrow; ++i) {
    for (int j = 0; j < ncol; ++j) {
      double tth = th[j], alf = al[i];
      long p = (long)i * ncol + j;
      if (qx) qx[p] = k0 * (cos(alf) * cos(tth) - cos(alpha_i));
      if (qy) qy[p] = k0 * (cos(alf) * sin(tth));
      if (qz) qz[p] = k0 * (sin(alf) + sin(alpha_i));
    }
  }
  if (alpha) memcpy(alpha, al, sizeof(double) * nrow);
  free(al);
  free(th);
  return 0;
}

/* src/model/qgrid.cpp:102-127 */
int orc_qz_extended(int n, const double* qz, double k0, double alpha_i, double dn2_re,
                    double dn2_im, double* qz_ext) {
  cplx dnl = cx(dn2_re, dn2_im);
  double sin_ai = sin(alpha_i);
  double kzi_0 = -1 * k0 * sin_ai;
  cplx kzi = rs(csqrt(sin_ai * sin_ai - dnl), -1 * k0);
  for (long i = 0; i < n; ++i) {
    double kzf_0 = qz[i] + kzi_0;
    cplx kzf = rs(csqrt(kzf_0 * kzf_0 - rs(dnl, k0 * k0)), (double)sgn_ref(kzf_0));
    st(qz_ext, i, kzf - kzi);
    st(qz_ext, n + i, -kzf - kzi);
    st(qz_ext, 2L * n + i, kzf + kzi);
    st(qz_ext, 3L * n + i, -kzf + kzi);
  }
  return 0;
}

/* ------------------------------------------------------------- multilayer ---- */

/* src/model/multilayer.cpp:65-108 */
int orc_parratt(int nl, const double* one_minus_n2, const double* z, double alpha, double k0,
                int order, double* tr) {
  cplx* T = (cplx*)calloc(nl, sizeof(cplx));
  cplx* R = (cplx*)calloc(nl, sizeof(cplx));
  cplx* kz = (cplx*)calloc(nl, sizeof(cplx));
  double sina = sin(alpha);
  T[nl - 1] = cx(1.0, 0.0);
  for (int i = 0; i < nl; ++i) kz[i] = rs(csqrt(sina * sina - ld(one_minus_n2, i)), -k0);
  for (int i = nl - 2; i > -1; --i) {
    cplx pij = (kz[i] + kz[i + 1]) / (rs(kz[i], 2.0));
    cplx mij = (kz[i] - kz[i + 1]) / (rs(kz[i], 2.0));
    double zi = z[i];
    cplx exp_p = cexp(rs(cx(0.0, -1.0) * (kz[i + 1] + kz[i]), zi));
    cplx exp_m = cexp(rs(cx(0.0, -1.0) * (kz[i + 1] - kz[i]), zi));
    cplx a00 = pij * exp_m;
    cplx a01 = mij * conj(exp_p);
    cplx a10 = mij * exp_p;
    cplx a11 = pij * conj(exp_m);
    T[i] = a00 * T[i + 1] + a01 * R[i + 1];
    R[i] = a10 * T[i + 1] + a11 * R[i + 1];
  }
  cplx t0 = T[0];
  for (int i = 0; i < nl; ++i) {
    T[i] /= t0;
    R[i] /= t0;
  }
  st(tr, 0, T[order]);
  st(tr, 1, R[order]);
  free(T);
  free(R);
  free(kz);
  return 0;
}

/* Builds the reference's layer stack (MultiLayer::init, multilayer.cpp:29-58):
 * vacuum first, user layers by ascending order, substrate (order -1) last. */
static int build_stack(int nlayers, const double* delta, const double* beta,
                       const double* thickness, const int* order, double** om_out,
                       double** z_out) {
  int nl = 0;
  double* om = (double*)calloc(2 * (nlayers + 2), sizeof(double));
  double* th = (double*)calloc(nlayers + 2, sizeof(double));
  double* z = (double*)calloc(nlayers + 2, sizeof(double));
  /* vacuum */
  om[0] = 0;
  om[1] = 0;
  th[0] = 0;
  nl = 1;
  /* user layers sorted by order (std::map<int, Layer>), substrate excluded */
  int* idx = (int*)malloc(sizeof(int) * (nlayers > 0 ? nlayers : 1));
  int nu = 0, sub = -1;
  for (int i = 0; i < nlayers; ++i) {
    if (order[i] == -1) {
      sub = i;
    } else {
      idx[nu++] = i;
    }
  }
  for (int a = 1; a < nu; ++a) { /* insertion sort by order */
    int v = idx[a], b = a - 1;
    while (b >= 0 && order[idx[b]] > order[v]) {
      idx[b + 1] = idx[b];
      --b;
    }
    idx[b + 1] = v;
  }
  for (int a = 0; a < nu; ++a) {
    int i = idx[a];
    om[2 * nl] = 2 * delta[i];
    om[2 * nl + 1] = 2 * beta[i];
    th[nl] = thickness[i];
    ++nl;
  }
  /* substrate (a default Layer when none was given) */
  if (sub >= 0) {
    om[2 * nl] = 2 * delta[sub];
    om[2 * nl + 1] = 2 * beta[sub];
    th[nl] = thickness[sub];
  }
  ++nl;
  double zz = 0;
  z[0] = 0;
  for (int i = 1; i < nl; ++i) {
    zz -= th[i];
    z[i] = zz;
  }
  free(idx);
  free(th);
  *om_out = om;
  *z_out = z;
  return nl;
}

/* src/model/multilayer.cpp:110-155 */
int orc_propagation_coeffs(int nlayers, const double* delta, const double* beta,
                           const double* thickness, const int* order, double k0,
                           double alpha_i, int particle_order, int nrow, int ncol,
                           const double* alpha, double* fc) {
  if (particle_order == -1) return -1;
  double *om, *z;
  int nl = build_stack(nlayers, delta, beta, thickness, order, &om, &z);
  double tr[4];
  orc_parratt(nl, om, z, alpha_i, k0, particle_order, tr);
  cplx Ti = ld(tr, 0), Ri = ld(tr, 1);
  cplx* Tf = (cplx*)calloc(nrow, sizeof(cplx));
  cplx* Rf = (cplx*)calloc(nrow, sizeof(cplx));
#pragma omp parallel for
  for (int i = 0; i < nrow; ++i) {
    if (alpha[i] > 0) {
      double t4[4];
      orc_parratt(nl, om, z, alpha[i], k0, particle_order, t4);
      Tf[i] = ld(t4, 0);
      Rf[i] = ld(t4, 1);
    }
  }
  long n = (long)nrow * ncol;
#pragma omp parallel for
  for (long i = 0; i < n; ++i) {
    long j = i / ncol;
    st(fc, i, Ti * conj(Tf[j]));
    st(fc, i + n, Ti * conj(Rf[j]));
    st(fc, i + 2 * n, Ri * conj(Tf[j]));
    st(fc, i + 3 * n, Ri * conj(Rf[j]));
  }
  free(Tf);
  free(Rf);
  free(om);
  free(z);
  return 0;
}

/* ---------------------------------------------------------------- rotation ---- */

void orc_rot_axis(int axis, double a, double* d) {
  double c = cos(a), s = sin(a);
  static const double eye[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  memcpy(d, eye, sizeof(eye));
  switch (axis) {
    case 0:
      d[4] = c; d[5] = -s; d[7] = s; d[8] = c;
      break;
    case 1:
      d[0] = c; d[2] = -s; d[6] = s; d[8] = c;
      break;
    case 2:
      d[0] = c; d[1] = -s; d[3] = s; d[4] = c;
      break;
    default:
      break;
  }
}

void orc_rot_mul(const double* a, const double* b, double* out) {
  double r[9] = {0};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) r[i * 3 + j] += a[i * 3 + k] * b[j + 3 * k];
  memcpy(out, r, sizeof(r));
}

/* RotMatrix_t::rotate(real x, real y, complex z), include/numerics/matrix.hpp:123-130 */
static inline void rotate(const double* d, double x, double y, cplx z, cplx* m) {
  m[0] = d[0] * x + d[1] * y + rs(z, d[2]);
  m[1] = d[3] * x + d[4] * y + rs(z, d[5]);
  m[2] = d[6] * x + d[7] * y + rs(z, d[8]);
}

/* ---------------------------------------------------------- numeric FF ---- */

/* src/ff/cpu/ff_tri_cpu.cpp:200-246 */
int orc_ff_approx_triangle(const double* sd, int ntri, int nqy, const double* qx,
                           const double* qy, int nqz, const double* qz, const double* rot9,
                           double* ff) {
  if (ntri < 1) return 0;
#pragma omp parallel for schedule(static)
  for (int iz = 0; iz < nqz; ++iz) {
    int iy = iz % nqy;
    cplx acc = 0;
    cplx m[3];
    rotate(rot9, qx[iy], qy[iy], ld(qz, iz), m);
    double q2 = cnorm(m[0]) + cnorm(m[1]) + cnorm(m[2]);
    for (int t = 0; t < ntri; ++t) {
      const double* p = sd + 8L * t;
      double s = p[0], nx = p[1], ny = p[2], nz = p[3], x = p[4], y = p[5], z = p[6];
      cplx qn = rs(m[0], nx) + rs(m[1], ny) + rs(m[2], nz);
      cplx qt = rs(m[0], x) + rs(m[1], y) + rs(m[2], z);
      cplx nj = cx(0.0, -1.0), np = cx(0.0, 1.0);
      acc += rdiv(rs(nj * qn, s) * cexp(np * qt), q2);
    }
    st(ff, iz, acc);
  }
  return ntri;
}

/* FormFactorTriangle, src/ff/cpu/ff_tri_cpu.cpp:46-153: the exact Fourier transform of one
 * triangle (vertices v1, v2, v3) at the rotated q-vector m, reduced to edges and vertices. */
static double vabs3(const double* v) {
  double n = 0.;
  for (int i = 0; i < 3; ++i) n += v[i] * v[i];
  return sqrt(n);
}
static void vcross3(const double* u, const double* v, double* w) {
  w[0] = u[1] * v[2] - u[2] * v[1];
  w[1] = u[2] * v[0] - u[0] * v[2];
  w[2] = u[0] * v[1] - u[1] * v[0];
}
static cplx cdot3(const cplx* m, const double* v) {
  cplx r = 0;
  for (int i = 0; i < 3; ++i) r += rs(m[i], v[i]);
  return r;
}
static cplx ff_triangle_exact(const cplx* m, const double* tri) {
  const cplx unitc = cx(0.0, 1.0), n_unitc = cx(0.0, -1.0);
  cplx ff = 0;
  double q_sqr = 0.;
  for (int i = 0; i < 3; ++i) q_sqr += cnorm(m[i]);
  const double* vertex[3] = {tri, tri + 3, tri + 6};
  double edge[3][3];
  for (int i = 0; i < 3; ++i) {
    edge[0][i] = vertex[1][i] - vertex[0][i];
    edge[1][i] = vertex[2][i] - vertex[1][i];
    edge[2][i] = vertex[0][i] - vertex[2][i];
  }
  double n_t[3];
  vcross3(edge[0], edge[1], n_t);
  double nabs = vabs3(n_t);
  double t_area = 0.5 * nabs;
  for (int i = 0; i < 3; ++i) n_t[i] = n_t[i] / nabs;
  cplx q_dot_nt = cdot3(m, n_t);
  double proj_tq = q_sqr - cnorm(q_dot_nt);
  if (fabs(proj_tq) < TINY_REF) {  /* case 1 */
    cplx q_dot_v = cdot3(m, vertex[0]);
    return rdiv(rs(unitc * q_dot_nt, t_area), q_sqr) * cexp(n_unitc * q_dot_v);
  }
  for (int e = 0; e < 3; ++e) {
    double n_e[3];
    vcross3(edge[e], n_t, n_e);
    double ea = vabs3(n_e);
    for (int i = 0; i < 3; ++i) n_e[i] = n_e[i] / ea;
    cplx q_dot_ne = cdot3(m, n_e);
    double proj_eq = proj_tq - cnorm(q_dot_ne);
    if (fabs(proj_eq) < TINY_REF) {  /* case 2 */
      cplx q_dot_v = cdot3(m, vertex[e]);
      double f0 = vabs3(edge[e]) / (q_sqr * proj_tq);
      cplx c0 = -q_dot_nt * q_dot_ne;
      cplx c1 = cexp(n_unitc * q_dot_v);
      ff += rs(c0, f0) * c1;
    } else {  /* case 3 */
      double f0 = q_sqr * proj_tq * proj_eq;
      cplx q_dot_v = cdot3(m, vertex[e]);
      double el = vabs3(edge[e]);
      double n_v[3] = {edge[e][0] / el, edge[e][1] / el, edge[e][2] / el};
      cplx q_dot_nv = cdot3(m, n_v);
      cplx c0 = n_unitc * q_dot_nt * q_dot_ne * q_dot_nv;
      cplx c1 = cexp(n_unitc * q_dot_v);
      ff += rdiv(c0 * c1, f0);
      int ep = (e + 1) % 3;
      q_dot_v = cdot3(m, vertex[ep]);
      q_dot_nv = 0;
      for (int i = 0; i < 3; ++i) q_dot_nv -= rs(m[i], n_v[i]);
      c0 = n_unitc * q_dot_nt * q_dot_ne * q_dot_nv;
      c1 = cexp(n_unitc * q_dot_v);
      ff += rdiv(c0 * c1, f0);
    }
  }
  return ff;
}

/* NumericFormFactorC::compute_exact_triangle, src/ff/cpu/ff_tri_cpu.cpp:157-196:
 * tris: ntri x 9 doubles (v1, v2, v3, triangle_t of include/common/typedefs.hpp:102-106). */
int orc_ff_exact_triangle(const double* tris, int ntri, int nqy, const double* qx,
                          const double* qy, int nqz, const double* qz, const double* rot9,
                          double* ff) {
  if (ntri < 1) return 0;
#pragma omp parallel for schedule(static)
  for (int iz = 0; iz < nqz; ++iz) {
    int iy = iz % nqy;
    cplx m[3];
    rotate(rot9, qx[iy], qy[iy], ld(qz, iz), m);
    cplx acc = 0;
    for (int t = 0; t < ntri; ++t) acc += ff_triangle_exact(m, tris + 9L * t);
    st(ff, iz, acc);
  }
  return ntri;
}

/* src/file/objectshape_reader.cpp:275-300 */
int orc_triangle_params(const double* v1, const double* v2, const double* v3, double* s,
                        double* n, double* c) {
  c[0] = (v1[0] + v2[0] + v3[0]) / 3.0;
  c[1] = (v1[1] + v2[1] + v3[1]) / 3.0;
  c[2] = (v1[2] + v2[2] + v3[2]) / 3.0;
  double a[3] = {v2[0] - v1[0], v2[1] - v1[1], v2[2] - v1[2]};
  double b[3] = {v3[0] - v1[0], v3[1] - v1[1], v3[2] - v1[2]};
  double na = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  double nb = sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
  double dot = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
  double cr[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                  a[0] * b[1] - a[1] * b[0]};
  double nc = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
  if (nc == 0 || na == 0 || nb == 0) return 0;
  n[0] = cr[0] / nc;
  n[1] = cr[1] / nc;
  n[2] = cr[2] / nc;
  double sth = sqrt(1 - (dot / (na * nb)) * (dot / (na * nb)));
  *s = na * nb * sth / 2;
  return 1;
}

/* src/file/objectshape_reader.cpp:248-269 + src/ff/ff_num.cpp:1016-1030 */
int orc_mesh_to_shape_def(int nv, const double* verts, int nf, const int* faces,
                          double* sd) {
  int t = 0;
  for (int f = 0; f < nf; ++f) {
    int i0 = faces[3 * f], i1 = faces[3 * f + 1], i2 = faces[3 * f + 2];
    if (i0 < 0 || i1 < 0 || i2 < 0 || i0 >= nv || i1 >= nv || i2 >= nv) return -1;
    double s, n[3], c[3];
    if (!orc_triangle_params(verts + 3 * i0, verts + 3 * i1, verts + 3 * i2, &s, n, c))
      continue;
    double* p = sd + 8L * t;
    p[0] = s; p[1] = n[0]; p[2] = n[1]; p[3] = n[2];
    p[4] = c[0]; p[5] = c[1]; p[6] = c[2]; p[7] = 0.0;
    ++t;
  }
  return t;
}

/* --------------------------------------------------------- analytic FF ---- */

/* ShapeParamType / StatisticType / ShapeName, include/common/enums.hpp */
enum { P_RADIUS = 2, P_XSIZE = 3, P_YSIZE = 4, P_HEIGHT = 5, P_EDGE = 6, P_BASEANGLE = 7 };
enum { ST_NULL = 0, ST_NONE = 2, ST_GAUSSIAN = 4, ST_UNIFORM = 8 };
enum { SH_BOX = 2, SH_CUBE = 3, SH_CYLINDER = 4, SH_SPHERE = 5, SH_PRISM3 = 8, SH_PRISM6 = 9,
       SH_PYRAMID = 14 };

/* src/ff/ff_ana.cpp:235-284 */
int orc_param_distribution(int stat, double pmin, double pmax, double mean, double dev,
                           int nvalues, double* dim, double* w, int cap) {
  if (nvalues < 1) return -1;
  double maxv = pmax;
  if (pmax < pmin) pmax = pmin;
  int n = 0;
  if (nvalues > 1) {
    double step = fabs(pmax - pmin) / (nvalues - 1);
    double curr = pmin;
    do {
      if (n >= cap) return -1;
      dim[n++] = curr;
      curr += step;
    } while (curr < maxv); /* compares against param.max(), not the clamped pmax */
  } else {
    dim[n++] = pmin;
  }
  if (stat == ST_NONE || stat == ST_NULL) {
    w[0] = 1.0; /* a single weight, as the reference pushes only one */
    for (int i = 1; i < n; ++i) w[i] = 0.0; /* never read by the reference for n > 1 */
  } else if (stat == ST_UNIFORM) {
    for (int i = 0; i < n; ++i) w[i] = 1.0;
  } else if (stat == ST_GAUSSIAN) {
    if (!isfinite(mean)) mean = (dim[0] + dim[n - 1]) / 2;
    for (int i = 0; i < n; ++i)
      w[i] = exp(-1.0 * pow((dim[i] - mean), 2) / (2 * pow(dev, 2))) /
             (sqrt(2 * PI_REF) * dev);
  } else {
    return -1;
  }
  return n;
}

/* hig::sinc, include/numerics/numeric_utils.hpp:54-63 (free function) */
static cplx sinc_free(cplx x) {
  if (cabs(x) > 1.0E-14) return csin(x) / x;
  return (1. - rdiv(x * x, 6.)) + rdiv(x * x * x * x, 120.);
}
/* AnalyticFormFactor::sinc, src/ff/ff_ana.cpp:222-227 (member; used by member functions) */
static cplx sinc_member(cplx v) {
  if (fabs(creal(v)) <= 1e-14 && fabs(cimag(v)) <= 1e-14) return cx(1.0, 0.0);
  return csin(v) / v;
}
/* AnalyticFormFactor::fq_inv, src/ff/ff_ana.cpp:190-196 */
static cplx fq_inv(cplx value, double y) {
  cplx unitc = cx(0, 1.0);
  cplx temp = rs(cexp(rdiv(rs(unitc * value, y), 2.0)), 2.0) * csin(rdiv(rs(value, y), 2.0)) /
              value;
  if (cabs(temp) <= 1e-14) temp = cx(y, 0);
  return temp;
}
/* phase factor exp(i q.T) written as exp(complex(-Im, Re)) as the reference does */
static inline cplx trans_phase(const cplx* m, const double* tv) {
  cplx t = rs(m[0], tv[0]) + rs(m[1], tv[1]) + rs(m[2], tv[2]);
  return cexp(cx(-cimag(t), creal(t)));
}

/* src/ff/ff_ana_cylinder.cpp:34-42 */
static cplx ff_cylinder_one(cplx qpar, cplx qz, double radius, double height) {
  double vol = 2. * PI_REF * radius * radius * height;
  cplx sinc_val = sinc_free(rs(rs(qz, 0.5), height));
  cplx expt_val = cexp(rs(rs(cx(0, 1), 0.5) * qz, height));
  cplx t1 = rs(qpar, radius);
  cplx bess = 0;
  if (cnorm(t1) > CUTINY_REF) bess = rdiv(cx(j1(creal(t1)), 0.0) * conj(t1), cnorm(t1));
  return rs(sinc_val, vol) * expt_val * bess;
}
/* src/ff/ff_ana_sphere.cpp:33-45 */
static cplx ff_sphere_one(cplx qx, cplx qy, cplx qz, double radius) {
  cplx qval = csqrt(qx * qx + qy * qy + qz * qz);
  if (cabs(qval) < TINY_REF) return 0;
  cplx qR = rs(qval, radius);
  cplx qR3 = qR * qR * qR;
  cplx t1 = rdiv(conj(qR3), cnorm(qR3));
  cplx c0 = (csin(qR) - qR * ccos(qR)) * t1;
  cplx c1 = cexp(rs(cx(0, 1) * qz, radius));
  double f0 = 4 * PI_REF * radius * radius * radius;
  return rs(c0, f0) * c1;
}
/* src/ff/ff_ana_box.cpp:35-42 */
static cplx ff_box_one(cplx qx, cplx qy, cplx qz, double L, double W, double H) {
  double vol = L * W * H;
  cplx e = cexp(rs(rs(cx(0, 1), 0.5) * qz, H));
  cplx s = sinc_free(rs(rs(qx, 0.5), L)) * sinc_free(rs(rs(qy, 0.5), W)) *
           sinc_free(rs(rs(qz, 0.5), H));
  return rs(e, vol) * s;
}
/* src/ff/ff_ana_cube.cpp:35-42 */
static cplx ff_cube_one(cplx qx, cplx qy, cplx qz, double L) {
  double vol = L * L * L;
  cplx e = cexp(rs(rs(cx(0, 1), 0.5) * qz, L));
  cplx s = sinc_free(rs(rs(qx, 0.5), L)) * sinc_free(rs(rs(qy, 0.5), L)) *
           sinc_free(rs(rs(qz, 0.5), L));
  return rs(e, vol) * s;
}
/* src/ff/ff_ana_pyramid.cpp:35-78 (angle in degrees) */
static cplx ff_pyramid_one(cplx qx, cplx qy, cplx qz, double L, double W, double H,
                           double angle) {
  double a = angle * PI_REF / 180.;
  double tan_a = tan(a);
  if ((2 * H / L >= tan_a) || (2 * H / W >= tan_a)) return 0;
  cplx tmp = qx * qy;
  if (cabs(tmp) < 1.0E-20) return 0;
  const cplx PJ = cx(0, 1), NJ = cx(0, -1);
  cplx q1 = rs(rdiv(qx - qy, tan_a) + qz, 0.5);
  cplx q2 = rs(rdiv(qx - qy, tan_a) - qz, 0.5);
  cplx q3 = rs(rdiv(qx + qy, tan_a) + qz, 0.5);
  cplx q4 = rs(rdiv(qx + qy, tan_a) - qz, 0.5);
  cplx k1 = sinc_free(rs(q1, H)) * cexp(rs(NJ * q1, H)) + sinc_free(rs(q2, H)) * cexp(rs(PJ * q2, H));
  cplx k2 = sinc_free(rs(q1, H)) * cexp(rs(NJ * q1, H)) * NJ +
            sinc_free(rs(q2, H)) * cexp(rs(PJ * q2, H)) * PJ;
  cplx k3 = sinc_free(rs(q3, H)) * cexp(rs(NJ * q3, H)) + sinc_free(rs(q4, H)) * cexp(rs(PJ * q4, H));
  cplx k4 = sinc_free(rs(q3, H)) * cexp(rs(NJ * q3, H)) * NJ +
            sinc_free(rs(q4, H)) * cexp(rs(PJ * q4, H)) * PJ;
  cplx t1 = k1 * ccos(rs(rs(qx, L) - rs(qy, W), 0.5));
  cplx t2 = k2 * csin(rs(rs(qx, L) - rs(qy, W), 0.5));
  cplx t3 = k3 * ccos(rs(rs(qx, L) + rs(qy, W), 0.5));
  cplx t4 = k4 * csin(rs(rs(qx, L) + rs(qy, W), 0.5));
  return (H / tmp) * (t1 + t2 - t3 - t4);
}

#define MAXV 4096
typedef struct {
  double v[MAXV];
  double w[MAXV];
  int n;
} dist_t;

static int push_dist(dist_t* d, const double* p) {
  int k = orc_param_distribution((int)p[1], p[2], p[3], p[4], p[5], (int)p[6], d->v + d->n,
                                 d->w + d->n, MAXV - d->n);
  if (k < 0) return -1;
  d->n += k;
  return 0;
}

/* src/ff/ff_ana.cpp:61-161 and the per-shape files named above */
int orc_ff_analytic(int shape, int nparam, const double* params, double tau, double eta,
                    const double* tv, const double* rot9, int nqy, const double* qx,
                    const double* qy, int nqz, const double* qz, double* ff) {
  dist_t* X = (dist_t*)calloc(1, sizeof(dist_t));
  dist_t* Y = (dist_t*)calloc(1, sizeof(dist_t));
  dist_t* Z = (dist_t*)calloc(1, sizeof(dist_t));
  dist_t* B = (dist_t*)calloc(1, sizeof(dist_t));
  int rc = 0;
  /* parameter routing per shape (compute_* switch statements) */
  for (int i = 0; i < nparam && rc == 0; ++i) {
    const double* p = params + 7 * i;
    int type = (int)p[0];
    switch (shape) {
      case SH_BOX: /* ff_ana_box.cpp:54-76 */
        if (type == P_EDGE) {
          rc |= push_dist(X, p); rc |= push_dist(Y, p); rc |= push_dist(Z, p);
        } else if (type == P_XSIZE) rc |= push_dist(X, p);
        else if (type == P_YSIZE) rc |= push_dist(Y, p);
        else if (type == P_HEIGHT) rc |= push_dist(Z, p);
        break;
      case SH_CUBE: /* ff_ana_cube.cpp:47-60: only 'height' is read */
        if (type == P_HEIGHT) rc |= push_dist(X, p);
        break;
      case SH_CYLINDER: /* ff_ana_cylinder.cpp:48-70 */
        if (type == P_HEIGHT) rc |= push_dist(Z, p);
        else if (type == P_RADIUS) rc |= push_dist(X, p);
        break;
      case SH_SPHERE: /* ff_ana_sphere.cpp:50-65 */
        if (type == P_RADIUS) rc |= push_dist(X, p);
        else if (type == P_EDGE || type == P_XSIZE || type == P_YSIZE || type == P_HEIGHT)
          rc |= push_dist(Z, p);
        break;
      case SH_PRISM3: /* ff_ana_prism.cpp:37-55 */
      case SH_PRISM6: /* ff_ana_prism6.cpp:37-55 */
        if (type == P_EDGE) rc |= push_dist(X, p);
        else if (type == P_HEIGHT) rc |= push_dist(Z, p);
        break;
      case SH_PYRAMID: /* ff_ana_pyramid.cpp:84-106 */
        if (type == P_XSIZE) rc |= push_dist(X, p);
        else if (type == P_YSIZE) rc |= push_dist(Y, p);
        else if (type == P_HEIGHT) rc |= push_dist(Z, p);
        else if (type == P_BASEANGLE) rc |= push_dist(B, p);
        break;
      default:
        rc = -1;
    }
  }
  if (rc == 0) {
    int ok = 1;
    switch (shape) {
      case SH_BOX: ok = X->n && Y->n && Z->n; break;
      case SH_CUBE: ok = X->n > 0; break;
      case SH_CYLINDER: ok = X->n && Z->n; break;
      case SH_SPHERE: ok = X->n > 0; break;
      case SH_PRISM3: ok = X->n && Z->n; break;
      default: break;
    }
    if (!ok) rc = -2;
  }
  if (rc == 0) {
    const double sqrt3 = sqrt(3.0);
#pragma omp parallel for schedule(static)
    for (int iz = 0; iz < nqz; ++iz) {
      int iy = iz % nqy;
      cplx m[3];
      rotate(rot9, qx[iy], qy[iy], ld(qz, iz), m);
      cplx acc = 0, out = 0;
      switch (shape) {
        case SH_CYLINDER: { /* ff_ana_cylinder.cpp:100-117 */
          cplx qpar = csqrt(m[0] * m[0] + m[1] * m[1]);
          for (int r = 0; r < X->n; ++r)
            for (int h = 0; h < Z->n; ++h) acc += ff_cylinder_one(qpar, m[2], X->v[r], Z->v[h]);
          out = acc * trans_phase(m, tv);
          break;
        }
        case SH_SPHERE: /* ff_ana_sphere.cpp:95-107 */
          for (int r = 0; r < X->n; ++r)
            acc += rs(ff_sphere_one(m[0], m[1], m[2], X->v[r]), X->w[r]);
          out = acc * trans_phase(m, tv);
          break;
        case SH_BOX: /* ff_ana_box.cpp:96-125 */
          for (int k = 0; k < Z->n; ++k)
            for (int j = 0; j < Y->n; ++j)
              for (int i = 0; i < X->n; ++i) {
                double wg = X->w[i] * Y->w[j] * Z->w[k];
                acc += rs(ff_box_one(m[0], m[1], m[2], X->v[i], Y->v[j], Z->v[k]), wg);
              }
          out = acc * trans_phase(m, tv);
          break;
        case SH_CUBE: /* ff_ana_cube.cpp:87-107 */
          for (int i = 0; i < X->n; ++i)
            acc += rs(ff_cube_one(m[0], m[1], m[2], X->v[i]), X->w[i]);
          out = acc * trans_phase(m, tv);
          break;
        case SH_PRISM3: { /* ff_ana_prism.cpp:82-108 */
          cplx t1 = m[0] * (m[0] * m[0] - rs(m[1], 3.0) * m[1]);
          cplx t2 = m[2] + rs(rs(m[0], sin(eta)) + rs(m[1], cos(eta)), tan(tau));
          for (int l = 0; l < X->n; ++l)
            for (int h = 0; h < Z->n; ++h) {
              double L = X->v[l];
              cplx t4 = m[0] * cexp(rs(rs(cx(0, 1) * m[1], L), sqrt3));
              cplx t5 = m[0] * ccos(rs(m[0], L));
              cplx t6 = rs(cx(0, 1), sqrt3) * m[1] * csin(rs(m[0], L));
              cplx t7 = fq_inv(t2, Z->v[h]);
              cplx t8 = (t4 - t5 - t6) * t7;
              cplx t3 = rdiv(rs(m[1], L), sqrt3);
              cplx t9 = rs(cexp(cx(cimag(t3), -creal(t3))), 2.0 * sqrt3);
              acc += (t9 / t1) * t8;
            }
          out = acc * trans_phase(m, tv);
          break;
        }
        case SH_PRISM6: { /* ff_ana_prism6.cpp:80-98 */
          cplx qm = rs(rs(m[0], sin(eta)) + rs(m[1], cos(eta)), tan(tau));
          cplx t1 = ((double)4.0 * sqrt3) / (rs(m[1], 3.0) * m[1] - m[0] * m[0]);
          for (int h = 0; h < Z->n; ++h)
            for (int l = 0; l < X->n; ++l) {
              double L = X->v[l];
              cplx rmqx = rdiv(rs(m[0], L), sqrt3);
              cplx rmqy = rs(m[1], L);
              cplx t2 = rmqy * rmqy * sinc_member(rmqx) * sinc_member(rmqy);
              cplx t3 = ccos(rs(rmqx, 2.0));
              cplx t4 = ccos(rmqy) * ccos(rmqx);
              cplx t5 = t1 * (t2 + t3 - t4);
              cplx t6 = fq_inv(m[2] + qm, Z->v[h]);
              acc += t5 * t6;
            }
          out = acc * trans_phase(m, tv);
          break;
        }
        case SH_PYRAMID: { /* ff_ana_pyramid.cpp:118-139 */
          for (int i = 0; i < X->n; ++i)
            for (int j = 0; j < Y->n; ++j)
              for (int h = 0; h < Z->n; ++h)
                for (int b = 0; b < B->n; ++b) {
                  double prob = X->w[i] * Y->w[j] * Z->w[h] * B->w[b];
                  acc += rs(ff_pyramid_one(m[0], m[1], m[2], X->v[i], Y->v[j], Z->v[h], B->v[b]),
                            prob);
                }
          cplx t1 = rs(m[0], tv[0]) + rs(m[1], tv[1]) + rs(m[2], tv[2]);
          out = acc * cexp(cx(0, 1) * t1);
          break;
        }
        default:
          break;
      }
      st(ff, iz, out);
    }
  }
  free(X);
  free(Y);
  free(Z);
  free(B);
  return rc == 0 ? nqz : rc;
}

/* ------------------------------------------------------ structure factor ---- */

/* LatticeType, include/common/enums.hpp:56-65 */
enum { L_NULL = 0, L_BCC = 2, L_CUBIC = 3, L_FCC = 4, L_FCO = 5, L_HCP = 6, L_HEX = 7 };

/* src/model/structure.cpp:86-182 (ca_ = 1, gamma_ = 0 as set by Lattice::Lattice) */
int orc_lattice_vectors(int type, const char* hkl, double* a, double* b, double* c, double* t) {
  const double sqrt3 = sqrt(3.0);
  const char* h = hkl ? hkl : "100";
#define SET3(v, x, y, z) (v[0] = (x), v[1] = (y), v[2] = (z))
  SET3(t, 0, 0, 0);
  switch (type) {
    case L_CUBIC:
      if (!strcmp(h, "100")) {
        SET3(a, 1, 0, 0); SET3(b, 0, 1, 0); SET3(c, 0, 0, 1);
      } else if (!strcmp(h, "110")) {
        SET3(a, 1, 0, 0); SET3(b, 0., 1.4142, 0); SET3(c, 0., 0.7071, 0.7071);
      } else return -1;
      break;
    case L_BCC:
      if (!strcmp(h, "100")) {
        SET3(a, 1., 0., 0.); SET3(b, 0., 1., 0.); SET3(c, 0.5, 0.5, 0.5);
      } else if (!strcmp(h, "110")) {
        SET3(a, 1.0, 0.0, 0); SET3(b, 0.5, 0.7071, 0); SET3(c, 0.0, 0.7071, 0.7071);
      } else return -1;
      break;
    case L_FCC:
      if (!strcmp(h, "100")) {
        SET3(a, 0.0, 0.5, 0.5); SET3(b, 0.5, 0.0, 0.5); SET3(c, 0.5, 0.5, 0.0);
      } else if (!strcmp(h, "111")) {
        SET3(a, 1., 0., 0); SET3(b, 0.5, 0.866, -0.); SET3(c, 1., 0.5773, 0.866);
      } else return -1;
      break;
    case L_FCO:
      SET3(a, 1, 0, 0); SET3(b, 0.5, tan(0.0) / 2.0, 0); SET3(c, 0, 0, 1.0);
      SET3(t, 0.5, 0, 1.0 / 2);
      break;
    case L_HCP:
      SET3(a, 1, 0, 0); SET3(b, 0.5, 0.866, 0); SET3(c, 0.5, 0.2887, 0.8165);
      break;
    case L_HEX:
      SET3(a, 1, 0, 0); SET3(b, 0.5, sqrt3 / 2.0, 0); SET3(c, 0, 0, 1);
      break;
    default:
      return -1;
  }
#undef SET3
  return 0;
}

/* src/sf/sf.cpp:164-246 */
/* StructureFactor::paracrystal1d / paracrystal2d_cubic / paracrystal2d_hex,
 * src/sf/liquid.cpp:29-110, chosen as compute_structure_factor chooses them
 * (src/sf/sf.cpp:116-151): dims 1, or dims 2 with lattice 3 (cubic) or 7 (hex). */
int orc_sf_paracrystal(int dims, int lattice, double dx, double dy, double sx, double sy,
                       double dom, int nqy, const double* qx, const double* qy, int nqz,
                       double* sf) {
  if (dims == 1) {
    double exp_v1 = exp(-2. * dy / dom);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nqz; ++i) {
      double q = qy[i % nqy];
      double qysy = sy * q;
      double exp_v2 = exp(-1.0 * qysy * qysy);
      double exp_v3 = exp(-0.5 * qysy * qysy);
      double tmp = (1. - exp_v2 * exp_v1) / (1. - 2. * exp_v3 * exp_v1 * cos(q * dy) + exp_v2 * exp_v1);
      st(sf, i, cx(sqrt(tmp), 0.));
    }
    return nqz;
  }
  if (dims != 2 || (lattice != 3 && lattice != 7)) return -1;
  double exp_v1x = exp(-2. * dx / dom);
  double exp_v1y = exp(-2. * dy / dom);
  const double C1 = 0.5 * sqrt(3.);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nqz; ++i) {
    int j = i % nqy;
    double x = qx[j], y = qy[j];
    double qpar = sqrt(x * x + y * y);
    double s1, s2;
    if (lattice == 3) {
      double cos_vx = cos(qpar * dx);
      double cos_vy = cos(qpar * dy);
      double qxsx = qpar * sx;
      double exp_v2x = exp(-1. * qxsx * qxsx);
      double exp_v3x = exp(-0.5 * qxsx * qxsx);
      double qysy = qpar * sy;
      double exp_v2y = exp(-1. * qysy * qysy);
      double exp_v3y = exp(-0.5 * qysy * qysy);
      s1 = (1. - exp_v2x * exp_v1x) / (1. - 2. * exp_v3x * exp_v1x * cos_vx + exp_v2x * exp_v1x);
      s2 = (1. - exp_v2y * exp_v1y) / (1. - 2. * exp_v3y * exp_v1y * cos_vy + exp_v2y * exp_v1y);
    } else {
      double qpsx = qpar * sx;
      double qpsy = qpar * sy;
      double phi_x = cos(C1 * x * dx + 0.5 * y * dy);
      double phi_y = cos(y * dy);
      double exp_v2x = exp(-1. * qpsx * qpsx);
      double exp_v2y = exp(-1. * qpsy * qpsy);
      double exp_v3x = exp(-0.5 * qpsx * qpsx);
      double exp_v3y = exp(-0.5 * qpsy * qpsy);
      s1 = (1. - exp_v2x * exp_v1x) / (1. - 2. * exp_v3x * exp_v1x * phi_x + exp_v2x * exp_v1x);
      s2 = (1. - exp_v2y * exp_v1y) / (1. - 2. * exp_v3y * exp_v1y * phi_y + exp_v2y * exp_v1y);
    }
    double tmp = fabs(s1 * s2);
    st(sf, i, cx(sqrt(tmp), 0.));
  }
  return nqz;
}

/* StructureFactor::PYFcn, src/sf/liquid.cpp:112-125 */
static double py_fcn(double alpha, double beta, double gamma, double x) {
  double sinx = sin(x);
  double cosx = cos(x);
  double x2 = x * x;
  double x3 = x2 * x;
  double x4 = x3 * x;
  double x5 = x4 * x;
  double t1 = alpha * (sinx - x * cosx) / x2;
  double t2 = beta * (2 * x * sinx + (2 - x2) * cosx - 2) / x3;
  double t3 = gamma * (-x4 * cosx + 4 * ((3 * x2 - 6) * cosx + (x3 - 6 * x) * sinx + 6)) / x5;
  return (t1 + t2 + t3);
}

/* StructureFactor::percus_yevik, src/sf/liquid.cpp:127-165: dims 2 uses |q_par|, dims 3 |q|
 * with complex qz (and takes a fourth root, as the reference does); other dims leave zeros. */
int orc_sf_percus_yevick(double dia, double volf, int dims, int nqy, const double* qx,
                         const double* qy, int nqz, const double* qz, double* sf) {
  double tmp0 = pow(1 - volf, 4);
  double alpha = pow(1 + 2 * volf, 2) / tmp0;
  double beta = -6 * volf * pow(1 + 0.5 * volf, 2) / tmp0;
  double gamma = 0.5 * volf * alpha;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nqz; ++i) {
    int j = i % nqy;
    double x0 = qx[j], y0 = qy[j];
    cplx out = 0;
    if (dims == 2 || dims == 3) {
      double qval = dims == 2 ? sqrt(x0 * x0 + y0 * y0)
                              : sqrt(x0 * x0 + y0 * y0 + cnorm(ld(qz, i)));
      if (qval < 1.0E-06) {
        out = cx(alpha / 3. + beta / 4. + gamma, 0.);
      } else {
        double x = qval * dia;
        double t = dims == 2 ? 1. / (1 + 24 * volf * py_fcn(alpha, beta, gamma, x) / x)
                             : 1. / sqrt(1 + 24 * volf * py_fcn(alpha, beta, gamma, x) / x);
        out = cx(sqrt(t), 0.);
      }
    }
    st(sf, i, out);
  }
  return nqz;
}

int orc_sf_lattice(const double* abc9, const double* repet_in, const double* sc,
                   const double* center, const double* rot9, int nqy, const double* qx,
                   const double* qy, int nqz, const double* qz, double* sf) {
  double repet[3] = {repet_in[0], repet_in[1], repet_in[2]};
  for (int i = 0; i < 3; ++i)
    if (repet[i] < 1) repet[i] = 1;
  double la[3], lb[3], lc[3];
  for (int i = 0; i < 3; ++i) {
    la[i] = abc9[i] * sc[0];
    lb[i] = abc9[3 + i] * sc[1];
    lc[i] = abc9[6 + i] * sc[2];
  }
  const double eps = DBL_EPSILON;
  const cplx uc = cx(1, 0), uci = cx(0, 1);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nqz; ++i) {
    int j = i % nqy;
    cplx m[3];
    rotate(rot9, qx[j], qy[j], ld(qz, i), m);
    cplx sa, sb, sc_;
    cplx e_iqa = cexp(uci * (rs(m[0], la[0]) + rs(m[1], la[1]) + rs(m[2], la[2])));
    cplx Xa = uc - cpow_std(e_iqa, repet[0]);
    cplx Ya = uc - e_iqa;
    if (fabs(cimag(Ya)) > eps || fabs(creal(Ya)) > eps) sa = Xa / Ya;
    else sa = repet[0];
    sa = cpow_std(e_iqa, ((double)1.0 - repet[0]) / (double)2.0) * sa;

    /* b axis: lb[2]*lb[2] where lb[2]*mq[2] is meant (sf.cpp:212), kept as the reference has it */
    cplx iqb = uci * (rs(m[0], lb[0]) + rs(m[1], lb[1]) + lb[2] * lb[2]);
    cplx iqNb = rs(iqb, repet[1]);
    cplx e_iqb = cexp(iqb);
    cplx Xb = uc - cexp(iqNb);
    cplx Yb = uc - cexp(iqb);
    if (fabs(cimag(Yb)) > eps || fabs(creal(Yb)) > eps) sb = Xb / Yb;
    else sb = repet[1];
    sb = cpow_std(e_iqb, ((double)1.0 - repet[1]) / (double)2.0) * sb;

    cplx e_iqc = cexp(uci * (rs(m[0], lc[0]) + rs(m[1], lc[1]) + rs(m[2], lc[2])));
    cplx Xc = uc - cpow_std(e_iqc, repet[2]);
    cplx Yc = uc - e_iqc;
    if (fabs(cimag(Yc)) > eps || fabs(creal(Yc)) > eps) sc_ = Xc / Yc;
    else sc_ = repet[2];
    sc_ = cpow_std(e_iqc, ((double)1.0 - repet[2]) / (double)2.0) * sc_;

    cplx t3 = rs(m[0], center[0]) + rs(m[1], center[1]) + rs(m[2], center[2]);
    t3 = cexp(cx(-cimag(t3), creal(t3)));
    st(sf, i, t3 * sa * sb * sc_);
  }
  return nqz;
}

/* ----------------------------------------------------------------- DWBA ---- */

/* src/sim/hipgisaxs_main.cpp:1086-1100 */
void orc_dwba_combine(int n, const double* fc, const double* sf, const double* ff, double w,
                      double* inten) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    long i0 = i, i1 = (long)n + i, i2 = 2L * n + i, i3 = 3L * n + i;
    cplx t = ld(fc, i0) * ld(sf, i0) * ld(ff, i0) + ld(fc, i1) * ld(sf, i1) * ld(ff, i1) +
             ld(fc, i2) * ld(sf, i2) * ld(ff, i2) + ld(fc, i3) * ld(sf, i3) * ld(ff, i3);
    t = w * t;
    inten[i] += creal(t) * creal(t) + cimag(t) * cimag(t);
  }
}

/* src/sim/hipgisaxs_main.cpp:1102-1105 */
void orc_saxs_combine(int n, const double* sf, const double* ff, double w, double* inten) {
  for (int i = 0; i < n; ++i) {
    cplx t = rs(ld(sf, i), w) * ld(ff, i);
    inten[i] = creal(t) * creal(t) + cimag(t) * cimag(t);
  }
}

/* ------------------------------------------------------------ distances ---- */

/* include/analyzer/distance_functions.hpp:125-143 */
double orc_abs_diff_square(int n, const double* ref, const double* data,
                           const unsigned* mask) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) {
    double t = mask[i] * fabs(ref[i] - data[i]);
    s += t * t;
  }
  return s;
}

/* include/analyzer/distance_functions.hpp:89-103 */
void orc_residual_vector(int n, const double* ref, const double* data, const unsigned* mask,
                         double* out) {
  for (int i = 0; i < n; ++i) out[i] = mask[i] * (ref[i] - data[i]);
}

double orc_chi2(int n, const double* model, const double* counts, const unsigned* mask,
                double scale) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) {
    if (!mask || mask[i]) {
      double d = scale * model[i] - counts[i];
      double c = counts[i] > 1.0 ? counts[i] : 1.0;
      s += d * d / c;
    }
  }
  return s;
}

/* ------------------------------------------------------- post-processing ---- */

/* Convolutions::gaussian, include/numerics/convolutions.hpp:122-124 */
static double gauss1(int x, double sigma) {
  return 1.0 / (sigma * sqrt(2 * PI_REF) * exp((x * x) / (2 * sigma * sigma)));
}

/* Convolutions::convolution_gaussian_2d, include/numerics/convolutions.hpp:127-174: two
 * normalised passes (horizontal, then vertical) over the window [i - r, i + r) with
 * r = ceil(6 sigma), the weights indexed from the window's start. data: ny rows of nx. */
int orc_smear_gaussian(double* data, int nx, int ny, double sigma) {
  int r = (int)ceil(6 * sigma);
  int gn = 2 * r + 1;
  double* gmap = (double*)malloc(sizeof(double) * gn);
  double* conv = (double*)malloc(sizeof(double) * (size_t)nx * ny);
  if (!gmap || !conv) {
    free(gmap);
    free(conv);
    return -1;
  }
  for (int i = 0; i < gn; ++i) gmap[i] = gauss1(i - r, sigma);
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      double sum = 0.0, norm = 0.0;
      int ibeg = i - r > 0 ? i - r : 0;
      int iend = i + r < nx ? i + r : nx;
      for (int k = ibeg; k < iend; ++k) {
        sum += data[(size_t)j * nx + k] * gmap[k - ibeg];
        norm += gmap[k - ibeg];
      }
      conv[(size_t)j * nx + i] = norm > TINY_REF ? sum / norm : 0;
    }
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      double sum = 0.0, norm = 0.0;
      int jbeg = j - r > 0 ? j - r : 0;
      int jend = j + r < ny ? j + r : ny;
      for (int l = jbeg; l < jend; ++l) {
        sum += conv[(size_t)l * nx + i] * gmap[l - jbeg];
        norm += gmap[l - jbeg];
      }
      data[(size_t)j * nx + i] = norm > TINY_REF ? sum / norm : 0;
    }
  free(gmap);
  free(conv);
  return 0;
}

/* HipGISAXS::normalize, src/sim/hipgisaxs_main.cpp:1439-1450: (x - min)/(max - min) for
 * every element but the first; returns 0 (and changes nothing) when max - min < 1e-30. */
int orc_normalize(double* data, long n) {
  double mn = data[0], mx = data[0];
  for (long i = 1; i < n; ++i) {
    mn = data[i] < mn ? data[i] : mn;
    mx = data[i] > mx ? data[i] : mx;
  }
  double d = mx - mn;
  if (d < 1e-30) return 0;
  for (long i = 1; i < n; ++i) data[i] = (data[i] - mn) / d;
  return 1;
}

/* HipGISAXS::run_gisaxs, uncorrelated structures (src/sim/hipgisaxs_main.cpp:1278-1293,
 * 1352-1362): iratios rescaled unless they sum to 1; out[z] = sum_s I[s n + z] r_s. */
void orc_structure_sum(int ns, long n, const double* img, const double* iratios, double* out) {
  double r[256];
  double rsum = 0.0;
  for (int s = 0; s < ns && s < 256; ++s) rsum += iratios[s];
  for (int s = 0; s < ns && s < 256; ++s) r[s] = rsum != 1.0 ? iratios[s] / rsum : iratios[s];
  for (long z = 0; z < n; ++z) {
    double sum = 0.0;
    for (int s = 0; s < ns && s < 256; ++s) sum += img[(long)s * n + z] * r[s];
    out[z] = sum;
  }
}

/* The fitter's distance measures (include/analyzer/distance_functions.hpp:387-844), numbered
 * as hgx_fit_distance numbers them, in the reference's sequential order: the masked norms
 * (DistanceMeasure::norm_l1/norm_l2/vec_dot, :31-55), then the terms.  Returns the number of
 * values written to out (1, or n for the residual forms), -1 for an unknown metric. */
static double fit_tr(int metric, double x) {
  return (metric == 2 || metric == 3 || metric == 7) ? cbrt(x) : sqrt(x);
}

long orc_fit_distance(int metric, long n, const double* ref, const double* dat, const unsigned* mask,
                      double* out) {
  if (metric < 0 || metric > 7) return -1;
  const int l1 = metric == 6 || metric == 7;
  double a = 0.0, b = 0.0, c = 0.0;
  for (long i = 0; i < n; ++i) {
    const double m = mask ? (double)mask[i] : 1.0;
    const double tr = fit_tr(metric, ref[i]), td = fit_tr(metric, dat[i]);
    if (l1) {
      a += m * fabs(tr);
      b += m * fabs(td);
    } else {
      const double rr = tr * tr, dd = td * td, rd = fabs(td * tr);
      a += m * (isnan(rr) ? 0 : rr);
      b += m * (isnan(dd) ? 0 : dd);
      c += m * (isnan(rd) ? 0 : rd);
    }
  }
  const double ref_norm = l1 ? a : sqrt(a), dat_norm = l1 ? b : sqrt(b);
  const double cc = c / (dat_norm * dat_norm);
  double sum = 0.0;
  for (long i = 0; i < n; ++i) {
    const double m = mask ? (double)mask[i] : 1.0;
    const double tr = fit_tr(metric, ref[i]), td = fit_tr(metric, dat[i]);
    double t, nd, nr;
    switch (metric) {
      case 0:
        nd = td / dat_norm; nr = tr / ref_norm;
        t = m * fabs(nr - nd);
        t = isfinite(t) ? t : 0.0;
        sum += t * t;
        break;
      case 1:
        nd = cc * td; nr = tr;
        t = m * fabs(nr - nd);
        t = isfinite(t) ? t : 0.0;
        sum += t * t;
        break;
      case 2:
        nd = td / dat_norm; nr = tr / ref_norm;
        t = m * (nd - nr);
        sum += t * t;
        break;
      case 3:
        nd = cc * td; nr = tr;
        t = m * fabs(nr - nd);
        sum += t * t;
        break;
      case 4:
        nd = td / dat_norm; nr = tr / ref_norm;
        t = m * fabs(nd - nr);
        out[i] = t * t;
        break;
      case 5:
        nd = cc * td; nr = tr;
        t = m * fabs(nr - nd);
        out[i] = t * t;
        break;
      default:
        nd = td / dat_norm; nr = tr / ref_norm;
        sum += m * fabs(nd - nr);
        break;
    }
  }
  if (metric == 4 || metric == 5) return n;
  out[0] = sum;
  return 1;
}

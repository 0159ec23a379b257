// Fused GISAXS model for fitting: cylinders on a 2-D lattice in DWBA, its Poisson chi^2 and
// the gradient of chi^2 with respect to theta = (radius R, height H, lattice constant a,
// in-plane rotation phi), for one or many candidate parameter sets with their own detector
// regions of interest.
//
// The model is the reference's simulation of one grain (HipGISAXS::run_gisaxs,
// src/sim/hipgisaxs_main.cpp:694-1100): rotation R_z(phi) (:698), cylinder form factor with
// the size distribution summed unweighted (src/ff/ff_ana_cylinder.cpp:34-117), lattice
// structure factor (src/sf/sf.cpp:164-246), DWBA combination with the Fresnel coefficients
// of the particle layer (:1086-1100), I = |w dn2 sum_k fc_k sf_k ff_k|^2.  It replaces the
// fitting front end's finite differences (src/analyzer/hipgisaxs_fit_lmvm.cpp:190-223: 1 + 2P
// forward runs per gradient) with one forward + adjoint pass.
//
// Factorisation used (vacuum particle layer: the four qz blocks are real and depend on the
// detector row only; lattice vectors a, b in the plane, c along z):
//   A(p) = K Fr(q||) Sa(theta_a) Sb(theta_b) Pc(p) Q(row),
//   Fr = sum_i 2 pi r_i^2 J1(q|| r_i)/(q|| r_i),  Q = sum_k fc_k e^{i qz_k cz} Sc_k G_k,
//   G_k = sum_j h_j sinc(qz_k h_j/2) e^{i qz_k h_j/2},  S_N(theta) = sin(N pi t)/sin(pi t)
//   with t = theta/2pi reduced to [-1/2, 1/2] (the reference's principal-branch Dirichlet
//   kernel written without its branch sign, which cancels), Pc = e^{i(cx q'x + cy q'y)}.
// Derivatives: dFr/dR = sum_i 2 pi r_i J0(q|| r_i) r_i / R; dG/dH = sum_j e^{i qz h_j} h_j / H;
// dS/dtheta from the closed form (series near t = 0); dtheta/dphi = a (u . dq'/dphi).
// Per-row factors are FP64; per-pixel Bessel sums in T (FP32 or FP64); lattice phases are
// reduced in FP64; chi^2 and gradient sums are FP64 and deterministic.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <type_traits>
#include <string>
#include <vector>

#include "cplx.cuh"
#include "hgx_internal.cuh"

namespace hgx {

int param_distribution_host(int stat, double pmin, double pmax, double mean, double dev,
                            int nvalues, std::vector<double>& dim, std::vector<double>& w);

constexpr int CYL_MAXS = 64;
constexpr int CYL_THREADS = 256;                   // block of the row-table and final kernels
// Tile shapes of the persistent pixel pass: threads per block x pixels per thread; one work
// item is one tile of threads*ppt consecutive ROI pixels.  Shape 0 is the default; the
// autotuner (hgx_cyl_batch_tune) times all of them on the batch's own ROIs.
struct CylShape {
  int threads, ppt;
};
constexpr CylShape CYL_SHAPES[] = {{256, 4}, {128, 1}, {128, 2}, {128, 4}, {256, 1},
                                   {256, 2}, {256, 8}, {512, 1}, {512, 2}};
constexpr int CYL_NSHAPES = sizeof(CYL_SHAPES) / sizeof(CYL_SHAPES[0]);
constexpr int CYL_MIN_TILE = 128;                  // smallest threads*ppt above
// Radial-sum tables of the FP32C pixel pass: per candidate, (fr, frR) of the sampled radii at
// the nodes q_j = (j - 1) h, j = 0 .. CYL_NTAB - 1, h = (largest q_par of the grid) / CYL_QT;
// the pixel pass interpolates them with 4-point Lagrange cubics (error ~ (h r)^4, about 1e-9
// relative for r ~ 6 nm) instead of summing 2 Bessel functions per radius per pixel.  Both sums
// depend on q_par only, which the in-plane rotation leaves unchanged.  Tables and interpolation
// are FP64: the gradient sums over a detector cancel near an optimum, and FP32 radial sums
// brought the batch's worst gradient error to 1e-5 of FP64.
constexpr int CYL_QT = 1024;
constexpr int CYL_NTAB = CYL_QT + 4;
constexpr double PI_D = 3.141592653589793;

// model parameter block of the C ABI (16 doubles)
enum { M_R = 0, M_H = 1, M_A = 2, M_PHI = 3, M_SPREAD = 4, M_NSAMP = 5, M_REP = 6, M_DN2 = 9,
       M_CENTER = 11, M_WEIGHT = 14, M_SAMPLING = 15 };

struct CylCand {
  double R, H, a, cphi, sphi;
  double rep[3];
  double K[2];       // weight * dn2
  double center[3];
  double ua[2], ub[2], uc;  // unscaled lattice vectors (in-plane a, b; c along z)
  int nr, nh;
  int row0, col0, nrows, ncols;
  long px_off;       // offset of this candidate's pixels in counts / intensity
  long item0, nitems;
  long rowtab0;      // offset of this candidate's rows in the row table
  double scale;
  double rmin;       // smallest radius sample (the q_par -> 0 guard of the radial sums)
  double r[CYL_MAXS];
  double h[CYL_MAXS];
};

struct RowTab {
  double2 Q, QH, Qa;
};

// S_N(theta) = sin(N pi t)/sin(pi t), t = theta/2pi reduced, and dS/dtheta (FP64).
__device__ __forceinline__ void dirichlet(double theta, double N, double* S, double* dS) {
  if (N == 1.0) {
    *S = 1.0;
    *dS = 0.0;
    return;
  }
  double t = theta * (1.0 / (2.0 * PI_D));
  t -= rint(t);
  double th = 2.0 * PI_D * t;  // reduced angle in [-pi, pi]
  if (fabs(th) * N < 0.1) {  // closed-form derivative cancels here; the series converges fast
    // series of sum_j cos(th c_j), c_j = j - (N-1)/2:  sum c^2, sum c^4, sum c^6
    double n2 = N * N;
    double s2 = N * (n2 - 1.0) / 12.0;
    double s4 = N * (n2 - 1.0) * (3.0 * n2 - 7.0) / 240.0;
    double s6 = N * (n2 - 1.0) * (3.0 * n2 * n2 - 18.0 * n2 + 31.0) / 1344.0;
    double x2 = th * th;
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

// ---------------------------------------------------------------- row table ----
__global__ void cyl_rows_kernel(const CylCand* __restrict__ cands,
                                const double2* __restrict__ rowqz,
                                const double2* __restrict__ rowfc, RowTab* __restrict__ tab) {
  const CylCand& c = cands[blockIdx.y];
  int lr = blockIdx.x * blockDim.x + threadIdx.x;
  if (lr >= c.nrows) return;
  int grow = c.row0 + lr;
  zd Q(0, 0), QH(0, 0), Qa(0, 0);
  for (int k = 0; k < 4; ++k) {
    double qz = rowqz[4L * grow + k].x;
    zd fc(rowfc[4L * grow + k]);
    zd G(0, 0), GH(0, 0);
    for (int j = 0; j < c.nh; ++j) {
      double h = c.h[j];
      double x = 0.5 * qz * h;  // sinc(qz h / 2) e^{i qz h / 2} h
      double sx, cx;
      sincos(x, &sx, &cx);
      double sincv = fabs(x) > 1.0e-14 ? sx / x : 1.0 - x * x / 6.0 + x * x * x * x / 120.0;
      G += zd(cx, sx) * (sincv * h);
      double s2, c2;
      sincos(2.0 * x, &s2, &c2);
      GH += zd(c2, s2) * (h / c.H);
    }
    double Sc, dSc;
    double thc = c.a * c.uc * qz;
    dirichlet(thc, c.rep[2], &Sc, &dSc);
    zd Zc = expi(c.center[2] * qz);
    zd f = fc * Zc;
    Q += f * (G * Sc);
    QH += f * (GH * Sc);
    Qa += f * (G * (dSc * thc / c.a));
  }
  RowTab t;
  t.Q = Q.d2();
  t.QH = QH.d2();
  t.Qa = Qa.d2();
  tab[c.rowtab0 + lr] = t;
}

// --------------------------------------------------------- radial-sum tables ----
// One node per thread: (fr, frR) at q = |j - 1| h, as the pixel pass would sum them, except
// that the q_par -> 0 guard takes the smooth limit (J1(x)/x -> 1/2, J0 -> 1) so that the
// interpolation near q = 0 is right; pixels that meet the guard sum directly.
__global__ void cyl_table_kernel(const CylCand* __restrict__ cands, double h, double2* __restrict__ table) {
  const CylCand& c = cands[blockIdx.y];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= CYL_NTAB) return;
  const double qp = fabs((double)(j - 1) * h);
  double fr = 0.0, frR = 0.0;
  for (int i = 0; i < c.nr; ++i) {
    const double r = c.r[i];
    const double x = qp * r;
    const double two_pi_r = 2.0 * PI_D * r;
    if (x * x > 1.0e-13) {
      fr += two_pi_r * r * j1(x) / x;
      frR += two_pi_r * r * j0(x);
    } else {
      fr += two_pi_r * r * 0.5;
      frR += two_pi_r * r;
    }
  }
  table[(long)blockIdx.y * CYL_NTAB + j] = make_double2(fr, frR / c.R);
}

// --------------------------------------------------------------- pixel pass ----
struct CylArgs {
  const CylCand* cands;
  const int2* items;     // (candidate, first pixel of the tile)
  long nitems;
  const RowTab* tab;
  const double* qx;
  const double* qy;
  int grid_ncol;
  const double* counts;  // may be NULL (forward only)
  const unsigned* mask;  // may be NULL
  double* intensity;     // may be NULL
  double* partial;       // 5 doubles per item (chi2, dR, dH, da, dphi)
  const double2* table;  // FP32C: CYL_NTAB (fr, frR) per candidate
  double inv_h;          // 1 / node spacing of the table
};

template <typename T>
struct BesselT;
template <>
struct BesselT<float> {
  static __device__ __forceinline__ float J0(float x) { return j0f(x); }
  static __device__ __forceinline__ float J1(float x) { return j1f(x); }
};
template <>
struct BesselT<double> {
  static __device__ __forceinline__ double J0(double x) { return j0(x); }
  static __device__ __forceinline__ double J1(double x) { return j1(x); }
};

template <int NT>
__device__ __forceinline__ double block_sum5(double* v, double* sh) {
  // v[5] per thread -> sh[0..4] in thread 0; fixed tree order
#pragma unroll
  for (int q = 0; q < 5; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int q = 0; q < 5; ++q) sh[w * 5 + q] = v[q];
  __syncthreads();
  if (threadIdx.x < 32) {
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      double t = threadIdx.x < NT / 32 ? sh[threadIdx.x * 5 + q] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      v[q] = t;
    }
  }
  __syncthreads();
  return v[0];
}

template <typename T, int NT, int PPT>
__global__ void __launch_bounds__(NT) cyl_pixels_kernel(CylArgs a) {
  __shared__ double sh[(NT / 32) * 5];
  for (long it = blockIdx.x; it < a.nitems; it += gridDim.x) {
    const int2 item = a.items[it];
    const CylCand& c = a.cands[item.x];
    const long npx = (long)c.nrows * c.ncols;
    double acc[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
      long idx = (long)item.y + threadIdx.x + (long)j * NT;
      if (idx >= npx) continue;
      int lr = (int)(idx / c.ncols), lc = (int)(idx - (long)lr * c.ncols);
      long p = (long)(c.row0 + lr) * a.grid_ncol + (c.col0 + lc);
      double qx = a.qx[p], qy = a.qy[p];
      double mx = c.cphi * qx - c.sphi * qy, my = c.sphi * qx + c.cphi * qy;
      double qpar = sqrt(mx * mx + my * my);
      // radial sums (precision T); FP32C interpolates the candidate's table except where a
      // radius sample meets the reference's q_par -> 0 guard (then the terms are summed)
      T fr = 0, frR = 0;
      double frt = 0.0, frRt = 0.0;  // interpolated (FP64 tables)
      bool direct = true;
      if constexpr (std::is_same<T, float>::value) {
        if (qpar * qpar * c.rmin * c.rmin > 1.0e-13) {
          direct = false;
          const double u = qpar * a.inv_h + 1.0;
          const int i0 = min(max((int)u, 1), CYL_NTAB - 3);
          const double t = u - i0;
          const double2* tb = a.table + (long)item.x * CYL_NTAB + (i0 - 1);
          const double w0 = -t * (t - 1.0) * (t - 2.0) * (1.0 / 6.0);
          const double w1 = (t + 1.0) * (t - 1.0) * (t - 2.0) * 0.5;
          const double w2 = -(t + 1.0) * t * (t - 2.0) * 0.5;
          const double w3 = (t + 1.0) * t * (t - 1.0) * (1.0 / 6.0);
          const double2 f0 = tb[0], f1 = tb[1], f2 = tb[2], f3 = tb[3];
          frt = w0 * f0.x + w1 * f1.x + w2 * f2.x + w3 * f3.x;
          frRt = w0 * f0.y + w1 * f1.y + w2 * f2.y + w3 * f3.y;
        }
      }
      if (direct) {
        const T qp = (T)qpar;
        for (int i = 0; i < c.nr; ++i) {
          T r = (T)c.r[i];
          T x = qp * r;
          if ((double)x * (double)x > 1.0e-13) {
            T two_pi_r = (T)(2.0 * PI_D) * r;
            fr += two_pi_r * r * BesselT<T>::J1(x) / x;
            frR += two_pi_r * r * BesselT<T>::J0(x);
          }
        }
        frR /= (T)c.R;
      }
      const double FR = direct ? (double)fr : frt, FRR = direct ? (double)frR : frRt;
      // lattice factors in FP64
      double tha = c.a * (c.ua[0] * mx + c.ua[1] * my);
      double thb = c.a * (c.ub[0] * mx + c.ub[1] * my);
      double Sa, dSa, Sb, dSb;
      dirichlet(tha, c.rep[0], &Sa, &dSa);
      dirichlet(thb, c.rep[1], &Sb, &dSb);
      double dtha_dphi = c.a * (c.ua[0] * (-my) + c.ua[1] * mx);
      double dthb_dphi = c.a * (c.ub[0] * (-my) + c.ub[1] * mx);
      double ph = c.center[0] * mx + c.center[1] * my;
      double dph = c.center[0] * (-my) + c.center[1] * mx;
      zd Pc = expi(ph);
      const RowTab rt = a.tab[c.rowtab0 + lr];
      // amplitude and its derivatives (FP64 combination of T radial sums)
      zd KQ = zd(c.K[0], c.K[1]) * zd(rt.Q);
      double SS = Sa * Sb;
      zd base = KQ * Pc;  // K Q Pc
      zd A = base * (FR * SS);
      zd dA_R = base * (FRR * SS);
      zd dA_H = (zd(c.K[0], c.K[1]) * zd(rt.QH)) * Pc * (FR * SS);
      zd dA_a = Pc * zd(c.K[0], c.K[1]) * FR *
                (zd(rt.Q) * ((dSa * tha / c.a) * Sb + Sa * (dSb * thb / c.a)) + zd(rt.Qa) * SS);
      zd dA_p = KQ * FR *
                (Pc * (dSa * dtha_dphi * Sb + Sa * dSb * dthb_dphi) + Pc * zd(0, dph) * SS);
      double I = A.x * A.x + A.y * A.y;
      if (a.intensity) a.intensity[c.px_off + idx] = I;
      if (a.counts) {
        double C = a.counts[c.px_off + idx];
        double m = a.mask ? (double)a.mask[c.px_off + idx] : 1.0;
        double w = m / (C > 1.0 ? C : 1.0);
        double res = c.scale * I - C;
        double g = 2.0 * w * res * c.scale;
        acc[0] += w * res * res;
        acc[1] += g * 2.0 * (A.x * dA_R.x + A.y * dA_R.y);
        acc[2] += g * 2.0 * (A.x * dA_H.x + A.y * dA_H.y);
        acc[3] += g * 2.0 * (A.x * dA_a.x + A.y * dA_a.y);
        acc[4] += g * 2.0 * (A.x * dA_p.x + A.y * dA_p.y);
      }
    }
    if (a.counts) {
      block_sum5<NT>(acc, sh);
      if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < 5; ++q) a.partial[5 * it + q] = acc[q];
    }
  }
}

// per-candidate sums of the items' partials, fixed order
__global__ void cyl_final_kernel(const CylCand* __restrict__ cands, const double* __restrict__ partial,
                                 double* __restrict__ out) {
  __shared__ double sh[(CYL_THREADS / 32) * 5];
  const CylCand& c = cands[blockIdx.x];
  double acc[5] = {0, 0, 0, 0, 0};
  for (long i = threadIdx.x; i < c.nitems; i += CYL_THREADS)
#pragma unroll
    for (int q = 0; q < 5; ++q) acc[q] += partial[5 * (c.item0 + i) + q];
  block_sum5<CYL_THREADS>(acc, sh);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < 5; ++q) out[5 * blockIdx.x + q] = acc[q];
}

// Launches tile shape `shape` of the pixel pass (a recursion over the shape table, so each
// table row names its own instantiation); with `occ` set it returns the shape's resident
// blocks per SM instead of launching.
template <typename T, int I>
static cudaError_t cyl_pixels_at(int shape, unsigned blocks, const CylArgs& a, cudaStream_t st,
                                 int* occ) {
  if constexpr (I < CYL_NSHAPES) {
    if (shape == I) {
      constexpr int NT = CYL_SHAPES[I].threads, PPT = CYL_SHAPES[I].ppt;
      static_assert(NT % 32 == 0 && NT <= 1024 && NT * PPT >= CYL_MIN_TILE, "bad tile shape");
      if (occ)
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, cyl_pixels_kernel<T, NT, PPT>, NT, 0);
      cyl_pixels_kernel<T, NT, PPT><<<blocks, NT, 0, st>>>(a);
      return cudaGetLastError();
    }
    return cyl_pixels_at<T, I + 1>(shape, blocks, a, st, occ);
  } else {
    return cudaErrorInvalidValue;
  }
}

// ------------------------------------------------- plain FP64 forward (baseline) ----
// One thread per pixel, the reference's loop structure: for each DWBA block, the cylinder
// double loop over (radius, height) (ff_ana_cylinder.cpp:107-111), the lattice factor with
// complex powers (sf.cpp:189-246), then the combination.  Used as the plain FP64 form whose
// 1 + 2P evaluations give the finite-difference gradient the fitter uses.
__global__ void __launch_bounds__(128) cyl_plain_kernel(const CylCand* __restrict__ cp,
                                                        const double2* __restrict__ rowqz,
                                                        const double2* __restrict__ rowfc,
                                                        const double* __restrict__ qxa,
                                                        const double* __restrict__ qya,
                                                        int grid_ncol, double* __restrict__ inten) {
  const CylCand& c = *cp;
  long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)c.nrows * c.ncols) return;
  int lr = (int)(idx / c.ncols), lc = (int)(idx - (long)lr * c.ncols);
  int grow = c.row0 + lr;
  long p = (long)grow * grid_ncol + (c.col0 + lc);
  double qx = qxa[p], qy = qya[p];
  zd acc(0, 0);
  for (int k = 0; k < 4; ++k) {
    zd qz(rowqz[4L * grow + k]);
    zd m0(c.cphi * qx - c.sphi * qy + 0.0 * qz.x, 0.0), m1(c.sphi * qx + c.cphi * qy, 0.0), m2 = qz;
    zd qpar = csqrt_(m0 * m0 + m1 * m1);
    zd ff(0, 0);
    for (int i = 0; i < c.nr; ++i)
      for (int j = 0; j < c.nh; ++j) {
        double r = c.r[i], h = c.h[j];
        double vol = 2. * PI_D * r * r * h;
        zd xs = (m2 * 0.5) * h;
        zd sincv = cabs_(xs) > 1e-14 ? csin_(xs) / xs : (1.0 - xs * xs / 6.0) + xs * xs * xs * xs / 120.0;
        zd ex = cexp_((zd(0, 0.5) * m2) * h);
        zd t1 = qpar * r;
        zd bess(0, 0);
        if (norm2(t1) > 1.0e-13) bess = zd(j1(t1.x), 0.0) * conj(t1) / norm2(t1);
        ff += ((sincv * vol) * ex) * bess;
      }
    // lattice factor (sf.cpp:189-246), lattice vectors scaled by a
    double la[3] = {c.ua[0] * c.a, c.ua[1] * c.a, 0.0}, lb[3] = {c.ub[0] * c.a, c.ub[1] * c.a, 0.0};
    double lc = c.uc * c.a;
    const zd one(1.0, 0.0);
    zd eqa = cexp_(zd(0, 1) * (m0 * la[0] + m1 * la[1]));
    zd Ya = one - eqa;
    zd sa = (fabs(Ya.y) > 2.220446049250313e-16 || fabs(Ya.x) > 2.220446049250313e-16)
                ? (one - cpow_std(eqa, c.rep[0])) / Ya : zd(c.rep[0], 0);
    sa = cpow_std(eqa, (1.0 - c.rep[0]) / 2.0) * sa;
    zd iqb = zd(0, 1) * (m0 * lb[0] + m1 * lb[1] + lb[2] * lb[2]);
    zd eqb = cexp_(iqb), Yb = one - eqb;
    zd sb = (fabs(Yb.y) > 2.220446049250313e-16 || fabs(Yb.x) > 2.220446049250313e-16)
                ? (one - cexp_(iqb * c.rep[1])) / Yb : zd(c.rep[1], 0);
    sb = cpow_std(eqb, (1.0 - c.rep[1]) / 2.0) * sb;
    zd eqc = cexp_(zd(0, 1) * (m2 * lc)), Yc = one - eqc;
    zd sc = (fabs(Yc.y) > 2.220446049250313e-16 || fabs(Yc.x) > 2.220446049250313e-16)
                ? (one - cpow_std(eqc, c.rep[2])) / Yc : zd(c.rep[2], 0);
    sc = cpow_std(eqc, (1.0 - c.rep[2]) / 2.0) * sc;
    zd t3 = m0 * c.center[0] + m1 * c.center[1] + m2 * c.center[2];
    zd sf = cexp_(zd(-t3.y, t3.x)) * sa * sb * sc;
    acc += zd(rowfc[4L * grow + k]) * sf * (zd(c.K[0], c.K[1]) * ff);
  }
  inten[idx] = acc.x * acc.x + acc.y * acc.y;
}

// ------------------------------------------------------------------- host ----
int cyl_fill_cand(const double* m, const double* abc9, const int* roi, double scale, CylCand& c) {
  c = CylCand();
  c.R = m[M_R];
  c.H = m[M_H];
  c.a = m[M_A];
  c.cphi = cos(m[M_PHI]);
  c.sphi = sin(m[M_PHI]);
  if (!(c.R > 0) || !(c.H > 0) || !(c.a > 0))
    return fail(HGX_ERR_INVALID_ARG, "cylinder model: radius, height and lattice constant must be > 0");
  for (int i = 0; i < 3; ++i) {
    c.rep[i] = m[M_REP + i] < 1 ? 1 : m[M_REP + i];
    c.center[i] = m[M_CENTER + i];
  }
  double w = m[M_WEIGHT];
  c.K[0] = w * m[M_DN2];
  c.K[1] = w * m[M_DN2 + 1];
  if (abc9[2] != 0.0 || abc9[5] != 0.0 || abc9[6] != 0.0 || abc9[7] != 0.0)
    return fail(HGX_ERR_INVALID_ARG, "cylinder model: lattice vectors a, b must lie in the plane and c along z");
  c.ua[0] = abc9[0];
  c.ua[1] = abc9[1];
  c.ub[0] = abc9[3];
  c.ub[1] = abc9[4];
  c.uc = abc9[8];
  // size distributions: Gaussian over +-3 sigma sampled as param_distribution does
  double s = m[M_SPREAD];
  int n = (int)m[M_NSAMP];
  std::vector<double> rv, rw, hv, hw;
  if (s > 0 && n > 1 && m[M_SAMPLING] == 1.0) {
    // exactly n evenly spaced samples: smooth in R and H (the reference's stepping below
    // can add or drop the last sample as R or H moves, a jump in the model)
    for (int i = 0; i < n; ++i) {
      double u = -3.0 * s + 6.0 * s * i / (n - 1);
      rv.push_back(c.R * (1.0 + u));
      hv.push_back(c.H * (1.0 + u));
    }
  } else if (s > 0 && n > 1) {
    HGX_TRY(param_distribution_host(4, c.R * (1 - 3 * s), c.R * (1 + 3 * s), c.R, s * c.R, n, rv, rw));
    HGX_TRY(param_distribution_host(4, c.H * (1 - 3 * s), c.H * (1 + 3 * s), c.H, s * c.H, n, hv, hw));
  } else {
    rv.push_back(c.R);
    hv.push_back(c.H);
  }
  if (rv.size() > CYL_MAXS || hv.size() > CYL_MAXS)
    return fail(HGX_ERR_INVALID_ARG, "cylinder model: at most 64 size samples");
  c.nr = (int)rv.size();
  c.nh = (int)hv.size();
  for (int i = 0; i < c.nr; ++i) c.r[i] = rv[i];
  c.rmin = c.nr > 0 ? *std::min_element(rv.begin(), rv.end()) : 0.0;
  for (int i = 0; i < c.nh; ++i) c.h[i] = hv[i];
  c.row0 = roi[0];
  c.col0 = roi[1];
  c.nrows = roi[2];
  c.ncols = roi[3];
  c.scale = scale;
  return HGX_OK;
}

}  // namespace hgx

// A prepared batch: candidates, work items, row table, device buffers, and a CUDA graph of
// (parameters H2D -> row table -> pixel pass -> per-candidate sums -> results D2H).
struct hgx_cyl_batch_s {
  hgx_ctx ctx = nullptr;
  hgx_qgrid grid = nullptr;
  int ncand = 0;
  long npx = 0, nitems = 0, nrowtab = 0;
  int precision = HGX_F32C;
  double abc9[9];
  std::vector<int> rois;
  double scale = 1.0;
  hgx::DevBuf d_cands, d_items, d_tab, d_partial, d_out, d_rowfc, d_counts, d_mask, d_inten;
  hgx::CylCand* h_cands = nullptr;  // pinned
  double* h_out = nullptr;          // pinned
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int persistent_blocks = 0;
  int shape = 0;  // tile shape of the pixel pass (index into the shape table)
  hgx::DevBuf d_table;  // FP32C radial-sum tables
  hgx::DevBuf d_plain;  // the candidate record of hgx_cyl_plain_forward
  double table_h = 1.0;  // their node spacing
};

namespace hgx {

static int cyl_enqueue(hgx_cyl_batch_s* b, bool with_counts, bool with_intensity) {
  cudaStream_t st = b->ctx->stream;
  HGX_CUDA(cudaMemcpyAsync(b->d_cands.p, b->h_cands, sizeof(CylCand) * b->ncand,
                           cudaMemcpyHostToDevice, st));
  int maxrows = 0;
  for (int i = 0; i < b->ncand; ++i) maxrows = std::max(maxrows, b->rois[4 * i + 2]);
  dim3 rg((maxrows + 127) / 128, b->ncand);
  cyl_rows_kernel<<<rg, 128, 0, st>>>((const CylCand*)b->d_cands.p, b->grid->rowqz,
                                      (const double2*)b->d_rowfc.p, (RowTab*)b->d_tab.p);
  CylArgs a;
  a.cands = (const CylCand*)b->d_cands.p;
  a.items = (const int2*)b->d_items.p;
  a.nitems = b->nitems;
  a.tab = (const RowTab*)b->d_tab.p;
  a.qx = b->grid->qx;
  a.qy = b->grid->qy;
  a.grid_ncol = b->grid->ncol;
  a.counts = with_counts ? (const double*)b->d_counts.p : nullptr;
  a.mask = with_counts ? (const unsigned*)b->d_mask.p : nullptr;
  a.intensity = with_intensity ? (double*)b->d_inten.p : nullptr;
  a.partial = (double*)b->d_partial.p;
  a.table = (const double2*)b->d_table.p;
  a.inv_h = 1.0 / b->table_h;
  if (b->precision == HGX_F32C)
    cyl_table_kernel<<<dim3((CYL_NTAB + 127) / 128, b->ncand), 128, 0, st>>>(
        (const CylCand*)b->d_cands.p, b->table_h, (double2*)b->d_table.p);
  long blocks = std::min<long>(b->nitems, (long)b->persistent_blocks);
  cudaError_t e = b->precision == HGX_F64
                      ? cyl_pixels_at<double, 0>(b->shape, (unsigned)blocks, a, st, nullptr)
                      : cyl_pixels_at<float, 0>(b->shape, (unsigned)blocks, a, st, nullptr);
  if (e != cudaSuccess) return cuda_fail(e, "cyl_pixels_kernel launch");
  if (with_counts) {
    cyl_final_kernel<<<b->ncand, CYL_THREADS, 0, st>>>((const CylCand*)b->d_cands.p,
                                                      (const double*)b->d_partial.p,
                                                      (double*)b->d_out.p);
    HGX_CUDA(cudaMemcpyAsync(b->h_out, b->d_out.p, sizeof(double) * 5 * b->ncand,
                             cudaMemcpyDeviceToHost, st));
  }
  HGX_CUDA(cudaGetLastError());
  return HGX_OK;
}

// Work items for tile shape `shape`: one per threads*ppt consecutive pixels of each ROI; sets
// the candidates' item ranges, grows and fills the item and partial-sum buffers, sizes the
// persistent grid from the shape's occupancy, and drops a captured graph (its launch shape
// and buffers are stale).
static int cyl_apply_shape(hgx_cyl_batch_s* b, int shape) {
  if (shape < 0 || shape >= CYL_NSHAPES)
    return fail(HGX_ERR_INVALID_ARG, "hgx_cyl_batch: unknown tile shape");
  const long tile = (long)CYL_SHAPES[shape].threads * CYL_SHAPES[shape].ppt;
  std::vector<int2> items;
  for (int i = 0; i < b->ncand; ++i) {
    CylCand& h = b->h_cands[i];
    long n = (long)b->rois[4 * i + 2] * b->rois[4 * i + 3];
    h.item0 = (long)items.size();
    for (long s = 0; s < n; s += tile) items.push_back(make_int2(i, (int)s));
    h.nitems = (long)items.size() - h.item0;
  }
  cudaStream_t st = b->ctx->stream;
  HGX_CUDA(cudaStreamSynchronize(st));
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  HGX_TRY(b->d_items.reserve(sizeof(int2) * items.size()));
  HGX_TRY(b->d_partial.reserve(sizeof(double) * 5 * items.size()));
  HGX_CUDA(cudaMemcpyAsync(b->d_items.p, items.data(), sizeof(int2) * items.size(),
                           cudaMemcpyHostToDevice, st));
  HGX_CUDA(cudaStreamSynchronize(st));  // `items` is pageable and about to go out of scope
  int per_sm = 0;
  CylArgs none{};
  cudaError_t e = b->precision == HGX_F64 ? cyl_pixels_at<double, 0>(shape, 0, none, st, &per_sm)
                                          : cyl_pixels_at<float, 0>(shape, 0, none, st, &per_sm);
  if (e != cudaSuccess) return cuda_fail(e, "hgx_cyl_batch: occupancy query");
  b->persistent_blocks = b->ctx->sm_count * std::max(1, per_sm);
  b->nitems = (long)items.size();
  b->shape = shape;
  return HGX_OK;
}

static int cyl_set_models(hgx_cyl_batch_s* b, const double* models) {
  for (int i = 0; i < b->ncand; ++i) {
    CylCand c;
    HGX_TRY(cyl_fill_cand(models + 16 * i, b->abc9, b->rois.data() + 4 * i, b->scale, c));
    CylCand& h = b->h_cands[i];
    // keep the layout fields computed at creation
    c.px_off = h.px_off;
    c.item0 = h.item0;
    c.nitems = h.nitems;
    c.rowtab0 = h.rowtab0;
    h = c;
  }
  return HGX_OK;
}

}  // namespace hgx

using namespace hgx;

extern "C" {

int hgx_cyl_batch_destroy(hgx_cyl_batch_s* b);

// Creates a batch of ncand candidates.  rois: 4 ints each (row0, col0, nrows, ncols) inside
// the grid; counts: concatenated ROI images (row-major per candidate, in candidate order),
// may be NULL for forward-only use; mask: same layout or NULL.
int hgx_cyl_batch_create(hgx_ctx c, hgx_qgrid g, const double* rowfc, const double* abc9,
                         int ncand, const int* rois, const double* counts,
                         const unsigned* mask, double scale, int precision,
                         hgx_cyl_batch_s** out) {
  if (!c || !g || !rowfc || !abc9 || !rois || !out || ncand < 1)
    return fail(HGX_ERR_INVALID_ARG, "hgx_cyl_batch_create: null argument");
  *out = nullptr;
  if (g->mode != 1 || g->nk != 4)
    return fail(HGX_ERR_INVALID_ARG, "hgx_cyl_batch_create: needs a DWBA grid with real qz "
                                     "constant along rows (vacuum particle layer)");
  if (precision != HGX_F32C && precision != HGX_F64)
    return fail(HGX_ERR_INVALID_ARG, "hgx_cyl_batch_create: unknown precision");
  HGX_CUDA(cudaSetDevice(c->device));
  auto b = new (std::nothrow) hgx_cyl_batch_s();
  if (!b) return fail(HGX_ERR_NO_MEMORY, "hgx_cyl_batch_create: host allocation");
  b->ctx = c;
  b->grid = g;
  b->ncand = ncand;
  b->precision = precision;
  b->scale = scale;
  for (int i = 0; i < 9; ++i) b->abc9[i] = abc9[i];
  b->rois.assign(rois, rois + 4 * ncand);
  auto bail = [&](int s) {
    hgx_cyl_batch_destroy(b);
    return s;
  };
  if (cudaMallocHost(&b->h_cands, sizeof(CylCand) * ncand) != cudaSuccess ||
      cudaMallocHost(&b->h_out, sizeof(double) * 5 * ncand) != cudaSuccess)
    return bail(fail(HGX_ERR_NO_MEMORY, "hgx_cyl_batch_create: pinned host memory"));
  long px = 0, rows = 0;
  for (int i = 0; i < ncand; ++i) {
    const int* r = rois + 4 * i;
    if (r[0] < 0 || r[1] < 0 || r[2] < 1 || r[3] < 1 || r[0] + r[2] > g->nrow || r[1] + r[3] > g->ncol)
      return bail(fail(HGX_ERR_INVALID_ARG, "hgx_cyl_batch_create: ROI outside the grid"));
    CylCand& h = b->h_cands[i];
    h = CylCand();
    long n = (long)r[2] * r[3];
    h.px_off = px;
    h.rowtab0 = rows;
    px += n;
    rows += r[2];
  }
  b->npx = px;
  b->nrowtab = rows;
  int s = HGX_OK;
  if ((s = b->d_cands.reserve(sizeof(CylCand) * ncand)) || (s = b->d_tab.reserve(sizeof(RowTab) * rows)) ||
      (s = b->d_out.reserve(sizeof(double) * 5 * ncand)) || (s = b->d_rowfc.reserve(sizeof(double2) * 4 * g->nrow)) ||
      (s = b->d_inten.reserve(sizeof(double) * px)))
    return bail(s);
  cudaStream_t st = c->stream;
  cudaError_t e = cudaMemcpyAsync(b->d_rowfc.p, rowfc, sizeof(double2) * 4 * g->nrow,
                                  is_device_ptr(rowfc) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && counts) {
    if ((s = b->d_counts.reserve(sizeof(double) * px))) return bail(s);
    e = cudaMemcpyAsync(b->d_counts.p, counts, sizeof(double) * px,
                        is_device_ptr(counts) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
  }
  if (e == cudaSuccess && mask) {
    if ((s = b->d_mask.reserve(sizeof(unsigned) * px))) return bail(s);
    e = cudaMemcpyAsync(b->d_mask.p, mask, sizeof(unsigned) * px,
                        is_device_ptr(mask) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return bail(cuda_fail(e, "hgx_cyl_batch_create: copies"));
  if (!mask) b->d_mask.release();
  if (precision == HGX_F32C) {
    // node spacing of the radial-sum tables: the grid's largest q_par over CYL_QT intervals
    std::vector<double> hx(g->nqy), hy(g->nqy);
    e = cudaMemcpy(hx.data(), g->qx, sizeof(double) * g->nqy, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(hy.data(), g->qy, sizeof(double) * g->nqy, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return bail(cuda_fail(e, "hgx_cyl_batch_create: read q-grid"));
    double qm = 0.0;
    for (int i = 0; i < g->nqy; ++i) qm = std::max(qm, sqrt(hx[i] * hx[i] + hy[i] * hy[i]));
    b->table_h = (qm > 0.0 ? qm : 1.0) * (1.0 + 1e-9) / CYL_QT;
    if ((s = b->d_table.reserve(sizeof(double2) * CYL_NTAB * (size_t)ncand))) return bail(s);
  }
  if ((s = cyl_apply_shape(b, 0))) return bail(s);
  *out = b;
  return HGX_OK;
}

// Evaluates chi^2 and its gradient for every candidate: models: 16 doubles per candidate;
// out: 5 doubles per candidate (chi2, dchi2/dR, dchi2/dH, dchi2/da, dchi2/dphi).  The first
// call captures the sequence into a CUDA graph; later calls replay it.
int hgx_cyl_batch_eval(hgx_cyl_batch_s* b, const double* models, double* out) {
  if (!b || !models || !out) return fail(HGX_ERR_INVALID_ARG, "hgx_cyl_batch_eval: null argument");
  if (!b->d_counts.p) return fail(HGX_ERR_INVALID_ARG, "hgx_cyl_batch_eval: batch has no counts");
  HGX_CUDA(cudaSetDevice(b->ctx->device));
  cudaStream_t st = b->ctx->stream;
  HGX_CUDA(cudaStreamSynchronize(st));  // the pinned parameter block is about to change
  HGX_TRY(cyl_set_models(b, models));
  if (!b->exec) {
    cudaStream_t cap = nullptr;
    HGX_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaStream_t saved = b->ctx->stream;
    b->ctx->stream = cap;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    int s = HGX_OK;
    if (e == cudaSuccess) s = cyl_enqueue(b, true, false);
    cudaGraph_t graph = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
    b->ctx->stream = saved;
    cudaStreamDestroy(cap);
    if (e != cudaSuccess || s != HGX_OK || e2 != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);  // a graph ended from a failed capture is not kept
      if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
      if (s != HGX_OK) return s;
      return cuda_fail(e2, "cudaStreamEndCapture");
    }
    b->graph = graph;
    HGX_CUDA(cudaGraphInstantiate(&b->exec, graph, 0));
  }
  HGX_CUDA(cudaGraphLaunch(b->exec, st));
  HGX_CUDA(cudaStreamSynchronize(st));
  for (int i = 0; i < 5 * b->ncand; ++i) out[i] = b->h_out[i];
  return hgx_synchronize(b->ctx);
}

// Model intensity of every candidate (no chi^2): intensity = concatenated ROI images.
int hgx_cyl_batch_forward(hgx_cyl_batch_s* b, const double* models, double* intensity) {
  if (!b || !models || !intensity) return fail(HGX_ERR_INVALID_ARG, "hgx_cyl_batch_forward: null argument");
  HGX_CUDA(cudaSetDevice(b->ctx->device));
  HGX_CUDA(cudaStreamSynchronize(b->ctx->stream));
  HGX_TRY(cyl_set_models(b, models));
  HGX_TRY(cyl_enqueue(b, false, true));
  HGX_CUDA(cudaMemcpyAsync(intensity, b->d_inten.p, sizeof(double) * b->npx,
                           is_device_ptr(intensity) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                           b->ctx->stream));
  return hgx_synchronize(b->ctx);
}

// The plain FP64 form (reference loop structure) of candidate `cand`'s intensity; with the
// distance kernels it gives the finite-difference chi^2 gradient of the reference's fitter.
int hgx_cyl_plain_forward(hgx_cyl_batch_s* b, int cand, const double* model, double* intensity) {
  if (!b || !model || !intensity || cand < 0 || cand >= b->ncand)
    return fail(HGX_ERR_INVALID_ARG, "hgx_cyl_plain_forward: bad argument");
  HGX_CUDA(cudaSetDevice(b->ctx->device));
  cudaStream_t st = b->ctx->stream;
  CylCand cnd;
  HGX_TRY(cyl_fill_cand(model, b->abc9, b->rois.data() + 4 * cand, b->scale, cnd));
  DevBuf dout;
  DevBuf& dc = b->d_plain;
  HGX_TRY(dc.reserve(sizeof(CylCand)));
  HGX_CUDA(cudaMemcpyAsync(dc.p, &cnd, sizeof(CylCand), cudaMemcpyHostToDevice, st));
  long n = (long)cnd.nrows * cnd.ncols;
  void* dI = nullptr;
  HGX_TRY(stage_out(b->ctx, intensity, sizeof(double) * n, dout, &dI));
  cyl_plain_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(
      (const CylCand*)dc.p, b->grid->rowqz, (const double2*)b->d_rowfc.p, b->grid->qx, b->grid->qy,
      b->grid->ncol, (double*)dI);
  HGX_CUDA(cudaGetLastError());
  HGX_TRY(finish_out(b->ctx, intensity, sizeof(double) * n, dI));
  return hgx_synchronize(b->ctx);
}

// Tile-shape table of the pixel pass: threads per block and pixels per thread of `shape`;
// HGX_ERR_INVALID_ARG past the end of the table (callers enumerate with it).
int hgx_cyl_shape_info(int shape, int* threads, int* pixels_per_thread) {
  if (shape < 0 || shape >= CYL_NSHAPES)
    return fail(HGX_ERR_INVALID_ARG, "hgx_cyl_shape_info: shape past the end of the table");
  if (threads) *threads = CYL_SHAPES[shape].threads;
  if (pixels_per_thread) *pixels_per_thread = CYL_SHAPES[shape].ppt;
  return HGX_OK;
}

int hgx_cyl_batch_set_shape(hgx_cyl_batch_s* b, int shape) {
  if (!b) return fail(HGX_ERR_INVALID_ARG, "hgx_cyl_batch_set_shape: null batch");
  HGX_CUDA(cudaSetDevice(b->ctx->device));
  return cyl_apply_shape(b, shape);
}

int hgx_cyl_batch_get_shape(hgx_cyl_batch_s* b, int* shape) {
  if (!b || !shape) return fail(HGX_ERR_INVALID_ARG, "hgx_cyl_batch_get_shape: null argument");
  *shape = b->shape;
  return HGX_OK;
}

// The autotuner: for every tile shape, one untimed evaluation and then `reps` evaluations timed
// together with CUDA events on the batch's stream (chi^2 + gradient when the batch has counts,
// else the forward intensities), at these models and on this batch's ROIs; keeps the fastest
// shape.  times_ms (may be NULL) receives the mean time of each shape, in table order.
int hgx_cyl_batch_tune(hgx_cyl_batch_s* b, const double* models, int reps, int* best_shape,
                       double* best_ms, double* times_ms) {
  if (!b || !models) return fail(HGX_ERR_INVALID_ARG, "hgx_cyl_batch_tune: null argument");
  if (reps < 1) reps = 1;
  HGX_CUDA(cudaSetDevice(b->ctx->device));
  cudaStream_t st = b->ctx->stream;
  HGX_CUDA(cudaStreamSynchronize(st));
  HGX_TRY(cyl_set_models(b, models));
  struct Events {
    cudaEvent_t e[2] = {nullptr, nullptr};
    ~Events() {
      for (auto x : e)
        if (x) cudaEventDestroy(x);
    }
  } ev;
  HGX_CUDA(cudaEventCreate(&ev.e[0]));
  HGX_CUDA(cudaEventCreate(&ev.e[1]));
  const bool chi = b->d_counts.p != nullptr;
  int best = 0;
  double bms = 0.0;
  for (int sh = 0; sh < CYL_NSHAPES; ++sh) {
    HGX_TRY(cyl_apply_shape(b, sh));
    HGX_TRY(cyl_enqueue(b, chi, !chi));
    HGX_CUDA(cudaEventRecord(ev.e[0], st));
    for (int r = 0; r < reps; ++r) HGX_TRY(cyl_enqueue(b, chi, !chi));
    HGX_CUDA(cudaEventRecord(ev.e[1], st));
    HGX_CUDA(cudaEventSynchronize(ev.e[1]));
    float ms = 0.f;
    HGX_CUDA(cudaEventElapsedTime(&ms, ev.e[0], ev.e[1]));
    double per = (double)ms / reps;
    if (times_ms) times_ms[sh] = per;
    if (sh == 0 || per < bms) {
      best = sh;
      bms = per;
    }
  }
  HGX_TRY(cyl_apply_shape(b, best));
  if (best_shape) *best_shape = best;
  if (best_ms) *best_ms = bms;
  return hgx_synchronize(b->ctx);
}

int hgx_cyl_batch_info(hgx_cyl_batch_s* b, long* npx, long* nitems) {
  if (!b) return fail(HGX_ERR_INVALID_ARG, "hgx_cyl_batch_info: null batch");
  if (npx) *npx = b->npx;
  if (nitems) *nitems = b->nitems;
  return HGX_OK;
}

int hgx_cyl_batch_destroy(hgx_cyl_batch_s* b) {
  if (!b) return HGX_OK;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->h_cands) cudaFreeHost(b->h_cands);
  if (b->h_out) cudaFreeHost(b->h_out);
  delete b;
  return HGX_OK;
}

}  // extern "C"

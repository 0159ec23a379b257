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
// |Pc| = 1, so I = |K Q|^2 (Fr Sa Sb)^2 and every derivative of I is real arithmetic on three
// FP64 row scalars and the pixel's Fr, dFr/dR, Sa, Sb, dSa, dSb.  Row factors are FP64; the
// pixel pass is FP64 throughout (HGX_F64) or FP32C (lattice turns reduced in FP64, radial sums
// interpolated from FP64 tables, Dirichlet kernels and derivative products in FP32); chi^2 and
// gradient sums are FP64 and deterministic.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <type_traits>
#include <string>
#include <vector>

#include "cplx.cuh"
#include "hgx_internal.cuh"
#include "turns.cuh"

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
  double ka[2], kb[2];      // a ua / 2pi, a ub / 2pi: lattice phases in turns
  float ser[2][8];          // FP32C Dirichlet series of the a- and b-directions (cyl_dirichlet_series)
  float fa, fua[2], fub[2], frep[2], fscale;  // FP32 copies for the FP32C pixel pass
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
  double q2, qh, qa;     // |K Q|^2, |K|^2 Re(conj(Q) dQ/dH), |K|^2 Re(conj(Q) dQ/da)
  float q2f, qhf, qaf;   // the same rounded to FP32 (the FP32C derivative products)
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

// The Dirichlet kernel in FP32 arithmetic at a turn t already reduced to [-1/2, 1/2] in FP64.
// N t is reduced modulo 2 in FP64 too (sin and cos of pi N t keep their values), so both sines
// keep FP32 accuracy for any N.  For |theta| N < 1 the closed form's derivative cancels; there
// the series in y = (theta N)^2 with the candidate's scaled power sums: e[0..3] for S, e[4..7]
// for dS.
__device__ __forceinline__ void dirichlet_f32(double t, double N, float Nf, const float* e,
                                              float* S, float* dS) {
  if (N == 1.0) {
    *S = 1.0f;
    *dS = 0.0f;
    return;
  }
  const float tf = (float)t;
  const float thN = 6.28318530718f * tf * Nf;
  if (fabsf(thN) < 1.0f) {
    const float y = thN * thN;
    *S = Nf * (1.0f - y * (e[0] - y * (e[1] - y * (e[2] - y * e[3]))));
    *dS = -thN * Nf * Nf * (e[4] - y * (e[5] - y * (e[6] - y * e[7])));
    return;
  }
  const double u = N * t;
  float sn, cn, s1, c1;
  sincospi_f32((float)(u - 2.0 * round_fp64(0.5 * u)), &sn, &cn);
  sincospi_f32(tf, &s1, &c1);
  const float inv = __frcp_rn(s1), Sv = sn * inv;
  *S = Sv;
  *dS = 0.5f * (Nf * cn - Sv * c1) * inv;
}

// ---------------------------------------------------------------- row table ----
// One warp per (candidate, ROI row): lane 8 k + j takes DWBA block k and the height samples
// j, j + 8, ...; xor shuffles close the height sums inside each group of 8 lanes and then the
// block sums across the groups (a fixed tree, so every lane holds the same bits).  The row's
// scalars of the intensity and its H- and a-derivatives: the centre phase has modulus 1 and
// drops out of |A|^2.
__device__ __forceinline__ void cyl_rows_body(const CylCand& c, int bx, const double2* __restrict__ rowqz,
                                              const double2* __restrict__ rowfc, RowTab* __restrict__ tab) {
  const int lr = (int)((bx * blockDim.x + threadIdx.x) >> 5);
  if (lr >= c.nrows) return;  // whole warps
  const int lane = threadIdx.x & 31, k = lane >> 3;
  const int grow = c.row0 + lr;
  const double qz = rowqz[4L * grow + k].x;
  zd G(0, 0), GH(0, 0);
  for (int j = lane & 7; j < c.nh; j += 8) {
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
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) {
    G.x += __shfl_xor_sync(0xffffffffu, G.x, o);
    G.y += __shfl_xor_sync(0xffffffffu, G.y, o);
    GH.x += __shfl_xor_sync(0xffffffffu, GH.x, o);
    GH.y += __shfl_xor_sync(0xffffffffu, GH.y, o);
  }
  double Sc, dSc;
  const double thc = c.a * c.uc * qz;
  dirichlet(thc, c.rep[2], &Sc, &dSc);
  const zd f = zd(rowfc[4L * grow + k]) * expi(c.center[2] * qz);
  zd Q = f * (G * Sc), QH = f * (GH * Sc), Qa = f * (G * (dSc * thc / c.a));
#pragma unroll
  for (int o = 8; o < 32; o <<= 1) {
    Q.x += __shfl_xor_sync(0xffffffffu, Q.x, o);
    Q.y += __shfl_xor_sync(0xffffffffu, Q.y, o);
    QH.x += __shfl_xor_sync(0xffffffffu, QH.x, o);
    QH.y += __shfl_xor_sync(0xffffffffu, QH.y, o);
    Qa.x += __shfl_xor_sync(0xffffffffu, Qa.x, o);
    Qa.y += __shfl_xor_sync(0xffffffffu, Qa.y, o);
  }
  if (lane == 0) {
    const double K2 = c.K[0] * c.K[0] + c.K[1] * c.K[1];
    RowTab t;
    t.q2 = K2 * norm2(Q);
    t.qh = K2 * (Q.x * QH.x + Q.y * QH.y);
    t.qa = K2 * (Q.x * Qa.x + Q.y * Qa.y);
    t.q2f = (float)t.q2;
    t.qhf = (float)t.qh;
    t.qaf = (float)t.qa;
    tab[c.rowtab0 + lr] = t;
  }
}

// --------------------------------------------------------- radial-sum tables ----
// 8 lanes per node: lane l sums the radius samples l, l + 8, ..., xor shuffles close the sum
// ((fr, frR) at q = |j - 1| h, as the pixel pass would sum them), except that the q_par -> 0
// guard takes the smooth limit (J1(x)/x -> 1/2, J0 -> 1) so that the interpolation near q = 0
// is right; pixels that meet the guard sum directly.  Each FP64 sum is stored as an FP32 pair
// (hi, lo = sum - hi): the pixel pass interpolates both in FP32, so no rounding of a node,
// common to every pixel near that q_par, reaches the intensity.
__device__ __forceinline__ void cyl_table_body(const CylCand& c, int bx, double h, float4* __restrict__ table) {
  const int j = (int)((bx * blockDim.x + threadIdx.x) >> 3), l = threadIdx.x & 7;
  const double qp = fabs((double)(j - 1) * h);
  double fr = 0.0, frR = 0.0;
  if (j < CYL_NTAB)  // lanes past the last node still join the shuffles
    for (int i = l; i < c.nr; i += 8) {
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
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) {
    fr += __shfl_xor_sync(0xffffffffu, fr, o);
    frR += __shfl_xor_sync(0xffffffffu, frR, o);
  }
  if (j < CYL_NTAB && l == 0) {
    const double v = frR / c.R;
    const float fh = (float)fr, vh = (float)v;
    table[(long)blockIdx.y * CYL_NTAB + j] = make_float4(fh, (float)(fr - fh), vh, (float)(v - vh));
  }
}

// The per-evaluation set-up in one launch: blocks [0, row_blocks) build the row table (a warp
// per ROI row), the rest (FP32C only) the radial-sum tables; grid y = candidate.
__global__ void cyl_prep_kernel(const CylCand* __restrict__ cands, int row_blocks,
                                const double2* __restrict__ rowqz, const double2* __restrict__ rowfc,
                                RowTab* __restrict__ tab, double h, float4* __restrict__ table) {
  const CylCand& c = cands[blockIdx.y];
  if ((int)blockIdx.x < row_blocks)
    cyl_rows_body(c, blockIdx.x, rowqz, rowfc, tab);
  else
    cyl_table_body(c, blockIdx.x - row_blocks, h, table);
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
  const float4* table;   // FP32C: CYL_NTAB (fr hi, lo, frR/R hi, lo) per candidate
  double inv_h;          // 1 / node spacing of the table
  const float* wf;       // FP32C: mask / max(counts, 1) per pixel (may be NULL: forward only)
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

// Per pixel: I = q2 (Fr Sa Sb)^2 and its derivatives
//   dI/dR = 2 q2 Fr dFr/dR (Sa Sb)^2,  dI/dH = 2 qh (Fr Sa Sb)^2,
//   dI/da = 2 Fr^2 Sa Sb (q2 d(Sa Sb)/da + qa Sa Sb),  dI/dphi = 2 q2 Fr^2 Sa Sb d(Sa Sb)/dphi,
// then the chi^2 terms w (s I - C)^2, w = mask / max(C, 1), and their derivatives.
// The FP64 form: every Bessel function and Dirichlet kernel in FP64 per pixel, FP64 sums.
template <typename T, int NT, int PPT>
__global__ void __launch_bounds__(NT) cyl_pixels_kernel(CylArgs a) {
  static_assert(std::is_same<T, double>::value, "FP32C has its own kernel");
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
      const double qx = a.qx[p], qy = a.qy[p];
      const double mx = c.cphi * qx - c.sphi * qy, my = c.sphi * qx + c.cphi * qy;
      const double qpar = sqrt(mx * mx + my * my);
      double Sa, dSa, Sb, dSb;
      dirichlet(c.a * (c.ua[0] * mx + c.ua[1] * my), c.rep[0], &Sa, &dSa);
      dirichlet(c.a * (c.ub[0] * mx + c.ub[1] * my), c.rep[1], &Sb, &dSb);
      double FR = 0.0, FRR = 0.0;
      for (int i = 0; i < c.nr; ++i) {
        const double r = c.r[i], x = qpar * r;
        if (x * x > 1.0e-13) {
          const double two_pi_r = 2.0 * PI_D * r;
          FR += two_pi_r * r * j1(x) / x;
          FRR += two_pi_r * r * j0(x);
        }
      }
      FRR /= c.R;
      const RowTab& rt = a.tab[c.rowtab0 + lr];
      const double SS = Sa * Sb, F = FR * SS;
      const double I = rt.q2 * (F * F);
      if (a.intensity) a.intensity[c.px_off + idx] = I;
      if (a.counts) {
        const double pa = c.ua[0] * mx + c.ua[1] * my, pb = c.ub[0] * mx + c.ub[1] * my;
        const double ra = c.ua[1] * mx - c.ua[0] * my, rb = c.ub[1] * mx - c.ub[0] * my;
        const double dSSa = dSa * pa * Sb + Sa * dSb * pb;
        const double dSSp = c.a * (dSa * ra * Sb + Sa * dSb * rb);
        const double FRF = FR * F;
        const double C = a.counts[c.px_off + idx];
        const double mk = a.mask ? (double)a.mask[c.px_off + idx] : 1.0;
        const double w = mk / (C > 1.0 ? C : 1.0);
        const double res = c.scale * I - C;
        const double g = 2.0 * w * res * c.scale;
        acc[0] += w * res * res;
        acc[1] += g * (2.0 * rt.q2 * F * FRR * SS);
        acc[2] += g * (2.0 * rt.qh * F * F);
        acc[3] += g * (2.0 * FRF * (rt.q2 * dSSa + rt.qa * SS));
        acc[4] += g * (2.0 * rt.q2 * FRF * dSSp);
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

// The FP32C form.  FP64: the rotated q (mx, my), q_par and the table coordinate, the lattice
// turns and N t (reduced with round_fp64), the residual s I - C and the sums over threads and
// items.  FP32: the radial sums interpolated from the (hi, lo) tables, the Dirichlet kernels
// (own sincospi on the FMA pipe) and all derivative products, and each thread's sums over its
// PPT pixels.  The row scalar q2 multiplies (Fr Sa Sb)^2 in FP64, so no rounding common to
// many pixels (a row or candidate constant) reaches I: the chi^2 gradient sums residuals of
// both signs over the detector, and such an error would add up where the residuals cancel.
// Row and column advance by integer steps (no division per pixel); weights w come from a
// per-pixel FP32 array made once when the batch is created.
template <int NT, int PPT>
__global__ void __launch_bounds__(NT) cyl_pixels_f32c_kernel(CylArgs a) {
  __shared__ double sh[(NT / 32) * 5];
  for (long it = blockIdx.x; it < a.nitems; it += gridDim.x) {
    const int2 item = a.items[it];
    const CylCand& c = a.cands[item.x];
    const int ncols = c.ncols;
    const long npx = (long)c.nrows * ncols;
    const int first = item.y + threadIdx.x;
    int lr = first / ncols, lc = first - lr * ncols;
    const int dq = NT / ncols, dr = NT - dq * ncols;
    float acc[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
      if (j > 0) {
        lr += dq;
        lc += dr;
        if (lc >= ncols) {
          lc -= ncols;
          ++lr;
        }
      }
      const long idx = (long)first + (long)j * NT;
      if (idx >= npx) continue;
      const long p = (long)(c.row0 + lr) * a.grid_ncol + (c.col0 + lc);
      const double qx = __ldg(a.qx + p), qy = __ldg(a.qy + p);
      // the pixel's counts and weight issued early (read-only loads, independent of the math)
      double C = 0.0;
      float w = 0.0f;
      if (a.counts) {
        C = __ldg(a.counts + c.px_off + idx);
        w = __ldg(a.wf + c.px_off + idx);
      }
      const double mx = c.cphi * qx - c.sphi * qy, my = c.sphi * qx + c.cphi * qy;
      const double q2d = mx * mx + my * my;
      float FR = 0.f, FRR = 0.f;
      if (q2d * c.rmin * c.rmin > 1.0e-13) {
        // node below u = q_par / h + 1 by the FP64 rounding constant (its low word is the index)
        const double u = sqrt(q2d) * a.inv_h + 1.0;
        const double rb = __dadd_rn(__dadd_rn(u, -0.5), RND52);
        const int k = __double2loint(rb), i0 = min(max(k, 1), CYL_NTAB - 3);
        float t = (float)(u - __dsub_rn(rb, RND52));
        if (i0 != k) t += (float)(k - i0);
        const float w0 = -t * (t - 1.0f) * (t - 2.0f) * (1.0f / 6.0f);
        const float w1 = (t + 1.0f) * (t - 1.0f) * (t - 2.0f) * 0.5f;
        const float w2 = -(t + 1.0f) * t * (t - 2.0f) * 0.5f;
        const float w3 = (t + 1.0f) * t * (t - 1.0f) * (1.0f / 6.0f);
        const float4* tb = a.table + (long)item.x * CYL_NTAB + (i0 - 1);
        const float4 f0 = __ldg(tb), f1 = __ldg(tb + 1), f2 = __ldg(tb + 2), f3 = __ldg(tb + 3);
        FR = (w0 * f0.x + w1 * f1.x + w2 * f2.x + w3 * f3.x) + (w0 * f0.y + w1 * f1.y + w2 * f2.y + w3 * f3.y);
        FRR = (w0 * f0.z + w1 * f1.z + w2 * f2.z + w3 * f3.z) + (w0 * f0.w + w1 * f1.w + w2 * f2.w + w3 * f3.w);
      } else {  // the reference's q_par -> 0 guard: sum the terms that pass it
        const float qp = (float)sqrt(q2d);
        for (int i = 0; i < c.nr; ++i) {
          const float r = (float)c.r[i], x = qp * r;
          if ((double)x * (double)x > 1.0e-13) {
            const float two_pi_r = (float)(2.0 * PI_D) * r;
            FR += two_pi_r * r * j1f(x) / x;
            FRR += two_pi_r * r * j0f(x);
          }
        }
        FRR /= (float)c.R;
      }
      double ta = c.ka[0] * mx + c.ka[1] * my, tb = c.kb[0] * mx + c.kb[1] * my;
      ta -= round_fp64(ta);
      tb -= round_fp64(tb);
      float Sa, dSa, Sb, dSb;
      dirichlet_f32(ta, c.rep[0], c.frep[0], c.ser[0], &Sa, &dSa);
      dirichlet_f32(tb, c.rep[1], c.frep[1], c.ser[1], &Sb, &dSb);
      const RowTab* rt = a.tab + c.rowtab0 + lr;
      const float SS = Sa * Sb, F = FR * SS;
      const double I = __ldg(&rt->q2) * (double)(F * F);
      if (a.intensity) a.intensity[c.px_off + idx] = I;
      if (a.counts) {
        const float X = (float)mx, Y = (float)my;
        const float pa = c.fua[0] * X + c.fua[1] * Y, pb = c.fub[0] * X + c.fub[1] * Y;
        const float ra = c.fua[1] * X - c.fua[0] * Y, rb = c.fub[1] * X - c.fub[0] * Y;
        const float dSSa = dSa * pa * Sb + Sa * dSb * pb;
        const float dSSp = c.fa * (dSa * ra * Sb + Sa * dSb * rb);
        const float FRF = FR * F;
        const float q2f = __ldg(&rt->q2f), qhf = __ldg(&rt->qhf), qaf = __ldg(&rt->qaf);
        const float res = (float)(c.scale * I - C);
        const float g = 2.0f * w * res * c.fscale;
        acc[0] += w * res * res;
        acc[1] += g * (2.0f * q2f * F * FRR * SS);
        acc[2] += g * (2.0f * qhf * F * F);
        acc[3] += g * (2.0f * FRF * (q2f * dSSa + qaf * SS));
        acc[4] += g * (2.0f * q2f * FRF * dSSp);
      }
    }
    if (a.counts) {
      double accd[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) accd[q] = (double)acc[q];
      block_sum5<NT>(accd, sh);
      if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < 5; ++q) a.partial[5 * it + q] = accd[q];
    }
  }
}

// FP32C: the per-pixel weights mask / max(C, 1) as FP32, once per batch.
__global__ void cyl_weights_kernel(const double* __restrict__ counts, const unsigned* __restrict__ mask,
                                   long n, float* __restrict__ wf) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double C = counts[i];
    const double m = mask ? (double)mask[i] : 1.0;
    wf[i] = (float)(m / (C > 1.0 ? C : 1.0));
  }
}

// per-candidate sums of the items' partials, fixed order
// (block 0 also copies the context's device error word behind the results, so that one copy
// brings both back)
__global__ void cyl_final_kernel(const CylCand* __restrict__ cands, const double* __restrict__ partial,
                                 double* __restrict__ out, const unsigned* __restrict__ err, int ncand) {
  __shared__ double sh[(CYL_THREADS / 32) * 5];
  const CylCand& c = cands[blockIdx.x];
  double acc[5] = {0, 0, 0, 0, 0};
  for (long i = threadIdx.x; i < c.nitems; i += CYL_THREADS)
#pragma unroll
    for (int q = 0; q < 5; ++q) acc[q] += partial[5 * (c.item0 + i) + q];
  block_sum5<CYL_THREADS>(acc, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < 5; ++q) out[5 * blockIdx.x + q] = acc[q];
    if (blockIdx.x == 0) {
      double e = 0.0;
      *reinterpret_cast<unsigned*>(&e) = *err;
      out[5 * ncand] = e;
    }
  }
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
      if constexpr (std::is_same<T, float>::value) {
        if (occ)
          return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, cyl_pixels_f32c_kernel<NT, PPT>, NT, 0);
        cyl_pixels_f32c_kernel<NT, PPT><<<blocks, NT, 0, st>>>(a);
      } else {
        if (occ)
          return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, cyl_pixels_kernel<T, NT, PPT>, NT, 0);
        cyl_pixels_kernel<T, NT, PPT><<<blocks, NT, 0, st>>>(a);
      }
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
// Scaled power sums of the FP32C Dirichlet series (dirichlet_f32): with c_j = j - (N-1)/2,
// s_2k = sum_j c_j^2k (polynomials in N, exact for integer N: N(N^2-1)/12,
// N(N^2-1)(3N^2-7)/240, N(N^2-1)(3N^4-18N^2+31)/1344, N(N^2-1)(5N^6-55N^4+239N^2-381)/11520),
//   S  = N (1 - y e0 + y^2 e1 - y^3 e2 + y^4 e3),          e_k = s_2k+2 / ((2k+2)! N^(2k+3)),
//   dS = -theta N^3 (e4 - y e5 + y^2 e6 - y^3 e7),       e_4+k = s_2k+2 / ((2k+1)! N^(2k+3)),
// y = (theta N)^2 < 1; the first omitted term is below 3e-10 of N.
void cyl_dirichlet_series(double N, float* e) {
  for (int i = 0; i < 8; ++i) e[i] = 0.0f;
  if (N == 1.0) return;
  const double n2 = N * N, base = N * (n2 - 1.0);
  const double s[4] = {base / 12.0, base * (3.0 * n2 - 7.0) / 240.0,
                       base * (3.0 * n2 * n2 - 18.0 * n2 + 31.0) / 1344.0,
                       base * (5.0 * n2 * n2 * n2 - 55.0 * n2 * n2 + 239.0 * n2 - 381.0) / 11520.0};
  const double fs[4] = {2.0, 24.0, 720.0, 40320.0}, fd[4] = {1.0, 6.0, 120.0, 5040.0};
  double np = N * n2;  // N^(2k+3)
  for (int k = 0; k < 4; ++k, np *= n2) {
    e[k] = (float)(s[k] / (fs[k] * np));
    e[4 + k] = (float)(s[k] / (fd[k] * np));
  }
}

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
  c.fa = (float)c.a;
  for (int i = 0; i < 2; ++i) {
    c.ka[i] = c.a * c.ua[i] / (2.0 * PI_D);
    c.kb[i] = c.a * c.ub[i] / (2.0 * PI_D);
    c.fua[i] = (float)c.ua[i];
    c.fub[i] = (float)c.ub[i];
    c.frep[i] = (float)c.rep[i];
    cyl_dirichlet_series(c.rep[i], c.ser[i]);
  }
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
  c.fscale = (float)scale;
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
  hgx::DevBuf d_wf;     // FP32C per-pixel weights mask / max(counts, 1)
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
  // row table (a warp per row, 4 rows per block) and, in FP32C, the radial-sum tables (16
  // nodes per block) in one launch
  const int row_blocks = (maxrows + 3) / 4;
  const int table_blocks = b->precision == HGX_F32C ? (8 * CYL_NTAB + 127) / 128 : 0;
  cyl_prep_kernel<<<dim3(row_blocks + table_blocks, b->ncand), 128, 0, st>>>(
      (const CylCand*)b->d_cands.p, row_blocks, b->grid->rowqz, (const double2*)b->d_rowfc.p,
      (RowTab*)b->d_tab.p, b->table_h, (float4*)b->d_table.p);
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
  a.table = (const float4*)b->d_table.p;
  a.inv_h = 1.0 / b->table_h;
  a.wf = with_counts ? (const float*)b->d_wf.p : nullptr;
  long blocks = std::min<long>(b->nitems, (long)b->persistent_blocks);
  cudaError_t e = b->precision == HGX_F64
                      ? cyl_pixels_at<double, 0>(b->shape, (unsigned)blocks, a, st, nullptr)
                      : cyl_pixels_at<float, 0>(b->shape, (unsigned)blocks, a, st, nullptr);
  if (e != cudaSuccess) return cuda_fail(e, "cyl_pixels_kernel launch");
  if (with_counts) {
    cyl_final_kernel<<<b->ncand, CYL_THREADS, 0, st>>>((const CylCand*)b->d_cands.p,
                                                      (const double*)b->d_partial.p,
                                                      (double*)b->d_out.p, b->ctx->d_err, b->ncand);
    // the results and, behind them, the context's device error word (read after the one
    // synchronisation)
    HGX_CUDA(cudaMemcpyAsync(b->h_out, b->d_out.p, sizeof(double) * (5 * b->ncand + 1),
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
      cudaMallocHost(&b->h_out, sizeof(double) * (5 * ncand + 1)) != cudaSuccess)
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
      (s = b->d_out.reserve(sizeof(double) * (5 * ncand + 1))) || (s = b->d_rowfc.reserve(sizeof(double2) * 4 * g->nrow)) ||
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
    if ((s = b->d_table.reserve(sizeof(float4) * CYL_NTAB * (size_t)ncand))) return bail(s);
    if (counts) {
      if ((s = b->d_wf.reserve(sizeof(float) * px))) return bail(s);
      cyl_weights_kernel<<<(unsigned)std::min<long>((px + 255) / 256, 4L * c->sm_count * 8), 256, 0, st>>>(
          (const double*)b->d_counts.p, (const unsigned*)b->d_mask.p, px, (float*)b->d_wf.p);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return bail(cuda_fail(e, "hgx_cyl_batch_create: weights"));
    }
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
  unsigned err = 0;
  memcpy(&err, b->h_out + 5 * b->ncand, sizeof(unsigned));
  if (err) {  // as hgx_synchronize reports the context's device error bits
    cudaMemset(b->ctx->d_err, 0, sizeof(unsigned));
    return fail(HGX_ERR_DEVICE, "hgx_cyl_batch_eval: device error bits set by a kernel on this context");
  }
  for (int i = 0; i < 5 * b->ncand; ++i) out[i] = b->h_out[i];
  return HGX_OK;
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

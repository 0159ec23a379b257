// Triangle-mesh model in DWBA: the mesh -> triangle tuple conversion on the device, the
// chi^2 of the mesh's scattering, and its gradient with respect to every vertex coordinate
// by a hand-written adjoint.
//
// Conversion: ObjectShapeReader::get_triangle_params (src/file/objectshape_reader.cpp:275-300)
// — s = area, n = unit normal, c = centroid; degenerate triangles get s = 0 (the reference
// drops them, which is the same contribution).
//
// Forward: F_k(p) = (-i)/|q_k|^2 sum_t (q_k . n~_t) e^{i q_k . c_t}, n~ = s n (the FP32C row
// kernel), A(p) = w dn2 sum_k fc_k(row) F_k(p), I = |A|^2, chi^2 = sum m (s I - C)^2/max(C,1).
// Adjoint: with lambda_p = dchi^2/dI_p and H_pk = 2 lambda_p conj(A_p) w dn2 fc_k (-i)/|q_k|^2,
//   dchi^2 = Re sum_{p,k} H_pk dS_k(p),  S_k = sum_t (q_k . n~_t) e^{i q_k . c_t},
//   dchi^2/dn~_t = Re sum_{p,k} H_pk e^{i q_k . c_t} q_k,
//   dchi^2/dc_t  = -Im sum_{p,k} H_pk e^{i q_k . c_t} (q_k . n~_t) q_k.
// The backward pass recomputes the phases tile by tile (no per-triangle phases are stored):
// each CTA owns a tile of triangles and a chunk of detector rows; per (row, triangle) it
// forms the row phasors Z_0, Z_2 once; per pixel it combines the four blocks through the
// pairing qz_3 = -qz_0, qz_1 = -qz_2 (Z_3 = conj Z_0, Z_1 = conj Z_2):
//   Psi = sum_k H_k Z_k, Psi_z = sum_k qz_k H_k Z_k, Psi_zz = sum_k qz_k^2 H_k Z_k,
//   g_n~ += (Re(E Psi) qx, Re(E Psi) qy, Re(E Psi_z)),
//   g_c  -= (A Im(E Psi) + n~z Im(E Psi_z)) (qx, qy) and (A Im(E Psi_z) + n~z Im(E Psi_zz)),
// with E = e^{i(qx c'x + qy c'y)} and A = qx n~'x + qy n~'y in the rotated frame.  Per-chunk
// partial gradients are summed in a fixed order (deterministic), rotated back, and chained
// to the vertices: n~ = (v2 - v1) x (v3 - v1) / 2, c = (v1 + v2 + v3)/3.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <vector>

#include "cplx.cuh"
#include "hgx_internal.cuh"

namespace hgx {

constexpr double TWO_PI_M = 6.283185307179586476925286766559;
constexpr double INV_TWO_PI_M = 0.15915494309189533576888376337251;

// -------------------------------------------------------------- conversion ----
__global__ void mesh_to_shape_kernel(const double* __restrict__ v, int nv, const int* __restrict__ f,
                                     int nf, double* __restrict__ sd, unsigned* __restrict__ err) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nf) return;
  int i0 = f[3 * t], i1 = f[3 * t + 1], i2 = f[3 * t + 2];
  double* p = sd + 8L * t;
  if (i0 < 0 || i1 < 0 || i2 < 0 || i0 >= nv || i1 >= nv || i2 >= nv) {
    atomicOr(err, (unsigned)DEV_ERR_BAD_INDEX);
    for (int k = 0; k < 8; ++k) p[k] = 0.0;
    return;
  }
  const double *v1 = v + 3L * i0, *v2 = v + 3L * i1, *v3 = v + 3L * i2;
  double c[3] = {(v1[0] + v2[0] + v3[0]) / 3.0, (v1[1] + v2[1] + v3[1]) / 3.0,
                 (v1[2] + v2[2] + v3[2]) / 3.0};
  double a[3] = {v2[0] - v1[0], v2[1] - v1[1], v2[2] - v1[2]};
  double b[3] = {v3[0] - v1[0], v3[1] - v1[1], v3[2] - v1[2]};
  double na = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  double nb = sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
  double dot = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
  double cr[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
  double nc = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
  if (nc == 0 || na == 0 || nb == 0) {  // degenerate: contributes nothing
    for (int k = 0; k < 8; ++k) p[k] = 0.0;
    p[4] = c[0];
    p[5] = c[1];
    p[6] = c[2];
    return;
  }
  double sth = sqrt(1 - (dot / (na * nb)) * (dot / (na * nb)));
  p[0] = na * nb * sth / 2;
  p[1] = cr[0] / nc;
  p[2] = cr[1] / nc;
  p[3] = cr[2] / nc;
  p[4] = c[0];
  p[5] = c[1];
  p[6] = c[2];
  p[7] = 0.0;
}

// ------------------------------------------------------------ adjoint seeds ----
// Per pixel: A, I, chi^2 term, and the paired seeds (H0+H3, H0-H3, H2+H1, H2-H1) in FP32.
struct SeedArgs {
  const void* F;           // 4N form factor (complex64 for FP32C, complex128 for FP64)
  const double2* rowfc;    // nrow x 4
  const double2* rowqz;    // nrow x 4
  const double* qx;
  const double* qy;
  int nrow, ncol;
  double K[2];             // w * dn2
  double R[9];
  const double* counts;
  const unsigned* mask;
  double scale;
  void* seeds;             // 2 float4 (FP32C) or 2 double4 (FP64) per pixel
  double* intensity;       // may be NULL
  double* partial;         // chi^2 per block
};

__device__ __forceinline__ zd load_ff(const float2* F, long i) {
  const float2 f = F[i];
  return zd((double)f.x, (double)f.y);
}
__device__ __forceinline__ zd load_ff(const double2* F, long i) { return zd(F[i]); }
__device__ __forceinline__ void store_seeds(float4* S, long p, const zd* H) {
  S[2 * p] = make_float4((float)(H[0].x + H[3].x), (float)(H[0].y + H[3].y),
                         (float)(H[0].x - H[3].x), (float)(H[0].y - H[3].y));
  S[2 * p + 1] = make_float4((float)(H[2].x + H[1].x), (float)(H[2].y + H[1].y),
                             (float)(H[2].x - H[1].x), (float)(H[2].y - H[1].y));
}
__device__ __forceinline__ void store_seeds(double4* S, long p, const zd* H) {
  S[2 * p] = make_double4(H[0].x + H[3].x, H[0].y + H[3].y, H[0].x - H[3].x, H[0].y - H[3].y);
  S[2 * p + 1] = make_double4(H[2].x + H[1].x, H[2].y + H[1].y, H[2].x - H[1].x, H[2].y - H[1].y);
}

template <typename FT, typename ST>
__global__ void __launch_bounds__(256) mesh_seed_kernel(SeedArgs a) {
  __shared__ double red[8];
  long n = (long)a.nrow * a.ncol;
  long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double chi = 0.0;
  if (p < n) {
    long row = p / a.ncol;
    zd K(a.K[0], a.K[1]);
    zd A(0, 0);
    zd fcK[4];
    double q2[4];
    double qx = a.qx[p], qy = a.qy[p];
    for (int k = 0; k < 4; ++k) {
      fcK[k] = zd(a.rowfc[4 * row + k]) * K;
      A += fcK[k] * load_ff(static_cast<const FT*>(a.F), (long)k * n + p);
      double qz = a.rowqz[4 * row + k].x, s = 0.0;
      for (int j = 0; j < 3; ++j) {
        double m = a.R[3 * j] * qx + a.R[3 * j + 1] * qy + a.R[3 * j + 2] * qz;
        s += m * m;
      }
      q2[k] = s;
    }
    double I = A.x * A.x + A.y * A.y;
    if (a.intensity) a.intensity[p] = I;
    double lam = 0.0;
    if (a.counts) {
      double C = a.counts[p];
      double m = a.mask ? (double)a.mask[p] : 1.0;
      double w = m / (C > 1.0 ? C : 1.0);
      double r = a.scale * I - C;
      chi = w * r * r;
      lam = 2.0 * w * r * a.scale;
    }
    // H_k = 2 lam conj(A) fcK_k (-i) / q2_k
    zd base = conj(A) * (2.0 * lam);
    zd H[4];
    for (int k = 0; k < 4; ++k) {
      zd h = base * fcK[k];
      H[k] = zd(h.y, -h.x) / q2[k];  // times -i
    }
    store_seeds(static_cast<ST*>(a.seeds), p, H);
  }
  // block sum of chi^2 (fixed order)
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) chi += __shfl_down_sync(0xffffffffu, chi, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = chi;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += red[w];
    a.partial[blockIdx.x] = s;
  }
}

// ------------------------------------------------------------- backward pass ----
// One CTA per triangle tile of the forward (TRI_TILE triangles, 2 per thread) and chunk of rows.
// The tile's offsets d = c' - c0 carry the FP32 phases; the anchor phasor e^{i q_par.c0}
// (FP64 phase) is folded into the seeds when a pixel is staged, and the row phasors take the
// full z centroid c0z + dz in FP64.
constexpr int BW_THREADS = TRI_TILE / 2;
constexpr int BW_TPT = 2;                       // triangles per thread
constexpr int BW_TRI = BW_THREADS * BW_TPT;     // triangles per CTA = one forward tile
constexpr int BW_COLS = 256;                    // pixels staged per step
// In-plane phases of a staged chunk with |q_par| x (tile's largest offset) up to 8 pi go to the
// SFU without the explicit reduction, as in the forward row kernel (ff_tri.cu)
constexpr float BW_WIDE_PHASE2 = 631.65468f;     // (8 pi)^2

struct BwArgs {
  const float* tiles;        // the forward's FP32 tiles (offsets in nm, s n' components)
  const double4* anchors;    // per tile: c0x/2pi, c0y/2pi, c0z, max in-plane offset
  const int* perm;           // slot -> triangle (-1: padding)
  int ntri;
  const float4* seeds;
  const double* qx;
  const double* qy;
  const double2* rowqz;
  int nrow, ncol, rows_per_chunk;
  double* partial;           // [chunk][ntri][6]
};

__device__ __forceinline__ float4 rotate2(float4 v, float ca, float sa) {
  return make_float4(v.x * ca - v.y * sa, v.x * sa + v.y * ca, v.z * ca - v.w * sa,
                     v.z * sa + v.w * ca);
}

__global__ void __launch_bounds__(BW_THREADS) mesh_backward_kernel(BwArgs a) {
  __shared__ float4 s_px[BW_COLS * 3];  // (qx, qy, -, -), seeds 0, seeds 1 (anchor-rotated)
  const int TILE_T = TRI_TILE;          // the forward's tile layout
  const int tile = blockIdx.x;
  const int chunk = blockIdx.y;
  const int r0 = chunk * a.rows_per_chunk;
  const int r1 = min(a.nrow, r0 + a.rows_per_chunk);
  const double4 anc = a.anchors[tile];
  const double cz0 = anc.z * INV_TWO_PI_M;
  // this thread's triangles
  float cx[BW_TPT], cy[BW_TPT], cz[BW_TPT], nx[BW_TPT], ny[BW_TPT], nz[BW_TPT];
  double acc[BW_TPT][6];
  int orig[BW_TPT];
  const float* tl = a.tiles + (size_t)tile * TILE_T * 6;
#pragma unroll
  for (int u = 0; u < BW_TPT; ++u) {
    const int j = u * BW_THREADS + threadIdx.x;
    orig[u] = a.perm[(size_t)tile * TILE_T + j];
    float4 A = reinterpret_cast<const float4*>(tl)[j];
    float2 B = reinterpret_cast<const float2*>(tl + 4 * TILE_T)[j];
    cx[u] = A.x; nx[u] = A.y; cy[u] = A.z; ny[u] = A.w; cz[u] = B.x; nz[u] = B.y;  // (dx, nx, dy, ny)
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[u][q] = 0.0;
  }
  for (int row = r0; row < r1; ++row) {
    const double qz0 = a.rowqz[4L * row].x, qz2 = a.rowqz[4L * row + 2].x;
    const float fq0 = (float)qz0, fq2 = (float)qz2;
    // row phasors Z_0 = (x0, y0), Z_2 = (x2, y2) of each triangle, paired across the two block
    // pairs for the FP32x2 operations below: X = (x0, x2), Y = (y0, y2), Yn = -Y
    float2 X[BW_TPT], Y[BW_TPT], Yn[BW_TPT];
#pragma unroll
    for (int u = 0; u < BW_TPT; ++u) {
      const double czt = cz0 + (double)cz[u] * INV_TWO_PI_M;  // full z centroid, turns
      double w0 = qz0 * czt, w2 = qz2 * czt;
      w0 -= rint(w0);
      w2 -= rint(w2);
      float x0, y0, x2, y2;
      sincospif((float)(2.0 * w0), &y0, &x0);
      sincospif((float)(2.0 * w2), &y2, &x2);
      X[u] = make_float2(x0, x2);
      Y[u] = make_float2(y0, y2);
      Yn[u] = make_float2(-y0, -y2);
    }
    const float fq00 = fq0 * fq0, fq22 = fq2 * fq2;
    const float rmax2 = (float)(anc.w * anc.w);
    for (int c0 = 0; c0 < a.ncol; c0 += BW_COLS) {
      float part[BW_TPT][6];  // FP32 sums over one chunk of pixels, folded into FP64 below
#pragma unroll
      for (int u = 0; u < BW_TPT; ++u)
#pragma unroll
        for (int q = 0; q < 6; ++q) part[u][q] = 0.f;
      const int nc = min(BW_COLS, a.ncol - c0);
      __syncthreads();
      int wide = 0;  // some staged pixel has |q_par| x (tile's largest offset) above 8 pi
      for (int i = threadIdx.x; i < nc; i += BW_THREADS) {
        long p = (long)row * a.ncol + c0 + i;
        const double qx = a.qx[p], qy = a.qy[p];
        double w = fma(qx, anc.x, qy * anc.y);
        w -= rint(w);
        float sa, ca;
        sincospif((float)(2.0 * w), &sa, &ca);
        const float fx = (float)qx, fy = (float)qy;
        wide |= (fx * fx + fy * fy) * rmax2 > BW_WIDE_PHASE2;
        s_px[3 * i] = make_float4(fx, fy, 0.f, 0.f);
        // the seeds (P03, M03) and (P21, M21) interleaved, so that each FP32x2 operand below is
        // an aligned register pair of one shared-memory load: (P03r, P21r, P03i, P21i) and
        // (M03r, M21r, M03i, M21i)
        const float4 s03 = rotate2(a.seeds[2 * p], ca, sa), s21 = rotate2(a.seeds[2 * p + 1], ca, sa);
        s_px[3 * i + 1] = make_float4(s03.x, s21.x, s03.y, s21.y);
        s_px[3 * i + 2] = make_float4(s03.z, s21.z, s03.w, s21.w);
      }
      wide = __syncthreads_or(wide);
      for (int i = 0; i < nc; ++i) {
        const float4 q = s_px[3 * i];
        const float4 A = s_px[3 * i + 1], B = s_px[3 * i + 2];
        const float2 sx = make_float2(A.x, A.y), sy = make_float2(A.z, A.w);
        const float2 sz = make_float2(B.x, B.y), sw = make_float2(B.z, B.w);
#pragma unroll
        for (int u = 0; u < BW_TPT; ++u) {
          float tp = fmaf(q.x, cx[u], q.y * cy[u]);  // in-plane phase offset, radians
          if (wide) {  // reduced to [-pi, pi] before the SFU
            const float tt = tp * 0.159154943091895336f;
            tp = (tt - ((tt + 12582912.0f) - 12582912.0f)) * 6.28318530717958648f;
          }
          float sn, cs;
          __sincosf(tp, &sn, &cs);
          const float aq = fmaf(q.x, nx[u], q.y * ny[u]);
          // Psi_03 = P03 x0 + i M03 y0, B03 = M03 x0 + i P03 y0 (likewise 21), as pairs (03, 21)
          const float2 pr = __ffma2_rn(sw, Yn[u], __fmul2_rn(sx, X[u]));  // Re Psi
          const float2 pim = __ffma2_rn(sz, Y[u], __fmul2_rn(sy, X[u]));  // Im Psi
          const float2 br = __ffma2_rn(sy, Yn[u], __fmul2_rn(sz, X[u]));  // Re B
          const float2 bim = __ffma2_rn(sx, Y[u], __fmul2_rn(sw, X[u]));  // Im B
          const float psr = pr.x + pr.y, psi = pim.x + pim.y;
          const float pzr = fq0 * br.x + fq2 * br.y, pzi = fq0 * bim.x + fq2 * bim.y;
          const float pzzr = fq00 * pr.x + fq22 * pr.y, pzzi = fq00 * pim.x + fq22 * pim.y;
          // E * Psi etc.
          const float eR = cs * psr - sn * psi, eI = cs * psi + sn * psr;
          const float ezR = cs * pzr - sn * pzi, ezI = cs * pzi + sn * pzr;
          const float ezzI = cs * pzzi + sn * pzzr;
          part[u][0] = fmaf(eR, q.x, part[u][0]);
          part[u][1] = fmaf(eR, q.y, part[u][1]);
          part[u][2] += ezR;
          const float gxy = fmaf(aq, eI, nz[u] * ezI);
          part[u][3] = fmaf(-gxy, q.x, part[u][3]);
          part[u][4] = fmaf(-gxy, q.y, part[u][4]);
          part[u][5] -= fmaf(aq, ezI, nz[u] * ezzI);
        }
      }
#pragma unroll
      for (int u = 0; u < BW_TPT; ++u)
#pragma unroll
        for (int q = 0; q < 6; ++q) acc[u][q] += (double)part[u][q];
    }
  }
#pragma unroll
  for (int u = 0; u < BW_TPT; ++u) {
    if (orig[u] < 0) continue;
    double* dst = a.partial + ((size_t)chunk * a.ntri + orig[u]) * 6;
#pragma unroll
    for (int q = 0; q < 6; ++q) dst[q] = acc[u][q];
  }
}

// The plain FP64 backward pass (the FP64 reference of the FP32 one): triangles read from the
// FP64 tuples and rotated in the kernel, every phase and sum in FP64, same CTA layout
// (TRI_TILE triangles per CTA, 2 per thread) and chunking; partial gradients in the caller's
// triangle order.
constexpr int BW64_COLS = 128;

struct Bw64Args {
  const double* sd;          // ntri x 8 tuples
  int ntri;
  Rot9d R;
  const double4* seeds;      // 2 per pixel: (P03, M03), (P21, M21)
  const double* qx;
  const double* qy;
  const double2* rowqz;
  int nrow, ncol, rows_per_chunk;
  double* partial;           // [chunk][ntri][6]
};

__global__ void __launch_bounds__(BW_THREADS) mesh_backward_f64_kernel(Bw64Args a) {
  __shared__ double2 s_q[BW64_COLS];
  __shared__ double4 s_s[BW64_COLS * 2];
  const int chunk = blockIdx.y;
  const int r0 = chunk * a.rows_per_chunk;
  const int r1 = min(a.nrow, r0 + a.rows_per_chunk);
  double c[BW_TPT][3], nn[BW_TPT][3], acc[BW_TPT][6];
  int tri[BW_TPT];
#pragma unroll
  for (int u = 0; u < BW_TPT; ++u) {
    const int t = blockIdx.x * BW_TRI + u * BW_THREADS + threadIdx.x;
    tri[u] = t < a.ntri ? t : -1;
    const double* p = a.sd + 8L * (t < a.ntri ? t : 0);
    const double s = t < a.ntri ? p[0] : 0.0;
#pragma unroll
    for (int l = 0; l < 3; ++l) {
      nn[u][l] = s * (a.R.r[l] * p[1] + a.R.r[3 + l] * p[2] + a.R.r[6 + l] * p[3]);
      c[u][l] = a.R.r[l] * p[4] + a.R.r[3 + l] * p[5] + a.R.r[6 + l] * p[6];
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[u][q] = 0.0;
  }
  for (int row = r0; row < r1; ++row) {
    const double qz0 = a.rowqz[4L * row].x, qz2 = a.rowqz[4L * row + 2].x;
    double x0[BW_TPT], y0[BW_TPT], x2[BW_TPT], y2[BW_TPT];
#pragma unroll
    for (int u = 0; u < BW_TPT; ++u) {
      sincos(qz0 * c[u][2], &y0[u], &x0[u]);
      sincos(qz2 * c[u][2], &y2[u], &x2[u]);
    }
    for (int c0 = 0; c0 < a.ncol; c0 += BW64_COLS) {
      const int nc = min(BW64_COLS, a.ncol - c0);
      __syncthreads();
      for (int i = threadIdx.x; i < nc; i += BW_THREADS) {
        const long p = (long)row * a.ncol + c0 + i;
        s_q[i] = make_double2(a.qx[p], a.qy[p]);
        s_s[2 * i] = a.seeds[2 * p];
        s_s[2 * i + 1] = a.seeds[2 * p + 1];
      }
      __syncthreads();
      for (int i = 0; i < nc; ++i) {
        const double2 q = s_q[i];
        const double4 s03 = s_s[2 * i], s21 = s_s[2 * i + 1];
#pragma unroll
        for (int u = 0; u < BW_TPT; ++u) {
          double sn, cs;
          sincos(q.x * c[u][0] + q.y * c[u][1], &sn, &cs);
          const double aq = q.x * nn[u][0] + q.y * nn[u][1];
          const double p03r = s03.x * x0[u] - s03.w * y0[u], p03i = s03.y * x0[u] + s03.z * y0[u];
          const double b03r = s03.z * x0[u] - s03.y * y0[u], b03i = s03.w * x0[u] + s03.x * y0[u];
          const double p21r = s21.x * x2[u] - s21.w * y2[u], p21i = s21.y * x2[u] + s21.z * y2[u];
          const double b21r = s21.z * x2[u] - s21.y * y2[u], b21i = s21.w * x2[u] + s21.x * y2[u];
          const double psr = p03r + p21r, psi = p03i + p21i;
          const double pzr = qz0 * b03r + qz2 * b21r, pzi = qz0 * b03i + qz2 * b21i;
          const double pzzr = qz0 * qz0 * p03r + qz2 * qz2 * p21r;
          const double pzzi = qz0 * qz0 * p03i + qz2 * qz2 * p21i;
          const double eR = cs * psr - sn * psi, eI = cs * psi + sn * psr;
          const double ezR = cs * pzr - sn * pzi, ezI = cs * pzi + sn * pzr;
          const double ezzI = cs * pzzi + sn * pzzr;
          acc[u][0] += eR * q.x;
          acc[u][1] += eR * q.y;
          acc[u][2] += ezR;
          const double gxy = aq * eI + nn[u][2] * ezI;
          acc[u][3] -= gxy * q.x;
          acc[u][4] -= gxy * q.y;
          acc[u][5] -= aq * ezI + nn[u][2] * ezzI;
        }
      }
    }
  }
#pragma unroll
  for (int u = 0; u < BW_TPT; ++u) {
    if (tri[u] < 0) continue;
    double* dst = a.partial + ((size_t)chunk * a.ntri + tri[u]) * 6;
#pragma unroll
    for (int q = 0; q < 6; ++q) dst[q] = acc[u][q];
  }
}

// Sums the chunks (fixed order), rotates back to the mesh frame and writes per-triangle
// gradients with respect to n~ = s n and c:  g[t] = (g_n~ (3), g_c (3)).
__global__ void mesh_tri_grad_kernel(const double* __restrict__ partial, int nchunks, int ntri,
                                     Rot9d R, double* __restrict__ gtri) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntri) return;
  double g[6] = {0, 0, 0, 0, 0, 0};
  for (int c = 0; c < nchunks; ++c)
    for (int q = 0; q < 6; ++q) g[q] += partial[((size_t)c * ntri + t) * 6 + q];
  // the prep used n' = R^T n, c' = R^T c: dL/dn = R dL/dn'
  for (int v = 0; v < 2; ++v)
    for (int i = 0; i < 3; ++i)
      gtri[6L * t + 3 * v + i] =
          R.r[3 * i] * g[3 * v] + R.r[3 * i + 1] * g[3 * v + 1] + R.r[3 * i + 2] * g[3 * v + 2];
}

// Chain rule to vertices, gathered per vertex over its faces (CSR, deterministic):
// n~ = (a x b)/2, a = v2 - v1, b = v3 - v1:  dL/da = (b x g_n)/2, dL/db = (g_n x a)/2;
// c = (v1+v2+v3)/3.
__global__ void mesh_vertex_grad_kernel(const double* __restrict__ v, const int* __restrict__ f,
                                        const int* __restrict__ vptr, const int* __restrict__ vfaces,
                                        int nv, const double* __restrict__ gtri,
                                        double* __restrict__ gv) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  double out[3] = {0, 0, 0};
  for (int e = vptr[i]; e < vptr[i + 1]; ++e) {
    int fs = vfaces[e];
    int t = fs >> 2, slot = fs & 3;
    const int* F = f + 3L * t;
    const double *v1 = v + 3L * F[0], *v2 = v + 3L * F[1], *v3 = v + 3L * F[2];
    double a[3] = {v2[0] - v1[0], v2[1] - v1[1], v2[2] - v1[2]};
    double b[3] = {v3[0] - v1[0], v3[1] - v1[1], v3[2] - v1[2]};
    const double* gn = gtri + 6L * t;
    const double* gc = gn + 3;
    double ga[3] = {(b[1] * gn[2] - b[2] * gn[1]) / 2, (b[2] * gn[0] - b[0] * gn[2]) / 2,
                    (b[0] * gn[1] - b[1] * gn[0]) / 2};
    double gb[3] = {(gn[1] * a[2] - gn[2] * a[1]) / 2, (gn[2] * a[0] - gn[0] * a[2]) / 2,
                    (gn[0] * a[1] - gn[1] * a[0]) / 2};
    for (int k = 0; k < 3; ++k) {
      double d = gc[k] / 3.0;
      if (slot == 0) d -= ga[k] + gb[k];
      else if (slot == 1) d += ga[k];
      else d += gb[k];
      out[k] += d;
    }
  }
  for (int k = 0; k < 3; ++k) gv[3L * i + k] = out[k];
}

int ff_triangles_device(hgx_ctx c, hgx_qgrid g, const double* sd, int ntri, const double* rot9,
                        int precision, void* out, int ff_type, int want_p);

}  // namespace hgx

using namespace hgx;

extern "C" {

int hgx_mesh_to_shape_def(hgx_ctx c, int nv, const double* verts, int nf, const int* faces,
                          double* shape_def) {
  if (!c || !verts || !faces || !shape_def || nv < 1 || nf < 1)
    return fail(HGX_ERR_INVALID_ARG, "hgx_mesh_to_shape_def: null argument or empty mesh");
  HGX_CUDA(cudaSetDevice(c->device));
  DevBuf bv, bf, bo;
  const void *dv, *df;
  HGX_TRY(stage_in(c, verts, sizeof(double) * 3 * nv, bv, &dv));
  HGX_TRY(stage_in(c, faces, sizeof(int) * 3 * nf, bf, &df));
  void* dout = nullptr;
  HGX_TRY(stage_out(c, shape_def, sizeof(double) * 8 * nf, bo, &dout));
  mesh_to_shape_kernel<<<(nf + 127) / 128, 128, 0, c->stream>>>((const double*)dv, nv, (const int*)df,
                                                                nf, (double*)dout, c->d_err);
  HGX_CUDA(cudaGetLastError());
  HGX_TRY(finish_out(c, shape_def, sizeof(double) * 8 * nf, dout));
  return hgx_synchronize(c);
}

int hgx_mesh_chi2_grad_ex(hgx_ctx c, hgx_qgrid g, int nv, const double* verts, int nf,
                          const int* faces, const double* rot9, const double* rowfc,
                          double dn2_re, double dn2_im, double weight, const double* counts,
                          const unsigned* mask, double scale, double* chi2, double* grad_verts,
                          double* intensity, int precision) {
  if (!c || !g || !verts || !faces || !rowfc || !chi2 || nv < 3 || nf < 1)
    return fail(HGX_ERR_INVALID_ARG, "hgx_mesh_chi2_grad: null argument or empty mesh");
  if (precision != HGX_F32C && precision != HGX_F64)
    return fail(HGX_ERR_INVALID_ARG, "hgx_mesh_chi2_grad: unknown precision");
  const bool f64 = precision == HGX_F64;
  if (g->mode != 1)
    return fail(HGX_ERR_INVALID_ARG, "hgx_mesh_chi2_grad: needs a DWBA grid with real qz constant "
                                     "along rows (vacuum particle layer)");
  if (!counts && grad_verts)
    return fail(HGX_ERR_INVALID_ARG, "hgx_mesh_chi2_grad: the gradient needs counts");
  HGX_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  const long n = (long)g->nrow * g->ncol;
  static const double eye[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  const double* R = rot9 ? rot9 : eye;
  // inputs on the device
  if (!c->mesh) c->mesh = new (std::nothrow) MeshWork();
  if (!c->mesh) return fail(HGX_ERR_NO_MEMORY, "hgx_mesh_chi2_grad: host allocation");
  MeshWork& w = *c->mesh;
  DevBuf &bv = w.bv, &bf = w.bf, &bfc = w.bfc, &bc = w.bc, &bm = w.bm, &sd = w.sd, &F = w.F,
         &seeds = w.seeds, &part = w.part, &gtri = w.gtri, &vptr = w.vptr, &vfac = w.vfac,
         &gvb = w.gvb, &Ib = w.Ib;
  const void *dv, *df, *dfc, *dc = nullptr, *dm = nullptr;
  HGX_TRY(stage_in(c, verts, sizeof(double) * 3 * nv, bv, &dv));
  HGX_TRY(stage_in(c, faces, sizeof(int) * 3 * nf, bf, &df));
  HGX_TRY(stage_in(c, rowfc, sizeof(double2) * 4 * g->nrow, bfc, &dfc));
  HGX_TRY(stage_in(c, counts, sizeof(double) * n, bc, &dc));
  HGX_TRY(stage_in(c, mask, sizeof(unsigned) * n, bm, &dm));
  // 1. triangle tuples, 2. forward form factor (FP32C)
  HGX_TRY(sd.reserve(sizeof(double) * 8 * nf));
  mesh_to_shape_kernel<<<(nf + 127) / 128, 128, 0, st>>>((const double*)dv, nv, (const int*)df, nf,
                                                         (double*)sd.p, c->d_err);
  HGX_TRY(F.reserve((f64 ? sizeof(double2) : sizeof(float2)) * 4 * n));
  // FP32C: the scalar row kernel (4 pixels/thread), whose triangle tiles the backward pass
  // reads; FP64: the plain FP64 kernel
  HGX_TRY(ff_triangles_device(c, g, (const double*)sd.p, nf, R, precision, F.p,
                              f64 ? HGX_C128 : HGX_C64, 4));
  // 3. intensity, chi^2, seeds
  const int sblocks = (int)((n + 255) / 256);
  HGX_TRY(seeds.reserve((f64 ? sizeof(double4) : sizeof(float4)) * 2 * n));
  HGX_TRY(part.reserve(sizeof(double) * (sblocks + 1)));
  void* dI = nullptr;
  if (intensity) HGX_TRY(stage_out(c, intensity, sizeof(double) * n, Ib, &dI));
  SeedArgs sa;
  sa.F = F.p;
  sa.rowfc = (const double2*)dfc;
  sa.rowqz = g->rowqz;
  sa.qx = g->qx;
  sa.qy = g->qy;
  sa.nrow = g->nrow;
  sa.ncol = g->ncol;
  sa.K[0] = weight * dn2_re;
  sa.K[1] = weight * dn2_im;
  for (int i = 0; i < 9; ++i) sa.R[i] = R[i];
  sa.counts = (const double*)dc;
  sa.mask = (const unsigned*)dm;
  sa.scale = scale;
  sa.seeds = seeds.p;
  sa.intensity = (double*)dI;
  sa.partial = (double*)part.p;
  if (f64) mesh_seed_kernel<double2, double4><<<sblocks, 256, 0, st>>>(sa);
  else mesh_seed_kernel<float2, float4><<<sblocks, 256, 0, st>>>(sa);
  HGX_CUDA(cudaGetLastError());
  std::vector<double> hpart(sblocks);
  HGX_CUDA(cudaMemcpyAsync(hpart.data(), part.p, sizeof(double) * sblocks, cudaMemcpyDeviceToHost, st));
  if (grad_verts) {
    // 4. backward over (triangle tiles) x (row chunks): the FP32C forward's tiles, or the
    // FP64 tuples in blocks of 128
    const TileView tv = c->tiles;
    if (!f64 && (tv.ntri != nf || !tv.perm))
      return fail(HGX_ERR_INVALID_ARG, "hgx_mesh_chi2_grad: the forward left no triangle tiles");
    const int ntile = f64 ? (nf + BW_TRI - 1) / BW_TRI : tv.ntiles;
    int chunks = std::max(1, (c->sm_count * 16) / std::max(1, ntile));
    chunks = std::min(chunks, g->nrow);
    const int rpc = (g->nrow + chunks - 1) / chunks;
    chunks = (g->nrow + rpc - 1) / rpc;
    HGX_TRY(gtri.reserve(sizeof(double) * 6 * nf));
    DevBuf& bwpart = w.bwpart;
    HGX_TRY(bwpart.reserve(sizeof(double) * 6 * (size_t)nf * chunks));
    dim3 grid(ntile, chunks);
    if (f64) {
      Bw64Args ba;
      ba.sd = (const double*)sd.p;
      ba.ntri = nf;
      for (int i2 = 0; i2 < 9; ++i2) ba.R.r[i2] = R[i2];
      ba.seeds = (const double4*)seeds.p;
      ba.qx = g->qx;
      ba.qy = g->qy;
      ba.rowqz = g->rowqz;
      ba.nrow = g->nrow;
      ba.ncol = g->ncol;
      ba.rows_per_chunk = rpc;
      ba.partial = (double*)bwpart.p;
      mesh_backward_f64_kernel<<<grid, BW_THREADS, 0, st>>>(ba);
    } else {
      BwArgs ba;
      ba.tiles = tv.tiles;  // tiles left by the forward
      ba.anchors = tv.anchors;
      ba.perm = tv.perm;
      ba.ntri = nf;
      ba.seeds = (const float4*)seeds.p;
      ba.qx = g->qx;
      ba.qy = g->qy;
      ba.rowqz = g->rowqz;
      ba.nrow = g->nrow;
      ba.ncol = g->ncol;
      ba.rows_per_chunk = rpc;
      ba.partial = (double*)bwpart.p;
      mesh_backward_kernel<<<grid, BW_THREADS, 0, st>>>(ba);
    }
    HGX_CUDA(cudaGetLastError());
    Rot9d Rd;
    for (int i = 0; i < 9; ++i) Rd.r[i] = R[i];
    mesh_tri_grad_kernel<<<(nf + 127) / 128, 128, 0, st>>>((const double*)bwpart.p, chunks, nf, Rd,
                                                          (double*)gtri.p);
    // 5. vertex gather (CSR of vertex -> (face, slot) built on the host)
    std::vector<int> hf(3 * (size_t)nf);
    if (is_device_ptr(faces)) {
      HGX_CUDA(cudaMemcpyAsync(hf.data(), faces, sizeof(int) * 3 * nf, cudaMemcpyDeviceToHost, st));
      HGX_CUDA(cudaStreamSynchronize(st));
    } else {
      std::copy(faces, faces + 3 * (size_t)nf, hf.begin());
    }
    std::vector<int> ptr(nv + 1, 0), idx(3 * (size_t)nf);
    for (int e = 0; e < 3 * nf; ++e) {
      if (hf[e] < 0 || hf[e] >= nv) return fail(HGX_ERR_INVALID_ARG, "hgx_mesh_chi2_grad: bad face index");
      ptr[hf[e] + 1]++;
    }
    for (int i = 0; i < nv; ++i) ptr[i + 1] += ptr[i];
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    for (int t = 0; t < nf; ++t)
      for (int s = 0; s < 3; ++s) idx[fill[hf[3 * t + s]]++] = (t << 2) | s;
    HGX_TRY(vptr.reserve(sizeof(int) * (nv + 1)));
    HGX_TRY(vfac.reserve(sizeof(int) * 3 * (size_t)nf));
    HGX_CUDA(cudaMemcpyAsync(vptr.p, ptr.data(), sizeof(int) * (nv + 1), cudaMemcpyHostToDevice, st));
    HGX_CUDA(cudaMemcpyAsync(vfac.p, idx.data(), sizeof(int) * 3 * nf, cudaMemcpyHostToDevice, st));
    void* dgv = nullptr;
    HGX_TRY(stage_out(c, grad_verts, sizeof(double) * 3 * nv, gvb, &dgv));
    mesh_vertex_grad_kernel<<<(nv + 127) / 128, 128, 0, st>>>(
        (const double*)dv, (const int*)df, (const int*)vptr.p, (const int*)vfac.p, nv,
        (const double*)gtri.p, (double*)dgv);
    HGX_CUDA(cudaGetLastError());
    HGX_TRY(finish_out(c, grad_verts, sizeof(double) * 3 * nv, dgv));
  }
  if (intensity) HGX_TRY(finish_out(c, intensity, sizeof(double) * n, dI));
  HGX_TRY(hgx_synchronize(c));
  double s = 0.0;
  for (int b = 0; b < sblocks; ++b) s += hpart[b];
  *chi2 = s;
  return HGX_OK;
}

int hgx_mesh_chi2_grad(hgx_ctx c, hgx_qgrid g, int nv, const double* verts, int nf,
                       const int* faces, const double* rot9, const double* rowfc,
                       double dn2_re, double dn2_im, double weight, const double* counts,
                       const unsigned* mask, double scale, double* chi2, double* grad_verts,
                       double* intensity) {
  return hgx_mesh_chi2_grad_ex(c, g, nv, verts, nf, faces, rot9, rowfc, dn2_re, dn2_im, weight,
                               counts, mask, scale, chi2, grad_verts, intensity, HGX_F32C);
}

}  // extern "C"

// Numeric (triangulated-mesh) form factor:  F(q) = sum_t (-i)(q'.n_t) s_t e^{i q'.c_t} / |q'|^2,
// q' = R q — the reference's "approx triangle" formula (src/ff/cpu/ff_tri_cpu.cpp:233-240,
// src/ff/gpu/ff_tri_gpu.cu:371-384).
//
// Triangle tiles (FP32 kernels).  The triangles are put in Morton order of their centroids
// (a stable radix sort of 30-bit keys) and cut into tiles of 512, so that each tile covers a
// compact patch of the mesh.  Each tile carries an FP64 anchor c0 (the mean of its rotated
// centroids); the FP32 tile data hold only the offsets c' - c0.  Then
//   e^{i q.c'} = e^{i q.c0} e^{i q.(c' - c0)},
// where the anchor phase q.c0 is formed and range-reduced in FP64 once per (q-point, tile)
// and applied as one complex rotation of the tile's partial sums, and the FP32 phase per
// (q-point, triangle) only spans the tile's extent.  A mesh far from the origin therefore
// loses no phase accuracy, and when the tile's in-plane phases stay within a few turns (the
// warp's largest |q_par| times the tile's largest offset) the row kernel feeds them to the SFU
// without a per-term reduction.
//
// Kernels:
//  * ff_tri_f64_kernel     — the plain FP64 form: one thread per q-point, triangles staged
//                            through shared memory, reference arithmetic.  Parity reference
//                            on the device and the denominator of the FP32 speed-up.
//  * ff_tri_rows_kernel    — FP32, for q-grids laid out by detector rows (QGrid layout: qz
//                            depends on the row only).  The rotation is folded into the
//                            triangles (q'.c = q.(R^T c)), the phase splits into an in-plane
//                            part e^{i(qx c'x + qy c'y)} evaluated per (pixel, triangle) and a
//                            row part e^{i qz_k c'z} evaluated once per (row, triangle) and
//                            block k in FP64.  With the four real DWBA blocks (qz_3 = -qz_0,
//                            qz_1 = -qz_2) one in-plane sincos serves all four blocks.
//                            Triangle tiles arrive in shared memory by TMA bulk copies,
//                            double-buffered on mbarriers.  Sums are blocked per tile, rotated
//                            by the tile's anchor phasor and folded with TwoSum (compensated).
//  * ff_tri_rows_x2_kernel — the same with packed FP32x2 arithmetic (two pixels per lane pair).
//  * ff_tri_points_kernel  — FP32 for arbitrary q-point sets (one thread per q-point), the
//                            same tiles and anchors without the row factorisation.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <cub/device/device_radix_sort.cuh>
#include <mutex>

#include "hgx_internal.cuh"
#include "ptx.cuh"

namespace hgx {

constexpr int TILE = TRI_TILE;              // triangles per shared-memory tile (512)
constexpr int TILE_FLOATS = TILE * 6;       // float4 A[TILE] (dx,nx,dy,ny) + float2 B[TILE] (dz,nz)
constexpr uint32_t TILE_BYTES = TILE_FLOATS * 4;
constexpr int TILE_X2_FLOATS = TILE * 10;   // float4 A2[2*TILE] ((dx,dx,dy,dy),(nx,nx,ny,ny)) + float2 B[TILE]
constexpr uint32_t TILE_X2_BYTES = TILE_X2_FLOATS * 4;
constexpr double TWO_PI = 6.283185307179586476925286766559;
constexpr double INV_TWO_PI = 0.15915494309189533576888376337251;
constexpr float TWO_PI_F = 6.28318530717958648f;
constexpr float INV_TWO_PI_F = 0.159154943091895336f;
// In-plane phases of a tile with |q_par| * (largest offset) above 8 pi radians get the
// explicit reduction to [-1/2, 1/2] turn before the SFU; below it they go straight in (the SFU
// reduces its argument itself; its error grows with |x| by the rounding of x / 2 pi, about
// 2^-24 |x|, 1.5e-6 rad at 8 pi).
constexpr float WIDE_PHASE2 = 631.65468f;   // (8 pi)^2

struct Rot9 {
  double r[9];
};

// ------------------------------------------------------------- triangle prep ----
// Morton order: bounding box of the centroids (per-block partials, then one block), 30-bit
// keys, stable radix sort (cub), then one CTA per tile writes the tile and its anchor.
constexpr int BBOX_THREADS = 256;
constexpr int BBOX_MAX_BLOCKS = 256;

__device__ __forceinline__ void bbox_block_reduce(double* lo, double* hi, double (*s)[6]) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo[k] = fmin(lo[k], __shfl_down_sync(0xffffffffu, lo[k], o));
      hi[k] = fmax(hi[k], __shfl_down_sync(0xffffffffu, hi[k], o));
    }
  if (l == 0)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      s[w][k] = lo[k];
      s[w][3 + k] = hi[k];
    }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int v = 1; v < BBOX_THREADS / 32; ++v)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        lo[k] = fmin(lo[k], s[v][k]);
        hi[k] = fmax(hi[k], s[v][3 + k]);
      }
}

__global__ void __launch_bounds__(BBOX_THREADS) tri_bbox_kernel(const double* __restrict__ sd, int ntri,
                                                                double* __restrict__ part) {
  __shared__ double s[BBOX_THREADS / 32][6];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int t = blockIdx.x * BBOX_THREADS + threadIdx.x; t < ntri; t += gridDim.x * BBOX_THREADS)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double c = sd[8L * t + 4 + k];
      lo[k] = fmin(lo[k], c);
      hi[k] = fmax(hi[k], c);
    }
  bbox_block_reduce(lo, hi, s);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      part[6 * blockIdx.x + k] = lo[k];
      part[6 * blockIdx.x + 3 + k] = hi[k];
    }
}

__global__ void __launch_bounds__(BBOX_THREADS) tri_bbox_final_kernel(double* __restrict__ part,
                                                                      int nparts) {
  __shared__ double s[BBOX_THREADS / 32][6];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int b = threadIdx.x; b < nparts; b += BBOX_THREADS)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      lo[k] = fmin(lo[k], part[6 * b + k]);
      hi[k] = fmax(hi[k], part[6 * b + 3 + k]);
    }
  bbox_block_reduce(lo, hi, s);
  __syncthreads();  // every thread has read the partials before block 0's slot is overwritten
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      part[k] = lo[k];
      part[3 + k] = hi[k];
    }
}

// 10 bits of v spread to every third bit.
__device__ __forceinline__ unsigned spread3(unsigned v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

__global__ void tri_key_kernel(const double* __restrict__ sd, int ntri, const double* __restrict__ bbox,
                               unsigned* __restrict__ keys, int* __restrict__ idx) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntri) return;
  unsigned q[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double lo = bbox[k], ext = bbox[3 + k] - lo;
    double u = ext > 0.0 ? (sd[8L * t + 4 + k] - lo) / ext : 0.0;
    int b = (int)(u * 1024.0);
    q[k] = (unsigned)min(1023, max(0, b));
  }
  keys[t] = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
  idx[t] = t;
}

// One CTA (128 threads) per tile.  order: the triangle of each sorted slot (NULL: slot i holds
// triangle i).  Writes the tile (n~ = s R^T n, offsets d = R^T c - c0; the scalar layout
// float4 (dx, n~x, dy, n~y) + float2 (dz, n~z) in nm, so that (dx, n~x) and (dy, n~y) load as
// FP32x2 pairs; the packed layout in turns), its anchor (c0x/2pi, c0y/2pi, c0z, max |d_par|)
// and, when perm is not NULL, the triangle index of each slot (-1 for padding).  The anchor's
// sums run in a fixed order (deterministic).  Padding slots are zero (they contribute nothing).
template <bool X2>
__global__ void __launch_bounds__(TILE) tri_tile_kernel(const double* __restrict__ sd, int ntri, Rot9 R,
                                                        const int* __restrict__ order,
                                                        float* __restrict__ tiles,
                                                        double4* __restrict__ anchors,
                                                        int* __restrict__ perm) {
  __shared__ double s_red[TILE / 32][4];
  __shared__ double s_c0[3];
  __shared__ double s_rmax[TILE / 32];
  const int tile = blockIdx.x, j = threadIdx.x;
  const long pos = (long)tile * TILE + j;
  const int t = pos < ntri ? (order ? order[pos] : (int)pos) : -1;
  if (perm) perm[pos] = t;
  double s = 0.0, np[3] = {0.0, 0.0, 0.0}, cp[3] = {0.0, 0.0, 0.0};
  if (t >= 0) {
    const double* p = sd + 8L * t;
    s = p[0];
    double n[3] = {p[1], p[2], p[3]}, c[3] = {p[4], p[5], p[6]};
#pragma unroll
    for (int l = 0; l < 3; ++l) {
      np[l] = R.r[0 * 3 + l] * n[0] + R.r[1 * 3 + l] * n[1] + R.r[2 * 3 + l] * n[2];
      cp[l] = R.r[0 * 3 + l] * c[0] + R.r[1 * 3 + l] * c[1] + R.r[2 * 3 + l] * c[2];
    }
  }
  double v[4] = {cp[0], cp[1], cp[2], t >= 0 ? 1.0 : 0.0};
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if ((j & 31) == 0)
#pragma unroll
    for (int k = 0; k < 4; ++k) s_red[j >> 5][k] = v[k];
  __syncthreads();
  if (j == 0) {
    double sum[4] = {0.0, 0.0, 0.0, 0.0};
    for (int w = 0; w < TILE / 32; ++w)
#pragma unroll
      for (int k = 0; k < 4; ++k) sum[k] += s_red[w][k];
#pragma unroll
    for (int k = 0; k < 3; ++k) s_c0[k] = sum[k] / sum[3];  // every tile holds >= 1 triangle
  }
  __syncthreads();
  double d[3] = {0.0, 0.0, 0.0};
  if (t >= 0)
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = cp[k] - s_c0[k];
  double r = sqrt(d[0] * d[0] + d[1] * d[1]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, o));
  if ((j & 31) == 0) s_rmax[j >> 5] = r;
  __syncthreads();
  if (j == 0) {
    double rm = s_rmax[0];
    for (int w = 1; w < TILE / 32; ++w) rm = fmax(rm, s_rmax[w]);
    anchors[tile] = make_double4(s_c0[0] * INV_TWO_PI, s_c0[1] * INV_TWO_PI, s_c0[2], rm);
  }
  const double u = X2 ? INV_TWO_PI : 1.0;
  const float dx = (float)(d[0] * u), dy = (float)(d[1] * u), dz = (float)(d[2] * u);
  const float nx = (float)(s * np[0]), ny = (float)(s * np[1]), nz = (float)(s * np[2]);
  if (X2) {
    float4* A2 = reinterpret_cast<float4*>(tiles + (size_t)tile * TILE_X2_FLOATS);
    float2* B = reinterpret_cast<float2*>(tiles + (size_t)tile * TILE_X2_FLOATS + 8 * TILE);
    A2[2 * j] = make_float4(dx, dx, dy, dy);
    A2[2 * j + 1] = make_float4(nx, nx, ny, ny);
    B[j] = make_float2(dz, nz);
  } else {
    float4* A = reinterpret_cast<float4*>(tiles + (size_t)tile * TILE_FLOATS);
    float2* B = reinterpret_cast<float2*>(tiles + (size_t)tile * TILE_FLOATS + 4 * TILE);
    A[j] = make_float4(dx, nx, dy, ny);
    B[j] = make_float2(dz, nz);
  }
}

// ------------------------------------------------------------------ helpers ----
__device__ __forceinline__ void two_sum_fold(float& sum, float& part, float& comp) {
  float s = sum + part;
  float bp = s - sum;
  float err = (sum - (s - bp)) + (part - bp);
  sum = s;
  comp += err;
  part = 0.f;
}

// |R (qx, qy, qz)|^2 with complex qz, as RotMatrix_t::rotate + cuCnorm3 evaluate it.
__device__ __forceinline__ double rotated_q2(const Rot9& R, double qx, double qy, double2 qz) {
  double q2 = 0.0;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    double re = R.r[3 * j] * qx + R.r[3 * j + 1] * qy + R.r[3 * j + 2] * qz.x;
    double im = R.r[3 * j + 2] * qz.y;
    q2 += re * re + im * im;
  }
  return q2;
}

template <typename OUT>
__device__ __forceinline__ void store_ff(OUT* out, long idx, double re, double im);
template <>
__device__ __forceinline__ void store_ff<float2>(float2* out, long idx, double re, double im) {
  out[idx] = make_float2((float)re, (float)im);
}
template <>
__device__ __forceinline__ void store_ff<double2>(double2* out, long idx, double re, double im) {
  out[idx] = make_double2(re, im);
}

// The anchor phasor e^{2 pi i u} of an FP64 phase u in turns, reduced exactly in FP64.
__device__ __forceinline__ float2 anchor_phasor(double u) {
  u -= rint(u);
  float s, c;
  sincospif((float)(2.0 * u), &s, &c);
  return make_float2(c, s);
}

// (re, im) <- (re, im) * (c + i s)
__device__ __forceinline__ void rotate_pair(float& re, float& im, float2 a) {
  const float r = re * a.x - im * a.y;
  im = re * a.y + im * a.x;
  re = r;
}

// Rounds x to the nearest integer (ties to even) with two FP32 adds — valid for
// |x| < 2^22 — so the reduction stays on the FMA pipe instead of the conversion unit.
__device__ __forceinline__ float round_nearest(float x) {
  const float magic = 12582912.0f;  // 1.5 * 2^23
  return (x + magic) - magic;
}

// ------------------------------------------------------------- row kernel ----
struct RowArgs {
  const float* tiles;
  const double4* anchors;
  int ntiles;
  const double* qx;
  const double* qy;
  const double2* rowqz;  // nrow x NK
  int nqy, nrow, ncol, rows_per_cta;
  Rot9 R;
  void* out;
  unsigned* err;
};

// Row factor of one (row, triangle) for a real block pair (qz, -qz), cz in turns (FP64):
// Z = e^{i 2pi qz cz} = (x, y), D = qz n~z; returns (x, y, D*y, D*x).
__device__ __forceinline__ float4 paired_factor(double q, double cz, float nz) {
  double u = q * cz;
  u -= rint(u);
  float s, c;
  sincospif((float)(2.0 * u), &s, &c);
  float D = (float)(q * (double)nz);
  return make_float4(c, s, D * s, D * c);
}

// Row factor for a general complex block, cz in turns: Z = e^{i 2pi qz cz}, D = qz n~z;
// returns (Z, D Z).
__device__ __forceinline__ float4 complex_factor(double2 q, double cz, float nz) {
  double u = q.x * cz;
  u -= rint(u);
  double amp = exp(-TWO_PI * q.y * cz);
  double s, c;
  sincospi(2.0 * u, &s, &c);
  double zr = amp * c, zi = amp * s;
  double dr = q.x * (double)nz, di = q.y * (double)nz;
  return make_float4((float)zr, (float)zi, (float)(dr * zr - di * zi), (float)(dr * zi + di * zr));
}

// One tile's partial sums of the row kernel (see ff_tri_rows_kernel).  WIDE: the in-plane
// phases get the explicit reduction to [-1/2, 1/2] turn before the SFU.
template <int P, int NK, bool PAIRED, bool WIDE>
__device__ __forceinline__ void row_tile_sums(const float4* __restrict__ A, const float4* __restrict__ RF,
                                              const float (&qxf)[P], const float (&qyf)[P],
                                              float (&acc)[P][PAIRED ? 8 : 2 * NK]) {
  constexpr int NF = PAIRED ? 2 : NK;
#pragma unroll 2
  for (int j = 0; j < TILE; ++j) {
    const float4 t = A[j];
    float4 f[NF];
#pragma unroll
    for (int n = 0; n < NF; ++n) f[n] = RF[j * NF + n];
#pragma unroll
    for (int i = 0; i < P; ++i) {
      // (q_par.d, q_par.n~) as one FP32x2 multiply and one FP32x2 FMA
      const float2 pa = __ffma2_rn(make_float2(qxf[i], qxf[i]), make_float2(t.x, t.y),
                                   __fmul2_rn(make_float2(qyf[i], qyf[i]), make_float2(t.z, t.w)));
      float tp = pa.x;  // in-plane phase offset, radians
      if (WIDE) {
        float tt = tp * INV_TWO_PI_F;
        tp = (tt - round_nearest(tt)) * TWO_PI_F;  // reduced to [-pi, pi]
      }
      float sn, cs;
      __sincosf(tp, &sn, &cs);
      const float aq = pa.y;  // in-plane part of q.n~
      float ur = aq * cs, ui = aq * sn;            // U = aq * E
      if (PAIRED) {
#pragma unroll
        for (int pr = 0; pr < 2; ++pr) {
          const float4 g = f[pr];  // (x, y, beta, gamma)
          float* q = acc[i] + 4 * pr;
          q[0] = fmaf(g.x, ur, q[0]);
          q[0] = fmaf(-g.z, sn, q[0]);  // P.re += x Ur - beta s
          q[1] = fmaf(g.x, ui, q[1]);
          q[1] = fmaf(g.z, cs, q[1]);   // P.im += x Ui + beta c
          q[2] = fmaf(-g.y, ui, q[2]);
          q[2] = fmaf(g.w, cs, q[2]);   // M.re += -y Ui + gamma c
          q[3] = fmaf(g.y, ur, q[3]);
          q[3] = fmaf(g.w, sn, q[3]);   // M.im += y Ur + gamma s
        }
      } else {
#pragma unroll
        for (int k = 0; k < NK; ++k) {
          const float4 g = f[k];  // (Zr, Zi, DZr, DZi)
          float* q = acc[i] + 2 * k;
          q[0] = fmaf(ur, g.x, q[0]);
          q[0] = fmaf(-ui, g.y, q[0]);
          q[0] = fmaf(g.z, cs, q[0]);
          q[0] = fmaf(-g.w, sn, q[0]);
          q[1] = fmaf(ur, g.y, q[1]);
          q[1] = fmaf(ui, g.x, q[1]);
          q[1] = fmaf(g.z, sn, q[1]);
          q[1] = fmaf(g.w, cs, q[1]);
        }
      }
    }
  }
}

template <int BLOCK, int P, int NK, bool PAIRED, typename OUT>
__global__ void __launch_bounds__(BLOCK, 2) ff_tri_rows_kernel(RowArgs a) {
  constexpr int NF = PAIRED ? 2 : NK;        // float4 row factors per (row, triangle)
  constexpr int NACC = PAIRED ? 8 : 2 * NK;  // float accumulators per pixel
  __shared__ __align__(128) float s_tile[2][TILE_FLOATS];
  __shared__ __align__(8) uint64_t s_bar[2];
  // dynamic: row factors (rows_per_cta x TILE x NF float4), then the compensation terms of
  // the running sums (P x NACC x BLOCK floats, thread-minor so accesses are conflict-free)
  extern __shared__ __align__(16) float4 s_dyn[];
  float4* s_rf = s_dyn;
  float* s_cmp = reinterpret_cast<float*>(s_dyn + (size_t)a.rows_per_cta * TILE * NF);

  const int R = a.rows_per_cta;
  const int tpr = BLOCK / R;
  const int lr = threadIdx.x / tpr;
  const int lane = threadIdx.x - lr * tpr;
  const int row = blockIdx.y * R + lr;
  // each warp takes 32 x P neighbouring columns of its row (a thread's pixel i at lane + 32 i of
  // the warp's block), so that the largest |q_par| of the warp's own pixels decides the explicit
  // phase reduction: warps near the detector's qy = 0 column skip it on wide tiles
  const int colbase = blockIdx.x * (tpr * P) + (lane >> 5) * (32 * P) + (lane & 31);

  float qxf[P], qyf[P];
  float acc[P][NACC], sum[P][NACC];
  float q2l = 0.f;
#pragma unroll
  for (int i = 0; i < P; ++i) {
    int col = colbase + i * 32;
    bool v = row < a.nrow && col < a.ncol;
    long p = (long)row * a.ncol + col;
    qxf[i] = v ? (float)a.qx[p] : 0.f;
    qyf[i] = v ? (float)a.qy[p] : 0.f;
    q2l = fmaxf(q2l, fmaf(qxf[i], qxf[i], qyf[i] * qyf[i]));
#pragma unroll
    for (int n = 0; n < NACC; ++n) {
      acc[i][n] = sum[i][n] = 0.f;
      s_cmp[(i * NACC + n) * BLOCK + threadIdx.x] = 0.f;
    }
  }

  if (threadIdx.x == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int s = 0; s < 2 && s < a.ntiles; ++s) {
      mbar_arrive_expect_tx(&s_bar[s], TILE_BYTES);
      bulk_g2s(s_tile[s], a.tiles + (size_t)s * TILE_FLOATS, TILE_BYTES, &s_bar[s]);
    }
  }
  // the warp's largest |q_par|^2 (non-negative floats order as their bits)
  const float q2max = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(q2l)));

  for (int s = 0; s < a.ntiles; ++s) {
    const int b = s & 1;
    const double4 anc = a.anchors[s];
    const bool ok = mbar_wait(&s_bar[b], (s >> 1) & 1);
    const float4* A = reinterpret_cast<const float4*>(s_tile[b]);
    const float2* B = reinterpret_cast<const float2*>(s_tile[b] + 4 * TILE);
    if (ok) {
      // one float4 row factor per item: (row, triangle, pair or block); z phases in FP64
      const double cz0 = anc.z * INV_TWO_PI;
      for (int it = threadIdx.x; it < R * TILE * NF; it += BLOCK) {
        const int f = it % NF;
        const int rj = it / NF;
        const int r = rj / TILE, j = rj - r * TILE;
        const int grow = blockIdx.y * R + r;
        const float2 bz = B[j];
        const double cz = cz0 + (double)bz.x * INV_TWO_PI;
        float4 v;
        if (PAIRED) {
          v = grow < a.nrow ? paired_factor(a.rowqz[(long)grow * 4 + 2 * f].x, cz, bz.y)
                            : make_float4(1.f, 0.f, 0.f, 0.f);
        } else {
          v = grow < a.nrow ? complex_factor(a.rowqz[(long)grow * NK + f], cz, bz.y)
                            : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        s_rf[it] = v;  // == ((r * TILE + j) * NF + f)
      }
    }
    if (__syncthreads_or(!ok)) {
      // A bulk copy did not arrive in time: record it, wait (bounded) for the copies this
      // CTA still has in flight so none lands after exit, then leave.
      if (threadIdx.x == 0) {
        atomicOr(a.err, (unsigned)DEV_ERR_WAIT_TIMEOUT);
        mbar_wait(&s_bar[b], (s >> 1) & 1);
        if (s + 1 < a.ntiles) mbar_wait(&s_bar[b ^ 1], ((s + 1) >> 1) & 1);
      }
      __syncthreads();
      return;
    }

    const float4* RF = s_rf + (size_t)lr * TILE * NF;
    if ((float)(anc.w * anc.w) * q2max > WIDE_PHASE2)  // uniform over the warp
      row_tile_sums<P, NK, PAIRED, true>(A, RF, qxf, qyf, acc);
    else
      row_tile_sums<P, NK, PAIRED, false>(A, RF, qxf, qyf, acc);
    // rotate the tile's partial sums by the anchor phasor e^{i(qx c0x + qy c0y)} (FP64
    // phase), then fold them into the running sums (TwoSum; error terms in smem)
#pragma unroll
    for (int i = 0; i < P; ++i) {
      const int col = colbase + i * 32;
      const bool v = row < a.nrow && col < a.ncol;
      const long p = (long)row * a.ncol + col;
      const float2 e = anchor_phasor(v ? fma(a.qx[p], anc.x, a.qy[p] * anc.y) : 0.0);
#pragma unroll
      for (int n = 0; n < NACC; n += 2) rotate_pair(acc[i][n], acc[i][n + 1], e);
#pragma unroll
      for (int n = 0; n < NACC; ++n) {
        float* cp = s_cmp + (i * NACC + n) * BLOCK + threadIdx.x;
        float c = *cp;
        two_sum_fold(sum[i][n], acc[i][n], c);
        *cp = c;
      }
    }
    __syncthreads();  // every thread is done with tile buffer b and the row factors
    if (threadIdx.x == 0 && s + 2 < a.ntiles) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&s_bar[b], TILE_BYTES);
      bulk_g2s(s_tile[b], a.tiles + (size_t)(s + 2) * TILE_FLOATS, TILE_BYTES, &s_bar[b]);
    }
  }

  // epilogue: F_k = (-i) S_k / |R q_k|^2
  OUT* out = reinterpret_cast<OUT*>(a.out);
#pragma unroll
  for (int i = 0; i < P; ++i) {
    int col = colbase + i * 32;
    if (row >= a.nrow || col >= a.ncol) continue;
    long p = (long)row * a.ncol + col;
    double qx = a.qx[p], qy = a.qy[p];
    double T[NACC];
#pragma unroll
    for (int n = 0; n < NACC; ++n)
      T[n] = (double)sum[i][n] + (double)s_cmp[(i * NACC + n) * BLOCK + threadIdx.x];
#pragma unroll
    for (int k = 0; k < NK; ++k) {
      double sr, si;
      if (PAIRED) {
        // blocks 0,3 from pair 0 (P0 +- M0); blocks 2,1 from pair 2 (P2 +- M2)
        const int pr = (k == 0 || k == 3) ? 0 : 1;
        const double sg = (k == 0 || k == 2) ? 1.0 : -1.0;
        sr = T[4 * pr + 0] + sg * T[4 * pr + 2];
        si = T[4 * pr + 1] + sg * T[4 * pr + 3];
      } else {
        sr = T[2 * k];
        si = T[2 * k + 1];
      }
      double2 qz = a.rowqz[(long)row * NK + k];
      double q2 = rotated_q2(a.R, qx, qy, qz);
      store_ff<OUT>(out, (long)k * a.nqy + p, si / q2, -sr / q2);
    }
  }
}

// ------------------------------------------------------- packed row kernel ----
// The paired-block row kernel with Blackwell's packed FP32x2 arithmetic (__ffma2_rn,
// __fadd2_rn, __fmul2_rn): each thread carries its pixels in pairs, so one instruction
// advances two pixels.  Operands shared by both pixels of a pair (triangle data, row
// factors) are stored duplicated, (v, v), so they load as packed operands; the signs of
// the two negative terms are folded into a negated sine instead of negated operands.  Its
// tiles carry the offsets in turns and every phase is reduced explicitly.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

template <int BLOCK, int PP, typename OUT>
__global__ void __launch_bounds__(BLOCK) ff_tri_rows_x2_kernel(RowArgs a) {
  constexpr int NACC = 8;
  constexpr int P = 2 * PP;
  __shared__ __align__(128) float s_tile[2][TILE_X2_FLOATS];
  __shared__ __align__(8) uint64_t s_bar[2];
  // dynamic: row factors (rows_per_cta x TILE x 4 float4, duplicated), then the
  // compensation terms (P x NACC x BLOCK floats)
  extern __shared__ __align__(16) float4 s_dyn[];
  float4* s_rf = s_dyn;
  float* s_cmp = reinterpret_cast<float*>(s_dyn + (size_t)a.rows_per_cta * TILE * 4);

  const int R = a.rows_per_cta;
  const int tpr = BLOCK / R;
  const int lr = threadIdx.x / tpr;
  const int lane = threadIdx.x - lr * tpr;
  const int row = blockIdx.y * R + lr;
  const int colbase = blockIdx.x * (tpr * P) + lane;

  float2 qx2[PP], qy2[PP];
  float2 acc[PP][NACC], sum[PP][NACC];
#pragma unroll
  for (int pp = 0; pp < PP; ++pp) {
    float q[2][2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      int col = colbase + (2 * pp + c) * tpr;
      bool v = row < a.nrow && col < a.ncol;
      long p = (long)row * a.ncol + col;
      q[c][0] = v ? (float)a.qx[p] : 0.f;
      q[c][1] = v ? (float)a.qy[p] : 0.f;
    }
    qx2[pp] = f2(q[0][0], q[1][0]);
    qy2[pp] = f2(q[0][1], q[1][1]);
#pragma unroll
    for (int n = 0; n < NACC; ++n) {
      acc[pp][n] = sum[pp][n] = f2(0.f, 0.f);
      s_cmp[((pp * NACC + n) * 2 + 0) * BLOCK + threadIdx.x] = 0.f;
      s_cmp[((pp * NACC + n) * 2 + 1) * BLOCK + threadIdx.x] = 0.f;
    }
  }

  if (threadIdx.x == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int s = 0; s < 2 && s < a.ntiles; ++s) {
      mbar_arrive_expect_tx(&s_bar[s], TILE_X2_BYTES);
      bulk_g2s(s_tile[s], a.tiles + (size_t)s * TILE_X2_FLOATS, TILE_X2_BYTES, &s_bar[s]);
    }
  }

  const float M = 12582912.0f;  // 1.5 * 2^23: (t + M) - M rounds t to an integer
  for (int s = 0; s < a.ntiles; ++s) {
    const int b = s & 1;
    const double4 anc = a.anchors[s];
    const bool ok = mbar_wait(&s_bar[b], (s >> 1) & 1);
    const float4* A2 = reinterpret_cast<const float4*>(s_tile[b]);
    const float2* B = reinterpret_cast<const float2*>(s_tile[b] + 8 * TILE);
    if (ok) {
      // two duplicated float4 per (row, triangle, block pair): (x,x,y,y), (beta,beta,gamma,gamma)
      const double cz0 = anc.z * INV_TWO_PI;
      for (int it = threadIdx.x; it < R * TILE * 2; it += BLOCK) {
        const int f = it & 1;
        const int rj = it >> 1;
        const int r = rj / TILE, j = rj - r * TILE;
        const int grow = blockIdx.y * R + r;
        const float2 bz = B[j];
        float4 v = grow < a.nrow ? paired_factor(a.rowqz[(long)grow * 4 + 2 * f].x, cz0 + (double)bz.x, bz.y)
                                 : make_float4(1.f, 0.f, 0.f, 0.f);
        float4* dst = s_rf + (size_t)(r * TILE + j) * 4 + 2 * f;
        dst[0] = make_float4(v.x, v.x, v.y, v.y);
        dst[1] = make_float4(v.z, v.z, v.w, v.w);
      }
    }
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicOr(a.err, (unsigned)DEV_ERR_WAIT_TIMEOUT);
        mbar_wait(&s_bar[b], (s >> 1) & 1);
        if (s + 1 < a.ntiles) mbar_wait(&s_bar[b ^ 1], ((s + 1) >> 1) & 1);
      }
      __syncthreads();
      return;
    }

    const float4* RF = s_rf + (size_t)lr * TILE * 4;
#pragma unroll 2
    for (int j = 0; j < TILE; ++j) {
      const float4 c4 = A2[2 * j], n4 = A2[2 * j + 1];
      float4 rf[4];
#pragma unroll
      for (int n = 0; n < 4; ++n) rf[n] = RF[4 * j + n];
#pragma unroll
      for (int pp = 0; pp < PP; ++pp) {
        float2 tp = __ffma2_rn(qx2[pp], f2(c4.x, c4.y), __fmul2_rn(qy2[pp], f2(c4.z, c4.w)));
        float2 k = __fadd2_rn(__fadd2_rn(tp, f2(M, M)), f2(-M, -M));
        float2 rr = __ffma2_rn(k, f2(-1.f, -1.f), tp);  // exact reduction to [-1/2, 1/2]
        float2 ang = __fmul2_rn(rr, f2(TWO_PI_F, TWO_PI_F));
        float s0, c0, s1, c1;
        __sincosf(ang.x, &s0, &c0);
        __sincosf(ang.y, &s1, &c1);
        const float2 sn = f2(s0, s1), cs = f2(c0, c1);
        const float2 nsn = __fmul2_rn(sn, f2(-1.f, -1.f));
        float2 aq = __ffma2_rn(qx2[pp], f2(n4.x, n4.y), __fmul2_rn(qy2[pp], f2(n4.z, n4.w)));
        const float2 ur = __fmul2_rn(aq, cs), ui = __fmul2_rn(aq, sn), nui = __fmul2_rn(aq, nsn);
#pragma unroll
        for (int pr = 0; pr < 2; ++pr) {
          const float4 xy = rf[2 * pr], bg = rf[2 * pr + 1];
          const float2 X = f2(xy.x, xy.y), Y = f2(xy.z, xy.w), Bt = f2(bg.x, bg.y), G = f2(bg.z, bg.w);
          float2* q = acc[pp] + 4 * pr;
          q[0] = __ffma2_rn(Bt, nsn, __ffma2_rn(X, ur, q[0]));  // P.re += x Ur - beta s
          q[1] = __ffma2_rn(Bt, cs, __ffma2_rn(X, ui, q[1]));   // P.im += x Ui + beta c
          q[2] = __ffma2_rn(G, cs, __ffma2_rn(Y, nui, q[2]));   // M.re += -y Ui + gamma c
          q[3] = __ffma2_rn(G, sn, __ffma2_rn(Y, ur, q[3]));    // M.im += y Ur + gamma s
        }
      }
    }
#pragma unroll
    for (int pp = 0; pp < PP; ++pp)
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int col = colbase + (2 * pp + c) * tpr;
        const bool v = row < a.nrow && col < a.ncol;
        const long p = (long)row * a.ncol + col;
        const float2 e = anchor_phasor(v ? fma(a.qx[p], anc.x, a.qy[p] * anc.y) : 0.0);
#pragma unroll
        for (int n = 0; n < NACC; n += 2) {
          float& re = c ? acc[pp][n].y : acc[pp][n].x;
          float& im = c ? acc[pp][n + 1].y : acc[pp][n + 1].x;
          rotate_pair(re, im, e);
        }
      }
#pragma unroll
    for (int pp = 0; pp < PP; ++pp)
#pragma unroll
      for (int n = 0; n < NACC; ++n) {
        float* cp0 = s_cmp + ((pp * NACC + n) * 2 + 0) * BLOCK + threadIdx.x;
        float* cp1 = s_cmp + ((pp * NACC + n) * 2 + 1) * BLOCK + threadIdx.x;
        float c0 = *cp0, c1 = *cp1;
        two_sum_fold(sum[pp][n].x, acc[pp][n].x, c0);
        two_sum_fold(sum[pp][n].y, acc[pp][n].y, c1);
        *cp0 = c0;
        *cp1 = c1;
      }
    __syncthreads();
    if (threadIdx.x == 0 && s + 2 < a.ntiles) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&s_bar[b], TILE_X2_BYTES);
      bulk_g2s(s_tile[b], a.tiles + (size_t)(s + 2) * TILE_X2_FLOATS, TILE_X2_BYTES, &s_bar[b]);
    }
  }

  OUT* out = reinterpret_cast<OUT*>(a.out);
#pragma unroll
  for (int pp = 0; pp < PP; ++pp)
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      int col = colbase + (2 * pp + c) * tpr;
      if (row >= a.nrow || col >= a.ncol) continue;
      long p = (long)row * a.ncol + col;
      double qx = a.qx[p], qy = a.qy[p];
      double T[NACC];
#pragma unroll
      for (int n = 0; n < NACC; ++n)
        T[n] = (double)(c ? sum[pp][n].y : sum[pp][n].x) +
               (double)s_cmp[((pp * NACC + n) * 2 + c) * BLOCK + threadIdx.x];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int pr = (k == 0 || k == 3) ? 0 : 1;
        const double sg = (k == 0 || k == 2) ? 1.0 : -1.0;
        double sr = T[4 * pr + 0] + sg * T[4 * pr + 2];
        double si = T[4 * pr + 1] + sg * T[4 * pr + 3];
        double2 qz = a.rowqz[(long)row * 4 + k];
        double q2 = rotated_q2(a.R, qx, qy, qz);
        store_ff<OUT>(out, (long)k * a.nqy + p, si / q2, -sr / q2);
      }
    }
}

// ----------------------------------------------------------- points kernel ----
struct PointArgs {
  const float* tiles;
  const double4* anchors;
  int ntiles;
  const double* qx;
  const double* qy;
  const double2* qz;
  int nqy, nqz;
  Rot9 R;
  void* out;
  unsigned* err;
};

template <int BLOCK, typename OUT>
__global__ void __launch_bounds__(BLOCK) ff_tri_points_kernel(PointArgs a) {
  __shared__ __align__(128) float s_tile[2][TILE_FLOATS];
  __shared__ __align__(8) uint64_t s_bar[2];
  const long iz = (long)blockIdx.x * BLOCK + threadIdx.x;
  const bool valid = iz < a.nqz;
  float qxf = 0.f, qyf = 0.f, qzr = 0.f, qzi = 0.f;
  double qxd = 0.0, qyd = 0.0, qzd = 0.0, qzid = 0.0;
  if (valid) {
    long iy = iz % a.nqy;
    qxd = a.qx[iy];
    qyd = a.qy[iy];
    double2 q = a.qz[iz];
    qzd = q.x;
    qzid = q.y;
    qxf = (float)qxd;
    qyf = (float)qyd;
    qzr = (float)q.x;
    qzi = (float)q.y;
  }
  float acc[2] = {0.f, 0.f}, sum[2] = {0.f, 0.f}, cmp[2] = {0.f, 0.f};

  if (threadIdx.x == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int s = 0; s < 2 && s < a.ntiles; ++s) {
      mbar_arrive_expect_tx(&s_bar[s], TILE_BYTES);
      bulk_g2s(s_tile[s], a.tiles + (size_t)s * TILE_FLOATS, TILE_BYTES, &s_bar[s]);
    }
  }
  for (int s = 0; s < a.ntiles; ++s) {
    const int b = s & 1;
    const double4 anc = a.anchors[s];
    const bool ok = mbar_wait(&s_bar[b], (s >> 1) & 1);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicOr(a.err, (unsigned)DEV_ERR_WAIT_TIMEOUT);
        mbar_wait(&s_bar[b], (s >> 1) & 1);
        if (s + 1 < a.ntiles) mbar_wait(&s_bar[b ^ 1], ((s + 1) >> 1) & 1);
      }
      __syncthreads();
      return;
    }
    const float4* A = reinterpret_cast<const float4*>(s_tile[b]);
    const float2* B = reinterpret_cast<const float2*>(s_tile[b] + 4 * TILE);
#pragma unroll 4
    for (int j = 0; j < TILE; ++j) {
      const float4 t = A[j];
      const float2 z = B[j];
      float tt = fmaf(qzr, z.x, fmaf(qxf, t.x, qyf * t.z)) * INV_TWO_PI_F;  // turns
      float rr = tt - rintf(tt);
      float sn, cs;
      __sincosf(rr * TWO_PI_F, &sn, &cs);
      if (qzi != 0.f) {
        float amp = __expf(-qzi * z.x);
        sn *= amp;
        cs *= amp;
      }
      float ar = fmaf(qzr, z.y, fmaf(qxf, t.y, qyf * t.w));
      float ai = qzi * z.y;
      acc[0] = fmaf(ar, cs, acc[0]);
      acc[0] = fmaf(-ai, sn, acc[0]);
      acc[1] = fmaf(ar, sn, acc[1]);
      acc[1] = fmaf(ai, cs, acc[1]);
    }
    // the anchor e^{i q.c0} (FP64 phase, amplitude e^{-Im(qz) c0z}) on the tile's sums
    float2 e = anchor_phasor(fma(qxd, anc.x, fma(qyd, anc.y, qzd * anc.z * INV_TWO_PI)));
    if (qzid != 0.0) {
      const float amp0 = (float)exp(-qzid * anc.z);
      e.x *= amp0;
      e.y *= amp0;
    }
    rotate_pair(acc[0], acc[1], e);
    two_sum_fold(sum[0], acc[0], cmp[0]);
    two_sum_fold(sum[1], acc[1], cmp[1]);
    __syncthreads();
    if (threadIdx.x == 0 && s + 2 < a.ntiles) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&s_bar[b], TILE_BYTES);
      bulk_g2s(s_tile[b], a.tiles + (size_t)(s + 2) * TILE_FLOATS, TILE_BYTES, &s_bar[b]);
    }
  }
  if (!valid) return;
  long iy = iz % a.nqy;
  double q2 = rotated_q2(a.R, a.qx[iy], a.qy[iy], a.qz[iz]);
  double sr = (double)sum[0] + (double)cmp[0], si = (double)sum[1] + (double)cmp[1];
  store_ff<OUT>(reinterpret_cast<OUT*>(a.out), iz, si / q2, -sr / q2);
}

// -------------------------------------------------------------- FP64 kernel ----
constexpr int TILE64 = 64;

struct F64Args {
  const double* sd;  // T x 8
  int ntri;
  const double* qx;
  const double* qy;
  const double2* qz;
  int nqy, nqz;
  Rot9 R;
  void* out;
};

// The plain FP64 form: one thread per q-point, reference arithmetic
// (src/ff/gpu/ff_tri_gpu.cu:319-390) without its shared-memory race; 1/|q'|^2 is applied
// once per q-point instead of once per term.
template <int BLOCK, typename OUT>
__global__ void __launch_bounds__(BLOCK) ff_tri_f64_kernel(F64Args a) {
  __shared__ double s_sd[TILE64 * 8];
  const long iz = (long)blockIdx.x * BLOCK + threadIdx.x;
  const bool valid = iz < a.nqz;
  double2 m[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
  double q2 = 1.0;
  if (valid) {
    long iy = iz % a.nqy;
    double qx = a.qx[iy], qy = a.qy[iy];
    double2 qz = a.qz[iz];
    q2 = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      m[j].x = a.R.r[3 * j] * qx + a.R.r[3 * j + 1] * qy + a.R.r[3 * j + 2] * qz.x;
      m[j].y = a.R.r[3 * j + 2] * qz.y;
      q2 += m[j].x * m[j].x + m[j].y * m[j].y;
    }
  }
  const bool real_q = m[0].y == 0.0 && m[1].y == 0.0 && m[2].y == 0.0;
  double accr = 0.0, acci = 0.0;
  for (int t0 = 0; t0 < a.ntri; t0 += TILE64) {
    __syncthreads();
    const int nt = min(TILE64, a.ntri - t0);
    for (int k = threadIdx.x; k < nt * 8; k += BLOCK) s_sd[k] = a.sd[8L * t0 + k];
    __syncthreads();
    for (int j = 0; j < nt; ++j) {
      const double* p = s_sd + 8 * j;
      double s = p[0];
      double qnr = m[0].x * p[1] + m[1].x * p[2] + m[2].x * p[3];
      double qni = m[0].y * p[1] + m[1].y * p[2] + m[2].y * p[3];
      double qtr = m[0].x * p[4] + m[1].x * p[5] + m[2].x * p[6];
      double sn, cs;
      sincos(qtr, &sn, &cs);
      if (!real_q) {
        double qti = m[0].y * p[4] + m[1].y * p[5] + m[2].y * p[6];
        double e = exp(-qti);
        sn *= e;
        cs *= e;
      }
      // (-i) qn s = (qni s, -qnr s); times e^{i qt}
      double ar = qni * s, ai = -qnr * s;
      accr += ar * cs - ai * sn;
      acci += ar * sn + ai * cs;
    }
  }
  if (valid) store_ff<OUT>(reinterpret_cast<OUT*>(a.out), iz, accr / q2, acci / q2);
}

// ------------------------------------------------------------------ launch ----
static Rot9 make_rot(const double* r9) {
  Rot9 R;
  static const double eye[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int i = 0; i < 9; ++i) R.r[i] = r9 ? r9[i] : eye[i];
  return R;
}

template <int BLOCK, int P, int NK, bool PAIRED, typename OUT>
static int launch_rows(const RowArgs& a, dim3 grid, cudaStream_t st) {
  constexpr int NF = PAIRED ? 2 : NK;
  constexpr int NACC = PAIRED ? 8 : 2 * NK;
  size_t smem = (size_t)a.rows_per_cta * TILE * NF * sizeof(float4) +
                (size_t)P * NACC * BLOCK * sizeof(float);
  // static + dynamic shared memory may pass 48 KB: opt in for the dynamic part every time
  HGX_CUDA(cudaFuncSetAttribute(ff_tri_rows_kernel<BLOCK, P, NK, PAIRED, OUT>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  ff_tri_rows_kernel<BLOCK, P, NK, PAIRED, OUT><<<grid, BLOCK, smem, st>>>(a);
  HGX_CUDA(cudaGetLastError());
  return HGX_OK;
}

template <int BLOCK, int PP, typename OUT>
static int launch_rows_x2(const RowArgs& a, dim3 grid, cudaStream_t st) {
  size_t smem = (size_t)a.rows_per_cta * TILE * 4 * sizeof(float4) +
                (size_t)2 * PP * 8 * BLOCK * sizeof(float);
  // static + dynamic shared memory may pass 48 KB: opt in for the dynamic part every time
  HGX_CUDA(cudaFuncSetAttribute(ff_tri_rows_x2_kernel<BLOCK, PP, OUT>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  ff_tri_rows_x2_kernel<BLOCK, PP, OUT><<<grid, BLOCK, smem, st>>>(a);
  HGX_CUDA(cudaGetLastError());
  return HGX_OK;
}

template <int P, typename OUT>
static int dispatch_rows(const RowArgs& a, dim3 grid, int nk, bool paired, cudaStream_t st) {
  if (paired) return launch_rows<256, P, 4, true, OUT>(a, grid, st);
  if (nk == 4) return launch_rows<256, P, 4, false, OUT>(a, grid, st);
  return launch_rows<256, P, 1, false, OUT>(a, grid, st);
}

// Launch shape for the row kernel: P pixels per thread, threads per row a power of two
// (>= 64) covering the row when it is short, up to 4 rows per CTA in that case (the row
// factors of R rows x 512 triangles must fit the CTA's shared memory: at most 227 KB with the
// static tiles, the row factors and the compensation terms; the packed kernel with 8 pixels
// per thread keeps R <= 2).
struct RowShape {
  int P, tpr, R;
  dim3 grid;
};

static RowShape row_shape(int nrow, int ncol, int sm_count, int want_p, bool packed = false) {
  const int BLOCK = 256;
  RowShape best{};
  for (int P = want_p; P >= 1; P >>= 1) {
    int tpr = (packed && P >= 8) ? 128 : 64;
    while (tpr < BLOCK && tpr * P < ncol) tpr <<= 1;
    int R = BLOCK / tpr;
    dim3 g((ncol + tpr * P - 1) / (tpr * P), (nrow + R - 1) / R);
    best = RowShape{P, tpr, R, g};
    if ((long)g.x * g.y >= 2L * sm_count) break;  // enough CTAs to fill the GPU
  }
  return best;
}

// Scratch of the FP32 tile preparation, carved from the context's scratch buffer.
struct TilePrep {
  float* tiles = nullptr;
  double4* anchors = nullptr;
  int* perm = nullptr;
  unsigned* keys[2] = {nullptr, nullptr};
  int* idx[2] = {nullptr, nullptr};
  double* bbox = nullptr;
  void* sort_tmp = nullptr;
  size_t sort_bytes = 0;
};

static size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

// Prepares the tiles of ntri triangles (layout: scalar or packed) in Morton order, with
// their anchors and slot -> triangle map, on the context's stream; records them in c->tiles.
static int prepare_tiles(hgx_ctx c, const double* sd, int ntri, const Rot9& R, bool x2,
                         TilePrep* out) {
  cudaStream_t st = c->stream;
  const int ntiles = (ntri + TILE - 1) / TILE;
  const size_t tile_bytes = (size_t)ntiles * (x2 ? TILE_X2_BYTES : TILE_BYTES);
  const int nparts = std::min(BBOX_MAX_BLOCKS, (ntri + BBOX_THREADS - 1) / BBOX_THREADS);
  const bool sort = ntiles > 1;
  size_t sort_bytes = 0;
  if (sort) {
    HGX_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const unsigned*)nullptr,
                                             (unsigned*)nullptr, (const int*)nullptr, (int*)nullptr,
                                             ntri, 0, 30, st));
  }
  size_t off[9];
  size_t total = 0;
  const size_t sizes[9] = {tile_bytes,
                           sizeof(double4) * (size_t)ntiles,
                           sizeof(int) * (size_t)ntiles * TILE,
                           sort ? sizeof(unsigned) * (size_t)ntri : 0,
                           sort ? sizeof(unsigned) * (size_t)ntri : 0,
                           sort ? sizeof(int) * (size_t)ntri : 0,
                           sort ? sizeof(int) * (size_t)ntri : 0,
                           sort ? sizeof(double) * 6 * (size_t)nparts : 0,
                           sort_bytes};
  for (int i = 0; i < 9; ++i) {
    off[i] = total;
    total += align256(sizes[i]);
  }
  HGX_TRY(c->scratch.reserve(total));
  char* base = reinterpret_cast<char*>(c->scratch.p);
  TilePrep t;
  t.tiles = reinterpret_cast<float*>(base + off[0]);
  t.anchors = reinterpret_cast<double4*>(base + off[1]);
  t.perm = reinterpret_cast<int*>(base + off[2]);
  const int* order = nullptr;
  if (sort) {
    t.keys[0] = reinterpret_cast<unsigned*>(base + off[3]);
    t.keys[1] = reinterpret_cast<unsigned*>(base + off[4]);
    t.idx[0] = reinterpret_cast<int*>(base + off[5]);
    t.idx[1] = reinterpret_cast<int*>(base + off[6]);
    t.bbox = reinterpret_cast<double*>(base + off[7]);
    t.sort_tmp = base + off[8];
    t.sort_bytes = sort_bytes;
    tri_bbox_kernel<<<nparts, BBOX_THREADS, 0, st>>>(sd, ntri, t.bbox);
    tri_bbox_final_kernel<<<1, BBOX_THREADS, 0, st>>>(t.bbox, nparts);
    tri_key_kernel<<<(ntri + 255) / 256, 256, 0, st>>>(sd, ntri, t.bbox, t.keys[0], t.idx[0]);
    HGX_CUDA(cudaGetLastError());
    size_t tb = sort_bytes;
    HGX_CUDA(cub::DeviceRadixSort::SortPairs(t.sort_tmp, tb, t.keys[0], t.keys[1], t.idx[0],
                                             t.idx[1], ntri, 0, 30, st));
    order = t.idx[1];
  }
  if (x2)
    tri_tile_kernel<true><<<ntiles, TILE, 0, st>>>(sd, ntri, R, order, t.tiles, t.anchors, t.perm);
  else
    tri_tile_kernel<false><<<ntiles, TILE, 0, st>>>(sd, ntri, R, order, t.tiles, t.anchors, t.perm);
  HGX_CUDA(cudaGetLastError());
  c->tiles = TileView{t.tiles, t.anchors, t.perm, ntiles, ntri};
  *out = t;
  return HGX_OK;
}

int ff_triangles_device(hgx_ctx c, hgx_qgrid g, const double* sd, int ntri, const double* rot9,
                        int precision, void* out, int ff_type, int want_p) {
  cudaStream_t st = c->stream;
  Rot9 R = make_rot(rot9);
  const bool c64 = ff_type == HGX_C64;
  if (precision == HGX_F64) {
    F64Args a{sd, ntri, g->qx, g->qy, g->qz, g->nqy, g->nqz, R, out};
    dim3 grid((g->nqz + 127) / 128);
    if (c64) ff_tri_f64_kernel<128, float2><<<grid, 128, 0, st>>>(a);
    else ff_tri_f64_kernel<128, double2><<<grid, 128, 0, st>>>(a);
    HGX_CUDA(cudaGetLastError());
    return HGX_OK;
  }
  if (want_p == 0) want_p = g->tuned_p;  // the autotuner's choice for this grid, if any
  if (want_p != 0 && want_p != 1 && want_p != 2 && want_p != 4 && want_p != -2 && want_p != -4 &&
      want_p != -8)
    return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles: pixels per thread must be 1, 2 or 4 (scalar) "
                                     "or -2, -4, -8 (packed)");
  const int ntiles = (ntri + TILE - 1) / TILE;
  // paired real DWBA blocks, packed FP32x2 kernel on request (want_p = -2, -4, -8 pixels per
  // thread); automatic (0) picks the scalar one.
  if (g->mode == 1 && want_p < 0) {
    const int P = -want_p;
    if (P != 2 && P != 4 && P != 8)
      return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles: packed kernel takes 2, 4 or 8 pixels per thread");
    RowShape sh = row_shape(g->nrow, g->ncol, c->sm_count, P, true);
    if (sh.P < 2) sh = row_shape(g->nrow, g->ncol, 0, 2, true);  // keep at least one pair
    if (sh.grid.y > 65535u)
      return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles: too many detector rows for one launch");
    TilePrep t;
    HGX_TRY(prepare_tiles(c, sd, ntri, R, true, &t));
    RowArgs a{t.tiles, t.anchors, ntiles, g->qx, g->qy, g->rowqz, g->nqy, g->nrow, g->ncol, sh.R, R,
              out, c->d_err};
    switch (sh.P) {
      case 8:
        return c64 ? launch_rows_x2<256, 4, float2>(a, sh.grid, st) : launch_rows_x2<256, 4, double2>(a, sh.grid, st);
      case 4:
        return c64 ? launch_rows_x2<256, 2, float2>(a, sh.grid, st) : launch_rows_x2<256, 2, double2>(a, sh.grid, st);
      default:
        return c64 ? launch_rows_x2<256, 1, float2>(a, sh.grid, st) : launch_rows_x2<256, 1, double2>(a, sh.grid, st);
    }
  }
  // FP32 scalar kernels
  if (g->mode == 0) {
    TilePrep t;
    HGX_TRY(prepare_tiles(c, sd, ntri, R, false, &t));
    PointArgs a{t.tiles, t.anchors, ntiles, g->qx, g->qy, g->qz, g->nqy, g->nqz, R, out, c->d_err};
    dim3 grid((g->nqz + 127) / 128);
    if (c64) ff_tri_points_kernel<128, float2><<<grid, 128, 0, st>>>(a);
    else ff_tri_points_kernel<128, double2><<<grid, 128, 0, st>>>(a);
    HGX_CUDA(cudaGetLastError());
    return HGX_OK;
  }
  RowShape sh = row_shape(g->nrow, g->ncol, c->sm_count, want_p > 0 ? want_p : 4);
  if (sh.grid.y > 65535u)
    return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles: too many detector rows for one launch");
  TilePrep t;
  HGX_TRY(prepare_tiles(c, sd, ntri, R, false, &t));
  RowArgs a{t.tiles, t.anchors, ntiles, g->qx, g->qy, g->rowqz, g->nqy, g->nrow, g->ncol, sh.R, R,
            out, c->d_err};
  const bool paired = g->mode == 1;
  switch (sh.P) {
    case 4:
      return c64 ? dispatch_rows<4, float2>(a, sh.grid, g->nk, paired, st)
                 : dispatch_rows<4, double2>(a, sh.grid, g->nk, paired, st);
    case 2:
      return c64 ? dispatch_rows<2, float2>(a, sh.grid, g->nk, paired, st)
                 : dispatch_rows<2, double2>(a, sh.grid, g->nk, paired, st);
    default:
      return c64 ? dispatch_rows<1, float2>(a, sh.grid, g->nk, paired, st)
                 : dispatch_rows<1, double2>(a, sh.grid, g->nk, paired, st);
  }
}

static size_t esz_of(int ff_type) { return ff_type == HGX_C64 ? sizeof(float2) : sizeof(double2); }

// The triangle tuples on the device: the caller's array, or a copy in the context's staging.
static int stage_shape_def(hgx_ctx c, const double* shape_def, int ntri, const double** sd) {
  *sd = shape_def;
  if (is_device_ptr(shape_def)) return HGX_OK;
  HGX_TRY(c->staging.reserve(sizeof(double) * 8 * (size_t)ntri));
  HGX_CUDA(cudaMemcpyAsync(c->staging.p, shape_def, sizeof(double) * 8 * (size_t)ntri,
                           cudaMemcpyHostToDevice, c->stream));
  *sd = reinterpret_cast<const double*>(c->staging.p);
  return HGX_OK;
}

// Where the kernels write a form factor of `bytes` for the caller's ff: device memory itself;
// page-locked host memory mapped into the device's address space directly (the kernels' stores
// cross the bus while they run, so no copy follows them); other host memory through the
// context's output staging (*staged: the caller copies it back after the kernels).
static int output_view(hgx_ctx c, void* ff, size_t bytes, void** dout, bool* staged) {
  *staged = false;
  *dout = ff;
  if (is_device_ptr(ff)) return HGX_OK;
  if (void* m = mapped_host_ptr(ff)) {
    *dout = m;
    return HGX_OK;
  }
  HGX_TRY(c->shaped_out.reserve(bytes));
  *dout = c->shaped_out.p;
  *staged = true;
  return HGX_OK;
}

}  // namespace hgx

using namespace hgx;

extern "C" {

int hgx_ff_triangles_q_ex(hgx_ctx c, hgx_qgrid g, const double* shape_def, int ntri,
                         const double* rot9, int precision, void* ff, int ff_type, int pixels) {
  if (!c || !g || !shape_def || !ff)
    return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles_q: null argument");
  if (ntri < 1) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles_q: no triangles");
  if (precision != HGX_F64 && precision != HGX_F32C)
    return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles_q: unknown precision");
  if (ff_type != HGX_C128 && ff_type != HGX_C64)
    return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles_q: unknown output type");
  if (g->ctx != c) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles_q: grid of another context");
  HGX_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  const double* sd = nullptr;
  HGX_TRY(stage_shape_def(c, shape_def, ntri, &sd));
  const bool host_out = !is_device_ptr(ff);
  bool staged = false;
  void* dout = nullptr;
  HGX_TRY(output_view(c, ff, esz_of(ff_type) * (size_t)g->nqz, &dout, &staged));
  HGX_TRY(ff_triangles_device(c, g, sd, ntri, rot9, precision, dout, ff_type, pixels));
  if (staged) HGX_CUDA(cudaMemcpyAsync(ff, dout, esz_of(ff_type) * (size_t)g->nqz, cudaMemcpyDeviceToHost, st));
  return host_out ? hgx_synchronize(c) : HGX_OK;
}

int hgx_ff_triangles_q(hgx_ctx c, hgx_qgrid g, const double* shape_def, int ntri,
                       const double* rot9, int precision, void* ff, int ff_type) {
  return hgx_ff_triangles_q_ex(c, g, shape_def, ntri, rot9, precision, ff, ff_type, 0);
}

// The launch-shape autotuner of the FP32C row kernel.  Candidates, in this order: scalar
// kernel with 4, 2, 1 pixels per thread, then (paired real grids only) the packed FP32x2
// kernel with 2, 4, 8.  Each is run once untimed and then `reps` times between two CUDA
// events on the context's stream, on the caller's triangles (the cost of every candidate is
// linear in the triangle count, so a few thousand triangles rank them); the fastest is stored
// in the grid and used by later calls that ask for the automatic shape.
static const int TUNE_CANDIDATES[] = {4, 2, 1, -2, -4, -8};
constexpr int TUNE_NCAND = sizeof(TUNE_CANDIDATES) / sizeof(TUNE_CANDIDATES[0]);

int hgx_ff_tune(hgx_ctx c, hgx_qgrid g, const double* shape_def, int ntri, const double* rot9,
                int ff_type, int reps, int* best_ppt, double* best_ms, double* times_ms) {
  if (!c || !g || !shape_def) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_tune: null argument");
  if (ntri < 1) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_tune: no triangles");
  if (ff_type != HGX_C128 && ff_type != HGX_C64)
    return fail(HGX_ERR_INVALID_ARG, "hgx_ff_tune: unknown output type");
  if (g->ctx != c) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_tune: grid of another context");
  if (reps < 1) reps = 1;
  if (times_ms)
    for (int i = 0; i < TUNE_NCAND; ++i) times_ms[i] = 0.0;
  if (g->mode == 0) {  // per-q-point kernel: one launch shape, nothing to choose
    if (best_ppt) *best_ppt = 0;
    if (best_ms) *best_ms = 0.0;
    return HGX_OK;
  }
  HGX_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  const double* sd = shape_def;
  DevBuf sdbuf, out;
  if (!is_device_ptr(shape_def)) {
    HGX_TRY(sdbuf.reserve(sizeof(double) * 8 * (size_t)ntri));
    HGX_CUDA(cudaMemcpyAsync(sdbuf.p, shape_def, sizeof(double) * 8 * (size_t)ntri,
                             cudaMemcpyHostToDevice, st));
    sd = reinterpret_cast<const double*>(sdbuf.p);
  }
  const size_t esz = ff_type == HGX_C64 ? sizeof(float2) : sizeof(double2);
  HGX_TRY(out.reserve(esz * (size_t)g->nqz));
  struct Events {
    cudaEvent_t e[2] = {nullptr, nullptr};
    ~Events() {
      for (auto x : e)
        if (x) cudaEventDestroy(x);
    }
  } ev;
  HGX_CUDA(cudaEventCreate(&ev.e[0]));
  HGX_CUDA(cudaEventCreate(&ev.e[1]));
  int best = 0;
  double bms = 0.0;
  for (int i = 0; i < TUNE_NCAND; ++i) {
    const int p = TUNE_CANDIDATES[i];
    if (p < 0 && g->mode != 1) continue;
    HGX_TRY(ff_triangles_device(c, g, sd, ntri, rot9, HGX_F32C, out.p, ff_type, p));
    HGX_CUDA(cudaEventRecord(ev.e[0], st));
    for (int r = 0; r < reps; ++r)
      HGX_TRY(ff_triangles_device(c, g, sd, ntri, rot9, HGX_F32C, out.p, ff_type, p));
    HGX_CUDA(cudaEventRecord(ev.e[1], st));
    HGX_CUDA(cudaEventSynchronize(ev.e[1]));
    float ms = 0.f;
    HGX_CUDA(cudaEventElapsedTime(&ms, ev.e[0], ev.e[1]));
    double per = (double)ms / reps;
    if (times_ms) times_ms[i] = per;
    if (best == 0 || per < bms) {
      best = p;
      bms = per;
    }
  }
  HGX_TRY(hgx_synchronize(c));  // device errors of the timed launches
  g->tuned_p = best;
  if (best_ppt) *best_ppt = best;
  if (best_ms) *best_ms = bms;
  return HGX_OK;
}

int hgx_ff_triangles(hgx_ctx c, const double* shape_def, int ntri, int nqy, const double* qx,
                     const double* qy, int nqz, const double* qz, const double* rot9,
                     int precision, double* ff) {
  if (ntri < 1) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles: no triangles");
  if (!c) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles: null context");
  HGX_CUDA(cudaSetDevice(c->device));
  hgx_qgrid g = nullptr;
  bool rows_first = false;
  if (precision == HGX_F32C && shape_def && ff && qx && qy && qz)
    HGX_TRY(shaped_rows_begin(c, nqy, qx, qy, nqz, qz, &g, &rows_first));
  else
    HGX_TRY(shaped_grid(c, nqy, qx, qy, nqz, qz, &g));
  if (!rows_first) {
    int s = hgx_ff_triangles_q(c, g, shape_def, ntri, rot9, precision, ff, HGX_C128);
    if (s == HGX_OK && is_device_ptr(ff)) s = hgx_synchronize(c);
    return s;
  }
  // The row kernel runs from qx, qy and the row table while the side stream copies the 4N qz
  // values and checks them; a grid that fails the check (qz not constant along its rows, or
  // blocks that do not pair as the first q-points of the rows suggested) is finalized from the
  // full qz and the form factor computed again.
  const double* sd = nullptr;
  HGX_TRY(stage_shape_def(c, shape_def, ntri, &sd));
  bool staged = false;
  void* dout = nullptr;
  HGX_TRY(output_view(c, ff, sizeof(double2) * (size_t)nqz, &dout, &staged));
  int s = ff_triangles_device(c, g, sd, ntri, rot9, HGX_F32C, dout, HGX_C128, 0);
  const int s_check = shaped_rows_check(c, g, qz);
  bool ok = true;
  const int s_settle = s_check == HGX_OK ? shaped_rows_settle(c, g, &ok) : s_check;
  if (s_settle != HGX_OK) s = s_settle;
  // a failed check: the first result (or its refusal of the guessed layout) is replaced
  else if (!ok) s = ff_triangles_device(c, g, sd, ntri, rot9, HGX_F32C, dout, HGX_C128, 0);
  if (s == HGX_OK && staged)
    HGX_CUDA(cudaMemcpyAsync(ff, dout, sizeof(double2) * (size_t)nqz, cudaMemcpyDeviceToHost, c->stream));
  if (s != HGX_OK) {
    cudaStreamSynchronize(c->stream);  // leave nothing of this call queued behind the error
    return s;
  }
  return hgx_synchronize(c);
}

}  // extern "C"

// ------------------------------------------------------ allocation-free entry ----
// hgx_ff_triangles_noalloc: the FP32C per-q-point form factor for callers that must not
// allocate device memory — a plug-in that lives inside another framework's memory pool and
// is handed only device pointers, a service held to a fixed device-memory budget, or a
// real-time loop in which a cudaMalloc/cudaFree would synchronise the whole device.  Its
// scratch (the FP32 triangle tiles, their anchors and an error word) lives in file-scope
// static device arrays of fixed size, reserved when the library's device code is loaded on a
// GPU and held until exit.
//
// In host code the array names below are only host-side stand-ins, not device addresses:
// the device addresses are obtained once per device with cudaGetSymbolAddress (set-up done by
// the first call on each device, with that device current; make that first call before any
// stream capture) and passed to the kernels.  Every call shares the array: the triangle
// tiles are fully rewritten by each call and the error word is cleared at its start; calls
// that overlap on the GPU (different streams, no ordering) race on the array and must be
// ordered by the caller.  hgx_ff_triangles_noalloc_status reads the error word back.
constexpr int NOALLOC_MAX_TRIANGLES = 65536;
constexpr int NOALLOC_MAX_TILES = NOALLOC_MAX_TRIANGLES / TILE;  // 128 tiles, 1.5 MiB + 4 KiB anchors
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) float g_noalloc_tiles[NOALLOC_MAX_TILES * TILE_FLOATS];
static __device__ __align__(256) double4 g_noalloc_anchors[NOALLOC_MAX_TILES];
static __device__ __align__(256) unsigned g_noalloc_err;

namespace {
struct NoallocSlot {
  float* tiles = nullptr;
  double4* anchors = nullptr;
  unsigned* err = nullptr;
};
NoallocSlot g_noalloc_slots[NOALLOC_MAX_DEVICES];
std::mutex g_noalloc_mutex;

int noalloc_setup(int dev, NoallocSlot* out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  NoallocSlot& s = g_noalloc_slots[dev];
  if (!s.tiles) {
    void* t = nullptr;
    void* an = nullptr;
    void* e = nullptr;
    cudaError_t rc = cudaGetSymbolAddress(&t, g_noalloc_tiles);
    if (rc != cudaSuccess) return cuda_fail(rc, "cudaGetSymbolAddress(g_noalloc_tiles)");
    rc = cudaGetSymbolAddress(&an, g_noalloc_anchors);
    if (rc != cudaSuccess) return cuda_fail(rc, "cudaGetSymbolAddress(g_noalloc_anchors)");
    rc = cudaGetSymbolAddress(&e, g_noalloc_err);
    if (rc != cudaSuccess) return cuda_fail(rc, "cudaGetSymbolAddress(g_noalloc_err)");
    s.tiles = static_cast<float*>(t);
    s.anchors = static_cast<double4*>(an);
    s.err = static_cast<unsigned*>(e);
  }
  *out = s;
  return HGX_OK;
}
}  // namespace

extern "C" int hgx_ff_triangles_noalloc(const double* shape_def, int ntri, int nqy,
                                        const double* qx, const double* qy, int nqz,
                                        const double* qz, const double* rot9, void* ff,
                                        int ff_type, void* stream) {
  if (!shape_def || !qx || !qy || !qz || !ff)
    return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles_noalloc: null argument");
  if (ntri < 1) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles_noalloc: no triangles");
  if (ntri > NOALLOC_MAX_TRIANGLES)
    return fail(HGX_ERR_INVALID_ARG,
                "hgx_ff_triangles_noalloc: more than 65536 triangles (the fixed scratch limit); "
                "use hgx_ff_triangles_q");
  if (nqy < 1 || nqz < 1) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles_noalloc: empty q-grid");
  if (ff_type != HGX_C128 && ff_type != HGX_C64)
    return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles_noalloc: unknown output type");
  int dev = 0;
  HGX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
    return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles_noalloc: device index too large");
  NoallocSlot slot;
  HGX_TRY(noalloc_setup(dev, &slot));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  Rot9 R = make_rot(rot9);
  const int ntiles = (ntri + TILE - 1) / TILE;
  HGX_CUDA(cudaMemsetAsync(slot.err, 0, sizeof(unsigned), st));
  // tiles in the caller's triangle order (no sort, which would need more scratch), each with
  // its FP64 anchor
  tri_tile_kernel<false><<<ntiles, TILE, 0, st>>>(shape_def, ntri, R, nullptr, slot.tiles,
                                                 slot.anchors, nullptr);
  HGX_CUDA(cudaGetLastError());
  PointArgs a{slot.tiles, slot.anchors, ntiles, qx, qy, reinterpret_cast<const double2*>(qz), nqy,
              nqz, R, ff, slot.err};
  dim3 grid((nqz + 127) / 128);
  if (ff_type == HGX_C64) ff_tri_points_kernel<128, float2><<<grid, 128, 0, st>>>(a);
  else ff_tri_points_kernel<128, double2><<<grid, 128, 0, st>>>(a);
  HGX_CUDA(cudaGetLastError());
  return HGX_OK;
}

// The device error word of the allocation-free entry: waits for `stream`, copies the word
// into *bits (host memory) and returns HGX_ERR_DEVICE when a kernel of the last call on this
// device recorded an error (a bounded wait that gave up leaves part of ff unwritten).
// Allocates nothing.
extern "C" int hgx_ff_triangles_noalloc_status(void* stream, unsigned* bits) {
  if (!bits) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles_noalloc_status: bits is NULL");
  *bits = 0;
  int dev = 0;
  HGX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
    return fail(HGX_ERR_INVALID_ARG, "hgx_ff_triangles_noalloc_status: device index too large");
  NoallocSlot slot;
  HGX_TRY(noalloc_setup(dev, &slot));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  unsigned word = 0;
  HGX_CUDA(cudaMemcpyAsync(&word, slot.err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  HGX_CUDA(cudaStreamSynchronize(st));
  *bits = word;
  if (word)
    return fail(HGX_ERR_DEVICE, "hgx_ff_triangles_noalloc: a kernel recorded device error bits " +
                                    std::to_string(word) + " (1 = a bounded wait gave up)");
  return HGX_OK;
}

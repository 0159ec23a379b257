// The exact (polyhedral) triangle form factor: FormFactorTriangle and
// NumericFormFactorC::compute_exact_triangle (src/ff/cpu/ff_tri_cpu.cpp:46-196; the GPU twin
// is ff_poly_kernel, src/ff/gpu/ff_tri_gpu.cu:46-205).  For each q-point (rotated, m = R q)
// and triangle (v1, v2, v3) the Fourier transform of the triangle reduces to its edges and
// vertices:
//   |m|^2 - |m.n_t|^2 = 0:  i (m.n_t) A / |m|^2 e^{-i m.v1}
//   else, per edge e:       -(m.n_t)(m.n_e) |e| / (|m|^2 proj_t) e^{-i m.v_e}      (case 2)
//                           -i (m.n_t)(m.n_e)(m.n_v)(e^{-i m.v_e} - e^{-i m.v_e+1}) / f0
// with the reference's sign convention (e^{-i q.v}) and thresholds (DBL_MIN).
//
// FP64 throughout, and compiled without fused multiply-adds (-fmad=false, hipgisaxs_b200/
// build.py): the vertex terms of a triangle are of size O(1 / (|m|^2 proj_t proj_e)) and
// cancel to O(A) — severely at small |q| — so the result is as sensitive to rounding as the
// reference's own; each product and sum here rounds as the reference's CPU code rounds it.
//
// Design: the reference recomputes the triangle geometry (edges, unit normal, area, edge
// normals, edge directions) for every (q, triangle); here a prep kernel computes it once per
// triangle in the reference's operation order, and the main kernel stages it through shared
// memory (one thread per q-point, tiles of EX_TILE triangles) and evaluates each vertex
// exponential once per (q, triangle) instead of twice (the same input, so the same value).
// A degenerate triangle (zero area) contributes nothing; the reference divides by zero there.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>

#include "cplx.cuh"
#include "hgx_internal.cuh"

namespace hgx {

constexpr int EX_TILE = 32;      // triangles per shared-memory tile
constexpr int EX_THREADS = 128;
constexpr int GEO_DOUBLES = 36;  // per triangle, padded

// per-triangle geometry, reference order (src/ff/cpu/ff_tri_cpu.cpp:59-80, 95-99, 122)
struct TriGeo {
  double v[9];   // v1, v2, v3
  double nt[3];  // unit normal
  double area;   // 0 = degenerate (skipped)
  double ne[9];  // unit edge normals n_e = (e x n_t)/|.|
  double nv[9];  // unit edge directions e/|e|
  double el[3];  // edge lengths
  double pad[2];
};
static_assert(sizeof(TriGeo) == GEO_DOUBLES * sizeof(double), "TriGeo layout");
constexpr int GEO_AREA = 12;     // index of `area` in the double view

__device__ __forceinline__ double vabs3(const double* v) {
  double n = 0.;
#pragma unroll
  for (int i = 0; i < 3; ++i) n += v[i] * v[i];
  return sqrt(n);
}
__device__ __forceinline__ void vcross3(const double* u, const double* v, double* w) {
  w[0] = u[1] * v[2] - u[2] * v[1];
  w[1] = u[2] * v[0] - u[0] * v[2];
  w[2] = u[0] * v[1] - u[1] * v[0];
}

__global__ void tri_geo_kernel(const double* __restrict__ tris, int ntri, int ntot,
                               TriGeo* __restrict__ geo) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntot) return;
  TriGeo g;
  for (int k = 0; k < GEO_DOUBLES; ++k) reinterpret_cast<double*>(&g)[k] = 0.0;
  if (t < ntri) {
    const double* p = tris + 9L * t;
    for (int k = 0; k < 9; ++k) g.v[k] = p[k];
    double edge[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      edge[0][i] = g.v[3 + i] - g.v[i];
      edge[1][i] = g.v[6 + i] - g.v[3 + i];
      edge[2][i] = g.v[i] - g.v[6 + i];
    }
    double n[3];
    vcross3(edge[0], edge[1], n);
    const double nabs = vabs3(n);
    if (nabs > 0.0) {
      g.area = 0.5 * nabs;
#pragma unroll
      for (int i = 0; i < 3; ++i) g.nt[i] = n[i] / nabs;
#pragma unroll
      for (int e = 0; e < 3; ++e) {
        double ne[3];
        vcross3(edge[e], g.nt, ne);
        const double ea = vabs3(ne);
        const double el = vabs3(edge[e]);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          g.ne[3 * e + i] = ne[i] / ea;
          g.nv[3 * e + i] = edge[e][i] / el;
        }
        g.el[e] = el;
      }
    }
  }
  geo[t] = g;
}

__device__ __forceinline__ zd mdot(const zd* m, const double* v) {
  zd r(0.0, 0.0);
#pragma unroll
  for (int i = 0; i < 3; ++i) r += m[i] * v[i];
  return r;
}

// e^{-i z} for complex z = a + bi:  e^{b} (cos a - i sin a)
__device__ __forceinline__ zd exp_minus_i(zd z) {
  double s, c;
  sincos(z.x, &s, &c);
  const double e = exp(z.y);
  return zd(e * c, -e * s);
}

// one triangle's exact form factor at the rotated q-vector m (|m|^2 = q2)
__device__ __forceinline__ zd triangle_exact(const double* G, const zd* m, double q2) {
  const TriGeo& g = *reinterpret_cast<const TriGeo*>(G);
  const zd qnt = mdot(m, g.nt);
  const double proj_tq = q2 - norm2(qnt);
  if (fabs(proj_tq) < DBL_MIN) {  // case 1: q along the normal
    const zd e0 = exp_minus_i(mdot(m, g.v));
    return (zd(0.0, 1.0) * qnt * g.area / q2) * e0;
  }
  zd E[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) E[k] = exp_minus_i(mdot(m, g.v + 3 * k));
  zd ff(0.0, 0.0);
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    const zd qne = mdot(m, g.ne + 3 * e);
    const double proj_eq = proj_tq - norm2(qne);
    if (fabs(proj_eq) < DBL_MIN) {  // case 2: q in the plane, normal to the edge
      const double f0 = g.el[e] / (q2 * proj_tq);
      const zd c0 = -(qnt * qne);
      ff += (c0 * f0) * E[e];
    } else {  // case 3: the two vertices of the edge
      const double f0 = q2 * proj_tq * proj_eq;
      const zd qnv = mdot(m, g.nv + 3 * e);
      const zd c0 = zd(0.0, -1.0) * qnt * qne * qnv;
      ff += (c0 * E[e]) / f0;
      ff += (-c0 * E[(e + 1) % 3]) / f0;
    }
  }
  return ff;
}

template <typename OUT>
__device__ __forceinline__ void store_c(OUT* out, long i, zd v);
template <>
__device__ __forceinline__ void store_c<float2>(float2* out, long i, zd v) {
  out[i] = make_float2((float)v.x, (float)v.y);
}
template <>
__device__ __forceinline__ void store_c<double2>(double2* out, long i, zd v) {
  out[i] = make_double2(v.x, v.y);
}

struct ExactArgs {
  const TriGeo* geo;
  int ntiles;
  const double* qx;
  const double* qy;
  const double2* qz;
  int nqy, nqz;
  Rot9d R;
  void* out;
};

template <typename OUT>
__global__ void __launch_bounds__(EX_THREADS) ff_exact_kernel(ExactArgs a) {
  __shared__ double s_geo[EX_TILE * GEO_DOUBLES];
  const long iz = (long)blockIdx.x * EX_THREADS + threadIdx.x;
  const bool valid = iz < a.nqz;
  zd m[3];
  double q2 = 1.0;
  if (valid) {
    const long iy = iz % a.nqy;
    rotate_q(a.R, a.qx[iy], a.qy[iy], zd(a.qz[iz]), m);
    q2 = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) q2 += norm2(m[j]);
  }
  zd acc(0.0, 0.0);
  const double* src = reinterpret_cast<const double*>(a.geo);
  for (int s = 0; s < a.ntiles; ++s) {
    __syncthreads();  // the previous tile is no longer read
    for (int k = threadIdx.x; k < EX_TILE * GEO_DOUBLES; k += EX_THREADS)
      s_geo[k] = src[(long)s * EX_TILE * GEO_DOUBLES + k];
    __syncthreads();
    if (valid) {
      for (int j = 0; j < EX_TILE; ++j) {
        const double* G = s_geo + j * GEO_DOUBLES;
        if (G[GEO_AREA] == 0.0) continue;  // degenerate, or the zero padding of the last tile
        acc += triangle_exact(G, m, q2);
      }
    }
  }
  if (valid) store_c<OUT>(reinterpret_cast<OUT*>(a.out), iz, acc);
}

static Rot9d rot9d(const double* r9) {
  Rot9d R;
  for (int i = 0; i < 9; ++i) R.r[i] = r9 ? r9[i] : (i % 4 == 0 ? 1.0 : 0.0);
  return R;
}

}  // namespace hgx

using namespace hgx;

extern "C" {

int hgx_ff_exact_triangles_q(hgx_ctx c, hgx_qgrid g, const double* tris, int ntri,
                             const double* rot9, void* ff, int ff_type) {
  if (!c || !g || !tris || !ff) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_exact_triangles_q: null argument");
  if (ntri < 1) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_exact_triangles_q: no triangles");
  if (ff_type != HGX_C128 && ff_type != HGX_C64)
    return fail(HGX_ERR_INVALID_ARG, "hgx_ff_exact_triangles_q: unknown output type");
  if (g->ctx != c) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_exact_triangles_q: grid of another context");
  HGX_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  DevBuf tb, ob;
  const void* dt = nullptr;
  HGX_TRY(stage_in(c, tris, sizeof(double) * 9 * (size_t)ntri, tb, &dt));
  const int ntiles = (ntri + EX_TILE - 1) / EX_TILE;
  const int ntot = ntiles * EX_TILE;
  HGX_TRY(c->scratch.reserve(sizeof(TriGeo) * (size_t)ntot));
  TriGeo* geo = reinterpret_cast<TriGeo*>(c->scratch.p);
  tri_geo_kernel<<<(ntot + 127) / 128, 128, 0, st>>>((const double*)dt, ntri, ntot, geo);
  HGX_CUDA(cudaGetLastError());
  const size_t esz = ff_type == HGX_C64 ? sizeof(float2) : sizeof(double2);
  void* dout = nullptr;
  HGX_TRY(stage_out(c, ff, esz * (size_t)g->nqz, ob, &dout));
  ExactArgs a{geo, ntiles, g->qx, g->qy, g->qz, g->nqy, g->nqz, rot9d(rot9), dout};
  const unsigned blocks = (unsigned)((g->nqz + EX_THREADS - 1) / EX_THREADS);
  if (ff_type == HGX_C64) ff_exact_kernel<float2><<<blocks, EX_THREADS, 0, st>>>(a);
  else ff_exact_kernel<double2><<<blocks, EX_THREADS, 0, st>>>(a);
  HGX_CUDA(cudaGetLastError());
  return finish_out(c, ff, esz * (size_t)g->nqz, dout);
}

int hgx_ff_exact_triangles(hgx_ctx c, const double* tris, int ntri, int nqy, const double* qx,
                           const double* qy, int nqz, const double* qz, const double* rot9,
                           double* ff) {
  if (ntri < 1) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_exact_triangles: no triangles");
  if (!c) return fail(HGX_ERR_INVALID_ARG, "hgx_ff_exact_triangles: null context");
  HGX_CUDA(cudaSetDevice(c->device));
  hgx_qgrid g = nullptr;
  HGX_TRY(shaped_grid(c, nqy, qx, qy, nqz, qz, &g));
  int s = hgx_ff_exact_triangles_q(c, g, tris, ntri, rot9, ff, HGX_C128);
  if (s == HGX_OK) s = hgx_synchronize(c);
  return s;
}

}  // extern "C"

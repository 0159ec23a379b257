// HipGISAXS::compute_gisaxs for a HiG description, on the device
// (src/sim/hipgisaxs_main.cpp:630-685 and run_gisaxs, :694-1440).
//
// For every structure: the grains of its ensemble (a regular grid of centres,
// spatial_distribution :1702-1867; one orientation per grain, orientation_distribution
// :1869-2010), for every grain the form factor of the unit cell (every element's shape at
// every location, weighted by dn2 = (1 - n^2)_layer - (1 - n^2)_shape, :976-1015), the
// structure factor (lattice, paracrystal or Percus-Yevick, :1045-1058) and the DWBA sum
// I += |w sum_k fc_k sf_k ff_k|^2 (:1086-1100); the structures' intensities are then summed
// with their iratios (:1352-1362, 1417-1431).  Structures and the elements of a unit cell are
// taken in key order; the reference walks unordered maps, whose order is unspecified (only
// the rounding of the sums depends on it).  The grid, the Fresnel coefficients and every
// per-grain array stay on the device; the host only walks the description.
//
// As in the reference: the particles sit in layer order 0 (the vacuum: the grain's layer
// order is never assigned, src/model/structure.cpp:389-398), so the DWBA grid is built with
// dn2 = 0 and the Fresnel coefficients for order 0; a custom (mesh) shape ignores its
// location (FormFactor::compute_form_factor passes no translation to the numeric form
// factor, src/ff/ff.cpp:40-48) but is added once per location; orientations drawn by the
// "range" and "random" statistics come from the C library's rand(), in the reference's
// order, while "gaussian", "normal" and "cauchy" step evenly over each axis's range and weight
// the grains; grain scalings and repetitions are sampled with the reference's seeded 64-bit
// Mersenne Twister.  The reference subtracts single_layer_thickness_, a member it never
// assigns, from the grain translation's z (:871-875), and spaces the grains by cell_, which it
// never assigns either; both are taken as 0 here.
//
// Refused with HGX_ERR_INVALID_ARG, naming the feature: clock-seeded random grain positions,
// "bragg" orientations (the reference's search reads q-grid extents it never sets and fails),
// structure correlations other than none (the reference indexes its single grain image as if
// it held one per grain), experiments other than gisaxs and saxs,
// and angle scans in hgx_hig_compute_gisaxs (more than one alpha_i, phi or tilt:
// compute_gisaxs itself refuses those; hgx_hig_compute_scan_point runs them).
//
// SAXS (expt = "saxs") follows run_gisaxs's other branch: the form factor as in GISAXS (its
// first block), the lattice structure factor at the detector's real qz, no Fresnel
// coefficients, and the intensity assigned rather than added, so a structure's image is its
// last grain's last scaling sample; only that one is computed (the orientations of all grains
// are still drawn, so rand() advances as in the reference).  Sliced layers (nslices > 1) give
// the reference's empty image: its slicing branch only prints a message.
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include <sys/stat.h>

#include <algorithm>
#include <array>
#include <map>
#include <new>
#include <random>
#include <string>
#include <vector>

#include "ana_sf.cuh"
#include "ana_sf_f32.cuh"
#include "ana_sf_tangent.cuh"
#include "hgx_internal.cuh"
#include "hig_config.hpp"

namespace hgx {

namespace {

constexpr double PI = 3.141592653589793;  // PI_, include/common/constants.hpp:29

// ff += dn2 * eff over n complex values, each product and sum rounded once (no fused
// multiply-add), as the reference's complex arithmetic rounds them
__global__ void add_scaled_kernel(long n, double dre, double dim, const double2* __restrict__ eff,
                                  double2* __restrict__ ff) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double2 e = eff[i];
  double2 f = ff[i];
  const double re = __dsub_rn(__dmul_rn(dre, e.x), __dmul_rn(dim, e.y));
  const double im = __dadd_rn(__dmul_rn(dre, e.y), __dmul_rn(dim, e.x));
  f.x = __dadd_rn(f.x, re);
  f.y = __dadd_rn(f.y, im);
  ff[i] = f;
}

// The SAXS intensity of one grain and scaling sample (run_gisaxs, :1099-1103): the form
// factor's first block (the reference sizes it for the extended qz in either experiment),
// the structure factor at the detector's real qz; the reference assigns (=) where GISAXS
// accumulates, so each sample replaces the structure's image.  Unfused products and sums, as
// the reference's complex arithmetic rounds them.
__global__ void saxs_intensity_kernel(long n, double w, const double2* __restrict__ sf,
                                      const double2* __restrict__ ff, double* __restrict__ out) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double2 a = sf[i], b = ff[i];
  const double ar = __dmul_rn(w, a.x), ai = __dmul_rn(w, a.y);
  const double tr = __dsub_rn(__dmul_rn(ar, b.x), __dmul_rn(ai, b.y));
  const double ti = __dadd_rn(__dmul_rn(ar, b.y), __dmul_rn(ai, b.x));
  out[i] = __dadd_rn(__dmul_rn(tr, tr), __dmul_rn(ti, ti));
}

// qz of the detector as complex values (imaginary part 0), for SAXS structure factors
// img[z] = sum_s I_s[z] r_s per image (grid y = image of a population, 0 otherwise), as
// hgx_structure_sum forms it: separate multiply and add, structures in order
// (src/sim/hipgisaxs_main.cpp:1352-1362)
__global__ void image_structure_sum_kernel(const double* __restrict__ I, const double* __restrict__ r,
                                           int ns, long n, double* __restrict__ out) {
  const long z = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= n) return;
  const double* Ic = I + (long)blockIdx.y * ns * n;
  double sum = 0.0;
  for (int s = 0; s < ns; ++s) sum = __dadd_rn(sum, __dmul_rn(Ic[(long)s * n + z], r[s]));
  out[(long)blockIdx.y * n + z] = sum;
}

// Room for `bytes` in the simulation's pinned arena (*host), and copies of host data to dev
// through it: one asynchronous copy from pinned memory (a copy from pageable memory waits for
// the host).  The arena in use is reset at the start of each simulation and grows only after
// the stream has finished reading it (a grown arena starts empty: earlier rooms are given up).
int arena_block(HigWork& w, cudaStream_t st, size_t bytes, unsigned char** host) {
  const size_t step = (bytes + 255) & ~(size_t)255;
  const int k = w.arena_cur;
  if (w.arena_off + step > w.arena_cap[k]) {
    // copies in flight still read the old arena; the copies made so far in this simulation
    // are complete after the synchronisation, so the new arena starts empty
    HGX_CUDA(cudaStreamSynchronize(st));
    if (w.h_arena[k]) cudaFreeHost(w.h_arena[k]);
    w.h_arena[k] = nullptr;
    w.arena_cap[k] = 0;
    w.arena_off = 0;
    const size_t cap = std::max<size_t>(2 * step, (size_t)1 << 20);
    HGX_CUDA(cudaMallocHost(&w.h_arena[k], cap));
    w.arena_cap[k] = cap;
  }
  *host = w.h_arena[k] + w.arena_off;
  w.arena_off += step;
  return HGX_OK;
}

int arena_copy(HigWork& w, cudaStream_t st, void* dev, const void* src, size_t bytes) {
  if (!bytes) return HGX_OK;
  unsigned char* dst = nullptr;
  HGX_TRY(arena_block(w, st, bytes, &dst));
  memcpy(dst, src, bytes);
  HGX_CUDA(cudaMemcpyAsync(dev, dst, bytes, cudaMemcpyHostToDevice, st));
  return HGX_OK;
}

__global__ void real_to_complex_kernel(long n, const double* __restrict__ x, double2* __restrict__ z) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) z[i] = make_double2(x[i], 0.0);
}

// The fused grain loop (structures whose unit cell holds analytic shapes only): a quad of
// threads per pixel loops over the grains and evaluates, for its DWBA block, every element's
// form factor at its own rotation and location and the grain's structure factor; the quad
// forms the DWBA sum and accumulates |sum|^2 in a register.  The per-grain form-factor and
// structure-factor arrays of the step-by-step path (4N complex each, written and read back
// per grain) never exist: per grain the kernel reads a few dozen parameters.  The arithmetic
// is the step-by-step path's (the same device functions, the same order of sums), so the two
// agree to rounding.
// One structure-factor evaluation of a grain: scaled lattice vectors, repetitions, weight.
struct ScaleEntry {
  double la[3], lb[3], lc[3], rep[3];
  double w;
};

struct FusedElem {
  double loc[3];
  double dre, dim;  // dn2 of the element's shape
};

struct FusedArgs {
  const AnaShape* shapes;  // one per element-location
  const FusedElem* elems;
  int nelem;
  const double* grains;    // per grain: rotation (9), centre (3)
  const double* elem_rot;  // per grain and element-location: rotation (9)
  int g0, g1;              // grains of this launch
  const ScaleEntry* scales;  // per grain: nscale structure-factor evaluations
  int nscale;
  const double2* sfbuf;    // grain-independent structure factor (4N), or NULL for the lattice
  const double* qx;
  const double* qy;
  const double2* qz;
  const double2* fc;
  long n;
  double* out;             // N intensities, accumulated
  // a population launch (grid y = candidate): per-candidate strides of shapes, elems and
  // scales (records), grains and elem_rot (doubles) and out (doubles); 0 otherwise
  long ps_shape = 0, ps_elem = 0, ps_grain = 0, ps_er = 0, ps_scale = 0, ps_out = 0;
};

// Four threads per pixel, one per DWBA block k: each evaluates fc_k sf_k ff_k and the quad
// adds the four terms in the order k = 0..3 (shuffles), as the step-by-step combination does.
// SHAPE: the one analytic shape of every element (0: any).  PAIRED: every grain of the launch
// keeps qz out of the rotated qx, qy and every lattice a vector has no z component, so the
// lattice factor takes sf_lattice_eval_paired (the same values; each variant carries one of
// the two structure-factor bodies, which keeps the kernel's code smaller).
template <int SHAPE, int PAIRED>
__global__ void __launch_bounds__(128, (SHAPE == SH_PYRAMID || SHAPE == 0) ? 3 : 5) grain_dwba_kernel(FusedArgs a) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long i = t >> 2;
  const int k = (int)(t & 3);
  const bool live = i < a.n;  // every lane takes part in the shuffles
  const long ii = live ? i : 0;
  const double qx = a.qx[ii], qy = a.qy[ii];
  const zd qz(a.qz[k * a.n + ii]);
  const zd fc(a.fc[k * a.n + ii]);
  const int base = (threadIdx.x & 31) & ~3;
  const long cy = blockIdx.y;  // the candidate of a population launch
  const AnaShape* shapes = a.shapes + cy * a.ps_shape;
  const FusedElem* elems = a.elems + cy * a.ps_elem;
  const double* grains = a.grains + cy * a.ps_grain;
  const double* elem_rot = a.elem_rot + cy * a.ps_er;
  const ScaleEntry* scales = a.scales + cy * a.ps_scale;
  double* out = a.out + cy * a.ps_out;
  double acc = (live && k == 0) ? out[i] : 0.0;
  for (int g = a.g0; g < a.g1; ++g) {
    const double* gp = grains + 12 * (long)g;
    zd ff(0, 0);
    for (int e = 0; e < a.nelem; ++e) {
      const double* er = elem_rot + 9 * ((long)g * a.nelem + e);
      Rot9d Re;
#pragma unroll
      for (int r = 0; r < 9; ++r) Re.r[r] = er[r];
      zd m[3];
      rotate_q(Re, qx, qy, qz, m);
      // the same grain and element in every lane of the warp: the test is warp-uniform
      const zd eff = (er[2] == 0.0 && er[5] == 0.0 && shapes[e].d[0].n >= 4)
                         ? ff_analytic_eval_quad<SHAPE>(shapes[e], m, elems[e].loc, k)
                         : ff_analytic_eval<SHAPE>(shapes[e], m, elems[e].loc);
      const double dre = elems[e].dre, dim = elems[e].dim;
      ff.x = __dadd_rn(ff.x, __dsub_rn(__dmul_rn(dre, eff.x), __dmul_rn(dim, eff.y)));
      ff.y = __dadd_rn(ff.y, __dadd_rn(__dmul_rn(dre, eff.y), __dmul_rn(dim, eff.x)));
    }
    Rot9d R;
#pragma unroll
    for (int r = 0; r < 9; ++r) R.r[r] = gp[r];
    zd mr[3];
    rotate_q(R, qx, qy, qz, mr);
    const ScaleEntry* sp = scales + (long)g * a.nscale;
    for (int si = 0; si < a.nscale; ++si) {
      zd sfv;
      if (a.sfbuf) {
        sfv = zd(a.sfbuf[k * a.n + ii]);
      } else {
        SfLat L;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          L.la[d] = sp[si].la[d];
          L.lb[d] = sp[si].lb[d];
          L.lc[d] = sp[si].lc[d];
          L.rep[d] = sp[si].rep[d];
          L.center[d] = gp[9 + d];
        }
        if (PAIRED)
          sfv = sf_lattice_eval_paired(L, mr, (k & 1) != 0);
        else
          sfv = sf_lattice_eval(L, mr);
      }
      const zd term = fc * sfv * ff;
      zd sum(0, 0);
#pragma unroll
      for (int j = 0; j < 4; ++j)
        sum += zd(__shfl_sync(0xffffffffu, term.x, base + j), __shfl_sync(0xffffffffu, term.y, base + j));
      sum = sp[si].w * sum;
      acc += sum.x * sum.x + sum.y * sum.y;
    }
  }
  if (live && k == 0) out[i] = acc;
}

// The fused grain loop in FP32C for grids with real qz and unit cells of one shape among
// cylinder, sphere and box: the same quad layout and order of sums as grain_dwba_kernel, the
// form and structure factors from ana_sf_f32.cuh (FP64 phases, FP32 transcendentals and
// sums), the DWBA terms in FP32 and the intensity accumulated in FP64.
template <int SHAPE>
__global__ void __launch_bounds__(128) grain_dwba_f32c_kernel(FusedArgs a) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long i = t >> 2;
  const int k = (int)(t & 3);
  const bool live = i < a.n;  // every lane takes part in the shuffles
  const long ii = live ? i : 0;
  const double qx = a.qx[ii], qy = a.qy[ii];
  const double qz = a.qz[k * a.n + ii].x;
  const double2 fcd = a.fc[k * a.n + ii];
  const cf fc{(float)fcd.x, (float)fcd.y};
  const int base = (threadIdx.x & 31) & ~3;
  const long cy = blockIdx.y;  // the candidate of a population launch
  const AnaShape* shapes = a.shapes + cy * a.ps_shape;
  const FusedElem* elems = a.elems + cy * a.ps_elem;
  const double* grains = a.grains + cy * a.ps_grain;
  const double* elem_rot = a.elem_rot + cy * a.ps_er;
  const ScaleEntry* scales = a.scales + cy * a.ps_scale;
  double* out = a.out + cy * a.ps_out;
  double acc = (live && k == 0) ? out[i] : 0.0;
  for (int g = a.g0; g < a.g1; ++g) {
    const double* gp = grains + 12 * (long)g;
    cf ff{0.f, 0.f};
    for (int e = 0; e < a.nelem; ++e) {
      const double* er = elem_rot + 9 * ((long)g * a.nelem + e);
      double m[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) m[j] = er[3 * j] * qx + er[3 * j + 1] * qy + er[3 * j + 2] * qz;
      // the same grain and element in every lane of the warp: the test is warp-uniform; the
      // split pays when the in-plane sums have four samples or more
      const cf eff = (er[2] == 0.0 && er[5] == 0.0 && shapes[e].d[0].n >= 4)
                         ? ff_analytic_f32c_quad<SHAPE>(shapes[e], m, elems[e].loc, k)
                         : ff_analytic_f32c<SHAPE>(shapes[e], m, elems[e].loc);
      ff = cadd(ff, cmul(cf{(float)elems[e].dre, (float)elems[e].dim}, eff));
    }
    double mr[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) mr[j] = gp[3 * j] * qx + gp[3 * j + 1] * qy + gp[3 * j + 2] * qz;
    const ScaleEntry* sp = scales + (long)g * a.nscale;
    const bool flat = gp[2] == 0.0 && gp[5] == 0.0;  // the grain rotation keeps qz out of mr[0], mr[1]
    for (int si = 0; si < a.nscale; ++si) {
      cf sfv;
      if (a.sfbuf) {
        const double2 v = a.sfbuf[k * a.n + ii];
        sfv = cf{(float)v.x, (float)v.y};
      } else {
        SfLat L;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          L.la[d] = sp[si].la[d];
          L.lb[d] = sp[si].lb[d];
          L.lc[d] = sp[si].lc[d];
          L.rep[d] = sp[si].rep[d];
          L.center[d] = gp[9 + d];
        }
        // warp-uniform: the same grain and sample in every lane
        sfv = (flat && L.la[2] == 0.0 && L.rep[1] == round_fp64(L.rep[1])) ? sf_lattice_f32c_paired(L, mr, k)
                                                                           : sf_lattice_f32c(L, mr);
      }
      const cf term = cmul(cmul(fc, sfv), ff);
      cf sum{0.f, 0.f};
#pragma unroll
      for (int j = 0; j < 4; ++j)
        sum = cadd(sum, cf{__shfl_sync(0xffffffffu, term.x, base + j),
                           __shfl_sync(0xffffffffu, term.y, base + j)});
      const float w = (float)sp[si].w;
      acc += (double)(w * w * (sum.x * sum.x + sum.y * sum.y));
    }
  }
  if (live && k == 0) out[i] = acc;
}

// true when the FP32C grain kernel has a body for this shape
static bool grain_f32c_shape(int shape) {
  return shape == SH_CYLINDER || shape == SH_SPHERE || shape == SH_BOX;
}

static void launch_grain_f32c(int shape, unsigned blocks, cudaStream_t st, const FusedArgs& a) {
  switch (shape) {
    case SH_CYLINDER: grain_dwba_f32c_kernel<SH_CYLINDER><<<blocks, 128, 0, st>>>(a); break;
    case SH_SPHERE: grain_dwba_f32c_kernel<SH_SPHERE><<<blocks, 128, 0, st>>>(a); break;
    default: grain_dwba_f32c_kernel<SH_BOX><<<blocks, 128, 0, st>>>(a); break;
  }
}

// The tangent of the fused grain loop (FP64, real qz): for one direction of the fit
// parameters, the change of every pixel's intensity.  Per grain and sample the quad forms the
// amplitude A = w sum_k fc_k sf_k ff_k with the forward's device functions and its change dA
// from the hand-written tangents (ana_sf_tangent.cuh) of the tables' changes (shape samples
// and weights, locations, grain and element rotations, grain centres, lattice vectors, sample
// weights); dI = 2 Re(conj(A) dA), accumulated over the grains into dI (scaled by `scale`,
// the structure's share of the image).  The Fresnel coefficients, dn2 and grain-independent
// structure factors do not change.
struct TangentArgs {
  FusedArgs a;                // the tables at the current parameters (a.out unused)
  const AnaShape* dshapes;    // their changes, same layout
  const FusedElem* delems;
  const double* dgrains;
  const double* delem_rot;
  const ScaleEntry* dscales;
  double scale;
  double* dI;                 // N, accumulated
};

template <int SHAPE>
__global__ void __launch_bounds__(128) grain_tangent_kernel(TangentArgs ta) {
  const FusedArgs& a = ta.a;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long i = t >> 2;
  const int k = (int)(t & 3);
  const bool live = i < a.n;  // every lane takes part in the shuffles
  const long ii = live ? i : 0;
  const double q[3] = {a.qx[ii], a.qy[ii], a.qz[k * a.n + ii].x};
  const zd qzc(q[2], 0.0);
  const zd fc(a.fc[k * a.n + ii]);
  const int base = (threadIdx.x & 31) & ~3;
  double acc = 0.0;
  for (int g = a.g0; g < a.g1; ++g) {
    const double* gp = a.grains + 12 * (long)g;
    const double* dgp = ta.dgrains + 12 * (long)g;
    zd ff(0, 0), dff(0, 0);
    for (int e = 0; e < a.nelem; ++e) {
      const double* er = a.elem_rot + 9 * ((long)g * a.nelem + e);
      const double* der = ta.delem_rot + 9 * ((long)g * a.nelem + e);
      double m[3], dm[3];
      zd mz[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        m[j] = er[3 * j] * q[0] + er[3 * j + 1] * q[1] + er[3 * j + 2] * q[2];
        dm[j] = der[3 * j] * q[0] + der[3 * j + 1] * q[1] + der[3 * j + 2] * q[2];
      }
      Rot9d Re;
#pragma unroll
      for (int r = 0; r < 9; ++r) Re.r[r] = er[r];
      rotate_q(Re, q[0], q[1], qzc, mz);
      const zd F = ff_analytic_eval<SHAPE>(a.shapes[e], mz, a.elems[e].loc);
      const zd dF = ff_analytic_tangent<SHAPE>(a.shapes[e], ta.dshapes[e], m, dm, a.elems[e].loc,
                                               ta.delems[e].loc);
      const zd dn2(a.elems[e].dre, a.elems[e].dim);
      ff += dn2 * F;
      dff += dn2 * dF;
    }
    double mr[3], dmr[3];
    zd mrz[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      mr[j] = gp[3 * j] * q[0] + gp[3 * j + 1] * q[1] + gp[3 * j + 2] * q[2];
      dmr[j] = dgp[3 * j] * q[0] + dgp[3 * j + 1] * q[1] + dgp[3 * j + 2] * q[2];
    }
    Rot9d R;
#pragma unroll
    for (int r = 0; r < 9; ++r) R.r[r] = gp[r];
    rotate_q(R, q[0], q[1], qzc, mrz);
    const ScaleEntry* sp = a.scales + (long)g * a.nscale;
    const ScaleEntry* dsp = ta.dscales + (long)g * a.nscale;
    for (int si = 0; si < a.nscale; ++si) {
      zd sfv, dsf(0, 0);
      if (a.sfbuf) {
        sfv = zd(a.sfbuf[k * a.n + ii]);
      } else {
        SfLat L, dL;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          L.la[d] = sp[si].la[d];
          L.lb[d] = sp[si].lb[d];
          L.lc[d] = sp[si].lc[d];
          L.rep[d] = sp[si].rep[d];
          L.center[d] = gp[9 + d];
          dL.la[d] = dsp[si].la[d];
          dL.lb[d] = dsp[si].lb[d];
          dL.lc[d] = dsp[si].lc[d];
          dL.rep[d] = 0.0;
          dL.center[d] = dgp[9 + d];
        }
        sfv = sf_lattice_eval(L, mrz);
        dsf = sf_lattice_tangent(L, dL, mr, dmr);
      }
      const zd term = fc * sfv * ff;
      const zd dterm = fc * (dsf * ff + sfv * dff);
      zd A(0, 0), dA(0, 0);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        A += zd(__shfl_sync(0xffffffffu, term.x, base + j), __shfl_sync(0xffffffffu, term.y, base + j));
        dA += zd(__shfl_sync(0xffffffffu, dterm.x, base + j), __shfl_sync(0xffffffffu, dterm.y, base + j));
      }
      const double w = sp[si].w, dw = dsp[si].w;
      // d |w A|^2 = 2 w dw |A|^2 + 2 w^2 Re(conj(A) dA)
      acc += 2.0 * w * dw * (A.x * A.x + A.y * A.y) + 2.0 * w * w * (A.x * dA.x + A.y * dA.y);
    }
  }
  if (live && k == 0) ta.dI[i] += ta.scale * acc;
}

static void launch_grain_tangent(int shape, unsigned blocks, cudaStream_t st, const TangentArgs& t) {
  switch (shape) {
    case SH_CYLINDER: grain_tangent_kernel<SH_CYLINDER><<<blocks, 128, 0, st>>>(t); break;
    case SH_SPHERE: grain_tangent_kernel<SH_SPHERE><<<blocks, 128, 0, st>>>(t); break;
    default: grain_tangent_kernel<SH_BOX><<<blocks, 128, 0, st>>>(t); break;
  }
}

constexpr int FUSED_GRAINS_PER_LAUNCH = 64;  // keeps each launch to tens of milliseconds

template <int PAIRED>
void launch_grain_kernel(int shape, unsigned blocks, cudaStream_t st, const FusedArgs& a) {
  switch (shape) {
    case SH_CYLINDER: grain_dwba_kernel<SH_CYLINDER, PAIRED><<<blocks, 128, 0, st>>>(a); break;
    case SH_SPHERE: grain_dwba_kernel<SH_SPHERE, PAIRED><<<blocks, 128, 0, st>>>(a); break;
    case SH_BOX: grain_dwba_kernel<SH_BOX, PAIRED><<<blocks, 128, 0, st>>>(a); break;
    case SH_CUBE: grain_dwba_kernel<SH_CUBE, PAIRED><<<blocks, 128, 0, st>>>(a); break;
    case SH_PRISM3: grain_dwba_kernel<SH_PRISM3, PAIRED><<<blocks, 128, 0, st>>>(a); break;
    case SH_PRISM6: grain_dwba_kernel<SH_PRISM6, PAIRED><<<blocks, 128, 0, st>>>(a); break;
    case SH_PYRAMID: grain_dwba_kernel<SH_PYRAMID, PAIRED><<<blocks, 128, 0, st>>>(a); break;
    default: grain_dwba_kernel<0, PAIRED><<<blocks, 128, 0, st>>>(a); break;
  }
}

// RotMatrix_t(axis, angle) and its product (include/numerics/matrix.hpp:43-117)
struct Rot {
  double m[9];
  static Rot axis(int ax, double a) {
    const double c = cos(a), s = sin(a);
    Rot r;
    switch (ax) {
      case 0: { const double v[9] = {1., 0., 0., 0., c, -s, 0., s, c}; for (int i = 0; i < 9; ++i) r.m[i] = v[i]; break; }
      case 1: { const double v[9] = {c, 0., -s, 0., 1., 0., s, 0., c}; for (int i = 0; i < 9; ++i) r.m[i] = v[i]; break; }
      case 2: { const double v[9] = {c, -s, 0., s, c, 0., 0., 0., 1.}; for (int i = 0; i < 9; ++i) r.m[i] = v[i]; break; }
      default: { const double v[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}; for (int i = 0; i < 9; ++i) r.m[i] = v[i]; }
    }
    return r;
  }
  Rot operator*(const Rot& b) const {
    Rot r;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double acc = 0.0;
        for (int k = 0; k < 3; ++k) acc += m[i * 3 + k] * b.m[j + 3 * k];
        r.m[i * 3 + j] = acc;
      }
    return r;
  }
  void apply(const double* v, double* out) const {
    for (int i = 0; i < 3; ++i) out[i] = m[3 * i] * v[0] + m[3 * i + 1] * v[1] + m[3 * i + 2] * v[2];
  }
};

int shape_code(const std::string& name) {  // ShapeName, include/common/enums.hpp:24-43
  if (name == "box") return 2;
  if (name == "cube") return 3;
  if (name == "cylinder") return 4;
  if (name == "sphere") return 5;
  if (name == "prism3") return 8;
  if (name == "prism6") return 9;
  if (name == "pyramid") return 14;
  return -1;
}
int param_code(const std::string& t) {  // ShapeParamType, enums.hpp:45-54
  if (t == "radius") return 2;
  if (t == "xsize") return 3;
  if (t == "ysize") return 4;
  if (t == "height") return 5;
  if (t == "edge") return 6;
  if (t == "baseangle") return 7;
  return 1;
}
int stat_code(const std::string& s) {  // StatisticType, enums.hpp:74-84
  if (s == "null") return 0;
  if (s == "none") return 2;
  if (s == "cauchy") return 3;
  if (s == "gaussian") return 4;
  if (s == "random") return 5;
  if (s == "range") return 6;
  if (s == "t") return 7;
  if (s == "uniform") return 8;
  return 1;
}
int lattice_code(const std::string& t) {
  if (t == "bcc") return 2;
  if (t == "cubic") return 3;
  if (t == "fcc") return 4;
  if (t == "fco") return 5;
  if (t == "hcp") return 6;
  if (t == "hex") return 7;
  return 1;
}

bool file_exists(const std::string& p) {
  FILE* f = fopen(p.c_str(), "rb");
  if (!f) return false;
  fclose(f);
  return true;
}

// how many values an angle scan takes (HipGISAXS::compute_gisaxs, :640-660)
int scan_count(double mn, double mx, double step, bool clamp_max) {
  if (clamp_max && mx < mn) mx = mn;
  if ((clamp_max && mn == mx) || step == 0) return 1;
  return (int)((mx - mn) / step + 1);
}

}  // namespace

// woo::MTRandomNumberGenerator (include/woo/random/woo_mtrandom.hpp): a 64-bit Mersenne
// Twister seeded with 0, rand() = (x - min) / (max - min) in doubles.
struct MtRand {
  std::mt19937_64 gen{0};
  double min_ = (double)std::mt19937_64::min(), max_ = (double)std::mt19937_64::max();
  double rand() { return (double)(gen() - min_) / (max_ - min_); }
};

// HipGISAXS::gaussian and ::cauchy (include/sim/hipgisaxs_main.hpp:151-172)
static double weight_gaussian(double x, double mean, double sigma) {
  const double tiny = 2.2250738585072014e-308, sqrt_2pi = 2.506628;  // TINY_, SQRT_2PI_
  if (sigma < tiny) return (x - mean < tiny) ? 1.0 : 0.0;
  return (1.0 / (sigma * sqrt_2pi) * exp(-(x - mean) * (x - mean) / (2 * sigma * sigma)));
}
static double weight_cauchy(double x, double l, double sc) {
  const double tiny = 2.2250738585072014e-308;
  if (sc > tiny) return 1.0 / (PI * sc * (1.0 + ((x - l) / sc) * ((x - l) / sc)));
  return (x - l > tiny) ? 0.0 : 1.0;
}

// The grain-scaling and repetition loops of run_gisaxs (:815-870, :1017-1040) with
// construct_scaling_distribution (:2179-2226), construct_repetition_distribution (:2100-2176)
// and generate_repetition_range (:2089-2098): for every grain the list of (scaling, repetition,
// weight) its structure factor is evaluated with, in the reference's order.  Reproduced as
// written: the samples of all three axes share one sample vector indexed as if each axis had
// samples.size() / 3 of them; each repetition axis draws from a fresh generator; with a
// repetition distribution the repetition list is zipped to its shortest axis and indexed by
// grain, and the scaling loop runs max(#scalings, #repetitions) times.  Where the reference
// reads past its sample vector (a repetition distribution with an undistributed scaling, in the
// branch its grain_scaling_is_dist() takes by undefined behaviour) the undistributed branch is
// taken.  Returns false (with a message) where the reference's own steps fail.
static bool scale_plan(const hig::Structure& s, int ngr, const std::vector<double>& gw,
                       std::vector<ScaleEntry>& plan, int& nscale, std::string& why) {
  // scaling samples
  std::vector<double> samples, weights;
  bool any_dist = false, dist_branch = false;
  int nv[3];
  for (int i = 0; i < 3; ++i) {
    const bool is_dist = s.scaling_stat[i] != "none";
    any_dist = any_dist || is_dist;
    nv[i] = (!is_dist || s.scaling_stddev[i] == 0) ? 1 : s.scaling_nsamples[i];
    if (s.scaling_stddev[i] > 0) dist_branch = true;  // grain_scaling_is_dist()
  }
  MtRand rng;
  const double width = 4;
  const int max_nvals = std::max(nv[0], std::max(nv[1], nv[2]));
  for (int i = 0; i < 3; ++i) {
    const std::string& st = s.scaling_stat[i];
    const double mean = s.scaling_mean[i];
    const double sd = st != "none" ? s.scaling_stddev[i] : 0.0;
    if (st == "none") {
      samples.push_back(mean);
      weights.push_back(1.0);
    } else if (st == "gaussian" || st == "cauchy") {
      if (!(sd > 0)) {
        why = "a " + st + " scaling distribution needs stddev > 0 (the reference divides by zero)";
        return false;
      }
      const double mn = mean - width * sd;
      const double dx = (2 * width) * sd / (max_nvals + 1);
      for (int j = 0; j < max_nvals; ++j) {
        const double t = mn + j * dx + rng.rand() * dx;
        samples.push_back(t);
        weights.push_back(st == "gaussian" ? weight_gaussian(t, mean, sd) : weight_cauchy(t, mean, sd));
      }
    } else {
      why = "scaling statistic '" + st + "' (the reference samples only gaussian and cauchy)";
      return false;
    }
  }
  (void)any_dist;
  // repetitions
  std::vector<std::array<double, 3>> repeats;
  if (s.repetition_dist) {
    const int nrep = samples.size() > 1 ? (int)samples.size() : ngr;
    const hig::Repetition* axes[3] = {&s.xrep, &s.yrep, &s.zrep};
    std::vector<unsigned> vals[3];
    for (int a = 0; a < 3; ++a) {
      const hig::Repetition& r = *axes[a];
      if (r.stat == "none") {
        vals[a].push_back(r.min);
      } else if (r.stat == "range") {
        MtRand rr;  // a fresh generator for every axis
        for (int i = 0; i < nrep; ++i) vals[a].push_back((unsigned)(r.min + rr.rand() * (double)(r.max - r.min)));
      } else {
        why = "repetition statistic '" + r.stat + "' (the reference supports none and range)";
        return false;
      }
    }
    const size_t sizes = std::min(std::min(vals[0].size(), vals[1].size()), vals[2].size());
    for (size_t i = 0; i < sizes; ++i) repeats.push_back({{(double)vals[0][i], (double)vals[1][i], (double)vals[2][i]}});
  } else {
    repeats.push_back({{s.repetition[0], s.repetition[1], s.repetition[2]}});
  }
  const int num_scaling = (int)samples.size() / 3, num_repeats = (int)repeats.size();
  if (num_scaling == num_repeats) nscale = num_scaling;
  else if (num_scaling == 1) nscale = num_repeats;
  else if (num_repeats == 1) nscale = num_scaling;
  else {
    why = "scaling and repetition sample counts differ (the reference refuses this)";
    return false;
  }
  plan.resize((size_t)ngr * nscale);
  for (int g = 0; g < ngr; ++g)
    for (int i = 0; i < nscale; ++i) {
      double sc[3], w;
      if (dist_branch) {
        for (int k = 0; k < 3; ++k) sc[k] = samples[i + num_scaling * k];
        w = weights[i];
      } else {
        for (int k = 0; k < 3; ++k) sc[k] = samples[k];
        w = weights[0];
      }
      const std::array<double, 3>& rp = repeats[s.repetition_dist ? g % num_repeats : 0];
      ScaleEntry& e = plan[(size_t)g * nscale + i];
      for (int k = 0; k < 3; ++k) {  // scaled and clamped as hgx_sf_lattice does (sf.cu)
        e.la[k] = s.lattice.a[k] * sc[0];
        e.lb[k] = s.lattice.b[k] * sc[1];
        e.lc[k] = s.lattice.c[k] * sc[2];
        e.rep[k] = rp[k] < 1 ? 1 : rp[k];
      }
      e.w = gw[g] * w;  // gauss_weight * scaling_wght (:1045)
    }
  return true;
}

// The grain centres of spatial_distribution's "regular" branch (:1765-1828) with the unit
// cell size cell_ = 0 (the reference never assigns it) and tz = 0: d[3][ngrains].
static void regular_centres(const hig::Structure& s, std::vector<double>& d, int& ngr) {
  const double nd[3] = {s.maxgrains[0], s.maxgrains[1], s.maxgrains[2]};
  const int n0 = (int)nd[0], n1 = (int)nd[1], n2 = (int)nd[2];
  ngr = (int)(nd[0] * nd[1] * nd[2]);
  d.assign(3 * (size_t)ngr, 0.0);
  std::vector<double> dx(n0), dy(n1), dz(n2);
  const double sc[3] = {s.spacing[0], s.spacing[1], s.spacing[2]};  // cell_ + spacing
  double val = 0, step = sc[0], mx = sc[0] * (nd[0] - 1);
  for (int i = 0; i < n0; ++i, val += step) dx[i] = val - mx / 2;
  val = 0, step = sc[1], mx = sc[1] * (nd[1] - 1);
  for (int i = 0; i < n1; ++i, val += step) dy[i] = val - mx / 2;
  val = 0, step = sc[2];
  for (int i = 0; i < n2; ++i, val += step) dz[i] = val + 0.0;
  double* d1 = d.data();
  double* d2 = d1 + ngr;
  double* d3 = d2 + ngr;
  for (int x = 0; x < n0; ++x)
    for (int yz = 0; yz < n1 * n2; ++yz) d1[n1 * n2 * x + yz] = dx[x];
  for (int x = 0; x < n0; ++x)
    for (int y = 0; y < n1; ++y)
      for (int z = 0; z < n2; ++z) d2[n1 * n2 * x + n2 * y + z] = dy[y];
  for (int xy = 0; xy < n0 * n1; ++xy)
    for (int z = 0; z < n2; ++z) d3[n2 * xy + z] = dz[z];
}

// rotation_rotN() of a structure: (axis - 'x', first angle, second angle), zeros for axis 'n'
static void rotation_of(const hig::Rotation& r, double out[3]) {
  if (r.axis == 'n') { out[0] = out[1] = out[2] = 0; return; }
  out[0] = (double)((char)r.axis - 'x');
  out[1] = r.angles[0];
  out[2] = r.angles[1];
}

// orientation_distribution (:1869-2085): nn[3][ngr] radians and the grain weights gw[ngr]
// (run_gisaxs applies the product of the three axes' weights for "gaussian" and "cauchy",
// :946-951; for "normal", the same angles, it does not).  "range"/"random" draw with the C
// library's rand(); "gaussian"/"normal"/"cauchy" step each axis evenly over its range (the
// reference's random sampling of them is commented out) and weight by the distribution.
static int orientations(const hig::Structure& s, int ngr, std::vector<double>& nn, std::vector<double>& gw) {
  const double tiny = 2.2250738585072014e-308;  // TINY_
  double r[3][3];
  rotation_of(s.rot1, r[0]);
  rotation_of(s.rot2, r[1]);
  rotation_of(s.rot3, r[2]);
  const hig::Rotation* rot[3] = {&s.rot1, &s.rot2, &s.rot3};
  nn.assign(3 * (size_t)ngr, 0.0);
  std::vector<double> wg(3 * (size_t)ngr, 1.0);
  const std::string& st = s.orientation_stat;
  if (st == "single") {
    for (int k = 0; k < 3; ++k)
      for (int x = 0; x < ngr; ++x) nn[k * ngr + x] = r[k][1] * PI / 180;
  } else if (st == "random") {
    for (int x = 0; x < 3 * ngr; ++x) nn[x] = (double(rand()) / RAND_MAX) * 2 * PI;
  } else if (st == "range") {
    for (int k = 0; k < 3; ++k) {
      const double dr = fabs(r[k][2] - r[k][1]);
      for (int x = 0; x < ngr; ++x) nn[k * ngr + x] = (r[k][1] + (double(rand()) / RAND_MAX) * dr) * PI / 180;
    }
  } else if (st == "gaussian" || st == "normal") {
    for (int k = 0; k < 3; ++k) {
      double dr = fabs(r[k][2] - r[k][1]);
      if (dr > tiny) {
        dr /= ngr;
        for (int x = 0; x < ngr; ++x) {
          const double t = r[k][1] + x * dr;
          nn[k * ngr + x] = t * PI / 180;
          wg[k * ngr + x] = weight_gaussian(t, rot[k]->mean, rot[k]->sd);
        }
      } else {
        for (int x = 0; x < ngr; ++x) nn[k * ngr + x] = r[k][1] * PI / 180;
      }
    }
  } else if (st == "cauchy") {
    for (int k = 0; k < 3; ++k) {
      if (ngr == 1 && fabs(r[k][2] - r[k][1]) > 0)
        return fail(HGX_ERR_INVALID_ARG, "hgx_hig_compute_gisaxs: structure '" + s.key +
                                             "': cauchy orientations over a range need more than one grain "
                                             "(the reference divides the range by ngrains - 1)");
      const double dr = fabs(r[k][2] - r[k][1]) / (ngr - 1);
      if (dr > tiny) {
        for (int x = 0; x < ngr; ++x) {
          const double t = r[k][1] + x * dr;
          nn[k * ngr + x] = t * PI / 180;
          wg[k * ngr + x] = weight_cauchy(t, rot[k]->location, rot[k]->scale);
        }
      } else {
        for (int x = 0; x < ngr; ++x) nn[k * ngr + x] = r[k][1] * PI / 180;
      }
    }
  } else if (st == "bragg") {
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_compute_gisaxs: structure '" + s.key +
                                         "': bragg orientations are not supported (the reference's Bragg search "
                                         "reads q-grid extents it never sets, finds no angle and fails)");
  } else {
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_compute_gisaxs: structure '" + s.key +
                                         "': orientation statistic '" + st + "' is not supported");
  }
  gw.assign(ngr, 1.0);
  if (st == "gaussian" || st == "cauchy")
    for (int g = 0; g < ngr; ++g) gw[g] = wg[g] * wg[ngr + g] * wg[2 * ngr + g];
  return HGX_OK;
}

// The fused path for one structure: element-location and grain tables on the device, the
// structure factor once when it does not depend on the grain, then the grain kernel in
// launches of FUSED_GRAINS_PER_LAUNCH grains (the grains in order, so the sums run as in the
// step-by-step path).
// The fused grain kernel's tables of one structure: every element-location's analytic shape,
// location and dn2 (unit-cell elements in shape-key order, locations in file order), and per
// grain its rotation and centre (12 doubles) and every element's rotation (9 doubles).
struct FusedTables {
  std::vector<AnaShape> shapes;
  std::vector<FusedElem> elems;
  std::vector<double> gt, er;
};

static int fused_tables(const hig::Structure& s, const hig::Unitcell& uc, const hig::Input& in,
                        const Rot& rot_phi, const std::vector<double>& dd, const std::vector<double>& nn,
                        int ngr, int ax1, int ax2, int ax3, FusedTables& T) {
  std::vector<AnaShape>& shapes = T.shapes;
  std::vector<FusedElem>& elems = T.elems;
  shapes.clear();
  elems.clear();
  std::vector<const hig::Shape*> owner;
  for (const auto& ekv : uc.elements) {  // in shape-key order, locations in file order
    const hig::Shape& sh = in.shapes.at(ekv.first);
    std::vector<double> prm;
    for (const auto& pk : sh.params) {
      const hig::ShapeParam& p = pk.second;
      const double row[7] = {(double)param_code(p.type), (double)stat_code(p.stat), p.min, p.max,
                             p.p1, p.p2, (double)p.nvalues};
      prm.insert(prm.end(), row, row + 7);
    }
    AnaShape as;
    HGX_TRY(ana_shape_from_params(shape_code(sh.name), (int)(prm.size() / 7), prm.data(), 0.0, 0.0, as));
    for (const hig::vec3& loc : ekv.second) {
      FusedElem fe;
      for (int k = 0; k < 3; ++k) fe.loc[k] = loc[k];
      fe.dre = 0.0 - 2 * sh.refindex.delta;
      fe.dim = 0.0 - 2 * sh.refindex.beta;
      shapes.push_back(as);
      elems.push_back(fe);
      owner.push_back(&sh);
    }
  }
  const int nelem = (int)elems.size();
  std::vector<double>& gt = T.gt;
  std::vector<double>& er = T.er;
  gt.assign(12 * (size_t)ngr, 0.0);
  er.assign(9 * (size_t)ngr * (nelem > 0 ? nelem : 1), 0.0);
  for (int gi = 0; gi < ngr; ++gi) {
    const Rot rot = ((rot_phi * Rot::axis(ax3, nn[2 * ngr + gi])) * Rot::axis(ax2, nn[ngr + gi])) *
                    Rot::axis(ax1, nn[gi]);
    const double ddv[3] = {dd[gi], dd[gi + ngr], dd[gi + 2 * ngr]};
    double center[3];
    rot.apply(ddv, center);
    for (int k = 0; k < 3; ++k) center[k] += s.transvec[k];
    for (int r = 0; r < 9; ++r) gt[12 * (size_t)gi + r] = rot.m[r];
    for (int k = 0; k < 3; ++k) gt[12 * (size_t)gi + 9 + k] = center[k];
    for (int e = 0; e < nelem; ++e) {
      const hig::Shape& sh = *owner[e];
      const Rot srot = ((rot * Rot::axis(0, sh.xrot)) * Rot::axis(1, sh.yrot)) * Rot::axis(2, sh.zrot);
      for (int r = 0; r < 9; ++r) er[9 * ((size_t)gi * nelem + e) + r] = srot.m[r];
    }
  }
  return HGX_OK;
}

static int fused_structure(hgx_ctx c, hgx_qgrid g, HigWork& w, const hig::Structure& s, const hig::Unitcell& uc,
                           const hig::Input& in, const Rot& rot_phi, const std::vector<double>& dd,
                           const std::vector<double>& nn, int ngr, int ax1, int ax2, int ax3,
                           const std::vector<ScaleEntry>& plan, int nscale, const double2* fc,
                           double* Is, int precision) {
  cudaStream_t st = c->stream;
  FusedTables T;
  HGX_TRY(fused_tables(s, uc, in, rot_phi, dd, nn, ngr, ax1, ax2, ax3, T));
  const std::vector<AnaShape>& shapes = T.shapes;
  const std::vector<FusedElem>& elems = T.elems;
  const std::vector<double>& gt = T.gt;
  const std::vector<double>& er = T.er;
  const int nelem = (int)elems.size();
  DevBuf& bsf = w.sf;
  // the five tables as one block of the arena, sent in one copy
  auto up = [](size_t o) { return (o + 255) & ~(size_t)255; };
  const size_t o_el = up(sizeof(AnaShape) * nelem);
  const size_t o_gt = o_el + up(sizeof(FusedElem) * nelem);
  const size_t o_er = o_gt + up(sizeof(double) * gt.size());
  const size_t o_sc = o_er + up(sizeof(double) * er.size());
  const size_t total = o_sc + sizeof(ScaleEntry) * plan.size();
  HGX_TRY(w.ftab.reserve(total));
  unsigned char* h = nullptr;
  HGX_TRY(arena_block(w, st, total, &h));
  if (nelem > 0) {
    memcpy(h, shapes.data(), sizeof(AnaShape) * nelem);
    memcpy(h + o_el, elems.data(), sizeof(FusedElem) * nelem);
  }
  if (!gt.empty()) memcpy(h + o_gt, gt.data(), sizeof(double) * gt.size());
  if (!er.empty()) memcpy(h + o_er, er.data(), sizeof(double) * er.size());
  if (!plan.empty()) memcpy(h + o_sc, plan.data(), sizeof(ScaleEntry) * plan.size());
  HGX_CUDA(cudaMemcpyAsync(w.ftab.p, h, total, cudaMemcpyHostToDevice, st));
  const unsigned char* d = (const unsigned char*)w.ftab.p;
  FusedArgs a;
  a.shapes = (const AnaShape*)d;
  a.elems = (const FusedElem*)(d + o_el);
  a.nelem = nelem;
  a.grains = (const double*)(d + o_gt);
  a.elem_rot = (const double*)(d + o_er);
  a.scales = (const ScaleEntry*)(d + o_sc);
  a.nscale = nscale;
  a.sfbuf = nullptr;
  if (s.type == "paracrystal") {
    HGX_TRY(hgx_sf_paracrystal(c, g, s.pc_dims, lattice_code(s.lattice.type), s.pc_dist[1], s.pc_dist[0],
                               s.pc_sdev[1], s.pc_sdev[0], s.pc_domain, bsf.p, HGX_C128));
    a.sfbuf = (const double2*)bsf.p;
  } else if (s.type == "percusyevick") {
    HGX_TRY(hgx_sf_percus_yevick(c, g, s.py_diameter, s.py_volfract, s.py_dims, bsf.p, HGX_C128));
    a.sfbuf = (const double2*)bsf.p;
  }
  a.qx = g->qx;
  a.qy = g->qy;
  a.qz = g->qz;
  a.fc = fc;
  a.n = (long)g->nqy;
  a.out = Is;
  const unsigned blocks = (unsigned)((4 * a.n + 127) / 128);
  int one = nelem > 0 ? shapes[0].shape : 0;  // the shape every element shares, if any
  for (int e = 1; e < nelem; ++e)
    if (shapes[e].shape != one) one = 0;
  // FP32C: grids with real qz blocks (paired rows) and one shape with an FP32C body
  const bool f32c = precision == HGX_F32C && g->mode == 1 && grain_f32c_shape(one);
  for (int g0 = 0; g0 < ngr; g0 += FUSED_GRAINS_PER_LAUNCH) {
    a.g0 = g0;
    a.g1 = g0 + FUSED_GRAINS_PER_LAUNCH < ngr ? g0 + FUSED_GRAINS_PER_LAUNCH : ngr;
    if (f32c) {
      launch_grain_f32c(one, blocks, st, a);
      HGX_CUDA(cudaGetLastError());
      continue;
    }
    // the paired lattice factor when it holds for every grain and sample of the launch
    bool paired = a.sfbuf == nullptr;
    for (int gi = a.g0; gi < a.g1 && paired; ++gi) {
      if (gt[12 * (size_t)gi + 2] != 0.0 || gt[12 * (size_t)gi + 5] != 0.0) paired = false;
      for (int k = 0; k < nscale && paired; ++k)
        if (plan[(size_t)gi * nscale + k].la[2] != 0.0) paired = false;
    }
    if (paired)
      launch_grain_kernel<1>(one, blocks, st, a);
    else
      launch_grain_kernel<0>(one, blocks, st, a);
    HGX_CUDA(cudaGetLastError());
  }
  // the tables stay in the context's buffers; the next structure rewrites them in stream order
  return HGX_OK;
}

}  // namespace hgx

using namespace hgx;

namespace {
// HipGISAXS::run_gisaxs (src/sim/hipgisaxs_main.cpp:694-1440) at incidence angle alpha_deg and
// in-plane rotation phi_deg (degrees, as the reference's scan loops hold them; the tilt is not
// used by run_gisaxs).  The detector grid is QGrid::create's at the description's first
// alpha_i (HipGISAXS::init); qz_extended and the Fresnel coefficients take alpha_deg.
int compute_at(hgx_ctx c, hgx_hig h, int precision, double alpha_deg, double phi_deg, double* image) {
  if (!c || !h || !image) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_compute_gisaxs: null argument");
  if (precision != HGX_F64 && precision != HGX_F32C)
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_compute_gisaxs: unknown precision");
  const hig::Input& in = h->in;
  const hig::Scattering& sc = in.scattering;
  const hig::Compute& cp = in.compute;
  auto refuse = [](const std::string& why) {
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_compute_gisaxs: " + why);
  };
  if (sc.expt != "gisaxs" && sc.expt != "saxs")  // StructureFactor refuses the others (sf.cpp:100-102)
    return refuse("experiment '" + sc.expt + "': only gisaxs and saxs are defined");
  // sliced layers: the reference only prints that slicing is not implemented and adds nothing
  // (:1106-1115), so every structure's image stays zero; the orientations are still drawn
  const bool sliced = cp.nslices > 1;
  if (cp.structcorrelation != "null" && cp.structcorrelation != "nGnE")
    return refuse("structure correlation '" + cp.structcorrelation + "' is not supported");
  if (in.structures.empty()) return refuse("the description has no structure");
  for (const auto& kv : in.structures) {
    const hig::Structure& s = kv.second;
    if (s.distribution != "regular")
      return refuse("structure '" + s.key + "': ensemble distribution '" + s.distribution + "' is not supported");
    if (!in.unitcells.count(s.unitcell_key))
      return refuse("structure '" + s.key + "': unknown unit cell '" + s.unitcell_key + "'");
    if (s.maxgrains[0] < 1 || s.maxgrains[1] < 1 || s.maxgrains[2] < 1)
      return refuse("structure '" + s.key + "': maxgrains must be >= 1");
  }
  HGX_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = c->stream;

  // beam, grid (vacuum layer: dn2 = 0) and Fresnel coefficients for layer order 0
  double k0, alpha_i;  // alpha_i: the first incidence angle, of the detector grid
  HGX_TRY(hgx_hig_beam(h, &k0, &alpha_i, nullptr));
  const double alpha_s = alpha_deg * PI / 180;  // this simulation's incidence angle
  const double phi = phi_deg * PI / 180;
  if (!c->hig) {
    c->hig = new (std::nothrow) HigWork;
    if (!c->hig) return fail(HGX_ERR_NO_MEMORY, "hgx_hig_compute_gisaxs: out of host memory");
  }
  HigWork& w = *c->hig;
  if (w.arena_off) {  // a simulation that ended early may still have copies in flight
    HGX_CUDA(cudaStreamSynchronize(st));
    w.arena_off = 0;
  }
  // the other arena: its last simulation's copies must have run before it is refilled (the
  // previous simulation may still be on the stream when its image is device memory)
  w.arena_cur ^= 1;
  if (w.arena_ev[w.arena_cur]) HGX_CUDA(cudaEventSynchronize(w.arena_ev[w.arena_cur]));
  const double key[8] = {(double)cp.resolution[0], (double)cp.resolution[1], cp.minpoint[0], cp.minpoint[1],
                         cp.maxpoint[0], cp.maxpoint[1], alpha_i, k0};
  bool same = w.grid != nullptr;
  for (int k = 0; k < 8 && same; ++k) same = w.key[k] == key[k];
  if (!same) {  // the grid of this description (vacuum layer: dn2 = 0)
    if (w.grid) hgx_qgrid_destroy(w.grid);
    w.grid = nullptr;
    HGX_TRY(hgx_hig_qgrid(c, h, 0.0, 0.0, &w.grid));
    for (int k = 0; k < 8; ++k) w.key[k] = key[k];
    w.ext_alpha = alpha_i;
    ++w.grid_gen;
  }
  hgx_qgrid g = w.grid;
  if (w.ext_alpha != alpha_s) {  // layer_qgrid_qz at this angle (vacuum layer: dn2 = 0)
    HGX_TRY(qgrid_reextend(g, alpha_s, k0, 0.0, 0.0));
    w.ext_alpha = alpha_s;
  }
  const long n = (long)g->nqy;
  const long nq = (long)g->nqz;  // 4n
  std::vector<double> ld, lb, lt;
  std::vector<int> lo;
  for (const auto& kv : in.layers) {
    ld.push_back(kv.second.refindex.delta);
    lb.push_back(kv.second.refindex.beta);
    lt.push_back(kv.second.thickness);
    lo.push_back(kv.second.order);
  }
  DevBuf &bfc = w.fc, &bff = w.ff, &beff = w.eff, &bsf = w.sf, &bI = w.I;
  const bool fc_grows = bfc.bytes < sizeof(double2) * nq;
  HGX_TRY(bfc.reserve(sizeof(double2) * nq));
  HGX_TRY(bff.reserve(sizeof(double2) * nq));
  HGX_TRY(beff.reserve(sizeof(double2) * nq));
  HGX_TRY(bsf.reserve(sizeof(double2) * nq));
  const int nstruct = (int)in.structures.size();
  HGX_TRY(bI.reserve(sizeof(double) * n * nstruct));
  // the Fresnel coefficients depend on the grid, the beam and the layers only: kept between
  // simulations of the same set-up (a fit moves none of them)
  std::vector<double> fkey = {(double)w.grid_gen, k0, alpha_s};
  for (size_t i = 0; i < ld.size(); ++i) fkey.insert(fkey.end(), {ld[i], lb[i], lt[i], (double)lo[i]});
  if (fc_grows || fkey != w.fc_key) {
    w.fc_key.clear();
    HGX_TRY(hgx_propagation_coeffs(c, g, (int)ld.size(), ld.data(), lb.data(), lt.data(), lo.data(),
                                   k0, alpha_s, 0, nullptr, (double*)bfc.p, 0));
    w.fc_key = fkey;
  }
  HGX_CUDA(cudaMemsetAsync(bI.p, 0, sizeof(double) * n * nstruct, st));
  // SAXS: the lattice structure factor takes the detector's real qz (sf.cpp:199-200)
  const bool saxs = sc.expt == "saxs";
  struct GridGuard {
    hgx_qgrid g = nullptr;
    ~GridGuard() {
      if (g) hgx_qgrid_destroy(g);
    }
  } gs;
  if (saxs) {
    HGX_TRY(w.saxs_qz.reserve(sizeof(double2) * n));
    real_to_complex_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, g->qz_det, (double2*)w.saxs_qz.p);
    HGX_CUDA(cudaGetLastError());
    HGX_TRY(hgx_qgrid_from_arrays(c, (int)n, g->qx, g->qy, (int)n, (const double*)w.saxs_qz.p, g->ncol, &gs.g));
  }

  // custom shapes: triangle tuples on the device, kept by the context across calls and read
  // again only when the file changes (the reference reads them on every form-factor call)
  std::map<std::string, const MeshTuples*> meshes;  // shape key -> tuples
  const std::string dir = in.path.rfind('/') == std::string::npos ? "" : in.path.substr(0, in.path.rfind('/') + 1);
  for (const auto& kv : in.shapes) {
    const hig::Shape& sh = kv.second;
    if (sh.name != "custom") continue;
    std::string path = sh.name_str;
    if (!file_exists(path) && !path.empty() && path[0] != '/' && file_exists(dir + path)) path = dir + path;
    long long size = -1, mtime = -1;
    struct stat sb;
    if (stat(path.c_str(), &sb) == 0) {
      size = (long long)sb.st_size;
      mtime = (long long)sb.st_mtim.tv_sec * 1000000000LL + sb.st_mtim.tv_nsec;
    }
    MeshTuples& m = w.meshes[path];
    if (size < 0 || m.ntri < 1 || m.size != size || m.mtime_ns != mtime) {
      m.ntri = 0;
      int ntri = 0;
      HGX_TRY(hgx_read_shapes_file(c, path.c_str(), nullptr, 0, &ntri));
      if (ntri < 1) return refuse("shape file '" + path + "' has no triangles");
      std::vector<double> sd(8 * (size_t)ntri);
      HGX_TRY(hgx_read_shapes_file(c, path.c_str(), sd.data(), ntri, &ntri));
      HGX_TRY(m.tri.reserve(sizeof(double) * sd.size()));
      HGX_CUDA(cudaMemcpyAsync(m.tri.p, sd.data(), sizeof(double) * sd.size(), cudaMemcpyHostToDevice, st));
      HGX_CUDA(cudaStreamSynchronize(st));
      m.ntri = ntri;
      m.size = size;
      m.mtime_ns = mtime;
    }
    meshes[kv.first] = &m;
  }

  const Rot rot_phi = Rot::axis(2, phi);  // rot_ = RotMatrix_t(2, phi)
  const unsigned blocks = (unsigned)((nq + 255) / 256);
  int si = 0;
  for (const auto& skv : in.structures) {  // in key order (the reference: unordered_map order)
    const hig::Structure& s = skv.second;
    const hig::Unitcell& uc = in.unitcells.at(s.unitcell_key);
    std::vector<double> dd, nn, gw;
    int ngr = 0;
    regular_centres(s, dd, ngr);
    HGX_TRY(orientations(s, ngr, nn, gw));
    double r1[3], r2[3], r3[3];
    rotation_of(s.rot1, r1);
    rotation_of(s.rot2, r2);
    rotation_of(s.rot3, r3);
    const int ax1 = (int)r1[0], ax2 = (int)r2[0], ax3 = (int)r3[0];
    std::vector<ScaleEntry> plan;
    int nscale = 0;
    std::string why;
    if (!scale_plan(s, ngr, gw, plan, nscale, why)) return refuse("structure '" + s.key + "': " + why);
    double* Is = (double*)bI.p + (size_t)si * n;
    bool all_analytic = true;
    for (const auto& ekv : uc.elements) {
      auto shp = in.shapes.find(ekv.first);
      if (shp == in.shapes.end()) return refuse("unit cell '" + uc.key + "': unknown shape '" + ekv.first + "'");
      if (shp->second.name == "custom") all_analytic = false;
      else if (shape_code(shp->second.name) < 0)
        return refuse("shape '" + shp->second.key + "': '" + shp->second.name + "' has no analytic form factor here");
    }
    if (sliced) {
      ++si;
      continue;
    }
    if (all_analytic && !saxs) {
      HGX_TRY(fused_structure(c, g, w, s, uc, in, rot_phi, dd, nn, ngr, ax1, ax2, ax3, plan, nscale,
                              (const double2*)bfc.p, Is, precision));
      ++si;
      continue;
    }
    // the paracrystal and Percus-Yevick structure factors do not depend on the grain
    if (s.type == "paracrystal") {
      HGX_TRY(hgx_sf_paracrystal(c, g, s.pc_dims, lattice_code(s.lattice.type), s.pc_dist[1], s.pc_dist[0],
                                 s.pc_sdev[1], s.pc_sdev[0], s.pc_domain, bsf.p, HGX_C128));
    } else if (s.type == "percusyevick") {
      HGX_TRY(hgx_sf_percus_yevick(c, g, s.py_diameter, s.py_volfract, s.py_dims, bsf.p, HGX_C128));
    }
    for (int gi = saxs ? std::max(ngr - 1, 0) : 0; gi < ngr; ++gi) {  // SAXS: the last grain's image stands
      const Rot rot = ((rot_phi * Rot::axis(ax3, nn[2 * ngr + gi])) * Rot::axis(ax2, nn[ngr + gi])) *
                      Rot::axis(ax1, nn[gi]);
      const double ddv[3] = {dd[gi], dd[gi + ngr], dd[gi + 2 * ngr]};
      double center[3];
      rot.apply(ddv, center);
      for (int k = 0; k < 3; ++k) center[k] += s.transvec[k];
      // the unit cell's form factor
      HGX_CUDA(cudaMemsetAsync(bff.p, 0, sizeof(double2) * nq, st));
      for (const auto& ekv : uc.elements) {  // in shape-key order
        const std::string& skey = ekv.first;
        auto shp = in.shapes.find(skey);
        if (shp == in.shapes.end()) return refuse("unit cell '" + uc.key + "': unknown shape '" + skey + "'");
        const hig::Shape& sh = shp->second;
        const Rot srot = ((rot * Rot::axis(0, sh.xrot)) * Rot::axis(1, sh.yrot)) * Rot::axis(2, sh.zrot);
        const double dre = 0.0 - 2 * sh.refindex.delta, dim = 0.0 - 2 * sh.refindex.beta;
        std::vector<double> prm;
        for (const auto& pk : sh.params) {
          const hig::ShapeParam& p = pk.second;
          const double row[7] = {(double)param_code(p.type), (double)stat_code(p.stat), p.min, p.max,
                                 p.p1, p.p2, (double)p.nvalues};
          prm.insert(prm.end(), row, row + 7);
        }
        const int code = shape_code(sh.name);
        if (sh.name != "custom" && code < 0)
          return refuse("shape '" + sh.key + "': '" + sh.name + "' has no analytic form factor here");
        // a custom shape ignores its location: its form factor at this rotation is computed once
        // and added once per location, as the reference adds it
        if (sh.name == "custom" && !ekv.second.empty()) {
          const MeshTuples& m = *meshes.at(skey);
          HGX_TRY(hgx_ff_triangles_q(c, g, (const double*)m.tri.p, m.ntri, srot.m, precision, beff.p,
                                     HGX_C128));
        }
        for (const hig::vec3& loc : ekv.second) {
          if (sh.name != "custom") {
            const double tv[3] = {loc[0], loc[1], loc[2]};
            HGX_TRY(hgx_ff_analytic_params(c, g, code, (int)(prm.size() / 7), prm.data(), 0.0, 0.0, tv,
                                           srot.m, beff.p, HGX_C128));
          }
          add_scaled_kernel<<<blocks, 256, 0, st>>>(nq, dre, dim, (const double2*)beff.p, (double2*)bff.p);
          HGX_CUDA(cudaGetLastError());
        }
      }
      // the grain's structure factors and intensity terms, one per scaling/repetition sample
      for (int k = saxs ? std::max(nscale - 1, 0) : 0; k < nscale; ++k) {  // SAXS: the last sample stands
        const ScaleEntry& e = plan[(size_t)gi * nscale + k];
        if (s.type == "paracrystal" || s.type == "percusyevick") {
          // grain-independent: computed once per structure, before the grain loop (in SAXS the
          // reference reads its first N values, the ones computed here for the first block)
        } else {
          const double abc9[9] = {e.la[0], e.la[1], e.la[2], e.lb[0], e.lb[1], e.lb[2], e.lc[0], e.lc[1], e.lc[2]};
          const double one[3] = {1.0, 1.0, 1.0};
          HGX_TRY(hgx_sf_lattice(c, saxs ? gs.g : g, abc9, e.rep, one, center, rot.m, bsf.p, HGX_C128));
        }
        if (saxs) {
          saxs_intensity_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, e.w, (const double2*)bsf.p,
                                                                          (const double2*)bff.p, Is);
          HGX_CUDA(cudaGetLastError());
        } else {
          HGX_TRY(hgx_dwba_combine(c, n, (const double*)bfc.p, (const double*)bsf.p, bff.p, HGX_C128, e.w, Is));
        }
      }
    }
    ++si;
  }
  // the structure sum (hgx_structure_sum's rescaling of the iratios and order of sums)
  std::vector<double> ratios;
  double rsum = 0.0;
  for (const auto& kv : in.structures) {
    ratios.push_back(kv.second.iratio);
    rsum += kv.second.iratio;
  }
  if (rsum != 1.0)
    for (double& v : ratios) v /= rsum;
  HGX_TRY(w.ratios.reserve(sizeof(double) * nstruct));
  HGX_TRY(arena_copy(w, st, w.ratios.p, ratios.data(), sizeof(double) * nstruct));
  const bool dev_out = is_device_ptr(image);
  if (!dev_out) HGX_TRY(w.img.reserve(sizeof(double) * n));
  double* dimg = dev_out ? image : (double*)w.img.p;
  image_structure_sum_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>((const double*)bI.p, (const double*)w.ratios.p,
                                                                        nstruct, n, dimg);
  HGX_CUDA(cudaGetLastError());
  if (!dev_out) HGX_CUDA(cudaMemcpyAsync(image, dimg, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  // the end of this simulation's work on the stream, after which its arena may be refilled
  if (!w.arena_ev[w.arena_cur])
    HGX_CUDA(cudaEventCreateWithFlags(&w.arena_ev[w.arena_cur], cudaEventDisableTiming));
  HGX_CUDA(cudaEventRecord(w.arena_ev[w.arena_cur], st));
  w.arena_off = 0;
  // a host image: synchronous, device errors reported here; a device image: asynchronous on the
  // context's stream, device errors reported by the next synchronising call
  return dev_out ? HGX_OK : hgx_synchronize(c);
}

}  // namespace

extern "C" {

int hgx_hig_image_size(hgx_hig h, int* nrow, int* ncol) {
  if (!h) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_image_size: null handle");
  if (nrow) *nrow = h->in.compute.resolution[1];
  if (ncol) *ncol = h->in.compute.resolution[0];
  return HGX_OK;
}

int hgx_hig_compute_gisaxs(hgx_ctx c, hgx_hig h, int precision, double* image) {
  if (!h) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_compute_gisaxs: null argument");
  const hig::Scattering& sc = h->in.scattering;
  if (scan_count(sc.alphai[0], sc.alphai[1], sc.alphai[2], true) > 1 ||
      scan_count(sc.inplanerot[0], sc.inplanerot[1], sc.inplanerot[2], false) > 1 ||
      scan_count(sc.tilt[0], sc.tilt[1], sc.tilt[2], false) > 1)
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_compute_gisaxs: more than one alpha_i, phi or tilt (the "
                                     "reference's compute_gisaxs refuses scans; hgx_hig_compute_scan_point "
                                     "runs them)");
  return compute_at(c, h, precision, sc.alphai[0], sc.inplanerot[0], image);
}

int hgx_hig_scan_size(hgx_hig h, int* nalphai, int* nphi, int* ntilt) {
  if (!h) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_scan_size: null handle");
  const hig::Scattering& sc = h->in.scattering;
  if (nalphai) *nalphai = std::max(0, scan_count(sc.alphai[0], sc.alphai[1], sc.alphai[2], true));
  if (nphi) *nphi = std::max(0, scan_count(sc.inplanerot[0], sc.inplanerot[1], sc.inplanerot[2], false));
  if (ntilt) *ntilt = std::max(0, scan_count(sc.tilt[0], sc.tilt[1], sc.tilt[2], false));
  return HGX_OK;
}

int hgx_hig_scan_point(hgx_hig h, int p, double* alphai_deg, double* phi_deg, double* tilt_deg) {
  if (!h) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_scan_point: null handle");
  int na = 0, np = 0, nt = 0;
  HGX_TRY(hgx_hig_scan_size(h, &na, &np, &nt));
  if (p < 0 || (long)p >= (long)na * np * nt) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_scan_point: index out of range");
  const int i = p / (np * nt), j = (p / nt) % np, k = p % nt;
  // the values as run_all_gisaxs's loops accumulate them (x += step, from the minimum)
  const hig::Scattering& sc = h->in.scattering;
  double a = sc.alphai[0], f = sc.inplanerot[0], t = sc.tilt[0];
  for (int q = 0; q < i; ++q) a += sc.alphai[2];
  for (int q = 0; q < j; ++q) f += sc.inplanerot[2];
  for (int q = 0; q < k; ++q) t += sc.tilt[2];
  if (alphai_deg) *alphai_deg = a;
  if (phi_deg) *phi_deg = f;
  if (tilt_deg) *tilt_deg = t;
  return HGX_OK;
}

int hgx_hig_compute_scan_point(hgx_ctx c, hgx_hig h, int precision, int p, double* image) {
  double a = 0.0, f = 0.0;
  HGX_TRY(hgx_hig_scan_point(h, p, &a, &f, nullptr));
  return compute_at(c, h, precision, a, f, image);
}

}  // extern "C"

// ------------------------------------------------------- tangent of the image ----
namespace hgx {
namespace {

// What a fit parameter must leave unchanged for the fused grain loop's tangent to be the
// image's: the layers and the beam (Fresnel coefficients, grid), the structures' types,
// iratios, liquid structure-factor parameters, grain counts and repetitions, and the shapes'
// refractive indices (dn2).
std::vector<double> fixed_quantities(const hig::Input& in) {
  std::vector<double> f;
  for (const auto& kv : in.layers) {
    const hig::Layer& l = kv.second;
    f.insert(f.end(), {l.refindex.delta, l.refindex.beta, l.thickness, (double)l.order});
  }
  for (const auto& kv : in.shapes)
    f.insert(f.end(), {kv.second.refindex.delta, kv.second.refindex.beta});
  for (const auto& kv : in.structures) {
    const hig::Structure& s = kv.second;
    f.insert(f.end(), {s.iratio, (double)s.pc_dims, s.pc_dist[0], s.pc_dist[1], s.pc_sdev[0], s.pc_sdev[1],
                       s.pc_domain, (double)s.py_dims, s.py_diameter, s.py_volfract, s.maxgrains[0],
                       s.maxgrains[1], s.maxgrains[2], s.repetition[0], s.repetition[1], s.repetition[2]});
  }
  const hig::Scattering& sc = in.scattering;
  f.insert(f.end(), {sc.alphai[0], sc.inplanerot[0], sc.photon_value});
  const hig::Compute& cp = in.compute;
  f.insert(f.end(), {cp.minpoint[0], cp.minpoint[1], cp.maxpoint[0], cp.maxpoint[1],
                     (double)cp.resolution[0], (double)cp.resolution[1]});
  return f;
}

// The tables of every structure at one parameter setting.
struct StructTables {
  FusedTables f;
  std::vector<ScaleEntry> plan;
  int ngr = 0, nscale = 0, shape = 0;
  bool liquid = false;
};

int all_tables(const hig::Input& in, std::vector<StructTables>& out, std::string& why) {
  out.clear();
  const Rot rot_phi = Rot::axis(2, in.scattering.inplanerot[0] * PI / 180);
  for (const auto& skv : in.structures) {
    const hig::Structure& s = skv.second;
    const hig::Unitcell& uc = in.unitcells.at(s.unitcell_key);
    StructTables T;
    std::vector<double> dd, nn, gw;
    regular_centres(s, dd, T.ngr);
    HGX_TRY(orientations(s, T.ngr, nn, gw));
    double r1[3], r2[3], r3[3];
    rotation_of(s.rot1, r1);
    rotation_of(s.rot2, r2);
    rotation_of(s.rot3, r3);
    if (!scale_plan(s, T.ngr, gw, T.plan, T.nscale, why)) return HGX_ERR_INVALID_ARG;
    HGX_TRY(fused_tables(s, uc, in, rot_phi, dd, nn, T.ngr, (int)r1[0], (int)r2[0], (int)r3[0], T.f));
    T.shape = T.f.shapes.empty() ? 0 : T.f.shapes[0].shape;
    for (const AnaShape& a : T.f.shapes)
      if (a.shape != T.shape) T.shape = 0;
    T.liquid = s.type == "paracrystal" || s.type == "percusyevick";
    out.push_back(std::move(T));
  }
  return HGX_OK;
}

}  // namespace

// dI/dx for the fit variable `var` at its current value x0 in h (FP64): the change of every
// pixel of hgx_hig_compute_gisaxs's image, added into dI (device, nrow x ncol).  The tables
// of the fused grain loop (shape samples and weights, locations, rotations, centres, lattice
// vectors, sample weights) are functions of the description that the host builds; their
// changes are taken by central differences of that set-up at x0 +- step (algebraic in x, so
// accurate to ~1e-10), and the kernel carries them through the form and structure factors and
// the DWBA sum with the hand-written tangents.  Needs a preceding hgx_hig_compute_gisaxs of h
// (its grid and Fresnel coefficients).  Refused: parameters that change a quantity listed in
// fixed_quantities or a table's size, grids with complex qz, shapes other than cylinders,
// spheres and boxes, SAXS, sliced layers, random orientations.
int hig_image_tangent(hgx_ctx c, hgx_hig h, const std::string& var, double x0, double step, double* dI) {
  auto refuse = [&](const std::string& why) {
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_objective_grad: parameter '" + var + "': " + why);
  };
  const hig::Input& in = h->in;
  if (in.scattering.expt != "gisaxs") return refuse("gradients are built for GISAXS (DWBA) descriptions");
  if (in.compute.nslices > 1) return refuse("sliced layers");
  if (!c->hig || !c->hig->grid) return refuse("no simulation of the description has run on this context");
  hgx_qgrid g = c->hig->grid;
  if (g->mode != 1) return refuse("the grid's qz blocks are complex");
  for (const auto& kv : in.structures) {
    const hig::Structure& s = kv.second;
    if (s.orientation_stat == "range" || s.orientation_stat == "random")
      return refuse("structure '" + s.key + "': orientations drawn at random change between evaluations");
    if (s.type == "paracrystal" && s.lattice.type == "") return refuse("paracrystal without lattice");
    const hig::Unitcell& uc = in.unitcells.at(s.unitcell_key);
    for (const auto& e : uc.elements) {
      const std::string& nm = in.shapes.at(e.first).name;
      if (nm != "cylinder" && nm != "sphere" && nm != "box")
        return refuse("shape '" + e.first + "' (" + nm + "): tangents are built for cylinders, spheres and boxes");
    }
  }
  // the set-up at x0 - step, x0 + step and x0
  std::string why, err;
  hig::Input ip = in, im = in;
  if (!hig::update_param(ip, var, x0 + step, err) || !hig::update_param(im, var, x0 - step, err))
    return refuse(err);
  if (fixed_quantities(ip) != fixed_quantities(im))
    return refuse("it changes a refractive index, a layer, the beam, a liquid structure factor, an iratio, "
                  "a grain count or a repetition");
  std::vector<StructTables> T0, Tp, Tm;
  int st0 = all_tables(in, T0, why);
  if (st0 != HGX_OK) return why.empty() ? st0 : refuse(why);
  if (all_tables(ip, Tp, why) != HGX_OK || all_tables(im, Tm, why) != HGX_OK) return refuse(why);
  const double inv = 1.0 / (2.0 * step);
  // iratios as the structure sum rescales them
  double rsum = 0.0;
  for (const auto& kv : in.structures) rsum += kv.second.iratio;
  cudaStream_t st = c->stream;
  HigWork& w = *c->hig;
  const long n = (long)g->nqy;
  size_t si = 0;
  for (const auto& skv : in.structures) {
    const StructTables &A = T0[si], &P = Tp[si], &M = Tm[si];
    ++si;
    if (P.ngr != M.ngr || P.nscale != M.nscale || P.f.shapes.size() != M.f.shapes.size() ||
        A.ngr != P.ngr || A.nscale != P.nscale || A.f.shapes.size() != P.f.shapes.size())
      return refuse("it changes the number of grains, samples or elements");
    if (A.shape == 0) return refuse("a unit cell mixes shapes");
    // table changes
    FusedTables D = A.f;
    for (size_t e = 0; e < D.shapes.size(); ++e) {
      for (int d = 0; d < 4; ++d) {
        const Dist &dp = P.f.shapes[e].d[d], &dm = M.f.shapes[e].d[d];
        if (dp.n != dm.n || dp.n != A.f.shapes[e].d[d].n)
          return refuse("it changes the number of a shape's samples (the reference's sampling steps)");
        for (int j = 0; j < dp.n; ++j) {
          D.shapes[e].d[d].v[j] = (dp.v[j] - dm.v[j]) * inv;
          D.shapes[e].d[d].w[j] = (dp.w[j] - dm.w[j]) * inv;
        }
      }
      for (int k = 0; k < 3; ++k) D.elems[e].loc[k] = (P.f.elems[e].loc[k] - M.f.elems[e].loc[k]) * inv;
    }
    for (size_t j = 0; j < D.gt.size(); ++j) D.gt[j] = (P.f.gt[j] - M.f.gt[j]) * inv;
    for (size_t j = 0; j < D.er.size(); ++j) D.er[j] = (P.f.er[j] - M.f.er[j]) * inv;
    std::vector<ScaleEntry> Dp = A.plan;
    for (size_t j = 0; j < Dp.size(); ++j) {
      for (int k = 0; k < 3; ++k) {
        if (P.plan[j].rep[k] != M.plan[j].rep[k]) return refuse("it changes a repetition");
        Dp[j].la[k] = (P.plan[j].la[k] - M.plan[j].la[k]) * inv;
        Dp[j].lb[k] = (P.plan[j].lb[k] - M.plan[j].lb[k]) * inv;
        Dp[j].lc[k] = (P.plan[j].lc[k] - M.plan[j].lc[k]) * inv;
        if (A.plan[j].rep[k] != rint(A.plan[j].rep[k])) return refuse("a repetition is not an integer");
      }
      Dp[j].w = (P.plan[j].w - M.plan[j].w) * inv;
    }
    // device tables: values in the forward's buffers, changes in the tangent buffers
    const int nelem = (int)A.f.elems.size();
    DevBuf &bs = w.shapes, &be = w.elems, &bg = w.gt, &br = w.er, &bc = w.sc;
    DevBuf &ds = w.tshapes, &de = w.telems, &dg = w.tgt, &dr = w.ter, &dc = w.tsc;
    auto up = [&](DevBuf& b, const void* p, size_t bytes) -> int {
      HGX_TRY(b.reserve(bytes > 0 ? bytes : 16));
      if (bytes) HGX_CUDA(cudaMemcpyAsync(b.p, p, bytes, cudaMemcpyHostToDevice, st));
      return HGX_OK;
    };
    HGX_TRY(up(bs, A.f.shapes.data(), sizeof(AnaShape) * nelem));
    HGX_TRY(up(be, A.f.elems.data(), sizeof(FusedElem) * nelem));
    HGX_TRY(up(bg, A.f.gt.data(), sizeof(double) * A.f.gt.size()));
    HGX_TRY(up(br, A.f.er.data(), sizeof(double) * A.f.er.size()));
    HGX_TRY(up(bc, A.plan.data(), sizeof(ScaleEntry) * A.plan.size()));
    HGX_TRY(up(ds, D.shapes.data(), sizeof(AnaShape) * nelem));
    HGX_TRY(up(de, D.elems.data(), sizeof(FusedElem) * nelem));
    HGX_TRY(up(dg, D.gt.data(), sizeof(double) * D.gt.size()));
    HGX_TRY(up(dr, D.er.data(), sizeof(double) * D.er.size()));
    HGX_TRY(up(dc, Dp.data(), sizeof(ScaleEntry) * Dp.size()));
    const hig::Structure& s = skv.second;
    TangentArgs ta;
    FusedArgs& a = ta.a;
    a.shapes = (const AnaShape*)bs.p;
    a.elems = (const FusedElem*)be.p;
    a.nelem = nelem;
    a.grains = (const double*)bg.p;
    a.elem_rot = (const double*)br.p;
    a.scales = (const ScaleEntry*)bc.p;
    a.nscale = A.nscale;
    a.sfbuf = nullptr;
    if (s.type == "paracrystal") {
      HGX_TRY(hgx_sf_paracrystal(c, g, s.pc_dims, lattice_code(s.lattice.type), s.pc_dist[1], s.pc_dist[0],
                                 s.pc_sdev[1], s.pc_sdev[0], s.pc_domain, w.sf.p, HGX_C128));
      a.sfbuf = (const double2*)w.sf.p;
    } else if (s.type == "percusyevick") {
      HGX_TRY(hgx_sf_percus_yevick(c, g, s.py_diameter, s.py_volfract, s.py_dims, w.sf.p, HGX_C128));
      a.sfbuf = (const double2*)w.sf.p;
    }
    a.qx = g->qx;
    a.qy = g->qy;
    a.qz = g->qz;
    a.fc = (const double2*)w.fc.p;
    a.n = n;
    a.out = nullptr;
    ta.dshapes = (const AnaShape*)ds.p;
    ta.delems = (const FusedElem*)de.p;
    ta.dgrains = (const double*)dg.p;
    ta.delem_rot = (const double*)dr.p;
    ta.dscales = (const ScaleEntry*)dc.p;
    ta.scale = rsum != 1.0 ? s.iratio / rsum : s.iratio;
    ta.dI = dI;
    const unsigned blocks = (unsigned)((4 * n + 127) / 128);
    for (int g0 = 0; g0 < A.ngr; g0 += FUSED_GRAINS_PER_LAUNCH) {
      a.g0 = g0;
      a.g1 = std::min(A.ngr, g0 + FUSED_GRAINS_PER_LAUNCH);
      launch_grain_tangent(A.shape, blocks, st, ta);
      HGX_CUDA(cudaGetLastError());
    }
    // the tables are read by the kernels before the next structure's copies (stream order)
  }
  return HGX_OK;
}

}  // namespace hgx

// ------------------------------------------------------- a fitting population ----
// The particle loop of the reference's PSO fitter (src/analyzer/hipgisaxs_fit_pso.cpp:521-545)
// calls the objective once per particle: per particle the parameters, one simulation, one
// distance.  A population here evaluates all candidates of a generation together: the host
// builds each candidate's fused grain tables from a copy of the description with the
// candidate's parameters, and one CUDA graph (recorded on the first evaluation, replayed after)
// copies the tables from pinned memory, runs every launch of the fused grain kernel for all
// candidates at once (grid y = candidate), sums the structures and reduces every candidate's
// distance, and copies the npop distances back.  The grid, the Fresnel coefficients and any
// grain-independent (paracrystal, Percus-Yevick) structure factor are made once, at creation:
// candidates may change only what the fused tables hold (shape samples, locations,
// orientations, lattice vectors, scalings), as for the objective's gradient.
namespace hgx {
namespace {

// one structure's per-candidate table sizes and its launch choices
struct PopStruct {
  int ngr = 0, nscale = 0, nelem = 0, shape = 0;
  bool liquid = false, f32c = false;
  // byte offsets in the staging block of each table's region; a region holds the table of every
  // candidate in turn (candidate i at i x the table's size)
  size_t o_shapes = 0, o_elems = 0, o_gt = 0, o_er = 0, o_sc = 0;
  size_t n_gt = 0, n_er = 0, n_sc = 0;                               // per candidate (doubles, doubles, entries)
  long sf_off = 0;                                                    // liquid: offset in sf (complex values)
};

}  // namespace
}  // namespace hgx

struct hgx_hig_pop_s {
  hgx_ctx ctx = nullptr;
  hig::Input in;                  // the description at creation (candidates change copies)
  std::vector<double> fixed;      // fixed_quantities(in)
  int npop = 0, nx = 0, metric = 0, precision = HGX_F64;
  double reg_alpha = 0.0;
  long n = 0;
  int nstruct = 0;
  hgx_qgrid grid = nullptr;
  std::vector<hgx::PopStruct> st;
  size_t stage_bytes = 0;         // the tables of all candidates and structures
  unsigned char* h_stage = nullptr;  // pinned: stage_bytes
  double* h_dist = nullptr;       // pinned: npop
  hgx::DevBuf d_stage, fc, sf, I, img, ref, mask, ratios, scratch, dist;
  std::vector<int> variants;      // the paired / per-block choice of every FP64 launch, as recorded
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace hgx {
namespace {

int pop_refuse(const std::string& why) { return fail(HGX_ERR_INVALID_ARG, "hgx_hig_population: " + why); }

// the description's fused tables with candidate x applied (a copy of the description)
int pop_tables(const hgx_hig_pop_s& P, const double* x, std::vector<StructTables>& T) {
  hig::Input ip = P.in;
  int i = 0;
  for (const auto& kv : ip.fit_params) {
    std::string err;
    if (!hig::update_param(ip, kv.second.variable, x[i++], err)) return pop_refuse(err);
  }
  if (fixed_quantities(ip) != P.fixed)
    return pop_refuse("a candidate changes a refractive index, a layer, the beam, a liquid structure factor, "
                      "an iratio, a grain count or a repetition");
  std::string why;
  const int s = all_tables(ip, T, why);
  if (s != HGX_OK) return why.empty() ? s : pop_refuse(why);
  if ((int)T.size() != P.nstruct) return pop_refuse("a candidate changes the structures");
  for (int k = 0; k < P.nstruct; ++k) {
    const PopStruct& ps = P.st[k];
    const StructTables& t = T[k];
    if (t.ngr != ps.ngr || t.nscale != ps.nscale || (int)t.f.elems.size() != ps.nelem ||
        t.f.gt.size() != ps.n_gt || t.f.er.size() != ps.n_er || t.plan.size() != ps.n_sc)
      return pop_refuse("a candidate changes the number of grains, samples or elements");
    for (const AnaShape& a : t.f.shapes)
      if (a.shape != t.f.shapes[0].shape || (ps.shape != 0 && a.shape != ps.shape))
        return pop_refuse("a candidate changes a shape");
  }
  return HGX_OK;
}

// the paired lattice factor of a launch holds when it holds for every candidate
bool pop_paired(const std::vector<std::vector<StructTables>>& all, int k, int g0, int g1) {
  for (const auto& T : all) {
    const StructTables& t = T[k];
    if (t.liquid) return false;
    for (int gi = g0; gi < g1; ++gi) {
      if (t.f.gt[12 * (size_t)gi + 2] != 0.0 || t.f.gt[12 * (size_t)gi + 5] != 0.0) return false;
      for (int s = 0; s < t.nscale; ++s)
        if (t.plan[(size_t)gi * t.nscale + s].la[2] != 0.0) return false;
    }
  }
  return true;
}

// grains per launch: about FUSED_GRAINS_PER_LAUNCH grain evaluations over all candidates
int pop_chunk(int npop) { return std::max(1, FUSED_GRAINS_PER_LAUNCH / npop); }


int pop_enqueue(hgx_hig_pop_s& P, cudaStream_t st) {
  const long n = P.n;
  HGX_CUDA(cudaMemcpyAsync(P.d_stage.p, P.h_stage, P.stage_bytes, cudaMemcpyHostToDevice, st));
  HGX_CUDA(cudaMemsetAsync(P.I.p, 0, sizeof(double) * n * P.nstruct * P.npop, st));
  const unsigned char* base = (const unsigned char*)P.d_stage.p;
  const int chunk = pop_chunk(P.npop);
  size_t vi = 0;
  for (int k = 0; k < P.nstruct; ++k) {
    const PopStruct& ps = P.st[k];
    FusedArgs a;
    a.shapes = (const AnaShape*)(base + ps.o_shapes);
    a.elems = (const FusedElem*)(base + ps.o_elems);
    a.nelem = ps.nelem;
    a.grains = (const double*)(base + ps.o_gt);
    a.elem_rot = (const double*)(base + ps.o_er);
    a.scales = (const ScaleEntry*)(base + ps.o_sc);
    a.nscale = ps.nscale;
    a.sfbuf = ps.liquid ? (const double2*)P.sf.p + ps.sf_off : nullptr;
    a.qx = P.grid->qx;
    a.qy = P.grid->qy;
    a.qz = P.grid->qz;
    a.fc = (const double2*)P.fc.p;
    a.n = n;
    a.out = (double*)P.I.p + (size_t)k * n;
    // candidate strides in records: each region holds one table per candidate
    a.ps_shape = ps.nelem;
    a.ps_elem = ps.nelem;
    a.ps_grain = (long)ps.n_gt;
    a.ps_er = (long)ps.n_er;
    a.ps_scale = (long)ps.n_sc;
    a.ps_out = n * P.nstruct;
    const dim3 grid((unsigned)((4 * n + 127) / 128), (unsigned)P.npop);
    for (int g0 = 0; g0 < ps.ngr; g0 += chunk) {
      a.g0 = g0;
      a.g1 = std::min(ps.ngr, g0 + chunk);
      if (ps.f32c) {
        switch (ps.shape) {
          case SH_CYLINDER: grain_dwba_f32c_kernel<SH_CYLINDER><<<grid, 128, 0, st>>>(a); break;
          case SH_SPHERE: grain_dwba_f32c_kernel<SH_SPHERE><<<grid, 128, 0, st>>>(a); break;
          default: grain_dwba_f32c_kernel<SH_BOX><<<grid, 128, 0, st>>>(a); break;
        }
      } else {
        const int paired = P.variants[vi++];
#define HGX_POP_LAUNCH(S)                                                   \
  (paired ? (void)(grain_dwba_kernel<S, 1><<<grid, 128, 0, st>>>(a))      \
          : (void)(grain_dwba_kernel<S, 0><<<grid, 128, 0, st>>>(a)))
        switch (ps.shape) {
          case SH_CYLINDER: HGX_POP_LAUNCH(SH_CYLINDER); break;
          case SH_SPHERE: HGX_POP_LAUNCH(SH_SPHERE); break;
          case SH_BOX: HGX_POP_LAUNCH(SH_BOX); break;
          case SH_CUBE: HGX_POP_LAUNCH(SH_CUBE); break;
          case SH_PRISM3: HGX_POP_LAUNCH(SH_PRISM3); break;
          case SH_PRISM6: HGX_POP_LAUNCH(SH_PRISM6); break;
          case SH_PYRAMID: HGX_POP_LAUNCH(SH_PYRAMID); break;
          default: HGX_POP_LAUNCH(0); break;
        }
#undef HGX_POP_LAUNCH
      }
      HGX_CUDA(cudaGetLastError());
    }
  }
  image_structure_sum_kernel<<<dim3((unsigned)((n + 255) / 256), (unsigned)P.npop), 256, 0, st>>>(
      (const double*)P.I.p, (const double*)P.ratios.p, P.nstruct, n, (double*)P.img.p);
  HGX_CUDA(cudaGetLastError());
  HGX_TRY(fit_distance_population(st, P.metric, n, (const double*)P.ref.p, (const double*)P.img.p,
                                  (const unsigned*)P.mask.p, P.npop, (double*)P.scratch.p, (double*)P.dist.p));
  HGX_CUDA(cudaMemcpyAsync(P.h_dist, P.dist.p, sizeof(double) * P.npop, cudaMemcpyDeviceToHost, st));
  return HGX_OK;
}

}  // namespace
}  // namespace hgx

extern "C" {

int hgx_hig_population_destroy(hgx_hig_pop p) {
  if (!p) return HGX_OK;
  cudaSetDevice(p->ctx->device);
  cudaStreamSynchronize(p->ctx->stream);
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->grid) hgx_qgrid_destroy(p->grid);
  if (p->h_stage) cudaFreeHost(p->h_stage);
  if (p->h_dist) cudaFreeHost(p->h_dist);
  delete p;
  return HGX_OK;
}

int hgx_hig_population_create(hgx_ctx c, hgx_hig h, int npop, const double* ref, const unsigned* mask,
                              int metric, double reg_alpha, int precision, hgx_hig_pop* out) {
  if (!c || !h || !ref || !out || npop < 1) return pop_refuse("null argument or empty population");
  *out = nullptr;
  if (metric < 0 || metric > 7 || metric == 4 || metric == 5)
    return pop_refuse("a scalar distance measure is needed (not the residual vectors)");
  if (precision != HGX_F64 && precision != HGX_F32C) return pop_refuse("unknown precision");
  if (npop > 65535) return pop_refuse("at most 65,535 candidates");
  const hig::Input& in = h->in;
  const hig::Compute& cp = in.compute;
  if (in.scattering.expt != "gisaxs") return pop_refuse("populations are built for GISAXS (DWBA) descriptions");
  if (cp.nslices > 1) return pop_refuse("sliced layers");
  if (cp.structcorrelation != "null" && cp.structcorrelation != "nGnE")
    return pop_refuse("structure correlation '" + cp.structcorrelation + "' is not supported");
  if (in.structures.empty()) return pop_refuse("the description has no structure");
  for (const auto& kv : in.structures) {
    const hig::Structure& s = kv.second;
    if (s.distribution != "regular") return pop_refuse("structure '" + s.key + "': ensemble distribution '" + s.distribution + "'");
    if (!in.unitcells.count(s.unitcell_key)) return pop_refuse("structure '" + s.key + "': unknown unit cell");
    if (s.maxgrains[0] < 1 || s.maxgrains[1] < 1 || s.maxgrains[2] < 1) return pop_refuse("maxgrains must be >= 1");
    if (s.orientation_stat == "range" || s.orientation_stat == "random")
      return pop_refuse("structure '" + s.key + "': orientations drawn at random change between candidates");
    if (s.type == "paracrystal" && s.lattice.type == "") return pop_refuse("paracrystal without lattice");
    for (const auto& e : in.unitcells.at(s.unitcell_key).elements) {
      auto shp = in.shapes.find(e.first);
      if (shp == in.shapes.end()) return pop_refuse("unknown shape '" + e.first + "'");
      if (shp->second.name == "custom" || shape_code(shp->second.name) < 0)
        return pop_refuse("shape '" + e.first + "' (" + shp->second.name + "): the fused grain loop takes analytic shapes");
    }
  }
  HGX_CUDA(cudaSetDevice(c->device));
  auto p = new (std::nothrow) hgx_hig_pop_s;
  if (!p) return fail(HGX_ERR_NO_MEMORY, "hgx_hig_population_create: host allocation");
  auto bail = [&](int s) {
    hgx_hig_population_destroy(p);
    return s;
  };
  p->ctx = c;
  p->in = in;
  p->fixed = fixed_quantities(in);
  p->npop = npop;
  p->nx = (int)in.fit_params.size();
  p->metric = metric;
  p->precision = precision;
  p->reg_alpha = reg_alpha;
  cudaStream_t st = c->stream;
  // grid and Fresnel coefficients as hgx_hig_compute_gisaxs makes them
  double k0, alpha_i;
  int s = hgx_hig_beam(h, &k0, &alpha_i, nullptr);
  if (s) return bail(s);
  const double alpha_s = in.scattering.alphai[0] * PI / 180;
  if ((s = hgx_hig_qgrid(c, h, 0.0, 0.0, &p->grid))) return bail(s);
  if (alpha_s != alpha_i && (s = qgrid_reextend(p->grid, alpha_s, k0, 0.0, 0.0))) return bail(s);
  hgx_qgrid g = p->grid;
  p->n = (long)g->nqy;
  const long n = p->n, nq = (long)g->nqz;
  std::vector<double> ld, lb, lt;
  std::vector<int> lo;
  for (const auto& kv : in.layers) {
    ld.push_back(kv.second.refindex.delta);
    lb.push_back(kv.second.refindex.beta);
    lt.push_back(kv.second.thickness);
    lo.push_back(kv.second.order);
  }
  if ((s = p->fc.reserve(sizeof(double2) * nq))) return bail(s);
  if ((s = hgx_propagation_coeffs(c, g, (int)ld.size(), ld.data(), lb.data(), lt.data(), lo.data(), k0, alpha_s, 0,
                                  nullptr, (double*)p->fc.p, 0)))
    return bail(s);
  // the table layout (from the description's own parameters) and the grain-independent factors
  std::vector<StructTables> T0;
  std::string why;
  s = all_tables(in, T0, why);
  if (s) return bail(why.empty() ? s : pop_refuse(why));
  p->nstruct = (int)T0.size();
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) & ~(size_t)255;
    return o;
  };
  int nliquid = 0;
  for (const StructTables& t : T0) {
    PopStruct ps;
    ps.ngr = t.ngr;
    ps.nscale = t.nscale;
    ps.nelem = (int)t.f.elems.size();
    ps.shape = t.shape;
    ps.liquid = t.liquid;
    ps.f32c = precision == HGX_F32C && g->mode == 1 && grain_f32c_shape(t.shape);
    ps.n_gt = t.f.gt.size();
    ps.n_er = t.f.er.size();
    ps.n_sc = t.plan.size();
    ps.o_shapes = take(sizeof(AnaShape) * ps.nelem * npop);
    ps.o_elems = take(sizeof(FusedElem) * ps.nelem * npop);
    ps.o_gt = take(sizeof(double) * ps.n_gt * npop);
    ps.o_er = take(sizeof(double) * ps.n_er * npop);
    ps.o_sc = take(sizeof(ScaleEntry) * ps.n_sc * npop);
    if (ps.liquid) ps.sf_off = (long)nliquid++ * nq;
    p->st.push_back(ps);
  }
  p->stage_bytes = std::max<size_t>(off, 256);
  if (cudaMallocHost(&p->h_stage, p->stage_bytes) != cudaSuccess ||
      cudaMallocHost(&p->h_dist, sizeof(double) * npop) != cudaSuccess)
    return bail(fail(HGX_ERR_NO_MEMORY, "hgx_hig_population_create: pinned host memory"));
  if ((s = p->d_stage.reserve(p->stage_bytes)) || (s = p->I.reserve(sizeof(double) * n * p->nstruct * npop)) ||
      (s = p->img.reserve(sizeof(double) * n * npop)) || (s = p->ref.reserve(sizeof(double) * n)) ||
      (s = p->ratios.reserve(sizeof(double) * p->nstruct)) ||
      (s = p->scratch.reserve(sizeof(double) * fit_population_scratch(npop))) ||
      (s = p->dist.reserve(sizeof(double) * npop)))
    return bail(s);
  if (nliquid > 0 && (s = p->sf.reserve(sizeof(double2) * nq * nliquid))) return bail(s);
  int li = 0;
  for (const auto& kv : in.structures) {
    const hig::Structure& S = kv.second;
    if (S.type == "paracrystal")
      s = hgx_sf_paracrystal(c, g, S.pc_dims, lattice_code(S.lattice.type), S.pc_dist[1], S.pc_dist[0], S.pc_sdev[1],
                             S.pc_sdev[0], S.pc_domain, (double2*)p->sf.p + (long)li++ * nq, HGX_C128);
    else if (S.type == "percusyevick")
      s = hgx_sf_percus_yevick(c, g, S.py_diameter, S.py_volfract, S.py_dims, (double2*)p->sf.p + (long)li++ * nq,
                               HGX_C128);
    if (s) return bail(s);
  }
  std::vector<double> r;
  double rsum = 0.0;
  for (const auto& kv : in.structures) {
    r.push_back(kv.second.iratio);
    rsum += kv.second.iratio;
  }
  if (rsum != 1.0)
    for (double& v : r) v /= rsum;
  cudaError_t e = cudaMemcpyAsync(p->ratios.p, r.data(), sizeof(double) * r.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(p->ref.p, ref, sizeof(double) * n, is_device_ptr(ref) ? cudaMemcpyDeviceToDevice
                                                                            : cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && mask) {
    if ((s = p->mask.reserve(sizeof(unsigned) * n))) return bail(s);
    e = cudaMemcpyAsync(p->mask.p, mask, sizeof(unsigned) * n, is_device_ptr(mask) ? cudaMemcpyDeviceToDevice
                                                                                  : cudaMemcpyHostToDevice, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return bail(cuda_fail(e, "hgx_hig_population_create: copies"));
  *out = p;
  return HGX_OK;
}

int hgx_hig_population_eval(hgx_hig_pop p, const double* X, int nx, double* dist) {
  if (!p || !X || !dist) return pop_refuse("null argument");
  if (nx != p->nx) return pop_refuse("X must hold one value per fit parameter and candidate");
  if (is_device_ptr(dist) || is_device_ptr(X)) return pop_refuse("X and dist are host arrays");
  HGX_CUDA(cudaSetDevice(p->ctx->device));
  cudaStream_t st = p->ctx->stream;
  HGX_CUDA(cudaStreamSynchronize(st));  // the pinned staging block is about to change
  // every candidate's tables from its own copy of the description, into its place in each
  // table's region of the staging block
  std::vector<std::vector<StructTables>> all((size_t)p->npop);
  for (int i = 0; i < p->npop; ++i) {
    HGX_TRY(pop_tables(*p, X + (size_t)i * nx, all[i]));
    unsigned char* h = p->h_stage;
    for (int k = 0; k < p->nstruct; ++k) {
      const PopStruct& ps = p->st[k];
      const StructTables& t = all[i][k];
      const size_t ne = (size_t)ps.nelem;
      memcpy(h + ps.o_shapes + sizeof(AnaShape) * ne * i, t.f.shapes.data(), sizeof(AnaShape) * ne);
      memcpy(h + ps.o_elems + sizeof(FusedElem) * ne * i, t.f.elems.data(), sizeof(FusedElem) * ne);
      memcpy(h + ps.o_gt + sizeof(double) * ps.n_gt * i, t.f.gt.data(), sizeof(double) * ps.n_gt);
      memcpy(h + ps.o_er + sizeof(double) * ps.n_er * i, t.f.er.data(), sizeof(double) * ps.n_er);
      memcpy(h + ps.o_sc + sizeof(ScaleEntry) * ps.n_sc * i, t.plan.data(), sizeof(ScaleEntry) * ps.n_sc);
    }
  }
  // the paired / per-block choice of every FP64 launch for this generation
  std::vector<int> v;
  const int chunk = pop_chunk(p->npop);
  for (int k = 0; k < p->nstruct; ++k) {
    const PopStruct& ps = p->st[k];
    if (ps.f32c) continue;
    for (int g0 = 0; g0 < ps.ngr; g0 += chunk) v.push_back(pop_paired(all, k, g0, std::min(ps.ngr, g0 + chunk)));
  }
  if (p->exec && v != p->variants) {  // another kernel variant: record the graph again
    cudaGraphExecDestroy(p->exec);
    cudaGraphDestroy(p->graph);
    p->exec = nullptr;
    p->graph = nullptr;
  }
  p->variants = v;
  if (!p->exec) {
    cudaStream_t cap = nullptr;
    HGX_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    int s = HGX_OK;
    if (e == cudaSuccess) s = pop_enqueue(*p, cap);
    cudaGraph_t graph = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
    cudaStreamDestroy(cap);
    if (e != cudaSuccess || s != HGX_OK || e2 != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
      if (s != HGX_OK) return s;
      return cuda_fail(e2, "cudaStreamEndCapture");
    }
    p->graph = graph;
    HGX_CUDA(cudaGraphInstantiate(&p->exec, graph, 0));
  }
  HGX_CUDA(cudaGraphLaunch(p->exec, st));
  HGX_CUDA(cudaStreamSynchronize(st));
  HGX_TRY(hgx_synchronize(p->ctx));
  // the regularisation of HipGISAXSObjectiveFunction::operator() (objective_func_hipgisaxs.cpp:300-320)
  for (int i = 0; i < p->npop; ++i) {
    double pmean = 0.0;
    int j = 0;
    for (const auto& kv : p->in.fit_params) {
      const double mean = (kv.second.range[1] - kv.second.range[0]) / 2.0 + kv.second.range[0];
      double t = X[(size_t)i * nx + j++] - mean;
      t *= t;
      pmean += t;
    }
    const double reg = (p->reg_alpha / 2) * pmean;
    dist[i] = isfinite(p->h_dist[i]) ? p->h_dist[i] + reg : 1e8;
  }
  return HGX_OK;
}

}  // extern "C"

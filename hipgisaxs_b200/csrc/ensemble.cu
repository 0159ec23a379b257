// The grain loop of HipGISAXS::run_gisaxs for one structure whose unit cell holds one
// triangulated particle (src/sim/hipgisaxs_main.cpp:794-1100), on the device: for every
// grain g (orientation R_g, unit-cell centre c_g, weight w_g — the reference's rot, center and
// gauss_weight * scaling weight, :946-951, :958-960, :1045),
//   ff_g = dn2 F(shape_def rotated by R_g)                       (:983-1015)
//   sf_g = lattice structure factor at (c_g, R_g)                (:1050-1058)
//   I   += | w_g sum_k fc_k sf_gk ff_gk |^2                      (:1086-1100)
// The grains run back to back on the context's stream with no host round trip: the mesh and
// the Fresnel coefficients are copied to the device once, the form-factor and
// structure-factor buffers are reused across grains, and the intensity stays on the device
// until the last grain.  The form factor dominates the cost (the structure factor and the
// combination read and write a few bytes per q-point), so the three steps stay separate
// kernels.
#include <cuda_runtime.h>
#include <math.h>

#include "hgx_internal.cuh"

using namespace hgx;

extern "C" {

int hgx_dwba_mesh_grains(hgx_ctx c, hgx_qgrid g, const double* shape_def, int ntri, int ngrains,
                         const double* rots, const double* centers, const double* weights,
                         const double* abc9, const double* repet, const double* scaling,
                         const double* fc, double dn2_re, double dn2_im, int precision,
                         double* intensity) {
  if (!c || !g || !shape_def || !rots || !centers || !weights || !abc9 || !repet || !scaling ||
      !fc || !intensity)
    return fail(HGX_ERR_INVALID_ARG, "hgx_dwba_mesh_grains: null argument");
  if (ntri < 1 || ngrains < 1)
    return fail(HGX_ERR_INVALID_ARG, "hgx_dwba_mesh_grains: no triangles or no grains");
  if (g->ctx != c) return fail(HGX_ERR_INVALID_ARG, "hgx_dwba_mesh_grains: grid of another context");
  if (g->nk != 4)
    return fail(HGX_ERR_INVALID_ARG, "hgx_dwba_mesh_grains: needs a DWBA grid (4 qz blocks per pixel)");
  if (precision != HGX_F64 && precision != HGX_F32C)
    return fail(HGX_ERR_INVALID_ARG, "hgx_dwba_mesh_grains: unknown precision");
  HGX_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  const long n = g->nqy;  // pixels
  const size_t nq = (size_t)g->nqz;
  DevBuf bsd, bfc, bff, bsf, bI;
  const void* dsd = nullptr;
  const void* dfc = nullptr;
  HGX_TRY(stage_in(c, shape_def, sizeof(double) * 8 * (size_t)ntri, bsd, &dsd));
  HGX_TRY(stage_in(c, fc, sizeof(double2) * nq, bfc, &dfc));
  const int fft = precision == HGX_F64 ? HGX_C128 : HGX_C64;
  HGX_TRY(bff.reserve((fft == HGX_C128 ? sizeof(double2) : sizeof(float2)) * nq));
  HGX_TRY(bsf.reserve(sizeof(double2) * nq));
  void* dI = nullptr;
  HGX_TRY(stage_out(c, intensity, sizeof(double) * n, bI, &dI));
  HGX_CUDA(cudaMemsetAsync(dI, 0, sizeof(double) * n, st));
  const double dn2_abs = hypot(dn2_re, dn2_im);  // |w dn2 X|^2 = (w |dn2|)^2 |X|^2
  for (int k = 0; k < ngrains; ++k) {
    HGX_TRY(hgx_ff_triangles_q(c, g, (const double*)dsd, ntri, rots + 9L * k, precision, bff.p, fft));
    HGX_TRY(hgx_sf_lattice(c, g, abc9, repet, scaling, centers + 3L * k, rots + 9L * k, bsf.p, HGX_C128));
    HGX_TRY(hgx_dwba_combine(c, n, (const double*)dfc, (const double*)bsf.p, bff.p, fft,
                             weights[k] * dn2_abs, (double*)dI));
  }
  HGX_TRY(finish_out(c, intensity, sizeof(double) * n, dI));
  return hgx_synchronize(c);
}

}  // extern "C"

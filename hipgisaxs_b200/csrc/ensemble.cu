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

#include <vector>

#include "hgx_internal.cuh"

namespace hgx {

// img[z] = sum_s I_s[z] r_s, structures in order (src/sim/hipgisaxs_main.cpp:1352-1362)
__global__ void structure_sum_kernel(const double* __restrict__ I, const double* __restrict__ r,
                                     int ns, long n, double* __restrict__ out) {
  const long z = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= n) return;
  double sum = 0.0;
  // separate multiply and add (no fused multiply-add), rounding as the reference's loop does
  for (int s = 0; s < ns; ++s) sum = __dadd_rn(sum, __dmul_rn(I[(long)s * n + z], r[s]));
  out[z] = sum;
}

}  // namespace hgx

using namespace hgx;

namespace hgx {

// The shared grain loop: form factor of grain k into F (callback), then the structure factor
// and the DWBA accumulation; everything on the context's stream.
template <typename FF>
static int grain_loop(hgx_ctx c, hgx_qgrid g, int ngrains, const double* rots, const double* centers,
                      const double* weights, const double* abc9, const double* repet,
                      const double* scaling, const double* fc, double dn2_re, double dn2_im,
                      int fft, double* intensity, FF&& form_factor) {
  if (g->ctx != c) return fail(HGX_ERR_INVALID_ARG, "grain loop: grid of another context");
  if (g->nk != 4) return fail(HGX_ERR_INVALID_ARG, "grain loop: needs a DWBA grid (4 qz blocks per pixel)");
  HGX_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  const long n = g->nqy;  // pixels
  const size_t nq = (size_t)g->nqz;
  DevBuf bfc, bff, bsf, bI;
  const void* dfc = nullptr;
  HGX_TRY(stage_in(c, fc, sizeof(double2) * nq, bfc, &dfc));
  HGX_TRY(bff.reserve((fft == HGX_C128 ? sizeof(double2) : sizeof(float2)) * nq));
  HGX_TRY(bsf.reserve(sizeof(double2) * nq));
  void* dI = nullptr;
  HGX_TRY(stage_out(c, intensity, sizeof(double) * n, bI, &dI));
  HGX_CUDA(cudaMemsetAsync(dI, 0, sizeof(double) * n, st));
  const double dn2_abs = hypot(dn2_re, dn2_im);  // |w dn2 X|^2 = (w |dn2|)^2 |X|^2
  for (int k = 0; k < ngrains; ++k) {
    HGX_TRY(form_factor(k, bff.p));
    HGX_TRY(hgx_sf_lattice(c, g, abc9, repet, scaling, centers + 3L * k, rots + 9L * k, bsf.p, HGX_C128));
    HGX_TRY(hgx_dwba_combine(c, n, (const double*)dfc, (const double*)bsf.p, bff.p, fft,
                             weights[k] * dn2_abs, (double*)dI));
  }
  HGX_TRY(finish_out(c, intensity, sizeof(double) * n, dI));
  return hgx_synchronize(c);
}

}  // namespace hgx

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
  if (precision != HGX_F64 && precision != HGX_F32C)
    return fail(HGX_ERR_INVALID_ARG, "hgx_dwba_mesh_grains: unknown precision");
  HGX_CUDA(cudaSetDevice(c->device));
  DevBuf bsd;
  const void* dsd = nullptr;
  HGX_TRY(stage_in(c, shape_def, sizeof(double) * 8 * (size_t)ntri, bsd, &dsd));
  const int fft = precision == HGX_F64 ? HGX_C128 : HGX_C64;
  return grain_loop(c, g, ngrains, rots, centers, weights, abc9, repet, scaling, fc, dn2_re, dn2_im,
                    fft, intensity, [&](int k, void* F) {
                      return hgx_ff_triangles_q(c, g, (const double*)dsd, ntri, rots + 9L * k,
                                                precision, F, fft);
                    });
}

int hgx_dwba_analytic_grains(hgx_ctx c, hgx_qgrid g, int shape, int nparam, const double* params,
                             double tau, double eta, const double* transvec, int ngrains,
                             const double* rots, const double* centers, const double* weights,
                             const double* abc9, const double* repet, const double* scaling,
                             const double* fc, double dn2_re, double dn2_im, double* intensity) {
  if (!c || !g || !params || !rots || !centers || !weights || !abc9 || !repet || !scaling || !fc ||
      !intensity)
    return fail(HGX_ERR_INVALID_ARG, "hgx_dwba_analytic_grains: null argument");
  if (ngrains < 1 || nparam < 1)
    return fail(HGX_ERR_INVALID_ARG, "hgx_dwba_analytic_grains: no grains or no shape parameters");
  return grain_loop(c, g, ngrains, rots, centers, weights, abc9, repet, scaling, fc, dn2_re, dn2_im,
                    HGX_C128, intensity, [&](int k, void* F) {
                      return hgx_ff_analytic_params(c, g, shape, nparam, params, tau, eta, transvec,
                                                    rots + 9L * k, F, HGX_C128);
                    });
}

// The sum over structures of HipGISAXS::run_gisaxs for uncorrelated structures (its default,
// src/sim/hipgisaxs_main.cpp:1278-1293, 1352-1362): the iratios are rescaled to sum to 1
// unless they already do, and img[z] = sum_s intensities[s n + z] iratio_s.
int hgx_structure_sum(hgx_ctx c, int nstruct, long n, const double* intensities,
                      const double* iratios, double* out) {
  if (!c || !intensities || !iratios || !out || nstruct < 1 || n < 1)
    return fail(HGX_ERR_INVALID_ARG, "hgx_structure_sum: null argument or empty input");
  std::vector<double> r(iratios, iratios + nstruct);
  double rsum = 0.0;
  for (double v : r) rsum += v;
  if (rsum != 1.0)
    for (double& v : r) v /= rsum;
  HGX_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  DevBuf bI, br, bo;
  const void* dI = nullptr;
  HGX_TRY(stage_in(c, intensities, sizeof(double) * (size_t)nstruct * n, bI, &dI));
  HGX_TRY(br.reserve(sizeof(double) * nstruct));
  HGX_CUDA(cudaMemcpyAsync(br.p, r.data(), sizeof(double) * nstruct, cudaMemcpyHostToDevice, st));
  void* dout = nullptr;
  HGX_TRY(stage_out(c, out, sizeof(double) * n, bo, &dout));
  structure_sum_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>((const double*)dI, (const double*)br.p,
                                                                   nstruct, n, (double*)dout);
  HGX_CUDA(cudaGetLastError());
  HGX_TRY(finish_out(c, out, sizeof(double) * n, dout));
  return hgx_synchronize(c);
}

}  // extern "C"

// C ABI of the HiG input reader (hig_input.cpp) and the device set-up that HipGISAXS::init
// derives from it (src/sim/hipgisaxs_main.cpp:106-216).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <iterator>
#include <new>
#include <string>

#include "hgx_internal.cuh"
#include "hig_config.hpp"

using namespace hgx;

extern "C" {

int hgx_hig_read(const char* path, hgx_hig* out) {
  if (!path || !out) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_read: null argument");
  *out = nullptr;
  hgx_hig h = new (std::nothrow) hgx_hig_s;
  if (!h) return fail(HGX_ERR_NO_MEMORY, "hgx_hig_read: out of host memory");
  std::string err;
  if (!hig::read_input(path, h->in, err)) {
    delete h;
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_read: " + err);
  }
  *out = h;
  return HGX_OK;
}

int hgx_hig_json(hgx_hig h, char* buf, size_t cap, size_t* len) {
  if (!h) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_json: null handle");
  if (h->json.empty()) h->json = hig::to_json(h->in);
  if (len) *len = h->json.size();
  if (!buf) return HGX_OK;
  if (cap <= h->json.size()) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_json: buffer too small");
  memcpy(buf, h->json.c_str(), h->json.size() + 1);
  return HGX_OK;
}

int hgx_hig_destroy(hgx_hig h) {
  delete h;
  return HGX_OK;
}

int hgx_hig_beam(hgx_hig h, double* k0, double* alpha_i, double* freq) {
  if (!h) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_beam: null handle");
  double k, f;
  if (!hig::photon_k0(h->in.scattering, &k, &f))
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_beam: photon unit must be \"ev\" or \"kev\"");
  if (k0) *k0 = k;
  if (freq) *freq = f;
  if (alpha_i) *alpha_i = h->in.scattering.alphai[0] * 3.141592653589793 / 180;
  return HGX_OK;
}

int hgx_hig_update_param(hgx_hig h, const char* variable, double value) {
  if (!h || !variable) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_update_param: null argument");
  std::string err;
  if (!hig::update_param(h->in, variable, value, err)) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_update_param: " + err);
  h->json.clear();
  return HGX_OK;
}

int hgx_hig_fit_count(hgx_hig h, int* n) {
  if (!h || !n) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_fit_count: null argument");
  *n = (int)h->in.fit_params.size();
  return HGX_OK;
}

int hgx_hig_fit_param(hgx_hig h, int i, char* key, size_t key_cap, char* variable, size_t var_cap,
                      double* range3, double* init) {
  if (!h) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_fit_param: null handle");
  if (i < 0 || i >= (int)h->in.fit_params.size())
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_fit_param: index out of range");
  auto it = h->in.fit_params.begin();
  std::advance(it, i);
  const hig::FitParam& p = it->second;
  if (key) {
    if (key_cap <= p.key.size()) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_fit_param: key buffer too small");
    memcpy(key, p.key.c_str(), p.key.size() + 1);
  }
  if (variable) {
    if (var_cap <= p.variable.size()) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_fit_param: variable buffer too small");
    memcpy(variable, p.variable.c_str(), p.variable.size() + 1);
  }
  if (range3)
    for (int k = 0; k < 3; ++k) range3[k] = p.range[k];
  if (init) *init = p.init;
  return HGX_OK;
}

namespace {
int put_str(const std::string& v, char* buf, size_t cap, const char* what) {
  if (!buf) return HGX_OK;
  if (cap <= v.size()) return fail(HGX_ERR_INVALID_ARG, std::string(what) + ": buffer too small");
  memcpy(buf, v.c_str(), v.size() + 1);
  return HGX_OK;
}
}  // namespace

int hgx_hig_fit_reference(hgx_hig h, int i, char* path, size_t path_cap, char* mask, size_t mask_cap,
                          int* npar, int* nperp) {
  if (!h) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_fit_reference: null handle");
  if (!h->in.reference_data_set || i != 0)
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_fit_reference: no referencedata block of that index");
  const hig::FitReferenceData& r = h->in.reference_data;
  HGX_TRY(put_str(r.path_set ? r.path : std::string(), path, path_cap, "hgx_hig_fit_reference"));
  HGX_TRY(put_str(r.mask_set ? r.mask : std::string(), mask, mask_cap, "hgx_hig_fit_reference"));
  if (npar) *npar = (int)r.npoints_parallel;
  if (nperp) *nperp = (int)r.npoints_perpendicular;
  return HGX_OK;
}

// HipGISAXS::override_qregion (src/sim/hipgisaxs_main.cpp:236-277) with QGrid::update
// (src/model/qgrid.cpp:133-197), whose arithmetic is QGrid::create's for the given size and
// region: the computation block takes the reference data's fit region and the image's size
int hgx_hig_override_qregion(hgx_hig h, int ny, int nz, int i) {
  if (!h) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_override_qregion: null handle");
  if (ny < 1 || nz < 1) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_override_qregion: empty size");
  if (!h->in.reference_data_set || i != 0)
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_override_qregion: no referencedata block of that index");
  hig::Compute& c = h->in.compute;
  if (c.region_type == "pixels" || c.region_type == "angles")  // "not yet implemented" there
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_override_qregion: only a qspace output region can be overridden");
  if (c.region_type != "qspace")
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_override_qregion: unknown output region type");
  const hig::FitReferenceData& r = h->in.reference_data;
  c.resolution[0] = ny;
  c.resolution[1] = nz;
  c.minpoint = r.region_min;
  c.maxpoint = r.region_max;
  h->json.clear();
  return HGX_OK;
}

int hgx_hig_output_names(hgx_hig h, char* pathprefix, size_t prefix_cap, char* runname, size_t run_cap) {
  if (!h) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_output_names: null handle");
  const hig::Compute& c = h->in.compute;
  HGX_TRY(put_str(c.pathprefix, pathprefix, prefix_cap, "hgx_hig_output_names"));
  HGX_TRY(put_str(c.runname_set ? c.runname : std::string(), runname, run_cap, "hgx_hig_output_names"));
  return HGX_OK;
}

int hgx_hig_fit_algorithm_count(hgx_hig h, int* n) {
  if (!h || !n) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_fit_algorithm_count: null argument");
  *n = (int)h->in.algorithms.size();
  return HGX_OK;
}

int hgx_hig_fit_algorithm(hgx_hig h, int i, char* name, size_t name_cap, int* metric, double* tolerance,
                          double* regularization) {
  if (!h) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_fit_algorithm: null handle");
  if (i < 0 || i >= (int)h->in.algorithms.size())
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_fit_algorithm: index out of range");
  const hig::FitAlgorithm& a = h->in.algorithms[i];
  HGX_TRY(put_str(a.name, name, name_cap, "hgx_hig_fit_algorithm"));
  if (metric) {
    static const char* const names[] = {"sqrt_unit_l2", "sqrt_c_l2", "cbrt_unit_l2", "cbrt_c_l2",
                                        "sqrt_unit_l2_residual", "sqrt_c_l2_residual",
                                        "sqrt_unit_l1", "cbrt_unit_l1"};
    *metric = -1;
    if (a.metric_set)
      for (int k = 0; k < 8; ++k)
        if (a.distance_metric == names[k]) *metric = k;
  }
  if (tolerance) *tolerance = a.tolerance;
  if (regularization) *regularization = a.regularization;
  return HGX_OK;
}

int hgx_hig_fit_update(hgx_hig h, const double* x, int n) {
  if (!h || (n > 0 && !x)) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_fit_update: null argument");
  if (n != (int)h->in.fit_params.size())
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_fit_update: one value per fit parameter expected");
  int i = 0;
  for (const auto& kv : h->in.fit_params) {  // in key order, as fit_param_keys() lists them
    std::string err;
    if (!hig::update_param(h->in, kv.second.variable, x[i++], err))
      return fail(HGX_ERR_INVALID_ARG, "hgx_hig_fit_update: " + err);
  }
  h->json.clear();
  return HGX_OK;
}

int hgx_hig_qgrid(hgx_ctx ctx, hgx_hig h, double dn2_re, double dn2_im, hgx_qgrid* out) {
  if (!ctx || !h || !out) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_qgrid: null argument");
  const hig::Compute& c = h->in.compute;
  // QGrid::create handles the q-space region only (src/model/qgrid.cpp:43-45, 94-96)
  if (c.region_type != "qspace")
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_qgrid: only a \"qspace\" output region is supported");
  double k0, alpha_i;
  HGX_TRY(hgx_hig_beam(h, &k0, &alpha_i, nullptr));
  return hgx_qgrid_create(ctx, c.resolution[0], c.resolution[1], c.minpoint[0], c.minpoint[1],
                          c.maxpoint[0], c.maxpoint[1], alpha_i, k0, dn2_re, dn2_im, out);
}

int hgx_hig_objective(hgx_ctx ctx, hgx_hig h, const double* x, int nx, const double* ref,
                      const unsigned* mask, int metric, double reg_alpha, double* dist, long* ndist) {
  if (!ctx || !h || !ref || !dist) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_objective: null argument");
  if (is_device_ptr(dist)) return fail(HGX_ERR_INVALID_ARG, "hgx_hig_objective: dist must be host memory");
  // HipGISAXSObjectiveFunction::operator() (src/analyzer/objective_func_hipgisaxs.cpp:263-320):
  // the parameters in key order, the simulation, the distance, the regularisation
  HGX_TRY(hgx_hig_fit_update(h, x, nx));
  int nrow = 0, ncol = 0;
  HGX_TRY(hgx_hig_image_size(h, &nrow, &ncol));
  const long n = (long)nrow * ncol;
  HGX_CUDA(cudaSetDevice(ctx->device));
  if (!ctx->hig) {
    ctx->hig = new (std::nothrow) HigWork;
    if (!ctx->hig) return fail(HGX_ERR_NO_MEMORY, "hgx_hig_objective: out of host memory");
  }
  DevBuf& img = ctx->hig->obj;
  HGX_TRY(img.reserve(sizeof(double) * n));
  HGX_TRY(hgx_hig_compute_gisaxs(ctx, h, HGX_F64, (double*)img.p));
  const bool residual = metric == 4 || metric == 5;  // the residual-vector measures
  HGX_TRY(hgx_fit_distance(ctx, metric, n, ref, (const double*)img.p, mask, dist));
  const long nd = residual ? n : 1;
  double pmean = 0.0;
  int i = 0;
  for (const auto& kv : h->in.fit_params) {
    const double mean = (kv.second.range[1] - kv.second.range[0]) / 2.0 + kv.second.range[0];
    double t = x[i++] - mean;
    t *= t;
    pmean += t;
  }
  const double reg = (reg_alpha / 2) * pmean;
  const double reg_dist = reg / nd;
  for (long k = 0; k < nd; ++k) dist[k] = isfinite(dist[k]) ? dist[k] + reg_dist : 1e8;
  if (ndist) *ndist = nd;
  return HGX_OK;
}

// The objective of hgx_hig_objective for a scalar distance measure and its gradient with
// respect to the fit parameters.  The reference's LMVM fitter takes this gradient by central
// differences, two simulations per parameter (src/analyzer/hipgisaxs_fit_lmvm.cpp:190-223, the
// objective dist[0], src/analyzer/objective_func.cpp:107-115).  Here: one simulation, then
// lambda = d(distance)/d(image) on the device, then per parameter the tangent of the image
// (hig_image_tangent) contracted with lambda, plus the regularisation's reg_alpha (x - mean).
int hgx_hig_objective_grad(hgx_ctx ctx, hgx_hig h, const double* x, int nx, const double* ref,
                           const unsigned* mask, int metric, double reg_alpha, double* dist, double* grad) {
  if (!ctx || !h || !x || !ref || !dist || !grad)
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_objective_grad: null argument");
  if (metric == 4 || metric == 5)
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_objective_grad: the gradient is defined for the scalar "
                                     "distance measures (not the residual vectors)");
  if (nx != (int)h->in.fit_params.size())
    return fail(HGX_ERR_INVALID_ARG, "hgx_hig_objective_grad: x must hold one value per fit parameter");
  long nd = 0;
  HGX_TRY(hgx_hig_objective(ctx, h, x, nx, ref, mask, metric, reg_alpha, dist, &nd));
  int nrow = 0, ncol = 0;
  HGX_TRY(hgx_hig_image_size(h, &nrow, &ncol));
  const long n = (long)nrow * ncol;
  HigWork& w = *ctx->hig;
  DevBuf bref, bmask;
  const void *dref = nullptr, *dmask = nullptr;
  HGX_TRY(stage_in(ctx, ref, sizeof(double) * n, bref, &dref));
  if (mask) HGX_TRY(stage_in(ctx, mask, sizeof(unsigned) * n, bmask, &dmask));
  HGX_TRY(w.lam.reserve(sizeof(double) * n));
  HGX_TRY(w.dimg.reserve(sizeof(double) * n));
  HGX_TRY(fit_distance_gradient(ctx, metric, n, (const double*)dref, (const double*)w.obj.p,
                                (const unsigned*)dmask, (double*)w.lam.p));
  const bool finite = dist[0] != 1e8;  // a non-finite distance is replaced by 1e8: no slope
  int i = 0;
  for (const auto& kv : h->in.fit_params) {
    const double mean = (kv.second.range[1] - kv.second.range[0]) / 2.0 + kv.second.range[0];
    const double step = 1e-6 * std::max(1.0, std::fabs(x[i]));
    double g = 0.0;
    if (finite) {
      HGX_CUDA(cudaMemsetAsync(w.dimg.p, 0, sizeof(double) * n, ctx->stream));
      HGX_TRY(hig_image_tangent(ctx, h, kv.second.variable, x[i], step, (double*)w.dimg.p));
      HGX_TRY(device_dot(ctx, n, (const double*)w.lam.p, (const double*)w.dimg.p, &g));
      g += reg_alpha * (x[i] - mean);
    }
    grad[i++] = g;
  }
  return hgx_synchronize(ctx);
}

}  // extern "C"


// C ABI of the HiG input reader (hig_input.cpp) and the device set-up that HipGISAXS::init
// derives from it (src/sim/hipgisaxs_main.cpp:106-216).
#include <math.h>
#include <string.h>

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

}  // extern "C"

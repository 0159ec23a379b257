// Fresnel (Parratt) coefficients of the DWBA: MultiLayer::init, parratt_recursion and
// propagation_coeffs (src/model/multilayer.cpp:29-58, 65-108, 110-155), FP64 — the
// coefficients are sensitive near the critical angle and cost one recursion per detector row.
//
// fc_k[i] = {Ti conj(Tf), Ti conj(Rf), Ri conj(Tf), Ri conj(Rf)}[row(i)], zero for rows with
// alpha_f <= 0 (the reference leaves Tf = Rf = 0 there, multilayer.cpp:138).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "cplx.cuh"
#include "hgx_internal.cuh"

namespace hgx {

constexpr int MAX_LAYERS = 32;

struct Stack {
  int nl, order;
  double om_re[MAX_LAYERS], om_im[MAX_LAYERS], z[MAX_LAYERS];
};

// MultiLayer::parratt_recursion: T and R at layer `order` for one angle.
__device__ void parratt(const Stack& S, double alpha, double k0, zd* T_out, zd* R_out) {
  zd T[MAX_LAYERS], R[MAX_LAYERS], kz[MAX_LAYERS];
  const int nl = S.nl;
  double sina = sin(alpha);
  for (int i = 0; i < nl; ++i) {
    T[i] = zd(0, 0);
    R[i] = zd(0, 0);
    kz[i] = csqrt_(sina * sina - zd(S.om_re[i], S.om_im[i])) * (-k0);
  }
  T[nl - 1] = zd(1.0, 0.0);
  for (int i = nl - 2; i > -1; --i) {
    zd pij = (kz[i] + kz[i + 1]) / (kz[i] * 2.0);
    zd mij = (kz[i] - kz[i + 1]) / (kz[i] * 2.0);
    double zi = S.z[i];
    zd exp_p = cexp_((zd(0.0, -1.0) * (kz[i + 1] + kz[i])) * zi);
    zd exp_m = cexp_((zd(0.0, -1.0) * (kz[i + 1] - kz[i])) * zi);
    zd a00 = pij * exp_m, a01 = mij * conj(exp_p), a10 = mij * exp_p, a11 = pij * conj(exp_m);
    T[i] = a00 * T[i + 1] + a01 * R[i + 1];
    R[i] = a10 * T[i + 1] + a11 * R[i + 1];
  }
  zd t0 = T[0];
  *T_out = T[S.order] / t0;
  *R_out = R[S.order] / t0;
}

// One thread per detector row: Tf, Rf (zero when alpha_f <= 0); thread 0 of block 0 also
// writes the incident coefficients into slot nrow.
__global__ void parratt_rows_kernel(Stack S, const double* __restrict__ alpha, int nrow,
                                    double alpha_i, double k0, double2* __restrict__ tr) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < nrow) {
    zd T(0, 0), R(0, 0);
    if (alpha[r] > 0) parratt(S, alpha[r], k0, &T, &R);
    tr[2 * r] = T.d2();
    tr[2 * r + 1] = R.d2();
  }
  if (r == 0) {
    zd T, R;
    parratt(S, alpha_i, k0, &T, &R);
    tr[2 * nrow] = T.d2();
    tr[2 * nrow + 1] = R.d2();
  }
}

// Per-row DWBA coefficients: rowfc[r*4 + k].
__global__ void row_fc_kernel(const double2* __restrict__ tr, int nrow, double2* __restrict__ rowfc) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrow) return;
  zd Ti(tr[2 * nrow]), Ri(tr[2 * nrow + 1]);
  zd Tf(tr[2 * r]), Rf(tr[2 * r + 1]);
  rowfc[4 * r + 0] = (Ti * conj(Tf)).d2();
  rowfc[4 * r + 1] = (Ti * conj(Rf)).d2();
  rowfc[4 * r + 2] = (Ri * conj(Tf)).d2();
  rowfc[4 * r + 3] = (Ri * conj(Rf)).d2();
}

// Expands per-row coefficients to the reference's per-pixel 4N layout.
__global__ void expand_fc_kernel(const double2* __restrict__ rowfc, int nrow, int ncol,
                                 double2* __restrict__ fc) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long n = (long)nrow * ncol;
  if (i >= n) return;
  long r = i / ncol;
#pragma unroll
  for (int k = 0; k < 4; ++k) fc[k * n + i] = rowfc[4 * r + k];
}

// MultiLayer::init: vacuum first, user layers by ascending order, substrate (order -1) last;
// z measured from the top, decreasing by each layer's thickness.
int build_stack(int nlayers, const double* delta, const double* beta, const double* thickness,
                const int* order, int particle_order, Stack& S) {
  if (nlayers < 0 || nlayers + 2 > MAX_LAYERS)
    return fail(HGX_ERR_INVALID_ARG, "propagation coefficients: at most 30 layers");
  if (particle_order == -1)
    return fail(HGX_ERR_INVALID_ARG, "propagation coefficients: shapes can't be buried inside "
                                     "the substrate (the reference refuses order -1)");
  std::vector<int> idx;
  int sub = -1;
  for (int i = 0; i < nlayers; ++i) {
    if (order[i] == -1) sub = i;
    else idx.push_back(i);
  }
  std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return order[x] < order[y]; });
  std::vector<double> th;
  S.nl = 0;
  S.om_re[0] = S.om_im[0] = 0.0;
  th.push_back(0.0);
  S.nl = 1;
  for (int i : idx) {
    S.om_re[S.nl] = 2 * delta[i];
    S.om_im[S.nl] = 2 * beta[i];
    th.push_back(thickness[i]);
    ++S.nl;
  }
  S.om_re[S.nl] = sub >= 0 ? 2 * delta[sub] : 0.0;
  S.om_im[S.nl] = sub >= 0 ? 2 * beta[sub] : 0.0;
  th.push_back(sub >= 0 ? thickness[sub] : 0.0);
  ++S.nl;
  double z = 0;
  S.z[0] = 0;
  for (int i = 1; i < S.nl; ++i) {
    z -= th[i];
    S.z[i] = z;
  }
  if (particle_order < 0 || particle_order >= S.nl)
    return fail(HGX_ERR_INVALID_ARG, "propagation coefficients: particle layer out of range");
  S.order = particle_order;
  return HGX_OK;
}

// Per-row coefficients (nrow x 4 complex128) into `rowfc` (device).
int row_fc_device(hgx_ctx c, const Stack& S, const double* alpha_dev, int nrow, double k0,
                  double alpha_i, double2* rowfc) {
  DevBuf tr;
  HGX_TRY(tr.reserve(sizeof(double2) * 2 * (size_t)(nrow + 1)));
  parratt_rows_kernel<<<(nrow + 63) / 64, 64, 0, c->stream>>>(S, alpha_dev, nrow, alpha_i, k0,
                                                              reinterpret_cast<double2*>(tr.p));
  row_fc_kernel<<<(nrow + 127) / 128, 128, 0, c->stream>>>(reinterpret_cast<double2*>(tr.p), nrow,
                                                           rowfc);
  HGX_CUDA(cudaGetLastError());
  HGX_CUDA(cudaStreamSynchronize(c->stream));  // `tr` is released on return
  return HGX_OK;
}

}  // namespace hgx

using namespace hgx;

extern "C" {

int hgx_propagation_coeffs(hgx_ctx c, hgx_qgrid g, int nlayers, const double* delta,
                           const double* beta, const double* thickness, const int* order,
                           double k0, double alpha_i, int particle_order, const double* alpha,
                           double* fc, int per_row) {
  if (!c || !g || !fc || (nlayers > 0 && (!delta || !beta || !thickness || !order)))
    return fail(HGX_ERR_INVALID_ARG, "hgx_propagation_coeffs: null argument");
  if (g->nrow < 1 || g->ncol < 1)
    return fail(HGX_ERR_INVALID_ARG, "hgx_propagation_coeffs: the grid has no detector rows");
  Stack S;
  HGX_TRY(build_stack(nlayers, delta, beta, thickness, order, particle_order, S));
  HGX_CUDA(cudaSetDevice(c->device));
  const double* al = alpha ? alpha : g->alpha;
  if (!al)
    return fail(HGX_ERR_INVALID_ARG, "hgx_propagation_coeffs: exit angles needed (grid from arrays)");
  DevBuf abuf, rowbuf, outbuf;
  const void* al_dev = nullptr;
  HGX_TRY(stage_in(c, al, sizeof(double) * g->nrow, abuf, &al_dev));
  const long n = (long)g->nrow * g->ncol;
  const size_t out_bytes = sizeof(double2) * (per_row ? 4 * (size_t)g->nrow : 4 * (size_t)n);
  void* dout = nullptr;
  HGX_TRY(stage_out(c, fc, out_bytes, outbuf, &dout));
  double2* rowfc = reinterpret_cast<double2*>(dout);
  if (!per_row) {
    HGX_TRY(rowbuf.reserve(sizeof(double2) * 4 * (size_t)g->nrow));
    rowfc = reinterpret_cast<double2*>(rowbuf.p);
  }
  HGX_TRY(row_fc_device(c, S, reinterpret_cast<const double*>(al_dev), g->nrow, k0, alpha_i, rowfc));
  if (!per_row) {
    expand_fc_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(rowfc, g->nrow, g->ncol,
                                                                        reinterpret_cast<double2*>(dout));
    HGX_CUDA(cudaGetLastError());
  }
  HGX_TRY(finish_out(c, fc, out_bytes, dout));
  return hgx_synchronize(c);
}

}  // extern "C"

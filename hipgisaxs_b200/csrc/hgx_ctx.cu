// Context, errors, device buffers and q-grid objects of the hgx C ABI.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <cmath>
#include <string>
#include <vector>

#include "hgx_internal.cuh"

namespace hgx {

static thread_local std::string g_last_error;

int fail(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}

int cuda_fail(cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();  // clear a non-sticky error so the context stays usable
  return fail(e == cudaErrorMemoryAllocation ? HGX_ERR_NO_MEMORY : HGX_ERR_CUDA, m);
}

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

void* mapped_host_ptr(const void* p) {
  if (!p) return nullptr;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}

int DevBuf::reserve(size_t n) {
  if (n <= bytes) return HGX_OK;
  release();
  size_t want = n < 4096 ? 4096 : n;
  cudaError_t e = cudaMalloc(&p, want);
  if (e != cudaSuccess) {
    p = nullptr;
    bytes = 0;
    return cuda_fail(e, "cudaMalloc(scratch)");
  }
  bytes = want;
  return HGX_OK;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

// ------------------------------------------------------------- row table ----
// For q-grids laid out by detector rows: records each row's qz per block and checks that
// qz is constant along every row and, for 4 blocks, that the blocks pair as the DWBA
// construction makes them (block 3 = -block 0, block 1 = -block 2, all real).
__global__ void row_table_kernel(const double2* __restrict__ qz, int nqy, int nk, int ncol,
                                 double2* __restrict__ rowqz, unsigned* __restrict__ flags) {
  long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nqy) return;
  int row = (int)(p / ncol);
  long first = (long)row * ncol;
  bool row_ok = true, paired = (nk == 4);
  for (int k = 0; k < nk; ++k) {
    double2 v = qz[(long)k * nqy + p];
    double2 f = qz[(long)k * nqy + first];
    if (v.x != f.x || v.y != f.y) row_ok = false;
    if (rowqz && p == first) rowqz[(long)row * nk + k] = v;
    if (v.y != 0.0) paired = false;
  }
  if (nk == 4) {
    double2 a = qz[p], b = qz[(long)nqy + p], c = qz[2L * nqy + p], d = qz[3L * nqy + p];
    if (d.x != -a.x || b.x != -c.x) paired = false;
  }
  if (!row_ok) atomicOr(flags, 1u);
  if (!paired) atomicOr(flags, 2u);
}

int stage_in(hgx_ctx c, const void* p, size_t bytes, DevBuf& buf, const void** dev) {
  if (!p) {
    *dev = nullptr;
    return HGX_OK;
  }
  if (is_device_ptr(p)) {
    *dev = p;
    return HGX_OK;
  }
  HGX_TRY(buf.reserve(bytes));
  HGX_CUDA(cudaMemcpyAsync(buf.p, p, bytes, cudaMemcpyHostToDevice, c->stream));
  *dev = buf.p;
  return HGX_OK;
}

int stage_out(hgx_ctx c, void* p, size_t bytes, DevBuf& buf, void** dev) {
  (void)c;
  if (is_device_ptr(p)) {
    *dev = p;
    return HGX_OK;
  }
  HGX_TRY(buf.reserve(bytes));
  *dev = buf.p;
  return HGX_OK;
}

int finish_out(hgx_ctx c, void* p, size_t bytes, const void* dev) {
  if (p == dev) return HGX_OK;
  HGX_CUDA(cudaMemcpyAsync(p, dev, bytes, cudaMemcpyDeviceToHost, c->stream));
  return hgx_synchronize(c);
}

// Detector row length of a grid given as arrays: where qz of block 0 first changes (the QGrid
// layout keeps qz constant along a row); 0 when that cannot be read.
static int detect_ncol(hgx_qgrid g, const double* qz, int* ncol) {
  *ncol = 0;
  if (g->nk < 1) return HGX_OK;
  std::vector<double> h;
  const double* src = qz;
  if (is_device_ptr(qz)) {
    h.resize(2 * (size_t)g->nqy);
    cudaError_t e = cudaMemcpyAsync(h.data(), qz, sizeof(double2) * g->nqy, cudaMemcpyDeviceToHost,
                                    g->ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "q-grid: read qz");
    src = h.data();
  }
  int n = 1;
  while (n < g->nqy && src[2 * n] == src[0] && src[2 * n + 1] == src[1]) ++n;
  *ncol = n;
  return HGX_OK;
}

int shaped_grid(hgx_ctx c, int nqy, const double* qx, const double* qy, int nqz, const double* qz,
                hgx_qgrid* out) {
  hgx_qgrid g = c->shaped;
  if (g && g->nqy == nqy && g->nqz == nqz) {
    cudaStream_t st = c->stream;
    auto kind = [](const void* p) { return is_device_ptr(p) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice; };
    cudaError_t e = cudaMemcpyAsync(g->qx, qx, sizeof(double) * nqy, kind(qx), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(g->qy, qy, sizeof(double) * nqy, kind(qy), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(g->qz, qz, sizeof(double2) * nqz, kind(qz), st);
    int s = e == cudaSuccess ? HGX_OK : cuda_fail(e, "q-grid refill: copy");
    int ncol = 0;
    if (s == HGX_OK) s = detect_ncol(g, qz, &ncol);
    if (s == HGX_OK) {
      g->ncol = ncol;
      s = qgrid_finalize(g);
    }
    if (s == HGX_OK) {
      *out = g;
      return HGX_OK;
    }
    hgx_qgrid_destroy(g);  // leave no half-refilled grid behind
    c->shaped = nullptr;
    return s;
  }
  if (g) {
    hgx_qgrid_destroy(g);
    c->shaped = nullptr;
  }
  HGX_TRY(hgx_qgrid_from_arrays(c, nqy, qx, qy, nqz, qz, 0, &g));
  c->shaped = g;
  *out = g;
  return HGX_OK;
}

int shaped_rows_begin(hgx_ctx c, int nqy, const double* qx, const double* qy, int nqz, const double* qz,
                      hgx_qgrid* out, bool* rows_first) {
  *rows_first = false;
  hgx_qgrid g = c->shaped;
  if (!g || g->nqy != nqy || g->nqz != nqz || (g->nk != 1 && g->nk != 4) || is_device_ptr(qz))
    return shaped_grid(c, nqy, qx, qy, nqz, qz, out);
  int ncol = 0;
  HGX_TRY(detect_ncol(g, qz, &ncol));  // host array: scans the first row only
  // detector rows of at least 64 q-points (shorter runs of equal qz, as on scattered q-points,
  // take the full path: a row kernel there would be mostly idle lanes)
  if (ncol < 64 || nqy % ncol != 0) return shaped_grid(c, nqy, qx, qy, nqz, qz, out);
  const int nk = g->nk, nrow = nqy / ncol;
  // each row's first q-point of every block, and whether the blocks pair (real, qz4 = -qz1,
  // qz2 = -qz3) there; the check on the side stream holds every q-point to the same values
  std::vector<double2> rt((size_t)nrow * nk);
  bool paired = nk == 4;
  for (int r = 0; r < nrow; ++r) {
    for (int k = 0; k < nk; ++k) {
      const double* v = qz + 2 * ((size_t)k * nqy + (size_t)r * ncol);
      rt[(size_t)r * nk + k] = make_double2(v[0], v[1]);
      if (v[1] != 0.0) paired = false;
    }
    if (nk == 4) {
      const double2* t = &rt[(size_t)r * 4];
      if (t[3].x != -t[0].x || t[1].x != -t[2].x) paired = false;
    }
  }
  if (!c->side) {  // made once per context, kept only when all three exist
    cudaStream_t sst = nullptr;
    cudaEvent_t sev = nullptr;
    void* sfl = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&sst, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&sfl, 256);
    if (e != cudaSuccess) {
      if (sfl) cudaFree(sfl);
      if (sev) cudaEventDestroy(sev);
      if (sst) cudaStreamDestroy(sst);
      return cuda_fail(e, "side stream of the reference-shaped call");
    }
    c->side = sst;
    c->side_ev = sev;
    c->side_flags = static_cast<unsigned*>(sfl);
  }
  const size_t need = (size_t)nrow * nk;
  if (need > g->rowqz_cap) {
    HGX_CUDA(cudaStreamSynchronize(c->stream));  // earlier kernels may still read the old table
    if (g->rowqz) cudaFree(g->rowqz);
    g->rowqz = nullptr;
    g->rowqz_cap = 0;
    HGX_CUDA(cudaMalloc(&g->rowqz, sizeof(double2) * need));
    g->rowqz_cap = need;
  }
  cudaStream_t st = c->stream;
  auto kind = [](const void* p) { return is_device_ptr(p) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice; };
  HGX_CUDA(cudaMemcpyAsync(g->qx, qx, sizeof(double) * nqy, kind(qx), st));
  HGX_CUDA(cudaMemcpyAsync(g->qy, qy, sizeof(double) * nqy, kind(qy), st));
  HGX_CUDA(cudaMemcpyAsync(g->rowqz, rt.data(), sizeof(double2) * need, cudaMemcpyHostToDevice, st));
  // the side stream's copy of qz may start once everything queued so far has run (earlier
  // kernels that read the grid's qz)
  HGX_CUDA(cudaEventRecord(c->side_ev, st));
  g->ncol = ncol;
  g->nrow = nrow;
  g->mode = paired ? 1 : 2;
  *out = g;
  *rows_first = true;
  return HGX_OK;
}

int shaped_rows_check(hgx_ctx c, hgx_qgrid g, const double* qz) {
  HGX_CUDA(cudaStreamWaitEvent(c->side, c->side_ev, 0));
  HGX_CUDA(cudaMemsetAsync(c->side_flags, 0, sizeof(unsigned), c->side));
  HGX_CUDA(cudaMemcpyAsync(g->qz, qz, sizeof(double2) * g->nqz, cudaMemcpyHostToDevice, c->side));
  const int blocks = (g->nqy + 255) / 256;
  row_table_kernel<<<blocks, 256, 0, c->side>>>(g->qz, g->nqy, g->nk, g->ncol, nullptr, c->side_flags);
  HGX_CUDA(cudaGetLastError());
  return HGX_OK;
}

int shaped_rows_settle(hgx_ctx c, hgx_qgrid g, bool* ok) {
  unsigned flags = 0;
  HGX_CUDA(cudaMemcpyAsync(&flags, c->side_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, c->side));
  HGX_CUDA(cudaStreamSynchronize(c->side));
  const int mode = (flags & 1u) ? 0 : ((g->nk == 4 && !(flags & 2u)) ? 1 : 2);
  *ok = mode == g->mode;
  if (!*ok) HGX_TRY(qgrid_finalize(g));  // the full qz is on the device: table and mode from it
  return HGX_OK;
}

int qgrid_finalize(hgx_qgrid g) {
  g->mode = 0;
  if (g->nk != 1 && g->nk != 4) return HGX_OK;
  if (g->ncol <= 0 || g->nqy % g->ncol != 0) return HGX_OK;
  g->nrow = g->nqy / g->ncol;
  const size_t need = (size_t)g->nrow * g->nk;
  if (need > g->rowqz_cap) {
    if (g->rowqz) cudaFree(g->rowqz);
    g->rowqz = nullptr;
    g->rowqz_cap = 0;
    HGX_CUDA(cudaMalloc(&g->rowqz, sizeof(double2) * need));
    g->rowqz_cap = need;
  }
  HGX_TRY(g->ctx->scratch.reserve(256));
  unsigned* d_flags = reinterpret_cast<unsigned*>(g->ctx->scratch.p);
  cudaStream_t st = g->ctx->stream;
  HGX_CUDA(cudaMemsetAsync(d_flags, 0, sizeof(unsigned), st));
  int threads = 256;
  int blocks = (g->nqy + threads - 1) / threads;
  row_table_kernel<<<blocks, threads, 0, st>>>(g->qz, g->nqy, g->nk, g->ncol, g->rowqz, d_flags);
  HGX_CUDA(cudaGetLastError());
  unsigned flags = 0;
  HGX_CUDA(cudaMemcpyAsync(&flags, d_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  HGX_CUDA(cudaStreamSynchronize(st));
  if (flags & 1u) {  // not row-constant: the per-q-point kernels handle it (row table unused)
    g->nrow = 0;
    g->mode = 0;
    return HGX_OK;
  }
  g->mode = (g->nk == 4 && !(flags & 2u)) ? 1 : 2;
  return HGX_OK;
}

}  // namespace hgx

using namespace hgx;

extern "C" {

const char* hgx_last_error(void) { return g_last_error.c_str(); }

const char* hgx_status_string(int s) {
  switch (s) {
    case HGX_OK: return "ok";
    case HGX_ERR_INVALID_ARG: return "invalid argument";
    case HGX_ERR_CUDA: return "CUDA error";
    case HGX_ERR_NO_MEMORY: return "out of memory";
    case HGX_ERR_DEVICE: return "device-side error";
    case HGX_ERR_NOT_FINITE: return "non-finite result";
    default: return "unknown status";
  }
}

int hgx_version(void) { return 10000; }

int hgx_create(int device, hgx_ctx* out) {
  if (!out) return fail(HGX_ERR_INVALID_ARG, "hgx_create: out is NULL");
  *out = nullptr;
  int dev = device;
  if (dev < 0) HGX_CUDA(cudaGetDevice(&dev));
  int ndev = 0;
  HGX_CUDA(cudaGetDeviceCount(&ndev));
  if (dev >= ndev) return fail(HGX_ERR_INVALID_ARG, "hgx_create: no such device");
  HGX_CUDA(cudaSetDevice(dev));
  hgx_ctx c = new (std::nothrow) hgx_ctx_s();
  if (!c) return fail(HGX_ERR_NO_MEMORY, "hgx_create: host allocation");
  c->device = dev;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
    c->sm_count = prop.multiProcessorCount;
    c->max_smem_optin = (int)prop.sharedMemPerBlockOptin;
  }
  cudaError_t e = cudaMalloc(&c->d_err, sizeof(unsigned));
  if (e != cudaSuccess) {
    delete c;
    return cuda_fail(e, "cudaMalloc(error word)");
  }
  cudaMemset(c->d_err, 0, sizeof(unsigned));
  *out = c;
  return HGX_OK;
}

int hgx_destroy(hgx_ctx c) {
  if (!c) return HGX_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  if (c->d_err) cudaFree(c->d_err);
  if (c->side) cudaStreamSynchronize(c->side);
  if (c->shaped) hgx_qgrid_destroy(c->shaped);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->side_ev) cudaEventDestroy(c->side_ev);
  if (c->side_flags) cudaFree(c->side_flags);
  delete c->mesh;
  if (c->hig && c->hig->grid) hgx_qgrid_destroy(c->hig->grid);
  delete c->hig;
  c->scratch.release();
  c->staging.release();
  c->shaped_out.release();
  delete c;
  return HGX_OK;
}

int hgx_set_stream(hgx_ctx c, void* stream) {
  if (!c) return fail(HGX_ERR_INVALID_ARG, "hgx_set_stream: ctx is NULL");
  cudaStream_t next = reinterpret_cast<cudaStream_t>(stream);
  if (next != c->stream) {
    // the context's buffers are reused in stream order: work still queued on the old stream
    // finishes before work on the new one can touch them (a stream being captured into a graph
    // has run nothing yet and is left alone: a synchronisation would end its capture)
    HGX_CUDA(cudaSetDevice(c->device));
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(c->stream, &cs) != cudaSuccess)
      cudaGetLastError();  // the legacy stream while another stream is captured: left alone too
    else if (cs == cudaStreamCaptureStatusNone)
      HGX_CUDA(cudaStreamSynchronize(c->stream));
  }
  c->stream = next;
  return HGX_OK;
}

void* hgx_get_stream(hgx_ctx c) { return c ? reinterpret_cast<void*>(c->stream) : nullptr; }

int hgx_synchronize(hgx_ctx c) {
  if (!c) return fail(HGX_ERR_INVALID_ARG, "hgx_synchronize: ctx is NULL");
  HGX_CUDA(cudaSetDevice(c->device));
  HGX_CUDA(cudaStreamSynchronize(c->stream));
  unsigned err = 0;
  HGX_CUDA(cudaMemcpy(&err, c->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (err) {
    cudaMemset(c->d_err, 0, sizeof(unsigned));
    char buf[160];
    snprintf(buf, sizeof buf, "device error bits 0x%x (1=wait timeout, 2=row mismatch, "
             "4=bad index, 8=queue timeout)", err);
    return fail(HGX_ERR_DEVICE, buf);
  }
  return HGX_OK;
}

int hgx_qgrid_from_arrays(hgx_ctx c, int nqy, const double* qx, const double* qy, int nqz,
                          const double* qz, int ncol, hgx_qgrid* out) {
  if (!c || !out || !qx || !qy || !qz) return fail(HGX_ERR_INVALID_ARG, "hgx_qgrid_from_arrays: null argument");
  *out = nullptr;
  if (nqy < 1 || nqz < 1) return fail(HGX_ERR_INVALID_ARG, "hgx_qgrid_from_arrays: empty grid");
  if (ncol < 0) return fail(HGX_ERR_INVALID_ARG, "hgx_qgrid_from_arrays: ncol < 0");
  HGX_CUDA(cudaSetDevice(c->device));
  hgx_qgrid g = new (std::nothrow) hgx_qgrid_s();
  if (!g) return fail(HGX_ERR_NO_MEMORY, "hgx_qgrid_from_arrays: host allocation");
  g->ctx = c;
  g->nqy = nqy;
  g->nqz = nqz;
  g->nk = (nqz % nqy == 0) ? nqz / nqy : 0;
  cudaStream_t st = c->stream;
  auto cleanup = [&](int s) {
    hgx_qgrid_destroy(g);
    return s;
  };
  if (cudaMalloc(&g->qx, sizeof(double) * nqy) != cudaSuccess ||
      cudaMalloc(&g->qy, sizeof(double) * nqy) != cudaSuccess ||
      cudaMalloc(&g->qz, sizeof(double2) * nqz) != cudaSuccess)
    return cleanup(cuda_fail(cudaErrorMemoryAllocation, "hgx_qgrid_from_arrays: cudaMalloc"));
  auto kind = [](const void* p) { return is_device_ptr(p) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice; };
  cudaError_t e = cudaMemcpyAsync(g->qx, qx, sizeof(double) * nqy, kind(qx), st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(g->qy, qy, sizeof(double) * nqy, kind(qy), st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(g->qz, qz, sizeof(double2) * nqz, kind(qz), st);
  if (e != cudaSuccess) return cleanup(cuda_fail(e, "hgx_qgrid_from_arrays: copy"));
  // detector row length: given, or found where qz of block 0 first changes
  if (ncol == 0 && g->nk >= 1) {
    int s0 = detect_ncol(g, qz, &ncol);
    if (s0 != HGX_OK) return cleanup(s0);
  }
  g->ncol = ncol;
  int s = qgrid_finalize(g);
  if (s != HGX_OK) return cleanup(s);
  *out = g;
  return HGX_OK;
}

int hgx_qgrid_info(hgx_qgrid g, int* nqy, int* nqz, int* nrow, int* ncol, int* mode) {
  if (!g) return fail(HGX_ERR_INVALID_ARG, "hgx_qgrid_info: grid is NULL");
  if (nqy) *nqy = g->nqy;
  if (nqz) *nqz = g->nqz;
  if (nrow) *nrow = g->nrow;
  if (ncol) *ncol = g->ncol;
  if (mode) *mode = g->mode;
  return HGX_OK;
}

int hgx_qgrid_read(hgx_ctx c, hgx_qgrid g, double* qx, double* qy, double* qz, double* alpha,
                   double* qz_ext) {
  if (!c || !g) return fail(HGX_ERR_INVALID_ARG, "hgx_qgrid_read: null argument");
  HGX_CUDA(cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  auto kind = [](const void* p) { return is_device_ptr(p) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost; };
  if (qx) HGX_CUDA(cudaMemcpyAsync(qx, g->qx, sizeof(double) * g->nqy, kind(qx), st));
  if (qy) HGX_CUDA(cudaMemcpyAsync(qy, g->qy, sizeof(double) * g->nqy, kind(qy), st));
  if (qz) {
    if (!g->qz_det) return fail(HGX_ERR_INVALID_ARG, "hgx_qgrid_read: grid has no detector qz");
    HGX_CUDA(cudaMemcpyAsync(qz, g->qz_det, sizeof(double) * g->nqy, kind(qz), st));
  }
  if (alpha) {
    if (!g->alpha) return fail(HGX_ERR_INVALID_ARG, "hgx_qgrid_read: grid has no exit angles");
    HGX_CUDA(cudaMemcpyAsync(alpha, g->alpha, sizeof(double) * g->nrow, kind(alpha), st));
  }
  if (qz_ext) HGX_CUDA(cudaMemcpyAsync(qz_ext, g->qz, sizeof(double2) * g->nqz, kind(qz_ext), st));
  HGX_CUDA(cudaStreamSynchronize(st));
  return HGX_OK;
}

int hgx_qgrid_destroy(hgx_qgrid g) {
  if (!g) return HGX_OK;
  if (g->ctx) cudaSetDevice(g->ctx->device);
  if (g->ctx) cudaStreamSynchronize(g->ctx->stream);
  cudaFree(g->qx);
  cudaFree(g->qy);
  cudaFree(g->qz);
  cudaFree(g->rowqz);
  cudaFree(g->qz_det);
  cudaFree(g->alpha);
  delete g;
  return HGX_OK;
}

}  // extern "C"

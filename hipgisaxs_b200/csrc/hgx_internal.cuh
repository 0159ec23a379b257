// Internal declarations shared by the hgx CUDA sources (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "hgx.h"

namespace hgx {

// ------------------------------------------------------------------ errors ----
// Records a message for hgx_last_error() and returns the status.
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
#define HGX_CUDA(call)                                        \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return ::hgx::cuda_fail(e_, #call); \
  } while (0)
#define HGX_TRY(call)          \
  do {                         \
    int s_ = (call);           \
    if (s_ != HGX_OK) return s_; \
  } while (0)

// Error bits a kernel may set in the context's device error word.
enum DeviceError : unsigned {
  DEV_ERR_WAIT_TIMEOUT = 1u << 0,   // a bounded mbarrier wait gave up
  DEV_ERR_ROW_MISMATCH = 1u << 1,   // qz not constant along a row the caller declared
  DEV_ERR_BAD_INDEX = 1u << 2,      // an index outside its array (mesh faces, ROIs)
  DEV_ERR_QUEUE_TIMEOUT = 1u << 3,  // the persistent work queue gave up
};

// ------------------------------------------------------------- memory kind ----
// True when p is device (or managed) memory usable by the current device.
bool is_device_ptr(const void* p);
// The device address of page-locked host memory mapped into the device's address space
// (cudaMallocHost / cudaHostAlloc / cudaHostRegister under unified addressing), else nullptr.
void* mapped_host_ptr(const void* p);

// A device buffer owned by an object.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int reserve(size_t n);  // grows (never shrinks); contents are not preserved
  void release();
  ~DevBuf() { release(); }
};

}  // namespace hgx

namespace hgx {
// Device buffers of hgx_mesh_chi2_grad, kept by the context between calls (grow-only): large
// cudaMalloc/cudaFree pairs per call cost tens to hundreds of milliseconds.
struct MeshWork {
  DevBuf bv, bf, bfc, bc, bm, sd, F, seeds, part, gtri, vptr, vfac, gvb, Ib, bwpart;
};
// Triangles per tile of the FP32C triangle kernels (ff_tri.cu) and of the mesh adjoint's
// backward pass, which reads the forward's tiles.
constexpr int TRI_TILE = 512;
// The FP32 triangle tiles that the last FP32C form-factor call of a context left in its
// scratch (ff_tri.cu), read by the mesh adjoint: TRI_TILE triangles per tile, per-tile anchors
// (FP64 tile centre: in-plane in turns, z in nm; largest in-plane offset from it, nm) and the
// caller's index of the triangle in each tile slot (-1 for padding).
struct TileView {
  const float* tiles = nullptr;
  const double4* anchors = nullptr;
  const int* perm = nullptr;
  int ntiles = 0, ntri = 0;
};
// A custom shape's triangle tuples on the device, with the file's identity when it was read.
struct MeshTuples {
  DevBuf tri;  // ntri x 8 doubles (read_shapes_file layout)
  int ntri = 0;
  long long size = -1, mtime_ns = -1;
};
// Work of hgx_hig_compute_gisaxs, kept by the context between calls: the last description's
// q-grid (rebuilt when its region, beam or resolution changes), the custom shapes' triangle
// tuples (re-read only when the file's size or modification time changes) and grow-only
// buffers.
struct HigWork {
  hgx_qgrid grid = nullptr;
  double key[8] = {0};
  double ext_alpha = 0.0;  // the incidence angle the grid's qz blocks were extended for
  long grid_gen = 0;       // counts the grids made, so that cached results can name theirs
  std::vector<double> fc_key;  // what the Fresnel coefficients in fc were made for
  // pinned staging of the host tables of one simulation: two arenas used in turn, each
  // bump-allocated from its start, so that the host can fill one while the stream still copies
  // from the other (a simulation with a device image returns before its copies run); an arena
  // is refilled only after the event recorded at the end of its last simulation has completed
  unsigned char* h_arena[2] = {nullptr, nullptr};
  size_t arena_cap[2] = {0, 0};
  cudaEvent_t arena_ev[2] = {nullptr, nullptr};
  int arena_cur = 0;
  size_t arena_off = 0;  // nonzero between a simulation's first copy and its end
  DevBuf fc, ff, eff, sf, I, img, shapes, elems, gt, er, sc, obj, saxs_qz, ratios;
  DevBuf ftab;  // the fused grain kernel's tables of one structure, as one block
  // the objective's gradient: the tables' changes, d(distance)/d(image), d(image)/dx
  DevBuf tshapes, telems, tgt, ter, tsc, lam, dimg;
  std::map<std::string, MeshTuples> meshes;  // by resolved path
  ~HigWork() {
    for (int k = 0; k < 2; ++k) {
      if (arena_ev[k]) cudaEventSynchronize(arena_ev[k]);
      if (h_arena[k]) cudaFreeHost(h_arena[k]);
      if (arena_ev[k]) cudaEventDestroy(arena_ev[k]);
    }
  }
};
// d(image)/dx of hgx_hig_compute_gisaxs for one fit variable, added into dI (hig_sim.cu).
int hig_image_tangent(hgx_ctx c, hgx_hig h, const std::string& var, double x0, double step, double* dI);
// d(distance)/d(data) of a scalar fitting distance (fit_distance.cu), and a deterministic dot
// product of two device vectors (FP64, result on the host).
int fit_distance_gradient(hgx_ctx c, int metric, long n, const double* ref, const double* data,
                          const unsigned* mask, double* lambda);
int device_dot(hgx_ctx c, long n, const double* a, const double* b, double* out);
// The scalar fitting distance of npop images (imgs: npop x n, device) against one reference,
// enqueued on st without a host round trip: dist (device, npop) holds each candidate's value
// as hgx_fit_distance computes it for one image (the same sums in the same order).  scratch:
// fit_population_scratch(npop) doubles.
long fit_population_scratch(int npop);
int fit_distance_population(cudaStream_t st, int metric, long n, const double* ref, const double* imgs,
                            const unsigned* mask, int npop, double* scratch, double* dist);
}  // namespace hgx

// -------------------------------------------------------------- the context ----
struct hgx_ctx_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  unsigned* d_err = nullptr;  // device error word (DeviceError bits)
  hgx::DevBuf scratch;        // per-call scratch, grown on demand
  hgx::TileView tiles;        // triangle tiles of the last FP32C form factor (in scratch)
  hgx::DevBuf staging;        // device copies of host inputs
  int sm_count = 148;
  int max_smem_optin = 227 * 1024;
  // the q-grid and device output of the reference-shaped calls (explicit host arrays in,
  // host array out), kept between calls and refilled in place while the sizes stay the same,
  // so that those calls allocate and free no device memory
  hgx_qgrid_s* shaped = nullptr;
  hgx::DevBuf shaped_out;
  // the reference-shaped FP32C call's side stream: it copies the 4N qz values to the kept grid
  // and checks them while the row kernel already runs from a row table read on the host
  cudaStream_t side = nullptr;
  cudaEvent_t side_ev = nullptr;    // recorded on the context's stream, waited for by the side
  unsigned* side_flags = nullptr;   // device word: the check's flags (row_table_kernel bits)
  hgx::MeshWork* mesh = nullptr;  // work buffers of the mesh chi^2 and gradient
  hgx::HigWork* hig = nullptr;    // work of the HiG-driven simulation
};

// -------------------------------------------------------------- the q-grid ----
struct hgx_qgrid_s {
  hgx_ctx ctx = nullptr;
  int nqy = 0, nqz = 0, nrow = 0, ncol = 0, nk = 0;  // nk = nqz / nqy when integral
  int mode = 0;                  // 0 per-q-point, 1 rows paired-real, 2 rows complex
  double* qx = nullptr;          // nqy
  double* qy = nullptr;          // nqy
  double2* qz = nullptr;         // nqz
  double2* rowqz = nullptr;      // nrow x nk: the row-constant qz of each block (modes 1, 2)
  double* qz_det = nullptr;      // nqy: detector qz (grids made by hgx_qgrid_create)
  double* alpha = nullptr;       // nrow exit angles (grids made by hgx_qgrid_create)
  size_t rowqz_cap = 0;          // allocated entries of rowqz
  int tuned_p = 0;               // FP32 row-kernel launch shape chosen by hgx_ff_tune (0: none)
};

namespace hgx {
// Prepares triangle tiles for the FP32 kernels (see ff_tri.cu).
int qgrid_finalize(hgx_qgrid g);  // builds the row table and picks the mode
// Recomputes the DWBA qz blocks of a grid made by hgx_qgrid_create for another incidence
// angle (the detector qx, qy, qz and exit angles stay), then the row table (qgrid.cu).
int qgrid_reextend(hgx_qgrid g, double alpha_i, double k0, double dn2_re, double dn2_im);
// The context's grid for reference-shaped calls with these arrays: the kept one refilled in
// place when nqy and nqz match, else a new one (the old one destroyed).
int shaped_grid(hgx_ctx c, int nqy, const double* qx, const double* qy, int nqz, const double* qz,
                hgx_qgrid* out);
// The same grid for the reference-shaped FP32C form factor with qz in host memory, the 4N qz
// values left for later: when the kept grid has these sizes and the host qz array has a
// detector-row layout, qx and qy are copied on the context's stream and the row table is read
// from each row's first q-point of the host array (as row_table_kernel takes it), with the mode
// guessed from those values; *rows_first is then true and the caller enqueues its row kernels,
// calls shaped_rows_check(qz) and then shaped_rows_settle.  Otherwise *rows_first is false and
// the grid is the one shaped_grid makes.
int shaped_rows_begin(hgx_ctx c, int nqy, const double* qx, const double* qy, int nqz, const double* qz,
                      hgx_qgrid* out, bool* rows_first);
// Copies the host qz into the grid on the side stream, after the work already queued on the
// context's stream, and checks there that it is constant along rows with the guessed pairing.
int shaped_rows_check(hgx_ctx c, hgx_qgrid g, const double* qz);
// Waits for that check.  *ok = false when the guess did not hold: the grid has then been
// finalized from its full qz (row table, mode) and the caller runs its kernels again.
int shaped_rows_settle(hgx_ctx c, hgx_qgrid g, bool* ok);
// Lattice vectors a, b, c (abc9) and basis offset t3 of a lattice type (LatticeType code) and
// hkl string; false when the type has no vectors for that hkl (sf.cu).
bool lattice_table(int type, const std::string& hkl, double* abc9, double* t3);
}  // namespace hgx

namespace hgx {
// Device view of a caller array: the array itself when it is device memory, else a copy in
// `buf` (host -> device on the context's stream).
int stage_in(hgx_ctx c, const void* p, size_t bytes, DevBuf& buf, const void** dev);
// Device buffer for an output: the array itself when device memory, else `buf`; after the
// kernels, finish_out copies back and synchronises when the output is host memory.
int stage_out(hgx_ctx c, void* p, size_t bytes, DevBuf& buf, void** dev);
int finish_out(hgx_ctx c, void* p, size_t bytes, const void* dev);
}  // namespace hgx

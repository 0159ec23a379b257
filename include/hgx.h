/*
 * hgx — B200-native GISAXS forward model: the C ABI.
 *
 * Plain C: pointers, sizes and status codes; no C++ or torch types.  Every entry point
 * returns an hgx_status; on failure hgx_last_error() gives a message for the calling
 * thread.  Nothing here calls exit().
 *
 * Memory: unless stated otherwise, an array argument may live in host memory or in device
 * memory of the context's GPU (the library asks the CUDA driver which).  A call whose
 * output is host memory is synchronous.  A call whose inputs and outputs are all device
 * memory is asynchronous on the context's stream.
 *
 * Layouts follow the reference simulator (tacaswell/hipgisaxs): a detector of nrow x ncol
 * pixels is flattened row-major into N = nrow*ncol q-points (qx, qy real; qz complex);
 * DWBA ("extended") arrays hold 4 blocks of N complex values in the order of
 * QGrid::create_qz_extended (src/model/qgrid.cpp:102-127).  Complex values are interleaved
 * (re, im) pairs.  Rotation matrices are 9 doubles, row-major, as RotMatrix_t stores them
 * (include/numerics/matrix.hpp:30-140).
 */
#ifndef HGX_H
#define HGX_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  HGX_OK = 0,
  HGX_ERR_INVALID_ARG = 1, /* bad size, null pointer, unsupported combination */
  HGX_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  HGX_ERR_NO_MEMORY = 3,   /* device or host allocation failed */
  HGX_ERR_DEVICE = 4,      /* a kernel reported an error (bounded wait expired, bad input) */
  HGX_ERR_NOT_FINITE = 5   /* a result contains NaN/Inf where the model must be finite */
} hgx_status;

typedef enum { HGX_F64 = 0, HGX_F32C = 1 } hgx_precision;
typedef enum { HGX_C128 = 0, HGX_C64 = 1 } hgx_complex_type;

typedef struct hgx_ctx_s* hgx_ctx;
typedef struct hgx_qgrid_s* hgx_qgrid;

/* ------------------------------------------------------------------ context ---- */
const char* hgx_last_error(void);
const char* hgx_status_string(int status);
int hgx_version(void);

/* One context per (thread, device).  `device` < 0 uses the current device. */
int hgx_create(int device, hgx_ctx* out);
int hgx_destroy(hgx_ctx ctx);
/* Stream for asynchronous work (a cudaStream_t; NULL = the legacy default stream). */
int hgx_set_stream(hgx_ctx ctx, void* stream);
void* hgx_get_stream(hgx_ctx ctx);
/* Waits for the context's stream and reports any error a kernel recorded. */
int hgx_synchronize(hgx_ctx ctx);

/* ------------------------------------------------------------------- q-grid ---- */
/* A device-resident q-grid prepared once and reused by every kernel call.
 * Replaces the per-call q-grid upload of the reference's GPU classes
 * (src/ff/gpu/ff_tri_gpu.cu:440-476, src/ff/gpu/ff_ana_gpu.cu:57-98).
 * qx, qy: nqy reals; qz: nqz complex with nqz a multiple of nqy (q-point i uses
 * qx/qy[i % nqy], as the reference's kernels do).  ncol: pixels per detector row when
 * qz is constant along rows (QGrid layout), which enables the row-factorised FP32 kernel;
 * 0 = unknown (detected when qz is host memory, otherwise the per-q-point kernel is used). */
int hgx_qgrid_from_arrays(hgx_ctx ctx, int nqy, const double* qx, const double* qy, int nqz,
                          const double* qz, int ncol, hgx_qgrid* out);
/* QGrid::create + QGrid::create_qz_extended computed on the device
 * (src/model/qgrid.cpp:30-127): a q-space output region of ncol x nrow pixels, incidence
 * angle alpha_i (radians), wave number k0 (1/nm), particle-layer one_minus_n2 = dn2. */
int hgx_qgrid_create(hgx_ctx ctx, int ncol, int nrow, double qmin_y, double qmin_z,
                     double qmax_y, double qmax_z, double alpha_i, double k0, double dn2_re,
                     double dn2_im, hgx_qgrid* out);
/* Copies the grid out (any pointer may be NULL): qx, qy, qz (N each; qz is the real
 * detector qz), alpha (nrow exit angles), qz_ext (4N complex). */
int hgx_qgrid_read(hgx_ctx ctx, hgx_qgrid g, double* qx, double* qy, double* qz, double* alpha,
                   double* qz_ext);
/* Sizes and the kernel mode chosen for the grid: mode 0 = per-q-point, 1 = rows with
 * real paired DWBA blocks, 2 = rows with general complex qz. */
int hgx_qgrid_info(hgx_qgrid g, int* nqy, int* nqz, int* nrow, int* ncol, int* mode);
int hgx_qgrid_destroy(hgx_qgrid g);

/* --------------------------------------------------- numeric (mesh) form factor ---- */
/* F(q) = sum_t (-i)(q'.n_t) s_t exp(i q'.c_t) / |q'|^2 with q' = rot*q, the reference's
 * "approx triangle" formula.  Replaces NumericFormFactorG::compute_approx_triangle
 * (include/ff/gpu/ff_num_gpu.cuh:55-58, src/ff/gpu/ff_tri_gpu.cu:395-521) and its CPU twin
 * NumericFormFactorC::compute_approx_triangle (src/ff/cpu/ff_tri_cpu.cpp:200-246).
 * shape_def: ntri x 8 doubles (s, nx, ny, nz, cx, cy, cz, pad) as read_shapes_file packs
 * them (src/ff/ff_num.cpp:1016-1030).  precision HGX_F64: FP64 throughout, one thread per
 * q-point (the plain form); HGX_F32C: FP32 phases and sums with compensated accumulation.
 * ff: nqz complex of type ff_type. */
int hgx_ff_triangles_q(hgx_ctx ctx, hgx_qgrid g, const double* shape_def, int ntri,
                       const double* rot9, int precision, void* ff, int ff_type);
/* As hgx_ff_triangles_q with an explicit launch shape for the FP32 row kernel:
 * pixels_per_thread 1, 2 or 4 (0 = automatic).  Used by the launch-shape tuner. */
int hgx_ff_triangles_q_ex(hgx_ctx ctx, hgx_qgrid g, const double* shape_def, int ntri,
                          const double* rot9, int precision, void* ff, int ff_type,
                          int pixels_per_thread);
/* The reference-shaped call: explicit q arrays, complex128 output, synchronous.
 * Returns HGX_ERR_INVALID_ARG for ntri < 1 (the reference returns 0 triangles). */
int hgx_ff_triangles(hgx_ctx ctx, const double* shape_def, int ntri, int nqy, const double* qx,
                     const double* qy, int nqz, const double* qz, const double* rot9,
                     int precision, double* ff);

/* The FP32C numeric form factor for callers that cannot allocate device memory: code
 * running inside CUDA graph capture, inside another framework's memory pool or under a
 * fixed memory budget, where a cudaMalloc would fail, break the capture or synchronise the
 * device.  No counterpart in the reference.  Allocates nothing: its scratch is a fixed
 * static device array (1.5 MiB per GPU, held until exit), so ntri <= 65536 (larger
 * requests return HGX_ERR_INVALID_ARG).  All array arguments are device memory (same
 * layouts as hgx_ff_triangles; q-point i uses qx/qy[i % nqy]); rot9 is 9 host doubles or
 * NULL for the identity; ff is nqz complex of type ff_type.  Asynchronous on `stream`
 * (a cudaStream_t; NULL = legacy default stream).  The first call on each device looks up
 * the scratch address (cudaGetSymbolAddress) with that device current; make that first
 * call before any stream capture.  Calls share the scratch: calls that can overlap on the
 * GPU (unordered streams) race and must be ordered by the caller. */
int hgx_ff_triangles_noalloc(const double* shape_def, int ntri, int nqy, const double* qx,
                             const double* qy, int nqz, const double* qz, const double* rot9,
                             void* ff, int ff_type, void* stream);

/* ------------------------------------------------------------- measurement ---- */
/* Throughput probes for roofline denominators (no reference counterpart): FP32 FFMA
 * throughput (TFLOP/s, an FMA counted as 2 FLOP) and SFU __sinf throughput (Gop/s),
 * each the best of three timed launches of a dependent-free chain kernel.  With
 * sustained_ms > 0 the FP32 pipe is first kept busy for that long so that the clocks
 * settle as they do under a long kernel (the sustained figure); 0 gives the burst figure. */
int hgx_measure_peaks(hgx_ctx ctx, int sustained_ms, double* fp32_tflops, double* sfu_gops);

#ifdef __cplusplus
}
#endif
#endif /* HGX_H */

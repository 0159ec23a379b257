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

/* One context per (thread, device).  `device` < 0 uses the current device.  Objects made on
 * a context (q-grids, batches) must be destroyed before the context; a batch must be
 * destroyed before its q-grid. */
int hgx_create(int device, hgx_ctx* out);
int hgx_destroy(hgx_ctx ctx);
/* Stream for asynchronous work (a cudaStream_t; NULL = the legacy default stream).  A change
 * of stream first waits for the work queued on the old one (the context's buffers are reused
 * in stream order), unless the old stream is being captured into a graph. */
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
 * pixels_per_thread 1, 2 or 4 selects the scalar kernel with that many pixels per thread;
 * -2, -4 or -8 the packed FP32x2 kernel (paired real grids only); 0 = automatic (scalar, 4,
 * fewer when the grid is too small to fill the GPU). */
int hgx_ff_triangles_q_ex(hgx_ctx ctx, hgx_qgrid g, const double* shape_def, int ntri,
                          const double* rot9, int precision, void* ff, int ff_type,
                          int pixels_per_thread);
/* The launch-shape autotuner of the FP32C kernel (no reference counterpart; the reference
 * launches one fixed shape).  Times the candidate pixels_per_thread values 4, 2, 1 (scalar)
 * and, on paired real grids, -2, -4, -8 (packed) on these triangles — one untimed launch,
 * then `reps` launches between CUDA events each — and stores the fastest in the grid, where
 * later calls with the automatic shape (hgx_ff_triangles_q, or pixels_per_thread 0) use it.
 * Cost is linear in ntri for every candidate, so a few thousand triangles rank them.
 * best_ppt, best_ms and times_ms (6 means in the order above; 0 for a candidate the grid
 * does not take) may each be NULL.  Per-q-point grids have one shape: best_ppt = 0. */
int hgx_ff_tune(hgx_ctx ctx, hgx_qgrid g, const double* shape_def, int ntri,
                const double* rot9, int ff_type, int reps, int* best_ppt, double* best_ms,
                double* times_ms);
/* The reference-shaped call: explicit q arrays, complex128 output, synchronous.
 * Returns HGX_ERR_INVALID_ARG for ntri < 1 (the reference returns 0 triangles).  The context
 * keeps the q-grid between calls of the same sizes; from the second FP32C call on, with qz in
 * host memory laid out by detector rows (at least 64 q-points per row), the kernel starts from
 * qx, qy and each row's first qz while the 4N qz values are copied and checked beside it (a grid
 * that fails the check is computed again on the full path: the result is the same either way).
 * ff in page-locked host memory is written by the kernel directly. */
int hgx_ff_triangles(hgx_ctx ctx, const double* shape_def, int ntri, int nqy, const double* qx,
                     const double* qy, int nqz, const double* qz, const double* rot9,
                     int precision, double* ff);

/* The exact (polyhedral) triangle form factor: FormFactorTriangle and
 * NumericFormFactorC::compute_exact_triangle (src/ff/cpu/ff_tri_cpu.cpp:46-196), the path of
 * NumericFormFactor::compute2 (src/ff/ff_num.cpp:47-178); GPU twin
 * NumericFormFactorG::compute_exact_triangle (src/ff/gpu/ff_tri_gpu.cu:46-205, 210-...).
 * tris: ntri x 9 doubles (v1, v2, v3 — triangle_t, include/common/typedefs.hpp:102-106),
 * rot9 as above (NULL = identity), FP64 throughout, the reference's sign convention
 * (e^{-i q.v}) and case thresholds.  A degenerate (zero-area) triangle contributes nothing;
 * the reference divides by zero there.  ff: nqz complex of type ff_type. */
int hgx_ff_exact_triangles_q(hgx_ctx ctx, hgx_qgrid g, const double* tris, int ntri,
                             const double* rot9, void* ff, int ff_type);
/* The reference-shaped call: explicit q arrays, complex128 output, synchronous. */
int hgx_ff_exact_triangles(hgx_ctx ctx, const double* tris, int ntri, int nqy, const double* qx,
                           const double* qy, int nqz, const double* qz, const double* rot9,
                           double* ff);

/* ------------------------------------------------------- analytic form factors ---- */
/* AnalyticFormFactor::param_distribution (src/ff/ff_ana.cpp:235-284): the sample values
 * and weights of one shape parameter.  stat: StatisticType (0 null, 2 none, 4 gaussian,
 * 8 uniform; include/common/enums.hpp:74-84).  Host-only, no GPU needed. */
int hgx_param_distribution(int stat, double pmin, double pmax, double mean, double dev,
                           int nvalues, double* values, double* weights, int cap, int* count);
/* The analytic form factor of one shape on the grid, FP64 — replaces the
 * AnalyticFormFactorG::compute_* family (include/ff/gpu/ff_ana_gpu.cuh:28-96) and the CPU
 * AnalyticFormFactor::compute_* functions (src/ff/ff_ana_*.cpp).  shape: ShapeName
 * (include/common/enums.hpp:24-43) among box 2, cube 3, cylinder 4, sphere 5, prism3 8,
 * prism6 9, pyramid 14.  Up to four sampled dimensions (n_i values v_i with weights w_i,
 * at most 64 each; w_i NULL = 1):
 *   box: x, y, height; cube: edge; cylinder: radius, -, height (unweighted, as the
 *   reference sums them); sphere: radius; prism3/prism6: edge, -, height (unweighted);
 *   pyramid: x, y, height, base angle (degrees).
 * tau, eta: the prism tilt angles; transvec: translation (3); rot9: rotation or NULL. */
int hgx_ff_analytic(hgx_ctx ctx, hgx_qgrid g, int shape, int n1, const double* v1,
                    const double* w1, int n2, const double* v2, const double* w2, int n3,
                    const double* v3, const double* w3, int n4, const double* v4,
                    const double* w4, double tau, double eta, const double* transvec,
                    const double* rot9, void* ff, int ff_type);
/* The same with a precision (no counterpart in the reference, which computes in its build's one
 * precision): HGX_F64 as above, or HGX_F32C on grids with real qz for cylinders, spheres and
 * boxes (phases formed and reduced in FP64, FP32 transcendentals and sums); other shapes and
 * complex-qz grids are evaluated in FP64. */
int hgx_ff_analytic_ex(hgx_ctx ctx, hgx_qgrid g, int shape, int n1, const double* v1,
                       const double* w1, int n2, const double* v2, const double* w2, int n3,
                       const double* v3, const double* w3, int n4, const double* v4,
                       const double* w4, double tau, double eta, const double* transvec,
                       const double* rot9, void* ff, int ff_type, int precision);
/* AnalyticFormFactor::compute (src/ff/ff_ana.cpp:61-161) from HiG-style shape parameters:
 * 7 doubles per parameter (ShapeParamType, StatisticType, min, max, mean, deviation,
 * nvalues), routed to dimensions and sampled as the reference's compute_* functions do. */
int hgx_ff_analytic_params(hgx_ctx ctx, hgx_qgrid g, int shape, int nparam,
                           const double* params, double tau, double eta,
                           const double* transvec, const double* rot9, void* ff, int ff_type);
/* hgx_ff_analytic_params with a precision, as hgx_ff_analytic_ex. */
int hgx_ff_analytic_params_ex(hgx_ctx ctx, hgx_qgrid g, int shape, int nparam, const double* params,
                              double tau, double eta, const double* transvec, const double* rot9,
                              void* ff, int ff_type, int precision);

/* ---------------------------------------------------------- structure factor ---- */
/* Lattice::construct_vectors (src/model/structure.cpp:86-182): unscaled a, b, c (9) and
 * basis offset t (3, may be NULL).  type: LatticeType (bcc 2, cubic 3, fcc 4, fco 5, hcp 6,
 * hex 7); hkl "100", "110" or "111" where the reference defines it. */
int hgx_lattice_vectors(int type, const char* hkl, double* abc9, double* t3);
/* StructureFactor::compute_structure_factor, lattice branch (src/sf/sf.cpp:85-285):
 * abc9 lattice vectors, repet (3) repetitions, scaling (3), center (3), rot9.  FP64. */
int hgx_sf_lattice(hgx_ctx ctx, hgx_qgrid g, const double* abc9, const double* repet,
                   const double* scaling, const double* center, const double* rot9, void* sf,
                   int sf_type);
/* The same with a precision: HGX_F32C on grids with real qz and integer repetitions takes the
 * closed form sin(N theta_r / 2) / sin(theta_r / 2) that the reference's principal-branch
 * powers reduce to for a real angle (FP64 angles and reductions, FP32 sines); otherwise FP64. */
int hgx_sf_lattice_ex(hgx_ctx ctx, hgx_qgrid g, const double* abc9, const double* repet,
                      const double* scaling, const double* center, const double* rot9, void* sf,
                      int sf_type, int precision);

/* Paracrystal structure factors: StructureFactor::paracrystal1d / paracrystal2d_cubic /
 * paracrystal2d_hex (src/sf/liquid.cpp:29-110), selected as compute_structure_factor selects
 * them (src/sf/sf.cpp:116-151): dims 1, or dims 2 with lattice 3 (cubic) or 7 (hex);
 * dist_x/dist_y the mean distances, sdev_x/sdev_y their standard deviations, domain the
 * domain size (the 1-D form uses the y values and qy only).  FP64; sf: nqz complex (real
 * values), q-point i uses qx/qy[i % nqy]. */
int hgx_sf_paracrystal(hgx_ctx ctx, hgx_qgrid g, int dims, int lattice, double dist_x,
                       double dist_y, double sdev_x, double sdev_y, double domain, void* sf,
                       int sf_type);
/* Percus-Yevick structure factor: StructureFactor::percus_yevik (src/sf/liquid.cpp:112-165):
 * hard spheres of `diameter` at volume fraction `volfract`; dims 2 uses |q_par|, dims 3 |q|
 * with the complex qz.  The reference's values are reproduced, including the fourth root of
 * the 3-D form and the unrooted alpha/3 + beta/4 + gamma below |q| = 1e-6.  FP64. */
int hgx_sf_percus_yevick(hgx_ctx ctx, hgx_qgrid g, double diameter, double volfract, int dims,
                         void* sf, int sf_type);

/* ---------------------------------------------------------------- DWBA terms ---- */
/* MultiLayer::init + propagation_coeffs (src/model/multilayer.cpp:29-58,110-155), FP64:
 * user layers (delta, beta, thickness, order; order -1 = substrate; host arrays), the
 * particle layer's order, the grid's exit angles (alpha: nrow values, or NULL for a grid
 * made by hgx_qgrid_create).  fc: 4N complex128 in the reference's layout, or with
 * per_row != 0 the nrow x 4 per-row coefficients. */
int hgx_propagation_coeffs(hgx_ctx ctx, hgx_qgrid g, int nlayers, const double* delta,
                           const double* beta, const double* thickness, const int* order,
                           double k0, double alpha_i, int particle_order, const double* alpha,
                           double* fc, int per_row);
/* The DWBA combination (src/sim/hipgisaxs_main.cpp:1086-1100):
 * intensity[i] += |weight * sum_k fc[k n + i] sf[k n + i] ff[k n + i]|^2 over 4 blocks of n;
 * sf may be NULL (1).  With fc NULL the SAXS branch (:1102-1105): intensity[i] =
 * |weight sf[i] ff[i]|^2.  fc, sf complex128; ff of type ff_type. */
int hgx_dwba_combine(hgx_ctx ctx, long n, const double* fc, const double* sf, const void* ff,
                     int ff_type, double weight, double* intensity);

/* ------------------------------------------------------------------ distances ---- */
/* AbsoluteDifferenceSquare (include/analyzer/distance_functions.hpp:125-143):
 * sum (mask |ref - data|)^2, deterministic FP64 reduction. */
int hgx_abs_diff_square(hgx_ctx ctx, long n, const double* ref, const double* data,
                        const unsigned* mask, double* out);
/* ResidualVector (include/analyzer/distance_functions.hpp:89-103): mask (ref - data). */
int hgx_residual_vector(hgx_ctx ctx, long n, const double* ref, const double* data,
                        const unsigned* mask, double* out);
/* Poisson-weighted chi^2 of the fitting front end: sum mask (scale model - counts)^2 /
 * max(counts, 1) (mask may be NULL); deterministic FP64 reduction. */
int hgx_chi2(hgx_ctx ctx, long n, const double* model, const double* counts,
             const unsigned* mask, double scale, double* out);

/* The grain loop of HipGISAXS::run_gisaxs (src/sim/hipgisaxs_main.cpp:794-1100) for one
 * structure whose unit cell holds one triangulated particle, run on the device with no host
 * round trip between grains: for each grain k, the form factor of shape_def (ntri x 8) rotated
 * by rots[9k..] (the grain's composed rotation, :946-951, times the shape's own, :986), the
 * lattice structure factor (abc9 unscaled lattice vectors, repet, scaling) at centre
 * centers[3k..] and rotation rots[9k..] (:1050-1058), and
 * intensity[i] += |weights[k] dn2 sum_j fc_j sf_j ff_j|^2 over the 4 DWBA blocks (:1086-1100).
 * fc: 4N complex (hgx_propagation_coeffs); precision HGX_F32C or HGX_F64 for the form factor
 * (the structure factor and combination are FP64).  intensity: N doubles, overwritten with the
 * sum over grains.  The grid must be a DWBA grid (4 qz blocks). */
int hgx_dwba_mesh_grains(hgx_ctx ctx, hgx_qgrid g, const double* shape_def, int ntri,
                         int ngrains, const double* rots, const double* centers,
                         const double* weights, const double* abc9, const double* repet,
                         const double* scaling, const double* fc, double dn2_re, double dn2_im,
                         int precision, double* intensity);

/* As hgx_dwba_mesh_grains for a unit cell holding one analytic shape: the form factor of each
 * grain is hgx_ff_analytic_params(shape, nparam, params, tau, eta, transvec) at rots[9k..]
 * (AnalyticFormFactor::compute, src/ff/ff_ana.cpp:61-161), FP64. */
int hgx_dwba_analytic_grains(hgx_ctx ctx, hgx_qgrid g, int shape, int nparam,
                             const double* params, double tau, double eta,
                             const double* transvec, int ngrains, const double* rots,
                             const double* centers, const double* weights, const double* abc9,
                             const double* repet, const double* scaling, const double* fc,
                             double dn2_re, double dn2_im, double* intensity);
/* The sum over structures of HipGISAXS::run_gisaxs with uncorrelated structures (its default,
 * src/sim/hipgisaxs_main.cpp:1278-1293, 1352-1362): iratios rescaled to sum to 1 unless they
 * already do; out[z] = sum_s intensities[s n + z] iratio_s.  intensities: nstruct x n. */
int hgx_structure_sum(hgx_ctx ctx, int nstruct, long n, const double* intensities,
                      const double* iratios, double* out);

/* ------------------------------------------------------------ post-processing ---- */
/* Gaussian smearing of a detector image in place (HipGISAXS::gaussian_smearing,
 * src/sim/hipgisaxs_helpers.cpp:25-27, i.e. Convolutions::convolution_gaussian_2d,
 * include/numerics/convolutions.hpp:127-174): image is nrow rows of ncol doubles; a
 * horizontal then a vertical normalised pass over the window [i - r, i + r), r = ceil(6 sigma),
 * with the reference's window arithmetic (right end excluded, weights indexed from the
 * window's start).  sigma > 0 in pixels, 2 r + 1 <= 8193.  FP64, synchronous. */
int hgx_gaussian_smearing(hgx_ctx ctx, double* image, int ncol, int nrow, double sigma);
/* HipGISAXS::normalize (src/sim/hipgisaxs_main.cpp:1439-1450) in place: (x - min) /
 * (max - min) for every element but the first (left as it is, as in the reference);
 * *normalized = 0 and nothing changes when max - min < 1e-30.  Synchronous. */
int hgx_normalize(hgx_ctx ctx, double* data, long n, int* normalized);
/* HipGISAXS::save_gisaxs (src/sim/hipgisaxs_main.cpp:2250-2260): the ".out" text image, each
 * value in the default C++ stream format (6 significant digits) followed by a tab, one
 * detector row per line.  image: nrow x ncol doubles, host memory or device memory of ctx's
 * GPU (ctx may be NULL for a host image). */
int hgx_save_gisaxs(hgx_ctx ctx, const double* image, int nrow, int ncol, const char* path);

/* -------------------------------------------- fitting: chi^2 and its gradient ---- */
/* A fused model for the fitting front end: cylinders on a 2-D lattice in DWBA (one grain,
 * as HipGISAXS::run_gisaxs computes it, src/sim/hipgisaxs_main.cpp:694-1100), its Poisson
 * chi^2 (hgx_chi2) and the gradient of chi^2 with respect to theta = (R, H, a, phi) by a
 * hand-written adjoint — in place of the central finite differences of the reference's
 * LMVM fitter (src/analyzer/hipgisaxs_fit_lmvm.cpp:190-223) and of PSO's one-particle-at-a-
 * time loop (src/analyzer/hipgisaxs_fit_pso.cpp:521-545): many candidates, each with its own
 * detector region of interest, evaluated in one CUDA-graph launch.
 *
 * Model block: 16 doubles per candidate
 *   [0] cylinder radius R   [1] height H   [2] lattice constant a (scales a, b, c)
 *   [3] in-plane rotation phi (radians)    [4] relative Gaussian size spread (0 = one size)
 *   [5] samples over +-3 spread (param_distribution stepping, summed unweighted)
 *   [6..8] lattice repetitions   [9..10] particle contrast dn2 (complex)
 *   [11..13] grain centre   [14] weight
 *   [15] sampling: 0 = the reference's param_distribution stepping (which can gain or lose
 *        the last sample as R or H moves — a jump in chi^2), 1 = exactly [5] evenly spaced
 *        samples (smooth in R and H, for gradient-based fitting).
 * The grid must be a DWBA grid with real qz constant along rows (a vacuum particle layer);
 * rowfc: the per-row Fresnel coefficients (hgx_propagation_coeffs with per_row = 1);
 * abc9: unscaled lattice vectors with a, b in the plane and c along z (hex, cubic).
 * rois: 4 ints per candidate (row0, col0, nrows, ncols); counts: the candidates' ROI images
 * concatenated (row-major), or NULL for forward-only batches; mask: same layout or NULL;
 * scale: the model-to-counts factor of the chi^2.  precision: HGX_F32C (per-pixel arithmetic
 * in FP32: the radial sums interpolated from per-candidate tables over q_par, the lattice
 * factors from FP64-reduced turns; FP64 q, residuals and reductions; about 1e-7 of the FP64
 * chi^2, 1e-6 of its gradient) or HGX_F64 (every Bessel function and lattice factor evaluated
 * per pixel in FP64).  An FP32C batch with counts keeps one FP32 weight per ROI pixel. */
typedef struct hgx_cyl_batch_s* hgx_cyl_batch;
int hgx_cyl_batch_create(hgx_ctx ctx, hgx_qgrid g, const double* rowfc, const double* abc9,
                         int ncand, const int* rois, const double* counts,
                         const unsigned* mask, double scale, int precision,
                         hgx_cyl_batch* out);
/* chi^2 and gradient of every candidate: out = 5 doubles per candidate (chi2, dR, dH, da,
 * dphi).  The first call records the work into a CUDA graph; later calls replay it. */
int hgx_cyl_batch_eval(hgx_cyl_batch b, const double* models, double* out);
/* Model intensities of every candidate (the ROI images concatenated). */
int hgx_cyl_batch_forward(hgx_cyl_batch b, const double* models, double* intensity);
/* The plain FP64 form of candidate `cand`'s intensity: one thread per pixel with the
 * reference's loop structure (per DWBA block, the (radius, height) double loop and the
 * complex-power lattice factor).  Baseline for the finite-difference gradient. */
int hgx_cyl_plain_forward(hgx_cyl_batch b, int cand, const double* model, double* intensity);
int hgx_cyl_batch_info(hgx_cyl_batch b, long* npx, long* nitems);
int hgx_cyl_batch_destroy(hgx_cyl_batch b);
/* Tile shapes of the batch's persistent pixel pass (no reference counterpart; the reference
 * launches one fixed shape per kernel).  A work item is one tile of threads x
 * pixels_per_thread consecutive pixels of a candidate's ROI; the persistent grid is the
 * shape's resident blocks per SM x SM count.  hgx_cyl_shape_info describes table entry
 * `shape` (HGX_ERR_INVALID_ARG past the end, for enumeration); set/get select and read the
 * batch's shape (0 at creation).  Changing the shape drops the recorded CUDA graph; the
 * next hgx_cyl_batch_eval records a new one. */
int hgx_cyl_shape_info(int shape, int* threads, int* pixels_per_thread);
int hgx_cyl_batch_set_shape(hgx_cyl_batch b, int shape);
int hgx_cyl_batch_get_shape(hgx_cyl_batch b, int* shape);
/* The autotuner: times every tile shape on this batch at these models (one untimed
 * evaluation, then `reps` evaluations timed with CUDA events: chi^2 + gradient when the
 * batch has counts, else forward intensities) and keeps the fastest.  best_shape, best_ms
 * and times_ms (one mean per table entry, table order) may each be NULL. */
int hgx_cyl_batch_tune(hgx_cyl_batch b, const double* models, int reps, int* best_shape,
                       double* best_ms, double* times_ms);

/* --------------------------------------------------------- shape-definition files ---- */
/* Wavefront OBJ meshes without Boost (ObjectShapeReader::load_object,
 * src/file/objectshape_reader.cpp:52-242): vertices ("v") and faces ("f" with items v, v/vt,
 * v/vt/vn or v//vn, 1-based); other lines are ignored.  Triangles are kept in file order with
 * 0-based indices; 4-vertex faces are counted (nquads) and left out, as the reference's
 * converter leaves them out; larger faces are counted (nskipped).  Differences from the
 * reference: lines of any length, tabs as separators, and a malformed, relative or
 * out-of-range index returns HGX_ERR_INVALID_ARG instead of undefined behaviour.  Host only. */
typedef struct hgx_mesh_s* hgx_mesh;
int hgx_obj_load(const char* path, hgx_mesh* out);
int hgx_mesh_info(hgx_mesh m, int* nv, int* nf, int* nquads, int* nskipped);
/* verts: nv x 3 doubles, faces: nf x 3 ints (0-based); either may be NULL. */
int hgx_mesh_read(hgx_mesh m, double* verts, int* faces);
int hgx_mesh_destroy(hgx_mesh m);
/* NumericFormFactor::read_shapes_file (src/ff/ff_num.cpp:985-1030): the shape_def rows
 * (T x 8: s, n, c, pad) of an .obj file (triangles converted on the device with the
 * get_triangle_params arithmetic, degenerate faces dropped as convert_to_shape drops them)
 * or of a raw .dat file (7 values per triangle, RawShapeReader::load_raw).  The format is
 * chosen by the extension (obj/Obj/OBJ, dat/Dat/DAT); HDF5 files are rejected, as by a
 * reference build without its optional HDF5 support.  *ntri receives the triangle count;
 * with shape_def NULL nothing else is written, otherwise shape_def must hold capacity >= *ntri
 * rows (host memory).  ctx may be NULL for .dat files (no device work). */
int hgx_read_shapes_file(hgx_ctx ctx, const char* path, double* shape_def, int capacity,
                         int* ntri);

/* ------------------------------------------------------------ triangle meshes ---- */
/* ObjectShapeReader::get_triangle_params / convert_to_shape
 * (src/file/objectshape_reader.cpp:248-300) on the device: vertices nv x 3, faces nf x 3
 * (0-based) -> shape_def nf x 8 (s, n, c, pad) in face order; a degenerate face (which the
 * reference drops) gets s = 0, n = 0 and contributes nothing.  Bad indices: HGX_ERR_DEVICE. */
int hgx_mesh_to_shape_def(hgx_ctx ctx, int nv, const double* verts, int nf, const int* faces,
                          double* shape_def);
/* chi^2 of a triangle mesh in DWBA and its gradient with respect to every vertex
 * coordinate (hand-written adjoint; no counterpart in the reference, whose fitter can only
 * difference the forward model).  I(p) = |weight dn2 sum_k fc_k F_k(p)|^2 with F_k the
 * FP32C mesh form factor of the rotated mesh (rot9 or NULL); rowfc: per-row Fresnel
 * coefficients (nrow x 4); chi^2 = sum mask (scale I - counts)^2 / max(counts, 1).
 * Outputs: chi2 (host double), grad_verts (nv x 3, may be NULL), intensity (N, may be
 * NULL).  The grid must be a DWBA grid with real qz constant along rows. */
int hgx_mesh_chi2_grad(hgx_ctx ctx, hgx_qgrid g, int nv, const double* verts, int nf,
                       const int* faces, const double* rot9, const double* rowfc,
                       double dn2_re, double dn2_im, double weight, const double* counts,
                       const unsigned* mask, double scale, double* chi2, double* grad_verts,
                       double* intensity);
/* The same with a precision: HGX_F32C (as above) or HGX_F64 (plain FP64 form factor, seeds
 * and backward pass, every phase in FP64: the reference of the FP32C gradient). */
int hgx_mesh_chi2_grad_ex(hgx_ctx ctx, hgx_qgrid g, int nv, const double* verts, int nf,
                          const int* faces, const double* rot9, const double* rowfc,
                          double dn2_re, double dn2_im, double weight, const double* counts,
                          const unsigned* mask, double scale, double* chi2, double* grad_verts,
                          double* intensity, int precision);

/* The FP32C numeric form factor for callers that cannot allocate device memory: a plug-in
 * that runs inside another framework's memory pool and is handed only device pointers, a
 * service held to a fixed device-memory budget, or a real-time loop in which a cudaMalloc
 * would synchronise the device.  No counterpart in the reference.  Allocates nothing: its
 * scratch is fixed static device arrays (about 1.5 MiB per GPU, held until exit), so
 * ntri <= 65536 (larger requests return HGX_ERR_INVALID_ARG).  All array arguments are
 * device memory (same layouts as hgx_ff_triangles; q-point i uses qx/qy[i % nqy]); rot9 is
 * 9 host doubles or NULL for the identity; ff is nqz complex of type ff_type.  Asynchronous
 * on `stream` (a cudaStream_t; NULL = legacy default stream).  The first call on each
 * device looks up the scratch address (cudaGetSymbolAddress) with that device current;
 * make that first call before any stream capture.  Calls share the scratch, which keeps the
 * last call's contents: calls that can overlap on the GPU (unordered streams) race and must
 * be ordered by the caller. */
int hgx_ff_triangles_noalloc(const double* shape_def, int ntri, int nqy, const double* qx,
                             const double* qy, int nqz, const double* qz, const double* rot9,
                             void* ff, int ff_type, void* stream);
/* Device errors of hgx_ff_triangles_noalloc (no counterpart in the reference): waits for
 * `stream`, writes the error bits its kernels recorded since the start of the last call on
 * this device into *bits (host memory; 1 = a bounded wait gave up and part of ff is
 * unwritten) and returns HGX_ERR_DEVICE when they are nonzero.  Allocates nothing. */
int hgx_ff_triangles_noalloc_status(void* stream, unsigned* bits);

/* -------------------------------------------------------------- HiG input files ---- */
/* A simulation description read from a HiG file: HiGInput::construct_input_config
 * (src/config/hig_input.cpp:61-104, tokenizer src/file/read_oo_input.cpp, keywords
 * include/config/token_mapper.hpp).  Files the reference reads are read to the same values,
 * `include = "file"` splicing and the reference's carry-over quirks included; a file it
 * rejects is rejected (HGX_ERR_INVALID_ARG, the message names file and line).  Host only. */
typedef struct hgx_hig_s* hgx_hig;
int hgx_hig_read(const char* path, hgx_hig* out);
/* The whole description as JSON (shapes, layers, unitcells, structures, scattering, detector,
 * computation, fitting).  buf may be NULL to ask for the size: *len receives the length
 * without the terminating NUL; with buf, cap must be > *len. */
int hgx_hig_json(hgx_hig h, char* buf, size_t cap, size_t* len);
int hgx_hig_destroy(hgx_hig h);
/* The beam of HipGISAXS::init (src/sim/hipgisaxs_main.cpp:146-160): wave number k0 (1/nm)
 * from the photon energy ("ev" or "kev"), incidence angle alphai.min in radians, frequency.
 * Any output may be NULL. */
int hgx_hig_beam(hgx_hig h, double* k0, double* alpha_i, double* freq);
/* QGrid::create for the computation block's q-space output region and resolution
 * (src/model/qgrid.cpp:30-101) at the file's beam, then create_qz_extended with
 * dn2 = dn2_re + i dn2_im (the layer's 1 - n^2): a DWBA grid, built on the device. */
int hgx_hig_qgrid(hgx_ctx ctx, hgx_hig h, double dn2_re, double dn2_im, hgx_qgrid* out);
/* The detector image size of the description (computation.resolution): nrow x ncol. */
int hgx_hig_image_size(hgx_hig h, int* nrow, int* ncol);
/* HipGISAXS::compute_gisaxs (src/sim/hipgisaxs_main.cpp:630-685, run_gisaxs :694-1440) on
 * the device: for every structure and every grain of its ensemble, the unit cell's form
 * factor (analytic shapes at each location, mesh shapes from their .obj/.dat file), the
 * structure factor (lattice, paracrystal or Percus-Yevick) and the DWBA intensity with the
 * layer stack's Fresnel coefficients; the structures summed with their iratios.  image:
 * nrow x ncol doubles (host or device).  precision: HGX_F64, or HGX_F32C for the mesh form
 * factors and, on grids with real qz blocks, the fused grain kernel's cylinder, sphere and box
 * unit cells with their lattice structure factors (FP64 phase reduction, FP32 transcendentals
 * and sums, FP64 intensity; other cells stay FP64).  Supported: GISAXS and SAXS (expt "saxs": run_gisaxs's Born branch, :1099-1103, whose
 * assignment leaves each structure the image of its last grain's last scaling sample), one
 * alpha_i/phi/tilt, no structure correlation,
 * regular grain grids; "single", "range", "random" (drawn with the C library's rand() in the
 * reference's order), "gaussian", "normal" and "cauchy" orientations; gaussian/cauchy grain
 * scalings and ranged repetitions (the reference's seeded Mersenne Twister).  Other
 * descriptions return HGX_ERR_INVALID_ARG naming the feature.  nslices > 1 gives the
 * reference's zero image (its slicing branch only prints that it is not implemented).
 * With a host image the call is synchronous; with a device image it is asynchronous on the
 * context's stream (errors of its kernels surface at the next synchronising call, e.g.
 * hgx_synchronize), so that the host prepares the next simulation while this one runs. */
int hgx_hig_compute_gisaxs(hgx_ctx ctx, hgx_hig h, int precision, double* image);
/* Angle scans, as HipGISAXS::run_all_gisaxs walks them (src/sim/hipgisaxs_main.cpp:283-613):
 * the numbers of incidence angles, in-plane rotations and tilts (alphai, inplanerot, tilt
 * blocks: (max - min) / step + 1 truncated, 1 for a zero step; alphai's max raised to its min),
 * and scan point p = (i * nphi + j) * ntilt + k with its angles in degrees accumulated from the
 * minimum as the reference's loops accumulate them.  hgx_hig_compute_scan_point is
 * hgx_hig_compute_gisaxs at point p: the detector grid of the first alpha_i (HipGISAXS::init),
 * qz_extended and the Fresnel coefficients at the point's alpha_i, the structures rotated by
 * its phi (run_gisaxs does not use the tilt).  The reference's per-alpha_i "averaged" output
 * is the plain sum of the point images over phi and tilt, in point order. */
/* The computation block's pathprefix ("." by default) and runname as written ("" when not
 * given); the reference writes a run's files under pathprefix/runname_<YYYYmmdd_HHMMSS>
 * (run_<...> without a runname; ComputeParams, src/model/compute_params.cpp:24-78). */
int hgx_hig_output_names(hgx_hig h, char* pathprefix, size_t prefix_cap, char* runname, size_t run_cap);
int hgx_hig_scan_size(hgx_hig h, int* nalphai, int* nphi, int* ntilt);
int hgx_hig_scan_point(hgx_hig h, int p, double* alphai_deg, double* phi_deg, double* tilt_deg);
int hgx_hig_compute_scan_point(hgx_ctx ctx, hgx_hig h, int precision, int p, double* image);

/* The fitting block of a HiG description: parameters in key order (the order of
 * HiGInput::fit_param_keys, which the reference's fitters use for their x vectors). */
int hgx_hig_fit_count(hgx_hig h, int* n);
/* Parameter i: key, variable (e.g. "shape['s1']:param['radius']:min"), range (min, max,
 * step) and init; any output may be NULL. */
int hgx_hig_fit_param(hgx_hig h, int i, char* key, size_t key_cap, char* variable, size_t var_cap,
                      double* range3, double* init);
/* HiGInput::update_params (src/config/hig_input.cpp:2712-2830) for one variable, with the
 * update_param methods of the model classes and their quirks (a rotation's value is taken in
 * radians; "rot2['..']:max" sets rot2's minimum; "spacing:2" is not accepted, "spacing:z" is;
 * "xrot" is refused where the reference throws). */
int hgx_hig_update_param(hgx_hig h, const char* variable, double value);
/* All fit parameters at once: x[i] for the i-th key (nx = hgx_hig_fit_count). */
int hgx_hig_fit_update(hgx_hig h, const double* x, int nx);

/* The fitting block's reference data (HiGInput::reference_data_path / reference_data_mask,
 * include/config/hig_input.hpp:327-328; FitReferenceData, include/config/temp_helpers.hpp:26-62):
 * one referencedata block, i = 0.  The image and mask paths as written ("" when not given;
 * the reference opens them relative to the working directory) and the npoints counts (0 when
 * not given).  Any output may be NULL. */
int hgx_hig_fit_reference(hgx_hig h, int i, char* path, size_t path_cap, char* mask, size_t mask_cap,
                          int* npar, int* nperp);
/* HipGISAXS::override_qregion (src/sim/hipgisaxs_main.cpp:236-277): the simulation re-gridded
 * to a reference image of ny x nz pixels over the referencedata block's fit region (regmin,
 * regmax; 0 when not given, as in the reference), i.e. the computation block's resolution and
 * q-space region replaced (QGrid::update, src/model/qgrid.cpp:133-197).  Only a qspace output
 * region (the reference has not implemented the others).  Host only. */
int hgx_hig_override_qregion(hgx_hig h, int ny, int nz, int i);
/* The fitting block's analysis algorithms in file order (HiGInput::analysis_algo,
 * analysis_distance_metric, analysis_tolerance, analysis_regularization,
 * include/config/hig_input.hpp:338-345): the name ("pso", "lmvm", "pounders", "bruteforce",
 * "none_pounders", "error" for an unknown one), the distance metric as an hgx_fit_metric (-1
 * when not given or not one of them), tolerance and regularization.  Any output may be NULL. */
int hgx_hig_fit_algorithm_count(hgx_hig h, int* n);
int hgx_hig_fit_algorithm(hgx_hig h, int i, char* name, size_t name_cap, int* metric, double* tolerance,
                          double* regularization);

/* A fit's reference image and mask as the reference reads them
 * (src/analyzer/objective_func_hipgisaxs.cpp:83-205): the type by extension (edf/EDF: EDF,
 * src/file/edf_reader.cpp; txt/TXT/dat/DAT/out/OUT: text, ImageData::read,
 * src/analyzer/ImageData.cpp:79-104, whose row count leaves out a last line without a newline).
 * *count receives the number of values read (it exceeds ncol x nrow by that last line); data
 * may be NULL to ask for the sizes, otherwise capacity must hold every value.  Masks: the unsigned integers of
 * a text file (a last value followed directly by the end of the file is dropped, as the
 * reference drops it) or an EDF image's values.  Host only. */
int hgx_read_image(const char* path, double* data, long capacity, long* count, int* ncol, int* nrow);
int hgx_read_mask(const char* path, unsigned* mask, long capacity, long* count);

/* ------------------------------------------------------------- fitting metrics ---- */
/* The distance measures of the reference's HiG-driven fitter
 * (include/analyzer/distance_functions.hpp:387-844, chosen by the fitting block's
 * distancemetric, src/analyzer/hipgisaxs_fit_main.cpp:82-104): square- or cube-rooted images,
 * unit-vector (L2 or L1) or c-normalised, masked.  out: 1 value, or n per-pixel values for the
 * residual forms.  mask may be NULL (all pixels).  FP64, deterministic order. */
typedef enum {
  HGX_METRIC_SQRT_UNIT_L2 = 0,
  HGX_METRIC_SQRT_C_L2 = 1,
  HGX_METRIC_CBRT_UNIT_L2 = 2,
  HGX_METRIC_CBRT_C_L2 = 3,
  HGX_METRIC_SQRT_UNIT_L2_RESIDUAL = 4,
  HGX_METRIC_SQRT_C_L2_RESIDUAL = 5,
  HGX_METRIC_SQRT_UNIT_L1 = 6,
  HGX_METRIC_CBRT_UNIT_L1 = 7
} hgx_fit_metric;
int hgx_fit_distance(hgx_ctx ctx, int metric, long n, const double* ref, const double* data,
                     const unsigned* mask, double* out);
/* HipGISAXSObjectiveFunction::operator() (src/analyzer/objective_func_hipgisaxs.cpp:263-320)
 * for a HiG description: set the fit parameters to x (key order), simulate
 * (hgx_hig_compute_gisaxs, FP64), measure the distance to ref (nrow x ncol) under mask, add
 * the regularisation (reg_alpha/2) |x - mean|^2 spread over the distance vector (mean = the
 * middle of each parameter's range; a non-finite entry becomes 1e8).  dist: host memory for
 * 1 value, or nrow*ncol for the residual forms; *ndist receives the count. */
int hgx_hig_objective(hgx_ctx ctx, hgx_hig h, const double* x, int nx, const double* ref,
                      const unsigned* mask, int metric, double reg_alpha, double* dist, long* ndist);
/* hgx_hig_objective for a scalar distance measure (not the residual vectors) and its
 * gradient with respect to the fit parameters (grad: nx host doubles, key order).  The
 * reference's LMVM fitter differentiates dist[0] by central differences, two simulations per
 * parameter (src/analyzer/hipgisaxs_fit_lmvm.cpp:190-223).  Here one FP64 simulation, the
 * derivative of the distance with respect to the image on the device, and per parameter the
 * tangent of the image through the fused grain loop's form factors, lattice structure factor
 * and DWBA sum (hand-written derivatives), contracted with it; the regularisation adds
 * reg_alpha (x - mean).  Parameters: anything that moves the analytic shapes' samples and
 * weights (cylinder, sphere, box), element locations, orientations (not "range"/"random"),
 * grain spacings, lattice vectors or scalings; parameters that change refractive indices,
 * layers, the beam, liquid structure factors, iratios or a sample count return
 * HGX_ERR_INVALID_ARG with the reason.  DWBA grids with real qz (vacuum particle layer). */
int hgx_hig_objective_grad(hgx_ctx ctx, hgx_hig h, const double* x, int nx, const double* ref,
                           const unsigned* mask, int metric, double reg_alpha, double* dist,
                           double* grad);
/* A fitting population of a HiG description: the particle loop of the reference's PSO fitter
 * (src/analyzer/hipgisaxs_fit_pso.cpp:521-545), which calls the objective
 * (HipGISAXSObjectiveFunction::operator(), src/analyzer/objective_func_hipgisaxs.cpp:263-320)
 * once per particle, for npop candidates at a time.  _create copies the description (later
 * changes to h do not reach the population), builds the grid, the Fresnel coefficients and any
 * paracrystal or Percus-Yevick structure factor once, and keeps ref (nrow x ncol) and mask.
 * _eval: X = npop x nx parameter vectors (host, key order per row), dist = npop host doubles,
 * each the value hgx_hig_objective returns for that row (the same simulation arithmetic and
 * distance sums at HGX_F64; HGX_F32C runs the fused grain kernel's FP32C bodies where
 * hgx_hig_compute_gisaxs would).  One evaluation: the host builds every candidate's grain
 * tables; a CUDA graph, recorded on the first evaluation and replayed after, copies them from
 * pinned memory, runs each fused grain launch for all candidates together, sums the
 * structures, reduces all distances and copies them back.  Candidates may move what those
 * tables hold (shape samples and weights, locations, orientations other than "range"/"random",
 * spacings, lattice vectors, scalings); a candidate that changes a refractive index, a layer,
 * the beam, a liquid structure factor, an iratio, a grain, sample or element count returns
 * HGX_ERR_INVALID_ARG with the reason.  GISAXS descriptions of analytic shapes; scalar
 * distance measures only. */
typedef struct hgx_hig_pop_s* hgx_hig_pop;
int hgx_hig_population_create(hgx_ctx ctx, hgx_hig h, int npop, const double* ref,
                              const unsigned* mask, int metric, double reg_alpha, int precision,
                              hgx_hig_pop* out);
int hgx_hig_population_eval(hgx_hig_pop pop, const double* X, int nx, double* dist);
int hgx_hig_population_destroy(hgx_hig_pop pop);

/* ------------------------------------------------------------- measurement ---- */
/* Throughput probes for roofline denominators (no reference counterpart): FP32 FFMA
 * throughput (TFLOP/s, an FMA counted as 2 FLOP) and SFU __sinf throughput (Gop/s),
 * each the best of three timed launches of a dependent-free chain kernel.  With
 * sustained_ms > 0 the FP32 pipe is first kept busy for that long so that the clocks
 * settle as they do under a long kernel (the sustained figure); 0 gives the burst figure. */
int hgx_measure_peaks(hgx_ctx ctx, int sustained_ms, double* fp32_tflops, double* sfu_gops);
/* FP64 FMA throughput (TFLOP/s, FMA = 2) of a DFMA-chain probe on the context's device: the
 * roofline denominator of the FP64-bound kernels (no counterpart in the reference). */
int hgx_measure_peak_fp64(hgx_ctx ctx, double* fp64_tflops);

#ifdef __cplusplus
}
#endif
#endif /* HGX_H */

/*
 * TEST INFRASTRUCTURE — the CPU oracle.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load this library, and only as the
 * checker.  The product (hipgisaxs_b200/) never links or calls it.
 *
 * A plain-C, FP64 restatement of the reference's CPU hot path (tacaswell/hipgisaxs),
 * following the reference's evaluation order so that results agree with the compiled
 * reference (oracle/_ref/libhigref.so) to rounding.  Complex values are interleaved
 * (re, im) doubles.  Array layouts follow the reference: a detector of nrow x ncol pixels
 * is flattened row-major (N = nrow*ncol); "extended" (DWBA) arrays hold 4 blocks of N.
 *
 * Parity is pinned against the compiled reference (tests/golden fixtures generated from
 * oracle/_ref by tests/golden/gen_golden.py) and against analytic known answers.
 */
#ifndef HGX_ORACLE_H
#define HGX_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

int orc_set_threads(int n);

/* QGrid::create, src/model/qgrid.cpp:30-99 (q-space output region). alpha: nrow. */
int orc_qgrid_create(int ncol, int nrow, double qmin_y, double qmin_z, double qmax_y,
                     double qmax_z, double alpha_i, double k0, double* qx, double* qy,
                     double* qz, double* alpha);
/* QGrid::create_qz_extended, src/model/qgrid.cpp:102-127.  qz_ext: 4N complex. */
int orc_qz_extended(int n, const double* qz, double k0, double alpha_i, double dn2_re,
                    double dn2_im, double* qz_ext);
/* MultiLayer::parratt_recursion, src/model/multilayer.cpp:65-108.
 * Layers in reference order (0 = vacuum ... last = substrate): one_minus_n2 (complex,
 * 2 doubles each) and z (cumulative depth).  Out: T, R at `order` (4 doubles). */
int orc_parratt(int nl, const double* one_minus_n2, const double* z, double alpha, double k0,
                int order, double* tr);
/* MultiLayer::init + propagation_coeffs, src/model/multilayer.cpp:29-58,110-155.
 * layers: (delta, beta, thickness, order) per user layer, order -1 = substrate.
 * alpha: nrow exit angles (QGrid order).  fc: 4N complex. */
int orc_propagation_coeffs(int nlayers, const double* delta, const double* beta,
                           const double* thickness, const int* order, double k0,
                           double alpha_i, int particle_order, int nrow, int ncol,
                           const double* alpha, double* fc);
/* RotMatrix_t(axis, angle), include/numerics/matrix.hpp:47-69; row-major 3x3. */
void orc_rot_axis(int axis, double angle, double* r9);
/* RotMatrix_t::operator*(RotMatrix_t), include/numerics/matrix.hpp:104-111. */
void orc_rot_mul(const double* a, const double* b, double* out);

/* NumericFormFactorC::compute_approx_triangle, src/ff/cpu/ff_tri_cpu.cpp:200-246.
 * shape_def: T x 8 (s, nx, ny, nz, cx, cy, cz, pad).  qz: nqz complex; ff: nqz complex. */
int orc_ff_approx_triangle(const double* shape_def, int ntri, int nqy, const double* qx,
                           const double* qy, int nqz, const double* qz, const double* rot9,
                           double* ff);
/* NumericFormFactorC::compute_exact_triangle (src/ff/cpu/ff_tri_cpu.cpp:46-196): tris is
 * ntri x 9 (v1, v2, v3); ff nqz complex. */
int orc_ff_exact_triangle(const double* tris, int ntri, int nqy, const double* qx,
                          const double* qy, int nqz, const double* qz, const double* rot9,
                          double* ff);
/* ObjectShapeReader::get_triangle_params, src/file/objectshape_reader.cpp:275-300.
 * Returns 0 for a degenerate triangle (dropped by the reference). */
int orc_triangle_params(const double* v1, const double* v2, const double* v3, double* s,
                        double* n3, double* c3);
/* ObjectShapeReader::convert_to_shape, src/file/objectshape_reader.cpp:248-269, with the
 * 7 -> 8 padding of NumericFormFactor::read_shapes_file (src/ff/ff_num.cpp:1016-1030).
 * faces: 0-based vertex indices.  Returns the number of triangles written. */
int orc_mesh_to_shape_def(int nv, const double* verts, int nf, const int* faces,
                          double* shape_def);

/* AnalyticFormFactor::param_distribution, src/ff/ff_ana.cpp:235-284.
 * Returns the count written to dim/weight (<= cap), or -1 on error. */
int orc_param_distribution(int stat, double pmin, double pmax, double mean, double dev,
                           int nvalues, double* dim, double* weight, int cap);
/* AnalyticFormFactor::compute, src/ff/ff_ana.cpp:61-161, for the shapes the reference
 * implements (box, cube, cylinder, sphere, prism3, prism6, pyramid).  shape: ShapeName
 * enum values of include/common/enums.hpp:24-43.  params: 7 doubles per parameter
 * (type, stat, min, max, mean, deviation, nvalues).  Grid arrays as in the triangle FF. */
int orc_ff_analytic(int shape, int nparam, const double* params, double tau, double eta,
                    const double* transvec, const double* rot9, int nqy, const double* qx,
                    const double* qy, int nqz, const double* qz, double* ff);

/* Lattice::construct_vectors, src/model/structure.cpp:86-182.  type: LatticeType enum;
 * hkl "100"/"110"/"111".  Out a, b, c, t (3 each).  Returns 0 on success. */
int orc_lattice_vectors(int type, const char* hkl, double* a, double* b, double* c, double* t);
/* StructureFactor::compute_structure_factor, src/sf/sf.cpp:85-285 (lattice branch). */
int orc_sf_lattice(const double* abc9, const double* repet, const double* scaling,
                   const double* center, const double* rot9, int nqy, const double* qx,
                   const double* qy, int nqz, const double* qz, double* sf);

/* Paracrystal SFs, src/sf/liquid.cpp:29-110 (dims 1; dims 2 with lattice 3 cubic / 7 hex). */
int orc_sf_paracrystal(int dims, int lattice, double dx, double dy, double sx, double sy,
                       double dom, int nqy, const double* qx, const double* qy, int nqz,
                       double* sf);
/* Percus-Yevick SF, src/sf/liquid.cpp:112-165 (dims 2 or 3). */
int orc_sf_percus_yevick(double dia, double volf, int dims, int nqy, const double* qx,
                         const double* qy, int nqz, const double* qz, double* sf);

/* DWBA combination, src/sim/hipgisaxs_main.cpp:1086-1100: I[i] += |w * sum_k fc sf ff|^2. */
void orc_dwba_combine(int n, const double* fc, const double* sf, const double* ff,
                      double weight, double* intensity);
/* SAXS branch, src/sim/hipgisaxs_main.cpp:1102-1105: I[i] = |w * sf * ff|^2. */
void orc_saxs_combine(int n, const double* sf, const double* ff, double weight,
                      double* intensity);

/* Distance measures, include/analyzer/distance_functions.hpp:89-143. */
double orc_abs_diff_square(int n, const double* ref, const double* data,
                           const unsigned* mask);
void orc_residual_vector(int n, const double* ref, const double* data, const unsigned* mask,
                         double* out);
/* Poisson-weighted chi^2 used by the fitting front end of this project:
 * sum mask*(scale*I - C)^2 / max(C, 1). */
double orc_chi2(int n, const double* model, const double* counts, const unsigned* mask,
                double scale);

/* HipGISAXS::run_gisaxs structure sum (src/sim/hipgisaxs_main.cpp:1278-1293, 1352-1362);
 * at most 256 structures. */
void orc_structure_sum(int ns, long n, const double* img, const double* iratios, double* out);
/* Convolutions::convolution_gaussian_2d (include/numerics/convolutions.hpp:127-174), in place
 * on ny rows of nx. */
int orc_smear_gaussian(double* data, int nx, int ny, double sigma);
/* HipGISAXS::normalize (src/sim/hipgisaxs_main.cpp:1439-1450), in place; 1 if normalised. */
int orc_normalize(double* data, long n);

/* The fitter's distance measures (distance_functions.hpp:387-844), numbered as
 * hgx_fit_distance numbers them.  Returns the count written to out (1 or n), -1 on error. */
long orc_fit_distance(int metric, long n, const double* ref, const double* dat, const unsigned* mask,
                      double* out);

#ifdef __cplusplus
}
#endif
#endif

// Test infrastructure only: a C-ABI wrapper over the reference's OWN CPU hot-path
// classes (HipGISAXS, tacaswell/hipgisaxs), compiled from the reference sources by
// oracle/Makefile into oracle/_ref/libhigref.so.  It is used to pin the plain-C
// restatement in oracle/hgx_oracle.c and to generate the committed golden fixtures
// (tests/golden/gen_golden.py); the CPU reference arm of bench.py times it.
// Nothing in the product (hipgisaxs_b200/) links or loads it.
//
// Every entry point drives the reference class that owns the computation:
//   QGrid::create / create_qz_extended  (src/model/qgrid.cpp:30-127)
//   MultiLayer::init / propagation_coeffs (src/model/multilayer.cpp:29-155)
//   NumericFormFactorC::compute_approx_triangle (src/ff/cpu/ff_tri_cpu.cpp:200-246)
//   AnalyticFormFactor::compute (src/ff/ff_ana.cpp:61-161)
//   StructureFactor::compute_structure_factor (src/sf/sf.cpp:85-285)
//   the fitter's distance measures (include/analyzer/distance_functions.hpp:387-844)
#include <complex>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include <common/typedefs.hpp>
#include <common/enums.hpp>
#include <model/qgrid.hpp>
#include <model/compute_params.hpp>
#include <model/layer.hpp>
#include <model/shape.hpp>
#include <model/structure.hpp>
#include <common/constants.hpp>  // PI_, TINY_ used by convolutions.hpp
#include <numerics/convolutions.hpp>
#include <numerics/matrix.hpp>
#include <ff/cpu/ff_num_cpu.hpp>
#include <ff/ff_ana.hpp>
#include <sf/sf.hpp>
#include <analyzer/distance_functions.hpp>
#include <analyzer/ImageData.hpp>
#include <file/edf_reader.hpp>

#ifdef _OPENMP
#include <omp.h>
#endif

using namespace hig;

namespace {
RotMatrix_t make_rot(const double* r9) {
  vector3_t a(r9[0], r9[1], r9[2]), b(r9[3], r9[4], r9[5]), c(r9[6], r9[7], r9[8]);
  return RotMatrix_t(a, b, c);
}
}  // namespace

extern "C" {

int ref_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

// QGrid::create with a q-space output region; fills the singleton and copies it out.
// qx,qy,qz: nrow*ncol doubles; alpha: nrow doubles (after the reference's reversal).
int ref_qgrid_create(int ncol, int nrow, double qmin_y, double qmin_z, double qmax_y,
                     double qmax_z, double alpha_i_rad, double k0, double* qx, double* qy,
                     double* qz, double* alpha) {
  ComputeParams cp;
  cp.init();
  cp.output_region_type(region_qspace);
  cp.output_region_minpoint(qmin_y, qmin_z);
  cp.output_region_maxpoint(qmax_y, qmax_z);
  cp.resolution(ncol, nrow);
  QGrid& g = QGrid::instance();
  // QGrid::create appends to the singleton's vectors (it is meant to run once per process);
  // later grids go through QGrid::update, which clears them and evaluates the same formulas
  // (src/model/qgrid.cpp:133-192 vs :30-99).
  if (g.nqy() == 0) {
    if (!g.create(cp, alpha_i_rad, k0, 1)) return -1;
  } else {
    if (!g.update(ncol, nrow, qmin_y, qmin_z, qmax_y, qmax_z, 0.0, alpha_i_rad, k0, 1))
      return -1;
  }
  int n = g.nqy();
  if (n != ncol * nrow) return -2;
  if (qx) for (int i = 0; i < n; ++i) qx[i] = g.qx(i);
  if (qy) for (int i = 0; i < n; ++i) qy[i] = g.qy(i);
  if (qz) for (int i = 0; i < n; ++i) qz[i] = g.qz(i);
  if (alpha) for (int i = 0; i < g.nalpha(); ++i) alpha[i] = g.alpha(i);
  return 0;
}

// QGrid::update (the fitting ROI override, src/model/qgrid.cpp:133-192).
int ref_qgrid_update(int nqy, int nqz, double qminy, double qminz, double qmaxy, double qmaxz,
                     double alpha_i_rad, double k0, double* qx, double* qy, double* qz,
                     double* alpha) {
  QGrid& g = QGrid::instance();
  if (!g.update(nqy, nqz, qminy, qminz, qmaxy, qmaxz, 0.0, alpha_i_rad, k0, 1)) return -1;
  int n = g.nqy();
  if (qx) for (int i = 0; i < n; ++i) qx[i] = g.qx(i);
  if (qy) for (int i = 0; i < n; ++i) qy[i] = g.qy(i);
  if (qz) for (int i = 0; i < n; ++i) qz[i] = g.qz(i);
  if (alpha) for (int i = 0; i < g.nalpha(); ++i) alpha[i] = g.alpha(i);
  return 0;
}

// QGrid::create_qz_extended on the current singleton grid; qz_ext: 4N complex (interleaved).
int ref_qz_extended(double k0, double alpha_i_rad, double dn2_re, double dn2_im,
                    double* qz_ext) {
  QGrid& g = QGrid::instance();
  if (!g.create_qz_extended(k0, alpha_i_rad, complex_t(dn2_re, dn2_im))) return -1;
  int n = g.nqz_extended();
  for (int i = 0; i < n; ++i) {
    complex_t v = g.qz_extended(i);
    qz_ext[2 * i] = v.real();
    qz_ext[2 * i + 1] = v.imag();
  }
  return 0;
}

// MultiLayer::init + propagation_coeffs on the current singleton grid.
// layers: nlayers entries (delta, beta, thickness, order); order -1 = substrate.
// fc: 4N complex (interleaved).
int ref_propagation_coeffs(int nlayers, const double* delta, const double* beta,
                           const double* thickness, const int* order, double k0,
                           double alpha_i_rad, int particle_order, double* fc) {
  layer_list_t layers;
  for (int i = 0; i < nlayers; ++i) {
    Layer l;
    l.init();
    l.refindex_delta(delta[i]);
    l.refindex_beta(beta[i]);
    l.thickness(thickness[i]);
    l.order(order[i]);
    layers[order[i]] = l;
  }
  MultiLayer ml;
  if (!ml.init(layers)) return -1;
  complex_vec_t coeff;
  if (!ml.propagation_coeffs(coeff, k0, alpha_i_rad, particle_order)) return -2;
  for (size_t i = 0; i < coeff.size(); ++i) {
    fc[2 * i] = coeff[i].real();
    fc[2 * i + 1] = coeff[i].imag();
  }
  return (int)coeff.size();
}

// MultiLayer::parratt_recursion for one angle: returns T, R at `order`.
int ref_parratt(int nlayers, const double* delta, const double* beta, const double* thickness,
                const int* order, double alpha, double k0, int particle_order, double* tr4) {
  layer_list_t layers;
  for (int i = 0; i < nlayers; ++i) {
    Layer l;
    l.init();
    l.refindex_delta(delta[i]);
    l.refindex_beta(beta[i]);
    l.thickness(thickness[i]);
    l.order(order[i]);
    layers[order[i]] = l;
  }
  MultiLayer ml;
  if (!ml.init(layers)) return -1;
  complex_vec_t c = ml.parratt_recursion(alpha, k0, particle_order);
  tr4[0] = c[0].real(); tr4[1] = c[0].imag();
  tr4[2] = c[1].real(); tr4[3] = c[1].imag();
  return 0;
}

// NumericFormFactorC::compute_approx_triangle on explicit arrays.
// shape_def: T x 8 doubles; qz: nqz complex interleaved; ff: nqz complex interleaved.
int ref_ff_approx_triangle(const double* shape_def, int ntri, int nqy, const double* qx,
                           const double* qy, int nqz, const double* qz, const double* rot9,
                           double* ff) {
  real_vec_t sd(shape_def, shape_def + 8 * (size_t)ntri);
  std::vector<complex_t> qzc(nqz);
  for (int i = 0; i < nqz; ++i) qzc[i] = complex_t(qz[2 * i], qz[2 * i + 1]);
  std::vector<real_t> qxv(qx, qx + nqy), qyv(qy, qy + nqy);
  RotMatrix_t rot = make_rot(rot9);
  NumericFormFactorC cff;
  complex_t* out = nullptr;
  real_t t = 0;
  unsigned r = cff.compute_approx_triangle(sd, out, nqy, qxv.data(), qyv.data(), nqz,
                                           qzc.data(), rot, t);
  if (r == 0 || out == nullptr) return -1;
  for (int i = 0; i < nqz; ++i) {
    ff[2 * i] = out[i].real();
    ff[2 * i + 1] = out[i].imag();
  }
  delete[] out;
  return (int)r;
}

int ref_ff_exact_triangle(const double* tris, int ntri, int nqy, const double* qx,
                          const double* qy, int nqz, const double* qz, const double* rot9,
                          double* ff) {
  std::vector<triangle_t> tv(ntri);
  for (int t = 0; t < ntri; ++t)
    for (int k = 0; k < 3; ++k) {
      tv[t].v1[k] = tris[9 * t + k];
      tv[t].v2[k] = tris[9 * t + 3 + k];
      tv[t].v3[k] = tris[9 * t + 6 + k];
    }
  std::vector<complex_t> qzc(nqz);
  for (int i = 0; i < nqz; ++i) qzc[i] = complex_t(qz[2 * i], qz[2 * i + 1]);
  std::vector<real_t> qxv(qx, qx + nqy), qyv(qy, qy + nqy);
  RotMatrix_t rot = make_rot(rot9);
  NumericFormFactorC cff;
  complex_t* out = nullptr;
  real_t t = 0;
  unsigned r = cff.compute_exact_triangle(tv.data(), ntri, out, nqy, qxv.data(), qyv.data(), nqz,
                                          qzc.data(), rot, t);
  if (r == 0 || out == nullptr) return -1;
  for (int i = 0; i < nqz; ++i) {
    ff[2 * i] = out[i].real();
    ff[2 * i + 1] = out[i].imag();
  }
  delete[] out;
  return (int)r;
}

// AnalyticFormFactor::compute on the current singleton grid (extended qz).
// params: nparam entries of (type, stat, min, max, mean, deviation, nvalues) as doubles.
int ref_ff_analytic(int shape, int nparam, const double* params, double tau, double eta,
                    const double* transvec, const double* rot9, double* ff) {
  shape_param_list_t plist;
  for (int i = 0; i < nparam; ++i) {
    const double* p = params + 7 * i;
    ShapeParam sp;
    sp.init();
    sp.type((ShapeParamType)(int)p[0]);
    sp.stat((StatisticType)(int)p[1]);
    sp.min(p[2]);
    sp.max(p[3]);
    sp.mean(p[4]);
    sp.deviation(p[5]);
    sp.nvalues(p[6]);
    sp.set();
    plist[std::string("p") + std::to_string(i)] = sp;
  }
  RotMatrix_t rot = make_rot(rot9);
  std::vector<complex_t> out;
  AnalyticFormFactor aff;
  aff.init(rot, out);
  vector3_t tv(transvec[0], transvec[1], transvec[2]);
  if (!aff.compute((ShapeName)shape, tau, eta, tv, out, plist, 0.0, rot)) return -1;
  for (size_t i = 0; i < out.size(); ++i) {
    ff[2 * i] = out[i].real();
    ff[2 * i + 1] = out[i].imag();
  }
  return (int)out.size();
}

// StructureFactor::compute_structure_factor (lattice sums) on the current grid.
// abc9: the lattice vectors a, b, c (unscaled).  Lattice::construct_vectors is private in the
// reference, so the caller passes the vectors it would produce (src/model/structure.cpp:86-182).
int ref_sf_lattice(const double* abc9, const double* repet, const double* scaling,
                   const double* center, const double* rot9, int gisaxs, double* sf) {
  Lattice lat;
  lat.init();
  lat.type(lattice_null);
  lat.a(abc9[0], abc9[1], abc9[2]);
  lat.b(abc9[3], abc9[4], abc9[5]);
  lat.c(abc9[6], abc9[7], abc9[8]);
  lat.abc_set(true);
  vector3_t sc(scaling[0], scaling[1], scaling[2]);
  StructureFactor s;
  RotMatrix_t rot = make_rot(rot9);
  vector3_t rp(repet[0], repet[1], repet[2]), ce(center[0], center[1], center[2]);
  if (!s.compute_structure_factor(gisaxs ? "gisaxs" : "saxs", ce, &lat, rp, sc, rot, nullptr,
                                  nullptr))
    return -2;
  QGrid& g = QGrid::instance();
  int n = gisaxs ? g.nqz_extended() : g.nqz();
  for (int i = 0; i < n; ++i) {
    sf[2 * i] = s[i].real();
    sf[2 * i + 1] = s[i].imag();
  }
  return n;
}

// StructureFactor::compute_structure_factor, paracrystal branch, on the singleton grid.
int ref_sf_paracrystal(int dims, int lattice, double dx, double dy, double sx, double sy,
                       double dom, int gisaxs, double* sf) {
  auto pc = std::make_shared<Paracrystal>();
  pc->putDims(dims);
  pc->putDistXMean(dx);
  pc->putDistYMean(dy);
  pc->putDistXStddev(sx);
  pc->putDistYStddev(sy);
  pc->putDomainSize(dom);
  Lattice lat;
  lat.init();
  lat.type((LatticeType)lattice);
  StructureFactor s;
  s.putStructureType(paracrystal_type);
  RotMatrix_t rot;
  vector3_t z(0, 0, 0);
  if (!s.compute_structure_factor(gisaxs ? "gisaxs" : "saxs", z, &lat, z, z, rot, pc, nullptr)) return -2;
  QGrid& g = QGrid::instance();
  int n = gisaxs ? g.nqz_extended() : g.nqz();
  for (int i = 0; i < n; ++i) {
    sf[2 * i] = s[i].real();
    sf[2 * i + 1] = s[i].imag();
  }
  return n;
}

// StructureFactor::compute_structure_factor, Percus-Yevick branch, on the singleton grid.
int ref_sf_percus_yevick(double dia, double volf, int dims, int gisaxs, double* sf) {
  auto py = std::make_shared<PercusYevick>();
  py->putDims(dims);
  py->putDiameter(dia);
  py->putVolfract(volf);
  Lattice lat;
  lat.init();
  StructureFactor s;
  s.putStructureType(percusyevick_type);
  RotMatrix_t rot;
  vector3_t z(0, 0, 0);
  if (!s.compute_structure_factor(gisaxs ? "gisaxs" : "saxs", z, &lat, z, z, rot, nullptr, py)) return -2;
  QGrid& g = QGrid::instance();
  int n = gisaxs ? g.nqz_extended() : g.nqz();
  for (int i = 0; i < n; ++i) {
    sf[2 * i] = s[i].real();
    sf[2 * i + 1] = s[i].imag();
  }
  return n;
}

// Convolutions::convolution_gaussian_2d, as HipGISAXS::gaussian_smearing calls it
// (src/sim/hipgisaxs_helpers.cpp:25-27): data of ny rows of nx, replaced in place.
int ref_smear_gaussian(double* data, int nx, int ny, double sigma) {
  real_t* buf = new real_t[(size_t)nx * ny];
  for (size_t i = 0; i < (size_t)nx * ny; ++i) buf[i] = data[i];
  if (!Convolutions::instance().convolution_gaussian_2d(buf, nx, ny, sigma)) return -1;
  for (size_t i = 0; i < (size_t)nx * ny; ++i) data[i] = buf[i];
  delete[] buf;
  return 0;
}

// RotMatrix_t(axis, angle) and products, for the rotation-composition checks.
void ref_rotmatrix(int axis, double angle, double* r9) {
  RotMatrix_t r(axis, angle);
  // RotMatrix_t keeps its data private; recover it by rotating the unit vectors.
  for (int j = 0; j < 3; ++j) {
    vector3_t e(j == 0, j == 1, j == 2);
    vector3_t c = r * e;
    r9[0 * 3 + j] = c[0];
    r9[1 * 3 + j] = c[1];
    r9[2 * 3 + j] = c[2];
  }
}

// The fitter's distance measures, chosen as hgx_fit_distance numbers them: 0 sqrt_unit_l2,
// 1 sqrt_c_l2, 2 cbrt_unit_l2, 3 cbrt_c_l2, 4 sqrt_unit_l2_residual, 5 sqrt_c_l2_residual,
// 6 sqrt_unit_l1, 7 cbrt_unit_l1.  Returns the number of values written to out, -1 on error.
long ref_fit_distance(int metric, long n, const double* ref, const double* dat, const unsigned* mask,
                      double* out) {
  std::unique_ptr<DistanceMeasure> d;
  switch (metric) {
    case 0: d.reset(new SqrtUnitVectorNormL2DistanceSquare()); break;
    case 1: d.reset(new SqrtCNormL2DistanceSquare()); break;
    case 2: d.reset(new CbrtUnitVectorNormL2DistanceSquare()); break;
    case 3: d.reset(new CbrtCNormL2DistanceSquare()); break;
    case 4: d.reset(new SqrtUnitVectorNormL2DistanceSquareResidualVector()); break;
    case 5: d.reset(new SqrtCNormL2DistanceSquareResidualVector()); break;
    case 6: d.reset(new SqrtUnitVectorNormL1Distance()); break;
    case 7: d.reset(new CbrtUnitVectorNormL1Distance()); break;
    default: return -1;
  }
  std::vector<real_t> r(ref, ref + n), x(dat, dat + n);
  std::vector<unsigned> m(n, 1);
  if (mask) m.assign(mask, mask + n);
  real_t* rp = r.data();
  real_t* xp = x.data();
  unsigned* mp = m.data();
  std::vector<real_t> dist;
  if (!(*d)(rp, xp, mp, (unsigned)n, dist)) return -1;
  for (size_t i = 0; i < dist.size(); ++i) out[i] = dist[i];
  return (long)dist.size();
}

// A reference image as the reference reads it: ImageData::read for text files
// (src/analyzer/ImageData.cpp:79-104), EDFReader for .edf (src/file/edf_reader.cpp).
// Returns the value count, -1 when the file cannot be read, -2 when cap is too small.
long ref_read_image(const char* path, int edf, double* data, long cap, int* ncol, int* nrow) {
  std::vector<double> v;
  if (edf) {
    EDFReader r(path);  // exits the process on a file it cannot read: call it on good files only
    real_t* d = nullptr;
    unsigned ny = 0, nz = 0;
    if (!r.get_data(d, ny, nz)) return -1;
    v.assign(d, d + (size_t)ny * nz);
    *ncol = (int)ny;
    *nrow = (int)nz;
  } else {
    ImageData img;
    if (!img.read(path)) return -1;
    v.assign(img.data(), img.data() + img.size());
    *ncol = (int)img.n_par();
    *nrow = (int)img.n_ver();
  }
  if ((long)v.size() > cap) return -2;
  for (size_t i = 0; i < v.size(); ++i) data[i] = v[i];
  return (long)v.size();
}

}  // extern "C"


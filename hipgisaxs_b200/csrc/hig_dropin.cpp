// Method bodies of the reference simulator's GPU classes over the hgx C ABI (see
// include/hgx_hig.hpp).  Compiled into libhgx.so against the standalone declarations; with
// -DHGX_IN_REFERENCE_TREE -I<reference>/include it compiles against the reference's own
// headers and replaces src/ff/gpu/ff_tri_gpu.cu (approx triangle), src/ff/gpu/ff_ana_*_gpu.cu
// and src/sf/gpu/sf_gpu.cu.
//
// The classes keep the reference's synchronous semantics (host vectors in, host vectors
// out).  Device state (one hgx context per device, the q-grid uploaded at init) lives in a
// registry keyed by object address, so the classes' own data members are not used and the
// same file works with either set of declarations.  Errors return false / 0 as the
// reference does and print hgx_last_error() to stderr; nothing calls exit().
//
// Precision: HGX_PRECISION=f64 in the environment selects the plain FP64 kernels; the
// default is the FP32-compensated path (within 1e-5 norm-wise of FP64).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <map>
#include <stdexcept>
#include <string>
#include <mutex>
#include <sstream>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>
#include <sys/stat.h>
#include <time.h>

#include "hgx_hig.hpp"

namespace {

// the current device of the calling thread, as the reference's classes use it
int current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  return dev;
}

std::mutex g_mu;
std::unordered_map<int, hgx_ctx> g_ctx;  // per device

struct GridEntry {
  hgx_qgrid grid = nullptr;
  unsigned nqy = 0, nqz = 0;
  std::vector<std::complex<double>> sf;
};
std::unordered_map<const void*, GridEntry> g_grids;

hgx_ctx context_on(int dev) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_ctx.find(dev);
  if (it != g_ctx.end()) return it->second;
  hgx_ctx c = nullptr;
  if (hgx_create(dev, &c) != HGX_OK) {
    std::cerr << "hgx: " << hgx_last_error() << std::endl;
    return nullptr;
  }
  g_ctx[dev] = c;
  return c;
}

hgx_ctx context() { return context_on(current_device()); }

int precision() {
  const char* p = std::getenv("HGX_PRECISION");
  return (p && std::strcmp(p, "f64") == 0) ? HGX_F64 : HGX_F32C;
}

bool report(int status, const char* where) {
  if (status == HGX_OK) return true;
  std::cerr << "hgx: " << where << ": " << hgx_last_error() << std::endl;
  return false;
}

// RotMatrix_t keeps its 3x3 private: recover it from the images of the unit vectors.
void rot_to_r9(const hig::RotMatrix_t& rot, double* r9) {
  hig::RotMatrix_t r = rot;
  for (int j = 0; j < 3; ++j) {
    hig::vector3_t e(j == 0 ? 1.0 : 0.0, j == 1 ? 1.0 : 0.0, j == 2 ? 1.0 : 0.0);
    hig::vector3_t c = r * e;
    r9[0 * 3 + j] = c[0];
    r9[1 * 3 + j] = c[1];
    r9[2 * 3 + j] = c[2];
  }
}

// Uploads the QGrid singleton (extended qz when nqz > nqy, else the detector qz).
bool upload_grid(const void* owner, unsigned nqy, unsigned nqz) {
  hgx_ctx c = context();
  if (!c) return false;
  hig::QGrid& Q = hig::QGrid::instance();
  if ((int)nqy > Q.nqy()) {
    std::cerr << "hgx: the QGrid holds fewer q-points than requested" << std::endl;
    return false;
  }
  std::vector<double> qx(nqy), qy(nqy), qz(2 * (size_t)nqz);
  for (unsigned i = 0; i < nqy; ++i) {
    qx[i] = Q.qx((int)i);
    qy[i] = Q.qy((int)i);
  }
  const bool ext = nqz > nqy;
  for (unsigned i = 0; i < nqz; ++i) {
    std::complex<double> v = ext ? std::complex<double>(Q.qz_extended((int)i))
                                 : std::complex<double>(Q.qz((int)i), 0.0);
    qz[2 * i] = v.real();
    qz[2 * i + 1] = v.imag();
  }
  hgx_qgrid g = nullptr;
  if (!report(hgx_qgrid_from_arrays(c, (int)nqy, qx.data(), qy.data(), (int)nqz, qz.data(),
                                    Q.ncols(), &g),
              "upload q-grid"))
    return false;
  std::lock_guard<std::mutex> lk(g_mu);
  GridEntry& e = g_grids[owner];
  if (e.grid) hgx_qgrid_destroy(e.grid);
  e.grid = g;
  e.nqy = nqy;
  e.nqz = nqz;
  return true;
}

GridEntry* entry(const void* owner) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_grids.find(owner);
  return it == g_grids.end() ? nullptr : &it->second;
}

void drop(const void* owner) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_grids.find(owner);
  if (it == g_grids.end()) return;
  if (it->second.grid) hgx_qgrid_destroy(it->second.grid);
  g_grids.erase(it);
}

template <typename V>
const double* dptr(const V& v) {
  return v.empty() ? nullptr : v.data();
}

bool analytic(const void* owner, int shape, const std::vector<const std::vector<hig::real_t>*>& dims,
              double tau, double eta, const hig::RotMatrix_t& rot,
              const std::vector<hig::real_t>& transvec, std::vector<hig::complex_t>& ff) {
  GridEntry* e = entry(owner);
  if (!e || !e->grid) {
    hig::QGrid& Q = hig::QGrid::instance();
    if (!upload_grid(owner, Q.nqy(), Q.nqz_extended() > 0 ? Q.nqz_extended() : Q.nqz())) return false;
    e = entry(owner);
  }
  double r9[9];
  rot_to_r9(rot, r9);
  std::vector<double> out(2 * (size_t)e->nqz);
  const std::vector<hig::real_t>* d[8] = {nullptr};
  for (size_t i = 0; i < dims.size() && i < 8; ++i) d[i] = dims[i];
  auto n = [&](int i) { return d[i] ? (int)d[i]->size() : 0; };
  auto p = [&](int i) { return d[i] ? dptr(*d[i]) : nullptr; };
  int s = hgx_ff_analytic(context(), e->grid, shape, n(0), p(0), p(1), n(2), p(2), p(3), n(4), p(4),
                          p(5), n(6), p(6), p(7), tau, eta, transvec.size() >= 3 ? transvec.data() : nullptr,
                          r9, out.data(), HGX_C128);
  if (!report(s, "analytic form factor")) return false;
  ff.resize(e->nqz);
  for (size_t i = 0; i < e->nqz; ++i) ff[i] = hig::complex_t(out[2 * i], out[2 * i + 1]);
  return true;
}

}  // namespace

namespace hig {

#ifndef HGX_IN_REFERENCE_TREE
RotMatrix_t::RotMatrix_t(int axis, real_t a) : RotMatrix_t() {
  real_t c = std::cos(a), s = std::sin(a);
  switch (axis) {  // include/numerics/matrix.hpp:47-69
    case 0: d_[4] = c; d_[5] = -s; d_[7] = s; d_[8] = c; break;
    case 1: d_[0] = c; d_[2] = -s; d_[6] = s; d_[8] = c; break;
    case 2: d_[0] = c; d_[1] = -s; d_[3] = s; d_[4] = c; break;
    default: break;
  }
}
RotMatrix_t RotMatrix_t::operator*(const RotMatrix_t& r) const {
  RotMatrix_t o;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      real_t s = 0;
      for (int k = 0; k < 3; ++k) s += d_[i * 3 + k] * r.d_[j + 3 * k];
      o.d_[i * 3 + j] = s;
    }
  return o;
}
#endif

// --------------------------------------------------------- NumericFormFactorG ----
unsigned int NumericFormFactorG::compute_approx_triangle(std::vector<real_t>& shape_def,
                                                         cucomplex_t*& ff, int nqy, real_t* qx,
                                                         real_t* qy, int nqz, cucomplex_t* qz,
                                                         RotMatrix_t& rot, real_t& kernel_time) {
  hgx_ctx c = context();
  if (!c) return 0;
  size_t nt8 = shape_def.size() / 8;
  std::vector<double> packed;
  const double* sd = shape_def.data();
  if (shape_def.size() % 8 != 0 && shape_def.size() % 7 == 0) {  // 7-value tuples
    size_t nt = shape_def.size() / 7;
    packed.assign(8 * nt, 0.0);
    for (size_t t = 0; t < nt; ++t)
      for (int k = 0; k < 7; ++k) packed[8 * t + k] = shape_def[7 * t + k];
    sd = packed.data();
    nt8 = nt;
  }
  unsigned ntri = (unsigned)nt8;
  if (ntri < 1) return 0;
  double r9[9];
  rot_to_r9(rot, r9);
  ff = new (std::nothrow) cucomplex_t[nqz];
  if (!ff) return 0;
  auto t0 = std::chrono::steady_clock::now();
  int s = hgx_ff_triangles(c, sd, (int)ntri, nqy, qx, qy, nqz, reinterpret_cast<const double*>(qz),
                           r9, precision(), reinterpret_cast<double*>(ff));
  kernel_time = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (!report(s, "compute_approx_triangle")) {
    delete[] ff;
    ff = nullptr;
    return 0;
  }
  return ntri;
}

// The exact triangle form factor (NumericFormFactor::compute2's path): FP64 always, as the
// reference computes it; the triangles are the reference's triangle_t (9 reals each).
unsigned int NumericFormFactorG::compute_exact_triangle(triangle_t* triangles, int num_triangles,
                                                        cucomplex_t*& ff, int nqy, real_t* qx,
                                                        real_t* qy, int nqz, cucomplex_t* qz,
                                                        RotMatrix_t& rot, real_t& kernel_time) {
  hgx_ctx c = context();
  if (!c || !triangles || num_triangles < 1) return 0;
  std::vector<double> tris(9 * (size_t)num_triangles);
  for (int t = 0; t < num_triangles; ++t)
    for (int k = 0; k < 3; ++k) {
      tris[9 * t + k] = triangles[t].v1[k];
      tris[9 * t + 3 + k] = triangles[t].v2[k];
      tris[9 * t + 6 + k] = triangles[t].v3[k];
    }
  double r9[9];
  rot_to_r9(rot, r9);
  ff = new (std::nothrow) cucomplex_t[nqz];
  if (!ff) return 0;
  auto t0 = std::chrono::steady_clock::now();
  int s = hgx_ff_exact_triangles(c, tris.data(), num_triangles, nqy, qx, qy, nqz,
                                 reinterpret_cast<const double*>(qz), r9, reinterpret_cast<double*>(ff));
  kernel_time = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (!report(s, "compute_exact_triangle")) {
    delete[] ff;
    ff = nullptr;
    return 0;
  }
  return (unsigned)num_triangles;
}

// -------------------------------------------------------- AnalyticFormFactorG ----
AnalyticFormFactorG::AnalyticFormFactorG(unsigned int nqy, unsigned int nqz) { init(nqy, nqz); }
AnalyticFormFactorG::AnalyticFormFactorG() {}
AnalyticFormFactorG::~AnalyticFormFactorG() { drop(this); }
bool AnalyticFormFactorG::init(unsigned int nqy, unsigned int nqz) { return upload_grid(this, nqy, nqz); }
bool AnalyticFormFactorG::clear() { return true; }
bool AnalyticFormFactorG::destroy() {
  drop(this);
  return true;
}

bool AnalyticFormFactorG::compute_box(const real_t tau, const real_t eta, const std::vector<real_t>& x,
                                      const std::vector<real_t>& distr_x, const std::vector<real_t>& y,
                                      const std::vector<real_t>& distr_y, const std::vector<real_t>& z,
                                      const std::vector<real_t>& distr_z, const RotMatrix_t& rot,
                                      const std::vector<real_t>& transvec, std::vector<complex_t>& ff) {
  return analytic(this, 2, {&x, &distr_x, &y, &distr_y, &z, &distr_z}, tau, eta, rot, transvec, ff);
}
bool AnalyticFormFactorG::compute_cube(const real_t tau, const real_t eta, const std::vector<real_t>& x,
                                       const std::vector<real_t>& distr_x, const RotMatrix_t& rot,
                                       const std::vector<real_t>& transvec, std::vector<complex_t>& ff) {
  return analytic(this, 3, {&x, &distr_x}, tau, eta, rot, transvec, ff);
}
bool AnalyticFormFactorG::compute_cylinder(const real_t tau, const real_t eta, const std::vector<real_t>& r,
                                           const std::vector<real_t>& distr_r, const std::vector<real_t>& h,
                                           const std::vector<real_t>& distr_h, const RotMatrix_t& rot,
                                           const std::vector<real_t>& transvec, std::vector<complex_t>& ff) {
  return analytic(this, 4, {&r, &distr_r, nullptr, nullptr, &h, &distr_h}, tau, eta, rot, transvec, ff);
}
bool AnalyticFormFactorG::compute_sphere(const std::vector<real_t>& r, const std::vector<real_t>& distr_r,
                                         const std::vector<real_t>& h, const std::vector<real_t>& distr_h,
                                         const RotMatrix_t& rot, const std::vector<real_t>& transvec,
                                         std::vector<complex_t>& ff) {
  return analytic(this, 5, {&r, &distr_r, nullptr, nullptr, &h, &distr_h}, 0.0, 0.0, rot, transvec, ff);
}
bool AnalyticFormFactorG::compute_prism3(const real_t tau, const real_t eta, const std::vector<real_t>& l,
                                         const std::vector<real_t>& distr_l, const std::vector<real_t>& h,
                                         const std::vector<real_t>& distr_h, const RotMatrix_t& rot,
                                         const std::vector<real_t>& transvec, std::vector<complex_t>& ff) {
  return analytic(this, 8, {&l, &distr_l, nullptr, nullptr, &h, &distr_h}, tau, eta, rot, transvec, ff);
}
bool AnalyticFormFactorG::compute_prism6(const real_t tau, const real_t eta, const std::vector<real_t>& l,
                                         const std::vector<real_t>& distr_l, const std::vector<real_t>& h,
                                         const std::vector<real_t>& distr_h, const RotMatrix_t& rot,
                                         const std::vector<real_t>& transvec, std::vector<complex_t>& ff) {
  return analytic(this, 9, {&l, &distr_l, nullptr, nullptr, &h, &distr_h}, tau, eta, rot, transvec, ff);
}
bool AnalyticFormFactorG::compute_pyramid(const real_t tau, const real_t eta, const std::vector<real_t>& x,
                                          const std::vector<real_t>& distr_x, const std::vector<real_t>& y,
                                          const std::vector<real_t>& distr_y, const std::vector<real_t>& h,
                                          const std::vector<real_t>& distr_h, const std::vector<real_t>& b,
                                          const std::vector<real_t>& distr_b, const RotMatrix_t& rot,
                                          const std::vector<real_t>& transvec, std::vector<complex_t>& ff) {
  return analytic(this, 14, {&x, &distr_x, &y, &distr_y, &h, &distr_h, &b, &distr_b}, tau, eta, rot,
                  transvec, ff);
}

// ------------------------------------------------------------ StructureFactorG ----
StructureFactorG::StructureFactorG(unsigned int nqx, unsigned int nqy, unsigned int nqz) {
  init(nqx, nqy, nqz);
}
StructureFactorG::StructureFactorG() {}
StructureFactorG::~StructureFactorG() { drop(this); }
bool StructureFactorG::init(unsigned int, unsigned int nqy, unsigned int nqz) {
  return upload_grid(this, nqy, nqz);
}
bool StructureFactorG::clear() { return true; }
bool StructureFactorG::destroy() {
  drop(this);
  return true;
}

// The lattice structure factor of the reference's CPU class (src/sf/sf.cpp:164-246); the
// reference's GPU class multiplied a basis factor (1 + e^{iq.t}) its CPU class does not have
// (src/sf/gpu/sf_gpu.cu:290-291), which this implementation does not reproduce.
bool StructureFactorG::compute(std::string expt, vector3_t center, Lattice* lattice, vector3_t repet,
                               vector3_t scaling, RotMatrix_t rot) {
  if (!lattice) return false;
  GridEntry* e = entry(this);
  if (!e || !e->grid) {
    hig::QGrid& Q = hig::QGrid::instance();
    unsigned nz = expt == "saxs" ? (unsigned)Q.nqz() : (unsigned)Q.nqz_extended();
    if (!upload_grid(this, Q.nqy(), nz)) return false;
    e = entry(this);
  }
  vector3_t a = lattice->a(), b = lattice->b(), c = lattice->c();
  double abc9[9] = {a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2]};
  double rep[3] = {repet[0], repet[1], repet[2]}, sc[3] = {scaling[0], scaling[1], scaling[2]};
  double ce[3] = {center[0], center[1], center[2]};
  double r9[9];
  rot_to_r9(rot, r9);
  std::vector<double> out(2 * (size_t)e->nqz);
  if (!report(hgx_sf_lattice(context(), e->grid, abc9, rep, sc, ce, r9, out.data(), HGX_C128),
              "structure factor"))
    return false;
  e->sf.resize(e->nqz);
  for (size_t i = 0; i < e->nqz; ++i) e->sf[i] = std::complex<double>(out[2 * i], out[2 * i + 1]);
  return true;
}

void StructureFactorG::get_sf(complex_t*& sf) {
  GridEntry* e = entry(this);
  if (!e || !sf) return;
  for (size_t i = 0; i < e->sf.size(); ++i) sf[i] = complex_t(e->sf[i].real(), e->sf[i].imag());
}

}  // namespace hig

// ------------------------------------------------- HipGISAXSObjectiveFunctionG ----
namespace hig {

struct HipGISAXSObjectiveFunctionG::Impl {
  CylinderLatticeSetup s;
  hgx_ctx ctx = nullptr;  // the per-device context shared with the classes above
  hgx_qgrid grid = nullptr;
  std::vector<double> rowfc, abc9, counts;
  std::vector<unsigned> mask;
  hgx_cyl_batch one = nullptr;  // a single full-detector candidate
  hgx_cyl_batch pop = nullptr;  // the population batch (rebuilt when its size changes)
  int pop_n = 0;
  real_t alpha = 0.0;
  real_vec_t mean;
  bool good = false;

  ~Impl() {
    if (pop) hgx_cyl_batch_destroy(pop);
    if (one) hgx_cyl_batch_destroy(one);
    if (grid) hgx_qgrid_destroy(grid);
  }

  // the 16-double model block of the hgx_cyl_batch functions
  void model(const real_vec_t& x, double* m) const {
    for (int i = 0; i < 16; ++i) m[i] = 0.0;
    m[0] = x[0];
    m[1] = x[1];
    m[2] = x[2];
    m[3] = x[3];
    m[4] = s.spread;
    m[5] = s.spread > 0 ? s.nsamples : 1;
    for (int i = 0; i < 3; ++i) m[6 + i] = s.repet[i];
    m[9] = s.dn2[0];
    m[10] = s.dn2[1];
    for (int i = 0; i < 3; ++i) m[11 + i] = s.center[i];
    m[14] = s.weight;
    m[15] = s.smooth_sampling ? 1.0 : 0.0;
  }

  hgx_cyl_batch make_batch(int n) {
    const long npx = (long)s.nrow * s.ncol;
    std::vector<int> rois(4 * (size_t)n);
    std::vector<double> cnt((size_t)n * npx);
    std::vector<unsigned> msk(mask.empty() ? 0 : (size_t)n * npx);
    for (int i = 0; i < n; ++i) {
      rois[4 * i + 0] = 0;
      rois[4 * i + 1] = 0;
      rois[4 * i + 2] = s.nrow;
      rois[4 * i + 3] = s.ncol;
      std::copy(counts.begin(), counts.end(), cnt.begin() + (size_t)i * npx);
      if (!mask.empty()) std::copy(mask.begin(), mask.end(), msk.begin() + (size_t)i * npx);
    }
    hgx_cyl_batch b = nullptr;
    if (!report(hgx_cyl_batch_create(ctx, grid, rowfc.data(), abc9.data(), n, rois.data(), cnt.data(),
                                     msk.empty() ? nullptr : msk.data(), s.scale,
                                     s.fp64 ? HGX_F64 : HGX_F32C, &b),
                "objective batch"))
      return nullptr;
    return b;
  }

  // regularisation (alpha/2)||x - mean||^2 and its gradient alpha (x - mean)
  real_t reg(const real_vec_t& x, real_vec_t* g) const {
    real_t r = 0.0;
    for (int i = 0; i < 4; ++i) {
      real_t d = x[i] - (mean.size() == 4 ? mean[i] : 0.0);
      r += d * d;
      if (g) (*g)[i] += alpha * d;
    }
    return 0.5 * alpha * r;
  }
};

HipGISAXSObjectiveFunctionG::HipGISAXSObjectiveFunctionG(const CylinderLatticeSetup& setup,
                                                         const std::vector<real_t>& counts,
                                                         const std::vector<unsigned int>& mask)
    : impl_(new Impl()) {
  Impl& m = *impl_;
  m.s = setup;
  const long npx = (long)setup.nrow * setup.ncol;
  if (setup.nrow < 1 || setup.ncol < 1 || (long)counts.size() != npx ||
      (!mask.empty() && (long)mask.size() != npx)) {
    std::cerr << "hgx: objective: counts/mask do not match the detector size" << std::endl;
    return;
  }
  m.ctx = context();
  if (!m.ctx) return;
  const double pi = 3.141592653589793;
  const double k0 = 2 * pi / (1.23984 / setup.energy_kev);  // src/sim/hipgisaxs_main.cpp:144-158
  const double ai = setup.alpha_i_deg * pi / 180.0;
  if (!report(hgx_qgrid_create(m.ctx, setup.ncol, setup.nrow, setup.qy_min, setup.qz_min, setup.qy_max,
                               setup.qz_max, ai, k0, 0.0, 0.0, &m.grid),
              "objective q-grid"))
    return;
  const double delta = setup.substrate_delta, beta = setup.substrate_beta, thick = 0.0;
  const int order = -1;
  m.rowfc.assign(8 * (size_t)setup.nrow, 0.0);
  if (!report(hgx_propagation_coeffs(m.ctx, m.grid, 1, &delta, &beta, &thick, &order, k0, ai, 0, nullptr,
                                     m.rowfc.data(), 1),
              "objective Fresnel coefficients"))
    return;
  const int type = setup.lattice == "cubic" ? 3 : setup.lattice == "hex" ? 7 : -1;
  if (type < 0) {
    std::cerr << "hgx: objective: lattice must be hex or cubic" << std::endl;
    return;
  }
  m.abc9.assign(9, 0.0);
  if (!report(hgx_lattice_vectors(type, "100", m.abc9.data(), nullptr), "objective lattice")) return;
  m.counts = counts;
  m.mask = mask;
  m.one = m.make_batch(1);
  m.good = m.one != nullptr;
}

HipGISAXSObjectiveFunctionG::~HipGISAXSObjectiveFunctionG() { delete impl_; }

bool HipGISAXSObjectiveFunctionG::ok() const { return impl_->good; }

std::vector<std::string> HipGISAXSObjectiveFunctionG::fit_param_keys() const {
  return {"radius", "height", "lattice_a", "phi"};
}

bool HipGISAXSObjectiveFunctionG::set_regularization(real_t alpha) {
  impl_->alpha = alpha;
  return true;
}

bool HipGISAXSObjectiveFunctionG::set_param_mean(const real_vec_t& mean) {
  if (mean.size() != 4) return false;
  impl_->mean = mean;
  return true;
}

unsigned int HipGISAXSObjectiveFunctionG::data_size() const {
  return (unsigned)(impl_->s.nrow * impl_->s.ncol);
}

bool HipGISAXSObjectiveFunctionG::value_and_gradient(const real_vec_t& x, real_t& f, real_vec_t& g) {
  Impl& m = *impl_;
  if (!m.good || x.size() != 4) return false;
  double mb[16], out[5];
  m.model(x, mb);
  if (!report(hgx_cyl_batch_eval(m.one, mb, out), "objective value_and_gradient")) return false;
  g.assign(out + 1, out + 5);
  f = out[0] + m.reg(x, &g);
  return true;
}

real_vec_t HipGISAXSObjectiveFunctionG::operator()(const real_vec_t& x) {
  real_t f = 0.0;
  real_vec_t g;
  if (!value_and_gradient(x, f, g) || !std::isfinite(f)) f = 1e8;  // the reference's stand-in
  return real_vec_t(1, f);
}

bool HipGISAXSObjectiveFunctionG::evaluate(const std::vector<real_vec_t>& population, real_vec_t& f,
                                           std::vector<real_vec_t>& g) {
  Impl& m = *impl_;
  const int n = (int)population.size();
  if (!m.good || n < 1) return false;
  for (const auto& x : population)
    if (x.size() != 4) return false;
  if (m.pop_n != n) {
    if (m.pop) hgx_cyl_batch_destroy(m.pop);
    m.pop = m.make_batch(n);
    m.pop_n = m.pop ? n : 0;
    if (!m.pop) return false;
  }
  std::vector<double> mb(16 * (size_t)n), out(5 * (size_t)n);
  for (int i = 0; i < n; ++i) m.model(population[i], mb.data() + 16 * i);
  if (!report(hgx_cyl_batch_eval(m.pop, mb.data(), out.data()), "objective evaluate")) return false;
  f.resize(n);
  g.assign(n, real_vec_t());
  for (int i = 0; i < n; ++i) {
    g[i].assign(out.begin() + 5 * i + 1, out.begin() + 5 * i + 5);
    f[i] = out[5 * i] + m.reg(population[i], &g[i]);
  }
  return true;
}

bool HipGISAXSObjectiveFunctionG::simulate(const real_vec_t& x, real_vec_t& intensity) {
  Impl& m = *impl_;
  if (!m.good || x.size() != 4) return false;
  double mb[16];
  m.model(x, mb);
  intensity.assign((size_t)m.s.nrow * m.s.ncol, 0.0);
  return report(hgx_cyl_batch_forward(m.one, mb, intensity.data()), "objective simulate");
}

}  // namespace hig

// ------------------------------------------------------------------- HipGISAXSG ----
namespace hig {

struct HipGISAXSG::Impl {
  int device = 0;
  std::string outdir;
  hgx_ctx ctx = nullptr;
  hgx_hig h = nullptr;
  int nrow = 0, ncol = 0;
  double k0 = 0.0;
  bool ready = false;
  std::string err;

  ~Impl() {
    if (h) hgx_hig_destroy(h);
  }
  bool check(int status, const char* where) {
    if (status == HGX_OK) return true;
    err = hgx_last_error();
    std::cerr << "hgx: " << where << ": " << err << std::endl;
    return false;
  }
  bool refuse(const std::string& msg) {
    err = msg;
    std::cerr << "hgx: " << msg << std::endl;
    return false;
  }
  // the fit parameters in key order (HiGInput::fit_param_keys and its parallel lists)
  struct Param {
    std::string key, variable;
    double range[3], init;
  };
  std::vector<Param> params() const {
    std::vector<Param> out;
    int n = 0;
    if (!h || hgx_hig_fit_count(h, &n) != HGX_OK) return out;
    for (int i = 0; i < n; ++i) {
      char key[512], var[1024];
      Param p;
      if (hgx_hig_fit_param(h, i, key, sizeof(key), var, sizeof(var), p.range, &p.init) != HGX_OK) break;
      p.key = key;
      p.variable = var;
      out.push_back(p);
    }
    return out;
  }
};

HipGISAXSG::HipGISAXSG(int device) : impl_(new Impl) { impl_->device = device; }
HipGISAXSG::~HipGISAXSG() { delete impl_; }

bool HipGISAXSG::construct_input(const char* filename) {
  if (impl_->h) hgx_hig_destroy(impl_->h);
  impl_->h = nullptr;
  impl_->ready = false;
  if (!filename) return impl_->refuse("construct_input: no file name");
  return impl_->check(hgx_hig_read(filename, &impl_->h), "construct_input");
}

// HipGISAXS::init (src/sim/hipgisaxs_main.cpp): the beam and the detector image's size; the
// q-grid and Fresnel coefficients are built on the device by the first compute_gisaxs
bool HipGISAXSG::init() {
  Impl& m = *impl_;
  if (!m.h) return m.refuse("init: no input (construct_input first)");
  double ai = 0.0, fr = 0.0;
  if (!m.check(hgx_hig_beam(m.h, &m.k0, &ai, &fr), "init")) return false;
  if (!m.check(hgx_hig_image_size(m.h, &m.nrow, &m.ncol), "init")) return false;
  m.ctx = context_on(m.device);
  if (!m.ctx) return m.refuse(std::string("init: no device context: ") + hgx_last_error());
  m.ready = true;
  return true;
}

bool HipGISAXSG::compute_gisaxs(real_t*& final_data) {
  Impl& m = *impl_;
  if (!m.ready && !init()) return false;
  if (!m.check(hgx_hig_image_size(m.h, &m.nrow, &m.ncol), "compute_gisaxs")) return false;
  const size_t n = (size_t)m.nrow * m.ncol;
  bool owned = false;
  if (!final_data) {
    final_data = new (std::nothrow) real_t[n];
    if (!final_data) return m.refuse("compute_gisaxs: out of host memory");
    owned = true;
  }
  static_assert(sizeof(real_t) == sizeof(double), "the HiG simulation computes in double");
  if (!m.check(hgx_hig_compute_gisaxs(m.ctx, m.h, precision(), reinterpret_cast<double*>(final_data)),
               "compute_gisaxs")) {
    if (owned) {
      delete[] final_data;
      final_data = nullptr;
    }
    return false;
  }
  return true;
}

// HiGInput::update_params (src/config/hig_input.cpp:2712-2830): fit keys -> values; an
// unknown key throws std::out_of_range, as the reference's map lookup does
bool HipGISAXSG::update_params(const std::map<std::string, real_t>& values) {
  Impl& m = *impl_;
  if (!m.h) return m.refuse("update_params: no input");
  const std::vector<Impl::Param> ps = m.params();
  for (const auto& kv : values) {
    const Impl::Param* p = nullptr;
    for (const auto& q : ps)
      if (q.key == kv.first) p = &q;
    if (!p) throw std::out_of_range("update_params: no fit parameter with key '" + kv.first + "'");
    if (!m.check(hgx_hig_update_param(m.h, p->variable.c_str(), kv.second), "update_params")) return false;
  }
  return true;
}

bool HipGISAXSG::update_param(const std::string& variable, real_t value) {
  Impl& m = *impl_;
  if (!m.h) return m.refuse("update_param: no input");
  return m.check(hgx_hig_update_param(m.h, variable.c_str(), value), "update_param");
}

bool HipGISAXSG::gaussian_smearing(real_t*& data, real_t sigma) {
  Impl& m = *impl_;
  if (!m.ready && !init()) return false;
  return m.check(hgx_gaussian_smearing(m.ctx, reinterpret_cast<double*>(data), m.ncol, m.nrow, sigma),
                 "gaussian_smearing");
}

bool HipGISAXSG::normalize(real_t*& data, unsigned int size) {
  Impl& m = *impl_;
  if (!m.ready && !init()) return false;
  int done = 0;
  if (!m.check(hgx_normalize(m.ctx, reinterpret_cast<double*>(data), (long)size, &done), "normalize"))
    return false;
  return done != 0;  // false when max - min < 1e-30, as in the reference
}

bool HipGISAXSG::save_gisaxs(real_t* final_data, std::string filename) {
  Impl& m = *impl_;
  if (!m.ready && !init()) return false;
  return m.check(hgx_save_gisaxs(m.ctx, reinterpret_cast<const double*>(final_data), m.nrow, m.ncol,
                                 filename.c_str()),
                 "save_gisaxs");
}

namespace {
// ComputeParams::timestamp (src/model/compute_params.cpp:68-78)
std::string run_timestamp() {
  time_t raw;
  time(&raw);
  char buf[16];
  strftime(buf, sizeof(buf), "%Y%m%d_%H%M%S", localtime(&raw));
  return buf;
}
// a value as std::stringstream << writes it (6 significant digits), for the file names
std::string angle_text(double v) {
  std::ostringstream o;
  o << v;
  return o.str();
}
}  // namespace

// HipGISAXS::init's output directory and run_all_gisaxs's loops (src/sim/hipgisaxs_main.cpp:
// 160-170, 283-613); each point is hgx_hig_compute_scan_point, the sums run in point order
bool HipGISAXSG::run_all_gisaxs(int, int, int) {
  Impl& m = *impl_;
  if (!init()) return false;
  char prefix[4096], run[4096];
  if (!m.check(hgx_hig_output_names(m.h, prefix, sizeof(prefix), run, sizeof(run)), "run_all_gisaxs")) return false;
  const std::string rn = run[0] ? std::string(run) + "_" + run_timestamp() : "run_" + run_timestamp();
  m.outdir = std::string(prefix) + "/" + rn;
  if (mkdir(m.outdir.c_str(), 0755) != 0) return m.refuse("run_all_gisaxs: could not create output directory " + m.outdir);
  int na = 0, np = 0, nt = 0;
  if (!m.check(hgx_hig_scan_size(m.h, &na, &np, &nt), "run_all_gisaxs")) return false;
  const size_t n = (size_t)m.nrow * m.ncol;
  std::vector<double> img(n), sum(n);
  int p = 0;
  for (int i = 0; i < na; ++i) {
    double a = 0.0;
    std::fill(sum.begin(), sum.end(), 0.0);
    for (int j = 0; j < np; ++j)
      for (int k = 0; k < nt; ++k, ++p) {
        double f = 0.0, t = 0.0;
        if (!m.check(hgx_hig_scan_point(m.h, p, &a, &f, &t), "run_all_gisaxs")) return false;
        if (!m.check(hgx_hig_compute_scan_point(m.ctx, m.h, precision(), p, img.data()), "run_all_gisaxs"))
          return false;
        const std::string name = m.outdir + "/gisaxs_ai=" + angle_text(a) + "_rot=" + angle_text(f) + "_tilt=" +
                                 angle_text(t) + ".out";
        if (!m.check(hgx_save_gisaxs(m.ctx, img.data(), m.nrow, m.ncol, name.c_str()), "run_all_gisaxs"))
          return false;
        if (np > 1 || nt > 1)
          for (size_t q = 0; q < n; ++q) sum[q] = sum[q] + img[q];
      }
    if ((np > 1 || nt > 1) && np * nt > 0) {
      const std::string name = m.outdir + "/gisaxs_ai=" + angle_text(a) + "_averaged.out";
      if (!m.check(hgx_save_gisaxs(m.ctx, sum.data(), m.nrow, m.ncol, name.c_str()), "run_all_gisaxs"))
        return false;
    }
  }
  return true;
}

const std::string& HipGISAXSG::output_dir() const { return impl_->outdir; }

unsigned int HipGISAXSG::nrow() const { return (unsigned)impl_->nrow; }
unsigned int HipGISAXSG::ncol() const { return (unsigned)impl_->ncol; }
real_t HipGISAXSG::k0() const { return impl_->k0; }
const char* HipGISAXSG::last_error() const { return impl_->err.c_str(); }

std::vector<std::string> HipGISAXSG::fit_param_keys() const {
  std::vector<std::string> keys;
  for (const auto& p : impl_->params()) keys.push_back(p.key);
  return keys;
}

// ------------------------------------------------------- HiGObjectiveFunctionG ----
struct HiGObjectiveFunctionG::Impl {
  HipGISAXSG sim;
  unsigned n_par = 0, n_ver = 0;
  int metric = -1;
  real_t alpha = 0.0;
  std::vector<double> ref;
  std::vector<unsigned> mask;  // empty: every pixel
  bool good = false;
  explicit Impl(int device) : sim(device) {}
};

namespace {
const char* const kMetricNames[] = {"sqrt_unit_l2", "sqrt_c_l2", "cbrt_unit_l2", "cbrt_c_l2",
                                    "sqrt_unit_l2_residual", "sqrt_c_l2_residual", "sqrt_unit_l1",
                                    "cbrt_unit_l1"};
}  // namespace

HiGObjectiveFunctionG::HiGObjectiveFunctionG(const char* hig_file, int device) : impl_(new Impl(device)) {
  Impl& m = *impl_;
  if (!m.sim.construct_input(hig_file) || !m.sim.init()) return;
  m.n_par = m.sim.ncol();
  m.n_ver = m.sim.nrow();
  int nalg = 0;
  if (hgx_hig_fit_algorithm_count(m.sim.impl_->h, &nalg) == HGX_OK && nalg > 0)
    hgx_hig_fit_algorithm(m.sim.impl_->h, 0, nullptr, 0, &m.metric, nullptr, nullptr);
  // set_mean_data: every fit parameter at the middle of its range (the image the reference
  // computes there is not used by its operator(), so it is not computed here)
  std::map<std::string, real_t> mean;
  for (const auto& p : m.sim.impl_->params()) mean[p.key] = (p.range[1] - p.range[0]) / 2.0 + p.range[0];
  if (!m.sim.update_params(mean)) return;
  m.good = true;
}

HiGObjectiveFunctionG::~HiGObjectiveFunctionG() { delete impl_; }

bool HiGObjectiveFunctionG::ok() const { return impl_->good; }

// HipGISAXSObjectiveFunction::set_reference_data, read_mask_data, read_edf_mask_data
// (src/analyzer/objective_func_hipgisaxs.cpp:116-205)
bool HiGObjectiveFunctionG::set_reference_data(int i) {
  Impl& m = *impl_;
  HipGISAXSG::Impl& s = *m.sim.impl_;
  if (!m.good) return s.refuse("set_reference_data: the objective did not initialise");
  char path[4096], maskp[4096];
  if (!s.check(hgx_hig_fit_reference(s.h, i, path, sizeof(path), maskp, sizeof(maskp), nullptr, nullptr),
               "set_reference_data"))
    return false;
  long count = 0;
  int nc = 0, nr = 0;
  if (!s.check(hgx_read_image(path, nullptr, 0, &count, &nc, &nr), "set_reference_data")) return false;
  std::vector<double> img((size_t)std::max(count, 1L));
  if (!s.check(hgx_read_image(path, img.data(), (long)img.size(), &count, &nc, &nr), "set_reference_data"))
    return false;
  if ((unsigned)nc != m.n_par || (unsigned)nr != m.n_ver) {
    // the reference warns and re-grids its simulation to the image (override_qregion)
    std::cerr << "hgx: set_reference_data: the reference image is " << nc << " x " << nr
              << ", the simulation " << m.n_par << " x " << m.n_ver
              << "; the simulation takes the reference data's region" << std::endl;
    if (!s.check(hgx_hig_override_qregion(s.h, nc, nr, i), "set_reference_data")) return false;
    if (!s.check(hgx_hig_image_size(s.h, &s.nrow, &s.ncol), "set_reference_data")) return false;
    m.n_par = (unsigned)nc;
    m.n_ver = (unsigned)nr;
  }
  const size_t n = (size_t)m.n_par * m.n_ver;
  img.resize(n);  // a text image may carry a last, uncounted row
  std::vector<unsigned> msk;
  const std::string mp = maskp;
  if (!mp.empty()) {  // EDF or text by the extension, as the reference reads it
    long mc = 0;
    if (!s.check(hgx_read_mask(mp.c_str(), nullptr, 0, &mc), "set_reference_data")) return false;
    msk.resize((size_t)std::max(mc, 1L));
    if (!s.check(hgx_read_mask(mp.c_str(), msk.data(), (long)msk.size(), &mc), "set_reference_data")) return false;
    msk.resize((size_t)mc);
    if (msk.size() != n)
      return s.refuse("set_reference_data: mask and reference data sizes differ (" + std::to_string(n) +
                      " != " + std::to_string(msk.size()) + ")");
  }
  m.ref.swap(img);
  m.mask.swap(msk);
  return true;
}

bool HiGObjectiveFunctionG::set_reference_data(const real_vec_t& ref, const std::vector<unsigned int>& mask) {
  Impl& m = *impl_;
  const size_t n = (size_t)m.n_par * m.n_ver;
  if (!m.good) return m.sim.impl_->refuse("set_reference_data: the objective did not initialise");
  if (ref.size() != n || (!mask.empty() && mask.size() != n))
    return m.sim.impl_->refuse("set_reference_data: " + std::to_string(n) + " values expected");
  m.ref.assign(ref.begin(), ref.end());
  m.mask.assign(mask.begin(), mask.end());
  return true;
}

// simulate_and_set_ref (src/analyzer/objective_func_hipgisaxs.cpp:336-374); the mask is kept
bool HiGObjectiveFunctionG::simulate_and_set_ref(const real_vec_t& x) {
  Impl& m = *impl_;
  if (!m.good) return m.sim.impl_->refuse("simulate_and_set_ref: the objective did not initialise");
  if (!x.empty()) {
    const std::vector<std::string> keys = m.sim.fit_param_keys();
    if (x.size() > keys.size()) return m.sim.impl_->refuse("simulate_and_set_ref: more values than fit parameters");
    std::map<std::string, real_t> vals;
    for (size_t i = 0; i < x.size(); ++i) vals[keys[i]] = x[i];
    if (!m.sim.update_params(vals)) return false;
  }
  std::vector<real_t> img((size_t)m.n_par * m.n_ver);
  real_t* p = img.data();
  if (!m.sim.compute_gisaxs(p)) return false;
  m.ref.assign(img.begin(), img.end());
  return true;
}

bool HiGObjectiveFunctionG::set_distance_metric(const std::string& name) {
  for (int k = 0; k < 8; ++k)
    if (name == kMetricNames[k]) {
      impl_->metric = k;
      return true;
    }
  return impl_->sim.impl_->refuse("set_distance_metric: unknown metric '" + name + "'");
}

bool HiGObjectiveFunctionG::set_regularization(real_t alpha) {
  impl_->alpha = alpha;
  return true;
}

// operator() (src/analyzer/objective_func_hipgisaxs.cpp:263-334) through hgx_hig_objective
real_vec_t HiGObjectiveFunctionG::operator()(const real_vec_t& x) {
  Impl& m = *impl_;
  HipGISAXSG::Impl& s = *m.sim.impl_;
  if (!m.good) {
    s.refuse("operator(): the objective did not initialise");
    return real_vec_t();
  }
  if (m.ref.empty()) {
    s.refuse("operator(): no reference data (set_reference_data first)");
    return real_vec_t();
  }
  if (m.metric < 0) {
    s.refuse("operator(): no distance metric (none in the fitting block; set_distance_metric)");
    return real_vec_t();
  }
  std::vector<double> xd(x.begin(), x.end());
  std::vector<double> dist((size_t)m.n_par * m.n_ver);
  long nd = 0;
  if (!s.check(hgx_hig_objective(s.ctx, s.h, xd.data(), (int)xd.size(), m.ref.data(),
                                 m.mask.empty() ? nullptr : m.mask.data(), m.metric, m.alpha, dist.data(), &nd),
               "operator()"))
    return real_vec_t();
  return real_vec_t(dist.begin(), dist.begin() + nd);
}

bool HiGObjectiveFunctionG::value_and_gradient(const real_vec_t& x, real_t& f, real_vec_t& g) {
  Impl& m = *impl_;
  HipGISAXSG::Impl& s = *m.sim.impl_;
  if (!m.good || m.ref.empty() || m.metric < 0) {
    s.refuse("value_and_gradient(): the objective has no reference data or distance metric");
    return false;
  }
  std::vector<double> xd(x.begin(), x.end()), gd(x.size());
  double dist = 0.0;
  if (!s.check(hgx_hig_objective_grad(s.ctx, s.h, xd.data(), (int)xd.size(), m.ref.data(),
                                      m.mask.empty() ? nullptr : m.mask.data(), m.metric, m.alpha, &dist,
                                      gd.data()),
               "value_and_gradient()"))
    return false;
  f = dist;
  g.assign(gd.begin(), gd.end());
  return true;
}

bool HiGObjectiveFunctionG::evaluate_population(const std::vector<real_vec_t>& X, real_vec_t& dist) {
  Impl& m = *impl_;
  HipGISAXSG::Impl& s = *m.sim.impl_;
  if (!m.good || m.ref.empty() || m.metric < 0) {
    s.refuse("evaluate_population(): the objective has no reference data or distance metric");
    return false;
  }
  if (X.empty()) {
    s.refuse("evaluate_population(): empty population");
    return false;
  }
  const size_t nx = s.params().size();
  std::vector<double> xs;
  for (const real_vec_t& x : X) {
    if (x.size() != nx) {
      s.refuse("evaluate_population(): each candidate needs one value per fit parameter");
      return false;
    }
    xs.insert(xs.end(), x.begin(), x.end());
  }
  hgx_hig_pop pop = nullptr;
  if (!s.check(hgx_hig_population_create(s.ctx, s.h, (int)X.size(), m.ref.data(),
                                         m.mask.empty() ? nullptr : m.mask.data(), m.metric, m.alpha,
                                         HGX_F64, &pop),
               "evaluate_population()"))
    return false;
  std::vector<double> d(X.size());
  const bool good = s.check(hgx_hig_population_eval(pop, xs.data(), (int)nx, d.data()), "evaluate_population()");
  hgx_hig_population_destroy(pop);
  if (!good) return false;
  dist.assign(d.begin(), d.end());
  return true;
}

int HiGObjectiveFunctionG::num_fit_params() const { return (int)impl_->sim.impl_->params().size(); }

std::vector<std::string> HiGObjectiveFunctionG::fit_param_keys() const { return impl_->sim.fit_param_keys(); }

std::vector<std::pair<real_t, real_t>> HiGObjectiveFunctionG::fit_param_limits() const {
  std::vector<std::pair<real_t, real_t>> out;
  for (const auto& p : impl_->sim.impl_->params()) out.emplace_back(p.range[0], p.range[1]);
  return out;
}

real_vec_t HiGObjectiveFunctionG::fit_param_step_values() const {
  real_vec_t out;
  for (const auto& p : impl_->sim.impl_->params()) out.push_back(p.range[2]);
  return out;
}

real_vec_t HiGObjectiveFunctionG::fit_param_init_values() const {
  real_vec_t out;
  for (const auto& p : impl_->sim.impl_->params()) out.push_back(p.init);
  return out;
}

// HiGInput::param_space_mean (include/config/hig_input.hpp:322-325); an unknown key throws
// std::out_of_range as the reference's map lookup does
real_t HiGObjectiveFunctionG::param_space_mean(const std::string& key) const {
  for (const auto& p : impl_->sim.impl_->params())
    if (p.key == key) return (p.range[1] - p.range[0]) / 2.0 + p.range[0];
  throw std::out_of_range("param_space_mean: no fit parameter with key '" + key + "'");
}

real_t HiGObjectiveFunctionG::analysis_tolerance(int n) const {
  double t = 0.0;
  hgx_hig_fit_algorithm(impl_->sim.impl_->h, n, nullptr, 0, nullptr, &t, nullptr);
  return t;
}

real_t HiGObjectiveFunctionG::analysis_regularization(int n) const {
  double r = 0.0;
  hgx_hig_fit_algorithm(impl_->sim.impl_->h, n, nullptr, 0, nullptr, nullptr, &r);
  return r;
}

unsigned int HiGObjectiveFunctionG::n_par() const { return impl_->n_par; }
unsigned int HiGObjectiveFunctionG::n_ver() const { return impl_->n_ver; }
unsigned int HiGObjectiveFunctionG::data_size() const { return impl_->n_par * impl_->n_ver; }
HipGISAXSG& HiGObjectiveFunctionG::simulator() { return impl_->sim; }

}  // namespace hig

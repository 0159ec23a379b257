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
#include <mutex>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

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

hgx_ctx context() {
  const int dev = current_device();
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

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
#include <chrono>
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

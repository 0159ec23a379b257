// hgx_hig.hpp — the reference simulator's GPU classes (NumericFormFactorG,
// AnalyticFormFactorG, StructureFactorG; tacaswell/hipgisaxs) with their method signatures,
// implemented over the hgx C ABI (hipgisaxs_b200/csrc/hig_dropin.cpp).
//
// Built inside the reference tree (-DHGX_IN_REFERENCE_TREE -I<reference>/include), the
// reference's own headers declare the classes and types and hig_dropin.cpp supplies the
// method bodies in place of src/ff/gpu/ff_tri_gpu.cu, src/ff/gpu/ff_ana_*_gpu.cu and
// src/sf/gpu/sf_gpu.cu.  Built standalone (the default), this header declares the same
// classes over minimal stand-ins for the reference types it uses (real_t, complex_t,
// cucomplex_t, vector3_t, RotMatrix_t, Lattice and the QGrid singleton).
#ifndef HGX_HIG_HPP
#define HGX_HIG_HPP

#include <complex>
#include <string>
#include <vector>

#include "hgx.h"

#ifdef HGX_IN_REFERENCE_TREE
#include <common/typedefs.hpp>
#include <ff/gpu/ff_ana_gpu.cuh>
#include <ff/gpu/ff_num_gpu.cuh>
#include <model/qgrid.hpp>
#include <model/structure.hpp>
#include <numerics/matrix.hpp>
#include <sf/gpu/sf_gpu.cuh>
#else

namespace hig {

typedef double real_t;                    // include/common/typedefs.hpp:47-65 (DOUBLEP)
typedef std::complex<real_t> complex_t;
struct cucomplex_t {                      // layout of cuDoubleComplex
  double x, y;
};

struct vector3_t {                        // include/common/globals.hpp:68-...
  real_t vec_[3];
  vector3_t() : vec_{0, 0, 0} {}
  vector3_t(real_t a, real_t b, real_t c) : vec_{a, b, c} {}
  real_t& operator[](int i) { return vec_[i]; }
  real_t operator[](int i) const { return vec_[i]; }
};

class RotMatrix_t {                       // include/numerics/matrix.hpp:30-140
 public:
  RotMatrix_t() : d_{1, 0, 0, 0, 1, 0, 0, 0, 1} {}
  RotMatrix_t(int axis, real_t angle);
  RotMatrix_t(const vector3_t& a, const vector3_t& b, const vector3_t& c)
      : d_{a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2]} {}
  RotMatrix_t operator*(const RotMatrix_t& r) const;
  vector3_t operator*(const vector3_t& v) const {
    return vector3_t(d_[0] * v[0] + d_[1] * v[1] + d_[2] * v[2],
                     d_[3] * v[0] + d_[4] * v[1] + d_[5] * v[2],
                     d_[6] * v[0] + d_[7] * v[1] + d_[8] * v[2]);
  }

 private:
  real_t d_[9];
};

class Lattice {                           // include/model/structure.hpp:88-148 (vectors only)
 public:
  Lattice(const vector3_t& a, const vector3_t& b, const vector3_t& c) : a_(a), b_(b), c_(c) {}
  vector3_t a() const { return a_; }
  vector3_t b() const { return b_; }
  vector3_t c() const { return c_; }

 private:
  vector3_t a_, b_, c_;
};

// The QGrid singleton's accessors the GPU classes read (include/model/qgrid.hpp:27-122),
// filled by set() in standalone use.
class QGrid {
 public:
  static QGrid& instance() {
    static QGrid g;
    return g;
  }
  void set(int nrow, int ncol, const std::vector<real_t>& qx, const std::vector<real_t>& qy,
           const std::vector<real_t>& qz, const std::vector<complex_t>& qz_extended) {
    nrow_ = nrow;
    ncol_ = ncol;
    qx_ = qx;
    qy_ = qy;
    qz_ = qz;
    qz_extended_ = qz_extended;
  }
  int nqx() const { return (int)qx_.size(); }
  int nqy() const { return (int)qy_.size(); }
  int nqz() const { return (int)qz_.size(); }
  int nqz_extended() const { return (int)qz_extended_.size(); }
  int nrows() const { return nrow_; }
  int ncols() const { return ncol_; }
  real_t qx(int i) const { return qx_[i]; }
  real_t qy(int i) const { return qy_[i]; }
  real_t qz(int i) const { return qz_[i]; }
  complex_t qz_extended(int i) const { return qz_extended_[i]; }

 private:
  int nrow_ = 0, ncol_ = 0;
  std::vector<real_t> qx_, qy_, qz_;
  std::vector<complex_t> qz_extended_;
};

// include/ff/gpu/ff_num_gpu.cuh:34-140 (the approx-triangle entry points)
class NumericFormFactorG {
 public:
  NumericFormFactorG(int block_cuda) : block_cuda_(block_cuda) {}
  NumericFormFactorG(int, int, int) {}
  NumericFormFactorG() {}
  ~NumericFormFactorG() {}
  unsigned int compute_approx_triangle(std::vector<real_t>& shape_def, cucomplex_t*& ff, int nqy,
                                       real_t* qx, real_t* qy, int nqz, cucomplex_t* qz,
                                       RotMatrix_t& rot, real_t& kernel_time);

 private:
  int block_cuda_ = 0;
};

// include/ff/gpu/ff_ana_gpu.cuh:28-96
class AnalyticFormFactorG {
 public:
  AnalyticFormFactorG(unsigned int nqy, unsigned int nqz);
  AnalyticFormFactorG();
  ~AnalyticFormFactorG();
  bool init(unsigned int nqy, unsigned int nqz);
  bool clear();
  bool destroy();
  bool compute_box(const real_t tau, const real_t eta, const std::vector<real_t>& x,
                   const std::vector<real_t>& distr_x, const std::vector<real_t>& y,
                   const std::vector<real_t>& distr_y, const std::vector<real_t>& z,
                   const std::vector<real_t>& distr_z, const RotMatrix_t& rot,
                   const std::vector<real_t>& transvec, std::vector<complex_t>& ff);
  bool compute_cube(const real_t tau, const real_t eta, const std::vector<real_t>& x,
                    const std::vector<real_t>& distr_x, const RotMatrix_t& rot,
                    const std::vector<real_t>& transvec, std::vector<complex_t>& ff);
  bool compute_cylinder(const real_t tau, const real_t eta, const std::vector<real_t>& r,
                        const std::vector<real_t>& distr_r, const std::vector<real_t>& h,
                        const std::vector<real_t>& distr_h, const RotMatrix_t& rot,
                        const std::vector<real_t>& transvec, std::vector<complex_t>& ff);
  bool compute_sphere(const std::vector<real_t>& r, const std::vector<real_t>& distr_r,
                      const std::vector<real_t>& h, const std::vector<real_t>& distr_h,
                      const RotMatrix_t& rot, const std::vector<real_t>& transvec,
                      std::vector<complex_t>& ff);
  bool compute_prism3(const real_t tau, const real_t eta, const std::vector<real_t>& l,
                      const std::vector<real_t>& distr_l, const std::vector<real_t>& h,
                      const std::vector<real_t>& distr_h, const RotMatrix_t& rot,
                      const std::vector<real_t>& transvec, std::vector<complex_t>& ff);
  bool compute_prism6(const real_t tau, const real_t eta, const std::vector<real_t>& l,
                      const std::vector<real_t>& distr_l, const std::vector<real_t>& h,
                      const std::vector<real_t>& distr_h, const RotMatrix_t& rot,
                      const std::vector<real_t>& transvec, std::vector<complex_t>& ff);
  bool compute_pyramid(const real_t tau, const real_t eta, const std::vector<real_t>& x,
                       const std::vector<real_t>& distr_x, const std::vector<real_t>& y,
                       const std::vector<real_t>& distr_y, const std::vector<real_t>& h,
                       const std::vector<real_t>& distr_h, const std::vector<real_t>& b,
                       const std::vector<real_t>& distr_b, const RotMatrix_t& rot,
                       const std::vector<real_t>& transvec, std::vector<complex_t>& ff);
  // not implemented by the reference either (its CPU dispatcher never calls them)
  bool compute_prism3x() { return false; }
  bool compute_sawtooth_up() { return false; }
  bool compute_sawtooth_down() { return false; }
  bool compute_truncated_cone() { return false; }

 private:
  unsigned int nqy_ = 0, nqz_ = 0;
};

// include/sf/gpu/sf_gpu.cuh:34-67
class StructureFactorG {
 public:
  StructureFactorG(unsigned int nqx, unsigned int nqy, unsigned int nqz);
  StructureFactorG();
  ~StructureFactorG();
  bool init(unsigned int nqx, unsigned int nqy, unsigned int nqz);
  bool clear();
  bool destroy();
  void get_sf(complex_t*& sf);
  bool compute(std::string expt, vector3_t center, Lattice* lattice, vector3_t repet,
               vector3_t scaling, RotMatrix_t rot);

 private:
  unsigned int nqx_ = 0, nqy_ = 0, nqz_ = 0;
  std::vector<complex_t> sf_;
};

}  // namespace hig
#endif  // HGX_IN_REFERENCE_TREE
#endif  // HGX_HIG_HPP

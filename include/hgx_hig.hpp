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
#include <map>
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
typedef std::vector<real_t> real_vec_t;   // include/common/typedefs.hpp:66
typedef struct Triangle {                 // include/common/typedefs.hpp:102-106
  real_t v1[3];
  real_t v2[3];
  real_t v3[3];
} triangle_t;
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
  unsigned int compute_exact_triangle(triangle_t* triangles, int num_triangles, cucomplex_t*& ff,
                                      int nqy, real_t* qx, real_t* qy, int nqz, cucomplex_t* qz,
                                      RotMatrix_t& rot, real_t& kernel_time);
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

namespace hig {

// ---------------------------------------------------------- fitting front end ----
// The objective of the reference's fitters (HipGISAXSObjectiveFunction,
// include/analyzer/objective_func_hipgisaxs.hpp; operator() at
// src/analyzer/objective_func_hipgisaxs.cpp:245-333) for one model family — cylinders on a
// 2-D lattice over a substrate, in DWBA — evaluated on the GPU, with the two calls the
// reference's fitters lack: the gradient by a hand-written adjoint (in place of LMVM's
// central differences, src/analyzer/hipgisaxs_fit_lmvm.cpp:190-223) and a whole population
// in one graph-captured launch (in place of PSO's one-particle-at-a-time loop,
// src/analyzer/hipgisaxs_fit_pso.cpp:521-545).  A new class: the reference's own
// HipGISAXSObjectiveFunction reads a HiG file and runs the full simulator.
//
// Fit parameters x = (radius, height, lattice constant, in-plane rotation phi [radians]).
// Distance: chi^2 = sum mask (scale I(x) - counts)^2 / max(counts, 1), plus the reference's
// regularisation (alpha/2) ||x - x_mean||^2 (objective_func_hipgisaxs.cpp:296-311).
struct CylinderLatticeSetup {
  int ncol = 1024, nrow = 1024;                       // detector pixels
  real_t qy_min = -2.0, qz_min = 0.0, qy_max = 2.0, qz_max = 3.0;  // 1/nm
  real_t alpha_i_deg = 0.20, energy_kev = 10.0;
  real_t substrate_delta = 4.88e-6, substrate_beta = 7.37e-8;
  std::string lattice = "hex";                        // "hex" or "cubic" (a, b in the plane)
  real_t repet[3] = {20, 20, 1};
  real_t spread = 0.05;                               // relative Gaussian size spread
  int nsamples = 11;                                  // size samples over +-3 spread
  bool smooth_sampling = true;                        // evenly spaced samples (smooth chi^2)
  real_t dn2[2] = {-2 * 4.88e-6, -2 * 7.37e-8};       // particle contrast (complex)
  real_t center[3] = {0, 0, 0};
  real_t weight = 1.0;
  real_t scale = 1.0;                                 // model-to-counts factor of the chi^2
  bool fp64 = false;                                  // plain FP64 instead of FP32C
};

class HipGISAXSObjectiveFunctionG {
 public:
  // counts: nrow x ncol measured image (row 0 = top, as QGrid orders rows); mask: same
  // size of 0/1, or empty for none.
  HipGISAXSObjectiveFunctionG(const CylinderLatticeSetup& setup, const std::vector<real_t>& counts,
                              const std::vector<unsigned int>& mask = std::vector<unsigned int>());
  ~HipGISAXSObjectiveFunctionG();
  HipGISAXSObjectiveFunctionG(const HipGISAXSObjectiveFunctionG&) = delete;
  HipGISAXSObjectiveFunctionG& operator=(const HipGISAXSObjectiveFunctionG&) = delete;

  bool ok() const;                                    // false when set-up failed
  // the reference's call: the distance vector (one element: chi^2 + regularisation); a
  // non-finite distance becomes 1e8 as in the reference
  real_vec_t operator()(const real_vec_t& x);
  // distance and its gradient with respect to x
  bool value_and_gradient(const real_vec_t& x, real_t& f, real_vec_t& g);
  // distances and gradients of a population in one launch
  bool evaluate(const std::vector<real_vec_t>& population, real_vec_t& f,
                std::vector<real_vec_t>& g);
  // the model image at x (nrow x ncol)
  bool simulate(const real_vec_t& x, real_vec_t& intensity);

  int num_fit_params() const { return 4; }
  std::vector<std::string> fit_param_keys() const;
  bool set_regularization(real_t alpha);
  bool set_param_mean(const real_vec_t& mean);        // x_mean of the regularisation
  unsigned int data_size() const;

 private:
  struct Impl;
  Impl* impl_;
};


// --------------------------------------------------------- HiG-driven simulation ----
// HipGISAXS (include/sim/hipgisaxs_main.hpp, src/sim/hipgisaxs_main.cpp) for the path built
// here: read a HiG description, simulate it on the GPU (hgx_hig_compute_gisaxs), update
// parameters, post-process.  The method names are the reference's; the class name carries the
// G of the GPU classes so that it can sit beside the reference's own HipGISAXS.
class HipGISAXSG {
 public:
  explicit HipGISAXSG(int device = 0);
  ~HipGISAXSG();
  HipGISAXSG(const HipGISAXSG&) = delete;
  HipGISAXSG& operator=(const HipGISAXSG&) = delete;

  bool construct_input(const char* filename);        // HiGInput::construct_input_config
  bool init();                                       // beam and q-grid (HipGISAXS::init)
  // the nrow x ncol image of all structures; `final_data` is allocated with new[] when NULL
  bool compute_gisaxs(real_t*& final_data);
  bool update_params(const std::map<std::string, real_t>& params);  // fit keys -> values
  bool update_param(const std::string& variable, real_t value);      // a variable name
  bool gaussian_smearing(real_t*& data, real_t sigma);               // in place
  bool normalize(real_t*& data, unsigned int size);                  // in place
  bool save_gisaxs(real_t* final_data, std::string filename);        // the .out text
  // the main simulation program's run (HipGISAXS::run_all_gisaxs): every alpha_i x phi x tilt
  // of the scattering block, each image written as output_dir()/gisaxs_ai=<a>_rot=<phi>_tilt=<t>.out
  // and, per alpha_i with more than one phi or tilt, their sum as gisaxs_ai=<a>_averaged.out;
  // output_dir() = pathprefix/runname_<timestamp>, created here (the .tif images of the
  // reference's image writer are not written)
  bool run_all_gisaxs(int x_min = 0, int x_max = 0, int x_step = 0);
  const std::string& output_dir() const;
  unsigned int nrow() const;
  unsigned int ncol() const;
  real_t k0() const;
  std::vector<std::string> fit_param_keys() const;
  const char* last_error() const;                    // the library's message after a false

 private:
  struct Impl;
  Impl* impl_;
  friend class HiGObjectiveFunctionG;
};

// HipGISAXSObjectiveFunction (src/analyzer/objective_func_hipgisaxs.cpp,
// include/analyzer/objective_func_hipgisaxs.hpp) for a HiG file: the fitting block's parameters
// (key order), its reference data and mask (read by extension as the reference reads them),
// the distance metric of its first algorithm, the regularisation.  As in the reference, the
// constructor sets every fit parameter to the middle of its range (set_mean_data) and the
// regularisation starts at 0; operator() returns one distance, or one per pixel for the
// residual metrics, each plus its share of (alpha/2)|x - mean|^2 (a non-finite one becomes 1e8).
class HiGObjectiveFunctionG {
 public:
  HiGObjectiveFunctionG(const char* hig_file, int device = 0);
  ~HiGObjectiveFunctionG();
  HiGObjectiveFunctionG(const HiGObjectiveFunctionG&) = delete;
  HiGObjectiveFunctionG& operator=(const HiGObjectiveFunctionG&) = delete;

  bool ok() const;
  // the fitting block's reference data and mask (i = 0); an image whose size differs from the
  // detector's re-grids the simulation to it over the block's fit region (override_qregion)
  bool set_reference_data(int i);
  bool set_reference_data(const real_vec_t& ref, const std::vector<unsigned int>& mask);
  bool simulate_and_set_ref(const real_vec_t& x);    // the simulation at x as the reference
  bool set_distance_metric(const std::string& name);  // sqrt_unit_l2, sqrt_c_l2, ...
  bool set_regularization(real_t alpha);
  real_vec_t operator()(const real_vec_t& x);        // empty on failure
  // the scalar objective (operator()'s one distance; not the residual metrics) and its
  // gradient by the simulation's tangent (hgx_hig_objective_grad), where the reference's LMVM
  // fitter takes two simulations per parameter; false on failure
  bool value_and_gradient(const real_vec_t& x, real_t& f, real_vec_t& g);
  // the scalar objective of every candidate of a population (the particle loop of the
  // reference's PSO fitter, src/analyzer/hipgisaxs_fit_pso.cpp:521-545) in one batched
  // evaluation (hgx_hig_population_*; a caller that evaluates many generations keeps a
  // population handle of the C ABI, whose graph is then replayed); false on failure
  bool evaluate_population(const std::vector<real_vec_t>& X, real_vec_t& dist);
  int num_fit_params() const;
  std::vector<std::string> fit_param_keys() const;
  std::vector<std::pair<real_t, real_t>> fit_param_limits() const;
  real_vec_t fit_param_step_values() const;
  real_vec_t fit_param_init_values() const;
  real_t param_space_mean(const std::string& key) const;
  real_t analysis_tolerance(int n) const;
  real_t analysis_regularization(int n) const;
  unsigned int n_par() const;                        // detector columns
  unsigned int n_ver() const;                        // detector rows
  unsigned int data_size() const;
  HipGISAXSG& simulator();

 private:
  struct Impl;
  Impl* impl_;
};

}  // namespace hig
#endif  // HGX_HIG_HPP

// Drives hig::HipGISAXSG and hig::HiGObjectiveFunctionG (include/hgx_hig.hpp) the way the
// reference's simulator and HiG fitter drive HipGISAXS and HipGISAXSObjectiveFunction.
// argv[1]: a HiG file whose fitting block has the keys radius, spacing, twist and whose
// referencedata path (and mask, when given) lie in the working directory.  Writes, in the
// working directory:
//   meta.txt      nrow ncol k0, the fit keys, limits, steps, inits and range middles,
//                 the first algorithm's tolerance and regularization, and "throws" when
//                 update_params refused an unknown key with std::out_of_range
//   sim0.bin      compute_gisaxs of the file as read
//   sim1.bin      after update_params {radius 5, spacing 25, twist 12}; sim1.out its .out text
//   norm.bin      sim1 normalised; smear.bin  sim1 smeared with sigma 1.5
//   dist0.bin     the objective at x = (4.2, 21, 3) against the file's reference data
//   dist1.bin     the same with regularization 0.5
//   dist2.bin     the same with the sqrt_c_l2_residual metric (one value per pixel)
//   dist3.bin     sqrt_unit_l2 after simulate_and_set_ref(5, 25, 12), at (5, 25, 12)
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "hgx_hig.hpp"

static bool save(const std::string& path, const double* v, size_t n) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const bool ok = std::fwrite(v, sizeof(double), n, f) == n;
  std::fclose(f);
  return ok;
}

// argv[2] == "regrid": only the objective, whose reference image differs in size from the
// detector; writes regrid.txt (n_par n_ver after set_reference_data) and dist_regrid.bin at
// x = (4.2, 21, 3).
static int regrid(const char* hig_file) {
  hig::HiGObjectiveFunctionG obj(hig_file);
  if (!obj.ok()) return 20;
  const unsigned np0 = obj.n_par(), nv0 = obj.n_ver();
  if (!obj.set_reference_data(0)) return 21;
  hig::real_vec_t d = obj({4.2, 21.0, 3.0});
  if (d.empty() || !save("dist_regrid.bin", d.data(), d.size())) return 22;
  std::ofstream f("regrid.txt");
  f << np0 << " " << nv0 << " " << obj.n_par() << " " << obj.n_ver() << " " << obj.simulator().ncol() << " "
    << obj.simulator().nrow() << "\n";
  return 0;
}

// argv[2] == "scan": HipGISAXSG::run_all_gisaxs of the file, the C library's rand() seeded with 1
// after the device context exists; writes scan.txt with the output directory
static int scan(const char* hig_file) {
  hig::HipGISAXSG sim(0);
  if (!sim.construct_input(hig_file) || !sim.init()) return 30;
  srand(1);
  if (!sim.run_all_gisaxs()) return 31;
  std::ofstream f("scan.txt");
  f << sim.output_dir() << "\n";
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  if (argc > 2 && std::string(argv[2]) == "regrid") return regrid(argv[1]);
  if (argc > 2 && std::string(argv[2]) == "scan") return scan(argv[1]);
  hig::HipGISAXSG sim(0);
  if (!sim.construct_input(argv[1]) || !sim.init()) return 3;
  const size_t n = (size_t)sim.nrow() * sim.ncol();
  std::ofstream meta("meta.txt");
  meta.precision(17);
  meta << sim.nrow() << " " << sim.ncol() << " " << sim.k0() << "\n";

  hig::real_t* img = nullptr;
  if (!sim.compute_gisaxs(img) || !save("sim0.bin", img, n)) return 4;
  std::map<std::string, hig::real_t> vals = {{"radius", 5.0}, {"spacing", 25.0}, {"twist", 12.0}};
  if (!sim.update_params(vals) || !sim.compute_gisaxs(img) || !save("sim1.bin", img, n)) return 5;
  if (!sim.save_gisaxs(img, "sim1.out")) return 6;
  try {
    sim.update_params({{"no_such_key", 1.0}});
  } catch (const std::out_of_range&) {
    meta << "throws\n";
  }
  std::vector<hig::real_t> work(img, img + n);
  hig::real_t* w = work.data();
  if (!sim.normalize(w, (unsigned)n) || !save("norm.bin", w, n)) return 7;
  work.assign(img, img + n);
  if (!sim.gaussian_smearing(w, 1.5) || !save("smear.bin", w, n)) return 8;
  delete[] img;

  hig::HiGObjectiveFunctionG obj(argv[1]);
  if (!obj.ok()) return 9;
  const std::vector<std::string> keys = obj.fit_param_keys();
  for (const auto& k : keys) meta << k << " ";
  meta << "\n";
  for (const auto& l : obj.fit_param_limits()) meta << l.first << " " << l.second << " ";
  meta << "\n";
  for (double s : obj.fit_param_step_values()) meta << s << " ";
  meta << "\n";
  for (double s : obj.fit_param_init_values()) meta << s << " ";
  meta << "\n";
  for (const auto& k : keys) meta << obj.param_space_mean(k) << " ";
  meta << "\n" << obj.analysis_tolerance(0) << " " << obj.analysis_regularization(0) << "\n";
  meta << obj.n_par() << " " << obj.n_ver() << " " << obj.data_size() << " " << obj.num_fit_params() << "\n";
  meta.close();

  if (!obj.set_reference_data(0)) return 10;
  const hig::real_vec_t x = {4.2, 21.0, 3.0};
  hig::real_vec_t d = obj(x);
  if (d.empty() || !save("dist0.bin", d.data(), d.size())) return 11;
  obj.set_regularization(0.5);
  d = obj(x);
  if (d.empty() || !save("dist1.bin", d.data(), d.size())) return 12;
  {  // a population of two candidates: each the operator() value of its row
    const std::vector<hig::real_vec_t> X = {x, {4.0, 20.0, 2.5}};
    hig::real_vec_t pd;
    if (!obj.evaluate_population(X, pd) || pd.size() != 2) return 18;
    const hig::real_vec_t d1 = obj(X[1]);
    if (d1.empty() || std::fabs(pd[0] - d[0]) > 1e-12 * std::fabs(d[0]) ||
        std::fabs(pd[1] - d1[0]) > 1e-12 * std::fabs(d1[0]))
      return 19;
  }
  if (!obj.set_distance_metric("sqrt_c_l2_residual")) return 13;
  d = obj(x);
  if (d.size() != n || !save("dist2.bin", d.data(), d.size())) return 14;
  obj.set_regularization(0.0);
  if (!obj.set_distance_metric("sqrt_unit_l2") || !obj.simulate_and_set_ref({5.0, 25.0, 12.0})) return 15;
  d = obj({5.0, 25.0, 12.0});
  if (d.empty() || !save("dist3.bin", d.data(), d.size())) return 16;
  if (obj.set_distance_metric("l2")) return 17;  // an unknown metric is refused
  return 0;
}

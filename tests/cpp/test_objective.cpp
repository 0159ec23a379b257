// Drives hig::HipGISAXSObjectiveFunctionG (include/hgx_hig.hpp) the way the reference's
// fitters drive HipGISAXSObjectiveFunction: operator(), plus value_and_gradient and the
// batched evaluate.  argv[1]: a directory holding meta.bin (nrow, ncol, scale as doubles),
// counts.bin (nrow*ncol doubles) and x.bin (4 x npop doubles: population, first row = x0);
// writes value_grad.bin (5 doubles), op.bin (1 double), pop.bin (5 x npop doubles) and
// image.bin (nrow*ncol doubles at x0).
#include <cstdio>
#include <string>
#include <vector>

#include "hgx_hig.hpp"

static std::vector<double> load(const std::string& path) {
  std::vector<double> v;
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return v;
  double x;
  while (std::fread(&x, sizeof(double), 1, f) == 1) v.push_back(x);
  std::fclose(f);
  return v;
}

static bool save(const std::string& path, const std::vector<double>& v) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  bool ok = std::fwrite(v.data(), sizeof(double), v.size(), f) == v.size();
  std::fclose(f);
  return ok;
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string d = argv[1];
  std::vector<double> meta = load(d + "/meta.bin"), counts = load(d + "/counts.bin"),
                      xs = load(d + "/x.bin");
  if (meta.size() != 3 || xs.size() < 4 || xs.size() % 4) return 3;
  hig::CylinderLatticeSetup s;
  s.nrow = (int)meta[0];
  s.ncol = (int)meta[1];
  s.scale = meta[2];
  hig::HipGISAXSObjectiveFunctionG obj(s, counts);
  if (!obj.ok() || obj.num_fit_params() != 4 || obj.data_size() != counts.size()) return 4;
  std::vector<hig::real_vec_t> pop;
  for (size_t i = 0; i < xs.size(); i += 4) pop.push_back(hig::real_vec_t(xs.begin() + i, xs.begin() + i + 4));
  double f = 0;
  hig::real_vec_t g;
  if (!obj.value_and_gradient(pop[0], f, g) || g.size() != 4) return 5;
  std::vector<double> vg{f, g[0], g[1], g[2], g[3]};
  hig::real_vec_t dist = obj(pop[0]);
  if (dist.size() != 1) return 6;
  hig::real_vec_t fp;
  std::vector<hig::real_vec_t> gp;
  if (!obj.evaluate(pop, fp, gp) || fp.size() != pop.size()) return 7;
  std::vector<double> po;
  for (size_t i = 0; i < pop.size(); ++i) {
    po.push_back(fp[i]);
    for (int k = 0; k < 4; ++k) po.push_back(gp[i][k]);
  }
  hig::real_vec_t img;
  if (!obj.simulate(pop[0], img)) return 8;
  // regularisation: (alpha/2)||x - mean||^2 on top of the same chi^2
  obj.set_regularization(2.0);
  obj.set_param_mean({5.0, 10.0, 20.0, 0.0});
  double fr = 0;
  hig::real_vec_t gr;
  if (!obj.value_and_gradient(pop[0], fr, gr)) return 9;
  vg.push_back(fr);
  for (int k = 0; k < 4; ++k) vg.push_back(gr[k]);
  if (!save(d + "/value_grad.bin", vg) || !save(d + "/op.bin", dist) || !save(d + "/pop.bin", po) ||
      !save(d + "/image.bin", img))
    return 10;
  std::printf("ok\n");
  return 0;
}

// Exercises the drop-in GPU classes with the reference simulator's signatures:
// NumericFormFactorG::compute_approx_triangle and compute_exact_triangle, AnalyticFormFactorG (init + compute_cylinder,
// compute_sphere), StructureFactorG (init, compute, get_sf).  Reads raw inputs from a
// directory, writes raw outputs there; tests/test_gpu_dropin.py compares them with the oracle.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "hgx_hig.hpp"

using namespace hig;

static std::vector<double> load(const std::string& path) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) {
    std::cerr << "missing " << path << std::endl;
    std::exit(2);
  }
  size_t n = (size_t)f.tellg() / sizeof(double);
  std::vector<double> v(n);
  f.seekg(0);
  f.read(reinterpret_cast<char*>(v.data()), n * sizeof(double));
  return v;
}

static void save(const std::string& path, const double* p, size_t n) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(p), n * sizeof(double));
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  std::string d = argv[1];
  std::vector<double> meta = load(d + "/meta.bin");  // nrow, ncol
  int nrow = (int)meta[0], ncol = (int)meta[1], n = nrow * ncol;
  std::vector<double> qx = load(d + "/qx.bin"), qy = load(d + "/qy.bin"), qz = load(d + "/qz.bin");
  std::vector<double> ext = load(d + "/qz_ext.bin");
  std::vector<complex_t> qzc(4 * (size_t)n);
  for (size_t i = 0; i < qzc.size(); ++i) qzc[i] = complex_t(ext[2 * i], ext[2 * i + 1]);
  QGrid::instance().set(nrow, ncol, qx, qy, qz, qzc);

  RotMatrix_t rot = RotMatrix_t(2, 0.3) * RotMatrix_t(0, 0.1);

  // numeric form factor through the reference-shaped call
  std::vector<double> sd = load(d + "/shape_def.bin");
  NumericFormFactorG nff(64);
  cucomplex_t* ff = nullptr;
  real_t t = 0;
  unsigned nt = nff.compute_approx_triangle(sd, ff, n, qx.data(), qy.data(), 4 * n,
                                            reinterpret_cast<cucomplex_t*>(ext.data()), rot, t);
  if (nt != sd.size() / 8 || !ff) return 3;
  save(d + "/out_ff_tri.bin", reinterpret_cast<double*>(ff), 8 * (size_t)n);
  delete[] ff;

  // exact triangle form factor (triangle_t vertex triples)
  std::vector<double> tv9 = load(d + "/tris.bin");
  std::vector<triangle_t> tris(tv9.size() / 9);
  for (size_t k = 0; k < tris.size(); ++k)
    for (int j = 0; j < 3; ++j) {
      tris[k].v1[j] = tv9[9 * k + j];
      tris[k].v2[j] = tv9[9 * k + 3 + j];
      tris[k].v3[j] = tv9[9 * k + 6 + j];
    }
  cucomplex_t* ffe = nullptr;
  unsigned ne = nff.compute_exact_triangle(tris.data(), (int)tris.size(), ffe, n, qx.data(), qy.data(),
                                           4 * n, reinterpret_cast<cucomplex_t*>(ext.data()), rot, t);
  if (ne != tris.size() || !ffe) return 9;
  save(d + "/out_ff_exact.bin", reinterpret_cast<double*>(ffe), 8 * (size_t)n);
  delete[] ffe;

  // analytic cylinder and sphere
  AnalyticFormFactorG aff;
  if (!aff.init(n, 4 * n)) return 4;
  std::vector<real_t> r = {4.5, 5.0, 5.5}, wr = {1, 1, 1}, h = {9.0, 10.0}, wh = {1, 1};
  std::vector<real_t> tv = {0.5, -1.0, 2.0};
  std::vector<complex_t> cyl, sph;
  if (!aff.compute_cylinder(0.0, 0.0, r, wr, h, wh, rot, tv, cyl)) return 5;
  std::vector<real_t> rs = {9.0, 10.0}, ws = {0.4, 0.6}, none;
  if (!aff.compute_sphere(rs, ws, none, none, rot, tv, sph)) return 6;
  save(d + "/out_cyl.bin", reinterpret_cast<double*>(cyl.data()), 8 * (size_t)n);
  save(d + "/out_sph.bin", reinterpret_cast<double*>(sph.data()), 8 * (size_t)n);

  // lattice structure factor
  StructureFactorG sfg;
  if (!sfg.init(n, n, 4 * n)) return 7;
  Lattice lat(vector3_t(1, 0, 0), vector3_t(0.5, 0.8660254037844386, 0), vector3_t(0, 0, 1));
  if (!sfg.compute("gisaxs", vector3_t(1, 2, 3), &lat, vector3_t(20, 20, 1), vector3_t(20, 20, 20), rot))
    return 8;
  std::vector<complex_t> sf(4 * (size_t)n);
  complex_t* sp = sf.data();
  sfg.get_sf(sp);
  save(d + "/out_sf.bin", reinterpret_cast<double*>(sf.data()), 8 * (size_t)n);
  std::printf("ok %u triangles, kernel %.3f ms\n", nt, t);
  return 0;
}

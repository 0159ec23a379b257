// Test infrastructure (checker only): reads a HiG file with the reference's own reader
// (HiGInput::construct_input_config, src/config/hig_input.cpp:61-104) and writes the object
// model it built as JSON, in the layout of the product's reader (hgx_hig_json), so that the
// two can be compared field by field.  Compiled into oracle/_ref/libhigref.so by
// oracle/Makefile; never part of the product.
//
// The reference keeps most of its fields private to the classes that its reader is a friend
// of; this translation unit alone opens them to read them.
#include <cstdio>
#include <cstring>
#include <iostream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#define private public
#define protected public
#include <config/hig_input.hpp>
#undef private
#undef protected

namespace {

using namespace hig;

std::string shape_name(ShapeName n) {  // include/common/enums.hpp:24-43 -> keyword
  switch (n) {
    case shape_box: return "box";
    case shape_cube: return "cube";
    case shape_cylinder: return "cylinder";
    case shape_sphere: return "sphere";
    case shape_trunccone: return "trunccone";
    case shape_prism3: return "prism3";
    case shape_prism6: return "prism6";
    case shape_prism3x: return "prism3x";
    case shape_sawtooth: return "sawtooth";
    case shape_random_cylinders: return "randcylinders";
    case shape_horizontal_cylinder: return "hcylinder";
    case shape_pyramid: return "pyramid";
    case shape_custom: return "custom";
    case shape_null: return "null";
    default: return "error";
  }
}
std::string param_name(ShapeParamType t) {
  switch (t) {
    case param_radius: return "radius";
    case param_xsize: return "xsize";
    case param_ysize: return "ysize";
    case param_height: return "height";
    case param_edge: return "edge";
    case param_baseangle: return "baseangle";
    case param_null: return "null";
    default: return "error";
  }
}
std::string stat_name(StatisticType s) {
  switch (s) {
    case stat_none: return "none";
    case stat_cauchy: return "cauchy";
    case stat_gaussian: return "gaussian";
    case stat_random: return "random";
    case stat_range: return "range";
    case stat_t: return "t";
    case stat_uniform: return "uniform";
    case stat_null: return "null";
    default: return "error";
  }
}
std::string lattice_name(LatticeType t) {
  switch (t) {
    case lattice_bcc: return "bcc";
    case lattice_cubic: return "cubic";
    case lattice_fcc: return "fcc";
    case lattice_fco: return "fco";
    case lattice_hcp: return "hcp";
    case lattice_hex: return "hex";
    case lattice_null: return "null";
    default: return "error";
  }
}
std::string region_name(OutputRegionType t) {
  switch (t) {
    case region_angles: return "angles";
    case region_pixels: return "pixels";
    case region_qspace: return "qspace";
    case region_null: return "null";
    default: return "error";
  }
}
std::string corr_name(StructCorrelationType t) {
  switch (t) {
    case structcorr_null: return "null";
    case structcorr_nGnE: return "nGnE";
    case structcorr_nGE: return "nGE";
    case structcorr_GnE: return "GnE";
    case structcorr_GE: return "GE";
    default: return "error";
  }
}
std::string algo_name(FittingAlgorithmName n) {
  switch (n) {
    case algo_null: return "null";
    case algo_pounders: return "pounders";
    case algo_pso: return "pso";
    case algo_lmvm: return "lmvm";
    case algo_bruteforce: return "bruteforce";
    case algo_none_pounders: return "none_pounders";
    default: return "error";
  }
}
std::string algo_param_name(FitAlgorithmParamType t) {
  switch (t) {
    case algo_param_null: return "null";
    case algo_pounders_param_delta: return "pounders_delta";
    case algo_pso_param_omega: return "pso_omega";
    case algo_pso_param_phi1: return "pso_phi1";
    case algo_pso_param_phi2: return "pso_phi2";
    case algo_pso_param_nparticle: return "pso_num_particles";
    case algo_pso_param_ngen: return "pso_num_generations";
    case algo_pso_param_tune_omega: return "pso_tune_omega";
    case algo_pso_param_type: return "pso_type";
    default: return "error";
  }
}
std::string metric_name(FittingDistanceMetric m) {
  switch (m) {
    case metric_sqrt_unit_norm_l1: return "sqrt_unit_l1";
    case metric_sqrt_unit_norm_l2: return "sqrt_unit_l2";
    case metric_sqrt_c_norm_l2: return "sqrt_c_l2";
    case metric_cbrt_unit_norm_l1: return "cbrt_unit_l1";
    case metric_cbrt_unit_norm_l2: return "cbrt_unit_l2";
    case metric_cbrt_c_norm_l2: return "cbrt_c_l2";
    case metric_sqrt_unit_norm_l1_residual: return "sqrt_unit_l1_residual";
    case metric_sqrt_unit_norm_l2_residual: return "sqrt_unit_l2_residual";
    case metric_sqrt_c_norm_l2_residual: return "sqrt_c_l2_residual";
    case metric_null: return "null";
    default: return "error";
  }
}

struct J {
  std::string s;
  void num(double v) {
    char b[40];
    snprintf(b, sizeof b, "%.17g", v);
    s += b;
  }
  void str(const std::string& v) {
    s += '"';
    for (char c : v) {
      if (c == '"' || c == '\\') { s += '\\'; s += c; }
      else s += c;
    }
    s += '"';
  }
  void key(const std::string& k) { str(k); s += ": "; }
  void v3(vector3_t v) { s += '['; num(v[0]); s += ", "; num(v[1]); s += ", "; num(v[2]); s += ']'; }
  void v2(vector2_t v) { s += '['; num(v[0]); s += ", "; num(v[1]); s += ']'; }
  void c() { s += ", "; }
};

std::string dump(HiGInput& in) {
  J j;
  j.s += '{';
  // shapes, sorted by key
  std::map<std::string, Shape*> shapes;
  for (auto& kv : in.shapes_) shapes[kv.first] = &kv.second;
  j.key("shapes"); j.s += '{';
  bool first = true;
  for (auto& kv : shapes) {
    if (!first) j.c();
    first = false;
    Shape& s = *kv.second;
    j.key(kv.first); j.s += '{';
    j.key("name"); j.str(shape_name(s.name_)); j.c();
    j.key("name_str"); j.str(s.name_str_); j.c();
    j.key("originvec"); j.v3(s.originvec_); j.c();
    j.key("rot"); j.v3(vector3_t(s.zrot_, s.yrot_, s.xrot_)); j.c();
    j.key("refindex"); j.v2(vector2_t(s.refindex_.delta(), s.refindex_.beta())); j.c();
    j.key("params"); j.s += '{';
    std::map<std::string, ShapeParam*> params;
    for (auto& p : s.params_) params[p.first] = &p.second;
    bool f2 = true;
    for (auto& pk : params) {
      if (!f2) j.c();
      f2 = false;
      ShapeParam& p = *pk.second;
      j.key(pk.first); j.s += '{';
      j.key("type"); j.str(param_name(p.type_)); j.c();
      j.key("stat"); j.str(stat_name(p.stat_)); j.c();
      j.key("min"); j.num(p.min_); j.c();
      j.key("max"); j.num(p.max_); j.c();
      j.key("p1"); j.num(p.p1_); j.c();
      j.key("p2"); j.num(p.p2_); j.c();
      j.key("nvalues"); j.num(p.nvalues_);
      j.s += '}';
    }
    j.s += "}}";
  }
  j.s += '}'; j.c();
  // layers (std::map by order)
  j.key("layers"); j.s += '{';
  first = true;
  for (auto& kv : in.layers_) {
    if (!first) j.c();
    first = false;
    Layer& l = kv.second;
    j.key(std::to_string(kv.first)); j.s += '{';
    j.key("key"); j.str(l.key_); j.c();
    j.key("order"); j.num(l.order_); j.c();
    j.key("thickness"); j.num(l.thickness_); j.c();
    j.key("refindex"); j.v2(vector2_t(l.refindex_.delta(), l.refindex_.beta()));
    j.s += '}';
  }
  j.s += '}'; j.c();
  j.key("layer_keys"); j.s += '{';
  std::map<std::string, int> lkeys(in.layer_key_map_.begin(), in.layer_key_map_.end());
  first = true;
  for (auto& kv : lkeys) {
    if (!first) j.c();
    first = false;
    j.key(kv.first); j.num(kv.second);
  }
  j.s += '}'; j.c();
  // unit cells
  std::map<std::string, Unitcell*> ucs;
  for (auto& kv : in.unitcells_) ucs[kv.first] = &kv.second;
  j.key("unitcells"); j.s += '{';
  first = true;
  for (auto& kv : ucs) {
    if (!first) j.c();
    first = false;
    j.key(kv.first); j.s += '{';
    std::map<std::string, std::vector<vector3_t>*> els;
    for (auto& e : kv.second->elements_) els[e.first] = &e.second;
    bool f2 = true;
    for (auto& e : els) {
      if (!f2) j.c();
      f2 = false;
      j.key(e.first); j.s += '[';
      for (size_t i = 0; i < e.second->size(); ++i) { if (i) j.c(); j.v3((*e.second)[i]); }
      j.s += ']';
    }
    j.s += '}';
  }
  j.s += '}'; j.c();
  // structures
  std::map<std::string, Structure*> sts;
  for (auto& kv : in.structures_) sts[kv.first] = &kv.second;
  j.key("structures"); j.s += '{';
  first = true;
  for (auto& kv : sts) {
    if (!first) j.c();
    first = false;
    Structure& s = *kv.second;
    Grain& g = s.grain_;
    Lattice& L = g.lattice_;
    j.key(kv.first); j.s += '{';
    j.key("iratio"); j.num(s.iratio_); j.c();
    const char* tname = s.type_ == paracrystal_type ? "paracrystal"
                        : s.type_ == percusyevick_type ? "percusyevick" : "default";
    j.key("type"); j.str(tname); j.c();
    j.key("unitcell_key"); j.str(g.unitcell_key_); j.c();
    j.key("layer_key"); j.str(g.layer_key_); j.c();
    j.key("layer_order"); j.num(g.layer_order_); j.c();
    j.key("lattice"); j.s += '{';
    j.key("type"); j.str(lattice_name(L.type_)); j.c();
    j.key("hkl"); j.str(L.hkl_); j.c();
    j.key("abc_set"); j.s += L.abc_set_ ? "true" : "false"; j.c();
    j.key("a"); j.v3(L.a_); j.c();
    j.key("b"); j.v3(L.b_); j.c();
    j.key("c"); j.v3(L.c_); j.c();
    j.key("t"); j.v3(L.t_); j.c();
    j.key("abangle"); j.num(L.abangle_); j.c();
    j.key("caratio"); j.num(L.caratio_);
    j.s += '}'; j.c();
    j.key("transvec"); j.v3(g.transvec_); j.c();
    j.key("repetition"); j.v3(g.repetition_); j.c();
    j.key("repetition_dist"); j.s += g.is_repetition_dist_ ? "true" : "false"; j.c();
    j.key("scaling_mean"); j.v3(g.scaling_.mean_); j.c();
    j.key("scaling_stddev"); j.v3(g.scaling_.stddev_); j.c();
    j.key("scaling_stat"); j.s += '[';
    for (int k = 0; k < 3; ++k) { if (k) j.c(); j.str(stat_name(g.scaling_.dist_[k])); }
    j.s += ']'; j.c();
    j.key("scaling_nsamples");
    j.v3(vector3_t(g.scaling_.nvals_[0], g.scaling_.nvals_[1], g.scaling_.nvals_[2])); j.c();
    Ensemble& e = s.ensemble_;
    j.key("spacing"); j.v3(e.spacing_); j.c();
    j.key("maxgrains"); j.v3(e.maxgrains_); j.c();
    j.key("distribution"); j.str(e.distribution_); j.c();
    j.key("orientation_stat"); j.str(e.orientations_.stat_);
    Rotation* rots[3] = {&e.orientations_.rot1_, &e.orientations_.rot2_, &e.orientations_.rot3_};
    for (int k = 0; k < 3; ++k) {
      Rotation& r = *rots[k];
      j.c();
      j.key("rot" + std::to_string(k + 1)); j.s += '{';
      j.key("axis"); j.str(std::string(1, r.axis_)); j.c();
      j.key("angles"); j.v2(r.angles_); j.c();
      j.key("mean"); j.num(r.mean_); j.c();
      j.key("sd"); j.num(r.sd_); j.c();
      j.key("location"); j.num(r.location_); j.c();
      j.key("scale"); j.num(r.scale_);
      j.s += '}';
    }
    GrainRepetitions& gr = g.repetitiondist_;
    // the axis type is private to GrainRepetitions: reached through auto
    auto rep = [&](const char* name, auto& r) {
      j.c();
      j.key(name); j.s += '{';
      j.key("stat"); j.str(stat_name(r.stat_)); j.c();
      j.key("min"); j.num(r.min_); j.c();
      j.key("max"); j.num(r.max_);
      j.s += '}';
    };
    rep("xrepetition", gr.xrepetition_);
    rep("yrepetition", gr.yrepetition_);
    rep("zrepetition", gr.zrepetition_);
    if (s.type_ == paracrystal_type && s.paracrystal_) {
      Paracrystal& pc = *s.paracrystal_;
      j.c();
      j.key("paracrystal_raw"); j.s += '{';
      j.key("dims"); j.num(pc.dims_); j.c();
      j.key("ymean"); j.num(pc.dist_[0]); j.c();
      j.key("xmean"); j.num(pc.dist_[1]); j.c();
      j.key("ystddev"); j.num(pc.sdev_[0]); j.c();
      j.key("xstddev"); j.num(pc.sdev_[1]); j.c();
      j.key("domain"); j.num(pc.domsize_);
      j.s += '}';
    }
    if (s.type_ == percusyevick_type && s.percusyevick_) {
      PercusYevick& py = *s.percusyevick_;
      j.c();
      j.key("percusyevick_raw"); j.s += '{';
      j.key("dims"); j.num(py.dims_); j.c();
      j.key("diameter"); j.num(py.dia_); j.c();
      j.key("volfraction"); j.num(py.volf_);
      j.s += '}';
    }
    j.s += '}';
  }
  j.s += '}'; j.c();
  j.key("struct_in_layer"); j.s += in.struct_in_layer_ ? "true" : "false"; j.c();
  ScatteringParams& sc = in.scattering_;
  j.key("scattering"); j.s += '{';
  j.key("expt"); j.str(sc.expt_); j.c();
  j.key("alphai"); j.v3(vector3_t(sc.alpha_i_.min_, sc.alpha_i_.max_, sc.alpha_i_.step_)); j.c();
  j.key("inplanerot"); j.v3(vector3_t(sc.inplane_rot_.min_, sc.inplane_rot_.max_, sc.inplane_rot_.step_)); j.c();
  j.key("tilt"); j.v3(vector3_t(sc.tilt_.min_, sc.tilt_.max_, sc.tilt_.step_)); j.c();
  j.key("photon_value"); j.num(sc.photon_.value_); j.c();
  j.key("photon_unit"); j.str(sc.photon_.unit_); j.c();
  j.key("polarization"); j.str(sc.polarization_); j.c();
  j.key("coherence"); j.num(sc.coherence_); j.c();
  j.key("spotarea"); j.num(sc.spot_area_); j.c();
  j.key("smearing"); j.num(sc.smearing_);
  j.s += '}'; j.c();
  DetectorParams& d = in.detector_;
  j.key("detector"); j.s += '{';
  j.key("origin"); j.str(d.origin_); j.c();
  j.key("totalpixels"); j.v2(d.total_pixels_); j.c();
  j.key("pixelsize"); j.num(d.pixel_size_); j.c();
  j.key("sdd"); j.num(d.sd_distance_); j.c();
  j.key("directbeam"); j.v2(d.direct_beam_);
  j.s += '}'; j.c();
  ComputeParams& cp = in.compute_;
  j.key("computation"); j.s += '{';
  j.key("pathprefix"); j.str(cp.pathprefix_); j.c();
  // the run name without the "_<yyyymmdd>_<hhmmss>" that ComputeParams::runname appends
  if (cp.runname_.compare(0, 4, "run_") != 0 || cp.runname_.size() != 19) {
    std::string rn = cp.runname_;
    if (rn.size() >= 16) rn = rn.substr(0, rn.size() - 16);
    j.key("runname"); j.str(rn); j.c();
  }
  j.key("method"); j.str(cp.method_); j.c();
  j.key("region_type"); j.str(region_name(cp.output_region_.type_)); j.c();
  j.key("minpoint"); j.v2(cp.output_region_.minpoint_); j.c();
  j.key("maxpoint"); j.v2(cp.output_region_.maxpoint_); j.c();
  j.key("resolution"); j.v2(vector2_t(cp.resolution_[0], cp.resolution_[1])); j.c();
  j.key("nslices"); j.num(cp.nslices_); j.c();
  j.key("structcorrelation"); j.str(corr_name(cp.correlation_)); j.c();
  j.key("palette"); j.str(cp.palette_);
  j.s += "}, \"saveff_savesf_raw\": [";
  j.num(cp.saveff_ ? 1 : 0); j.c(); j.num(cp.savesf_ ? 1 : 0);
  j.s += "]"; j.c();
  j.key("fitparams"); j.s += '{';
  first = true;
  for (auto& kv : in.param_data_key_map_) {
    if (!first) j.c();
    first = false;
    FitParam& p = kv.second;
    j.key(kv.first); j.s += '{';
    j.key("variable"); j.str(p.variable_); j.c();
    j.key("range"); j.v3(vector3_t(p.range_.min_, p.range_.max_, p.range_.step_)); j.c();
    j.key("init"); j.num(p.init_);
    j.s += '}';
  }
  j.s += '}';
  if (in.reference_data_set_) {
    FitReferenceData& r = in.reference_data_[0];
    j.c();
    j.key("referencedata_raw"); j.s += '{';
    j.key("path"); j.str(r.image_path_); j.c();
    j.key("mask"); j.str(r.image_mask_); j.c();
    j.key("region_type"); j.str(region_name(r.region_type_)); j.c();
    j.key("region_min"); j.v2(vector2_t(r.x_min_, r.y_min_)); j.c();
    j.key("region_max"); j.v2(vector2_t(r.x_max_, r.y_max_)); j.c();
    j.key("npoints_parallel"); j.num(r.np_parallel_); j.c();
    j.key("npoints_perpendicular"); j.num(r.np_perpendicular_);
    j.s += '}';
  }
  j.c();
  j.key("algorithms_raw"); j.s += '[';
  for (size_t i = 0; i < in.analysis_algos_.size(); ++i) {
    AnalysisAlgorithmData& a = in.analysis_algos_[i];
    if (i) j.c();
    j.s += '{';
    j.key("regularization"); j.num(a.regularization_); j.c();
    j.key("name"); j.str(algo_name(a.name_)); j.c();
    j.key("name_str"); j.str(a.name_str_); j.c();
    j.key("order"); j.num(a.order_); j.c();
    j.key("tolerance"); j.num(a.tolerance_); j.c();
    j.key("distance_metric"); j.str(metric_name(a.distance_metric_)); j.c();
    j.key("restart"); j.s += a.restart_ ? "true" : "false"; j.c();
    j.key("params"); j.s += '{';
    std::map<std::string, double> ps;
    for (auto& p : a.params_map_) ps[algo_param_name(p.first)] = p.second.value_;
    bool f2 = true;
    for (auto& p : ps) {
      if (!f2) j.c();
      f2 = false;
      j.key(p.first); j.num(p.second);
    }
    j.s += "}}";
  }
  j.s += "]}";
  return j.s;
}

}  // namespace

extern "C" {

// Parses `path` with the reference's reader and writes the JSON (NUL-terminated) into buf.
// Returns the JSON length, -1 when the reader rejected the file, -2 when buf is too small.
long ref_hig_json(const char* path, char* buf, long cap) {
  static std::string out;
  {
    HiGInput in;
    in.init();
    // the reader's stream keeps its end-of-file state from the previous file read in this
    // process, which makes the reference skip its include pass; start each file as the
    // first file of a process starts
    InputReader::instance().input_stream_.clear();
    // the reference reports its errors on std::cerr; keep them out of the caller's output
    std::streambuf* old = std::cerr.rdbuf();
    std::ostringstream sink;
    std::cerr.rdbuf(sink.rdbuf());
    std::streambuf* old_out = std::cout.rdbuf();
    std::cout.rdbuf(sink.rdbuf());
    const bool ok = in.construct_input_config(path);
    std::cerr.rdbuf(old);
    std::cout.rdbuf(old_out);
    if (!ok) return -1;
    out = dump(in);
  }
  if ((long)out.size() + 1 > cap) return -2;
  memcpy(buf, out.c_str(), out.size() + 1);
  return (long)out.size();
}

// As ref_hig_json, after HiGInput::update_params with the fit parameters keys[i] = vals[i]
// (the keys of the file's fitting block).  -3 when update_params refused.
long ref_hig_json_updated(const char* path, const char** keys, const double* vals, int n, char* buf,
                          long cap) {
  static std::string out;
  {
    HiGInput in;
    in.init();
    std::streambuf* old = std::cerr.rdbuf();
    std::ostringstream sink;
    std::cerr.rdbuf(sink.rdbuf());
    std::streambuf* old_out = std::cout.rdbuf();
    std::cout.rdbuf(sink.rdbuf());
    InputReader::instance().input_stream_.clear();
    bool ok = in.construct_input_config(path);
    if (ok) {
      map_t m;
      for (int i = 0; i < n; ++i) m[keys[i]] = vals[i];
      ok = in.update_params(m);
      if (!ok) {
        std::cerr.rdbuf(old);
        std::cout.rdbuf(old_out);
        return -3;
      }
    }
    std::cerr.rdbuf(old);
    std::cout.rdbuf(old_out);
    if (!ok) return -1;
    out = dump(in);
  }
  if ((long)out.size() + 1 > cap) return -2;
  memcpy(buf, out.c_str(), out.size() + 1);
  return (long)out.size();
}

}  // extern "C"


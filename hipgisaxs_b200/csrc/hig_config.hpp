// The simulation description read from a HiG input file: the reference's HiGInput object
// model (include/config/hig_input.hpp, include/model/{shape,layer,unitcell,structure,
// inst_scattering,inst_detector,compute_params}.hpp, include/config/temp_helpers.hpp) as plain
// host structs.  Enumerations are kept as the keyword strings the file uses ("cylinder",
// "hcp", "qspace", ...) with "error" where the reference stores its error enumerator.
// Fields that the reference leaves uninitialised until the file sets them carry a *_set flag.
#pragma once

#include <array>
#include <map>
#include <string>
#include <vector>

namespace hgx {
namespace hig {

using vec2 = std::array<double, 2>;
using vec3 = std::array<double, 3>;

struct RefIndex {
  double delta = 0.0, beta = 0.0;
};

struct ShapeParam {                // ShapeParam, include/model/shape.hpp:30-98
  std::string type_name;           // the file's type string, the key in Shape::params
  std::string type = "error";      // radius, xsize, ysize, height, edge, baseangle or error
  std::string stat = "none";       // none, uniform, random, range, gaussian, cauchy, t, error
  double min = 0.0, max = 0.0, p1 = 0.0, p2 = 0.0;
  int nvalues = 1;
};

struct Shape {                     // Shape, include/model/shape.hpp:103-180
  std::string key;
  std::string name;                // shape keyword, or "custom" for a shape file
  std::string name_str;            // the name as written (the file name for a custom shape)
  vec3 originvec{{0.0, 0.0, 0.0}};
  double zrot = 0.0, yrot = 0.0, xrot = 0.0;  // radians
  RefIndex refindex;
  std::map<std::string, ShapeParam> params;   // keyed by type_name
};

struct Layer {                     // Layer, include/model/layer.hpp
  std::string key;
  int order = 0;
  double thickness = 0.0;
  RefIndex refindex;
};

struct Unitcell {                  // Unitcell, include/model/unitcell.hpp
  std::string key;
  std::map<std::string, std::vector<vec3>> elements;  // shape key -> locations
  std::vector<std::string> element_order;             // shape keys in file order
};

struct Rotation {                  // Rotation, include/model/structure.hpp:166-219
  char axis = 'n';
  vec2 angles{{0.0, 0.0}};
  double mean = 0.0, sd = 0.0, location = 0.0, scale = 0.0;
  bool mean_set = false;           // an anglemean was given: angles_min no longer moves the mean
};

struct Lattice {                   // Lattice, include/model/structure.hpp:88-160
  std::string type = "cubic";
  std::string hkl = "100";
  bool abc_set = false;
  vec3 a{{1, 0, 0}}, b{{0, 1, 0}}, c{{0, 0, 1}}, t{{0, 0, 0}};
  double abangle = 60.0, caratio = 1.0;
};

struct Repetition {                // one axis of GrainRepetitions, structure.hpp:281-305
  std::string stat = "null";
  unsigned min = 0, max = 0;
};

struct Structure {                 // Structure, include/model/structure.hpp:481-733
  std::string key;
  double iratio = 1.0;
  std::string type = "default";    // default, paracrystal, percusyevick
  // grain
  std::string unitcell_key;
  RefIndex grain_refindex;         // Grain::refindex_, settable by a fit, unused by the simulation
  std::string layer_key = "air";
  int layer_order = 0;             // never set from layer:key by the reference's reader
  Lattice lattice;
  vec3 transvec{{0, 0, 0}};
  vec3 repetition{{1, 1, 1}};
  bool repetition_dist = false;
  Repetition xrep, yrep, zrep;
  vec3 scaling_mean{{1, 1, 1}}, scaling_stddev{{0, 0, 0}};
  std::array<std::string, 3> scaling_stat{{"none", "none", "none"}};
  std::array<int, 3> scaling_nsamples{{40, 40, 40}};
  // ensemble
  vec3 spacing{{0, 0, 0}};
  vec3 maxgrains{{1, 1, 1}};
  std::string distribution = "regular";
  std::string orientation_stat = "single";
  Rotation rot1, rot2, rot3;
  // paracrystal / Percus-Yevick (include/model/structure.hpp:37-85)
  int pc_dims = 1;
  double pc_dist[2] = {0, 0}, pc_sdev[2] = {0, 0}, pc_domain = 0;
  bool pc_dist_set[2] = {false, false}, pc_sdev_set[2] = {false, false}, pc_domain_set = false;
  int py_dims = 2;
  double py_diameter = 0, py_volfract = 0;
  bool py_diameter_set = false, py_volfract_set = false;
};

struct Scattering {                // ScatteringParams, src/model/inst_scattering.cpp:24-34
  std::string expt = "gisaxs";
  vec3 alphai{{0.1, 0.1, 0.1}};    // min, max, step (degrees)
  vec3 inplanerot{{0, 0, 0}};
  vec3 tilt{{0, 0, 0}};
  double photon_value = 10000;
  std::string photon_unit = "ev";
  std::string polarization = "s";
  double coherence = 300, spotarea = 0.01, smearing = 1.0;
};

struct Detector {                  // DetectorParams, src/model/inst_detector.cpp:25-33
  std::string origin = "bottom-left";
  vec2 totalpixels{{5000, 5000}};
  double pixelsize = 0.172, sdd = 4000;
  vec2 directbeam{{0, 0}};
};

struct Compute {                   // ComputeParams, src/model/compute_params.cpp:24-38
  std::string pathprefix = ".";
  std::string runname;             // as written; the reference appends "_<timestamp>"
  bool runname_set = false;
  std::string method = "dwba";
  std::string region_type = "qspace";
  vec2 minpoint{{-1, -1}}, maxpoint{{-1, -1}};
  int resolution[2] = {1, 1};
  unsigned nslices = 0;
  std::string structcorrelation = "null";
  std::string palette = "default";
  bool saveff = false, savesf = false, saveff_set = false, savesf_set = false;
};

struct FitParam {                  // FitParam, include/model/fitting_params.hpp:35-43
  std::string key, variable;
  vec3 range{{0, 0, -1}};          // min, max, step
  double init = 0.0;
};

struct FitReferenceData {          // FitReferenceData, include/config/temp_helpers.hpp:26-62
  std::string path, mask;
  bool path_set = false, mask_set = false;
  std::string region_type;
  bool region_type_set = false;
  vec2 region_min{{0, 0}}, region_max{{0, 0}};
  bool region_min_set = false, region_max_set = false;
  unsigned npoints_parallel = 0, npoints_perpendicular = 0;
  bool npar_set = false, nperp_set = false;
};

struct FitAlgorithm {              // AnalysisAlgorithmData, temp_helpers.hpp:84-148
  std::string name = "null", name_str;
  bool name_set = false;
  int order = 0;
  bool order_set = false;
  double tolerance = 0.0, regularization = 0.0;
  bool tolerance_set = false;
  std::string distance_metric;
  bool metric_set = false;
  bool restart = false, restart_set = false;
  std::map<std::string, double> params;  // parameter type keyword -> value
};

struct Input {
  std::string path;                // the file read
  std::map<std::string, Shape> shapes;
  std::map<int, Layer> layers;     // by order, as the reference keeps them
  std::map<std::string, int> layer_keys;
  std::map<std::string, Unitcell> unitcells;
  std::map<std::string, Structure> structures;
  std::vector<std::string> structure_order;  // keys in file order
  bool struct_in_layer = false;
  Scattering scattering;
  Detector detector;
  Compute compute;
  std::map<std::string, FitParam> fit_params;
  FitReferenceData reference_data;
  bool reference_data_set = false;
  std::vector<FitAlgorithm> algorithms;
};

// HiGInput::update_params for one parameter variable (src/config/hig_input.cpp:2712-2830 and
// the update_param methods of the model classes), e.g. "shape['s1']:param['radius']:min".
bool update_param(Input& in, const std::string& variable, double value, std::string& err);

// Reads a HiG file (HiGInput::construct_input_config).  Returns false with a message naming the
// line on a syntax or semantic error.
bool read_input(const std::string& path, Input& out, std::string& err);

// The whole description as one JSON object (numbers with 17 significant digits).
std::string to_json(const Input& in);

// Wave number k0 (1/nm) and frequency from the photon energy (HipGISAXS::init,
// src/sim/hipgisaxs_main.cpp:146-160); false for a unit other than "ev" or "kev".
bool photon_k0(const Scattering& s, double* k0, double* freq);

}  // namespace hig
}  // namespace hgx

// the handle behind hgx_hig (include/hgx.h)
struct hgx_hig_s {
  hgx::hig::Input in;
  std::string json;  // built on first request
};

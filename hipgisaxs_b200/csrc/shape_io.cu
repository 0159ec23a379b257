// Shape-definition files of the numeric form factor, without Boost: the front end of
// NumericFormFactor::read_shapes_file (src/ff/ff_num.cpp:985-1030).
//
//  * Wavefront OBJ (ObjectShapeReader::load_object, src/file/objectshape_reader.cpp:52-242):
//    "v x y z" vertices; "f" faces whose items are v, v/vt, v/vt/vn or v//vn with 1-based
//    vertex indices; vt, vn, g, o, s, l, mtllib, usemtl, comments and unknown lines are
//    ignored.  Faces with 3 vertices are kept in file order; faces with 4 vertices are counted
//    and left out, as the reference's converter leaves them out (objectshape_reader.cpp:39-40);
//    faces with more vertices are counted and skipped.  Unlike the reference, lines of any
//    length are read, tabs separate items like spaces, and a non-integer, non-positive
//    (relative) or out-of-range vertex index is an error instead of undefined behaviour.
//  * raw ".dat" (RawShapeReader::load_raw, src/file/rawshape_reader.cpp:37-60): whitespace-
//    separated records of 7 values (s, nx, ny, nz, cx, cy, cz) until the first incomplete one.
//  * HDF5 shape files need the reference's optional USE_HDF5 build; they are rejected here as
//    the reference rejects them without it.
//
// The OBJ triangles become shape_def rows on the device (hgx_mesh_to_shape_def, the
// get_triangle_params arithmetic); degenerate faces are dropped as convert_to_shape drops them
// (objectshape_reader.cpp:256-259).
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "hgx_internal.cuh"

struct hgx_mesh_s {
  std::vector<double> v;  // nv x 3
  std::vector<int> f;     // nf x 3, 0-based
  int nquads = 0;         // 4-vertex faces left out
  int nskipped = 0;       // faces with more than 4 (or fewer than 3) vertices
};

namespace hgx {
namespace {

// strict decimal integer (the whole string), as a lexical cast would accept it
bool parse_int(const std::string& s, long* out) {
  if (s.empty()) return false;
  errno = 0;
  char* end = nullptr;
  long v = std::strtol(s.c_str(), &end, 10);
  if (errno != 0 || end == s.c_str() || *end != '\0') return false;
  *out = v;
  return true;
}

int load_obj(const char* path, hgx_mesh_s& m) {
  std::ifstream in(path);
  if (!in.is_open()) return fail(HGX_ERR_INVALID_ARG, std::string("hgx_obj_load: cannot open ") + path);
  std::string line;
  long lineno = 0;
  std::vector<int> idx;
  while (std::getline(in, line)) {
    ++lineno;
    line.erase(std::remove(line.begin(), line.end(), '\r'), line.end());
    std::istringstream ss(line);
    std::string tok;
    if (!(ss >> tok)) continue;  // blank line
    if (tok == "v") {
      double x, y, z;
      if (!(ss >> x >> y >> z))
        return fail(HGX_ERR_INVALID_ARG, "hgx_obj_load: bad vertex at line " + std::to_string(lineno));
      m.v.push_back(x);
      m.v.push_back(y);
      m.v.push_back(z);
    } else if (tok == "f") {
      idx.clear();
      std::string item;
      while (ss >> item) {
        // v | v/vt | v/vt/vn | v//vn: the vertex index is the text before the first '/'
        const size_t s1 = item.find('/');
        const size_t nslash = std::count(item.begin(), item.end(), '/');
        long vi = 0;
        if (nslash > 2 || !parse_int(item.substr(0, s1), &vi))
          return fail(HGX_ERR_INVALID_ARG,
                      "hgx_obj_load: could not understand face item '" + item + "' at line " +
                          std::to_string(lineno));
        if (vi < 1 || vi > 0x7fffffffL)
          return fail(HGX_ERR_INVALID_ARG,
                      "hgx_obj_load: vertex index " + std::to_string(vi) + " at line " +
                          std::to_string(lineno) + " (1-based, relative indices are not supported)");
        idx.push_back((int)(vi - 1));
      }
      if (idx.size() == 3) {
        m.f.insert(m.f.end(), idx.begin(), idx.end());
      } else if (idx.size() == 4) {
        ++m.nquads;
      } else {
        ++m.nskipped;
      }
    }
    // everything else (vt, vn, g, o, s, l, mtllib, usemtl, comments, unknown) is ignored
  }
  const long nv = (long)(m.v.size() / 3);
  for (size_t i = 0; i < m.f.size(); ++i)
    if (m.f[i] >= nv)
      return fail(HGX_ERR_INVALID_ARG, "hgx_obj_load: face " + std::to_string(i / 3) +
                                           " refers to vertex " + std::to_string(m.f[i] + 1) +
                                           " of " + std::to_string(nv));
  if (nv > 0x7fffffffL || m.f.size() / 3 > 0x7fffffffUL)
    return fail(HGX_ERR_INVALID_ARG, "hgx_obj_load: mesh too large");
  return HGX_OK;
}

// the last '.'-separated component of the file name (NumericFormFactor::get_shapes_file_format,
// src/ff/ff_num.cpp:948-966, which compares the same spellings)
enum FileType { FT_OBJ, FT_DAT, FT_HDF5, FT_UNKNOWN };
FileType file_type(const char* path) {
  std::string p(path);
  size_t dot = p.find_last_of('.');
  size_t slash = p.find_last_of('/');
  if (dot == std::string::npos || (slash != std::string::npos && dot < slash)) return FT_UNKNOWN;
  std::string e = p.substr(dot + 1);
  if (e == "obj" || e == "Obj" || e == "OBJ") return FT_OBJ;
  if (e == "dat" || e == "Dat" || e == "DAT") return FT_DAT;
  if (e == "hd5" || e == "Hd5" || e == "HD5" || e == "hdf5" || e == "Hdf5" || e == "HDF5") return FT_HDF5;
  return FT_UNKNOWN;
}

int load_dat(const char* path, std::vector<double>& rows) {
  std::ifstream in(path);
  if (!in.is_open()) return fail(HGX_ERR_INVALID_ARG, std::string("hgx_read_shapes_file: cannot open ") + path);
  double r[7];
  while (true) {
    int k = 0;
    while (k < 7 && (in >> r[k])) ++k;
    if (k < 7) break;  // the first incomplete record ends the file, as in the reference
    rows.insert(rows.end(), r, r + 7);
    rows.push_back(0.0);  // padding of the 8-value layout
  }
  return HGX_OK;
}

}  // namespace
}  // namespace hgx

using namespace hgx;

extern "C" {

int hgx_obj_load(const char* path, hgx_mesh* out) {
  if (!path || !out) return fail(HGX_ERR_INVALID_ARG, "hgx_obj_load: null argument");
  *out = nullptr;
  auto m = new (std::nothrow) hgx_mesh_s();
  if (!m) return fail(HGX_ERR_NO_MEMORY, "hgx_obj_load: host allocation");
  int s = load_obj(path, *m);
  if (s != HGX_OK) {
    delete m;
    return s;
  }
  *out = m;
  return HGX_OK;
}

int hgx_mesh_info(hgx_mesh m, int* nv, int* nf, int* nquads, int* nskipped) {
  if (!m) return fail(HGX_ERR_INVALID_ARG, "hgx_mesh_info: null mesh");
  if (nv) *nv = (int)(m->v.size() / 3);
  if (nf) *nf = (int)(m->f.size() / 3);
  if (nquads) *nquads = m->nquads;
  if (nskipped) *nskipped = m->nskipped;
  return HGX_OK;
}

int hgx_mesh_read(hgx_mesh m, double* verts, int* faces) {
  if (!m) return fail(HGX_ERR_INVALID_ARG, "hgx_mesh_read: null mesh");
  if (verts) std::copy(m->v.begin(), m->v.end(), verts);
  if (faces) std::copy(m->f.begin(), m->f.end(), faces);
  return HGX_OK;
}

int hgx_mesh_destroy(hgx_mesh m) {
  delete m;
  return HGX_OK;
}

int hgx_read_shapes_file(hgx_ctx c, const char* path, double* shape_def, int capacity, int* ntri) {
  if (!path || !ntri) return fail(HGX_ERR_INVALID_ARG, "hgx_read_shapes_file: null argument");
  if (shape_def && capacity < 0) return fail(HGX_ERR_INVALID_ARG, "hgx_read_shapes_file: capacity < 0");
  *ntri = 0;
  std::vector<double> rows;
  switch (file_type(path)) {
    case FT_DAT:
      HGX_TRY(load_dat(path, rows));
      break;
    case FT_OBJ: {
      if (!c) return fail(HGX_ERR_INVALID_ARG, "hgx_read_shapes_file: .obj files need a context");
      hgx_mesh_s m;
      HGX_TRY(load_obj(path, m));
      const int nv = (int)(m.v.size() / 3), nf = (int)(m.f.size() / 3);
      if (nf > 0) {
        std::vector<double> all(8 * (size_t)nf);
        HGX_TRY(hgx_mesh_to_shape_def(c, nv, m.v.data(), nf, m.f.data(), all.data()));
        for (int t = 0; t < nf; ++t) {
          const double* p = all.data() + 8 * (size_t)t;
          if (p[1] == 0.0 && p[2] == 0.0 && p[3] == 0.0) continue;  // degenerate: dropped
          rows.insert(rows.end(), p, p + 8);
        }
      }
      break;
    }
    case FT_HDF5:
      return fail(HGX_ERR_INVALID_ARG, "hgx_read_shapes_file: HDF5 shape files are not supported "
                                       "(the reference needs its optional HDF5 build for them too)");
    default:
      return fail(HGX_ERR_INVALID_ARG, std::string("hgx_read_shapes_file: unknown shape file format: ") + path);
  }
  const int n = (int)(rows.size() / 8);
  *ntri = n;
  if (shape_def) {
    if (capacity < n)
      return fail(HGX_ERR_INVALID_ARG, "hgx_read_shapes_file: shape_def holds " + std::to_string(capacity) +
                                           " rows, the file has " + std::to_string(n));
    std::copy(rows.begin(), rows.end(), shape_def);
  }
  return HGX_OK;
}

}  // extern "C"

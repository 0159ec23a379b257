// Reference images and masks of a fit, read as the reference reads them
// (HipGISAXSObjectiveFunction::set_reference_data / read_mask_data / read_edf_mask_data,
// src/analyzer/objective_func_hipgisaxs.cpp:83-205):
//   * the file type by extension (get_reference_file_type, :60-81): edf/EDF -> EDF;
//     txt/TXT/dat/DAT/out/OUT -> text;
//   * text images (ImageData::read, src/analyzer/ImageData.cpp:79-104): the values of every
//     line in order; the row length is the first line's count; the row count is the number of
//     getline calls before end-of-file minus one, so a last line without a newline is read
//     but not counted;
//   * EDF (EDFReader, src/file/edf_reader.cpp): "key = value ;" items in 512-byte blocks up to
//     the closing '}', then EDF_BinarySize bytes of 32-bit floats from the next block boundary;
//     Dim_1 is the row length, Dim_2 the row count, and their product must match the data;
//   * masks: unsigned integers of a text file until its end, or an EDF image's values.
// Host only.
#include <stdlib.h>
#include <string.h>

#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "hgx_internal.cuh"

namespace hgx {
namespace {

enum FileKind { KIND_ERROR, KIND_TEXT, KIND_EDF };

FileKind file_kind(const std::string& name) {
  const size_t dot = name.rfind('.');
  if (dot == std::string::npos) return KIND_ERROR;
  const std::string ext = name.substr(dot + 1);
  if (ext == "edf" || ext == "EDF") return KIND_EDF;
  if (ext == "txt" || ext == "TXT" || ext == "dat" || ext == "DAT" || ext == "out" || ext == "OUT")
    return KIND_TEXT;
  return KIND_ERROR;
}

bool read_text_image(const std::string& path, std::vector<double>& data, int& ncol, int& nrow) {
  std::ifstream f(path);
  if (!f.is_open()) return false;
  int nv = -1, np = 0;
  std::string line;
  while (!f.eof()) {
    std::getline(f, line);
    ++nv;
    std::istringstream ss(line);
    std::vector<double> row;
    double v;
    while (ss >> v) row.push_back(v);
    if (nv == 0) np = (int)row.size();
    data.insert(data.end(), row.begin(), row.end());
  }
  ncol = np;
  nrow = nv;
  return true;
}

bool is_space(char c) { return c == ' ' || c == '\n' || c == '\t' || c == '\r'; }

bool read_edf(const std::string& path, std::vector<double>& data, int& ncol, int& nrow, std::string& err) {
  std::ifstream f(path, std::ios::binary);
  if (!f.is_open()) { err = "cannot open"; return false; }
  const size_t B = 512;
  std::map<std::string, std::string> header;
  std::string key, value;
  bool in_value = false, done = false;
  std::vector<char> chunk(B);
  while (!done) {
    f.read(chunk.data(), B);
    if (f.gcount() <= 0) { err = "end of file inside the header"; return false; }
    for (size_t i = 0; i < B && !done; ++i) {
      const char c = chunk[i];
      if (!in_value) {
        if (c == '}') { done = true; break; }
        if (c == '=') { in_value = true; continue; }
        if (!is_space(c)) key += c;
      } else {
        if (c == ';') {
          header[key] = value;
          key.clear();
          value.clear();
          in_value = false;
          // the header ends at a '}' that follows only white space
          size_t j = i + 1;
          while (j < B && is_space(chunk[j])) ++j;
          if (j < B && chunk[j] == '}') done = true;
          continue;
        }
        if (!is_space(c)) value += c;
      }
    }
  }
  ncol = atoi(header["Dim_1"].c_str());
  nrow = atoi(header["Dim_2"].c_str());
  const unsigned long bytes = strtoul(header["EDF_BinarySize"].c_str(), nullptr, 10);
  std::vector<char> raw(bytes);
  if (bytes) f.read(raw.data(), bytes);
  if ((unsigned long)f.gcount() != bytes) { err = "fewer data bytes than EDF_BinarySize"; return false; }
  data.resize(bytes / sizeof(float));
  for (size_t i = 0; i < data.size(); ++i) {
    float v;
    memcpy(&v, raw.data() + i * sizeof(float), sizeof(float));
    data[i] = v;
  }
  if (data.size() != (size_t)ncol * (size_t)nrow) { err = "Dim_1 x Dim_2 does not match the data"; return false; }
  return true;
}

}  // namespace
}  // namespace hgx

using namespace hgx;

extern "C" {

int hgx_read_image(const char* path, double* data, long capacity, long* count, int* ncol, int* nrow) {
  if (!path || !count || !ncol || !nrow) return fail(HGX_ERR_INVALID_ARG, "hgx_read_image: null argument");
  std::vector<double> v;
  std::string err;
  switch (file_kind(path)) {
    case KIND_TEXT:
      if (!read_text_image(path, v, *ncol, *nrow))
        return fail(HGX_ERR_INVALID_ARG, std::string("hgx_read_image: cannot open ") + path);
      break;
    case KIND_EDF:
      if (!read_edf(path, v, *ncol, *nrow, err))
        return fail(HGX_ERR_INVALID_ARG, std::string("hgx_read_image: ") + path + ": " + err);
      break;
    default:
      return fail(HGX_ERR_INVALID_ARG, std::string("hgx_read_image: unknown image type of ") + path);
  }
  *count = (long)v.size();
  if (data) {
    if (capacity < (long)v.size()) return fail(HGX_ERR_INVALID_ARG, "hgx_read_image: capacity too small");
    memcpy(data, v.data(), sizeof(double) * v.size());
  }
  return HGX_OK;
}

int hgx_read_mask(const char* path, unsigned* mask, long capacity, long* count) {
  if (!path || !count) return fail(HGX_ERR_INVALID_ARG, "hgx_read_mask: null argument");
  std::vector<unsigned> m;
  if (file_kind(path) == KIND_EDF) {
    std::vector<double> v;
    int nc = 0, nr = 0;
    std::string err;
    if (!read_edf(path, v, nc, nr, err))
      return fail(HGX_ERR_INVALID_ARG, std::string("hgx_read_mask: ") + path + ": " + err);
    for (double x : v) m.push_back((unsigned)x);
  } else {
    std::ifstream f(path);
    if (!f.is_open()) return fail(HGX_ERR_INVALID_ARG, std::string("hgx_read_mask: cannot open ") + path);
    while (true) {  // read_mask_data: unsigned values until end of file
      unsigned val = 0;
      f >> val;
      if (f.eof()) break;
      if (f.fail()) return fail(HGX_ERR_INVALID_ARG, std::string("hgx_read_mask: not an unsigned integer in ") + path);
      m.push_back(val);
    }
  }
  *count = (long)m.size();
  if (mask) {
    if (capacity < (long)m.size()) return fail(HGX_ERR_INVALID_ARG, "hgx_read_mask: capacity too small");
    memcpy(mask, m.data(), sizeof(unsigned) * m.size());
  }
  return HGX_OK;
}

}  // extern "C"

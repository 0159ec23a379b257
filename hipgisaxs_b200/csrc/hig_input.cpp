// HiG input reader: the reference's HiGInput::construct_input_config
// (src/config/hig_input.cpp:61-104, with the tokenizer InputReader of
// src/file/read_oo_input.cpp and the keyword tables of include/config/token_mapper.hpp).
//
// The reference drives its object model token by token from a keyword stack.  This reader
// tokenizes the file, checks every token against the token that precedes it by the same
// rules the reference applies (so separators, comments and brackets are accepted or rejected
// alike), builds a tree of `keyword = value` entries and then fills the model block by block.
// Inputs the reference reads are read to the same values, including its quirks:
//   * a shape without a refindex block keeps the previous shape's refractive index
//     (Shape::init and Shape::clear leave refindex_ as it was, src/model/shape.cpp:46-62);
//   * alphai's step also sets the in-plane rotation step (missing break,
//     src/config/hig_input.cpp:1027-1030);
//   * a Percus-Yevick volfraction also sets the structure's iratio and must be > 0 (missing
//     break, src/config/hig_input.cpp:1110-1116);
//   * a second element with the same shape:key in one unit cell discards the first one's
//     locations (curr_element_list_[str].clear(), src/config/hig_input.cpp:1643);
//   * an orientation's anglemean/anglesd/anglelocation/anglescale carry over to the next
//     structure (Rotation keeps them through GrainOrientations::init/clear);
//   * an algorithm block starts from the previous block's name, order, tolerance,
//     regularization, metric and restart (AnalysisAlgorithmData::clear keeps them);
//   * the grain's layer order stays 0 whatever layer:key says (Grain::init,
//     src/model/structure.cpp:389-398; nothing in the reader assigns it);
//   * the run name is stored as written; the reference appends "_<timestamp>".
// Where the reference would dereference a missing object (a Percus-Yevick structure with more
// than one shape, domain/xspacing/yspacing outside a paracrystal) or loop on an unterminated
// string, this reader reports an error.  Keywords placed in a block that the reference would
// silently accept but never use are reported as misplaced.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <time.h>

#include <cstring>
#include <fstream>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "hgx_internal.cuh"
#include "hig_config.hpp"

namespace hgx {
namespace hig {

namespace {

constexpr double PI = 3.141592653589793;  // PI_, include/common/constants.hpp:29

// ------------------------------------------------------------------------- tokens ----

enum Kind { K_NONE, K_WORD, K_NUM, K_STR, K_LBRACE, K_RBRACE, K_LBRACK, K_RBRACK, K_ASSIGN,
            K_COMMA, K_COMMENT, K_END };

struct Tok {
  Kind k;
  std::string s;
  double v = 0.0;
  int line = 0;
  int file = 0;  // index into the file name list
};

// every keyword of the language (TokenMapper::KeyWords_, include/config/token_mapper.hpp:179-300)
const std::set<std::string>& keywords() {
  static const std::set<std::string> k = {
      "a", "abangle", "algorithm", "algoname", "algoorder", "algoparam", "alphai", "angles",
      "anglelocation", "anglemean", "anglescale", "anglesd", "axis", "b", "beta", "c", "caratio",
      "coherence", "computation", "delta", "detector", "dimensions", "directbeam",
      "distancemetric", "distribution", "domain", "element", "ensemble", "expt", "fitparam",
      "fitregion", "fitting", "grain", "hipGisaxsInput", "hkl", "include", "init", "inplanerot",
      "instrumentation", "iratio", "key", "lattice", "layer", "layer:key", "locations", "mask",
      "max", "maxgrains", "maxpoint", "mean", "method", "min", "minpoint", "name", "npoints",
      "nsamples", "nslices", "nvalues", "order", "orientations", "origin", "originvec",
      "outputregion", "p1", "p2", "palette", "paracrystal", "parallel", "param", "path",
      "pathprefix", "percusyevick", "perpendicular", "photon", "pixelsize", "polarization",
      "pvalue", "range", "regmax", "regmin", "regularization", "repetition", "repetitiondist",
      "restart", "referencedata", "refindex", "resolution", "rot", "rot1", "rot2", "rot3",
      "runname", "saveff", "savesf", "scaling", "scattering", "sdd", "shape", "shape:key",
      "smearing", "spacing", "spotarea", "stat", "stddev", "step", "structcorrelation",
      "structure", "thickness", "tilt", "tolerance", "totalpixels", "transvec", "type", "unit",
      "unitcell", "unitcell:key", "value", "variable", "volfraction", "xrepetition", "xrot",
      "xspacing", "yrepetition", "yrot", "yspacing", "zrepetition", "zrot"};
  return k;
}

struct Lexer {
  std::vector<std::string> files;
  std::string err;

  bool fail_at(int file, int line, const std::string& msg) {
    err = files[file] + ":" + std::to_string(line) + ": " + msg;
    return false;
  }

  static bool read_file(const std::string& path, std::string& text) {
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) return false;
    std::ostringstream ss;
    ss << f.rdbuf();
    text = ss.str();
    return true;
  }

  // InputReader::get_next_token (src/file/read_oo_input.cpp:151-229) over a whole file
  bool lex(const std::string& text, int file, std::vector<Tok>& out) {
    int line = 1;
    size_t i = 0;
    const size_t n = text.size();
    auto is_alpha = [](char c) { return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || c == ':'; };
    auto is_digit = [](char c) { return c >= '0' && c <= '9'; };
    while (i < n) {
      const char c = text[i];
      if (c == ' ' || c == '\t' || c == '\v' || c == '\f' || c == '\r' || c == '\n') {
        if (c == '\n') ++line;
        ++i;
        continue;
      }
      Tok t;
      t.line = line;
      t.file = file;
      if (c == '#') {  // comment to the end of the line
        while (i < n && text[i] != '\n') ++i;
        t.k = K_COMMENT;
      } else if (is_alpha(c)) {  // keyword: letters, ':' then also digits and '-'
        size_t j = i;
        while (j < n && (is_alpha(text[j]) || is_digit(text[j]) || text[j] == '-')) ++j;
        t.k = K_WORD;
        t.s = text.substr(i, j - i);
        i = j;
        if (!keywords().count(t.s)) return fail_at(file, line, "unknown keyword '" + t.s + "'");
      } else if (is_digit(c) || c == '-') {  // a number as istream >> double reads it
        size_t j = i;
        if (text[j] == '-') ++j;
        size_t digits = 0;
        while (j < n && is_digit(text[j])) ++j, ++digits;
        if (j < n && text[j] == '.') {
          ++j;
          while (j < n && is_digit(text[j])) ++j, ++digits;
        }
        if (digits == 0) return fail_at(file, line, "malformed number");
        if (j < n && (text[j] == 'e' || text[j] == 'E')) {
          size_t k = j + 1;
          if (k < n && (text[k] == '+' || text[k] == '-')) ++k;
          size_t ed = 0;
          while (k < n && is_digit(text[k])) ++k, ++ed;
          if (ed == 0) return fail_at(file, line, "malformed number (exponent without digits)");
          j = k;
        }
        const std::string num = text.substr(i, j - i);
        t.k = K_NUM;
        t.v = strtod(num.c_str(), nullptr);
        t.s = num;
        i = j;
      } else if (c == '"') {
        size_t j = text.find('"', i + 1);
        if (j == std::string::npos) return fail_at(file, line, "unterminated string");
        t.k = K_STR;
        t.s = text.substr(i + 1, j - i - 1);
        for (char ch : t.s)
          if (ch == '\n') ++line;
        i = j + 1;
      } else {
        switch (c) {
          case '{': t.k = K_LBRACE; break;
          case '}': t.k = K_RBRACE; break;
          case '[': t.k = K_LBRACK; break;
          case ']': t.k = K_RBRACK; break;
          case '=': t.k = K_ASSIGN; break;
          case ',': t.k = K_COMMA; break;
          default:
            return fail_at(file, line, std::string("unexpected character '") + c + "'");
        }
        ++i;
      }
      out.push_back(t);
    }
    return true;
  }

  // `include = "file"` is replaced by the file's tokens (HiGInput::construct_input_config's
  // first pass with InputReader::read_include_file, src/file/read_oo_input.cpp:55-90).  The
  // file is looked up as written (relative to the working directory, as the reference does),
  // then relative to the including file's directory.
  bool lex_file(const std::string& path, std::vector<Tok>& out, int depth) {
    if (depth > 16) return fail_at(0, 0, "include nesting deeper than 16 files");
    std::string text;
    if (!read_file(path, text)) {
      err = "cannot open input file '" + path + "'";
      return false;
    }
    const int file = (int)files.size();
    files.push_back(path);
    std::vector<Tok> toks;
    if (!lex(text, file, toks)) return false;
    for (size_t i = 0; i < toks.size(); ++i) {
      if (toks[i].k == K_WORD && toks[i].s == "include" && i + 2 < toks.size() &&
          toks[i + 1].k == K_ASSIGN && toks[i + 2].k == K_STR) {
        std::string inc = toks[i + 2].s;
        std::string probe;
        if (!read_file(inc, probe) && !inc.empty() && inc[0] != '/') {
          const size_t slash = path.rfind('/');
          if (slash != std::string::npos) inc = path.substr(0, slash + 1) + inc;
        }
        if (!lex_file(inc, out, depth + 1)) return false;
        i += 2;
        continue;
      }
      out.push_back(toks[i]);
    }
    return true;
  }
};

// The reference's token-order rules (HiGInput::process_curr_token,
// src/config/hig_input.cpp:109-601): which token may precede each kind of token.
bool check_order(const std::vector<Tok>& t, const Lexer& lx, std::string& err) {
  Kind prev = K_NONE;
  for (const Tok& k : t) {
    bool ok = true;
    switch (k.k) {
      case K_WORD:
        ok = (k.s == "hipGisaxsInput") ? prev == K_NONE
                                       : (prev == K_LBRACE || prev == K_COMMA || prev == K_COMMENT);
        break;
      case K_ASSIGN: ok = prev == K_WORD; break;
      case K_LBRACE: ok = prev == K_ASSIGN || prev == K_COMMENT; break;
      case K_RBRACE:
        ok = prev == K_NUM || prev == K_STR || prev == K_RBRACE || prev == K_RBRACK ||
             prev == K_LBRACE || prev == K_COMMENT;
        break;
      case K_LBRACK: ok = prev == K_ASSIGN || prev == K_LBRACK || prev == K_RBRACK; break;
      case K_RBRACK: ok = prev == K_NUM || prev == K_LBRACK || prev == K_COMMENT || prev == K_RBRACK; break;
      case K_NUM: ok = prev == K_ASSIGN || prev == K_LBRACK || prev == K_NUM || prev == K_COMMENT; break;
      case K_STR: ok = prev == K_ASSIGN || prev == K_COMMENT; break;
      case K_COMMA:
        ok = prev == K_RBRACK || prev == K_RBRACE || prev == K_STR || prev == K_NUM || prev == K_COMMENT;
        break;
      default: break;
    }
    if (!ok) {
      static const char* names[] = {"start", "keyword", "number", "string", "'{'", "'}'", "'['",
                                    "']'", "'='", "','", "comment", "end"};
      std::string what = k.k == K_WORD ? "keyword '" + k.s + "'" : names[k.k];
      err = lx.files[k.file] + ":" + std::to_string(k.line) + ": " + what + " cannot follow " +
            names[prev];
      return false;
    }
    prev = k.k;
  }
  return true;
}

// --------------------------------------------------------------------------- tree ----

struct Node {
  enum Type { NUM, STR, ARR, OBJ } type = OBJ;
  std::string key;  // for entries of an object
  double num = 0.0;
  std::string str;
  std::vector<Node> kids;  // array elements (NUM or ARR) or object entries
  int line = 0, file = 0;
  bool comment_before_close = false;  // an array whose ']' follows a comment
};

struct Parser {
  const std::vector<Tok>& t;
  const Lexer& lx;
  size_t i = 0;
  std::string err;

  Parser(const std::vector<Tok>& toks, const Lexer& l) : t(toks), lx(l) {}

  const Tok& cur() {
    static Tok end{K_END, "", 0.0, 0, 0};
    return i < t.size() ? t[i] : end;
  }
  bool fail(const std::string& msg) {
    const Tok& k = cur();
    err = (k.k == K_END ? std::string("end of input") : lx.files[k.file] + ":" + std::to_string(k.line)) +
          ": " + msg;
    return false;
  }
  void skip(bool commas) {
    while (i < t.size() && (t[i].k == K_COMMENT || (commas && t[i].k == K_COMMA))) ++i;
  }

  bool array(Node& n) {  // at '['
    n.type = Node::ARR;
    n.line = cur().line;
    n.file = cur().file;
    ++i;
    for (;;) {
      const size_t before = i;
      skip(false);
      const Tok& k = cur();
      if (k.k == K_RBRACK) {
        n.comment_before_close = i > before;
        ++i;
        return true;
      }
      if (k.k == K_NUM) {
        Node e;
        e.type = Node::NUM;
        e.num = k.v;
        e.line = k.line;
        e.file = k.file;
        n.kids.push_back(e);
        ++i;
      } else if (k.k == K_LBRACK) {
        Node e;
        if (!array(e)) return false;
        n.kids.push_back(std::move(e));
      } else {
        return fail("expected a number or ']' in an array");
      }
    }
  }

  bool object(Node& n) {  // at '{'
    n.type = Node::OBJ;
    n.line = cur().line;
    n.file = cur().file;
    ++i;
    for (;;) {
      skip(true);
      const Tok& k = cur();
      if (k.k == K_RBRACE) { ++i; return true; }
      if (k.k != K_WORD) return fail("expected a keyword or '}'");
      Node e;
      if (!entry(e)) return false;
      n.kids.push_back(std::move(e));
    }
  }

  bool entry(Node& e) {  // at a keyword
    e.key = cur().s;
    e.line = cur().line;
    e.file = cur().file;
    ++i;
    if (cur().k != K_ASSIGN) return fail("expected '=' after '" + e.key + "'");
    ++i;
    skip(false);
    const Tok& v = cur();
    switch (v.k) {
      case K_NUM: e.type = Node::NUM; e.num = v.v; ++i; break;
      case K_STR: e.type = Node::STR; e.str = v.s; ++i; break;
      case K_LBRACE: { Node o; if (!object(o)) return false; e.type = Node::OBJ; e.kids = std::move(o.kids); break; }
      case K_LBRACK: {
        Node a;
        if (!array(a)) return false;
        e.type = Node::ARR;
        e.kids = std::move(a.kids);
        e.comment_before_close = a.comment_before_close;
        break;
      }
      default: return fail("expected a value after '" + e.key + " ='");
    }
    // what may follow a value (a separator, a comment, the end of the block) is checked by
    // check_order; the enclosing block then expects a keyword or its end
    return true;
  }

  bool file(Node& root) {
    if (cur().k != K_WORD || cur().s != "hipGisaxsInput")
      return fail("the input must start with 'hipGisaxsInput ='");
    if (!entry(root)) return false;
    if (root.type != Node::OBJ) return fail("'hipGisaxsInput' must be an object");
    skip(true);
    if (cur().k != K_END) return fail("text after the closing '}' of hipGisaxsInput");
    return true;
  }
};

// ---------------------------------------------------------------------- semantics ----

// keyword tables of include/config/token_mapper.hpp:301-398
const std::set<std::string> kShapeNames = {"box", "cube", "cylinder", "hcylinder", "randcylinders",
                                           "sphere", "pyramid", "trunccone", "prism3", "prism6",
                                           "prism3x", "sawtooth", "custom"};
const std::set<std::string> kParamTypes = {"radius", "xsize", "ysize", "height", "edge", "baseangle"};
const std::set<std::string> kLattices = {"bcc", "cubic", "fcc", "fco", "hcp", "hex"};
const std::set<std::string> kRegions = {"angles", "pixels", "qspace"};
const std::set<std::string> kCorrelations = {"nGnE", "nGE", "GnE", "GE"};
const std::set<std::string> kAlgorithms = {"lmvm", "pounders", "pso", "bruteforce", "none_pounders"};
const std::set<std::string> kAlgoParams = {"pounders_delta", "pso_omega", "pso_phi1", "pso_phi2",
                                           "pso_num_particles", "pso_num_generations",
                                           "pso_tune_omega", "pso_type"};
const std::set<std::string> kMetrics = {"sqrt_unit_l1", "sqrt_unit_l2", "sqrt_c_l2", "cbrt_unit_l1",
                                        "cbrt_unit_l2", "cbrt_c_l2", "sqrt_unit_l1_residual",
                                        "sqrt_unit_l2_residual", "sqrt_c_l2_residual"};

std::string stat_name(const std::string& s) {  // StatisticKeyWords_: "single" is "none"
  static const std::set<std::string> k = {"none", "uniform", "random", "range", "gaussian", "cauchy", "t"};
  if (s == "single") return "none";
  return k.count(s) ? s : "error";
}
std::string lookup(const std::set<std::string>& table, const std::string& s) {
  return table.count(s) ? s : "error";
}
bool boolean(const std::string& s) {  // TokenMapper::get_boolean
  return s == "true" || s == "True" || s == "TRUE" || s == "yes" || s == "Yes" || s == "YES";
}
bool has_suffix(const std::string& s, const std::string& e) {
  return s.size() >= e.size() && s.compare(s.size() - e.size(), e.size(), e) == 0;
}

int lattice_code(const std::string& name) {  // LatticeType, include/common/enums.hpp:56-65
  if (name == "bcc") return 2;
  if (name == "cubic") return 3;
  if (name == "fcc") return 4;
  if (name == "fco") return 5;
  if (name == "hcp") return 6;
  if (name == "hex") return 7;
  return 1;
}

struct Builder {
  Input& in;
  const Lexer& lx;
  std::string err;
  RefIndex shape_refindex;  // carried from shape to shape
  Rotation rot_extra[3];    // mean/sd/location/scale carried from structure to structure
  Repetition rep_carry[3];  // the repetition distribution, never reset by the reference
  FitAlgorithm algo_carry;  // carried from algorithm to algorithm

  Builder(Input& i, const Lexer& l) : in(i), lx(l) {}

  bool fail(const Node& n, const std::string& msg) {
    err = lx.files[n.file] + ":" + std::to_string(n.line) + ": " + msg;
    return false;
  }
  bool misplaced(const Node& n, const char* block) {
    return fail(n, "keyword '" + n.key + "' is not valid in " + block);
  }
  bool number(const Node& n, double& v) {
    if (n.type != Node::NUM) return fail(n, "'" + n.key + "' takes a number");
    v = n.num;
    return true;
  }
  bool string(const Node& n, std::string& s) {
    if (n.type != Node::STR) return fail(n, "'" + n.key + "' takes a quoted string");
    s = n.str;
    return true;
  }
  bool object(const Node& n) {
    if (n.type != Node::OBJ) return fail(n, "'" + n.key + "' takes a { ... } block");
    return true;
  }
  template <size_t N>
  bool vec(const Node& n, std::array<double, N>& v) {
    if (n.type != Node::ARR || n.kids.size() != N)
      return fail(n, "'" + n.key + "' takes [" + std::to_string(N) + " numbers]");
    for (size_t k = 0; k < N; ++k) {
      if (n.kids[k].type != Node::NUM) return fail(n, "'" + n.key + "' takes a flat array of numbers");
      v[k] = n.kids[k].num;
    }
    return true;
  }

  // refindex = { delta, beta }, for a layer or a shape (hig_input.cpp:1037-1064)
  bool refindex(const Node& n, RefIndex& r) {
    if (!object(n)) return false;
    for (const Node& e : n.kids) {
      if (e.key == "delta") { if (!number(e, r.delta)) return false; }
      else if (e.key == "beta") { if (!number(e, r.beta)) return false; }
      else return misplaced(e, "refindex");
    }
    return true;
  }

  bool shape(const Node& n) {
    if (!object(n)) return false;
    Shape s;
    s.name = "error";
    s.refindex = shape_refindex;
    for (const Node& e : n.kids) {
      double v;
      if (e.key == "key") { if (!string(e, s.key)) return false; }
      else if (e.key == "name") {
        std::string nm;
        if (!string(e, nm)) return false;
        if (kShapeNames.count(nm)) s.name = nm;
        else if (has_suffix(nm, ".shp") || has_suffix(nm, ".hd5") || has_suffix(nm, ".dat") ||
                 has_suffix(nm, ".obj")) s.name = "custom";
        else return fail(e, "unknown shape name '" + nm + "'");
        s.name_str = nm;
      }
      else if (e.key == "originvec") { if (!vec(e, s.originvec)) return false; }
      else if (e.key == "zrot") { if (!number(e, v)) return false; s.zrot = v * PI / 180.; }
      else if (e.key == "yrot") { if (!number(e, v)) return false; s.yrot = v * PI / 180.; }
      else if (e.key == "xrot") { if (!number(e, v)) return false; s.xrot = v * PI / 180.; }
      else if (e.key == "refindex") { if (!refindex(e, s.refindex)) return false; shape_refindex = s.refindex; }
      else if (e.key == "param") {
        if (!object(e)) return false;
        ShapeParam p;
        for (const Node& f : e.kids) {
          if (f.key == "type") {
            if (!string(f, p.type_name)) return false;
            p.type = lookup(kParamTypes, p.type_name);
          }
          else if (f.key == "stat") { std::string st; if (!string(f, st)) return false; p.stat = stat_name(st); }
          else if (f.key == "min") { if (!number(f, p.min)) return false; }
          else if (f.key == "max") { if (!number(f, p.max)) return false; }
          else if (f.key == "p1") { if (!number(f, p.p1)) return false; }
          else if (f.key == "p2") { if (!number(f, p.p2)) return false; }
          else if (f.key == "nvalues") { if (!number(f, v)) return false; p.nvalues = (int)v; }
          else return misplaced(f, "param");
        }
        s.params[p.type_name] = p;
      }
      else return misplaced(e, "shape");
    }
    // Shape::operator= (include/model/shape.hpp:142-155) merges the parameters into those of
    // an earlier shape with the same key
    auto prev = in.shapes.find(s.key);
    if (prev != in.shapes.end()) {
      for (const auto& kv : prev->second.params)
        if (!s.params.count(kv.first)) s.params[kv.first] = kv.second;
    }
    in.shapes[s.key] = s;
    return true;
  }

  bool layer(const Node& n) {
    if (!object(n)) return false;
    Layer l;
    for (const Node& e : n.kids) {
      double v;
      if (e.key == "key") { if (!string(e, l.key)) return false; }
      else if (e.key == "order") { if (!number(e, v)) return false; l.order = (int)v; }
      else if (e.key == "thickness") { if (!number(e, l.thickness)) return false; }
      else if (e.key == "refindex") { if (!refindex(e, l.refindex)) return false; }
      else return misplaced(e, "layer");
    }
    in.layers[l.order] = l;
    in.layer_keys[l.key] = l.order;
    return true;
  }

  bool unitcell(const Node& n) {
    if (!object(n)) return false;
    Unitcell u;
    for (const Node& e : n.kids) {
      if (e.key == "key") { if (!string(e, u.key)) return false; }
      else if (e.key == "element") {
        if (!object(e)) return false;
        std::string skey;
        bool have_key = false;
        for (const Node& f : e.kids) {
          if (f.key == "shape:key") {
            if (!string(f, skey)) return false;
            have_key = true;
            if (!u.elements.count(skey)) u.element_order.push_back(skey);
            u.elements[skey].clear();
          } else if (f.key == "locations") {
            // nested arrays of 3 numbers, at least one (hig_input.cpp:445-461).  The reference
            // tells a location's ']' from the list's ']' by the token before it, so a comment
            // just before either bracket derails it: an error there and here
            if (f.type != Node::ARR || f.kids.empty())
              return fail(f, "'locations' takes [[x y z] ...]");
            bool comment_close = f.comment_before_close;
            for (const Node& p : f.kids) comment_close = comment_close || p.comment_before_close;
            if (comment_close)
              return fail(f, "a comment just before a ']' of 'locations'");
            if (!have_key) {
              if (!u.elements.count(skey)) u.element_order.push_back(skey);
            }
            for (const Node& p : f.kids) {
              if (p.type != Node::ARR || p.kids.size() != 3)
                return fail(f, "'locations' takes [[x y z] ...]");
              vec3 v;
              for (int k = 0; k < 3; ++k) {
                if (p.kids[k].type != Node::NUM) return fail(f, "'locations' takes [[x y z] ...]");
                v[k] = p.kids[k].num;
              }
              u.elements[skey].push_back(v);
            }
          } else {
            return misplaced(f, "element");
          }
        }
      }
      else return misplaced(e, "unitcell");
    }
    in.unitcells[u.key] = u;
    return true;
  }

  bool repetition_axis(const Node& n, Repetition& r) {
    if (!object(n)) return false;
    for (const Node& e : n.kids) {
      double v;
      if (e.key == "min" || e.key == "max") {
        if (!number(e, v)) return false;
        if (v < 0) return fail(e, "a repetition count must be >= 0");
        (e.key == "min" ? r.min : r.max) = (unsigned)v;
      }
      else if (e.key == "stat") { std::string st; if (!string(e, st)) return false; r.stat = stat_name(st); }
      else return misplaced(e, n.key.c_str());
    }
    return true;
  }

  // lattice = { type, a, b, c, hkl, abangle, caratio } or lattice = "type"
  bool lattice(const Node& n, Structure& s) {
    if (n.type == Node::STR) { s.lattice.type = lookup(kLattices, n.str); return true; }
    if (!object(n)) return false;
    for (const Node& e : n.kids) {
      if (e.key == "type") { std::string t; if (!string(e, t)) return false; s.lattice.type = lookup(kLattices, t); }
      else if (e.key == "hkl") { if (!string(e, s.lattice.hkl)) return false; }
      else if (e.key == "abangle") { if (!number(e, s.lattice.abangle)) return false; }
      else if (e.key == "caratio") { if (!number(e, s.lattice.caratio)) return false; }
      else if (e.key == "a" || e.key == "b" || e.key == "c") {
        const int ax = e.key[0] - 'a';
        if (e.type == Node::ARR) {
          vec3& dst = ax == 0 ? s.lattice.a : ax == 1 ? s.lattice.b : s.lattice.c;
          if (!vec(e, dst)) return false;
          s.lattice.abc_set = true;
        } else if (e.type == Node::OBJ) {  // the grain scaling of this axis (hig_input.cpp:1148-1196)
          for (const Node& f : e.kids) {
            double v;
            if (f.key == "mean") { if (!number(f, s.scaling_mean[ax])) return false; }
            else if (f.key == "stddev") { if (!number(f, s.scaling_stddev[ax])) return false; }
            else if (f.key == "nsamples") { if (!number(f, v)) return false; s.scaling_nsamples[ax] = (int)v; }
            else if (f.key == "stat") { std::string st; if (!string(f, st)) return false; s.scaling_stat[ax] = stat_name(st); }
            else return misplaced(f, "a lattice vector block");
          }
        } else {
          return fail(e, "'" + e.key + "' takes [x y z] or a { mean, stddev, stat, nsamples } block");
        }
      }
      else return misplaced(e, "lattice");
    }
    return true;
  }

  bool grain(const Node& n, Structure& s) {
    if (!object(n)) return false;
    for (const Node& e : n.kids) {
      double v;
      if (e.key == "unitcell:key") { if (!string(e, s.unitcell_key)) return false; }
      else if (e.key == "layer:key") { if (!string(e, s.layer_key)) return false; in.struct_in_layer = true; }
      else if (e.key == "lattice") { if (!lattice(e, s)) return false; }
      else if (e.key == "transvec") { if (!vec(e, s.transvec)) return false; }
      else if (e.key == "repetition") { if (!vec(e, s.repetition)) return false; }
      else if (e.key == "scaling") {
        if (e.type == Node::NUM) s.scaling_mean = {{e.num, e.num, e.num}};
        else if (e.type == Node::ARR) { if (!vec(e, s.scaling_mean)) return false; }
        else return fail(e, "'scaling' takes a number or [3 numbers]");
      }
      else if (e.key == "repetitiondist") {
        if (!object(e)) return false;
        for (const Node& f : e.kids) {
          if (f.key == "xrepetition") { if (!repetition_axis(f, s.xrep)) return false; }
          else if (f.key == "yrepetition") { if (!repetition_axis(f, s.yrep)) return false; }
          else if (f.key == "zrepetition") { if (!repetition_axis(f, s.zrep)) return false; }
          else return misplaced(f, "repetitiondist");
        }
        s.repetition_dist = true;
      }
      else if (e.key == "type") {  // paracrystal / percusyevick (hig_input.cpp:1561-1594)
        std::string t;
        if (!string(e, t)) return false;
        if (t == "paracrystal") {
          s.type = "paracrystal";
          s.pc_dims = 1;
          s.pc_dist_set[0] = s.pc_dist_set[1] = s.pc_sdev_set[0] = s.pc_sdev_set[1] = false;
          s.pc_domain_set = false;
        } else if (t == "percusyevick") {
          s.type = "percusyevick";
          s.py_dims = 2;
          s.py_volfract_set = false;
          if (in.shapes.size() == 1) {
            const Shape& sh = in.shapes.begin()->second;
            if (sh.name != "sphere") return fail(e, "Percus-Yevick needs a sphere");
            auto r = sh.params.find("radius");
            s.py_diameter = 2. * (r == sh.params.end() ? 0.0 : r->second.min);
            s.py_diameter_set = true;
          } else if (in.shapes.size() > 1) {
            return fail(e, "Percus-Yevick with more than one shape defined is not supported");
          } else {
            return fail(e, "Percus-Yevick needs a sphere shape defined before the structure");
          }
        }
      }
      else if (e.key == "dimensions") {
        if (!number(e, v)) return false;
        if (s.type == "paracrystal") s.pc_dims = (int)v;
        else if (s.type == "percusyevick") s.py_dims = (int)v;
      }
      else if (e.key == "domain") {
        if (!number(e, v)) return false;
        if (s.type != "paracrystal") return fail(e, "'domain' needs type = \"paracrystal\" first");
        s.pc_domain = v;
        s.pc_domain_set = true;
      }
      else if (e.key == "xspacing" || e.key == "yspacing") {
        if (!object(e)) return false;
        if (s.type != "paracrystal") return fail(e, "'" + e.key + "' needs type = \"paracrystal\" first");
        const int k = e.key[0] == 'y' ? 0 : 1;  // dist_[0] is y, dist_[1] is x
        for (const Node& f : e.kids) {
          if (f.key == "mean") { if (!number(f, s.pc_dist[k])) return false; s.pc_dist_set[k] = true; }
          else if (f.key == "stddev") { if (!number(f, s.pc_sdev[k])) return false; s.pc_sdev_set[k] = true; }
          else return misplaced(f, e.key.c_str());
        }
        if (k == 1 && s.pc_dims == 1) return fail(e, "'xspacing' needs a 2-dimensional paracrystal");
      }
      else if (e.key == "volfraction") {
        if (!number(e, v)) return false;
        if (s.type != "percusyevick") return fail(e, "'volfraction' needs type = \"percusyevick\" first");
        s.py_volfract = v;
        s.py_volfract_set = true;
        if (v <= 0) return fail(e, "'volfraction' must be > 0 (it also sets the iratio)");
        s.iratio = v;
      }
      else return misplaced(e, "grain");
    }
    if (s.type == "paracrystal" && s.pc_dims != 1 && s.pc_dims != 2)
      return fail(n, "a paracrystal has 1 or 2 dimensions");
    if (s.type == "percusyevick" && s.py_dims != 2 && s.py_dims != 3)
      return fail(n, "a Percus-Yevick structure has 2 or 3 dimensions");
    return true;
  }

  bool rotation(const Node& n, Rotation& r) {
    if (!object(n)) return false;
    for (const Node& e : n.kids) {
      if (e.key == "axis") { std::string a; if (!string(e, a)) return false; r.axis = a.empty() ? '\0' : a[0]; }
      else if (e.key == "angles") { if (!vec(e, r.angles)) return false; }
      else if (e.key == "anglemean") { if (!number(e, r.mean)) return false; r.mean_set = true; }
      else if (e.key == "anglesd") { if (!number(e, r.sd)) return false; }
      else if (e.key == "anglelocation") { if (!number(e, r.location)) return false; }
      else if (e.key == "anglescale") { if (!number(e, r.scale)) return false; }
      else return misplaced(e, n.key.c_str());
    }
    return true;
  }

  bool ensemble(const Node& n, Structure& s) {
    if (!object(n)) return false;
    for (const Node& e : n.kids) {
      if (e.key == "spacing") { if (!vec(e, s.spacing)) return false; }
      else if (e.key == "maxgrains") { if (!vec(e, s.maxgrains)) return false; }
      else if (e.key == "distribution") { if (!string(e, s.distribution)) return false; }
      else if (e.key == "orientations") {
        if (!object(e)) return false;
        for (const Node& f : e.kids) {
          if (f.key == "stat") { if (!string(f, s.orientation_stat)) return false; }
          else if (f.key == "rot1") { if (!rotation(f, s.rot1)) return false; }
          else if (f.key == "rot2") { if (!rotation(f, s.rot2)) return false; }
          else if (f.key == "rot3") { if (!rotation(f, s.rot3)) return false; }
          else return misplaced(f, "orientations");
        }
      }
      else return misplaced(e, "ensemble");
    }
    return true;
  }

  bool structure(const Node& n) {
    if (!object(n)) return false;
    Structure s;
    Rotation* rots[3] = {&s.rot1, &s.rot2, &s.rot3};
    const char axes[3] = {'x', 'y', 'z'};
    for (int k = 0; k < 3; ++k) {  // GrainOrientations::init keeps the carried extras
      *rots[k] = rot_extra[k];
      rots[k]->axis = axes[k];
      rots[k]->angles = {{0.0, 0.0}};
    }
    s.xrep = rep_carry[0];
    s.yrep = rep_carry[1];
    s.zrep = rep_carry[2];
    for (const Node& e : n.kids) {
      double v;
      if (e.key == "key") { if (!string(e, s.key)) return false; }
      else if (e.key == "iratio") {
        if (!number(e, v)) return false;
        if (v <= 0) return fail(e, "'iratio' must be > 0");
        s.iratio = v;
      }
      else if (e.key == "grain") { if (!grain(e, s)) return false; }
      else if (e.key == "ensemble") { if (!ensemble(e, s)) return false; }
      else if (e.key == "type") { std::string t; if (!string(e, t)) return false; }  // read, unused
      else return misplaced(e, "structure");
    }
    for (int k = 0; k < 3; ++k) rot_extra[k] = *rots[k];
    rep_carry[0] = s.xrep;
    rep_carry[1] = s.yrep;
    rep_carry[2] = s.zrep;
    // Lattice::construct_vectors (its result is not checked by the reference's reader)
    if (!s.lattice.abc_set) {
      double abc9[9], t3[3];
      if (lattice_table(lattice_code(s.lattice.type), s.lattice.hkl, abc9, t3)) {
        for (int k = 0; k < 3; ++k) {
          s.lattice.a[k] = abc9[k];
          s.lattice.b[k] = abc9[3 + k];
          s.lattice.c[k] = abc9[6 + k];
          s.lattice.t[k] = t3[k];
        }
      }
    }
    if (!in.structures.count(s.key)) in.structure_order.push_back(s.key);
    in.structures[s.key] = s;
    return true;
  }

  bool range3(const Node& n, vec3& r) {  // { min, max, step }
    if (!object(n)) return false;
    for (const Node& e : n.kids) {
      if (e.key == "min") { if (!number(e, r[0])) return false; }
      else if (e.key == "max") { if (!number(e, r[1])) return false; }
      else if (e.key == "step") { if (!number(e, r[2])) return false; }
      else return misplaced(e, n.key.c_str());
    }
    return true;
  }

  bool instrumentation(const Node& n) {
    if (!object(n)) return false;
    for (const Node& e : n.kids) {
      if (e.key == "scattering") {
        if (!object(e)) return false;
        Scattering& sc = in.scattering;
        for (const Node& f : e.kids) {
          if (f.key == "expt") { if (!string(f, sc.expt)) return false; }
          else if (f.key == "alphai") {
            if (!range3(f, sc.alphai)) return false;
            for (const Node& g : f.kids)
              if (g.key == "step") sc.inplanerot[2] = g.num;  // falls through in the reference
          }
          else if (f.key == "inplanerot") { if (!range3(f, sc.inplanerot)) return false; }
          else if (f.key == "tilt") { if (!range3(f, sc.tilt)) return false; }
          else if (f.key == "photon") {
            if (!object(f)) return false;
            for (const Node& g : f.kids) {
              if (g.key == "value") { if (!number(g, sc.photon_value)) return false; }
              else if (g.key == "unit") { if (!string(g, sc.photon_unit)) return false; }
              else return misplaced(g, "photon");
            }
          }
          else if (f.key == "polarization") { if (!string(f, sc.polarization)) return false; }
          else if (f.key == "coherence") { if (!number(f, sc.coherence)) return false; }
          else if (f.key == "spotarea") { if (!number(f, sc.spotarea)) return false; }
          else if (f.key == "smearing") { if (!number(f, sc.smearing)) return false; }
          else return misplaced(f, "scattering");
        }
      } else if (e.key == "detector") {
        if (!object(e)) return false;
        Detector& d = in.detector;
        for (const Node& f : e.kids) {
          if (f.key == "origin") { if (!string(f, d.origin)) return false; }
          else if (f.key == "totalpixels") { if (!vec(f, d.totalpixels)) return false; }
          else if (f.key == "sdd") { if (!number(f, d.sdd)) return false; }
          else if (f.key == "pixelsize") { if (!number(f, d.pixelsize)) return false; }
          else if (f.key == "directbeam") { if (!vec(f, d.directbeam)) return false; }
          else return misplaced(f, "detector");
        }
      } else {
        return misplaced(e, "instrumentation");
      }
    }
    return true;
  }

  bool computation(const Node& n) {
    if (!object(n)) return false;
    Compute& c = in.compute;
    for (const Node& e : n.kids) {
      double v;
      std::string str;
      if (e.key == "pathprefix") { if (!string(e, c.pathprefix)) return false; }
      else if (e.key == "runname") { if (!string(e, c.runname)) return false; c.runname_set = true; }
      else if (e.key == "method") { if (!string(e, c.method)) return false; }
      else if (e.key == "outputregion") {
        if (!object(e)) return false;
        for (const Node& f : e.kids) {
          if (f.key == "type") { if (!string(f, str)) return false; c.region_type = lookup(kRegions, str); }
          else if (f.key == "minpoint") { if (!vec(f, c.minpoint)) return false; }
          else if (f.key == "maxpoint") { if (!vec(f, c.maxpoint)) return false; }
          else return misplaced(f, "outputregion");
        }
      }
      else if (e.key == "resolution") {
        vec2 r;
        if (!vec(e, r)) return false;
        c.resolution[0] = (int)r[0];
        c.resolution[1] = (int)r[1];
      }
      else if (e.key == "nslices") {
        if (!number(e, v)) return false;
        if (v < 0) return fail(e, "'nslices' must be >= 0");
        c.nslices = (unsigned)v;
      }
      else if (e.key == "structcorrelation") { if (!string(e, str)) return false; c.structcorrelation = lookup(kCorrelations, str); }
      else if (e.key == "palette") { if (!string(e, c.palette)) return false; }
      else if (e.key == "saveff") { if (!string(e, str)) return false; c.saveff = boolean(str); c.saveff_set = true; }
      else if (e.key == "savesf") { if (!string(e, str)) return false; c.savesf = boolean(str); c.savesf_set = true; }
      else return misplaced(e, "computation");
    }
    return true;
  }

  bool fitting(const Node& n) {
    if (!object(n)) return false;
    for (const Node& e : n.kids) {
      double v;
      std::string str;
      if (e.key == "fitparam") {  // hig_input.cpp:287-303
        if (!object(e)) return false;
        FitParam p;
        for (const Node& f : e.kids) {
          if (f.key == "key") { if (!string(f, p.key)) return false; }
          else if (f.key == "variable") { if (!string(f, p.variable)) return false; }
          else if (f.key == "range") { if (!range3(f, p.range)) return false; }
          else if (f.key == "init") { if (!number(f, p.init)) return false; }
          else return misplaced(f, "fitparam");
        }
        if (p.key.empty() || p.variable.empty()) return fail(e, "a fitparam needs a key and a variable");
        if (in.fit_params.count(p.key)) return fail(e, "fitparam key '" + p.key + "' used twice");
        in.fit_params[p.key] = p;
      } else if (e.key == "referencedata") {
        if (!object(e)) return false;
        FitReferenceData& r = in.reference_data;
        for (const Node& f : e.kids) {
          if (f.key == "path") { if (!string(f, r.path)) return false; r.path_set = true; }
          else if (f.key == "mask") { if (!string(f, r.mask)) return false; r.mask_set = true; }
          else if (f.key == "fitregion") {
            if (!object(f)) return false;
            for (const Node& g : f.kids) {
              if (g.key == "type") { if (!string(g, str)) return false; r.region_type = lookup(kRegions, str); r.region_type_set = true; }
              else if (g.key == "regmin") { if (!vec(g, r.region_min)) return false; r.region_min_set = true; }
              else if (g.key == "regmax") { if (!vec(g, r.region_max)) return false; r.region_max_set = true; }
              else return misplaced(g, "fitregion");
            }
          } else if (f.key == "npoints") {
            if (!object(f)) return false;
            for (const Node& g : f.kids) {
              if (g.key == "parallel") { if (!number(g, v)) return false; r.npoints_parallel = (unsigned)v; r.npar_set = true; }
              else if (g.key == "perpendicular") { if (!number(g, v)) return false; r.npoints_perpendicular = (unsigned)v; r.nperp_set = true; }
              else return misplaced(g, "npoints");
            }
          } else {
            return misplaced(f, "referencedata");
          }
        }
        in.reference_data_set = true;
      } else if (e.key == "algorithm") {
        if (!object(e)) return false;
        FitAlgorithm a = algo_carry;
        a.params.clear();
        for (const Node& f : e.kids) {
          if (f.key == "algoname") {
            if (!string(f, a.name_str)) return false;
            a.name = lookup(kAlgorithms, a.name_str);
            a.name_set = true;
          }
          else if (f.key == "algoorder") { if (!number(f, v)) return false; a.order = (int)v; a.order_set = true; }
          else if (f.key == "tolerance") { if (!number(f, a.tolerance)) return false; a.tolerance_set = true; }
          else if (f.key == "regularization") { if (!number(f, a.regularization)) return false; }
          else if (f.key == "distancemetric") { if (!string(f, str)) return false; a.distance_metric = lookup(kMetrics, str); a.metric_set = true; }
          else if (f.key == "restart") { if (!string(f, str)) return false; a.restart = boolean(str); a.restart_set = true; }
          else if (f.key == "algoparam") {
            if (!object(f)) return false;
            std::string type = "null";
            double value = 0.0;
            for (const Node& g : f.kids) {
              if (g.key == "type") { if (!string(g, str)) return false; type = lookup(kAlgoParams, str); }
              else if (g.key == "pvalue") { if (!number(g, value)) return false; }
              else return misplaced(g, "algoparam");
            }
            a.params[type] = value;
          }
          else return misplaced(f, "algorithm");
        }
        in.algorithms.push_back(a);
        algo_carry = a;
      } else {
        return misplaced(e, "fitting");
      }
    }
    return true;
  }

  bool top(const Node& root) {
    for (const Node& e : root.kids) {
      bool ok;
      if (e.key == "shape") ok = shape(e);
      else if (e.key == "layer") ok = layer(e);
      else if (e.key == "unitcell") ok = unitcell(e);
      else if (e.key == "structure") ok = structure(e);
      else if (e.key == "instrumentation") ok = instrumentation(e);
      else if (e.key == "computation") ok = computation(e);
      else if (e.key == "fitting") ok = fitting(e);
      else ok = misplaced(e, "hipGisaxsInput");
      if (!ok) return false;
    }
    return true;
  }
};

// ---------------------------------------------------------------------------- json ----

struct Json {
  std::string s;
  void num(double v) {
    if (isnan(v)) { s += "NaN"; return; }
    if (isinf(v)) { s += v > 0 ? "Infinity" : "-Infinity"; return; }
    char b[40];
    snprintf(b, sizeof b, "%.17g", v);
    s += b;
  }
  void str(const std::string& v) {
    s += '"';
    for (char c : v) {
      if (c == '"' || c == '\\') { s += '\\'; s += c; }
      else if ((unsigned char)c < 0x20) { char b[8]; snprintf(b, sizeof b, "\\u%04x", c); s += b; }
      else s += c;
    }
    s += '"';
  }
  void key(const std::string& k) { str(k); s += ": "; }
  template <size_t N>
  void arr(const std::array<double, N>& v) {
    s += '[';
    for (size_t i = 0; i < N; ++i) { if (i) s += ", "; num(v[i]); }
    s += ']';
  }
  void open() { s += '{'; }
  void close() { s += '}'; }
  void comma() { s += ", "; }
};

}  // namespace

bool read_input(const std::string& path, Input& out, std::string& err) {
  out = Input();
  out.path = path;
  Lexer lx;
  std::vector<Tok> toks;
  if (!lx.lex_file(path, toks, 0)) { err = lx.err; return false; }
  if (!check_order(toks, lx, err)) return false;
  Parser ps(toks, lx);
  Node root;
  if (!ps.file(root)) { err = ps.err; return false; }
  Builder b(out, lx);
  if (!b.top(root)) { err = b.err; return false; }
  return true;
}

// ---------------------------------------------------------------- parameter updates ----

namespace {

// extract_first_keyword / extract_keyword_name_and_key (src/utils/string_utils.cpp:23-90)
void first_keyword(const std::string& str, std::string& kw, std::string& rest) {
  const size_t pos = str.find(':');
  kw = str.substr(0, pos);
  rest = pos == std::string::npos ? "" : str.substr(pos + 1);
}
bool name_and_key(const std::string& kw, std::string& name, std::string& key) {
  const size_t pos = kw.find('[');
  if (pos == std::string::npos) { name = kw; key = ""; return true; }
  name = kw.substr(0, pos);
  std::string rem = kw.substr(pos + 1);
  if (rem.empty() || rem.back() != ']') return false;
  rem.pop_back();
  if (rem.size() < 2 || rem.front() != '\'' || rem.back() != '\'') return false;
  key = rem.substr(1, rem.size() - 2);
  return true;
}
// "x"/"0", "y"/"1", "z"/"2" -> 0, 1, 2; -1 otherwise
int coordinate(const std::string& c) {
  if (c == "x" || c == "0") return 0;
  if (c == "y" || c == "1") return 1;
  if (c == "z" || c == "2") return 2;
  return -1;
}

struct Updater {
  Input& in;
  std::string err;
  bool bad(const std::string& m) { err = m; return false; }

  bool shape_param(ShapeParam& p, const std::string& rest, double v) {  // shape.cpp:114-150
    std::string kw, r2, name, key;
    first_keyword(rest, kw, r2);
    if (!name_and_key(kw, name, key)) return bad("malformed keyword '" + kw + "'");
    if (name == "min") p.min = v;
    else if (name == "max") p.max = v;
    else if (name == "p1") p.p1 = v;
    else if (name == "p2") p.p2 = v;
    else if (name == "nvalues") p.nvalues = (int)v;
    else if (name == "stat") {}
    else return bad("'" + name + "' is not a shape parameter field");
    return true;
  }

  bool shape(Shape& s, const std::string& rest, double v) {  // Shape::update_param, shape.cpp:190-247
    std::string kw, r2, name, key, coord, r3;
    first_keyword(rest, kw, r2);
    if (!name_and_key(kw, name, key)) return bad("malformed keyword '" + kw + "'");
    if (name == "key" || name == "name" || name == "originvec") {  // all three set originvec
      first_keyword(r2, coord, r3);
      const int c = coordinate(coord);
      if (c < 0) return bad("'" + coord + "' is not a coordinate");
      s.originvec[c] = v;
    } else if (name == "zrot") {
      s.zrot = v;  // radians: the update takes the value as it is
    } else if (name == "yrot") {
      s.yrot = v;
    } else if (name == "xrot") {
      return bad("'xrot' cannot be updated (the reference falls through into the parameter "
                 "branch and throws)");
    } else if (name == "param") {
      auto it = s.params.find(key);
      if (it == s.params.end()) return bad("shape '" + s.key + "' has no parameter '" + key + "'");
      return shape_param(it->second, r2, v);
    } else {
      return bad("'" + name + "' cannot be updated in a shape");
    }
    return true;
  }

  bool layer(Layer& l, const std::string& rest, double v) {  // Layer::update_param, layer.cpp
    std::string kw, r2, kw2, r3;
    first_keyword(rest, kw, r2);
    if (kw == "key" || kw == "order") return true;
    if (kw == "thickness") { l.thickness = v; return true; }
    if (kw == "refindex") {
      first_keyword(r2, kw2, r3);
      if (kw2 == "beta") { l.refindex.beta = v; return true; }
      if (kw2 == "delta") { l.refindex.delta = v; return true; }
      return bad("'" + kw2 + "' is not a refindex field");
    }
    return bad("'" + kw + "' cannot be updated in a layer");
  }

  bool rotation(Rotation& r, const std::string& name, const std::string& key, const std::string& rest,
                double v) {  // GrainOrientations::update_param, structure.cpp:237-330
    if (key != std::string(1, r.axis)) return bad("'" + name + "' is about axis '" + std::string(1, r.axis) + "'");
    std::string kw2, r2;
    first_keyword(rest, kw2, r2);
    if (kw2 == "min" || kw2 == "0") {
      r.angles[0] = v;
      if (!r.mean_set) r.mean = v;  // Rotation::angles_min
    } else if (kw2 == "max" || kw2 == "1") {
      if (name == "rot2") {  // the reference sets rot2's minimum here
        r.angles[0] = v;
        if (!r.mean_set) r.mean = v;
      } else {
        r.angles[1] = v;
      }
    } else if (kw2 == "anglelocation") r.location = v;
    else if (kw2 == "anglemean") { r.mean = v; r.mean_set = true; }
    else if (kw2 == "anglescale") r.scale = v;
    else if (kw2 == "anglesd") r.sd = v;
    else return bad("'" + kw2 + "' is not an orientation field");
    return true;
  }

  bool structure(Structure& s, const std::string& rest, double v) {  // structure.cpp:486-820
    std::string kw, r2, kw2, r3, kw3, r4, kw4, r5;
    first_keyword(rest, kw, r2);
    if (kw == "key") return true;
    if (kw == "iratio") { s.iratio = v; return true; }
    if (kw == "grain") {
      first_keyword(r2, kw2, r3);
      if (kw2 == "refindex") {
        first_keyword(r3, kw3, r4);
        if (kw3 == "delta") { s.grain_refindex.delta = v; return true; }
        if (kw3 == "beta") { s.grain_refindex.beta = v; return true; }
        return bad("'" + kw3 + "' is not a refindex field");
      }
      if (kw2 == "lattice") {
        first_keyword(r3, kw3, r4);
        if (kw3 == "a" || kw3 == "b" || kw3 == "c") {
          first_keyword(r4, kw4, r5);
          const int c = coordinate(kw4);
          if (c < 0) return bad("'" + kw4 + "' is not a coordinate");
          vec3& vec = kw3 == "a" ? s.lattice.a : kw3 == "b" ? s.lattice.b : s.lattice.c;
          vec[c] = v;
          return true;
        }
        if (kw3 == "type" || kw3 == "hkl") return true;  // immutable: a warning, no change
        if (kw3 == "abangle") { s.lattice.abangle = v; return true; }
        if (kw3 == "caratio") { s.lattice.caratio = v; return true; }
        return bad("'" + kw3 + "' cannot be updated in a lattice");
      }
      if (kw2 == "scaling") {
        if (r3.empty()) { s.scaling_mean = {{v, v, v}}; return true; }
        first_keyword(r3, kw3, r4);
        if (kw3 == "a" || kw3 == "b" || kw3 == "c") {
          const int ax = kw3[0] - 'a';
          first_keyword(r4, kw4, r5);
          if (kw4 == "mean") s.scaling_mean[ax] = v;
          else if (kw4 == "stddev") s.scaling_stddev[ax] = v;
          else if (kw4 == "nsamples") s.scaling_nsamples[ax] = (int)v;
          else return bad("'" + kw4 + "' is not a scaling field");
          return true;
        }
        return bad("'" + kw3 + "' is not a scaling axis");
      }
      if (kw2 == "transvec" || kw2 == "repetition") {
        first_keyword(r3, kw3, r4);
        const int c = coordinate(kw3);
        if (c < 0) return bad("'" + kw3 + "' is not a coordinate");
        (kw2 == "transvec" ? s.transvec : s.repetition)[c] = v;
        return true;
      }
      return bad("'" + kw2 + "' cannot be updated in a grain");
    }
    if (kw == "ensemble") {
      first_keyword(r2, kw2, r3);
      if (kw2 == "spacing" || kw2 == "maxgrains") {
        first_keyword(r3, kw3, r4);
        // x/0, y/1, and z only by name: the reference tests "1" again instead of "2"
        const int c = (kw3 == "x" || kw3 == "0") ? 0 : (kw3 == "y" || kw3 == "1") ? 1 : kw3 == "z" ? 2 : -1;
        if (c < 0) return bad("'" + kw3 + "' is not a coordinate here");
        (kw2 == "spacing" ? s.spacing : s.maxgrains)[c] = v;
        return true;
      }
      if (kw2 == "orientations") {
        first_keyword(r3, kw3, r4);
        std::string name, key;
        if (!name_and_key(kw3, name, key)) return bad("malformed keyword '" + kw3 + "'");
        if (name == "rot1") return rotation(s.rot1, name, key, r4, v);
        if (name == "rot2") return rotation(s.rot2, name, key, r4, v);
        if (name == "rot3") return rotation(s.rot3, name, key, r4, v);
        return bad("'" + name + "' cannot be updated in orientations");
      }
      if (kw2 == "distribution") return true;
      return bad("'" + kw2 + "' cannot be updated in an ensemble");
    }
    return bad("'" + kw + "' cannot be updated in a structure");
  }

  bool range(vec3& r, const std::string& rest, double v) {
    std::string kw, r2;
    first_keyword(rest, kw, r2);
    if (kw == "min") r[0] = v;
    else if (kw == "max") r[1] = v;
    else if (kw == "step") r[2] = v;
    else return bad("'" + kw + "' is not min, max or step");
    return true;
  }

  bool scattering(const std::string& rest, double v) {  // inst_scattering.cpp:36-120
    Scattering& sc = in.scattering;
    std::string kw, r2, kw2, r3;
    first_keyword(rest, kw, r2);
    if (kw == "expt" || kw == "polarization" || kw == "smearing") return true;
    if (kw == "alphai") return range(sc.alphai, r2, v);
    if (kw == "inplanerot") return range(sc.inplanerot, r2, v);
    if (kw == "tilt") return range(sc.tilt, r2, v);
    if (kw == "photon") {
      first_keyword(r2, kw2, r3);
      if (kw2 == "value") { sc.photon_value = v; return true; }
      if (kw2 == "unit") return true;
      return bad("'" + kw2 + "' is not a photon field");
    }
    if (kw == "coherence") { sc.coherence = v; return true; }
    if (kw == "spotarea") { sc.spotarea = v; return true; }
    return bad("'" + kw + "' cannot be updated in scattering");
  }

  bool detector(const std::string& rest, double v) {  // inst_detector.cpp:35-60
    std::string kw, r2;
    first_keyword(rest, kw, r2);
    if (kw == "origin" || kw == "totalpixels" || kw == "directbeam") return true;
    if (kw == "pixelsize") { in.detector.pixelsize = v; return true; }
    if (kw == "sdd") { in.detector.sdd = v; return true; }
    return bad("'" + kw + "' cannot be updated in the detector");
  }

  bool top(const std::string& var, double v) {  // HiGInput::update_params, hig_input.cpp:2712-2830
    std::string kw, rest, name, key, kw2, r2;
    if (var.empty()) return bad("empty parameter variable");
    first_keyword(var, kw, rest);
    if (!name_and_key(kw, name, key)) return bad("malformed keyword '" + kw + "'");
    if (name == "shape") {
      auto it = in.shapes.find(key);
      if (it == in.shapes.end()) return bad("no shape '" + key + "'");
      return shape(it->second, rest, v);
    }
    if (name == "layer") {
      auto lk = in.layer_keys.find(key);
      if (lk == in.layer_keys.end() || !in.layers.count(lk->second)) return bad("no layer '" + key + "'");
      return layer(in.layers[lk->second], rest, v);
    }
    if (name == "structure") {
      auto it = in.structures.find(key);
      if (it == in.structures.end()) return bad("no structure '" + key + "'");
      return structure(it->second, rest, v);
    }
    if (name == "instrumentation") {
      first_keyword(rest, kw2, r2);
      if (kw2 == "scattering") return scattering(r2, v);
      if (kw2 == "detector") return detector(r2, v);
      return bad("'" + kw2 + "' cannot be updated in instrumentation");
    }
    if (name == "computation") {  // ComputeParams::update_param: nothing changes
      first_keyword(rest, kw2, r2);
      if (kw2 == "pathprefix" || kw2 == "runname" || kw2 == "method" || kw2 == "outputregion" ||
          kw2 == "resolution" || kw2 == "nslices")
        return true;
      return bad("'" + kw2 + "' cannot be updated in computation");
    }
    return bad("'" + name + "' is not an updatable block");
  }
};

}  // namespace

bool update_param(Input& in, const std::string& variable, double value, std::string& err) {
  Updater u{in, ""};
  if (!u.top(variable, value)) {
    err = "parameter '" + variable + "': " + u.err;
    return false;
  }
  return true;
}

bool photon_k0(const Scattering& s, double* k0, double* freq) {
  double photon = s.photon_value;
  if (s.photon_unit == "ev") photon = photon / 1000;  // in keV
  else if (s.photon_unit != "kev") return false;
  const double lambda = 1.23984 / photon;
  if (freq) *freq = 1e-9 * photon * 1.60217646e-19 * 1000 / 6.626068e-34;
  if (k0) *k0 = 2 * PI / lambda;
  return true;
}

std::string to_json(const Input& in) {
  Json j;
  j.open();
  // shapes
  j.key("shapes"); j.open();
  bool first = true;
  for (const auto& kv : in.shapes) {
    if (!first) j.comma();
    first = false;
    const Shape& s = kv.second;
    j.key(kv.first); j.open();
    j.key("name"); j.str(s.name); j.comma();
    j.key("name_str"); j.str(s.name_str); j.comma();
    j.key("originvec"); j.arr(s.originvec); j.comma();
    j.key("rot"); j.arr(vec3{{s.zrot, s.yrot, s.xrot}}); j.comma();
    j.key("refindex"); j.arr(vec2{{s.refindex.delta, s.refindex.beta}}); j.comma();
    j.key("params"); j.open();
    bool f2 = true;
    for (const auto& pk : s.params) {
      if (!f2) j.comma();
      f2 = false;
      const ShapeParam& p = pk.second;
      j.key(pk.first); j.open();
      j.key("type"); j.str(p.type); j.comma();
      j.key("stat"); j.str(p.stat); j.comma();
      j.key("min"); j.num(p.min); j.comma();
      j.key("max"); j.num(p.max); j.comma();
      j.key("p1"); j.num(p.p1); j.comma();
      j.key("p2"); j.num(p.p2); j.comma();
      j.key("nvalues"); j.num(p.nvalues);
      j.close();
    }
    j.close(); j.close();
  }
  j.close(); j.comma();
  // layers
  j.key("layers"); j.open();
  first = true;
  for (const auto& kv : in.layers) {
    if (!first) j.comma();
    first = false;
    const Layer& l = kv.second;
    j.key(std::to_string(kv.first)); j.open();
    j.key("key"); j.str(l.key); j.comma();
    j.key("order"); j.num(l.order); j.comma();
    j.key("thickness"); j.num(l.thickness); j.comma();
    j.key("refindex"); j.arr(vec2{{l.refindex.delta, l.refindex.beta}});
    j.close();
  }
  j.close(); j.comma();
  j.key("layer_keys"); j.open();
  first = true;
  for (const auto& kv : in.layer_keys) {
    if (!first) j.comma();
    first = false;
    j.key(kv.first); j.num(kv.second);
  }
  j.close(); j.comma();
  // unit cells
  j.key("unitcells"); j.open();
  first = true;
  for (const auto& kv : in.unitcells) {
    if (!first) j.comma();
    first = false;
    j.key(kv.first); j.open();
    bool f2 = true;
    for (const auto& el : kv.second.elements) {
      if (!f2) j.comma();
      f2 = false;
      j.key(el.first); j.s += '[';
      for (size_t i = 0; i < el.second.size(); ++i) { if (i) j.comma(); j.arr(el.second[i]); }
      j.s += ']';
    }
    j.close();
  }
  j.close(); j.comma();
  // structures
  j.key("structures"); j.open();
  first = true;
  for (const auto& kv : in.structures) {
    if (!first) j.comma();
    first = false;
    const Structure& s = kv.second;
    j.key(kv.first); j.open();
    j.key("iratio"); j.num(s.iratio); j.comma();
    j.key("type"); j.str(s.type); j.comma();
    j.key("unitcell_key"); j.str(s.unitcell_key); j.comma();
    j.key("layer_key"); j.str(s.layer_key); j.comma();
    j.key("layer_order"); j.num(s.layer_order); j.comma();
    j.key("lattice"); j.open();
    j.key("type"); j.str(s.lattice.type); j.comma();
    j.key("hkl"); j.str(s.lattice.hkl); j.comma();
    j.key("abc_set"); j.s += s.lattice.abc_set ? "true" : "false"; j.comma();
    j.key("a"); j.arr(s.lattice.a); j.comma();
    j.key("b"); j.arr(s.lattice.b); j.comma();
    j.key("c"); j.arr(s.lattice.c); j.comma();
    j.key("t"); j.arr(s.lattice.t); j.comma();
    j.key("abangle"); j.num(s.lattice.abangle); j.comma();
    j.key("caratio"); j.num(s.lattice.caratio);
    j.close(); j.comma();
    j.key("transvec"); j.arr(s.transvec); j.comma();
    j.key("repetition"); j.arr(s.repetition); j.comma();
    j.key("repetition_dist"); j.s += s.repetition_dist ? "true" : "false"; j.comma();
    j.key("scaling_mean"); j.arr(s.scaling_mean); j.comma();
    j.key("scaling_stddev"); j.arr(s.scaling_stddev); j.comma();
    j.key("scaling_stat"); j.s += '[';
    for (int k = 0; k < 3; ++k) { if (k) j.comma(); j.str(s.scaling_stat[k]); }
    j.s += ']'; j.comma();
    j.key("scaling_nsamples"); j.arr(vec3{{(double)s.scaling_nsamples[0], (double)s.scaling_nsamples[1], (double)s.scaling_nsamples[2]}}); j.comma();
    j.key("spacing"); j.arr(s.spacing); j.comma();
    j.key("maxgrains"); j.arr(s.maxgrains); j.comma();
    j.key("distribution"); j.str(s.distribution); j.comma();
    j.key("orientation_stat"); j.str(s.orientation_stat);
    const Rotation* rots[3] = {&s.rot1, &s.rot2, &s.rot3};
    for (int k = 0; k < 3; ++k) {
      const Rotation& r = *rots[k];
      j.comma();
      j.key("rot" + std::to_string(k + 1)); j.open();
      j.key("axis"); j.str(std::string(1, r.axis)); j.comma();
      j.key("angles"); j.arr(r.angles); j.comma();
      j.key("mean"); j.num(r.mean); j.comma();
      j.key("sd"); j.num(r.sd); j.comma();
      j.key("location"); j.num(r.location); j.comma();
      j.key("scale"); j.num(r.scale);
      j.close();
    }
    const Repetition* reps[3] = {&s.xrep, &s.yrep, &s.zrep};
    const char* rep_names[3] = {"xrepetition", "yrepetition", "zrepetition"};
    for (int k = 0; k < 3; ++k) {
      j.comma();
      j.key(rep_names[k]); j.open();
      j.key("stat"); j.str(reps[k]->stat); j.comma();
      j.key("min"); j.num(reps[k]->min); j.comma();
      j.key("max"); j.num(reps[k]->max);
      j.close();
    }
    if (s.type == "paracrystal") {
      j.comma();
      j.key("paracrystal"); j.open();
      j.key("dims"); j.num(s.pc_dims);
      if (s.pc_dist_set[0]) { j.comma(); j.key("ymean"); j.num(s.pc_dist[0]); }
      if (s.pc_dist_set[1]) { j.comma(); j.key("xmean"); j.num(s.pc_dist[1]); }
      if (s.pc_sdev_set[0]) { j.comma(); j.key("ystddev"); j.num(s.pc_sdev[0]); }
      if (s.pc_sdev_set[1]) { j.comma(); j.key("xstddev"); j.num(s.pc_sdev[1]); }
      if (s.pc_domain_set) { j.comma(); j.key("domain"); j.num(s.pc_domain); }
      j.close();
    } else if (s.type == "percusyevick") {
      j.comma();
      j.key("percusyevick"); j.open();
      j.key("dims"); j.num(s.py_dims);
      if (s.py_diameter_set) { j.comma(); j.key("diameter"); j.num(s.py_diameter); }
      if (s.py_volfract_set) { j.comma(); j.key("volfraction"); j.num(s.py_volfract); }
      j.close();
    }
    j.close();
  }
  j.close(); j.comma();
  j.key("struct_in_layer"); j.s += in.struct_in_layer ? "true" : "false"; j.comma();
  // instrumentation
  const Scattering& sc = in.scattering;
  j.key("scattering"); j.open();
  j.key("expt"); j.str(sc.expt); j.comma();
  j.key("alphai"); j.arr(sc.alphai); j.comma();
  j.key("inplanerot"); j.arr(sc.inplanerot); j.comma();
  j.key("tilt"); j.arr(sc.tilt); j.comma();
  j.key("photon_value"); j.num(sc.photon_value); j.comma();
  j.key("photon_unit"); j.str(sc.photon_unit); j.comma();
  j.key("polarization"); j.str(sc.polarization); j.comma();
  j.key("coherence"); j.num(sc.coherence); j.comma();
  j.key("spotarea"); j.num(sc.spotarea); j.comma();
  j.key("smearing"); j.num(sc.smearing);
  j.close(); j.comma();
  const Detector& d = in.detector;
  j.key("detector"); j.open();
  j.key("origin"); j.str(d.origin); j.comma();
  j.key("totalpixels"); j.arr(d.totalpixels); j.comma();
  j.key("pixelsize"); j.num(d.pixelsize); j.comma();
  j.key("sdd"); j.num(d.sdd); j.comma();
  j.key("directbeam"); j.arr(d.directbeam);
  j.close(); j.comma();
  const Compute& c = in.compute;
  j.key("computation"); j.open();
  j.key("pathprefix"); j.str(c.pathprefix); j.comma();
  if (c.runname_set) { j.key("runname"); j.str(c.runname); j.comma(); }
  j.key("method"); j.str(c.method); j.comma();
  j.key("region_type"); j.str(c.region_type); j.comma();
  j.key("minpoint"); j.arr(c.minpoint); j.comma();
  j.key("maxpoint"); j.arr(c.maxpoint); j.comma();
  j.key("resolution"); j.arr(vec2{{(double)c.resolution[0], (double)c.resolution[1]}}); j.comma();
  j.key("nslices"); j.num(c.nslices); j.comma();
  j.key("structcorrelation"); j.str(c.structcorrelation); j.comma();
  j.key("palette"); j.str(c.palette);
  if (c.saveff_set) { j.comma(); j.key("saveff"); j.s += c.saveff ? "true" : "false"; }
  if (c.savesf_set) { j.comma(); j.key("savesf"); j.s += c.savesf ? "true" : "false"; }
  j.close(); j.comma();
  // fitting
  j.key("fitparams"); j.open();
  first = true;
  for (const auto& kv : in.fit_params) {
    if (!first) j.comma();
    first = false;
    j.key(kv.first); j.open();
    j.key("variable"); j.str(kv.second.variable); j.comma();
    j.key("range"); j.arr(kv.second.range); j.comma();
    j.key("init"); j.num(kv.second.init);
    j.close();
  }
  j.close();
  if (in.reference_data_set) {
    const FitReferenceData& r = in.reference_data;
    j.comma();
    j.key("referencedata"); j.open();
    bool f2 = true;
    auto sep = [&]() { if (!f2) j.comma(); f2 = false; };
    if (r.path_set) { sep(); j.key("path"); j.str(r.path); }
    if (r.mask_set) { sep(); j.key("mask"); j.str(r.mask); }
    if (r.region_type_set) { sep(); j.key("region_type"); j.str(r.region_type); }
    if (r.region_min_set) { sep(); j.key("region_min"); j.arr(r.region_min); }
    if (r.region_max_set) { sep(); j.key("region_max"); j.arr(r.region_max); }
    if (r.npar_set) { sep(); j.key("npoints_parallel"); j.num(r.npoints_parallel); }
    if (r.nperp_set) { sep(); j.key("npoints_perpendicular"); j.num(r.npoints_perpendicular); }
    j.close();
  }
  j.comma();
  j.key("algorithms"); j.s += '[';
  for (size_t i = 0; i < in.algorithms.size(); ++i) {
    const FitAlgorithm& a = in.algorithms[i];
    if (i) j.comma();
    j.open();
    j.key("regularization"); j.num(a.regularization);
    if (a.name_set) { j.comma(); j.key("name"); j.str(a.name); j.comma(); j.key("name_str"); j.str(a.name_str); }
    if (a.order_set) { j.comma(); j.key("order"); j.num(a.order); }
    if (a.tolerance_set) { j.comma(); j.key("tolerance"); j.num(a.tolerance); }
    if (a.metric_set) { j.comma(); j.key("distance_metric"); j.str(a.distance_metric); }
    if (a.restart_set) { j.comma(); j.key("restart"); j.s += a.restart ? "true" : "false"; }
    j.comma();
    j.key("params"); j.open();
    bool f2 = true;
    for (const auto& p : a.params) {
      if (!f2) j.comma();
      f2 = false;
      j.key(p.first); j.num(p.second);
    }
    j.close();
    j.close();
  }
  j.s += ']';
  j.close();
  return j.s;
}

}  // namespace hig
}  // namespace hgx

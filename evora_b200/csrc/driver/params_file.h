// params_file.h -- the reference's run parameters as the two drivers read and
// write them: the namelist group para of the parameter file
// (parameter.f90:26-105), its copy data/parameter (writeparameter,
// parameter.f90:267-337) and the post-processor's reading of that copy
// (rereadparameter, parameter.f90:339-411).
#pragma once

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../../include/evora_gpu.h"
#include "../fortran_fmt.h"

namespace evora {
namespace driver {

inline std::string lower(std::string s) {
  for (auto& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

inline bool read_text(const std::string& path, std::string* out) {
  std::ifstream in(path);
  if (!in) return false;
  std::stringstream ss;
  ss << in.rdbuf();
  *out = ss.str();
  return true;
}

// The items of namelist group `name` ('&name' or '$name' up to the closing
// '/', '!' comments dropped) as key -> value text; a key given twice keeps
// its last value, as a namelist read does.
inline bool read_group(const std::string& text, const std::string& name, std::map<std::string, std::string>* out) {
  const std::string t = lower(text);
  size_t pos = std::string::npos;
  for (const char lead : {'&', '$'}) {
    size_t p = 0;
    const std::string key = std::string(1, lead) + name;
    while ((p = t.find(key, p)) != std::string::npos) {
      const size_t e = p + key.size();
      if (e >= t.size() || !(std::isalnum((unsigned char)t[e]) || t[e] == '_')) {
        if (pos == std::string::npos || p < pos) pos = p;
        break;
      }
      p = e;
    }
  }
  if (pos == std::string::npos) return false;
  std::string body;
  bool quote = false;
  for (size_t i = pos + 1 + name.size(); i < t.size(); ++i) {
    const char c = t[i];
    if (c == '\'' || c == '"') quote = !quote;
    if (!quote && c == '!') {
      while (i < t.size() && t[i] != '\n') ++i;
      body += ' ';
      continue;
    }
    if (!quote && c == '/') break;
    body += c;
  }
  std::vector<std::pair<size_t, std::string>> keys;   // (start of key, key)
  for (size_t k = 0; k < body.size(); ++k) {
    if (body[k] != '=') continue;
    size_t e = k;
    while (e > 0 && std::isspace((unsigned char)body[e - 1])) --e;
    size_t b = e;
    while (b > 0 && (std::isalnum((unsigned char)body[b - 1]) || body[b - 1] == '_')) --b;
    if (b < e) keys.push_back({b, body.substr(b, e - b)});
  }
  for (size_t j = 0; j < keys.size(); ++j) {
    const size_t vb = body.find('=', keys[j].first) + 1;
    const size_t ve = j + 1 < keys.size() ? keys[j + 1].first : body.size();
    std::string v = body.substr(vb, ve - vb);
    while (!v.empty() && (std::isspace((unsigned char)v.back()) || v.back() == ',')) v.pop_back();
    size_t s = 0;
    while (s < v.size() && std::isspace((unsigned char)v[s])) ++s;
    (*out)[keys[j].second] = v.substr(s);
  }
  return true;
}

// A namelist real read into a real(8) variable: the decimal text rounded to
// FP64 (a 'd' exponent is an 'e').
inline double to_real(const std::string& v) {
  std::string s = v;
  for (auto& c : s)
    if (c == 'd' || c == 'D') c = 'e';
  return std::strtod(s.c_str(), nullptr);
}

inline bool to_logical(const std::string& v) {
  const std::string s = lower(v);
  const size_t i = s.find_first_not_of(" .");
  return i != std::string::npos && s[i] == 't';
}

// One entry of namelist para: name, edit type (L logical, I integer, E real)
// and the default of parameter.f90:41-82.  Real defaults are default-real
// (single precision) literals there, except j0 = 1d-21.
struct Entry {
  const char* name;
  char type;
  double def;
};

inline double sp(float f) { return (double)f; }

// In the order writeparameter writes them (parameter.f90:279-333).
inline const std::vector<Entry>& entries() {
  static const std::vector<Entry> e = {
      {"iconly", 'L', 0},          {"hydro", 'L', 1},          {"secondorder", 'L', 1},
      {"solver", 'I', 2},          {"limiter", 'I', 1},        {"cfl", 'E', sp(0.5f)},
      {"g", 'E', sp(1.4f)},        {"atomic", 'L', 0},         {"nx", 'I', 32},
      {"ny", 'I', 32},             {"nz", 'I', 32},            {"xmin", 'E', 0.0},
      {"xmax", 'E', 1.0},          {"ymin", 'E', 0.0},         {"ymax", 'E', 1.0},
      {"zmin", 'E', 0.0},          {"zmax", 'E', 1.0},         {"boundtype", 'I', 2},
      {"cut", 'L', 0},             {"slice", 'L', 0},          {"bov", 'L', 0},
      {"nsnap", 'I', 100},         {"gravity", 'L', 0},        {"tstart", 'E', 0.0},
      {"tend", 'E', 1.0},          {"supercomoving", 'L', 0},  {"c_cosmo", 'E', sp(0.1f)},
      {"omega0", 'E', 1.0},        {"lambda0", 'E', 0.0},      {"fb", 'E', 1.0},
      {"hubble0", 'E', 50.0},      {"box", 'E', 1.0},          {"zstart", 'E', 99.0},
      {"zend", 'E', 0.0},          {"chemistry", 'L', 0},      {"noncie", 'L', 0},
      {"cooling", 'L', 0},         {"background", 'L', 0},     {"bg", 'I', 0},
      {"j0", 'E', 1e-21},          {"c_chem", 'E', sp(0.1f)},  {"substep", 'E', sp(0.1f)},
      {"rhoh", 'E', sp(0.76f)},    {"rhohe", 'E', sp(0.24f)},  {"cooldt", 'L', 0},
      {"c_cooldt", 'E', 0.0},      {"tempfloor", 'L', 0},      {"temp_fl", 'E', 0.0},
      {"jeansfloor", 'L', 0},      {"c_jeans", 'E', 0.0},      {"conduction", 'L', 0},
      {"c_cond", 'E', sp(0.1f)},   {"simplekappa", 'L', 0},    {"dualenergy", 'L', 0},
      {"de_thresh", 'E', 0.0}};
  return e;
}

// The labels of writeparameter (16 columns, name as the source spells it).
inline std::string label(const char* name) {
  std::string n = name;
  if (n == "rhoh") n = "rhoH";
  if (n == "rhohe") n = "rhoHe";
  std::string s = n + " =";
  s.resize(16, ' ');
  return s;
}

// The run's parameter values (all of namelist para), keyed by lower-case
// name, and the array dump_redshift (global.f90:137-138).
struct RunParams {
  std::map<std::string, double> v;
  std::vector<double> dump_redshift = std::vector<double>(EVORA_NDUMP, -1.0);   // parameter.f90:82
  double operator[](const char* k) const { return v.at(k); }
  bool flag(const char* k) const { return v.at(k) != 0.0; }
};

inline RunParams defaults() {
  RunParams r;
  for (const auto& e : entries()) r.v[e.name] = e.def;
  return r;
}

// A namelist value list: items separated by commas or blanks, each a value
// or r*value (r repetitions).  False on an item that is not a number.
inline bool value_list(const std::string& text, std::vector<double>* out) {
  std::string t = text;
  for (auto& c : t)
    if (c == ',') c = ' ';
  std::istringstream in(t);
  std::string item;
  while (in >> item) {
    long rep = 1;
    const size_t star = item.find('*');
    if (star != std::string::npos) {
      char* end = nullptr;
      rep = std::strtol(item.c_str(), &end, 10);
      if (end != item.c_str() + star || rep < 1) return false;
      item = item.substr(star + 1);
    }
    std::string s = item;
    for (auto& c : s)
      if (c == 'd' || c == 'D') c = 'e';
    char* end = nullptr;
    const double x = std::strtod(s.c_str(), &end);
    if (end == s.c_str() || *end != '\0') return false;
    for (long i = 0; i < rep; ++i) out->push_back(x);
  }
  return true;
}

// readparameter (parameter.f90:26-105): defaults, then the namelist values.
// Unknown keys are reported in *unknown; dump_redshift takes a value list
// (at most EVORA_NDUMP values, filled from the first element on).
inline void apply_namelist(const std::map<std::string, std::string>& kv, RunParams* r, std::string* unknown) {
  for (const auto& [k, val] : kv) {
    if (k == "dump_redshift") {
      std::vector<double> z;
      if (!value_list(val, &z) || z.size() > (size_t)EVORA_NDUMP) {
        if (unknown) *unknown += (unknown->empty() ? "" : ", ") + std::string("dump_redshift (bad value list)");
        continue;
      }
      for (size_t i = 0; i < z.size(); ++i) r->dump_redshift[i] = z[i];
      continue;
    }
    auto it = r->v.find(k);
    if (it == r->v.end()) {
      if (unknown) *unknown += (unknown->empty() ? "" : ", ") + k;
      continue;
    }
    char type = 'E';
    for (const auto& e : entries())
      if (k == e.name) type = e.type;
    if (type == 'L') it->second = to_logical(val) ? 1.0 : 0.0;
    else if (type == 'I') it->second = (double)std::atol(val.c_str());
    else it->second = to_real(val);
  }
  // parameter.f90:95-104
  if (r->v["chemistry"] == 0.0) {
    r->v["background"] = 0.0;
    r->v["cooling"] = 0.0;
    r->v["cooldt"] = 0.0;
  }
}

// writeparameter (parameter.f90:267-337)
inline std::string parameter_text(const RunParams& r) {
  namespace ft = fortran;
  std::string s;
  for (const auto& e : entries()) {
    const double x = r.v.at(e.name);
    s += label(e.name);
    if (e.type == 'L') s += ft::L(x != 0.0, 16);
    else if (e.type == 'I') s += ft::I((long long)x, 16);
    else s += ft::E(x, 16, 8);
    s += '\n';
  }
  return s;
}

// rereadparameter (parameter.f90:339-411): the values of data/parameter,
// read back through their E16.8 text.  The reference reads the line of
// simplekappa into conduction (parameter.f90:405); neither reaches the hydro
// path.
inline bool reread(const std::string& text, RunParams* r) {
  *r = defaults();
  std::istringstream in(text);
  std::string line;
  size_t i = 0;
  const auto& es = entries();
  while (std::getline(in, line) && i < es.size()) {
    const Entry& e = es[i++];
    const std::string f = line.size() > 16 ? line.substr(16, 16) : "";
    if (e.type == 'L') r->v[e.name] = to_logical(f) ? 1.0 : 0.0;
    else if (e.type == 'I') r->v[e.name] = (double)std::atol(f.c_str());
    else {
      std::string s = f;
      // an E16.8 field with a three-digit exponent has no letter E
      if (s.find_first_of("eEdD") == std::string::npos) {
        const size_t k = s.find_last_of("+-");
        if (k != std::string::npos && k > 0 && s.find_first_not_of(' ') < k) s.insert(k, "E");
      }
      r->v[e.name] = to_real(s);
    }
  }
  return i == es.size();
}

// The hydro subset for the C ABI.
inline evora_params hydro_params(const RunParams& r) {
  evora_params p;
  evora_params_default(&p);
  p.nx = (int)r["nx"];
  p.ny = (int)r["ny"];
  p.nz = (int)r["nz"];
  p.solver = (int)r["solver"];
  p.limiter = (int)r["limiter"];
  p.boundtype = (int)r["boundtype"];
  p.secondorder = r.flag("secondorder");
  p.gravity = r.flag("gravity");
  p.conduction = r.flag("conduction");
  p.simplekappa = r.flag("simplekappa");
  p.c_cond = r["c_cond"];
  p.tempfloor = r.flag("tempfloor");
  p.jeansfloor = r.flag("jeansfloor");
  p.temp_fl = r["temp_fl"];
  p.c_jeans = r["c_jeans"];
  p.fb = r["fb"];
  p.dualenergy = r.flag("dualenergy");
  p.atomic = r.flag("atomic");
  p.g = r["g"];
  p.cfl = r["cfl"];
  p.de_thresh = r["de_thresh"];
  p.xmin = r["xmin"];
  p.xmax = r["xmax"];
  p.ymin = r["ymin"];
  p.ymax = r["ymax"];
  p.zmin = r["zmin"];
  p.zmax = r["zmax"];
  p.tstart = r["tstart"];
  p.tend = r["tend"];
  p.supercomoving = r.flag("supercomoving");
  p.c_cosmo = r["c_cosmo"];
  p.omega0 = r["omega0"];
  p.lambda0 = r["lambda0"];
  p.hubble0 = r["hubble0"];
  p.box = r["box"];
  p.zstart = r["zstart"];
  p.zend = r["zend"];
  for (int i = 0; i < EVORA_NDUMP; ++i) p.dump_redshift[i] = r.dump_redshift[i];
  p.chemistry = r.flag("chemistry");
  p.noncie = r.flag("noncie");
  p.cooling = r.flag("cooling");
  p.background = r.flag("background");
  p.bg = (int32_t)r["bg"];
  p.cooldt = r.flag("cooldt");
  p.j0 = r["j0"];
  p.c_chem = r["c_chem"];
  p.substep = r["substep"];
  p.rhoh = r["rhoh"];
  p.rhohe = r["rhohe"];
  p.c_cooldt = r["c_cooldt"];
  return p;
}

// The parts of a run these drivers do not have: the non-equilibrium
// chemistry build (grids do not advect its 12 fields).
inline std::string unsupported(const RunParams& r) {
  std::string s;
  if (r.flag("chemistry") && r.flag("noncie")) s += "noncie";
  if (!r.flag("hydro")) s += (s.empty() ? "" : ", ") + std::string("hydro = .false.");
  return s;
}

}  // namespace driver
}  // namespace evora

// param.cc -- param.in reader (see param.h).
#include "param.h"

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace dspw_host {

namespace {

class Tokens {
 public:
  explicit Tokens(const std::string& text) : s_(text) {}

  // skip whitespace, ',' ';' and comments (enflo/src/reader.h:49-88)
  void skip() {
    for (;;) {
      while (p_ < s_.size() && (std::isspace((unsigned char)s_[p_]) || s_[p_] == ',' || s_[p_] == ';')) ++p_;
      if (p_ >= s_.size()) return;
      if (s_[p_] == '#' || s_[p_] == '%' || (s_[p_] == '/' && p_ + 1 < s_.size() && s_[p_ + 1] == '/')) {
        while (p_ < s_.size() && s_[p_] != '\n') ++p_;
        continue;
      }
      if (s_[p_] == '/' && p_ + 1 < s_.size() && s_[p_ + 1] == '*') {
        size_t e = s_.find("*/", p_ + 2);
        p_ = e == std::string::npos ? s_.size() : e + 2;
        continue;
      }
      return;
    }
  }
  std::string word() {
    skip();
    size_t b = p_;
    while (p_ < s_.size() && !std::isspace((unsigned char)s_[p_])) ++p_;
    return s_.substr(b, p_ - b);
  }
  std::string rest_of_line() {
    skip();
    size_t b = p_;
    while (p_ < s_.size() && s_[p_] != '\n') ++p_;
    std::string r = s_.substr(b, p_ - b);
    while (!r.empty() && std::isspace((unsigned char)r.back())) r.pop_back();
    return r;
  }
  // numbers are read like stream extraction: the longest numeric prefix, so
  // that "100,200" yields 100 and leaves ",200" (skipped as a separator)
  double number() {
    skip();
    const char* b = s_.c_str() + p_;
    char* end = nullptr;
    double v = std::strtod(b, &end);
    if (end == b) fail("number", word());
    p_ += end - b;
    return v;
  }
  int integer() {
    skip();
    const char* b = s_.c_str() + p_;
    char* end = nullptr;
    long v = std::strtol(b, &end, 10);
    if (end == b) fail("integer", word());
    p_ += end - b;
    return (int)v;
  }
  void entry(const std::string& want) {
    std::string got = word();
    if (got != want) fail(want, got);
  }
  void begin(const std::string& name) {
    entry(name);
    entry("{");
  }
  bool end_of_section() {   // true and consumed if the next token is "}"
    size_t keep = p_;
    if (word() == "}") return true;
    p_ = keep;
    return false;
  }
  std::string peek() {
    size_t keep = p_;
    std::string w = word();
    p_ = keep;
    return w;
  }
  [[noreturn]] void fail(const std::string& want, const std::string& got) {
    throw std::runtime_error("param.in: expecting " + want + ", found '" + got + "'");
  }

 private:
  const std::string& s_;
  size_t p_ = 0;
};

std::vector<int> int_list(Tokens& t) {
  std::vector<int> v;
  t.entry("{");
  while (!t.end_of_section()) v.push_back(t.integer());
  return v;
}

}  // namespace

Param read_param(const std::string& path) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("param.in: cannot open " + path);
  std::stringstream ss;
  ss << in.rdbuf();
  std::string text = ss.str();
  Tokens t(text);
  Param P;
  // grid (enflo/src/parameter.cc:34-96)
  t.begin("grid");
  t.entry("x_min"); P.xmin = t.rest_of_line();
  t.entry("x_max"); P.xmax = t.rest_of_line();
  t.entry("Nx_cell"); P.nx = int_list(t);
  t.entry("y_min"); P.ymin = t.rest_of_line();
  t.entry("y_max"); P.ymax = t.rest_of_line();
  t.entry("Ny_cell"); P.ny = int_list(t);
  t.entry("z_min"); P.zmin = t.rest_of_line();
  t.entry("z_max"); P.zmax = t.rest_of_line();
  t.entry("Nz_cell"); P.nz = int_list(t);
  t.entry("}");
  if (P.nx.size() != P.ny.size() || P.nx.size() != P.nz.size() || P.nx.empty())
    throw std::runtime_error("param.in: Nx_cell, Ny_cell, Nz_cell need the same number of levels");
  // numeric (:101-217)
  t.begin("numeric");
  t.entry("time_scheme"); P.time_scheme = t.word();
  t.entry("cfl"); P.cfl = t.number();
  t.entry("max_iter"); P.max_iter = t.integer();
  t.entry("final_time"); P.final_time = t.number();
  t.entry("min_residue"); P.min_residue = t.number();
  t.entry("reconstruct"); P.reconstruct = t.word();
  if (P.reconstruct == "eno") P.reconstruct += std::to_string(t.integer());   // "eno <level>", :178-184
  t.entry("net_file"); P.net_file = t.word();
  t.entry("}");
  // material: scalar files start with 'model', system files with 'gamma'
  t.begin("material");
  if (t.peek() == "model") {
    P.scalar = true;
    t.entry("model"); P.model = t.word();
    if (P.model == "linadv") {
      t.entry("vel");
      t.entry("{");
      std::vector<double> v;
      while (!t.end_of_section()) v.push_back(t.number());
      if (v.size() != 3) throw std::runtime_error("param.in: need three linear advection velocity components");
      for (int k = 0; k < 3; k++) P.lin_vel[k] = v[k];
    }
    t.entry("flux"); P.flux = t.word();
  } else {
    t.entry("gamma"); P.gamma = t.number();
    t.entry("gas_const"); P.gas_const = t.number();
    t.begin("viscosity");
    t.entry("model"); P.mu_model = t.word();
    t.entry("mu_ref"); P.mu_ref = t.number();
    if (P.mu_model == "sutherland") { t.entry("T_ref"); P.T_ref = t.number(); t.entry("T_0"); P.T_0 = t.number(); }
    else if (P.mu_model == "power") { t.entry("T_ref"); P.T_ref = t.number(); t.entry("omega"); P.omega = t.number(); }
    t.entry("}");
    t.entry("prandtl"); P.prandtl = t.number();
    t.entry("model"); P.model = t.word();
    t.entry("flux"); P.flux = t.word();
    t.entry("EC1_fix");
    std::string e = t.word();
    if (e != "yes" && e != "no") t.fail("yes/no for EC1_fix", e);
    P.ec1_fix = e == "yes";
  }
  t.entry("}");
  // constants (:412-431)
  t.begin("constants");
  while (!t.end_of_section()) {
    std::string name = t.word();
    P.constants[name] = t.number();
  }
  // initial condition / exact solution (:436-525)
  t.begin("initial_condition");
  if (P.scalar) {
    P.ic.push_back(t.rest_of_line());
  } else {
    for (const char* k : {"density", "xvelocity", "yvelocity", "zvelocity", "pressure"}) {
      t.entry(k);
      P.ic.push_back(t.rest_of_line());
    }
  }
  t.entry("}");
  t.begin("exact_soln");
  t.entry("available");
  std::string a = t.word();
  if (a != "yes" && a != "no") t.fail("yes/no for available", a);
  P.exact_available = a == "yes";
  if (P.exact_available) {
    if (P.scalar) {
      P.exact.push_back(t.rest_of_line());
    } else {
      for (const char* k : {"density", "xvelocity", "yvelocity", "zvelocity", "pressure"}) {
        t.entry(k);
        P.exact.push_back(t.rest_of_line());
      }
    }
    t.entry("}");
  } else {
    while (!t.end_of_section()) t.word();
  }
  // boundary conditions (:530-586)
  t.begin("boundary_condition");
  const char* names[6] = {"xleft", "xright", "yleft", "yright", "zleft", "zright"};
  for (int f = 0; f < 6; f++) {
    t.begin(names[f]);
    t.entry("type");
    P.bc[f] = t.word();
    t.entry("}");
  }
  t.entry("}");
  // output (:591-641)
  t.begin("output");
  t.entry("OOC_study");
  std::string o = t.word();
  if (o != "yes" && o != "no") t.fail("yes/no for OOC_study", o);
  P.ooc = o == "yes";
  t.entry("problem_dim"); P.problem_dim = t.integer();
  t.entry("time_stamps"); P.time_stamps = t.integer();
  t.entry("output_path"); P.output_path = t.word();
  t.entry("}");
  if (P.ooc && (P.nx.size() < 2 || !P.exact_available))
    throw std::runtime_error("param.in: an OOC study needs two or more mesh levels and an exact solution");
  return P;
}

}  // namespace dspw_host

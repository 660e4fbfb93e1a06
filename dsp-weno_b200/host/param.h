// param.h -- reader of the reference's param.in files (the surface of
// Parameter::read, enflo/src/parameter.cc:16-29 and
// enflo_scalar/src_scalar/parameter.cc), written for this project.  Sections
// are read in the reference's order with the same keywords; comments are
// '#', '%', '//' lines and '/* */' blocks, and ',' / ';' separate tokens like
// whitespace (enflo/src/reader.h:49-88).  Errors are reported as exceptions
// instead of exit(0)/abort().
#pragma once
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace dspw_host {

struct Param {
  bool scalar = false;                 // enflo_scalar file (material section starts with 'model')
  std::string xmin, xmax, ymin, ymax, zmin, zmax;   // expressions
  std::vector<int> nx, ny, nz;
  std::string time_scheme;
  double cfl = 0, final_time = 0, min_residue = 0;
  int max_iter = 0;
  std::string reconstruct, net_file;
  // material
  std::string model, flux;
  double lin_vel[3] = {0, 0, 0};
  double gamma = 1.4, gas_const = 1.0, prandtl = 1.0;
  std::string mu_model = "constant";
  double mu_ref = 0, T_ref = 1, T_0 = 1, omega = 1;
  bool ec1_fix = false;
  std::map<std::string, double> constants;
  std::vector<std::string> ic;         // scalar: 1; systems: density, x/y/z velocity, pressure
  bool exact_available = false;
  std::vector<std::string> exact;
  std::string bc[6];
  bool ooc = false;
  int problem_dim = 1;
  int time_stamps = 1;
  std::string output_path = ".";
};

// throws std::runtime_error naming the expected and found entries
Param read_param(const std::string& path);

}  // namespace dspw_host

// output.h -- the reference's solution files: FV::output of enflo
// (enflo/src/output.cc:10-172: sol####.vtk, omg####.vtk, 1Dsol####.dat) and of
// enflo_scalar (enflo_scalar/src_scalar/output.cc:10-68: sol####.vtk,
// 1Dsol####.dat), written from a primitive state held on the host.
#pragma once
#include <string>
#include <vector>

namespace dspw_host {

struct OutGrid {
  int nx, ny, nz;
  double dx, dy, dz;
  double xmin, ymin, zmin;
  int bc[6];                // enum dspw_bc per face
  double bc_state[6][5];    // primitive state of dirichlet faces
  double gamma;
  bool scalar;
};

// The files of output number `counter` in `dir` for the primitive planes
// `prim` (nvar x nz x ny x nx) at `time`; returns the lines FV::output prints.
std::string write_output(const std::string& dir, int counter, double time, const OutGrid& g,
                         const std::vector<double>& prim);

// Node vorticity of find_vorticity (enflo/src/find_vort.cc:18-28) from the
// primitive planes, nodes (Nx+1)(Ny+1)(Nz+1) with x fastest, 3 values each.
std::vector<double> node_vorticity(const OutGrid& g, const std::vector<double>& prim);

}  // namespace dspw_host

// output.cc -- FV::output's files from a host primitive state (see output.h).
#include "output.h"

#include <cmath>
#include <fstream>
#include <sstream>

#include "../../include/dspw.h"

namespace dspw_host {

namespace {

// primitive state of cell (ci, cj, ck), each in -1 .. N, with the reference's
// one-layer ghost cells: one coordinate outside -> that face's boundary
// condition (apply_bc, enflo/src/fv.cc:121-315), two or three outside ->
// periodic wrap of all of them (edges and corners, :317-358)
void ghost_prim(const OutGrid& g, const std::vector<double>& prim, int ci, int cj, int ck, double p[5]) {
  const int N[3] = {g.nx, g.ny, g.nz};
  int c[3] = {ci, cj, ck};
  int out = 0, axis = -1;
  for (int a = 0; a < 3; a++)
    if (c[a] < 0 || c[a] >= N[a]) { out++; axis = a; }
  int flip = -1;
  if (out >= 2) {
    for (int a = 0; a < 3; a++) c[a] = (c[a] + N[a]) % N[a];
  } else if (out == 1) {
    const int face = 2 * axis + (c[axis] < 0 ? 0 : 1);
    const int kind = g.bc[face];
    if (kind == DSPW_BC_DIRICHLET) {
      for (int v = 0; v < 5; v++) p[v] = g.bc_state[face][v];
      return;
    }
    const int n = N[axis], x = c[axis];
    if (kind == DSPW_BC_PERIODIC) c[axis] = (x % n + n) % n;
    else if (kind == DSPW_BC_WALL) { c[axis] = x < 0 ? -1 - x : 2 * n - 1 - x; flip = axis; }
    else c[axis] = x < 0 ? 0 : n - 1;
  }
  const size_t ncell = (size_t)g.nx * g.ny * g.nz;
  const size_t cell = ((size_t)c[2] * g.ny + c[1]) * g.nx + c[0];
  for (int v = 0; v < 5; v++) p[v] = prim[v * ncell + cell];
  if (flip >= 0) p[1 + flip] = -p[1 + flip];
}

std::string counter_tag(int counter) {
  std::ostringstream ss;
  const char* pre = counter <= 9 ? "000" : (counter <= 99 ? "00" : (counter <= 999 ? "0" : ""));
  ss << pre << counter;
  return ss.str();
}

void vtk_header(std::ofstream& f, double time, const OutGrid& g) {
  f << "# vtk DataFile Version 3.0" << std::endl;
  f << "enflo" << std::endl;
  f << "ASCII" << std::endl;
  f << "DATASET STRUCTURED_POINTS" << std::endl;
  f << "FIELD FieldData 1" << std::endl;
  f << "TIME 1 1 double" << std::endl;
  f << time << std::endl;
  f << "DIMENSIONS " << (g.nx + 1) << " " << (g.ny + 1) << " " << (g.nz + 1) << std::endl;
  f << "SPACING " << g.dx << " " << g.dy << " " << g.dz << " " << std::endl;
  f << "ORIGIN " << g.xmin << " " << g.ymin << " " << g.zmin << " " << std::endl;
}

}  // namespace

std::vector<double> node_vorticity(const OutGrid& g, const std::vector<double>& prim) {
  const int NX = g.nx + 1, NY = g.ny + 1, NZ = g.nz + 1;
  std::vector<double> w((size_t)3 * NX * NY * NZ);
  const double vx = 1.0 / (4.0 * g.dx), vy = 1.0 / (4.0 * g.dy), vz = 1.0 / (4.0 * g.dz);
  for (int c = 0; c < NZ; c++)
    for (int b = 0; b < NY; b++)
      for (int a = 0; a < NX; a++) {
        double vel[8][3];   // index 4*dk + 2*dj + di; d = 1: cell a (b, c), 0: cell a-1
        for (int q = 0; q < 8; q++) {
          double p[5];
          ghost_prim(g, prim, a - 1 + (q & 1), b - 1 + ((q >> 1) & 1), c - 1 + (q >> 2), p);
          vel[q][0] = p[1]; vel[q][1] = p[2]; vel[q][2] = p[3];
        }
#define Q(i, j, k) ((k) * 4 + (j) * 2 + (i))
        // nodal_avg_and_vel_derivatives, enflo/src/nodal_avg_and_der.cc:37-81
        double Tx[3], Ty[3], Tz[3];
        for (int v = 0; v < 3; v++) {
          Tx[v] = vel[Q(1, 1, 1)][v] * vx + vel[Q(1, 1, 0)][v] * vx + vel[Q(1, 0, 1)][v] * vx + vel[Q(1, 0, 0)][v] * vx;
          Tx[v] += vel[Q(0, 1, 1)][v] * -vx + vel[Q(0, 1, 0)][v] * -vx + vel[Q(0, 0, 1)][v] * -vx +
                   vel[Q(0, 0, 0)][v] * -vx;
          Ty[v] = vel[Q(1, 1, 1)][v] * vy + vel[Q(1, 1, 0)][v] * vy + vel[Q(0, 1, 1)][v] * vy + vel[Q(0, 1, 0)][v] * vy;
          Ty[v] += vel[Q(1, 0, 1)][v] * -vy + vel[Q(1, 0, 0)][v] * -vy + vel[Q(0, 0, 1)][v] * -vy +
                   vel[Q(0, 0, 0)][v] * -vy;
          Tz[v] = vel[Q(1, 1, 1)][v] * vz + vel[Q(1, 0, 1)][v] * vz + vel[Q(0, 1, 1)][v] * vz + vel[Q(0, 0, 1)][v] * vz;
          Tz[v] += vel[Q(1, 1, 0)][v] * -vz + vel[Q(1, 0, 0)][v] * -vz + vel[Q(0, 1, 0)][v] * -vz +
                   vel[Q(0, 0, 0)][v] * -vz;
        }
#undef Q
        double* o = &w[3 * (((size_t)c * NY + b) * NX + a)];
        o[0] = Ty[2] - Tz[1];
        o[1] = Tz[0] - Tx[2];
        o[2] = Tx[1] - Ty[0];
      }
  return w;
}

std::string write_output(const std::string& dir, int counter, double time, const OutGrid& g,
                         const std::vector<double>& prim) {
  const std::string tag = counter_tag(counter);
  const std::string sol = dir + "/sol" + tag + ".vtk", line = dir + "/1Dsol" + tag + ".dat";
  std::ostringstream log;
  log << "Saving solutions in " << sol << std::endl;
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  {
    std::ofstream vtk(sol);
    vtk_header(vtk, time, g);
    vtk << "CELL_DATA  " << n << std::endl;
    if (g.scalar) {
      vtk << "SCALARS solution double 1" << std::endl;
      vtk << "LOOKUP_TABLE default" << std::endl;
      for (size_t c = 0; c < n; c++) vtk << prim[c] << std::endl;
    } else {
      vtk << "SCALARS density float 1" << std::endl;
      vtk << "LOOKUP_TABLE default" << std::endl;
      for (size_t c = 0; c < n; c++) vtk << prim[c] << std::endl;
      vtk << "VECTORS velocity float" << std::endl;
      for (size_t c = 0; c < n; c++) vtk << prim[n + c] << " " << prim[2 * n + c] << " " << prim[3 * n + c] << std::endl;
      vtk << "SCALARS pressure float 1" << std::endl;
      vtk << "LOOKUP_TABLE default" << std::endl;
      for (size_t c = 0; c < n; c++) vtk << prim[4 * n + c] << std::endl;
      vtk << "SCALARS physical_entropy float 1" << std::endl;
      vtk << "LOOKUP_TABLE default" << std::endl;
      // Entropy, enflo/src/fv.cc:557-560
      for (size_t c = 0; c < n; c++) vtk << std::log(prim[4 * n + c]) - g.gamma * std::log(prim[c]) << std::endl;
    }
  }
  if (!g.scalar) {
    const std::string omg = dir + "/omg" + tag + ".vtk";
    log << "Saving vorticty in " << omg << std::endl;   // the reference's message
    std::ofstream vtk(omg);
    vtk_header(vtk, time, g);
    const size_t nn = (size_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
    vtk << "POINT_DATA  " << nn << std::endl;
    vtk << "VECTORS vorticity float" << std::endl;
    const std::vector<double> w = node_vorticity(g, prim);
    for (size_t q = 0; q < nn; q++) vtk << w[3 * q] << " " << w[3 * q + 1] << " " << w[3 * q + 2] << std::endl;
  }
  {
    std::ofstream f(line);
    for (int i = 0; i < g.nx; i++) {
      const double x = (g.xmin + g.dx / 2) + g.dx * i;
      if (g.scalar) f << x << "\t" << prim[i] << "\t" << std::endl;
      else f << x << "\t" << prim[i] << "\t" << prim[n + i] << "\t" << prim[4 * n + i] << std::endl;
    }
  }
  return log.str();
}

}  // namespace dspw_host

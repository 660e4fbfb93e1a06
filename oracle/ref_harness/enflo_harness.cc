// Test-infrastructure harness around the reference Euler/Navier-Stokes solver
// (enflo/src).  It is compiled together with the reference's own, unmodified
// sources where they lie (see oracle/Makefile) into oracle/_ref/libenflo_ref.so
// and is only ever used as a checker: golden-vector generation and the CPU
// baseline.  Nothing here is part of the product.
//
// The reference exposes no API: the solver state and the per-stage functions
// are private members of class FV (enflo/src/fv.h:79-250).  The harness opens
// them with `#define private public` after every standard header has been
// included, and drives them in the order FV::run uses (enflo/src/fv.cc:1231-1324),
// minus file output and the per-step diagnostics, which do not touch the state.
//
// Array layout across this C surface: planes of shape (nvar, Nz, Ny, Nx), x
// fastest, interior cells only, FP64.

#include <algorithm>
#include <cassert>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>
#include <regex>

#define private public
#include "fv.h"
#undef private

std::map<std::string, double> constants;   // defined by enflo/src/main.cc:7 in the reference binary

namespace {

struct Quiet {   // the reference prints progress to std::cout; silence it inside calls
  std::streambuf* old;
  std::ostringstream sink;
  Quiet() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~Quiet() { std::cout.rdbuf(old); }
};

struct Handle {
  FV* fv;
  double t_interval, t_soln_save;
  int write_output;   // call FV::output at the time stamps, as FV::run does with print_soln
};

inline int ncell(const FV* f) { return f->Nx_cell * f->Ny_cell * f->Nz_cell; }
inline size_t plane_index(const FV* f, int i, int j, int k) {
  return ((size_t)k * f->Ny_cell + j) * f->Nx_cell + i;
}

}  // namespace

#define HX __attribute__((visibility("default")))

extern "C" {

// Build the solver for mesh level `level` of `param_path` and initialise it the
// way FV::run does before its time loop (enflo/src/fv.cc:1235-1244).
HX void* refE_create(const char* param_path, int level) {
  Quiet q;
  constants.clear();
  FV* fv = new FV(const_cast<char*>(param_path));
  if (level < 0 || level >= (int)fv->param.Nx_cell.size()) { delete fv; return nullptr; }
  fv->Nx_cell = fv->param.Nx_cell[level];
  fv->Ny_cell = fv->param.Ny_cell[level];
  fv->Nz_cell = fv->param.Nz_cell[level];
  fv->initialize();
  fv->prim_to_con();
  fv->prim_to_ent();
  fv->time = 0.0;
  fv->iter = 0;
  fv->counter = 0;   // output file numbering, FV::run (enflo/src/fv.cc:1245)
  Handle* h = new Handle();
  h->fv = fv;
  h->t_interval = fv->param.final_time / fv->param.t_stamps;
  h->t_soln_save = h->t_interval;
  return h;
}

HX void refE_destroy(void* hp) {
  Handle* h = (Handle*)hp;
  Quiet q;
  delete h->fv;
  delete h;
}

HX void refE_dims(void* hp, int* n, double* d) {
  FV* f = ((Handle*)hp)->fv;
  n[0] = f->Nx_cell; n[1] = f->Ny_cell; n[2] = f->Nz_cell; n[3] = f->ng_cell;
  d[0] = f->dx; d[1] = f->dy; d[2] = f->dz;
  d[3] = f->time; d[4] = f->dt;
  n[4] = f->iter;
}

HX void refE_get_prim(void* hp, double* out) {
  FV* f = ((Handle*)hp)->fv;
  int g = f->ng_cell, N = ncell(f);
  for (int k = 0; k < f->Nz_cell; ++k)
    for (int j = 0; j < f->Ny_cell; ++j)
      for (int i = 0; i < f->Nx_cell; ++i) {
        const PrimVar& p = f->primitive[i + g][j + g][k + g];
        size_t c = plane_index(f, i, j, k);
        out[0 * N + c] = p.density;
        out[1 * N + c] = p.velocity.x;
        out[2 * N + c] = p.velocity.y;
        out[3 * N + c] = p.velocity.z;
        out[4 * N + c] = p.pressure;
      }
}

HX void refE_get_cons(void* hp, double* out) {
  FV* f = ((Handle*)hp)->fv;
  int N = ncell(f);
  for (int k = 0; k < f->Nz_cell; ++k)
    for (int j = 0; j < f->Ny_cell; ++j)
      for (int i = 0; i < f->Nx_cell; ++i) {
        const ConVar& c0 = f->conserved[i][j][k];
        size_t c = plane_index(f, i, j, k);
        out[0 * N + c] = c0.density;
        out[1 * N + c] = c0.momentum.x;
        out[2 * N + c] = c0.momentum.y;
        out[3 * N + c] = c0.momentum.z;
        out[4 * N + c] = c0.energy;
      }
}

// Replace the interior primitive state, then rebuild ghosts, conserved and
// entropy variables exactly as FV::run's preamble does.
HX void refE_set_prim(void* hp, const double* in) {
  FV* f = ((Handle*)hp)->fv;
  int g = f->ng_cell, N = ncell(f);
  for (int k = 0; k < f->Nz_cell; ++k)
    for (int j = 0; j < f->Ny_cell; ++j)
      for (int i = 0; i < f->Nx_cell; ++i) {
        PrimVar& p = f->primitive[i + g][j + g][k + g];
        size_t c = plane_index(f, i, j, k);
        p.density = in[0 * N + c];
        p.velocity.x = in[1 * N + c];
        p.velocity.y = in[2 * N + c];
        p.velocity.z = in[3 * N + c];
        p.pressure = in[4 * N + c];
      }
  f->apply_bc();
  f->prim_to_con();
  f->prim_to_ent();
}

// Residual of one stage for the current state (enflo/src/fv.cc:1278-1279),
// in the reference's sign convention (U_t = -R / volume).
HX void refE_residual(void* hp, int rk, double* out) {
  Quiet q;
  FV* f = ((Handle*)hp)->fv;
  int N = ncell(f);
  f->prim_to_ent();
  f->compute_residual(rk);
  for (int k = 0; k < f->Nz_cell; ++k)
    for (int j = 0; j < f->Ny_cell; ++j)
      for (int i = 0; i < f->Nx_cell; ++i) {
        const Flux& r = f->residual[i][j][k];
        size_t c = plane_index(f, i, j, k);
        out[0 * N + c] = r.mass_flux;
        out[1 * N + c] = r.momentum_flux.x;
        out[2 * N + c] = r.momentum_flux.y;
        out[3 * N + c] = r.momentum_flux.z;
        out[4 * N + c] = r.energy_flux;
      }
}

HX double refE_compute_dt(void* hp) {
  FV* f = ((Handle*)hp)->fv;
  f->compute_dt();
  return f->dt;
}

// Advance up to `nsteps` steps with the loop body of FV::run
// (enflo/src/fv.cc:1262-1313): CFL dt, clipping to the next time stamp, the
// Runge-Kutta stages (the classic RK4 accumulator zeroed first).  If fixed_dt > 0 the CFL step is replaced by that value (the
// clipping still applies).  Returns the number of steps taken.
// With `rows`, each step also records the reference's own per-step
// diagnostics, 12 doubles: iter, time, total_ent, KE, KE_diss_pr,
// KE_diss_stress (0 for Euler), Enstrophy from compute_global at stage 0
// (fv.cc:1280-1281, with find_vorticity as FV::run calls it, :1244,1307), and
// the five components of compute_residual_norm after the step (:1286).
static int step_impl(Handle* h, int nsteps, double fixed_dt, double* rows) {
  FV* f = h->fv;
  int taken = 0;
  while (taken < nsteps && f->time < f->param.final_time && f->iter < f->param.max_iter) {
    double* row = rows ? rows + 12 * (size_t)taken : nullptr;
    if (row) f->find_vorticity();
    f->conserved_old = f->conserved;
    if (fixed_dt > 0) f->dt = fixed_dt; else f->compute_dt();
    if (f->time + f->dt > h->t_soln_save) f->dt = h->t_soln_save - f->time;
    if (f->param.time_scheme == rk4)   // enflo/src/fv.cc:1268-1275
      for (int i = 0; i < f->Nx_cell; ++i)
        for (int j = 0; j < f->Ny_cell; ++j)
          for (int k = 0; k < f->Nz_cell; ++k) f->residual2[i][j][k].zero();
    for (int rk = 0; rk < f->param.n_rks; ++rk) {
      f->prim_to_ent();
      f->compute_residual(rk);
      if (row && rk == 0) {
        f->compute_global();
        const bool ns = f->param.model == ns_es || f->param.model == ns_kep;
        row[0] = f->iter;
        row[1] = f->time;
        row[2] = f->total_ent;
        row[3] = f->KE;
        row[4] = f->KE_diss_pr;
        row[5] = ns ? f->KE_diss_stress : 0.0;
        row[6] = f->Enstrophy;
      }
      f->update_solution(rk);
      f->con_to_prim();
    }
    f->time += f->dt;
    ++f->iter;
    if (row) {
      f->compute_residual_norm();
      row[7] = f->res_norm.mass_flux;
      row[8] = f->res_norm.momentum_flux.x;
      row[9] = f->res_norm.momentum_flux.y;
      row[10] = f->res_norm.momentum_flux.z;
      row[11] = f->res_norm.energy_flux;
    }
    if (f->time == h->t_soln_save) {
      if (h->write_output) {
        f->find_vorticity();
        f->output();
      }
      h->t_soln_save += h->t_interval;
    }
    ++taken;
  }
  return taken;
}

HX int refE_step(void* hp, int nsteps, double fixed_dt) {
  Quiet q;
  return step_impl((Handle*)hp, nsteps, fixed_dt, nullptr);
}

HX int refE_step_diag(void* hp, int nsteps, double fixed_dt, double* rows) {
  Quiet q;
  return step_impl((Handle*)hp, nsteps, fixed_dt, rows);
}

// One face flux num_flux(P, V, n) (enflo/src/num_flux.cc:12-72) for a stencil
// of 2 ng cells (4; 6 for eno 3).  The stencil is written into an x-line of the
// mesh and V is taken from the reference's own prim_to_ent
// (enflo/src/fv.cc:421-552); the mesh must have Nx >= 2.  pin: (2 ng, 5)
// primitive rows; vout: (2 ng, 5) entropy variables used; flux: 5 values.
// dir 0/1/2 selects the unit normal.
HX void refE_face_flux(void* hp, const double* pin, int dir, double* vout, double* flux) {
  FV* f = ((Handle*)hp)->fv;
  int g = f->ng_cell;
  std::vector<PrimVar> P(2 * g);
  std::vector<EntVar> V(2 * g);
  for (int l = 0; l < 2 * g; ++l) {
    PrimVar& p = f->primitive[l][g][g];
    p.density = pin[5 * l + 0];
    p.velocity.x = pin[5 * l + 1];
    p.velocity.y = pin[5 * l + 2];
    p.velocity.z = pin[5 * l + 3];
    p.pressure = pin[5 * l + 4];
  }
  f->prim_to_ent();
  for (int l = 0; l < 2 * g; ++l) {
    P[l] = f->primitive[l][g][g];
    V[l] = f->entropy_var[l][g][g];
    vout[5 * l + 0] = V[l].entf;
    vout[5 * l + 1] = V[l].entv.x;
    vout[5 * l + 2] = V[l].entv.y;
    vout[5 * l + 3] = V[l].entv.z;
    vout[5 * l + 4] = V[l].entl;
  }
  Vector n;
  n = 0;
  if (dir == 0) n.x = 1; else if (dir == 1) n.y = 1; else n.z = 1;
  Flux fl;
  f->num_flux(P, V, n, fl);
  flux[0] = fl.mass_flux;
  flux[1] = fl.momentum_flux.x;
  flux[2] = fl.momentum_flux.y;
  flux[3] = fl.momentum_flux.z;
  flux[4] = fl.energy_flux;
}

// Component-wise reconstruction of a 4-cell stencil of 5-vectors with the
// configured scheme (enflo/src/reconstruct.cc:192-239).  zin: (4, 5).
HX void refE_reconstruct(void* hp, const double* zin, double* recl, double* recr) {
  FV* f = ((Handle*)hp)->fv;
  std::vector<std::vector<double> > Z(4, std::vector<double>(NVAR));
  for (int l = 0; l < 4; ++l)
    for (int v = 0; v < NVAR; ++v) Z[l][v] = zin[NVAR * l + v];
  double a[NVAR], b[NVAR];
  f->reconstruct(f->param.reconstruct_scheme, f->dx, Z, a, b);
  for (int v = 0; v < NVAR; ++v) { recl[v] = a[v]; recr[v] = b[v]; }
}

// Neural_Network::forward on one 4-value stencil (enflo/src/neural_network.cc:16-77).
HX void refE_nn_forward(void* hp, const double* u4, double* recl, double* recr) {
  FV* f = ((Handle*)hp)->fv;
  f->net.forward(u4, *recl, *recr);
}

HX double refE_logavg(double a, double b) { return logavg(a, b); }

// Write FV::output's files now (the reference's solution writer,
// enflo/src/output.cc:10-172) into the run's SOLN_FILES directory, as FV::run
// does before its time loop, and (on = 1) at every time stamp reached by
// later steps.
HX void refE_output(void* hp, int on) {
  Quiet q;
  Handle* h = (Handle*)hp;
  FV* f = h->fv;
  f->find_vorticity();
  f->output();
  h->write_output = on;
}

}  // extern "C"

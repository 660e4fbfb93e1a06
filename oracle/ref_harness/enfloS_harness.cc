// Test-infrastructure harness around the reference scalar solver
// (enflo_scalar/src_scalar), compiled with the reference's own unmodified
// sources where they lie (see oracle/Makefile) into oracle/_ref/libenfloS_ref.so.
// Used only as a checker (golden vectors, CPU baseline).
//
// The solver's state and per-stage functions are private members of class FV
// (enflo_scalar/src_scalar/fv.h:75-182); they are opened with
// `#define private public` after the standard headers and driven in the order
// FV::run uses (enflo_scalar/src_scalar/fv.cc:522-607) without file output.
//
// Array layout: (Nz, Ny, Nx) planes, x fastest, interior cells only, FP64.

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
#include "limiter.h"

std::map<std::string, double> constants;   // defined by src_scalar/main.cc in the reference binary

namespace {

struct Quiet {
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

inline size_t plane_index(const FV* f, int i, int j, int k) {
  return ((size_t)k * f->Ny_cell + j) * f->Nx_cell + i;
}

}  // namespace

#define HX __attribute__((visibility("default")))

extern "C" {

// Mesh level `level` of `param_path`, initialised as FV::run does before its
// loop (enflo_scalar/src_scalar/fv.cc:526-547).
HX void* refS_create(const char* param_path, int level) {
  Quiet q;
  constants.clear();
  FV* fv = new FV(const_cast<char*>(param_path));
  if (level < 0 || level >= (int)fv->param.Nx_cell.size()) { delete fv; return nullptr; }
  fv->Nx_cell = fv->param.Nx_cell[level];
  fv->Ny_cell = fv->param.Ny_cell[level];
  fv->Nz_cell = fv->param.Nz_cell[level];
  fv->initialize();
  fv->counter = 0;
  fv->time = 0.0;
  fv->iter = 0;
  Handle* h = new Handle();
  h->fv = fv;
  h->t_interval = fv->param.final_time / fv->param.t_stamps;
  h->t_soln_save = h->t_interval;
  return h;
}

HX void refS_destroy(void* hp) {
  Handle* h = (Handle*)hp;
  Quiet q;
  delete h->fv;
  delete h;
}

HX void refS_dims(void* hp, int* n, double* d) {
  FV* f = ((Handle*)hp)->fv;
  n[0] = f->Nx_cell; n[1] = f->Ny_cell; n[2] = f->Nz_cell; n[3] = f->ng_cell;
  n[4] = f->iter;
  d[0] = f->dx; d[1] = f->dy; d[2] = f->dz; d[3] = f->time; d[4] = f->dt;
}

HX void refS_get(void* hp, double* out) {
  FV* f = ((Handle*)hp)->fv;
  int g = f->ng_cell;
  for (int k = 0; k < f->Nz_cell; ++k)
    for (int j = 0; j < f->Ny_cell; ++j)
      for (int i = 0; i < f->Nx_cell; ++i)
        out[plane_index(f, i, j, k)] = f->solution[i + g][j + g][k + g];
}

HX void refS_set(void* hp, const double* in) {
  FV* f = ((Handle*)hp)->fv;
  int g = f->ng_cell;
  for (int k = 0; k < f->Nz_cell; ++k)
    for (int j = 0; j < f->Ny_cell; ++j)
      for (int i = 0; i < f->Nx_cell; ++i)
        f->solution[i + g][j + g][k + g] = in[plane_index(f, i, j, k)];
  f->apply_bc();
}

HX void refS_residual(void* hp, int rk, double* out) {
  FV* f = ((Handle*)hp)->fv;
  f->compute_residual(rk);
  for (int k = 0; k < f->Nz_cell; ++k)
    for (int j = 0; j < f->Ny_cell; ++j)
      for (int i = 0; i < f->Nx_cell; ++i)
        out[plane_index(f, i, j, k)] = f->residual[i][j][k];
}

HX double refS_compute_dt(void* hp) {
  FV* f = ((Handle*)hp)->fv;
  f->compute_dt();
  return f->dt;
}

// Loop body of FV::run (enflo_scalar/src_scalar/fv.cc:553-597) without output.
// With `rows`, each step also records 12 doubles: iter, time and total_ent of
// compute_global after the step (:573-576), zeros in the systems-only columns
// 3-6, the residual norm of compute_residual_norm in column 7, zeros after it.
static int step_impl(Handle* h, int nsteps, double fixed_dt, double* rows) {
  FV* f = h->fv;
  int taken = 0;
  while (taken < nsteps && f->time < f->param.final_time && f->iter < f->param.max_iter) {
    double* row = rows ? rows + 12 * (size_t)taken : nullptr;
    f->solution_old = f->solution;
    if (fixed_dt > 0) f->dt = fixed_dt; else f->compute_dt();
    if (f->time + f->dt > h->t_soln_save) f->dt = h->t_soln_save - f->time;
    if (f->param.time_scheme == rk4)   // enflo_scalar/src_scalar/fv.cc:560-566
      for (int i = 0; i < f->Nx_cell; ++i)
        for (int j = 0; j < f->Ny_cell; ++j)
          for (int k = 0; k < f->Nz_cell; ++k) f->residual2[i][j][k] = 0.0;
    for (int rk = 0; rk < f->param.n_rks; ++rk) {
      f->compute_residual(rk);
      f->update_solution(rk);
      f->apply_bc();
    }
    f->time += f->dt;
    ++f->iter;
    if (row) {
      f->compute_residual_norm();
      f->compute_global();
      for (int c = 0; c < 12; c++) row[c] = 0.0;
      row[0] = f->iter;
      row[1] = f->time;
      row[2] = f->total_ent;
      row[7] = f->res_norm;
    }
    if (f->time == h->t_soln_save) {
      if (h->write_output) {
        f->output();
      }
      h->t_soln_save += h->t_interval;
    }
    ++taken;
  }
  return taken;
}

HX int refS_step(void* hp, int nsteps, double fixed_dt) {
  Quiet q;
  return step_impl((Handle*)hp, nsteps, fixed_dt, nullptr);
}

HX int refS_step_diag(void* hp, int nsteps, double fixed_dt, double* rows) {
  Quiet q;
  return step_impl((Handle*)hp, nsteps, fixed_dt, rows);
}

// Run every remaining step of the current mesh level and return the L1, L2 and
// Linf errors against the exact solution (enflo_scalar/src_scalar/compute_errors.cc:9-30).
HX void refS_run_errors(void* hp, double* err3) {
  Handle* h = (Handle*)hp;
  FV* f = h->fv;
  refS_step(hp, 1 << 30, 0.0);
  Quiet q;
  std::vector<double> l1(1), l2(1), li(1);
  std::swap(l1, f->L1_err); std::swap(l2, f->L2_err); std::swap(li, f->Linf_err);
  f->L1_err.assign(1, 0.0); f->L2_err.assign(1, 0.0); f->Linf_err.assign(1, 0.0);
  f->compute_error(0);
  err3[0] = f->L1_err[0]; err3[1] = f->L2_err[0]; err3[2] = f->Linf_err[0];
  std::swap(l1, f->L1_err); std::swap(l2, f->L2_err); std::swap(li, f->Linf_err);
}

// cells of a face stencil passed in: 4, or 2 ng_cell when that is more (eno 3)
static int stencil_len(const FV* f) { return std::max(4, 2 * f->ng_cell); }

// One face flux num_flux(Soln, n) (enflo_scalar/src_scalar/num_flux.cc:12-57)
// of a stencil of stencil_len values.
HX double refS_face_flux(void* hp, const double* u4, int dir) {
  FV* f = ((Handle*)hp)->fv;
  std::vector<double> s(u4, u4 + stencil_len(f));
  Vector n;
  n = 0;
  if (dir == 0) n.x = 1; else if (dir == 1) n.y = 1; else n.z = 1;
  double fl;
  f->num_flux(s, n, fl);
  return fl;
}

// Configured reconstruction of one stencil of stencil_len values
// (enflo_scalar/src_scalar/reconstruct.cc:181-228).
HX void refS_reconstruct(void* hp, const double* u4, double* recl, double* recr) {
  FV* f = ((Handle*)hp)->fv;
  std::vector<double> s(u4, u4 + stencil_len(f));
  f->reconstruct(f->param.reconstruct_scheme, f->dx, s, *recl, *recr);
}

// sp_weno_rec (enflo_scalar/src_scalar/limiter.h:193-252) with an explicit corr_type.
HX void refS_sp_weno(const double* u4, int corr_type, double* recl, double* recr) {
  sp_weno_rec(u4, *recl, *recr, corr_type);
}

// Write FV::output's files now (the reference's solution writer,
// enflo_scalar/src_scalar/output.cc:10-68) into the run's SOLN_FILES directory, as FV::run
// does before its time loop, and (on = 1) at every time stamp reached by
// later steps.
HX void refS_output(void* hp, int on) {
  Quiet q;
  Handle* h = (Handle*)hp;
  FV* f = h->fv;
  f->output();
  h->write_output = on;
}

}  // extern "C"

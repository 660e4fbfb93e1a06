// enflo_b200.cc -- command-line driver, a drop-in for the reference's
// `enflo -i param.in` / `enfloS -i param.in` (enflo/src/main.cc:12-29).
//
// It reads the same param.in (param.h), evaluates the domain limits, initial
// condition and exact solution (expr.h), and for every mesh level (all levels
// when OOC_study is yes, the first otherwise, as FV::run, enflo/src/fv.cc:1231-1324)
// runs the stage path through the C ABI (include/dspw.h).  It writes the
// reference's SOLN_FILES_<reconstruction>/ directory: globals.dat with one row
// per step in compute_global's layout (enflo/src/compute_global.cc:80-88,
// enflo_scalar/src_scalar/compute_global.cc:34-38), from the diagnostics the
// library records on the device, the final solution, and for OOC studies
// l1_err.dat / l2_err.dat / linf_err.dat with the table layout of compute_OOC
// (enflo_scalar/src_scalar/compute_ooc.cc:10-141).  Errors of systems are those
// of the density.  Runs that are not OOC studies print the reference's per-step
// residual line (enflo/src/fv.cc:1289-1299, enflo_scalar/src_scalar/fv.cc:578-584)
// and write the solution files of FV::output (output.h) at t = 0 and at every
// time stamp, from snapshots the library takes on the device; the files are
// written by background threads while the GPU keeps stepping.
//
//   enflo_b200 -i param.in [--precision fp64|fp32_bf16] [--chunk K]
//   enflo_b200 -i param.in --check          parse and print the descriptor, no GPU
//   enflo_b200 -i param.in --dump-ic FILE   write level 0's initial state (FP64), no GPU
//   enflo_b200 -i param.in --output-ic      write the t = 0 solution files of FV::output, no GPU
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include <deque>
#include <thread>

#include "../../include/dspw.h"
#include "expr.h"
#include "output.h"
#include "param.h"

using dspw_host::Expr;
using dspw_host::Param;
using dspw_host::read_param;

namespace {

struct Fail : std::runtime_error {
  using std::runtime_error::runtime_error;
};

int flux_enum(const std::string& f) {
  static const std::map<std::string, int> m = {
      {"lin_ec", DSPW_LIN_EC}, {"lin_ec4", DSPW_LIN_EC4}, {"lin_tecno", DSPW_LIN_TECNO},
      {"lin_tecno4", DSPW_LIN_TECNO4}, {"bur_ec", DSPW_BUR_EC}, {"bur_ec4", DSPW_BUR_EC4},
      {"bur_tecno", DSPW_BUR_TECNO}, {"bur_tecno4", DSPW_BUR_TECNO4}, {"roe", DSPW_ROE}, {"kep", DSPW_KEP},
      {"kep4", DSPW_KEP4}, {"kepec", DSPW_KEPEC}, {"kepec4", DSPW_KEPEC4}, {"roe_ec", DSPW_ROE_EC},
      {"roe_ec4", DSPW_ROE_EC4}, {"keps", DSPW_KEPS}, {"keps4", DSPW_KEPS4}, {"kep_tecno_roe", DSPW_KEP_TECNO_ROE},
      {"kepes_tecno_roe", DSPW_KEPES_TECNO_ROE}, {"kepes_tecno_rusanov", DSPW_KEPES_TECNO_RUSANOV},
      {"roe_tecno_roe", DSPW_ROE_TECNO_ROE}, {"kepes_tecno4_roe", DSPW_KEPES_TECNO4_ROE},
      {"kepes_tecno4_rusanov", DSPW_KEPES_TECNO4_RUSANOV}, {"roe_tecno4_roe", DSPW_ROE_TECNO4_ROE}};
  auto it = m.find(f);
  if (it == m.end()) throw Fail("unknown flux scheme: " + f);
  return it->second;
}

int recon_enum(const std::string& r) {
  static const std::map<std::string, int> m = {{"sp_weno", DSPW_REC_SP_WENO}, {"sp_wenoc", DSPW_REC_SP_WENOC},
                                               {"sp_weno_corr2", DSPW_REC_SP_WENO_CORR2},
                                               {"sp_weno_dl", DSPW_REC_SP_WENO_DL}, {"first", DSPW_REC_FIRST},
                                               {"second", DSPW_REC_SECOND}, {"minmod", DSPW_REC_MINMOD},
                                               {"minabs", DSPW_REC_MINABS}, {"eno2", DSPW_REC_ENO2},
                                               {"eno3", DSPW_REC_ENO3}};
  auto it = m.find(r);
  if (it == m.end()) throw Fail("reconstruction not supported by the GPU path: " + r);
  return it->second;
}

int bc_enum(const std::string& b) {
  if (b == "periodic") return DSPW_BC_PERIODIC;
  if (b == "dirichlet") return DSPW_BC_DIRICHLET;
  if (b == "neumann") return DSPW_BC_NEUMANN;
  if (b == "wall") return DSPW_BC_WALL;
  throw Fail("unknown boundary type: " + b);
}

// network file in the format of Neural_Network::load_network (enflo/src/neural_network.cc:82-130)
void load_network(const std::string& path, dspw_desc& d) {
  std::ifstream in(path);
  if (!in) throw Fail("DSP-WENO network file does not exist: " + path);
  std::string line;
  bool weights = true;
  int wl = 0, bl = 0;
  while (std::getline(in, line)) {
    while (!line.empty() && std::isspace((unsigned char)line.back())) line.pop_back();
    if (line == "Biases") weights = false;
    if (line != "BEGIN") continue;
    int row = 0;
    while (std::getline(in, line)) {
      while (!line.empty() && std::isspace((unsigned char)line.back())) line.pop_back();
      if (line == "END") break;
      std::istringstream is(line);
      std::vector<double> v;
      double x;
      while (is >> x) v.push_back(x);
      if (v.empty()) continue;
      if (weights) {
        if (wl >= 4 || row >= 5 || v.size() != 5) throw Fail("network file: expected 4 layers of 5x5 weights");
        for (int k = 0; k < 5; k++) d.nn_w[wl][row][k] = v[k];
      } else {
        if (bl >= 4 || row >= 5) throw Fail("network file: expected 4 layers of 5 biases");
        d.nn_b[bl][row] = v[0];
      }
      row++;
    }
    if (weights) wl++; else bl++;
  }
  if (wl != 4 || bl != 4) throw Fail("network file: expected 4 weight and 4 bias blocks");
}

struct Level {
  dspw_desc d;
  int nvar;
  long long n;
  double xmin, xmax, ymin, ymax, zmin, zmax, dx, dy, dz;
};

// globals.dat rows in compute_global's layout, and the per-step residual line
// of FV::run when `log` is set.  Systems rows hold iter / time at the start of
// their step (compute_global runs at stage 0), scalar rows after it.
void write_globals(std::ostream& glob, std::ostream& out, const double* rows, int n, bool scalar, bool log,
                   double t_final, double& ent0) {
  for (int r = 0; r < n; r++) {
    const double* w = rows + (size_t)r * DSPW_DIAG_COLS;
    const double t = w[DSPW_DIAG_TIME], ent = w[DSPW_DIAG_ENTROPY];
    if (scalar) {
      glob << t << " " << std::setprecision(10) << ent << " " << (ent - ent0) / ent0 << " " << std::endl;
    } else {
      if (t == 0.0) {   // compute_global.cc:69-77
        ent0 = ent;
        if (ent0 == 0.0) {
          out << "WARNING: Initial total entropy is zero!! Re-setting it to 1.0" << std::endl;
          ent0 = 1.0;
        }
      }
      glob << t << " " << std::setprecision(10) << ent << " " << (ent - ent0) / std::fabs(ent0) << " "
           << w[DSPW_DIAG_KE] << " " << w[DSPW_DIAG_KE_DISS_PR] << " " << w[DSPW_DIAG_KE_DISS_STRESS] << " "
           << w[DSPW_DIAG_ENSTROPHY] << " " << std::endl;
    }
    if (!log) continue;
    std::ios saved(nullptr);
    saved.copyfmt(out);
    const double* res = w + DSPW_DIAG_RES;
    if (scalar) {
      out << std::left << "ITER = " << std::setw(8) << (long long)w[DSPW_DIAG_ITER] << " " << std::scientific
          << std::setprecision(4) << "TIME = " << t << " " << "RES = " << res[0] << std::endl;
    } else {
      // iter and time after the step; the reference prints the x-momentum
      // norm under RES_MOM_y (fv.cc:1296)
      const double t_after = r + 1 < n ? rows[(size_t)(r + 1) * DSPW_DIAG_COLS + DSPW_DIAG_TIME] : t_final;
      out << std::left << "ITER = " << std::setw(8) << (long long)w[DSPW_DIAG_ITER] + 1 << " " << std::scientific
          << std::setprecision(4) << "TIME = " << t_after << " " << "RES_MASS = " << res[0] << " "
          << "RES_MOM_X = " << res[1] << " " << "RES_MOM_y = " << res[1] << " " << "RES_MOM_z = " << res[3] << " "
          << "RES_ENERGY = " << res[4] << std::endl;
    }
    out.copyfmt(saved);
  }
}

dspw_host::OutGrid out_grid(const Level& L) {
  dspw_host::OutGrid g;
  g.nx = L.d.nx; g.ny = L.d.ny; g.nz = L.d.nz;
  g.dx = L.dx; g.dy = L.dy; g.dz = L.dz;
  g.xmin = L.xmin; g.ymin = L.ymin; g.zmin = L.zmin;
  for (int f = 0; f < 6; f++) {
    g.bc[f] = L.d.bc[f];
    for (int v = 0; v < 5; v++) g.bc_state[f][v] = L.d.bc_state[f][v];
  }
  g.gamma = L.d.gamma;
  g.scalar = L.nvar == 1;
  return g;
}

// FV::output files written by background threads, at most `max_inflight` at a
// time; each thread owns its state copy
struct Writers {
  std::vector<std::thread> threads;
  std::deque<std::string> logs;   // stable addresses for the running threads
  size_t done = 0;
  void add(const std::string& dir, int counter, double time, const dspw_host::OutGrid& g, std::vector<double> prim,
           size_t max_inflight = 3) {
    while (threads.size() - done >= max_inflight) join_one();
    logs.emplace_back();
    std::string* log = &logs.back();
    threads.emplace_back([=, prim = std::move(prim)]() { *log = dspw_host::write_output(dir, counter, time, g, prim); });
  }
  void join_one() {
    threads[done].join();
    std::cout << logs[done];
    ++done;
  }
  void join_all() {
    while (done < threads.size()) join_one();
  }
};

Level make_level(const Param& P, int rl, const std::string& precision) {
  Level L;
  dspw_desc& d = L.d;
  memset(&d, 0, sizeof(d));
  d.abi_version = DSPW_ABI_VERSION;
  if (P.scalar) d.model = P.model == "linadv" ? DSPW_LINADV : DSPW_BURGERS;
  else if (P.model == "euler") d.model = DSPW_EULER;
  else if (P.model == "ns_es") d.model = DSPW_NS_ES;
  else if (P.model == "ns_kep") d.model = DSPW_NS_KEP;
  else throw Fail("unknown model: " + P.model);
  d.flux = flux_enum(P.flux);
  d.recon = recon_enum(P.reconstruct);
  if (P.time_scheme == "ssprk3") d.time_scheme = DSPW_SSPRK3;
  else if (P.time_scheme == "rk1") d.time_scheme = DSPW_RK1;
  else if (P.time_scheme == "jameson_rk4") d.time_scheme = DSPW_JAMESON_RK4;
  else if (P.time_scheme == "rk4") d.time_scheme = DSPW_RK4;
  else throw Fail("time scheme not supported by the GPU path: " + P.time_scheme);
  d.precision = precision == "fp32_bf16" ? DSPW_FP32_BF16 : DSPW_FP64;
  d.nx = P.nx[rl];
  d.ny = P.ny[rl];
  d.nz = P.nz[rl];
  for (int f = 0; f < 6; f++) d.bc[f] = bc_enum(P.bc[f]);
  d.ec1_fix = P.ec1_fix;
  d.mu_model = P.mu_model == "sutherland" ? DSPW_MU_SUTHERLAND : (P.mu_model == "power" ? DSPW_MU_POWER : DSPW_MU_CONSTANT);
  d.max_iter = P.max_iter;
  d.t_stamps = P.time_stamps;
  L.xmin = Expr(P.xmin, P.constants).eval(0, 0, 0, 0);
  L.xmax = Expr(P.xmax, P.constants).eval(0, 0, 0, 0);
  L.ymin = Expr(P.ymin, P.constants).eval(0, 0, 0, 0);
  L.ymax = Expr(P.ymax, P.constants).eval(0, 0, 0, 0);
  L.zmin = Expr(P.zmin, P.constants).eval(0, 0, 0, 0);
  L.zmax = Expr(P.zmax, P.constants).eval(0, 0, 0, 0);
  d.xmin = L.xmin; d.xmax = L.xmax; d.ymin = L.ymin; d.ymax = L.ymax; d.zmin = L.zmin; d.zmax = L.zmax;
  d.gamma = P.gamma;
  d.gas_const = P.gas_const;
  d.prandtl = P.prandtl;
  d.mu_ref = P.mu_ref;
  d.T_ref = P.T_ref;
  d.T_0 = P.T_0;
  d.omega = P.omega;
  for (int k = 0; k < 3; k++) d.lin_vel[k] = P.lin_vel[k];
  d.cfl = P.cfl;
  d.final_time = P.final_time;
  if (P.reconstruct == "sp_weno_dl") load_network(P.net_file, d);
  L.nvar = P.scalar ? 1 : 5;
  L.n = (long long)d.nx * d.ny * d.nz;
  L.dx = (L.xmax - L.xmin) / d.nx;   // enflo/src/fv.cc:29-31
  L.dy = (L.ymax - L.ymin) / d.ny;
  L.dz = (L.zmax - L.zmin) / d.nz;
  return L;
}

// values of expressions at the cell centres xmin + 0.5 dx + i dx (enflo/src/fv.cc:41-43)
std::vector<double> evaluate(const Level& L, const std::vector<std::string>& exprs,
                             const std::map<std::string, double>& constants, double t) {
  std::vector<Expr> ex;
  for (auto& s : exprs) ex.emplace_back(s, constants);
  std::vector<double> out(ex.size() * L.n);
  const dspw_desc& d = L.d;
  for (int k = 0; k < d.nz; k++)
    for (int j = 0; j < d.ny; j++)
      for (int i = 0; i < d.nx; i++) {
        double x = L.xmin + 0.5 * L.dx + i * L.dx;
        double y = L.ymin + 0.5 * L.dy + j * L.dy;
        double z = L.zmin + 0.5 * L.dz + k * L.dz;
        long long c = ((long long)k * d.ny + j) * d.nx + i;
        for (size_t v = 0; v < ex.size(); v++) out[v * L.n + c] = ex[v].eval(x, y, z, t);
      }
  return out;
}

void check(int rc, const char* what) {
  if (rc != DSPW_OK) throw Fail(std::string(what) + ": " + dspw_error_string(rc));
}

void write_ooc(const std::string& path, const Param& P, const std::vector<double>& err,
               const std::vector<Level>& levels) {
  std::ofstream f(path);
  f << std::left << std::setw(40) << std::setfill('-') << "" << "\n";
  f << std::left << std::setfill(' ') << std::setw(6) << "Nx" << std::setw(6) << "Ny" << std::setw(6) << "Nz"
    << std::setw(17) << "ERR" << std::setw(8) << "OOC" << "\n";
  f << std::left << std::setw(40) << std::setfill('-') << "" << "\n" << std::setfill(' ');
  for (size_t i = 0; i < err.size(); i++) {
    const Level& L = levels[i];
    f << std::left << std::setw(6) << L.d.nx << std::setw(6) << L.d.ny << std::setw(6) << L.d.nz << std::scientific
      << std::setw(17) << std::setprecision(5) << err[i];
    if (i == 0) {
      f << std::setw(8) << " - ";
    } else {
      // rate from the mesh-size measure of compute_OOC (problem_dim directions)
      auto h2 = [&](const Level& M) {
        double s = M.dx * M.dx;
        if (P.problem_dim >= 2) s += M.dy * M.dy;
        if (P.problem_dim >= 3) s += M.dz * M.dz;
        return s;
      };
      double rate = std::log(err[i - 1] / err[i]) / std::log(std::sqrt(h2(levels[i - 1]) / h2(L)));
      f << std::fixed << std::setprecision(2) << std::setw(8) << rate;
    }
    f << "\n";
  }
}

}  // namespace

int main(int argc, char** argv) {
  std::string file, precision = "fp64", dump;
  bool check_only = false, output_ic = false;
  int chunk = 64;
  for (int a = 1; a < argc; a++) {
    std::string s = argv[a];
    if (s == "-i" && a + 1 < argc) file = argv[++a];
    else if (s == "--precision" && a + 1 < argc) precision = argv[++a];
    else if (s == "--chunk" && a + 1 < argc) chunk = std::atoi(argv[++a]);
    else if (s == "--check") check_only = true;
    else if (s == "--dump-ic" && a + 1 < argc) dump = argv[++a];
    else if (s == "--output-ic") output_ic = true;
    else {
      std::cerr << "usage: enflo_b200 -i param.in [--precision fp64|fp32_bf16] [--chunk K] [--check] "
                   "[--dump-ic FILE] [--output-ic]\n";
      return 2;
    }
  }
  if (file.empty()) {
    std::cerr << "enflo_b200: -i param.in is required\n";
    return 2;
  }
  try {
    Param P = read_param(file);
    int nlev = P.ooc ? (int)P.nx.size() : 1;
    std::vector<Level> levels;
    for (int rl = 0; rl < nlev; rl++) levels.push_back(make_level(P, rl, precision));
    if (check_only) {
      // parse every expression so that syntax errors surface without a GPU
      for (auto& e : P.ic) Expr(e, P.constants);
      for (auto& e : P.exact) Expr(e, P.constants);
      const dspw_desc& d = levels[0].d;
      std::cout << "{\"model\": " << d.model << ", \"flux\": " << d.flux << ", \"recon\": " << d.recon
                << ", \"nx\": " << d.nx << ", \"ny\": " << d.ny << ", \"nz\": " << d.nz << ", \"bc\": [" << d.bc[0]
                << ", " << d.bc[1] << ", " << d.bc[2] << ", " << d.bc[3] << ", " << d.bc[4] << ", " << d.bc[5]
                << "], \"xmin\": " << std::setprecision(17) << d.xmin << ", \"xmax\": " << d.xmax
                << ", \"cfl\": " << d.cfl << ", \"final_time\": " << d.final_time << ", \"t_stamps\": " << d.t_stamps
                << ", \"levels\": " << nlev << ", \"nn_w000\": " << d.nn_w[0][0][0] << "}\n";
      return 0;
    }
    if (!dump.empty()) {
      std::vector<double> ic = evaluate(levels[0], P.ic, P.constants, 0.0);
      std::ofstream f(dump, std::ios::binary);
      f.write(reinterpret_cast<const char*>(ic.data()), sizeof(double) * ic.size());
      return 0;
    }
    std::string soln_dir = P.output_path + "/SOLN_FILES_" + P.reconstruct;   // enflo/src/fv.h:28-34
    std::filesystem::remove_all(soln_dir);
    std::filesystem::create_directories(soln_dir);
    if (output_ic) {
      std::vector<double> ic = evaluate(levels[0], P.ic, P.constants, 0.0);
      std::cout << dspw_host::write_output(soln_dir, 0, 0.0, out_grid(levels[0]), ic);
      return 0;
    }
    std::ofstream glob(soln_dir + "/globals.dat");
    std::vector<double> l1, l2, linf;
    for (int rl = 0; rl < nlev; rl++) {
      Level& L = levels[rl];
      std::cout << "   Solving on mesh with size " << L.d.nx << "x" << L.d.ny << "x" << L.d.nz << std::endl;
      std::vector<double> ic = evaluate(L, P.ic, P.constants, 0.0);
      dspw_handle* h = nullptr;
      check(dspw_create(&L.d, &h), "dspw_create");
      int rc = dspw_upload_prim(h, 0, ic.data());
      if (rc) { dspw_destroy(h); check(rc, "dspw_upload_prim"); }
      if (rc == DSPW_OK) rc = dspw_diag_enable(h, chunk);
      if (rc) { dspw_destroy(h); check(rc, "dspw_diag_enable"); }
      double ent0 = 0.0;
      if (P.scalar) {   // compute_global before the time loop (enflo_scalar/src_scalar/fv.cc:544)
        dspw_globals_out g0;
        rc = dspw_globals(h, 0, &g0);
        if (rc) { dspw_destroy(h); check(rc, "dspw_globals"); }
        ent0 = g0.total_entropy != 0.0 ? g0.total_entropy : 1.0;
        glob << 0.0 << " " << std::setprecision(10) << g0.total_entropy << " " << (g0.total_entropy - ent0) / ent0
             << " " << std::endl;
      }
      int steps = 0;
      dspw_globals_out g;
      if (P.ooc) {
        rc = dspw_run(h, chunk, &steps);
        if (rc == DSPW_OK) rc = dspw_globals(h, 0, &g);
        if (rc) { dspw_destroy(h); check(rc, "dspw_run"); }
      } else {
        // solution files at t = 0 and at every time stamp (fv.cc:1242-1243,1309-1313)
        const dspw_host::OutGrid og = out_grid(L);
        int counter = 0;
        Writers writers;
        writers.add(soln_dir, counter++, 0.0, og, ic);
        rc = dspw_snap_enable(h, std::max(1, std::min(P.time_stamps, 8)));
        if (rc) { dspw_destroy(h); check(rc, "dspw_snap_enable"); }
        long long dropped = 0;
        for (;;) {
          rc = dspw_step(h, chunk, 0.0);
          if (rc == DSPW_OK) rc = dspw_globals(h, 0, &g);
          dspw_status_out st;
          if (rc == DSPW_OK && dspw_last_status(h, &st) == DSPW_OK && st.code) rc = st.code;
          int ns = 0;
          if (rc == DSPW_OK) rc = dspw_snap_pending(h, 0, &ns, &dropped);
          for (int q = 0; rc == DSPW_OK && q < ns; q++) {
            std::vector<double> snap(L.nvar * L.n);
            double t = 0.0;
            rc = dspw_snap_read(h, 0, snap.data(), &t, nullptr);
            if (rc == DSPW_OK) writers.add(soln_dir, counter++, t, og, std::move(snap));
          }
          if (rc || g.finished) break;
        }
        writers.join_all();
        if (rc) { dspw_destroy(h); check(rc, "dspw_step"); }
        if (dropped) std::cerr << "   " << dropped << " solution snapshots were dropped" << std::endl;
      }
      int nrows = 0, nread = 0;
      check(dspw_diag_pending(h, 0, &nrows, nullptr), "dspw_diag_pending");
      std::vector<double> rows((size_t)nrows * DSPW_DIAG_COLS);
      check(dspw_diag_read(h, 0, rows.data(), nrows, &nread), "dspw_diag_read");
      write_globals(glob, std::cout, rows.data(), nread, P.scalar, !P.ooc, g.time, ent0);
      std::vector<double> prim(L.nvar * L.n);
      check(dspw_download_prim(h, 0, prim.data()), "dspw_download_prim");
      if (P.ooc) {
        std::vector<std::string> ex = {P.exact[0]};
        std::vector<double> exact = evaluate(L, ex, P.constants, g.time);
        double e[3];
        check(dspw_errors(h, 0, 0, exact.data(), e), "dspw_errors");
        l1.push_back(e[0]);
        l2.push_back(e[1]);
        linf.push_back(e[2]);
        std::cout << "   L1 error " << std::scientific << std::setprecision(5) << e[0] << " after " << g.iter
                  << " steps, t = " << std::defaultfloat << g.time << std::endl;
      } else {
        std::ofstream sol(soln_dir + "/sol_final.dat");
        sol << std::setprecision(17);
        for (long long c = 0; c < L.n; c++) {
          for (int v = 0; v < L.nvar; v++) sol << prim[v * L.n + c] << (v + 1 < L.nvar ? " " : "\n");
        }
        std::cout << "   " << g.iter << " steps, t = " << g.time << std::endl;
      }
      dspw_status_out st;
      dspw_last_status(h, &st);
      if (st.code) std::cerr << "   device status: " << dspw_error_string(st.code) << std::endl;
      dspw_destroy(h);
    }
    if (P.ooc) {
      write_ooc(soln_dir + "/l1_err.dat", P, l1, levels);
      write_ooc(soln_dir + "/l2_err.dat", P, l2, levels);
      write_ooc(soln_dir + "/linf_err.dat", P, linf, levels);
    }
  } catch (const std::exception& e) {
    std::cerr << "enflo_b200: " << e.what() << std::endl;
    return 1;
  }
  return 0;
}

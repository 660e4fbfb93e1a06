// dspw_capi.cu -- the C ABI of include/dspw.h: handle lifetime, validation,
// device buffers, per-problem tables, the per-step CUDA graph and the
// host<->device copies.  All arithmetic runs in the kernels of
// dspw_kernels.cuh (instantiated by dspw_fp64.cu / dspw_fp32.cu).
#include <cuda.h>
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cmath>
#include <deque>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "dspw_launch.h"

using namespace dspw;

namespace dspw {

// -------------------------------------------------------- step control kernels

__global__ void k_begin_step_wrap(const ProbDev* prob, ProbState* st, int nprob, double fixed_dt, int* nactive) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nprob) return;
  const ProbDev& P = prob[p];
  ProbState& S = st[p];
  S.snap = 0;
  if (!(S.time < P.final_time && S.iter < P.max_iter)) {
    S.active = 0;
    S.dt = 0.0;
    S.factor = 0.0;
    return;
  }
  atomicAdd(nactive, 1);
  S.active = 1;
  double dt;
  if (fixed_dt > 0) {
    dt = fixed_dt;
  } else {
    unsigned long long sb = 0ull;   // max over the slots (ordered bits of non-negative speeds)
    for (int k = 0; k < EPI_SLOTS; k++) sb = S.smax[k] > sb ? S.smax[k] : sb;
    double smax = __longlong_as_double((long long)sb);
    dt = 1.0e20;
    double c = P.hmin / smax;
    if (c < dt) dt = c;
    dt *= P.cfl;
  }
  if (S.time + dt > S.t_save) dt = S.t_save - S.time;
  S.dt = dt;
  S.factor = dt / (P.dx * P.dy * P.dz);
  for (int k = 0; k < EPI_SLOTS; k++) {
    S.smax[k] = 0ull;
    S.ent_acc[k] = 0.0;
  }
}

// sum of the entropy slots of a problem
__device__ inline double ent_sum(const ProbState& S) {
  double e = 0.0;
  for (int k = 0; k < EPI_SLOTS; k++) e += S.ent_acc[k];
  return e;
}

cudaError_t launch_begin_step(const ProbDev* prob, ProbState* st, int nprob, double fixed_dt, int* nactive,
                              cudaStream_t s) {
  k_begin_step_wrap<<<(nprob + 127) / 128, 128, 0, s>>>(prob, st, nprob, fixed_dt, nactive);
  return cudaGetLastError();
}

// time += dt, ++iter, advance the time stamp (enflo/src/fv.cc:1285-1312), and
// the discrete entropy inequality bookkeeping.
__global__ void k_end_step(const ProbDev* prob, ProbState* st, int nprob) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nprob) return;
  ProbState& S = st[p];
  if (!S.active) return;
  S.time += S.dt;
  S.iter += 1;
  const int stamp = S.time == S.t_save;   // output time stamp (fv.cc:1309-1313)
  if (stamp) S.t_save += prob[p].t_interval;
  S.snap = stamp;
  // discrete entropy inequality: relative change of the total entropy
  const double e = ent_sum(S) * prob[p].vol;
  const double rise = (e - S.ent) / fabs(S.ent);
  if (rise > S.ent_max_rise) S.ent_max_rise = rise;
  S.ent = e;
  S.ent_steps += 1;
}

// total entropy of an uploaded state; the inequality's record starts anew
__global__ void k_init_entropy(const ProbDev* prob, ProbState* st, int p) {
  ProbState& S = st[p];
  S.ent = ent_sum(S) * prob[p].vol;
  for (int k = 0; k < EPI_SLOTS; k++) S.ent_acc[k] = 0.0;
  S.ent_max_rise = -1.0e300;
  S.ent_steps = 0;
}


// checks of an uploaded primitive state (nvar planes of n values, FP64):
// bad[0] counts cells with density or pressure <= 0 or NaN (systems), bad[1]
// non-finite values; the initial state must be positive (enflo/src/fv.cc:88-89)
__global__ void k_check_prim(const double* prim, long long n, int nv, unsigned long long* bad) {
  unsigned long long pos = 0, fin = 0;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    if (nv == 5 && (!(prim[c] > 0.0) || !(prim[4 * n + c] > 0.0))) pos++;
    for (int v = 0; v < nv; v++) fin += !isfinite(prim[v * n + c]);
  }
  pos = __reduce_add_sync(0xffffffffu, (unsigned)pos);
  fin = __reduce_add_sync(0xffffffffu, (unsigned)fin);
  if ((threadIdx.x & 31) == 0 && (pos | fin)) {
    atomicAdd(bad, pos);
    atomicAdd(bad + 1, fin);
  }
}

int device_sms() {
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 148;
  if (dev < 64 && cache[dev] > 0) return cache[dev];
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 148;
  if (dev < 64) cache[dev] = n;
  return n;
}

cudaError_t launch_check_prim(const double* prim, long long n, int nv, unsigned long long* bad, cudaStream_t s) {
  long long g = (n + 255) / 256;
  if (g > device_sms() * 8LL) g = device_sms() * 8LL;
  k_check_prim<<<(int)(g < 1 ? 1 : g), 256, 0, s>>>(prim, n, nv, bad);
  return cudaGetLastError();
}

cudaError_t launch_end_step(const ProbDev* prob, ProbState* st, int nprob, cudaStream_t s) {
  k_end_step<<<(nprob + 127) / 128, 128, 0, s>>>(prob, st, nprob);
  return cudaGetLastError();
}

}  // namespace dspw

// ------------------------------------------------------------------ handle --

// Problems of a batch that run the same sweep kernels: one launch per
// direction and class, over the class's own task prefix sums; pmap maps the
// class's entries to the batch's problem indices (null when the class is the
// whole batch in order).
struct SweepClass {
  int spec = 0;                        // spec_code of the class's kernels, 0 generic
  std::vector<int> probs;
  std::vector<int> task_start[3];
  int* dtask[3] = {nullptr, nullptr, nullptr};
  int* dpmap = nullptr;
  int grid[3] = {0, 0, 0};             // launch grid chosen by dspw_tune (0: one block per block-worth of tasks)
  // TMA staging of the specialised y / z sweeps: the class's tensor maps
  // (tma_map_index layout; null when the class does not qualify or its
  // problems ask for cp.async) and, per direction, whether the sweep stages
  // with TMA (1) or with per-thread cp.async copies (0).  tma_forced: the
  // problems ask for TMA (tile_staging 2), else dspw_tune picks.
  void* dtmap = nullptr;
  int use_tma[3] = {0, 0, 0};
  int tma_forced = 0;
  // narrow tiles of the specialised y / z sweeps (k_sweep_narrow: 4-column
  // blocks, cp.async staging) per direction; the direction's task list then
  // counts groups of 4 columns.  narrow_forced: the problems ask for them
  // (tile_staging 3), else dspw_tune picks.
  int narrow[3] = {0, 0, 0};
  int narrow_forced = 0;
};

struct dspw_handle {
  int nprob = 0;
  int precision = 0;
  int nrk = 3;
  int time_scheme = 1;
  int has_ns = 0;
  int has_halo = 0;   // some problem stores halo layers (DSPW_BC_HALO faces)
  // slab of a decomposition over NCCL ranks (dspw_slab_connect): the step
  // graph exchanges halo layers with the neighbours and reduces the CFL speed
  ncclComm_t comm = nullptr;
  int rank = 0, nranks = 1, up = -1, down = -1;
  int maxdim = 1;
  std::vector<SweepClass> classes;
  std::vector<dspw_desc> desc;
  std::vector<ProbDev> hprob;
  std::vector<long long> cell_start;   // nprob + 1
  long long ctot = 0;
  long long maxcells = 0;
  ProbDev* dprob = nullptr;
  ProbState* dst = nullptr;
  StatusDev* dstatus = nullptr;
  NetParams* dnet = nullptr;
  long long* dcell_start = nullptr;
  int* dnactive = nullptr;
  void* Un = nullptr;
  void* Ua = nullptr;
  void* Ub = nullptr;
  void* R = nullptr;
  void* R2 = nullptr;                  // classic RK4 only
  // per-step diagnostics (dspw_diag_enable): accumulators, the row ring
  // (slot-major, diag_cap slots of nprob rows) and the rows drained to the host
  int diag_cap = 0;
  DiagAcc* ddiag = nullptr;
  double* ddiag_part = nullptr;        // block partial rows of one diagnostics launch
  double* drows = nullptr;
  long long* dnode_start = nullptr;
  long long nodes_tot = 0;
  std::vector<unsigned long long> diag_taken;   // rows of each problem moved to the host so far
  std::vector<long long> diag_dropped;
  std::vector<std::vector<double>> diag_host;
  // snapshots at the output time stamps (dspw_snap_enable): a ring of
  // snap_slots state-shaped buffers, per-problem counts and (time, iter), and
  // the snapshots drained to the host as primitive planes
  int snap_slots = 0;
  void* dsnap = nullptr;
  unsigned long long* dsnap_count = nullptr;
  SnapMeta* dsnap_meta = nullptr;
  struct HostSnap { double time; int iter; std::vector<double> prim; };
  std::vector<unsigned long long> snap_taken;
  std::vector<long long> snap_dropped;
  std::vector<std::deque<HostSnap>> snap_host;
  void* V = nullptr;
  void* node = nullptr;
  double* dstage = nullptr;
  double* dscratch = nullptr;
  double* dred = nullptr;         // block rows of the deterministic reductions (reduce_rows_max() x 8)
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  double graph_dt = -1.0;
  // training-pair collection during residual evaluations (trainer only)
  float* collect_buf = nullptr;
  unsigned long long* collect_count = nullptr;
  unsigned long long collect_cap = 0;
  unsigned collect_stride = 1;
  // profiling: when set, an event is recorded after every launch
  std::vector<cudaEvent_t>* prof_ev = nullptr;
  std::vector<std::string>* prof_names = nullptr;
  int last_error = 0;
  size_t elem = 8;
};

extern "C" {
static int download(dspw_handle* h, int p, double* out, int prim, void* src);
}

namespace {

#define CK(x)                                  \
  do {                                         \
    cudaError_t e__ = (x);                     \
    if (e__ != cudaSuccess) {                  \
      h->last_error = DSPW_ERR_CUDA;           \
      return DSPW_ERR_CUDA;                    \
    }                                          \
  } while (0)

void prof_mark(dspw_handle* h, const char* name) {
  if (!h->prof_ev) return;
  cudaEvent_t e;
  cudaEventCreate(&e);
  cudaEventRecord(e, h->stream);
  h->prof_ev->push_back(e);
  h->prof_names->push_back(name);
}

int problem_dim(const dspw_desc& d) {
  if (d.nz > 1) return 3;
  if (d.ny > 1) return 2;
  return 1;
}

// ghost layers per side of a face stencil: 3 for eno 3, else 2
int ghost_width(const dspw_desc& d) { return d.recon == DSPW_REC_ENO3 ? 3 : 2; }

// halo layers stored on each side of the last swept direction (0: none)
int halo_layers(const dspw_desc& d) {
  const int D = problem_dim(d) - 1;
  return (d.bc[2 * D] == DSPW_BC_HALO || d.bc[2 * D + 1] == DSPW_BC_HALO) ? ghost_width(d) : 0;
}

// cells of one layer across the last swept direction (the layers are
// contiguous in memory: that direction is the outermost one of the problem)
long long layer_cells(const dspw_desc& d) {
  const int D = problem_dim(d) - 1;
  return D == 0 ? 1LL : (D == 1 ? (long long)d.nx : (long long)d.nx * d.ny);
}

int validate(const dspw_desc& d) {
  if (d.abi_version != DSPW_ABI_VERSION) return DSPW_ERR_ARG;
  if (d.model < 0 || d.model > 4) return DSPW_ERR_ARG;
  if (d.nx < 1 || d.ny < 1 || d.nz < 1) return DSPW_ERR_ARG;
  int dim = problem_dim(d);
  int N[3] = {d.nx, d.ny, d.nz};
  for (int k = 0; k < dim; k++)
    if (N[k] < 2) return DSPW_ERR_UNSUPPORTED;   // a swept direction needs >= 2 cells
  // eno 3 has three ghost cells: on a line of two cells the wall mirror of the
  // third would lie outside the line (periodic ghosts wrap, neumann ones copy)
  if (d.recon == DSPW_REC_ENO3)
    for (int k = 0; k < dim; k++)
      if (N[k] < 3 && (d.bc[2 * k] == DSPW_BC_WALL || d.bc[2 * k + 1] == DSPW_BC_WALL)) return DSPW_ERR_UNSUPPORTED;
  if (!(d.xmax > d.xmin) || !(d.ymax > d.ymin) || !(d.zmax > d.zmin)) return DSPW_ERR_ARG;
  if (d.precision != DSPW_FP64 && d.precision != DSPW_FP32_BF16) return DSPW_ERR_ARG;
  if (d.time_scheme < DSPW_RK1 || d.time_scheme > DSPW_RK4) return DSPW_ERR_UNSUPPORTED;
  if (d.recon < DSPW_REC_SP_WENO || d.recon > DSPW_REC_ENO3) return DSPW_ERR_UNSUPPORTED;
  bool scalar = d.model <= DSPW_BURGERS;
  if (scalar) {
    if (d.model == DSPW_LINADV && !(d.flux >= DSPW_LIN_EC && d.flux <= DSPW_LIN_TECNO4)) return DSPW_ERR_ARG;
    if (d.model == DSPW_BURGERS && !(d.flux >= DSPW_BUR_EC && d.flux <= DSPW_BUR_TECNO4)) return DSPW_ERR_ARG;
  } else {
    switch (d.flux) {
      case DSPW_KEPEC: case DSPW_KEPEC4: case DSPW_KEP: case DSPW_KEP4: case DSPW_ROE_EC: case DSPW_ROE_EC4:
      case DSPW_KEPS: case DSPW_KEPS4: case DSPW_ROE:
      case DSPW_KEP_TECNO_ROE: case DSPW_KEPES_TECNO_ROE: case DSPW_KEPES_TECNO_RUSANOV:
      case DSPW_ROE_TECNO_ROE: case DSPW_KEPES_TECNO4_ROE: case DSPW_KEPES_TECNO4_RUSANOV:
      case DSPW_ROE_TECNO4_ROE: break;
      default: return DSPW_ERR_UNSUPPORTED;
    }
    if (!(d.gamma > 1.0) || !(d.gas_const > 0.0)) return DSPW_ERR_ARG;
    if (d.model == DSPW_NS_ES || d.model == DSPW_NS_KEP) {
      if (dim != 3) return DSPW_ERR_UNSUPPORTED;
      for (int f = 0; f < 6; f++)
        if (d.bc[f] != DSPW_BC_PERIODIC) return DSPW_ERR_UNSUPPORTED;   // enflo/src/parameter.cc:564-568
      if (!(d.mu_ref > 0.0) || !(d.prandtl > 0.0)) return DSPW_ERR_ARG;
    }
  }
  for (int f = 0; f < 6; f++)
    if (d.bc[f] < 0 || d.bc[f] > DSPW_BC_HALO) return DSPW_ERR_ARG;
  // halo faces: the two faces of the last swept direction only, for the Euler
  // and scalar models, with at least one ghost width of interior layers to send
  for (int f = 0; f < 6; f++) {
    if (d.bc[f] != DSPW_BC_HALO) continue;
    if (f / 2 != dim - 1 || d.model == DSPW_NS_ES || d.model == DSPW_NS_KEP) return DSPW_ERR_UNSUPPORTED;
    if (N[dim - 1] < ghost_width(d)) return DSPW_ERR_UNSUPPORTED;
  }
  for (int a = 0; a < 3; a++)   // periodic must pair with periodic (enflo/src/parameter.cc:570-581)
    if ((d.bc[2 * a] == DSPW_BC_PERIODIC) != (d.bc[2 * a + 1] == DSPW_BC_PERIODIC)) return DSPW_ERR_ARG;
  if (!(d.cfl > 0.0) || !(d.final_time >= 0.0) || d.max_iter < 1 || d.t_stamps < 1) return DSPW_ERR_ARG;
  if (d.nn_use_box != 0 && d.nn_use_box != 1) return DSPW_ERR_ARG;
  if (d.nn_use_box)
    for (int k = 0; k < 5; k++)
      if (!(d.nn_feat_lo[k] <= d.nn_feat_hi[k])) return DSPW_ERR_ARG;   // also rejects NaN bounds
  if (d.generic_kernels != 0 && d.generic_kernels != 1) return DSPW_ERR_ARG;
  if (d.tile_staging < 0 || d.tile_staging > 3) return DSPW_ERR_ARG;
  for (int k = 0; k < 3; k++)
    if (!(d.cell_size[k] >= 0.0) || !std::isfinite(d.cell_size[k])) return DSPW_ERR_ARG;
  // unused slots stay zero, so that a later ABI version can give them a meaning
  for (int k = 0; k < 5; k++)
    if (d.reserved_i[k] != 0) return DSPW_ERR_ARG;
  for (int k = 0; k < 5; k++)
    if (d.reserved_d[k] != 0.0) return DSPW_ERR_ARG;
  return DSPW_OK;
}

// stages per time step (enflo/src/fv.cc:1268-1310)
int stages_of(int time_scheme) {
  return time_scheme == DSPW_RK1 ? 1 : (time_scheme == DSPW_SSPRK3 ? 3 : 4);
}

ProbDev make_prob(const dspw_desc& d, long long off) {
  ProbDev P;
  memset(&P, 0, sizeof(P));
  P.model = d.model;
  P.flux = d.flux;
  P.recon = d.recon;
  P.dim = problem_dim(d);
  P.is_scalar = d.model <= DSPW_BURGERS;
  P.nv = P.is_scalar ? 1 : P.dim + 2;
  P.nrk = stages_of(d.time_scheme);
  P.nx = d.nx; P.ny = d.ny; P.nz = d.nz;
  for (int f = 0; f < 6; f++) P.bc[f] = d.bc[f];
  P.ec1 = d.ec1_fix;
  P.mu_model = d.mu_model;
  P.max_iter = d.max_iter;
  P.off = off;
  P.dx = (d.xmax - d.xmin) / d.nx;   // enflo/src/fv.cc:29-31
  P.dy = (d.ymax - d.ymin) / d.ny;
  P.dz = (d.zmax - d.zmin) / d.nz;
  // a slab of a decomposed domain keeps the domain's cell size bit for bit
  // (its own bounds divided by its own cell count need not round to it)
  if (d.cell_size[0] > 0.0) P.dx = d.cell_size[0];
  if (d.cell_size[1] > 0.0) P.dy = d.cell_size[1];
  if (d.cell_size[2] > 0.0) P.dz = d.cell_size[2];
  P.hmin = std::min(P.dx, std::min(P.dy, P.dz));
  P.vol = P.dx * P.dy * P.dz;
  P.node_vol = (d.xmax - d.xmin) / (d.nx + 1) * (d.ymax - d.ymin) / (d.ny + 1) * (d.zmax - d.zmin) / (d.nz + 1);
  P.area[0] = P.dy * P.dz;           // num_flux face areas (enflo/src/kepec.cc:38-44)
  P.area[1] = P.dx * P.dz;
  P.area[2] = P.dx * P.dy;
  for (int k = 0; k < 3; k++) P.rarea[k] = 1 / P.area[k];
  P.gamma = d.gamma; P.gas_const = d.gas_const; P.prandtl = d.prandtl;
  P.mu_ref = d.mu_ref; P.T_ref = d.T_ref; P.T_0 = d.T_0; P.omega = d.omega;
  P.Cp = d.gamma * d.gas_const / (d.gamma - 1.0);
  for (int k = 0; k < 3; k++) P.lin_vel[k] = d.lin_vel[k];
  P.lin_speed = std::sqrt(d.lin_vel[0] * d.lin_vel[0] + d.lin_vel[1] * d.lin_vel[1] + d.lin_vel[2] * d.lin_vel[2]);
  for (int k = 0; k < 3; k++) {
    double n[3] = {0, 0, 0};
    n[k] = 1;
    P.lin_vn[k] = n[0] * d.lin_vel[0] + n[1] * d.lin_vel[1] + n[2] * d.lin_vel[2];
  }
  P.cfl = d.cfl;
  P.final_time = d.final_time;
  P.t_interval = d.final_time / d.t_stamps;
  for (int f = 0; f < 6; f++)
    for (int c = 0; c < 5; c++) P.bc_state[f][c] = d.bc_state[f][c];
  // flux structure
  P.central = 0; P.fourth = 0; P.tecno = 0; P.rusanov = 0;
  switch (d.flux) {
    case DSPW_LIN_EC4: case DSPW_BUR_EC4: P.fourth = 1; break;
    case DSPW_LIN_TECNO: case DSPW_BUR_TECNO: P.tecno = 1; break;
    case DSPW_LIN_TECNO4: case DSPW_BUR_TECNO4: P.tecno = 1; P.fourth = 1; break;
    case DSPW_KEPEC: break;
    case DSPW_KEPEC4: P.fourth = 1; break;
    case DSPW_KEP: P.central = 1; break;
    case DSPW_KEP4: P.central = 1; P.fourth = 1; break;
    case DSPW_ROE_EC: P.central = 2; break;
    case DSPW_ROE_EC4: P.central = 2; P.fourth = 1; break;
    case DSPW_KEPS: P.central = 3; break;
    case DSPW_KEPS4: P.central = 3; P.fourth = 1; break;
    case DSPW_ROE: P.central = 4; break;
    case DSPW_KEP_TECNO_ROE: P.central = 1; P.tecno = 1; P.ec1 = 0; break;   // no EC1_fix (kep_tecno_roe.cc)
    case DSPW_KEPES_TECNO_ROE: P.tecno = 1; break;
    case DSPW_KEPES_TECNO_RUSANOV: P.tecno = 1; P.rusanov = 1; P.ec1 = 0; break;
    case DSPW_ROE_TECNO_ROE: P.central = 2; P.tecno = 1; break;
    case DSPW_KEPES_TECNO4_ROE: P.tecno = 1; P.fourth = 1; break;
    case DSPW_KEPES_TECNO4_RUSANOV: P.tecno = 1; P.fourth = 1; P.rusanov = 1; P.ec1 = 0; break;
    case DSPW_ROE_TECNO4_ROE: P.central = 2; P.tecno = 1; P.fourth = 1; break;
    default: break;
  }
  P.spw_corr = d.recon == DSPW_REC_SP_WENO_DL ? -1 : (d.recon == DSPW_REC_SP_WENOC ? 1 : (d.recon == DSPW_REC_SP_WENO_CORR2 ? 2 : 0));
  return P;
}

NetParams make_net(const dspw_desc& dn) {
  NetParams np;
  memset(&np, 0, sizeof(np));
  // the FP32 form's last layer yields base-2 logits (its softmax uses 2^x)
  const double log2e = 1.4426950408889634;
  for (int l = 0; l < 4; l++)
    for (int j = 0; j < 5; j++) {
      const double f = l == 3 ? log2e : 1.0;
      np.b[l][j] = dn.nn_b[l][j];
      np.bf[l][j] = (float)(dn.nn_b[l][j] * f);
      for (int k = 0; k < 5; k++) {
        np.w[l][j][k] = dn.nn_w[l][j][k];
        np.wf[l][j][k] = (float)(dn.nn_w[l][j][k] * f);
      }
    }
  // nn_use_box: the network carries a training box of its inputs; inputs
  // outside it use plain SP-WENO
  np.use_box = dn.nn_use_box ? 1 : 0;
  for (int k = 0; k < 5; k++) { np.feat_lo[k] = -1e30f; np.feat_hi[k] = 1e30f; }
  if (np.use_box)
    for (int k = 0; k < 5; k++) { np.feat_lo[k] = (float)dn.nn_feat_lo[k]; np.feat_hi[k] = (float)dn.nn_feat_hi[k]; }
  return np;
}

// Sweep kernels of one problem: Euler / NS problems with the 4th-order KEPEC
// central part plus TeCNO dissipation run the kernels specialised for their
// dimension and reconstruction family; every other problem the generic ones.
int spec_of(const ProbDev& P, const dspw_desc& d) {
  if (d.generic_kernels == 1) return 0;   // generic kernels requested
  if (P.is_scalar)   // 1-D linear advection / Burgers with an SP-WENO-family or network reconstruction
    return (P.dim == 1 && P.recon < DSPW_REC_FIRST) ? scalar_spec_code(P.spw_corr < 0 ? 2 : 1) : 0;
  if (P.central != 0 || !P.fourth || !P.tecno || P.recon >= DSPW_REC_FIRST) return 0;
  return spec_code(P.dim, P.spw_corr < 0 ? 2 : 1);
}

// Tasks of one problem in direction dir: warp tasks (one line segment each),
// or, for the y / z sweeps of a specialised batch, block tasks of `cols`
// adjacent columns (decode_group: 8, or 4 for the narrow tiles).
long long tasks_for(const ProbDev& P, int dir, bool groups, int cols = WARPS_PER_BLOCK) {
  if (dir >= P.dim) return 0;
  int N[3] = {P.nx, P.ny, P.nz};
  long long nseg = (N[dir] + SEG_CELLS - 1) / SEG_CELLS;
  long long other = (long long)P.nx * P.ny * P.nz / N[dir];
  if (groups && dir >= 1) return nseg * (other / P.nx) * ((P.nx + cols - 1) / cols);
  return nseg * other;
}

// The task list (prefix sums over the class's problems) of one direction, for
// the class's current tile width; uploaded when the device copy exists.
int class_tasks(SweepClass& c, const std::vector<ProbDev>& prob, int dir) {
  const int cols = (c.spec != 0 && dir >= 1 && c.narrow[dir]) ? NARROW_COLS : WARPS_PER_BLOCK;
  std::vector<int> ts(1, 0);
  for (int p : c.probs) {
    const long long nt = (long long)ts.back() + tasks_for(prob[p], dir, c.spec != 0, cols);
    if (nt > (1LL << 30)) return DSPW_ERR_ARG;
    ts.push_back((int)nt);
  }
  c.task_start[dir] = ts;
  if (c.dtask[dir] &&
      cudaMemcpy(c.dtask[dir], ts.data(), sizeof(int) * ts.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return DSPW_ERR_CUDA;
  return DSPW_OK;
}

void* buf(dspw_handle* h, int which) {
  switch (which) {
    case 0: return h->Un;
    case 1: return h->Ua;
    default: return h->Ub;
  }
}

template <typename T>
DiagArgs<T> diag_args(dspw_handle* h, const long long* start, const T* U) {
  DiagArgs<T> d;
  memset(&d, 0, sizeof(d));
  d.prob = h->dprob;
  d.st = h->dst;
  d.acc = h->ddiag;
  d.part = h->ddiag_part;
  d.nprob = h->nprob;
  d.start = start;
  d.U = U;
  d.R = (const T*)h->R;
  d.node = (const T*)h->node;
  d.ctot = h->ctot;
  d.rows = h->drows;
  d.cap = h->diag_cap;
  return d;
}

// Move the rows written since the last drain from the device ring into the
// per-problem host lists.  Rows of a problem beyond the ring's capacity since
// the last drain were overwritten and are counted as dropped.
int drain_diag(dspw_handle* h) {
  if (h->diag_cap == 0) return DSPW_OK;
  const int np = h->nprob;
  std::vector<DiagAcc> acc(np);
  CK(cudaMemcpyAsync(acc.data(), h->ddiag, sizeof(DiagAcc) * np, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  unsigned long long lo = ~0ull, hi = 0;
  for (int p = 0; p < np; p++) {
    unsigned long long from = h->diag_taken[p], to = acc[p].count;
    if (to - from > (unsigned long long)h->diag_cap) {
      h->diag_dropped[p] += (long long)(to - from - h->diag_cap);
      from = to - h->diag_cap;
      h->diag_taken[p] = from;
    }
    if (to > from) { lo = std::min(lo, from); hi = std::max(hi, to); }
  }
  if (hi == 0) return DSPW_OK;
  // slots lo .. hi-1 (at most diag_cap of them), in one or two contiguous runs
  const size_t row_bytes = sizeof(double) * DIAG_COLS * np;
  const unsigned long long n = hi - lo, cap = h->diag_cap;
  std::vector<double> buf((size_t)n * DIAG_COLS * np);
  const unsigned long long s0 = lo % cap, first = std::min(n, cap - s0);
  CK(cudaMemcpyAsync(buf.data(), h->drows + s0 * DIAG_COLS * np, first * row_bytes, cudaMemcpyDeviceToHost,
                     h->stream));
  if (n > first)
    CK(cudaMemcpyAsync(buf.data() + first * DIAG_COLS * np, h->drows, (n - first) * row_bytes,
                       cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int p = 0; p < np; p++) {
    for (unsigned long long r = h->diag_taken[p]; r < acc[p].count; r++) {
      const double* row = buf.data() + ((r - lo) * np + p) * DIAG_COLS;
      h->diag_host[p].insert(h->diag_host[p].end(), row, row + DIAG_COLS);
    }
    h->diag_taken[p] = acc[p].count;
  }
  return DSPW_OK;
}

// Move the snapshots taken since the last drain from the device ring to host
// memory as primitive planes.  A problem with more than snap_slots new
// snapshots lost the oldest ones (counted as dropped).
int drain_snap(dspw_handle* h) {
  if (h->snap_slots == 0) return DSPW_OK;
  const int np = h->nprob;
  std::vector<unsigned long long> count(np);
  std::vector<SnapMeta> meta((size_t)np * h->snap_slots);
  CK(cudaMemcpyAsync(count.data(), h->dsnap_count, sizeof(unsigned long long) * np, cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaMemcpyAsync(meta.data(), h->dsnap_meta, sizeof(SnapMeta) * meta.size(), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const size_t slot_bytes = (size_t)h->elem * 5 * (size_t)h->ctot;
  for (int p = 0; p < np; p++) {
    unsigned long long from = h->snap_taken[p];
    if (count[p] - from > (unsigned long long)h->snap_slots) {
      h->snap_dropped[p] += (long long)(count[p] - from - h->snap_slots);
      from = count[p] - h->snap_slots;
    }
    const dspw_desc& d = h->desc[p];
    const size_t nvals = (size_t)(d.model <= DSPW_BURGERS ? 1 : 5) * (size_t)d.nx * d.ny * d.nz;
    for (unsigned long long c = from; c < count[p]; c++) {
      const unsigned long long slot = c % (unsigned long long)h->snap_slots;
      dspw_handle::HostSnap s;
      s.time = meta[slot * np + p].time;
      s.iter = meta[slot * np + p].iter;
      s.prim.resize(nvals);
      int r = download(h, p, s.prim.data(), 1, (char*)h->dsnap + slot * slot_bytes);
      if (r) return r;
      h->snap_host[p].push_back(std::move(s));
    }
    h->snap_taken[p] = count[p];
  }
  return DSPW_OK;
}

// state buffer that stage rk reads (0: U^n, 1: Ua, 2: Ub), see stage_args
int stage_input(const dspw_handle* h, int rk) {
  static const int in4[4] = {0, 1, 2, 1};
  if (h->nrk == 1) return 0;
  if (h->nrk == 3) return rk == 0 ? 0 : (rk == 1 ? 1 : 2);
  return in4[rk];
}

// sweep arguments of stage rk (residual_only: write R in every sweep)
template <typename T>
SweepArgs<T> stage_args(dspw_handle* h, int rk, int residual_only) {
  SweepArgs<T> a;
  memset(&a, 0, sizeof(a));
  a.prob = h->dprob;
  a.st = h->dst;
  a.nprob = h->nprob;
  // stage buffers: SSPRK3 U^n -> Ua -> Ub -> U^n, the four-stage schemes
  // U^n -> Ua -> Ub -> Ua -> U^n (the last stage writes in place: every cell
  // reads its own U^n entry before overwriting it, and no sweep of that stage
  // reads U^n); RK1 U^n -> Ua, copied back after the stage
  static const int out4[4] = {1, 2, 1, 0};
  int in = stage_input(h, rk), out;
  if (h->nrk == 1) out = 1;
  else if (h->nrk == 3) out = rk == 0 ? 1 : (rk == 1 ? 2 : 0);
  else out = out4[rk];
  if (residual_only) { in = 0; out = 1; }
  a.Uin = (const T*)buf(h, in);
  a.tma_in = in;
  a.Un = (const T*)h->Un;
  a.Uout = (T*)buf(h, out);
  a.R = (T*)h->R;
  a.ctot = h->ctot;
  a.rk = rk;
  a.scheme = h->time_scheme;
  a.R2 = (T*)h->R2;
  static const double ark[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0};   // enflo/src/ext_constants.h:7-8
  static const double brk[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
  a.a_rk = rk < 3 ? ark[rk] : 0.0;
  a.b_rk = rk < 3 ? brk[rk] : 0.0;
  a.final_stage = (rk == h->nrk - 1) && !residual_only;
  a.residual_only = residual_only;
  a.store_R = h->diag_cap > 0 && !residual_only && (rk == 0 || rk == h->nrk - 1);
  a.status = h->dstatus;
  a.net = h->dnet;
  a.collect_buf = residual_only ? h->collect_buf : nullptr;
  a.collect_count = h->collect_count;
  a.collect_cap = h->collect_cap;
  a.collect_stride = h->collect_stride ? h->collect_stride : 1;
  // NS problems never update in a sweep; mixed batches are not formed with NS
  a.viscous = h->has_ns ? 1 : 0;
  return a;
}

// grid of one class's sweep: the tuned one, else one block per 8 warp tasks or
// per column group (specialised y / z sweeps)
int default_grid(const SweepClass& c, int dir) {
  int nt = c.task_start[dir].back();
  return (c.spec && dir >= 1) ? nt : (nt + WARPS_PER_BLOCK - 1) / WARPS_PER_BLOCK;
}

template <typename T>
cudaError_t launch_class_sweep(dspw_handle* h, SweepArgs<T> a, const SweepClass& c, int dir) {
  a.task_start = c.dtask[dir];
  a.pmap = c.dpmap;
  a.nprob = (int)c.probs.size();
  a.ntask = c.task_start[dir].back();
  a.tmaps = c.dtmap;
  a.narrow = (c.spec != 0 && dir >= 1 && c.narrow[dir]) ? 1 : 0;
  a.tma = (!a.narrow && c.dtmap && dir >= 1 && c.use_tma[dir]) ? 1 : 0;
  int grid = c.grid[dir] ? c.grid[dir] : default_grid(c, dir);
  return Launch<T>::sweep(dir, a, grid, h->stream, c.spec);
}

int enqueue_halo_exchange(dspw_handle* h, int rk);

// cuTensorMapEncodeTiled of the driver, found through the runtime (no link
// against libcuda); null when the driver does not offer it
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiledFn) nullptr;
    return (EncodeTiledFn)f;
  }();
  return fn;
}

// Tensor maps of the TMA staging for every specialised class of dimension 2
// or 3 whose problems all have nx a multiple of 8 and 16-byte aligned rows and
// planes: per problem and y / z direction, the three stage inputs with a box of
// 8 x SEG_LOAD rows x nv planes, the residual and U^n with a box of
// 8 x SEG_CELLS rows (tma_map_index).  The tensor of a problem is its interior
// (nx, ny, nz) x nv planes; the box moves along the sweep direction.  A class
// that does not qualify, or any encoding failure, keeps dtmap null: its sweeps
// stage with cp.async.
void build_tma_maps(dspw_handle* h) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return;
  const int w = (int)h->elem, vec = 16 / w;
  void* bufs[5] = {h->Un, h->Ua, h->Ub, h->R, h->Un};
  for (SweepClass& c : h->classes) {
    const int dim = c.spec >= 100 ? 1 : c.spec / 10;
    if (c.spec == 0 || dim < 2) continue;
    bool ok = h->ctot % vec == 0;
    bool forced = true;
    for (int p : c.probs) {
      const ProbDev& P = h->hprob[p];
      ok = ok && P.nx % COOP_COLS == 0 && P.off % vec == 0 && h->desc[p].tile_staging != 1 &&
           h->desc[p].tile_staging != 3;
      forced = forced && h->desc[p].tile_staging == 2;
    }
    if (!ok) continue;
    const size_t n = c.probs.size();
    std::vector<CUtensorMap> maps(n * 2 * TMA_SLOTS);
    static_assert(sizeof(CUtensorMap) == TMA_MAP_BYTES, "tensor map size");
    for (size_t i = 0; i < n && ok; i++) {
      const ProbDev& P = h->hprob[c.probs[i]];
      const cuuint64_t gdim[4] = {(cuuint64_t)P.nx, (cuuint64_t)P.ny, (cuuint64_t)P.nz, (cuuint64_t)P.nv};
      const cuuint64_t gstride[3] = {(cuuint64_t)P.nx * w, (cuuint64_t)P.nx * P.ny * w, (cuuint64_t)h->ctot * w};
      const cuuint32_t estride[4] = {1, 1, 1, 1};
      for (int dir = 1; dir < dim && ok; dir++)
        for (int slot = 0; slot < TMA_SLOTS && ok; slot++) {
          const cuuint32_t rows = slot < 3 ? SEG_LOAD : SEG_CELLS;
          const cuuint32_t box[4] = {(cuuint32_t)COOP_COLS, dir == 1 ? rows : 1u, dir == 2 ? rows : 1u,
                                     (cuuint32_t)P.nv};
          void* addr = (char*)bufs[slot] + (size_t)w * P.off;
          ok = enc(&maps[tma_map_index((int)i, dir, slot)],
                   w == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, addr, gdim, gstride,
                   box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
        }
    }
    if (!ok) continue;
    void* d = nullptr;
    if (cudaMalloc(&d, maps.size() * sizeof(CUtensorMap)) != cudaSuccess) continue;
    if (cudaMemcpy(d, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaFree(d);
      continue;
    }
    c.dtmap = d;
    c.tma_forced = forced ? 1 : 0;
    c.use_tma[1] = c.use_tma[2] = c.tma_forced;
  }
}

template <typename T>
int enqueue_stage(dspw_handle* h, int rk, int residual_only) {
  SweepArgs<T> a = stage_args<T>(h, rk, residual_only);
  if (!residual_only) {   // the collective path only (residuals and tuning stay rank-local)
    int rx = enqueue_halo_exchange(h, rk);
    if (rx) return rx;
  }
  if (h->has_ns) {
    CK(Launch<T>::entvars(h->dprob, h->nprob, h->dcell_start, h->ctot, a.Uin, h->ctot, (T*)h->V, h->stream));
    prof_mark(h, "entvars");
    CK(Launch<T>::visc_nodes(h->dprob, h->nprob, h->dcell_start, h->ctot, (const T*)h->V, h->ctot, (T*)h->node,
                             h->stream));
    prof_mark(h, "visc_nodes");
  }
  for (int dir = 0; dir < h->maxdim; dir++) {
    for (const SweepClass& c : h->classes) {
      if (c.task_start[dir].back() == 0) continue;
      CK(launch_class_sweep<T>(h, a, c, dir));
      std::string name = dir == 0 ? "sweep_x" : (dir == 1 ? "sweep_y" : "sweep_z");
      if (h->classes.size() > 1) name += ".c" + std::to_string(c.spec);
      prof_mark(h, name.c_str());
    }
  }
  const bool diag = h->diag_cap > 0 && !residual_only;
  if (diag && rk == 0) {
    // U^n is intact during stage 0 (it writes Ua); R holds its inviscid residual
    DiagArgs<T> da = diag_args<T>(h, h->dcell_start, (const T*)h->Un);
    CK(Launch<T>::diag_cells(da, 0, h->ctot, h->stream));
    if (h->nodes_tot > 0) {
      da.start = h->dnode_start;
      CK(Launch<T>::diag_nodes(da, h->nodes_tot, h->stream));
    }
    prof_mark(h, "diag_stage0");
  }
  if (h->has_ns) {
    CK(Launch<T>::visc_update(a, h->dcell_start, h->ctot, (const T*)h->node, h->stream));
    prof_mark(h, "visc_update");
  }
  if (h->nrk == 1 && !residual_only)
    CK(cudaMemcpyAsync(h->Un, h->Ua, h->elem * h->ctot * 5, cudaMemcpyDeviceToDevice, h->stream));
  if (diag && rk == h->nrk - 1) {
    // U^(n+1) is in U^n's buffer; R holds the last stage's residual
    DiagArgs<T> da = diag_args<T>(h, h->dcell_start, (const T*)h->Un);
    CK(Launch<T>::diag_cells(da, 1, h->ctot, h->stream));
    CK(Launch<T>::diag_row(da, h->stream));
    prof_mark(h, "diag_row");
  }
  return DSPW_OK;
}

// Launch autotuner: for every kernel class and direction, time the sweep
// (residual evaluation of the current state, which writes only the residual
// buffer) with its default grid and with persistent grids of 1, 2 and 4 times
// the resident blocks of the whole GPU; the specialised y / z sweeps also with
// both tile widths (8 columns, 4 columns) and, for 8 columns with tensor maps,
// both stagings (cp.async, TMA).  The fastest candidate is kept.
template <typename T>
int tune_grids(dspw_handle* h, int reps, double* before_ms, double* after_ms) {
  int dev = 0, nsm = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  StatusDev saved;
  CK(cudaMemcpy(&saved, h->dstatus, sizeof(saved), cudaMemcpyDeviceToHost));
  SweepArgs<T> a = stage_args<T>(h, 0, 1);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  double tot_before = 0.0, tot_after = 0.0;
  int ret = DSPW_OK;
  for (SweepClass& c : h->classes) {
    for (int dir = 0; dir < h->maxdim; dir++) {
      if (c.task_start[dir].back() == 0) continue;
      // tile widths: the specialised y / z sweeps of a 2-D / 3-D class also
      // try the narrow tiles (4 columns, cp.async), unless the problems fix
      // the staging
      const int tma0 = c.use_tma[dir], nw0 = c.narrow[dir];
      std::vector<int> widths = {nw0};
      if (c.spec != 0 && c.spec < 100 && dir >= 1 && !c.tma_forced && !c.narrow_forced) widths.push_back(1 - nw0);
      double best = 1e300;
      int best_grid = 0, best_tma = tma0, best_nw = nw0;
      for (int nw : widths) {
        if (c.narrow[dir] != nw) {
          c.narrow[dir] = nw;
          if (class_tasks(c, h->hprob, dir) != DSPW_OK) { ret = DSPW_ERR_CUDA; break; }
        }
        const int g0 = default_grid(c, dir);
        const int bpsm = Launch<T>::sweep_blocks_per_sm(dir, c.spec, nw);
        std::vector<int> grids = {0};
        for (int k : {1, 2, 4})
          if (bpsm > 0 && (long long)nsm * bpsm * k < g0) grids.push_back(nsm * bpsm * k);
        // candidates (grid, staging): the 8-column y / z sweeps of a class
        // with tensor maps also try the other staging (TMA / cp.async)
        std::vector<std::pair<int, int>> cand;
        for (int g : grids) {
          cand.push_back({g, nw ? 0 : tma0});
          if (!nw && c.dtmap && dir >= 1 && !c.tma_forced) cand.push_back({g, 1 - tma0});
        }
        for (auto [g, tm] : cand) {
          c.grid[dir] = g;
          c.use_tma[dir] = tm;
          std::vector<float> t(reps);
          for (int r = 0; r < reps && ret == DSPW_OK; r++) {
            if (cudaEventRecord(e0, h->stream) != cudaSuccess ||
                launch_class_sweep<T>(h, a, c, dir) != cudaSuccess ||
                cudaEventRecord(e1, h->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                cudaEventElapsedTime(&t[r], e0, e1) != cudaSuccess)
              ret = DSPW_ERR_CUDA;
          }
          if (ret) break;
          std::sort(t.begin(), t.end());
          const double med = t[reps / 2];
          if (g == 0 && tm == tma0 && nw == nw0) tot_before += med;
          if (med < best) { best = med; best_grid = g; best_tma = tm; best_nw = nw; }
        }
        if (ret) break;
      }
      if (ret) break;
      if (c.narrow[dir] != best_nw) {
        c.narrow[dir] = best_nw;
        if (class_tasks(c, h->hprob, dir) != DSPW_OK) { ret = DSPW_ERR_CUDA; break; }
      }
      c.grid[dir] = best_grid;
      c.use_tma[dir] = best_tma;
      tot_after += best;
    }
    if (ret) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ret) {
    for (SweepClass& c : h->classes) {
      c.grid[0] = c.grid[1] = c.grid[2] = 0;
      c.use_tma[0] = 0;
      c.use_tma[1] = c.use_tma[2] = c.dtmap ? c.tma_forced : 0;
      c.narrow[1] = c.narrow[2] = c.narrow_forced;
      for (int dir = 1; dir < 3; dir++) class_tasks(c, h->hprob, dir);
    }
  }
  // the timing runs counted faces; the status is the solver's, not the tuner's
  if (cudaMemcpy(h->dstatus, &saved, sizeof(saved), cudaMemcpyHostToDevice) != cudaSuccess) ret = DSPW_ERR_CUDA;
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
  if (before_ms) *before_ms = tot_before;
  if (after_ms) *after_ms = tot_after;
  return ret;
}

int enqueue_stage_any(dspw_handle* h, int rk, int residual_only) {
  return h->precision == DSPW_FP64 ? enqueue_stage<double>(h, rk, residual_only)
                                   : enqueue_stage<float>(h, rk, residual_only);
}

// end of a step: time, iteration and time-stamp bookkeeping, then the
// snapshot of the problems that reached a stamp
template <typename T>
int enqueue_end_step_t(dspw_handle* h) {
  CK(launch_end_step(h->dprob, h->dst, h->nprob, h->stream));
  if (h->snap_slots > 0) {
    SnapArgs<T> a;
    memset(&a, 0, sizeof(a));
    a.prob = h->dprob;
    a.st = h->dst;
    a.nprob = h->nprob;
    a.cell_start = h->dcell_start;
    a.U = (const T*)h->Un;
    a.slots = (T*)h->dsnap;
    a.ctot = h->ctot;
    a.nslots = h->snap_slots;
    a.count = h->dsnap_count;
    a.meta = h->dsnap_meta;
    CK(Launch<T>::snap(a, h->ctot, h->stream));
  }
  return DSPW_OK;
}

int enqueue_end_step(dspw_handle* h) {
  return h->precision == DSPW_FP64 ? enqueue_end_step_t<double>(h) : enqueue_end_step_t<float>(h);
}

// NCCL, opened at run time (the process's own libnccl.so.2 when one is loaded,
// e.g. by torch), so that the library loads and runs without it
struct NcclApi {
  bool ok = false;
  ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
  ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
  ncclResult_t (*send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*group_start)() = nullptr;
  ncclResult_t (*group_end)() = nullptr;
  ncclResult_t (*all_reduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                             cudaStream_t) = nullptr;
};

const NcclApi& nccl() {
  static const NcclApi api = [] {
    NcclApi a;
    void* lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!lib) return a;
    a.get_unique_id = (decltype(a.get_unique_id))dlsym(lib, "ncclGetUniqueId");
    a.comm_init_rank = (decltype(a.comm_init_rank))dlsym(lib, "ncclCommInitRank");
    a.comm_destroy = (decltype(a.comm_destroy))dlsym(lib, "ncclCommDestroy");
    a.send = (decltype(a.send))dlsym(lib, "ncclSend");
    a.recv = (decltype(a.recv))dlsym(lib, "ncclRecv");
    a.group_start = (decltype(a.group_start))dlsym(lib, "ncclGroupStart");
    a.group_end = (decltype(a.group_end))dlsym(lib, "ncclGroupEnd");
    a.all_reduce = (decltype(a.all_reduce))dlsym(lib, "ncclAllReduce");
    a.ok = a.get_unique_id && a.comm_init_rank && a.comm_destroy && a.send && a.recv && a.group_start &&
           a.group_end && a.all_reduce;
    return a;
  }();
  return api;
}

#define NCK(x)                                                     \
  do {                                                             \
    if ((x) != ncclSuccess) {                                      \
      h->last_error = DSPW_ERR_CUDA;                               \
      return DSPW_ERR_CUDA;                                        \
    }                                                              \
  } while (0)

// CFL speed of the newest state in slot 0 (max of the slots), the others
// cleared: the value an all-reduce(max) over the ranks combines
__global__ void k_smax_pack(ProbState* st) {
  unsigned long long m = 0ull;
  for (int k = 0; k < EPI_SLOTS; k++) m = st->smax[k] > m ? st->smax[k] : m;
  for (int k = 1; k < EPI_SLOTS; k++) st->smax[k] = 0ull;
  st->smax[0] = m;
}

// the speed of the whole decomposed domain: max over the ranks of each
// slab's (non-negative doubles order as their bit patterns)
int enqueue_speed_reduce(dspw_handle* h) {
  if (!h->comm) return DSPW_OK;
  k_smax_pack<<<1, 1, 0, h->stream>>>(h->dst);
  CK(cudaGetLastError());
  unsigned long long* s0 = (unsigned long long*)((char*)h->dst + offsetof(ProbState, smax));
  NCK(nccl().all_reduce(s0, s0, 1, ncclUint64, ncclMax, h->comm, h->stream));
  return DSPW_OK;
}

// Halo layers of the state stage rk reads, from the neighbouring ranks: phase
// 1 upwards (send_hi to the upper rank, recv_lo from the lower), phase 2
// downwards, each one NCCL group in which every pair of ranks has one message
// per component in component order on both sides, so the pairs match also
// when both neighbours are one rank (two slabs, periodic) or this rank itself
// (one periodic slab).
int enqueue_halo_exchange(dspw_handle* h, int rk) {
  if (!h->comm) return DSPW_OK;
  dspw_halo_out v;
  if (dspw_halo_view(h, 0, rk, &v) != DSPW_OK) return DSPW_OK;   // no halo faces: nothing to exchange
  const ncclDataType_t t = h->elem == 8 ? ncclFloat64 : ncclFloat32;
  const size_t cs = (size_t)v.comp_stride * h->elem;
  const NcclApi& n = nccl();
  // a failed send / recv still closes its group, so that no NCCL group stays
  // open on this thread
#define NCKG(x)                                  \
  do {                                           \
    if ((x) != ncclSuccess) {                    \
      n.group_end();                             \
      h->last_error = DSPW_ERR_CUDA;             \
      return DSPW_ERR_CUDA;                      \
    }                                            \
  } while (0)
  NCK(n.group_start());
  for (int c = 0; c < v.ncomp; c++) {
    if (h->up >= 0) NCKG(n.send((char*)v.send_hi + c * cs, v.count, t, h->up, h->comm, h->stream));
    if (h->down >= 0) NCKG(n.recv((char*)v.recv_lo + c * cs, v.count, t, h->down, h->comm, h->stream));
  }
  NCK(n.group_end());
  NCK(n.group_start());
  for (int c = 0; c < v.ncomp; c++) {
    if (h->down >= 0) NCKG(n.send((char*)v.send_lo + c * cs, v.count, t, h->down, h->comm, h->stream));
    if (h->up >= 0) NCKG(n.recv((char*)v.recv_hi + c * cs, v.count, t, h->up, h->comm, h->stream));
  }
  NCK(n.group_end());
#undef NCKG
  return DSPW_OK;
}

int enqueue_step(dspw_handle* h, double fixed_dt) {
  CK(cudaMemsetAsync(h->dnactive, 0, sizeof(int), h->stream));
  if (fixed_dt <= 0) {
    int rs = enqueue_speed_reduce(h);
    if (rs) return rs;
  }
  CK(launch_begin_step(h->dprob, h->dst, h->nprob, fixed_dt, h->dnactive, h->stream));
  prof_mark(h, "begin_step");
  for (int rk = 0; rk < h->nrk; rk++) {
    int r = enqueue_stage_any(h, rk, 0);
    if (r) return r;
  }
  int re = enqueue_end_step(h);
  if (re) return re;
  prof_mark(h, "end_step");
  return DSPW_OK;
}

int build_graph(dspw_handle* h, double fixed_dt) {
  if (h->graph && h->graph_dt == fixed_dt) return DSPW_OK;
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int r = enqueue_step(h, fixed_dt);
  cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  if (r) return r;
  if (e != cudaSuccess) { h->last_error = DSPW_ERR_CUDA; return DSPW_ERR_CUDA; }
  e = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { h->graph = nullptr; h->last_error = DSPW_ERR_CUDA; return DSPW_ERR_CUDA; }
  h->graph_dt = fixed_dt;
  return DSPW_OK;
}

long long ncells(const dspw_desc& d) { return (long long)d.nx * d.ny * d.nz; }

int check_p(dspw_handle* h, int p) { return (!h || p < 0 || p >= h->nprob) ? DSPW_ERR_ARG : DSPW_OK; }

}  // namespace

namespace dspw {
int handle_collect(dspw_handle* h, float* buf, unsigned long long* count, unsigned long long cap, unsigned stride) {
  h->collect_buf = buf;
  h->collect_count = count;
  h->collect_cap = cap;
  h->collect_stride = stride;
  int r = enqueue_stage_any(h, 0, 1);
  h->collect_buf = nullptr;
  h->collect_count = nullptr;
  if (r) return r;
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return DSPW_ERR_CUDA;
  return DSPW_OK;
}
int handle_precision(const dspw_handle* h) { return h->precision; }
ProbDev make_prob_public(const dspw_desc& d, long long off) { return make_prob(d, off); }
NetParams make_net_public(const dspw_desc& d) { return make_net(d); }
}  // namespace dspw

// ------------------------------------------------------------------ C ABI --

extern "C" {

const char* dspw_error_string(int code) {
  switch (code) {
    case DSPW_OK: return "DSPW_OK";
    case DSPW_ERR_ARG: return "DSPW_ERR_ARG: bad argument or descriptor";
    case DSPW_ERR_CUDA: return "DSPW_ERR_CUDA: a CUDA runtime call failed";
    case DSPW_ERR_NONFINITE: return "DSPW_ERR_NONFINITE: NaN or Inf in the state";
    case DSPW_ERR_NONPOSITIVE: return "DSPW_ERR_NONPOSITIVE: density or pressure <= 0";
    case DSPW_ERR_TIMEOUT: return "DSPW_ERR_TIMEOUT: a bounded device wait gave up";
    case DSPW_ERR_UNSUPPORTED: return "DSPW_ERR_UNSUPPORTED: combination not implemented";
    case DSPW_ERR_NOMEM: return "DSPW_ERR_NOMEM: device allocation failed";
    case DSPW_ERR_FINISHED: return "DSPW_ERR_FINISHED: problem reached final_time or max_iter";
    default: return "unknown dspw status";
  }
}

int dspw_version(void) { return DSPW_ABI_VERSION; }

int dspw_create(const dspw_desc* desc, dspw_handle** out) { return dspw_create_batch(desc, 1, out); }

int dspw_create_batch(const dspw_desc* descs, int nprob, dspw_handle** out) {
  if (!descs || !out || nprob < 1) return DSPW_ERR_ARG;
  *out = nullptr;
  for (int p = 0; p < nprob; p++) {
    int r = validate(descs[p]);
    if (r) return r;
    if (descs[p].precision != descs[0].precision || descs[p].time_scheme != descs[0].time_scheme) return DSPW_ERR_ARG;
  }
  dspw_handle* h = new dspw_handle;
  h->nprob = nprob;
  h->precision = descs[0].precision;
  h->time_scheme = descs[0].time_scheme;
  h->nrk = stages_of(h->time_scheme);
  h->elem = h->precision == DSPW_FP64 ? 8 : 4;
  h->desc.assign(descs, descs + nprob);
  long long off = 0;
  h->cell_start.push_back(0);
  for (int p = 0; p < nprob; p++) {
    // a problem with halo faces stores its ghost layers beside the interior:
    // its block is [halo, interior, halo]; cell_start bounds whole blocks
    const long long hc = halo_layers(descs[p]) * layer_cells(descs[p]);
    if (hc) h->has_halo = 1;
    h->hprob.push_back(make_prob(descs[p], off + hc));
    off += ncells(descs[p]) + 2 * hc;
    h->cell_start.push_back(off);
    h->maxcells = std::max(h->maxcells, ncells(descs[p]));
    h->maxdim = std::max(h->maxdim, h->hprob.back().dim);
    if (descs[p].model == DSPW_NS_ES || descs[p].model == DSPW_NS_KEP) h->has_ns = 1;
  }
  if (h->has_ns) {   // the viscous kernels run over the whole batch: Navier-Stokes problems only
    for (int p = 0; p < nprob; p++)
      if (descs[p].model != DSPW_NS_ES && descs[p].model != DSPW_NS_KEP) { delete h; return DSPW_ERR_UNSUPPORTED; }
  }
  h->ctot = off;
  // classes of problems sharing sweep kernels, in order of first appearance
  for (int p = 0; p < nprob; p++) {
    const int sc = spec_of(h->hprob[p], descs[p]);
    SweepClass* c = nullptr;
    for (SweepClass& k : h->classes)
      if (k.spec == sc) c = &k;
    if (!c) {
      h->classes.emplace_back();
      c = &h->classes.back();
      c->spec = sc;
    }
    c->probs.push_back(p);
  }
  for (SweepClass& c : h->classes) {
    // narrow tiles when every problem of a specialised 2-D / 3-D class asks for them
    bool narrow = c.spec != 0 && c.spec < 100;
    for (int p : c.probs) narrow = narrow && descs[p].tile_staging == 3 && h->hprob[p].dim >= 2;
    c.narrow_forced = narrow ? 1 : 0;
    c.narrow[1] = c.narrow[2] = c.narrow_forced;
    for (int dir = 0; dir < 3; dir++)
      if (class_tasks(c, h->hprob, dir) != DSPW_OK) { delete h; return DSPW_ERR_ARG; }
  }
  // network parameters (shared by the batch; taken from the first DL problem)
  const dspw_desc* dnet = &descs[0];
  for (int p = 0; p < nprob; p++)
    if (descs[p].recon == DSPW_REC_SP_WENO_DL) { dnet = &descs[p]; break; }
  NetParams np = make_net(*dnet);
  int ret = DSPW_OK;
#define CKC(x)                                   \
  do {                                           \
    if ((x) != cudaSuccess) {                    \
      ret = DSPW_ERR_NOMEM;                      \
      goto fail;                                 \
    }                                            \
  } while (0)
  {
    size_t state_bytes = (size_t)h->elem * (size_t)std::max<long long>(h->ctot, 1) * 5;
    CKC(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CKC(h->precision == DSPW_FP64 ? Launch<double>::prepare() : Launch<float>::prepare());
    CKC(cudaMalloc(&h->dprob, sizeof(ProbDev) * nprob));
    CKC(cudaMalloc(&h->dst, sizeof(ProbState) * nprob));
    CKC(cudaMalloc(&h->dstatus, sizeof(StatusDev)));
    CKC(cudaMalloc(&h->dnet, sizeof(NetParams)));
    CKC(cudaMalloc(&h->dcell_start, sizeof(long long) * (nprob + 1)));
    CKC(cudaMalloc(&h->dnactive, sizeof(int)));
    for (SweepClass& c : h->classes) {
      const size_t n = c.probs.size();
      for (int dir = 0; dir < 3; dir++) CKC(cudaMalloc(&c.dtask[dir], sizeof(int) * (n + 1)));
      if (h->classes.size() > 1) CKC(cudaMalloc(&c.dpmap, sizeof(int) * n));
    }
    CKC(cudaMalloc(&h->Un, state_bytes));
    CKC(cudaMalloc(&h->Ua, state_bytes));
    CKC(cudaMalloc(&h->Ub, state_bytes));
    CKC(cudaMalloc(&h->R, state_bytes));
    if (h->time_scheme == DSPW_RK4) CKC(cudaMalloc(&h->R2, state_bytes));
    if (h->has_ns) {
      CKC(cudaMalloc(&h->V, state_bytes));
      CKC(cudaMalloc(&h->node, state_bytes * 3));
    }
    CKC(cudaMalloc(&h->dstage, sizeof(double) * 5 * (size_t)std::max<long long>(h->maxcells, 1)));
    CKC(cudaMalloc(&h->dscratch, sizeof(double) * 16));
    CKC(cudaMalloc(&h->dred, sizeof(double) * 8 * (size_t)reduce_rows_max()));
    CKC(cudaMemcpy(h->dprob, h->hprob.data(), sizeof(ProbDev) * nprob, cudaMemcpyHostToDevice));
    CKC(cudaMemset(h->dst, 0, sizeof(ProbState) * nprob));
    CKC(cudaMemset(h->dstatus, 0, sizeof(StatusDev)));
    CKC(cudaMemcpy(h->dnet, &np, sizeof(NetParams), cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(h->dcell_start, h->cell_start.data(), sizeof(long long) * (nprob + 1), cudaMemcpyHostToDevice));
    for (SweepClass& c : h->classes) {
      const size_t n = c.probs.size();
      for (int dir = 0; dir < 3; dir++)
        CKC(cudaMemcpy(c.dtask[dir], c.task_start[dir].data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
      if (c.dpmap) CKC(cudaMemcpy(c.dpmap, c.probs.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    }
    CKC(cudaMemset(h->Un, 0, state_bytes));
    CKC(cudaMemset(h->Ua, 0, state_bytes));
    CKC(cudaMemset(h->Ub, 0, state_bytes));
    CKC(cudaMemset(h->R, 0, state_bytes));
    // problems start finished until their state is uploaded
    std::vector<ProbState> hs(nprob);
    memset(hs.data(), 0, sizeof(ProbState) * nprob);
    for (int p = 0; p < nprob; p++) {
      hs[p].time = h->hprob[p].final_time;
      hs[p].iter = h->hprob[p].max_iter;
    }
    CKC(cudaMemcpy(h->dst, hs.data(), sizeof(ProbState) * nprob, cudaMemcpyHostToDevice));
  }
  build_tma_maps(h);
  *out = h;
  return DSPW_OK;
fail:
  dspw_destroy(h);
  return ret;
#undef CKC
}

int dspw_destroy(dspw_handle* h) {
  if (!h) return DSPW_ERR_ARG;
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  if (h->comm) nccl().comm_destroy(h->comm);
  void* ptrs[] = {h->dprob, h->dst, h->dstatus, h->dnet, h->dcell_start, h->dnactive,
                  h->Un, h->Ua, h->Ub, h->R, h->R2, h->V, h->node, h->dstage, h->dscratch, h->dred,
                  h->ddiag, h->ddiag_part, h->drows, h->dnode_start, h->dsnap, h->dsnap_count, h->dsnap_meta};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (SweepClass& c : h->classes) {
    for (int dir = 0; dir < 3; dir++)
      if (c.dtask[dir]) cudaFree(c.dtask[dir]);
    if (c.dpmap) cudaFree(c.dpmap);
    if (c.dtmap) cudaFree(c.dtmap);
  }
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return DSPW_OK;
}

int dspw_upload_prim(dspw_handle* h, int p, const double* prim) {
  if (check_p(h, p) || !prim) return DSPW_ERR_ARG;
  const dspw_desc& d = h->desc[p];
  long long n = ncells(d);
  int nv = d.model <= DSPW_BURGERS ? 1 : 5;
  CK(cudaMemcpyAsync(h->dstage, prim, sizeof(double) * nv * n, cudaMemcpyHostToDevice, h->stream));
  // positivity (enflo/src/fv.cc:88-89 asserts it) and finiteness, checked on
  // the staged copy before the state is touched
  unsigned long long* bad = (unsigned long long*)h->dscratch;
  unsigned long long hb[2] = {0, 0};
  CK(cudaMemsetAsync(bad, 0, sizeof(hb), h->stream));
  CK(launch_check_prim(h->dstage, n, nv, bad, h->stream));
  CK(cudaMemcpyAsync(hb, bad, sizeof(hb), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (hb[0]) return DSPW_ERR_NONPOSITIVE;
  if (hb[1]) return DSPW_ERR_NONFINITE;
  ProbState s;
  memset(&s, 0, sizeof(s));
  s.time = 0.0;
  s.iter = 0;
  s.t_save = h->hprob[p].t_interval;
  s.active = 1;
  CK(cudaMemcpyAsync(h->dst + p, &s, sizeof(s), cudaMemcpyHostToDevice, h->stream));
  if (h->precision == DSPW_FP64)
    CK(Launch<double>::upload(h->dprob, h->dst, p, h->dstage, (double*)h->Un, h->ctot, n, h->stream));
  else
    CK(Launch<float>::upload(h->dprob, h->dst, p, h->dstage, (float*)h->Un, h->ctot, n, h->stream));
  k_init_entropy<<<1, 1, 0, h->stream>>>(h->dprob, h->dst, p);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  return DSPW_OK;
}

int dspw_entropy_check(dspw_handle* h, int p, double* max_rise, long long* steps) {
  if (check_p(h, p) || !max_rise) return DSPW_ERR_ARG;
  ProbState s;
  CK(cudaMemcpyAsync(&s, h->dst + p, sizeof(s), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  *max_rise = s.ent_max_rise;
  if (steps) *steps = s.ent_steps;
  return DSPW_OK;
}

static int download(dspw_handle* h, int p, double* out, int prim, void* src) {
  if (check_p(h, p) || !out) return DSPW_ERR_ARG;
  const dspw_desc& d = h->desc[p];
  long long n = ncells(d);
  int nv = d.model <= DSPW_BURGERS ? 1 : 5;
  if (h->precision == DSPW_FP64)
    CK(Launch<double>::download(h->dprob, p, (const double*)src, h->ctot, n, h->dstage, prim, h->stream));
  else
    CK(Launch<float>::download(h->dprob, p, (const float*)src, h->ctot, n, h->dstage, prim, h->stream));
  CK(cudaMemcpyAsync(out, h->dstage, sizeof(double) * nv * n, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return DSPW_OK;
}

int dspw_download_prim(dspw_handle* h, int p, double* prim) { return download(h, p, prim, 1, h ? h->Un : nullptr); }
int dspw_download_cons(dspw_handle* h, int p, double* cons) { return download(h, p, cons, 0, h ? h->Un : nullptr); }

int dspw_compute_dt(dspw_handle* h, int p, double* dt) {
  if (check_p(h, p) || !dt) return DSPW_ERR_ARG;
  long long n = ncells(h->desc[p]);
  CK(cudaMemsetAsync(h->dscratch, 0, sizeof(double), h->stream));
  if (h->precision == DSPW_FP64)
    CK(Launch<double>::speed(h->dprob, h->dst, p, (const double*)h->Un, h->ctot, n, h->dscratch, h->stream));
  else
    CK(Launch<float>::speed(h->dprob, h->dst, p, (const float*)h->Un, h->ctot, n, h->dscratch, h->stream));
  double smax = 0;
  CK(cudaMemcpyAsync(&smax, h->dscratch, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const ProbDev& P = h->hprob[p];
  double v = 1.0e20;   // enflo/src/fv.cc:366-383
  double c = P.hmin / smax;
  if (c < v) v = c;
  *dt = v * P.cfl;
  return DSPW_OK;
}

int dspw_residual(dspw_handle* h, int p, double* res) {
  if (check_p(h, p) || !res) return DSPW_ERR_ARG;
  int r = enqueue_stage_any(h, 0, 1);
  if (r) return r;
  return download(h, p, res, 0, h->R);
}

// first health error the device recorded since the last dspw_last_status
// (DSPW_ERR_NONFINITE / DSPW_ERR_NONPOSITIVE), DSPW_OK if none; the counters
// are left for dspw_last_status
static int device_health(dspw_handle* h) {
  int code = 0;
  CK(cudaMemcpyAsync(&code, &h->dstatus->code, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return code;
}

int dspw_stage(dspw_handle* h, int rk, double dt) {
  if (!h || rk < 0 || rk >= h->nrk) return DSPW_ERR_ARG;
  if (rk == 0) {
    CK(cudaMemsetAsync(h->dnactive, 0, sizeof(int), h->stream));
    if (dt <= 0) {
      int rs = enqueue_speed_reduce(h);
      if (rs) return rs;
    }
    CK(launch_begin_step(h->dprob, h->dst, h->nprob, dt, h->dnactive, h->stream));
  }
  int r = enqueue_stage_any(h, rk, 0);
  if (r) return r;
  if (rk == h->nrk - 1) {
    r = enqueue_end_step(h);
    if (r) return r;
  }
  return device_health(h);
}

int dspw_step(dspw_handle* h, int nsteps, double fixed_dt) {
  if (!h || nsteps < 0) return DSPW_ERR_ARG;
  int r = build_graph(h, fixed_dt > 0 ? fixed_dt : 0.0);
  if (r) return r;
  for (int s = 0; s < nsteps; s++) {
    CK(cudaGraphLaunch(h->graph, h->stream));
    // keep the diagnostics and snapshot rings from wrapping
    if (h->diag_cap > 0 && (s + 1) % h->diag_cap == 0) { r = drain_diag(h); if (r) return r; }
    if (h->snap_slots > 0 && (s + 1) % h->snap_slots == 0) { r = drain_snap(h); if (r) return r; }
  }
  CK(cudaStreamSynchronize(h->stream));
  r = drain_diag(h);
  if (r) return r;
  r = drain_snap(h);
  if (r) return r;
  return device_health(h);
}

int dspw_run(dspw_handle* h, int chunk, int* steps) {
  if (!h || chunk < 1) return DSPW_ERR_ARG;
  int r = build_graph(h, 0.0);
  if (r) return r;
  // bounded by the largest max_iter of the batch; a health error ends the run
  long long limit = 0;
  for (auto& d : h->desc) limit = std::max<long long>(limit, d.max_iter);
  long long total = 0;
  int status = DSPW_OK;
  for (;;) {
    for (int s = 0; s < chunk; s++) {
      CK(cudaGraphLaunch(h->graph, h->stream));
      if (h->diag_cap > 0 && (s + 1) % h->diag_cap == 0) { r = drain_diag(h); if (r) return r; }
      if (h->snap_slots > 0 && (s + 1) % h->snap_slots == 0) { r = drain_snap(h); if (r) return r; }
    }
    r = drain_diag(h);
    if (r) return r;
    r = drain_snap(h);
    if (r) return r;
    total += chunk;
    int nact = 0;
    StatusDev sd;
    CK(cudaMemcpyAsync(&nact, h->dnactive, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(&sd, h->dstatus, sizeof(sd), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (sd.code) { status = sd.code; break; }
    if (nact == 0 || total > limit) break;
  }
  // exact count of steps of the longest problem
  std::vector<ProbState> hs(h->nprob);
  CK(cudaMemcpy(hs.data(), h->dst, sizeof(ProbState) * h->nprob, cudaMemcpyDeviceToHost));
  int mx = 0;
  for (auto& s : hs) mx = std::max(mx, s.iter);
  if (steps) *steps = mx;
  return status;
}

int dspw_globals(dspw_handle* h, int p, dspw_globals_out* g) {
  if (check_p(h, p) || !g) return DSPW_ERR_ARG;
  long long n = ncells(h->desc[p]);
  if (h->precision == DSPW_FP64)
    CK(Launch<double>::globals(h->dprob, p, (const double*)h->Un, h->ctot, n, h->dred, h->dscratch, h->stream));
  else
    CK(Launch<float>::globals(h->dprob, p, (const float*)h->Un, h->ctot, n, h->dred, h->dscratch, h->stream));
  double acc[8];
  ProbState s;
  CK(cudaMemcpyAsync(acc, h->dscratch, sizeof(double) * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(&s, h->dst + p, sizeof(s), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const ProbDev& P = h->hprob[p];
  g->time = s.time;
  g->dt = s.dt;
  g->iter = s.iter;
  g->finished = !(s.time < P.final_time && s.iter < P.max_iter);
  g->total_entropy = acc[0] * P.vol;
  g->kinetic_energy = acc[1] * P.vol;
  for (int v = 0; v < 5; v++) g->conserved[v] = acc[2 + v] * P.vol;
  return DSPW_OK;
}

int dspw_diag_enable(dspw_handle* h, int capacity) {
  if (!h || capacity < 0) return DSPW_ERR_ARG;
  if (h->has_halo && capacity > 0) return DSPW_ERR_UNSUPPORTED;   // node sums need the whole domain
  CK(cudaStreamSynchronize(h->stream));
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }   // the step graph changes
  if (h->ddiag) cudaFree(h->ddiag);
  if (h->ddiag_part) cudaFree(h->ddiag_part);
  if (h->drows) cudaFree(h->drows);
  if (h->dnode_start) cudaFree(h->dnode_start);
  h->ddiag = nullptr; h->ddiag_part = nullptr; h->drows = nullptr; h->dnode_start = nullptr;
  h->diag_cap = 0;
  h->nodes_tot = 0;
  h->diag_taken.assign(h->nprob, 0);
  h->diag_dropped.assign(h->nprob, 0);
  h->diag_host.assign(h->nprob, std::vector<double>());
  if (capacity == 0) return DSPW_OK;
  // node prefix: (Nx+1)(Ny+1)(Nz+1) nodes per system, none for scalar problems
  std::vector<long long> ns(h->nprob + 1, 0);
  for (int p = 0; p < h->nprob; p++) {
    const ProbDev& P = h->hprob[p];
    ns[p + 1] = ns[p] + (P.is_scalar ? 0 : (long long)(P.nx + 1) * (P.ny + 1) * (P.nz + 1));
  }
  const size_t ring = sizeof(double) * DIAG_COLS * (size_t)h->nprob * (size_t)capacity;
  // partial rows: (blocks + problems) of the largest diagnostics launch
  const size_t part = sizeof(double) * DIAG_NACC * (size_t)(device_sms() * 8LL + h->nprob);
  if (cudaMalloc(&h->ddiag, sizeof(DiagAcc) * h->nprob) != cudaSuccess ||
      cudaMalloc(&h->ddiag_part, part) != cudaSuccess ||
      cudaMalloc(&h->drows, ring) != cudaSuccess ||
      cudaMalloc(&h->dnode_start, sizeof(long long) * (h->nprob + 1)) != cudaSuccess) {
    if (h->ddiag) cudaFree(h->ddiag);
    if (h->ddiag_part) cudaFree(h->ddiag_part);
    if (h->drows) cudaFree(h->drows);
    if (h->dnode_start) cudaFree(h->dnode_start);
    h->ddiag = nullptr; h->ddiag_part = nullptr; h->drows = nullptr; h->dnode_start = nullptr;
    h->last_error = DSPW_ERR_CUDA;
    return DSPW_ERR_CUDA;
  }
  CK(cudaMemset(h->ddiag, 0, sizeof(DiagAcc) * h->nprob));
  CK(cudaMemset(h->drows, 0, ring));
  CK(cudaMemcpy(h->dnode_start, ns.data(), sizeof(long long) * (h->nprob + 1), cudaMemcpyHostToDevice));
  h->nodes_tot = ns[h->nprob];
  h->diag_cap = capacity;
  return DSPW_OK;
}

int dspw_diag_pending(dspw_handle* h, int p, int* nrows, long long* ndropped) {
  if (check_p(h, p) || !nrows) return DSPW_ERR_ARG;
  int r = drain_diag(h);
  if (r) return r;
  *nrows = h->diag_cap ? (int)(h->diag_host[p].size() / DIAG_COLS) : 0;
  if (ndropped) *ndropped = h->diag_cap ? h->diag_dropped[p] : 0;
  return DSPW_OK;
}

int dspw_diag_read(dspw_handle* h, int p, double* rows, int max_rows, int* nread) {
  if (check_p(h, p) || !nread || max_rows < 0 || (max_rows > 0 && !rows)) return DSPW_ERR_ARG;
  int r = drain_diag(h);
  if (r) return r;
  *nread = 0;
  if (h->diag_cap == 0) return DSPW_OK;
  std::vector<double>& q = h->diag_host[p];
  const int n = std::min<int>(max_rows, (int)(q.size() / DIAG_COLS));
  memcpy(rows, q.data(), sizeof(double) * DIAG_COLS * n);
  q.erase(q.begin(), q.begin() + (size_t)n * DIAG_COLS);
  *nread = n;
  return DSPW_OK;
}

int dspw_snap_enable(dspw_handle* h, int slots) {
  if (!h || slots < 0) return DSPW_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }   // the step graph changes
  if (h->dsnap) cudaFree(h->dsnap);
  if (h->dsnap_count) cudaFree(h->dsnap_count);
  if (h->dsnap_meta) cudaFree(h->dsnap_meta);
  h->dsnap = nullptr; h->dsnap_count = nullptr; h->dsnap_meta = nullptr;
  h->snap_slots = 0;
  h->snap_taken.assign(h->nprob, 0);
  h->snap_dropped.assign(h->nprob, 0);
  h->snap_host.assign(h->nprob, std::deque<dspw_handle::HostSnap>());
  if (slots == 0) return DSPW_OK;
  const size_t bytes = (size_t)h->elem * 5 * (size_t)h->ctot * (size_t)slots;
  if (cudaMalloc(&h->dsnap, bytes) != cudaSuccess ||
      cudaMalloc(&h->dsnap_count, sizeof(unsigned long long) * h->nprob) != cudaSuccess ||
      cudaMalloc(&h->dsnap_meta, sizeof(SnapMeta) * (size_t)h->nprob * slots) != cudaSuccess) {
    if (h->dsnap) cudaFree(h->dsnap);
    if (h->dsnap_count) cudaFree(h->dsnap_count);
    if (h->dsnap_meta) cudaFree(h->dsnap_meta);
    h->dsnap = nullptr; h->dsnap_count = nullptr; h->dsnap_meta = nullptr;
    h->last_error = DSPW_ERR_CUDA;
    return DSPW_ERR_CUDA;
  }
  CK(cudaMemset(h->dsnap_count, 0, sizeof(unsigned long long) * h->nprob));
  CK(cudaMemset(h->dsnap_meta, 0, sizeof(SnapMeta) * (size_t)h->nprob * slots));
  h->snap_slots = slots;
  return DSPW_OK;
}

int dspw_snap_pending(dspw_handle* h, int p, int* n, long long* ndropped) {
  if (check_p(h, p) || !n) return DSPW_ERR_ARG;
  int r = drain_snap(h);
  if (r) return r;
  *n = h->snap_slots ? (int)h->snap_host[p].size() : 0;
  if (ndropped) *ndropped = h->snap_slots ? h->snap_dropped[p] : 0;
  return DSPW_OK;
}

int dspw_snap_read(dspw_handle* h, int p, double* prim, double* time, int* iter) {
  if (check_p(h, p) || !prim) return DSPW_ERR_ARG;
  int r = drain_snap(h);
  if (r) return r;
  if (h->snap_slots == 0 || h->snap_host[p].empty()) return DSPW_ERR_ARG;
  dspw_handle::HostSnap& s = h->snap_host[p].front();
  memcpy(prim, s.prim.data(), sizeof(double) * s.prim.size());
  if (time) *time = s.time;
  if (iter) *iter = s.iter;
  h->snap_host[p].pop_front();
  return DSPW_OK;
}

int dspw_last_status(dspw_handle* h, dspw_status_out* s) {
  if (!h || !s) return DSPW_ERR_ARG;
  StatusDev d;
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaMemcpy(&d, h->dstatus, sizeof(d), cudaMemcpyDeviceToHost));
  CK(cudaMemset(h->dstatus, 0, sizeof(d)));
  s->code = d.code ? d.code : h->last_error;
  s->nonfinite_cells = (long long)d.nonfinite;
  s->nonpositive_cells = (long long)d.nonpositive;
  s->sign_violations = (long long)d.sign_viol;
  s->faces_checked = 0;
  s->limiter_acts = 0;
  for (int k = 0; k < EPI_SLOTS; k++) {
    s->faces_checked += (long long)d.faces_checked[k];
    s->limiter_acts += (long long)d.limiter_acts[k];
  }
  h->last_error = 0;
  return DSPW_OK;
}

int dspw_errors(dspw_handle* h, int p, int comp, const double* exact, double err[3]) {
  if (check_p(h, p) || !exact || !err || comp < 0 || comp > 4) return DSPW_ERR_ARG;
  long long n = ncells(h->desc[p]);
  CK(cudaMemcpyAsync(h->dstage, exact, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
  if (h->precision == DSPW_FP64)
    CK(Launch<double>::errors(h->dprob, p, (const double*)h->Un, h->ctot, n, comp, h->dstage, h->dred, h->dscratch,
                              h->stream));
  else
    CK(Launch<float>::errors(h->dprob, p, (const float*)h->Un, h->ctot, n, comp, h->dstage, h->dred, h->dscratch,
                             h->stream));
  double acc[3];
  CK(cudaMemcpyAsync(acc, h->dscratch, sizeof(double) * 3, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const ProbDev& P = h->hprob[p];
  err[0] = acc[0] * (P.dx * P.dy * P.dz);   // enflo_scalar/src_scalar/compute_errors.cc:26-29
  err[1] = std::sqrt(acc[1] * (P.dx * P.dy * P.dz));
  err[2] = acc[2];
  return DSPW_OK;
}

int dspw_tune(dspw_handle* h, int reps, double* before_ms, double* after_ms) {
  if (!h || reps < 1 || reps > 1000) return DSPW_ERR_ARG;
  return h->precision == DSPW_FP64 ? tune_grids<double>(h, reps, before_ms, after_ms)
                                   : tune_grids<float>(h, reps, before_ms, after_ms);
}

int dspw_profile_step(dspw_handle* h, double* kernel_ms, char* names, int max_k, int* nk) {
  if (!h || !kernel_ms || max_k < 1) return DSPW_ERR_ARG;
  std::vector<cudaEvent_t> ev;
  std::vector<std::string> nm;
  cudaEvent_t e0;
  CK(cudaEventCreate(&e0));
  CK(cudaEventRecord(e0, h->stream));
  h->prof_ev = &ev;
  h->prof_names = &nm;
  int r = enqueue_step(h, 0.0);
  h->prof_ev = nullptr;
  h->prof_names = nullptr;
  CK(cudaStreamSynchronize(h->stream));
  int n = 0;
  cudaEvent_t prev = e0;
  for (size_t i = 0; i < ev.size(); i++) {
    float ms = 0;
    cudaEventElapsedTime(&ms, prev, ev[i]);
    if (n < max_k) {
      kernel_ms[n] = ms;
      if (names) {
        memset(names + 16 * n, 0, 16);
        strncpy(names + 16 * n, nm[i].c_str(), 15);
      }
      n++;
    }
    prev = ev[i];
  }
  for (auto e : ev) cudaEventDestroy(e);
  cudaEventDestroy(e0);
  if (nk) *nk = n;
  return r;
}

int dspw_reconstruct_batch(const dspw_desc* d, const double* u4, long long n, double* recl, double* recr,
                           long long* limiter_acts) {
  if (!d || !u4 || !recl || !recr || n < 0) return DSPW_ERR_ARG;
  if (d->recon < DSPW_REC_SP_WENO || d->recon > DSPW_REC_ENO2) return DSPW_ERR_UNSUPPORTED;
  if (d->precision != DSPW_FP64 && d->precision != DSPW_FP32_BF16) return DSPW_ERR_ARG;
  if (n == 0) return DSPW_OK;
  ProbDev P = make_prob(*d, 0);
  NetParams np = make_net(*d);
  ProbDev* dp = nullptr;
  NetParams* dn = nullptr;
  double *du = nullptr, *dl = nullptr, *dr = nullptr;
  unsigned long long* dacts = nullptr;
  unsigned long long acts = 0;
  int ret = DSPW_OK;
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return DSPW_ERR_CUDA;
  if (cudaMalloc(&dp, sizeof(P)) != cudaSuccess || cudaMalloc(&dn, sizeof(np)) != cudaSuccess ||
      cudaMalloc(&du, sizeof(double) * 4 * n) != cudaSuccess || cudaMalloc(&dl, sizeof(double) * n) != cudaSuccess ||
      cudaMalloc(&dr, sizeof(double) * n) != cudaSuccess || cudaMalloc(&dacts, sizeof(acts)) != cudaSuccess) {
    ret = DSPW_ERR_NOMEM;
  } else {
    cudaError_t e = cudaMemcpyAsync(dp, &P, sizeof(P), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dn, &np, sizeof(np), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(du, u4, sizeof(double) * 4 * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(dacts, 0, sizeof(acts), s);
    if (e == cudaSuccess)
      e = d->precision == DSPW_FP64 ? Launch<double>::recon_batch(dp, dn, du, n, dl, dr, dacts, s)
                                    : Launch<float>::recon_batch(dp, dn, du, n, dl, dr, dacts, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(recl, dl, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(recr, dr, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&acts, dacts, sizeof(acts), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) ret = DSPW_ERR_CUDA;
  }
  if (limiter_acts) *limiter_acts = (long long)acts;
  cudaFree(dp); cudaFree(dn); cudaFree(du); cudaFree(dl); cudaFree(dr); cudaFree(dacts);
  cudaStreamDestroy(s);
  return ret;
}

int dspw_sync(dspw_handle* h) {
  if (!h) return DSPW_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  return h->last_error;
}

void* dspw_stream(dspw_handle* h) { return h ? (void*)h->stream : nullptr; }

int dspw_nccl_id(unsigned char id[128]) {
  if (!id) return DSPW_ERR_ARG;
  if (!nccl().ok) return DSPW_ERR_UNSUPPORTED;
  ncclUniqueId u;
  if (nccl().get_unique_id(&u) != ncclSuccess) return DSPW_ERR_CUDA;
  static_assert(sizeof(u) == 128, "ncclUniqueId is 128 bytes");
  memcpy(id, &u, sizeof(u));
  return DSPW_OK;
}

int dspw_slab_connect(dspw_handle* h, const unsigned char id[128], int rank, int nranks) {
  if (!h || !id || nranks < 1 || rank < 0 || rank >= nranks || h->nprob != 1 || h->comm) return DSPW_ERR_ARG;
  if (!nccl().ok) return DSPW_ERR_UNSUPPORTED;
  const dspw_desc& d = h->desc[0];
  const int D = problem_dim(d) - 1;
  const bool lo_halo = d.bc[2 * D] == DSPW_BC_HALO, hi_halo = d.bc[2 * D + 1] == DSPW_BC_HALO;
  // a periodic domain wraps its first and last slab around; an inner slab
  // has halo faces on both sides
  if ((rank > 0 && !lo_halo) || (rank + 1 < nranks && !hi_halo)) return DSPW_ERR_ARG;
  ncclUniqueId u;
  memcpy(&u, id, sizeof(u));
  CK(cudaStreamSynchronize(h->stream));
  ncclComm_t c = nullptr;
  if (nccl().comm_init_rank(&c, nranks, u, rank) != ncclSuccess) return DSPW_ERR_CUDA;
  h->comm = c;
  h->rank = rank;
  h->nranks = nranks;
  h->down = lo_halo ? (rank > 0 ? rank - 1 : nranks - 1) : -1;
  h->up = hi_halo ? (rank + 1 < nranks ? rank + 1 : 0) : -1;
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }   // the step graph changes
  return DSPW_OK;
}

int dspw_halo_view(dspw_handle* h, int p, int rk, dspw_halo_out* out) {
  if (check_p(h, p) || !out || rk < 0 || rk >= h->nrk) return DSPW_ERR_ARG;
  const dspw_desc& d = h->desc[p];
  const int ng = halo_layers(d);
  if (!ng) return DSPW_ERR_ARG;
  const ProbDev& P = h->hprob[p];
  const long long lc = layer_cells(d);
  const int D = P.dim - 1;
  const long long N = D == 0 ? P.nx : (D == 1 ? P.ny : P.nz);
  char* base = (char*)buf(h, stage_input(h, rk)) + h->elem * P.off;
  out->recv_lo = base - h->elem * ng * lc;
  out->recv_hi = base + h->elem * N * lc;
  out->send_lo = base;
  out->send_hi = base + h->elem * (N - ng) * lc;
  out->count = ng * lc;
  out->comp_stride = h->ctot;
  out->ncomp = P.nv;
  out->elem_bytes = (int)h->elem;
  out->ng = ng;
  out->layer_cells = (int)lc;
  return DSPW_OK;
}

int dspw_device_state(dspw_handle* h, int p, void** ptr, long long* stride, int* elem_bytes) {
  if (check_p(h, p) || !ptr) return DSPW_ERR_ARG;
  *ptr = (char*)h->Un + h->elem * h->hprob[p].off;
  if (stride) *stride = h->ctot;
  if (elem_bytes) *elem_bytes = (int)h->elem;
  return DSPW_OK;
}

}  // extern "C"

// dspw_kernels.cuh -- device data structures and the stage kernels.
//
// Work decomposition.  A stage is one sweep kernel per active direction.  The
// unit of work is a warp task: one line segment of SEG_CELLS cells along the
// sweep direction of one problem.  A warp stages the SEG_CELLS + 4 cells it
// needs (2 ghost/halo cells per side) in shared memory, converts them to
// primitive and entropy variables once, evaluates the SEG_CELLS + 1 faces (one
// lane per face, the wide 4th-order two-point fluxes shared between
// neighbouring faces), and then either accumulates the residual of its cells
// (non-final sweep) or applies the SSPRK stage update (final sweep).  Warps of
// a block are independent (only __syncwarp), so problems of any size and mix
// share one launch: the global task index is mapped to (problem, line,
// segment) through per-problem prefix sums.
//
// Cell data in HBM: structure-of-arrays planes U[c * ctot + cell], cells of
// problem p at [off_p, off_p + nx*ny*nz) with x fastest.  Euler problems store
// dim+2 components (rho, rho u[, rho v[, rho w]], E): the momentum components
// of inactive directions are identically zero in the reference and are not
// stored.
#pragma once
#include <cstddef>
#include "dspw_math.cuh"
#include "../../include/dspw.h"

namespace dspw {

constexpr int SEG_CELLS = 30;               // cells per warp task
constexpr int SEG_FACES = SEG_CELLS + 1;    // faces per warp task (lanes 0..30)
constexpr int SEG_LOAD = SEG_CELLS + 4;     // staged cells per warp task
constexpr int WARPS_PER_BLOCK = 8;
#ifndef DSPW_MINB_F64
#define DSPW_MINB_F64 2
#endif
#ifndef DSPW_MINB_F32
#define DSPW_MINB_F32 3
#endif
// resident blocks per SM requested from the register allocator
template <typename T> struct MinBlocks { static constexpr int value = sizeof(T) == 8 ? DSPW_MINB_F64 : DSPW_MINB_F32; };

struct ProbDev {
  int model, flux, recon, dim, nv, nrk;
  int nx, ny, nz;
  int bc[6];
  int ec1, mu_model, max_iter, is_scalar;
  int central;        // 0 kepec, 1 kep, 2 roe_ec, 3 keps, 4 roe (two-point flux; TeCNO central part)
  int fourth;         // 1: 4th-order central combination
  int tecno;          // 1: entropy-stable dissipation added
  int rusanov;        // 1: Rusanov Lambda, 0: Roe Lambda
  int spw_corr;       // SP-WENO correction type, -1 for the network
  long long off;      // first cell
  double dx, dy, dz, hmin, vol;
  double node_vol;    // (xmax-xmin)/(Nx+1) * (ymax-ymin)/(Ny+1) * (zmax-zmin)/(Nz+1) (compute_global.cc:59-61)
  double area[3], rarea[3];
  double gamma, gas_const, prandtl, mu_ref, T_ref, T_0, omega, Cp;
  double lin_vel[3], lin_speed, lin_vn[3];
  double cfl, final_time, t_interval;
  double bc_state[6][5];
};

// Compile-time specialisation of the sweep kernels.  The generic kernel reads
// the flux structure and the reconstruction from ProbDev at run time and holds
// the code of every model, dimension and flux.  A batch whose problems are all
// Euler / Navier-Stokes of one dimension with the 4th-order KEPEC central part
// and TeCNO dissipation (kepes_tecno4_roe, kepes_tecno4_rusanov) and one
// reconstruction family runs a kernel with those choices fixed (Roe / Rusanov,
// EC1_fix and the SP-WENO correction stay run-time flags).
struct SpecGeneric {
  static constexpr bool fixed = false;
  static constexpr int dim = 0;
  static constexpr int rec = 0;
};
template <int DIM_, int REC_>   // REC_: 1 SP-WENO family, 2 DSP-WENO network
struct SpecHot {
  static constexpr bool fixed = true;
  static constexpr int dim = DIM_;
  static constexpr int rec = REC_;
};
// host-side code of a specialisation: 0 generic, else 10 * dim + rec
constexpr int spec_code(int dim, int rec) { return 10 * dim + rec; }
// 1-D scalar problems (linear advection, Burgers) with the reconstruction
// family rec fixed: k_sweep_scalar
constexpr int scalar_spec_code(int rec) { return 100 + rec; }
// resident blocks per SM of k_sweep_scalar: 64 registers per thread for FP32,
// 128 for FP64 (the FP64 network forward spills at 64)
template <typename T> struct ScalarMinBlocks { static constexpr int value = sizeof(T) == 8 ? 2 : 4; };

// The per-step reductions of a problem (wave-speed max, entropy sum) go to
// EPI_SLOTS slots picked by block index, so that the one atomic per warp of
// the sweeps does not queue on a single address; the step kernels combine them.
constexpr int EPI_SLOTS = 16;

struct ProbState {
  double time, dt, t_save, factor;
  unsigned long long smax[EPI_SLOTS];   // bits of the max wave speed of the newest state
  // discrete entropy inequality: total entropy of the newest state, the sum
  // of the step being built, the largest relative one-step rise, steps checked
  double ent, ent_max_rise;
  double ent_acc[EPI_SLOTS];
  long long ent_steps;
  int iter, active;
  int snap;                  // 1: this step ended on an output time stamp
  int pad;
};

struct StatusDev {
  int code;
  int pad;
  unsigned long long nonfinite, nonpositive, sign_viol;
  // incremented by nearly every warp of every sweep: slots by block index
  unsigned long long faces_checked[EPI_SLOTS], limiter_acts[EPI_SLOTS];
};

template <typename T>
struct SweepArgs {
  const ProbDev* prob;
  ProbState* st;
  const int* task_start;   // nprob + 1 prefix of tasks in this direction
  const int* pmap;         // problem index of each entry of task_start (null: identity)
  int nprob, ntask;
  const T* Uin;            // U^(k), stage input
  const T* Un;             // U^n
  T* Uout;                 // U^(k+1)
  T* R;                    // residual accumulator (non-final sweeps)
  long long ctot;
  int rk;
  int scheme;              // enum dspw_time
  double a_rk, b_rk;       // SSPRK3 / RK1 stage coefficients
  T* R2;                   // classic RK4: weighted sum of the stage residuals
  int final_stage;         // 1: this stage produces U^(n+1)
  int residual_only;       // 1: write R in every sweep, never update
  int store_R;             // 1: the updating sweep also stores the stage residual (diagnostics)
  int viscous;             // 1: the NS viscous kernel performs the update
  StatusDev* status;
  const NetParams* net;
  // optional collection of (stencil, reconstruction) pairs for training:
  // every collect_stride-th reconstruction appends 6 floats (u0..u3, l, r)
  float* collect_buf;
  unsigned long long* collect_count;
  unsigned long long collect_cap;
  unsigned collect_stride;
  // TMA staging of the specialised y / z sweeps (tma = 1): tensor maps of the
  // class's problems in global memory, TMA_SLOTS per problem and direction
  // (tma_map_index), and the slot of the state this stage reads
  const void* tmaps;
  int tma;
  int tma_in;              // 0: U^n, 1: Ua, 2: Ub
  int narrow;              // 1: the specialised y / z sweep runs k_sweep_narrow (4-column tiles)
};

// Tensor maps of the TMA staging, per (class problem, direction 1 / 2):
// slots 0-2 the stage input U^n / Ua / Ub with a box of SEG_LOAD rows, slot 3
// the residual and slot 4 U^n with a box of SEG_CELLS rows.  A map is 128 bytes.
constexpr int TMA_SLOTS = 5;
constexpr int TMA_MAP_BYTES = 128;
__host__ __device__ constexpr inline int tma_map_index(int p, int dir, int slot) { return (p * 2 + (dir - 1)) * TMA_SLOTS + slot; }

// append one training pair (sampled by a hash of the reconstruction's position)
template <typename T>
__device__ inline void collect_pair(const SweepArgs<T>& A, unsigned key, T s0, T s1, T s2, T s3, T l, T r) {
  if (!A.collect_buf) return;
  unsigned h = key * 2654435761u;
  h ^= h >> 15;
  if (h % A.collect_stride) return;
  unsigned long long i = atomicAdd(A.collect_count, 1ull);
  if (i >= A.collect_cap) return;
  float* o = A.collect_buf + 6 * i;
  o[0] = (float)s0; o[1] = (float)s1; o[2] = (float)s2; o[3] = (float)s3; o[4] = (float)l; o[5] = (float)r;
}

// ----------------------------------------------------------- small helpers --

template <typename T> struct Vec5 { T v[5]; };

DSPW_HD unsigned long long speed_bits(double s) { return (unsigned long long)__double_as_longlong(s); }

template <typename T>
DSPW_HD void load_cons(const T* U, long long ctot, long long cell, int nv, int dim, T u[5]) {
  u[0] = U[cell];
  u[1] = U[ctot + cell];
  if (nv == 5) {
    u[2] = U[2 * ctot + cell];
    u[3] = U[3 * ctot + cell];
    u[4] = U[4 * ctot + cell];
  } else if (nv == 4) {
    u[2] = U[2 * ctot + cell];
    u[3] = T(0);
    u[4] = U[3 * ctot + cell];
  } else {
    u[2] = T(0);
    u[3] = T(0);
    u[4] = U[2 * ctot + cell];
  }
  (void)dim;
}

template <typename T>
DSPW_HD void store_cons(T* U, long long ctot, long long cell, int nv, const T u[5]) {
  U[cell] = u[0];
  U[ctot + cell] = u[1];
  if (nv == 5) {
    U[2 * ctot + cell] = u[2];
    U[3 * ctot + cell] = u[3];
    U[4 * ctot + cell] = u[4];
  } else if (nv == 4) {
    U[2 * ctot + cell] = u[2];
    U[3 * ctot + cell] = u[4];
  } else {
    U[2 * ctot + cell] = u[4];
  }
}

// con_to_prim, enflo/src/fv.cc:388-400
template <typename T>
DSPW_HD void cons_to_prim(const T u[5], T gamma, T p[5]) {
  typedef Mth<T> m;
  p[0] = u[0];
  T r = m::rcp(u[0]);
  p[1] = u[1] * r;
  p[2] = u[2] * r;
  p[3] = u[3] * r;
  T msq = u[1] * u[1] + u[2] * u[2] + u[3] * u[3];
  p[4] = (gamma - T(1.0)) * (u[4] - m::div(T(0.5) * msq, u[0]));
}

// prim_to_con, enflo/src/fv.cc:405-416
template <typename T>
DSPW_HD void prim_to_cons(const T p[5], T gamma, T u[5]) {
  typedef Mth<T> m;
  u[0] = p[0];
  u[1] = p[1] * p[0];
  u[2] = p[2] * p[0];
  u[3] = p[3] * p[0];
  T vsq = p[1] * p[1] + p[2] * p[2] + p[3] * p[3];
  u[4] = T(0.5) * p[0] * vsq + m::div(p[4], gamma - T(1.0));
}

// entropy variables, enflo/src/fv.cc:427-433 with Entropy :557-560
template <typename T>
DSPW_HD void prim_to_ent(const T p[5], T gamma, T v[5]) {
  typedef Mth<T> m;
  T beta = m::div(p[0], T(2) * p[4]);
  T s = m::log(p[4]) - gamma * m::log(p[0]);
  T vsq = p[1] * p[1] + p[2] * p[2] + p[3] * p[3];
  v[0] = m::div(gamma - s, gamma - T(1)) - vsq * beta;
  v[1] = p[1] * (T(2) * beta);
  v[2] = p[2] * (T(2) * beta);
  v[3] = p[3] * (T(2) * beta);
  v[4] = T(-2) * beta;
}

// Viscosity, enflo/src/parameter.cc:646-663
DSPW_HD double viscosity(const ProbDev& P, double T) {
  if (P.mu_model == DSPW_MU_SUTHERLAND) return P.mu_ref * ::pow(T / P.T_ref, 1.5) * (P.T_ref + P.T_0) / (T + P.T_0);
  if (P.mu_model == DSPW_MU_POWER) return P.mu_ref * ::pow(T / P.T_ref, P.omega);
  return P.mu_ref;
}

// wave speed of compute_dt, enflo/src/fv.cc:366-383 (+ viscous term for NS)
template <typename T>
DSPW_HD double wave_speed(const ProbDev& P, const T p[5]) {
  if (P.model == DSPW_LINADV) return P.lin_speed;
  if (P.model == DSPW_BURGERS) return (double)Mth<T>::abs(p[0]);
  if constexpr (sizeof(T) == 4) {
    // FP32 state: its speed in FP32 (the FP64 square roots cost 4 % of the
    // FP32 step); the viscous term stays in FP64
    if (P.model == DSPW_EULER) {
      const float s = sqrtf(p[1] * p[1] + p[2] * p[2] + p[3] * p[3]) + sqrtf((float)P.gamma * p[4] / p[0]);
      return (double)s;
    }
  }
  double rho = (double)p[0], pr = (double)p[4];
  double u = p[1], v = p[2], w = p[3];
  double s = ::sqrt(u * u + v * v + w * w) + ::sqrt(P.gamma * pr / rho);
  if (P.model == DSPW_NS_ES || P.model == DSPW_NS_KEP)
    s += viscosity(P, pr / (P.gas_const * rho)) / rho / P.hmin;
  return s;
}

DSPW_HD unsigned warp_max_u64_lane0(unsigned long long& v) {
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return 0;
}

DSPW_HD double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// global task -> problem (binary search in the prefix sums)
DSPW_HD int find_problem(const int* start, int nprob, int task) {
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(start + mid) <= task) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <int DIR>
DSPW_HD int dir_len(const ProbDev& P) { return DIR == 0 ? P.nx : (DIR == 1 ? P.ny : P.nz); }

// (line index, segment) of a local task.  DIR 0: seg fastest, then j, then k
// (consecutive warps extend the same x line).  DIR 1/2: x fastest so the warps
// of a block read adjacent x columns.
template <int DIR>
DSPW_HD void decode_task(const ProbDev& P, int lt, int& i0, int& j0, int& k0, int& c0, int& ncell) {
  int N = dir_len<DIR>(P);
  int nseg = (N + SEG_CELLS - 1) / SEG_CELLS;
  int seg;
  if (DIR == 0) {
    seg = lt % nseg; lt /= nseg;
    j0 = lt % P.ny; k0 = lt / P.ny; i0 = 0;
  } else if (DIR == 1) {
    i0 = lt % P.nx; lt /= P.nx;
    seg = lt % nseg; k0 = lt / nseg; j0 = 0;
  } else {
    i0 = lt % P.nx; lt /= P.nx;
    seg = lt % nseg; j0 = lt / nseg; k0 = 0;
  }
  c0 = seg * SEG_CELLS;
  ncell = min(SEG_CELLS, N - c0);
}

// (column group, segment) of a local group task of the specialised y / z
// sweeps: groups of COLS adjacent x columns (8, or 4 for the narrow tiles; the
// last of a row may be partial, ncols < COLS), then segments, then the
// remaining direction.
template <int DIR, int COLS = WARPS_PER_BLOCK>
DSPW_HD void decode_group(const ProbDev& P, int lg, int& i0, int& j0, int& k0, int& c0, int& ncell, int& ncols) {
  const int N = dir_len<DIR>(P);
  const int nseg = (N + SEG_CELLS - 1) / SEG_CELLS;
  const int ngx = (P.nx + COLS - 1) / COLS;
  const int ig = lg % ngx;
  lg /= ngx;
  const int seg = lg % nseg, o = lg / nseg;
  i0 = ig * COLS;
  ncols = min(COLS, P.nx - i0);
  if (DIR == 1) { k0 = o; j0 = 0; } else { j0 = o; k0 = 0; }
  c0 = seg * SEG_CELLS;
  ncell = min(SEG_CELLS, N - c0);
}

template <int DIR>
DSPW_HD long long cell_index(const ProbDev& P, int i0, int j0, int k0, int c) {
  if (DIR == 0) return P.off + ((long long)k0 * P.ny + j0) * P.nx + c;
  if (DIR == 1) return P.off + ((long long)k0 * P.ny + c) * P.nx + i0;
  return P.off + ((long long)c * P.ny + j0) * P.nx + i0;
}

// Ghost handling of apply_bc (enflo/src/fv.cc:121-361): source cell along the
// line for a (possibly ghost) index c, and the boundary kind used.  A halo
// face (slab decomposition) reads its stored ghost layers in place.
DSPW_HD int ghost_source(int c, int N, int kind, int& flip) {
  flip = 0;
  if (c >= 0 && c < N) return c;
  if (kind == DSPW_BC_HALO) return c;   // the stored halo layer beside the interior
  if (kind == DSPW_BC_PERIODIC) return ((c % N) + N) % N;
  if (kind == DSPW_BC_WALL) { flip = 1; return c < 0 ? -1 - c : 2 * N - 1 - c; }
  return c < 0 ? 0 : N - 1;   // neumann (and dirichlet, which ignores it)
}

// Sign property of the reconstruction (the trainer's sign_property,
// DSP-WENO_trainer/DSP-WENO_network_trainer.py:110-116): the reconstructed jump
// zr - zl has the sign of the cell jump z2 - z1 or is zero.  "Zero" allows the
// rounding of the arithmetic type (the trainer uses 1e-14 for FP64 data of
// order one): 8 ulps of the largest value involved.
template <typename T>
DSPW_HD bool sign_violation(T z0, T z1, T z2, T z3, T zl, T zr) {
  T rj = zr - zl, cj = z2 - z1;
  if (!(rj * cj < T(0))) return false;
  typedef Mth<T> m;
  T sc = m::max(m::max(m::max(m::abs(zl), m::abs(zr)), m::max(m::abs(z1), m::abs(z2))),
                m::max(m::abs(z0), m::abs(z3)));
  const T eps = sizeof(T) == 8 ? T(2.220446049250313e-16) : T(1.1920929e-07);
  return m::abs(rj) > T(64) * eps * sc;
}

// ------------------------------------------------------ warp shared memory --

// staging of the network inputs / outputs of one warp (FP32 form only)
// per-warp scratch of the tensor-core network (FP32 form): the staged inputs,
// the logits, and each lane's B fragments and biases (loaded once per kernel)
template <typename T> struct NetScratch { float feat[32][8]; float logit[32][8]; uint32_t frag[32][12]; };
template <> struct NetScratch<double> { float feat[1][8]; float logit[1][8]; uint32_t frag[1][12]; };

// P and V hold the staged cells of a warp task: SEG_LOAD of them (two ghost
// cells per side), two more for the three-cell halo of point-wise ENO of
// level 3, which the generic kernel stages one slot further right (eno_shift).
template <typename T>
struct WarpSmem {
  T P[5][SEG_LOAD + 2];
  T V[5][SEG_LOAD + 2];
  T W[5][32];      // wide two-point fluxes, centre g = c0 - 1 + idx
  T F[5][32];      // face fluxes, face f = c0 + idx
  NetScratch<T> ns;
  // padding to a length of 12 words mod 32 (FP32: 1580 words, FP64: 1420):
  // the cooperative block's accesses to 8 warps' scratch at one index (4 rows
  // x 8 columns per warp instruction) then hit 32 different banks
  T pad[sizeof(T) == 4 ? 4 : 16];
};
// mlp_warp_tiles addresses the scratch by these byte offsets, with 16-byte
// vector accesses to the rows of every warp's scratch
static_assert(offsetof(NetScratch<float>, logit) == 1024 && offsetof(NetScratch<float>, frag) == 2048,
              "NetScratch<float> layout");
static_assert(offsetof(WarpSmem<float>, ns) % 16 == 0 && sizeof(WarpSmem<float>) % 16 == 0,
              "WarpSmem<float> alignment");
static_assert((sizeof(WarpSmem<float>) / 4) % 32 == 12, "WarpSmem<float> bank spread");

// ---------------------------------------------------- two-point fluxes ------

// face-average state shared by kepec and the TeCNO dissipation
// (enflo/src/kepec.cc:18-30, kepes_tecno4_roe.cc:34-48)
template <typename T>
struct FaceAvg {
  T rho, beta, p, betal, betar, vel[3], vn;
};

template <typename T, int DIR>
DSPW_HD void face_avg(const T* Pl, const T* Pr, T Rg, FaceAvg<T>& f) {
  typedef Mth<T> m;
  T rhol = Pl[0], rhor = Pr[0];
  f.rho = logavg<T>(rhol, rhor);
  T templ = m::div(Pl[4], Rg * rhol);
  T tempr = m::div(Pr[4], Rg * rhor);
  f.betal = m::div(T(0.5), Rg * templ);
  f.betar = m::div(T(0.5), Rg * tempr);
  f.beta = logavg<T>(f.betal, f.betar);
  f.p = m::div(T(0.5) * (rhol + rhor), f.betal + f.betar);
  f.vel[0] = Pl[1] * T(0.5) + Pr[1] * T(0.5);
  f.vel[1] = Pl[2] * T(0.5) + Pr[2] * T(0.5);
  f.vel[2] = Pl[3] * T(0.5) + Pr[3] * T(0.5);
  // vel * unit_normal with n = e_DIR: the other products are +-0
  f.vn = f.vel[0] * T(DIR == 0) + f.vel[1] * T(DIR == 1) + f.vel[2] * T(DIR == 2);
}

// kepec_flux from a face average, enflo/src/kepec.cc:30-48
template <typename T, int DIR>
DSPW_HD void kepec_from_avg(const FaceAvg<T>& f, const T* Pl, const T* Pr, T gamma, T area, T F[5]) {
  typedef Mth<T> m;
  T vel2 = T(0.5) * ((Pl[1] * Pl[1] + Pl[2] * Pl[2] + Pl[3] * Pl[3]) + (Pr[1] * Pr[1] + Pr[2] * Pr[2] + Pr[3] * Pr[3]));
  F[0] = f.rho * f.vn;
  F[1] = T(DIR == 0) * f.p + f.vel[0] * F[0];
  F[2] = T(DIR == 1) * f.p + f.vel[1] * F[0];
  F[3] = T(DIR == 2) * f.p + f.vel[2] * F[0];
  F[4] = T(0.5) * (m::div(T(1.0), (gamma - T(1.0)) * f.beta) - vel2) * F[0] +
         (F[1] * f.vel[0] + F[2] * f.vel[1] + F[3] * f.vel[2]);
#pragma unroll
  for (int c = 0; c < 5; c++) F[c] *= area;
}

template <typename T, int DIR>
DSPW_HD void kepec_pair(const T* Pl, const T* Pr, T gamma, T Rg, T area, T F[5]) {
  FaceAvg<T> f;
  face_avg<T, DIR>(Pl, Pr, Rg, f);
  kepec_from_avg<T, DIR>(f, Pl, Pr, gamma, area, F);
}

// kep_flux, enflo/src/kep.cc:10-44 (Enthalpy enflo/src/fv.cc:565-569)
template <typename T, int DIR>
DSPW_HD void kep_pair(const T* Pl, const T* Pr, T gamma, T area, T F[5]) {
  typedef Mth<T> m;
  T rho = T(0.5) * (Pl[0] + Pr[0]);
  T p = T(0.5) * (Pl[4] + Pr[4]);
  T vel[3] = {Pl[1] * T(0.5) + Pr[1] * T(0.5), Pl[2] * T(0.5) + Pr[2] * T(0.5), Pl[3] * T(0.5) + Pr[3] * T(0.5)};
  T al = m::sqrt(m::div(gamma * Pl[4], Pl[0]));
  T ar = m::sqrt(m::div(gamma * Pr[4], Pr[0]));
  T Hl = m::div(al * al, gamma - T(1.0)) + T(0.5) * (Pl[1] * Pl[1] + Pl[2] * Pl[2] + Pl[3] * Pl[3]);
  T Hr = m::div(ar * ar, gamma - T(1.0)) + T(0.5) * (Pr[1] * Pr[1] + Pr[2] * Pr[2] + Pr[3] * Pr[3]);
  T H = T(0.5) * (Hl + Hr);
  T vn = vel[0] * T(DIR == 0) + vel[1] * T(DIR == 1) + vel[2] * T(DIR == 2);
  F[0] = rho * vn;
  F[1] = T(DIR == 0) * p + vel[0] * F[0];
  F[2] = T(DIR == 1) * p + vel[1] * F[0];
  F[3] = T(DIR == 2) * p + vel[2] * F[0];
  F[4] = rho * H * vn;
#pragma unroll
  for (int c = 0; c < 5; c++) F[c] *= area;
}

// roe_ec_flux, enflo/src/roe_ec.cc:10-69
template <typename T, int DIR>
DSPW_HD void roe_ec_pair(const T* Pl, const T* Pr, T gamma, T area, T F[5]) {
  typedef Mth<T> m;
  T rhol = Pl[0], rhor = Pr[0], pl = Pl[4], pr = Pr[4];
  T bl = m::sqrt(m::div(rhol, pl));
  T br = m::sqrt(m::div(rhor, pr));
  T z1b = T(0.5) * (bl + br);
  T zvb[3] = {Pl[1] * (T(0.5) * bl) + Pr[1] * (T(0.5) * br), Pl[2] * (T(0.5) * bl) + Pr[2] * (T(0.5) * br),
              Pl[3] * (T(0.5) * bl) + Pr[3] * (T(0.5) * br)};
  T z5b = T(0.5) * (bl * pl + br * pr);
  T zn = zvb[0] * T(DIR == 0) + zvb[1] * T(DIR == 1) + zvb[2] * T(DIR == 2);
  T z1l = logavg<T>(bl, br);
  T z5l = logavg<T>(bl * pl, br * pr);
  F[0] = z5l * zn;
  T c1 = m::div(z5b, z1b), c2 = m::div(F[0], z1b);
  F[1] = T(DIR == 0) * c1 + zvb[0] * c2;
  F[2] = T(DIR == 1) * c1 + zvb[1] * c2;
  F[3] = T(DIR == 2) * c1 + zvb[2] * c2;
  F[4] = m::div(T(0.5) * (m::div(m::div(gamma + T(1.0), gamma - T(1.0)) * F[0], z1l) +
                          (F[1] * zvb[0] + F[2] * zvb[1] + F[3] * zvb[2])), z1b);
#pragma unroll
  for (int c = 0; c < 5; c++) F[c] *= area;
}

// keps_flux, enflo/src/keps.cc:10-48 (arithmetic means of rho and beta)
template <typename T, int DIR>
DSPW_HD void keps_pair(const T* Pl, const T* Pr, T gamma, T Rg, T area, T F[5]) {
  typedef Mth<T> m;
  T rhol = Pl[0], rhor = Pr[0];
  T rho = T(0.5) * (rhol + rhor);
  T templ = m::div(Pl[4], Rg * rhol);
  T tempr = m::div(Pr[4], Rg * rhor);
  T vel2 = T(0.5) * ((Pl[1] * Pl[1] + Pl[2] * Pl[2] + Pl[3] * Pl[3]) + (Pr[1] * Pr[1] + Pr[2] * Pr[2] + Pr[3] * Pr[3]));
  T betal = m::div(T(0.5), Rg * templ);
  T betar = m::div(T(0.5), Rg * tempr);
  T beta = T(0.5) * (betal + betar);
  T p = m::div(T(0.5) * rho, beta);
  T vel[3] = {Pl[1] * T(0.5) + Pr[1] * T(0.5), Pl[2] * T(0.5) + Pr[2] * T(0.5), Pl[3] * T(0.5) + Pr[3] * T(0.5)};
  T vn = vel[0] * T(DIR == 0) + vel[1] * T(DIR == 1) + vel[2] * T(DIR == 2);
  F[0] = rho * vn;
  F[1] = T(DIR == 0) * p + vel[0] * F[0];
  F[2] = T(DIR == 1) * p + vel[1] * F[0];
  F[3] = T(DIR == 2) * p + vel[2] * F[0];
  F[4] = T(0.5) * (m::div(T(1.0), (gamma - T(1.0)) * beta) - vel2) * F[0] +
         (F[1] * vel[0] + F[2] * vel[1] + F[3] * vel[2]);
#pragma unroll
  for (int c = 0; c < 5; c++) F[c] *= area;
}

// roe_flux (Roe's flux without entropy fix), enflo/src/roe.cc:10-86
template <typename T, int DIR>
DSPW_HD void roe_pair(const T* Pl, const T* Pr, T gamma, T area, T F[5]) {
  typedef Mth<T> m;
  const T n[3] = {T(DIR == 0), T(DIR == 1), T(DIR == 2)};
  T rhol = Pl[0], rhor = Pr[0], pl = Pl[4], pr = Pr[4];
  T hl = m::div(m::div(gamma * pl, rhol), gamma - T(1.0)) + T(0.5) * (Pl[1] * Pl[1] + Pl[2] * Pl[2] + Pl[3] * Pl[3]);
  T hr = m::div(m::div(gamma * pr, rhor), gamma - T(1.0)) + T(0.5) * (Pr[1] * Pr[1] + Pr[2] * Pr[2] + Pr[3] * Pr[3]);
  T rls = m::sqrt(rhol), rrs = m::sqrt(rhor);
  T fl = m::div(rls, rls + rrs);
  T fr = T(1.0) - fl;
  T rho = rls * rrs;
  T vel[3] = {Pl[1] * fl + Pr[1] * fr, Pl[2] * fl + Pr[2] * fr, Pl[3] * fl + Pr[3] * fr};
  T h = hl * fl + hr * fr;
  T vn = vel[0] * n[0] + vel[1] * n[1] + vel[2] * n[2];
  T a = m::sqrt((gamma - T(1.0)) * (h - T(0.5) * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2])));
  T dp = pr - pl;
  T vln = Pl[1] * n[0] + Pl[2] * n[1] + Pl[3] * n[2];
  T vrn = Pr[1] * n[0] + Pr[2] * n[1] + Pr[3] * n[2];
  T dV = vrn - vln;
  if (vn >= T(0.0)) {
    T lambda = vn - a;
    T coeff = m::div(T(0.5) * (dp - rho * a * dV), a * a);
    T factor = ((T(0.0) < lambda) ? T(0.0) : lambda) * coeff;   // std::min(lambda, 0.0)
    F[0] = rhol * vln;
#pragma unroll
    for (int c = 0; c < 3; c++) F[1 + c] = n[c] * pl + Pl[1 + c] * (rhol * vln);
    F[4] = hl * F[0];
    F[0] += factor;
#pragma unroll
    for (int c = 0; c < 3; c++) F[1 + c] += vel[c] * factor + n[c] * (-a * factor);
    F[4] += (h - a * vn) * factor;
  } else {
    T lambda = vn + a;
    T coeff = m::div(T(0.5) * (dp + rho * a * dV), a * a);
    T factor = ((lambda < T(0.0)) ? T(0.0) : lambda) * coeff;   // std::max(lambda, 0.0)
    F[0] = rhor * vrn;
#pragma unroll
    for (int c = 0; c < 3; c++) F[1 + c] = n[c] * pr + Pr[1 + c] * (rhor * vrn);
    F[4] = hr * F[0];
    F[0] -= factor;
#pragma unroll
    for (int c = 0; c < 3; c++) F[1 + c] += vel[c] * (-factor) + n[c] * (-a * factor);
    F[4] -= (h + a * vn) * factor;
  }
#pragma unroll
  for (int c = 0; c < 5; c++) F[c] *= area;
}

// two-point flux of kind 0 kepec, 1 kep, 2 roe_ec, 3 keps, 4 roe
template <typename T, int DIR>
DSPW_HD void central_pair(int kind, const T* Pl, const T* Pr, T gamma, T Rg, T area, T F[5]) {
  if (kind == 0) kepec_pair<T, DIR>(Pl, Pr, gamma, Rg, area, F);
  else if (kind == 1) kep_pair<T, DIR>(Pl, Pr, gamma, area, F);
  else if (kind == 2) roe_ec_pair<T, DIR>(Pl, Pr, gamma, area, F);
  else if (kind == 3) keps_pair<T, DIR>(Pl, Pr, gamma, Rg, area, F);
  else roe_pair<T, DIR>(Pl, Pr, gamma, area, F);
}

// ------------------------------------------------- BF16 tensor-core network --

// One warp evaluates the 5-5-5-5-5 network for 32 instances (one per lane) as
// two m16n8k8 BF16 MMA tiles per layer, FP32 accumulation; layer outputs stay
// in registers (the C fragment of one layer is the A fragment of the next).
struct NetFrag {
  uint32_t b[4];       // B fragment per layer: W^T (k = input, n = output)
  float bias0[4], bias1[4];   // bias of output columns n = 2*(lane%4), +1
};

DSPW_HD uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&h);
}

__device__ inline void net_frag_load(const NetParams& P, int lane, NetFrag& nf) {
  int n = lane >> 2, k0 = (lane & 3) * 2;
#pragma unroll
  for (int l = 0; l < 4; l++) {
    float w0 = (n < 5 && k0 < 5) ? P.wf[l][n][k0] : 0.f;
    float w1 = (n < 5 && k0 + 1 < 5) ? P.wf[l][n][k0 + 1] : 0.f;
    nf.b[l] = pack_bf16(w0, w1);
    nf.bias0[l] = (k0 < 5) ? P.bf[l][k0] : 0.f;
    nf.bias1[l] = (k0 + 1 < 5) ? P.bf[l][k0 + 1] : 0.f;
  }
}

// each lane stores its fragments into its warp's scratch (once per kernel)
template <typename T>
__device__ inline void net_frag_stage(const NetParams& P, int lane, NetScratch<T>& ns) {
  if constexpr (sizeof(T) == 4) {
    NetFrag nf;
    net_frag_load(P, lane, nf);
#pragma unroll
    for (int l = 0; l < 4; l++) {
      ns.frag[lane][l] = nf.b[l];
      ns.frag[lane][4 + l] = __float_as_uint(nf.bias0[l]);
      ns.frag[lane][8 + l] = __float_as_uint(nf.bias1[l]);
    }
    __syncwarp();
  }
}

// The four layers of one 16-row tile as one PTX block: A fragments loaded from
// the staged inputs (rows r and r + 8, columns kq and kq + 1) and rounded to
// BF16, m16n8k8 BF16 MMA with the layer's FP32 biases as the C operand, ReLU
// fused into the BF16 repacking of the result as the next layer's A fragment
// (cvt.rn.relu: max(x, 0) then round), and the logits stored back to shared
// memory.
__device__ inline void mlp_tile_bf16(const NetFrag& nf, unsigned in_lo, unsigned in_hi, unsigned out_lo,
                                     unsigned out_hi) {
  asm volatile(
      "{\n\t"
      ".reg .f32 %%x<4>, %%c<4>;\n\t"
      ".reg .b32 %%a<2>;\n\t"
      "ld.shared.v2.f32 {%%x0, %%x1}, [%0];\n\t"
      "ld.shared.v2.f32 {%%x2, %%x3}, [%1];\n\t"
      "cvt.rn.bf16x2.f32 %%a0, %%x1, %%x0;\n\t"
      "cvt.rn.bf16x2.f32 %%a1, %%x3, %%x2;\n\t"
      "mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%%c0,%%c1,%%c2,%%c3}, {%%a0,%%a1}, {%4}, "
      "{%8,%9,%8,%9};\n\t"
      "cvt.rn.relu.bf16x2.f32 %%a0, %%c1, %%c0;\n\t"
      "cvt.rn.relu.bf16x2.f32 %%a1, %%c3, %%c2;\n\t"
      "mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%%c0,%%c1,%%c2,%%c3}, {%%a0,%%a1}, {%5}, "
      "{%10,%11,%10,%11};\n\t"
      "cvt.rn.relu.bf16x2.f32 %%a0, %%c1, %%c0;\n\t"
      "cvt.rn.relu.bf16x2.f32 %%a1, %%c3, %%c2;\n\t"
      "mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%%c0,%%c1,%%c2,%%c3}, {%%a0,%%a1}, {%6}, "
      "{%12,%13,%12,%13};\n\t"
      "cvt.rn.relu.bf16x2.f32 %%a0, %%c1, %%c0;\n\t"
      "cvt.rn.relu.bf16x2.f32 %%a1, %%c3, %%c2;\n\t"
      "mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%%c0,%%c1,%%c2,%%c3}, {%%a0,%%a1}, {%7}, "
      "{%14,%15,%14,%15};\n\t"
      "st.shared.v2.f32 [%2], {%%c0, %%c1};\n\t"
      "st.shared.v2.f32 [%3], {%%c2, %%c3};\n\t"
      "}\n"
      :
      : "r"(in_lo), "r"(in_hi), "r"(out_lo), "r"(out_hi), "r"(nf.b[0]), "r"(nf.b[1]), "r"(nf.b[2]), "r"(nf.b[3]),
        "f"(nf.bias0[0]), "f"(nf.bias1[0]), "f"(nf.bias0[1]), "f"(nf.bias1[1]), "f"(nf.bias0[2]), "f"(nf.bias1[2]),
        "f"(nf.bias0[3]), "f"(nf.bias1[3])
      : "memory");
}

// The warp-wide part of one network evaluation: both tiles, between two warp
// barriers.  mma.sync.aligned requires every lane of the warp to execute the
// same instruction.  Inlined into lane-divergent code, the compiler may emit
// several copies of the MMA sequence and send different lanes through
// different copies, which yields wrong logits; as a separate function there
// is exactly one copy that every lane calls.  ns_addr is the shared-memory
// address of the warp's NetScratch.
static __device__ __noinline__ void mlp_warp_tiles(unsigned ns_addr) {
  __syncwarp();
  unsigned lane;
  asm("mov.u32 %0, %%laneid;" : "=r"(lane));
  NetFrag nf;
  const unsigned fa = ns_addr + 2048u + lane * 48u;   // frag[lane][0..11]
  asm volatile("ld.shared.v4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(nf.b[0]), "=r"(nf.b[1]), "=r"(nf.b[2]), "=r"(nf.b[3]) : "r"(fa));
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(nf.bias0[0]), "=f"(nf.bias0[1]), "=f"(nf.bias0[2]), "=f"(nf.bias0[3]) : "r"(fa + 16u));
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(nf.bias1[0]), "=f"(nf.bias1[1]), "=f"(nf.bias1[2]), "=f"(nf.bias1[3]) : "r"(fa + 32u));
  // rows 16 t + r and 16 t + r + 8 share the half swap of rows with bit 2 set
  // (warp_mlp_bf16): (16 t + r) >> 2 & 1 = r >> 2 & 1 = lane >> 4 & 1
  const unsigned r = lane >> 2, kq = ((lane & 3) * 2) ^ (((lane >> 4) & 1u) << 2);
#pragma unroll
  for (unsigned t = 0; t < 2; t++) {
    const unsigned lo = ((16 * t + r) * 8 + kq) * 4, hi = ((16 * t + r + 8) * 8 + kq) * 4;
    mlp_tile_bf16(nf, ns_addr + lo, ns_addr + hi, ns_addr + 1024u + lo, ns_addr + 1024u + hi);
  }
  __syncwarp();
}

// in: this lane's 5 inputs; out: this lane's 5 logits.  Every lane of the
// warp must call it.  A row of 8 floats holds columns 0-3 and 4-7 in its two
// 16-byte halves, swapped in rows with bit 2 set: the 16-byte accesses of 8
// consecutive lanes (rows 32 bytes apart) then fall into 32 different banks.
__device__ inline void warp_mlp_bf16(NetScratch<float>& ns, const float in[5], float out[5], int lane) {
  const int h = (lane >> 2) & 1;
  float4* f = reinterpret_cast<float4*>(&ns.feat[lane][0]);
  f[h] = make_float4(in[0], in[1], in[2], in[3]);
  f[h ^ 1] = make_float4(in[4], 0.f, 0.f, 0.f);
  mlp_warp_tiles((unsigned)__cvta_generic_to_shared(&ns));
  const float4* o = reinterpret_cast<const float4*>(&ns.logit[lane][0]);
  const float4 lo = o[h], hi = o[h ^ 1];
  out[0] = lo.x; out[1] = lo.y; out[2] = lo.z; out[3] = lo.w;
  out[4] = hi.x;
}

// DSP-WENO reconstruction of one stencil per lane, warp-cooperative network.
// Every lane of the warp must call it (the MMA is warp-wide); `valid` masks
// lanes whose result is unused.  Returns 1 if the sign-preserving limiter had
// to act (FP32 form).
template <typename T>
__device__ inline int dsp_weno_warp(const NetParams& NP, WarpSmem<T>* sm, int lane, bool valid,
                                    T u0, T u1, T u2, T u3, T& l, T& r, unsigned long long& signv);

template <>
__device__ inline int dsp_weno_warp<double>(const NetParams& NP, WarpSmem<double>*, int, bool valid,
                                            double u0, double u1, double u2, double u3, double& l, double& r,
                                            unsigned long long&) {
  if (valid) dsp_weno_fp64(NP, u0, u1, u2, u3, l, r);
  return 0;
}

template <>
__device__ inline int dsp_weno_warp<float>(const NetParams& NP, WarpSmem<float>* sm, int lane,
                                           bool valid, float u0, float u1, float u2, float u3, float& l, float& r,
                                           unsigned long long& signv) {
  // The reference skips the network when |u2 - u1| < 1e-15 (reconstruct.cc:152);
  // in FP32 the equivalent "no jump" test is a jump of a few ulps of the values,
  // below which the scaled differences of the features are rounding noise.
  float mag = fmaxf(fabsf(u1), fabsf(u2));
  bool guard = fabsf(u2 - u1) < fmaxf(1e-15f, 4.0f * 1.1920929e-07f * mag);
  // the inputs before the network call, the vertices after it: the code in
  // front of the warp-wide MMA is free of lane-dependent branches, and the ten
  // vertices are not held across the call
  float feat[5], tm, tp, md;
  nn_inputs<float>(u0, u1, u2, u3, feat, tm, tp, md);
  bool inbox = true;
  if (NP.use_box) {
#pragma unroll
    for (int k = 0; k < 5; k++) inbox = inbox && feat[k] >= NP.feat_lo[k] && feat[k] <= NP.feat_hi[k];
  }
  // Every lane's features go through the tiles, whatever they hold: each
  // instance is one row of the A operand, so a NaN or infinity of one lane (a
  // guard lane, an invalid lane, degenerate features) reaches only that lane's
  // logits and never another's.
  float lg[5];
  warp_mlp_bf16(sm->ns, feat, lg, lane);
  if (!valid) return 0;
  if (guard) { l = 0.f; r = 0.f; return 0; }
  if (inbox) {
    float vx[5], vy[5];
    nn_vertices<float>(tm, tp, md, vx, vy);
    nn_finish<float>(lg, vx, vy, u0, u1, u2, u3, l, r);
    // non-finite features or vertices (the only way to a non-finite
    // reconstruction of a finite stencil) fall back to SP-WENO below; so does
    // an overflow of l + r of huge finite values, which SP-WENO also handles
    if (isfinite(l + r)) {
      // sign-preserving limiter: the reconstructed jump must not oppose the
      // cell jump; an opposing jump is replaced by zero, so the property holds
      // exactly.
      const float dj = u2 - u1, rj = r - l;
      if (dj * rj < 0.f) {
        const float c = 0.5f * (l + r);
        l = c; r = c;
        return 1;
      }
      return 0;
    }
  }
  // degenerate features or outside the training range: plain SP-WENO
  sp_weno<float>(u0, u1, u2, u3, 0, l, r);
  if (sign_violation<float>(u0, u1, u2, u3, l, r)) signv++;   // not limited: checked here
  return 0;
}

// The FP32 network path ends in a sign-preserving limiter that tests the same
// two jumps (dsp_weno_warp<float>), so there the property holds by
// construction and the caller does not re-check it; the path's SP-WENO
// fallback faces, which are not limited, are checked inside it.  SP-WENO, the
// lower-order reconstructions and the FP64 (unlimited) network are checked by
// the caller.
template <typename T, typename Sp>
__device__ __forceinline__ bool sign_checked(const ProbDev& P) {
  if constexpr (sizeof(T) == 4) {
    if constexpr (Sp::fixed) return Sp::rec != 2;
    else return !(P.recon < DSPW_REC_FIRST && P.spw_corr < 0);
  }
  return true;
}

// Staging shift of the six-cell stencils of point-wise ENO of level 3 (generic
// kernel only; the specialised kernels never see it, and fold it to 0).
template <typename Sp>
__device__ inline int eno_shift(const ProbDev& P) {
  return (!Sp::fixed && P.recon == DSPW_REC_ENO3) ? 1 : 0;
}

template <typename T, typename Sp>
__device__ inline void reconstruct_lane(const ProbDev& P, const NetParams& NP, WarpSmem<T>* sm,
                                        int lane, bool valid, T s0, T s1, T s2, T s3, T& l, T& r, int& viol,
                                        unsigned long long& signv) {
  if (!Sp::fixed && P.recon >= DSPW_REC_FIRST) {
    if (valid) simple_recon<T>(P.recon, s0, s1, s2, s3, l, r);
  } else if (Sp::fixed ? Sp::rec == 1 : P.spw_corr >= 0) {
    if (valid) sp_weno<T>(s0, s1, s2, s3, P.spw_corr, l, r);
  } else {
    viol += dsp_weno_warp<T>(NP, sm, lane, valid, s0, s1, s2, s3, l, r, signv);
  }
}

// ------------------------------------------------------------ Euler sweep --

// TeCNO dissipation -0.5 R Lambda [[Z]] for one face (enflo/src/kepes_tecno4_roe.cc:59-171
// and the Roe / Rusanov variants), R = eigenvectors scaled by S^(1/2), Z = R^T V
// of the 4 stencil cells, component-wise reconstruction.  Columns of R are
// built one at a time; Diff[i] accumulates over j in the reference's order.
template <typename T, int DIR, int DIM, typename Sp>
__device__ inline void tecno_dissipation(const SweepArgs<T>& A, const ProbDev& P, const NetParams& NP,
                                         WarpSmem<T>* sm, int lane, bool valid, int q0,
                                         const FaceAvg<T>& fa, T flux[5], int& viol, unsigned long long& signv,
                                         unsigned collect_salt) {
  typedef Mth<T> m;
  const T G = T(P.gamma);
  const T n0 = T(DIR == 0), n1 = T(DIR == 1), n2 = T(DIR == 2);
  const T* vel = fa.vel;
  const int qb = eno_shift<Sp>(P);
  const int cq = q0 + qb;   // first of the four cells around the face
  T a = m::sqrt(m::div(T(0.5) * G, fa.beta));
  T vsq = vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2];
  T H = m::div(a * a, G - T(1.0)) + T(0.5) * vsq;
  T v1 = vel[0] * n1 - vel[1] * n0;
  T v2 = vel[2] * n0 - vel[0] * n2;
  T const1 = m::sqrt(m::div(fa.rho, G));
  T psqrt = m::sqrt(fa.p);
  const T sh = m::sqrt(T(0.5));
  T S[5] = {sh * const1, m::sqrt(G - T(1.0)) * const1, psqrt, psqrt, sh * const1};
  T Lam[5];
  if (!P.rusanov) {
    T l2 = m::abs(fa.vn);
    T ma = T(0.0);
    T L0 = m::abs(fa.vn - a), L4 = m::abs(fa.vn + a);
    if (P.ec1) {
      // LambdaL[0]-LambdaR[0] and LambdaL[3]-LambdaR[3] (kepes_tecno4_roe.cc:92-113)
      T vnl = sm->P[1 + DIR][cq + 1], vnr = sm->P[1 + DIR][cq + 2];
      T al = m::sqrt(m::div(T(0.5) * G, fa.betal));
      T ar = m::sqrt(m::div(T(0.5) * G, fa.betar));
      ma = T(1.0 / 6.0);
      L0 = L0 + ma * m::abs((vnl - al) - (vnr - ar));
      L4 = L4 + ma * m::abs(vnl - vnr);
    }
    Lam[0] = L0; Lam[1] = l2; Lam[2] = l2; Lam[3] = l2; Lam[4] = L4;
  } else {
    T lr = m::abs(fa.vn) + m::abs(a);
    Lam[0] = Lam[1] = Lam[2] = Lam[3] = Lam[4] = lr;
  }
  T Diff[5] = {T(0), T(0), T(0), T(0), T(0)};
  auto component = [&](int j) {
    // components that are identically zero in lower dimensions (exact skip)
    if (DIM == 1 && (j == 2 || j == 3)) return;
    if (DIM == 2 && j == 3) return;
    // column j of R (kepes_tecno4_roe.cc:66-72), scaled by S[j]
    T col[5];
    if (j == 0) { col[0] = T(1); col[1] = vel[0] - a * n0; col[2] = vel[1] - a * n1; col[3] = vel[2] - a * n2; col[4] = H - a * fa.vn; }
    else if (j == 1) { col[0] = T(1); col[1] = vel[0]; col[2] = vel[1]; col[3] = vel[2]; col[4] = T(0.5) * vsq; }
    else if (j == 2) { col[0] = T(0); col[1] = n1; col[2] = -n0; col[3] = T(0); col[4] = v1; }
    else if (j == 3) { col[0] = T(0); col[1] = -n2; col[2] = T(0); col[3] = n0; col[4] = v2; }
    else { col[0] = T(1); col[1] = vel[0] + a * n0; col[2] = vel[1] + a * n1; col[3] = vel[2] + a * n2; col[4] = H + a * fa.vn; }
    // S[j] and Lam[j] by selects: j may be a run-time value (no local memory)
    const T Sj = j == 0 ? S[0] : (j == 1 ? S[1] : (j == 2 ? S[2] : (j == 3 ? S[3] : S[4])));
#pragma unroll
    for (int r = 0; r < 5; r++) col[r] *= Sj;
    // Z_k = (R S^(1/2))^T V_k of staged cell q
    auto zdot = [&](int q) {
      T acc = col[0] * sm->V[0][q] + col[1] * sm->V[1][q];
      if (DIM >= 2) acc = acc + col[2] * sm->V[2][q];
      if (DIM >= 3) acc = acc + col[3] * sm->V[3][q];
      acc = acc + col[4] * sm->V[4][q];
      return T(0.0) + acc;
    };
    T z[4];
#pragma unroll
    for (int k = 0; k < 4; k++) z[k] = zdot(cq + k);
    T zl = T(0), zr = T(0);
    if (qb) {
      const T zo0 = zdot(q0), zo5 = zdot(q0 + 5);
      if (valid) eno3_recon<T>(zo0, z[0], z[1], z[2], z[3], zo5, zl, zr);
    } else {
      reconstruct_lane<T, Sp>(P, NP, sm, lane, valid, z[0], z[1], z[2], z[3], zl, zr, viol, signv);
    }
    if (A.collect_buf && valid)
      collect_pair<T>(A, (unsigned)(blockIdx.x * 1024 + threadIdx.x) * 8u + (unsigned)j + 977u * collect_salt,
                      z[0], z[1], z[2], z[3], zl, zr);
    T dZ = zr - zl;
    if (valid && sign_checked<T, Sp>(P) && sign_violation<T>(z[0], z[1], z[2], z[3], zl, zr)) signv++;
    T ld = j == 0 ? Lam[0] : (j == 1 ? Lam[1] : (j == 2 ? Lam[2] : (j == 3 ? Lam[3] : Lam[4])));
#pragma unroll
    for (int i = 0; i < 5; i++) Diff[i] += col[i] * ld * dZ;
  };
  // The 2-D / 3-D FP32 DSP-WENO kernels keep this loop rolled: one copy of
  // the reconstruction (features, network, limiter) instead of four or five
  // relieves the instruction cache (KH 2048^2: 3.31 -> 3.23 ms per step).
  // Unrolled is faster for the SP-WENO family and for FP64 (1-3 %), and for
  // the 1-D kernels (3 components; the small 1-D grids of the matched-error
  // runs are bound by the latency of one warp task: 5 % faster).
  if constexpr (sizeof(T) == 4 && Sp::rec == 2 && DIM > 1) {
#pragma unroll 1
    for (int j = 0; j < 5; j++) component(j);
  } else {
#pragma unroll
    for (int j = 0; j < 5; j++) component(j);
  }
  flux[0] -= T(0.5) * Diff[0];
  flux[1] -= T(0.5) * Diff[1];
  flux[2] -= T(0.5) * Diff[2];
  if (DIM >= 3) flux[2] -= T(0.5) * Diff[3];   // momentum y, as the reference (kepes_tecno4_roe.cc:170)
  flux[4] -= T(0.5) * Diff[4];
}

// ------------------------------------------------------------ warp tasks --

// load the SEG_LOAD staged cells of a line segment (interior + ghosts) as
// primitive and entropy variables; ghost cells follow apply_bc
// (enflo/src/fv.cc:121-361): periodic wrap, wall mirror with the normal
// velocity negated, neumann copy of the boundary cell, dirichlet fixed state.
// qb = eno_shift(): staged cell q is c0 - 2 - qb + q, so that point-wise ENO
// of level 3 finds its third ghost cell at q = 0 and every other reader the
// four-cell stencil of face c0 + lane at q = lane + qb .. lane + qb + 3.
template <typename T, int DIR>
__device__ inline void euler_stage_cells(const SweepArgs<T>& A, const ProbDev& P, WarpSmem<T>* sm, int lane, int i0,
                                         int j0, int k0, int c0, int ncell, int qb) {
  const int N = dir_len<DIR>(P);
  const T G = T(P.gamma);
  for (int q = lane; q < ncell + 4 + 2 * qb; q += 32) {
    int c = c0 - 2 - qb + q;
    int side = c < 0 ? 0 : 1;
    int kind = (c >= 0 && c < N) ? DSPW_BC_PERIODIC : P.bc[2 * DIR + side];
    T p[5];
    if (kind == DSPW_BC_DIRICHLET) {
#pragma unroll
      for (int v = 0; v < 5; v++) p[v] = T(P.bc_state[2 * DIR + side][v]);
    } else {
      int flip;
      int src = ghost_source(c, N, kind, flip);
      T u[5];
      load_cons<T>(A.Uin, A.ctot, cell_index<DIR>(P, i0, j0, k0, src), P.nv, P.dim, u);
      cons_to_prim<T>(u, G, p);
      if (flip) p[1 + DIR] = -p[1 + DIR];
    }
    T v[5];
    prim_to_ent<T>(p, G, v);
#pragma unroll
    for (int w = 0; w < 5; w++) { sm->P[w][q] = p[w]; sm->V[w][q] = v[w]; }
  }
  __syncwarp();
}

// stage coefficients of the four-stage schemes (enflo/src/ext_constants.h:9-10)
DSPW_HD double jameson_coef(int rk) { return rk == 0 ? 1.0 / 4.0 : (rk == 1 ? 1.0 / 3.0 : (rk == 2 ? 1.0 / 2.0 : 1.0)); }
DSPW_HD double rk4_coef(int rk) { return (rk == 1 || rk == 2) ? 1.0 / 2.0 : 1.0; }

// stage update of one cell of a system (u holds the stage input on entry):
// SSPRK3 / RK1  U = b U + (a U^n + R (-factor b))        enflo/src/fv.cc:1163-1175
// Jameson RK4   U = U^n + R (-factor alpha_k)             enflo/src/fv.cc:1176-1184
// classic RK4   R2 += R / c_k; U = U^n + R (-factor c_(k+1)),
//               last stage U = U^n + R2 (-factor / 6)     enflo/src/fv.cc:1185-1197
// (R2 starts every step at zero: stage 0 does not read it)
template <typename T>
__device__ inline void stage_combine(const SweepArgs<T>& A, const ProbDev& P, const ProbState& S, long long cell,
                                     const T R[5], T u[5], const T un[5]) {
  if (A.scheme == DSPW_JAMESON_RK4) {
    const T c = T(-S.factor * jameson_coef(A.rk));
#pragma unroll
    for (int v = 0; v < 5; v++) u[v] = un[v] * T(1.0) + R[v] * c;
  } else if (A.scheme == DSPW_RK4) {
    T r2[5] = {T(0), T(0), T(0), T(0), T(0)};
    if (A.rk > 0) load_cons<T>(A.R2, A.ctot, cell, P.nv, P.dim, r2);
    const T inv = T(1.0 / rk4_coef(A.rk));
#pragma unroll
    for (int v = 0; v < 5; v++) r2[v] += R[v] * inv;
    if (A.rk < 3) {
      store_cons<T>(A.R2, A.ctot, cell, P.nv, r2);
      const T c = T(-S.factor * rk4_coef(A.rk + 1));
#pragma unroll
      for (int v = 0; v < 5; v++) u[v] = un[v] * T(1.0) + R[v] * c;
    } else {
      const T c = T(-S.factor / 6.0);
#pragma unroll
      for (int v = 0; v < 5; v++) u[v] = un[v] * T(1.0) + r2[v] * c;
    }
  } else {
    const T a = T(A.a_rk), b = T(A.b_rk);
    const T c2 = T(-S.factor * A.b_rk);
#pragma unroll
    for (int v = 0; v < 5; v++) {
      u[v] *= b;
      u[v] += un[v] * a + R[v] * c2;
    }
  }
}

// stage update of one Euler cell from its residual R, U^(k) (u) and U^n (un),
// stored to Uout, with the CFL speed / health epilogue on the stage
// that yields U^(n+1).
template <typename T>
__device__ inline void update_euler_cell(const SweepArgs<T>& A, const ProbDev& P, const ProbState& S, long long cell,
                                         const T R[5], T u[5], const T un[5], double& smax, double& ent,
                                         unsigned& bad_fin, unsigned& bad_pos) {
  stage_combine<T>(A, P, S, cell, R, u, un);
  store_cons<T>(A.Uout, A.ctot, cell, P.nv, u);
  if (A.store_R) store_cons<T>(A.R, A.ctot, cell, P.nv, R);
  if (A.final_stage) {
    T p[5];
    cons_to_prim<T>(u, T(P.gamma), p);
    double sp = wave_speed<T>(P, p);
    if (sp > smax) smax = sp;
    double rho = p[0], pr = p[4];
    if (!(rho > 0.0) || !(pr > 0.0)) bad_pos++;
    if (!isfinite(rho) || !isfinite(pr) || !isfinite((double)u[1]) || !isfinite((double)u[4])) bad_fin++;
    // entropy -rho s / (gamma - 1), s = ln p - gamma ln rho: the cell's term in
    // the state's type, the sum in FP64
    const T sT = Mth<T>::log(p[4]) - T(P.gamma) * Mth<T>::log(p[0]);
    ent += (double)(-p[0] * sT / T(P.gamma - 1.0));
  }
}

// final combination for one cell: residual (reference order
// ((R_prev - F_left) + F_right)) then either store R or apply the SSPRK stage
// update U = b U + (a U^n + R (-factor b)) (enflo/src/fv.cc:1163-1175), with
// the CFL speed / health epilogue on the stage that yields U^(n+1).
template <typename T>
__device__ inline void finish_cell(const SweepArgs<T>& A, const ProbDev& P, const ProbState& S, long long cell,
                                   bool first, bool final_sweep, const T Fl[5], const T Fr[5], int nv_eff,
                                   double& smax, double& ent, unsigned& bad_fin, unsigned& bad_pos) {
  T R[5];
  if (first) {
#pragma unroll
    for (int v = 0; v < 5; v++) R[v] = (T(0.0) - Fl[v]) + Fr[v];
  } else {
    T r0[5];
    if (P.is_scalar) { r0[0] = A.R[cell]; r0[1] = r0[2] = r0[3] = r0[4] = T(0); }
    else load_cons<T>(A.R, A.ctot, cell, P.nv, P.dim, r0);
#pragma unroll
    for (int v = 0; v < 5; v++) R[v] = (r0[v] - Fl[v]) + Fr[v];
  }
  if (!final_sweep) {
    if (P.is_scalar) A.R[cell] = R[0];
    else store_cons<T>(A.R, A.ctot, cell, P.nv, R);
    return;
  }
  const T a = T(A.a_rk), b = T(A.b_rk);
  const T c2 = T(-S.factor * A.b_rk);
  T u[5], un[5];
  if (P.is_scalar) {
    u[0] = A.Uin[cell];
    un[0] = A.Un[cell];
    T x;
    if (A.scheme == DSPW_JAMESON_RK4) {   // enflo_scalar/src_scalar/fv.cc:477-486
      x = un[0] - T(S.factor * jameson_coef(A.rk)) * R[0];
    } else if (A.scheme == DSPW_RK4) {    // enflo_scalar/src_scalar/fv.cc:487-499
      T r2 = (A.rk > 0 ? A.R2[cell] : T(0)) + R[0] / T(rk4_coef(A.rk));
      if (A.rk < 3) {
        A.R2[cell] = r2;
        x = un[0] - T(S.factor * rk4_coef(A.rk + 1)) * R[0];
      } else {
        x = un[0] - (T(S.factor) * r2) / T(6.0);
      }
    } else {
      x = u[0] * b;
      x = x + (un[0] * a - T(S.factor * A.b_rk) * R[0]);
    }
    A.Uout[cell] = x;
    if (A.store_R) A.R[cell] = R[0];
    if (A.final_stage) {
      T pp[5] = {x, T(0), T(0), T(0), T(0)};
      double sp = wave_speed<T>(P, pp);
      if (sp > smax) smax = sp;   // NaN speeds are skipped, as std::min skips them in compute_dt
      ent += 0.5 * (double)x * (double)x;   // entropy u^2 / 2, summed in FP64
      if (!isfinite((double)x)) bad_fin++;
    }
    return;
  }
  load_cons<T>(A.Uin, A.ctot, cell, P.nv, P.dim, u);
  load_cons<T>(A.Un, A.ctot, cell, P.nv, P.dim, un);
  update_euler_cell<T>(A, P, S, cell, R, u, un, smax, ent, bad_fin, bad_pos);
  (void)a; (void)c2; (void)nv_eff;
}

template <typename T>
__device__ inline void warp_epilogue(const SweepArgs<T>& A, bool final_stage, ProbState& S, int lane, double smax,
                                     double ent,
                                     unsigned bad_fin, unsigned bad_pos, unsigned long long signv, int viol,
                                     unsigned checked) {
  if (final_stage && !A.residual_only) {
    unsigned long long sb = (unsigned long long)__double_as_longlong(smax);
    warp_max_u64_lane0(sb);
    const double es = warp_sum(ent);
    if (lane == 0) {
      const int sl = blockIdx.x & (EPI_SLOTS - 1);
      atomicMax(&S.smax[sl], sb);
      atomicAdd(&S.ent_acc[sl], es);
    }
  }
  unsigned bf = __reduce_add_sync(0xffffffffu, bad_fin);
  unsigned bp = __reduce_add_sync(0xffffffffu, bad_pos);
  unsigned sv = __reduce_add_sync(0xffffffffu, (unsigned)signv);
  unsigned vv = __reduce_add_sync(0xffffffffu, (unsigned)viol);
  unsigned ck = __reduce_add_sync(0xffffffffu, checked);
  if (lane == 0) {
    const int sl = blockIdx.x & (EPI_SLOTS - 1);
    if (ck) atomicAdd(&A.status->faces_checked[sl], (unsigned long long)ck);
    if (bf) { atomicAdd(&A.status->nonfinite, (unsigned long long)bf); atomicCAS(&A.status->code, 0, DSPW_ERR_NONFINITE); }
    if (bp) { atomicAdd(&A.status->nonpositive, (unsigned long long)bp); atomicCAS(&A.status->code, 0, DSPW_ERR_NONPOSITIVE); }
    if (sv) atomicAdd(&A.status->sign_viol, (unsigned long long)sv);
    if (vv) atomicAdd(&A.status->limiter_acts[sl], (unsigned long long)vv);
  }
}

// Faces of one staged line segment (phases B and C): wide two-point fluxes,
// face central flux, TeCNO dissipation; face fluxes end in sm->F.
template <typename T, int DIR, int DIM, typename Sp>
__device__ inline void euler_faces(const SweepArgs<T>& A, const ProbDev& P, WarpSmem<T>* sm,
                                   int lane, int ncell, int& viol, unsigned long long& signv, unsigned& checked,
                                   unsigned collect_salt = 0) {
  const T G = T(P.gamma), Rg = T(P.gas_const), area = T(P.area[DIR]);
  const int qb = eno_shift<Sp>(P);
  // phase B: wide two-point flux centred at g = c0 - 1 + lane (cells g-1, g+1)
  const bool fourth = Sp::fixed || P.fourth;
  if (fourth && lane <= ncell + 1) {
    T Fw[5], Pl[5], Pr[5];
#pragma unroll
    for (int v = 0; v < 5; v++) { Pl[v] = sm->P[v][lane + qb]; Pr[v] = sm->P[v][lane + 2 + qb]; }
    if (Sp::fixed) kepec_pair<T, DIR>(Pl, Pr, G, Rg, area, Fw);
    else central_pair<T, DIR>(P.central, Pl, Pr, G, Rg, area, Fw);
#pragma unroll
    for (int v = 0; v < 5; v++) sm->W[v][lane] = Fw[v];
  }
  __syncwarp();
  // phase C: face f = c0 + lane between staged cells q = lane+1+qb and lane+2+qb
  const bool valid = lane <= ncell;
  const int lq = valid ? lane : 0;
  T flux[5] = {T(0), T(0), T(0), T(0), T(0)};
  FaceAvg<T> fa;
  {
    T Pl[5], Pr[5];
    const int ql = lq + 1 + qb;
#pragma unroll
    for (int v = 0; v < 5; v++) { Pl[v] = sm->P[v][ql]; Pr[v] = sm->P[v][ql + 1]; }
    face_avg<T, DIR>(Pl, Pr, Rg, fa);
    T Fn[5];
    if (Sp::fixed || P.central == 0) kepec_from_avg<T, DIR>(fa, Pl, Pr, G, area, Fn);
    else central_pair<T, DIR>(P.central, Pl, Pr, G, Rg, area, Fn);
    if (fourth) {
      // kepec4 / roe_ec4 / kep4: 4/3 F(1,2) - 1/6 F(0,2) - 1/6 F(1,3) (enflo/src/kepec4.cc:10-38)
      const T fact = T(-1.0 / 6.0);
#pragma unroll
      for (int v = 0; v < 5; v++) {
        T f = T(0.0);
        f += Fn[v] * T(4.0 / 3.0);
        f += sm->W[v][lq] * fact;
        f += sm->W[v][lq + 1] * fact;
        flux[v] = f;
      }
    } else {
#pragma unroll
      for (int v = 0; v < 5; v++) flux[v] = Fn[v];
    }
  }
  if (Sp::fixed || P.tecno) {
    const T ra = T(P.rarea[DIR]);
#pragma unroll
    for (int v = 0; v < 5; v++) flux[v] *= ra;
    tecno_dissipation<T, DIR, DIM, Sp>(A, P, *A.net, sm, lane, valid, lq, fa, flux, viol, signv, collect_salt);
#pragma unroll
    for (int v = 0; v < 5; v++) flux[v] *= area;
    checked = valid ? (DIM == 1 ? 3u : (DIM == 2 ? 4u : 5u)) : 0u;
  }
  if (valid) {
#pragma unroll
    for (int v = 0; v < 5; v++) sm->F[v][lane] = flux[v];
  }
  __syncwarp();
}

template <typename T, int DIR, int DIM, typename Sp>
__device__ void euler_task(const SweepArgs<T>& A, const ProbDev& P, ProbState& S,
                           WarpSmem<T>* sm, int lane, int lt) {
  int i0, j0, k0, c0, ncell;
  decode_task<DIR>(P, lt, i0, j0, k0, c0, ncell);
  euler_stage_cells<T, DIR>(A, P, sm, lane, i0, j0, k0, c0, ncell, eno_shift<Sp>(P));
  int viol = 0;
  unsigned long long signv = 0;
  unsigned checked = 0;
  euler_faces<T, DIR, DIM, Sp>(A, P, sm, lane, ncell, viol, signv, checked, (unsigned)lt);
  // phase D: cells
  const bool first = (DIR == 0);
  const bool final_sweep = !A.residual_only && !A.viscous && (DIR == DIM - 1);
  double smax = 0.0;
  double ent = 0.0;
  unsigned bad_fin = 0, bad_pos = 0;
  if (lane < ncell) {
    T Fl[5], Fr[5];
#pragma unroll
    for (int v = 0; v < 5; v++) { Fl[v] = sm->F[v][lane]; Fr[v] = sm->F[v][lane + 1]; }
    long long cell = cell_index<DIR>(P, i0, j0, k0, c0 + lane);
    finish_cell<T>(A, P, S, cell, first, final_sweep, Fl, Fr, P.nv, smax, ent, bad_fin, bad_pos);
  }
  if (!final_sweep) { smax = 0.0; ent = 0.0; }
  warp_epilogue<T>(A, A.final_stage && final_sweep, S, lane, smax, ent, bad_fin, bad_pos, signv, viol, checked);
  __syncwarp();
}

// Block-cooperative variant for the y and z sweeps: the 8 warps of the block
// hold 8 adjacent x-columns of the same line segment.  The staging loads and
// the cell epilogue run with threads laid out as 4 rows x 8 columns per warp
// instruction (8 consecutive x per row), instead of one strided cell per lane;
// the faces are evaluated per warp exactly as in euler_task.
constexpr int COOP_COLS = WARPS_PER_BLOCK;
// the narrow tiles of the y / z sweeps: 4 columns, one block of 4 warps
constexpr int NARROW_COLS = 4;

// Block-wide tiles of the cooperative sweep, behind the per-warp scratch in
// dynamic shared memory: the staged conserved rows of the 8 columns (ghost rows
// resolved), and the residual and U^n of the segment's cells for the epilogue.
// Planes are the stored components 0 .. nv-1.
template <typename T, int COLS = COOP_COLS>
struct CoopTiles {
  T U[5][SEG_LOAD][COLS];
  T R[5][SEG_CELLS][COLS];
  T Un[5][SEG_CELLS][COLS];
};
static_assert(sizeof(WarpSmem<double>) % 16 == 0, "WarpSmem<double> alignment");
static_assert((sizeof(WarpSmem<double>) / 4) % 32 == 12, "WarpSmem<double> bank spread");

// 16-byte global -> shared copy that completes asynchronously (L2 only)
__device__ inline void cp_async16(void* smem, const void* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ inline void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// u[5] of one tile entry (plane layout of load_cons)
template <typename T, int ROWS, int COLS>
__device__ inline void tile_cons(const T (*U)[ROWS][COLS], int nv, int q, int col, T u[5]) {
  u[0] = U[0][q][col];
  u[1] = U[1][q][col];
  if (nv == 5) { u[2] = U[2][q][col]; u[3] = U[3][q][col]; u[4] = U[4][q][col]; }
  else if (nv == 4) { u[2] = U[2][q][col]; u[3] = T(0); u[4] = U[3][q][col]; }
  else { u[2] = T(0); u[3] = T(0); u[4] = U[2][q][col]; }
}

// Block-cooperative variant for the y and z sweeps: the 8 warps of the block
// hold 8 adjacent x-columns of the same line segment.  The block first issues
// asynchronous row copies (8 adjacent x per row and plane) of the staged cells
// and, as a second group, of the residual and U^n of its cells; it converts the
// staged rows once the first group has landed, evaluates the faces per warp as
// in euler_task while the second group is in flight, and runs the cell
// epilogue from shared memory.  When the rows are not 16-byte aligned in
// global memory (nx, the problem offset or the plane stride not a multiple of
// 16 bytes) the same tiles are filled by plain loads.
// Conversion of the staged rows of a block task: row q = tid / 8 (+ 32) of
// column col, from the tile U (ghost rows already resolved to their source
// rows), into the per-warp primitive / entropy rows of warp `col`.
template <typename T, int DIR, int COLS>
__device__ __forceinline__ void coop_convert(const ProbDev& P, WarpSmem<T>* sm0, const T (*U)[SEG_LOAD][COLS], int c0,
                                    int nrow, int ncols) {
  const int tid = threadIdx.x, col = tid % COLS;
  const int N = dir_len<DIR>(P);
  const T G = T(P.gamma);
  for (int q = tid / COLS; q < nrow && col < ncols; q += 32) {   // COLS warps: 32 rows per pass
    const int c = c0 - 2 + q;
    const int side = c < 0 ? 0 : 1;
    const int kind = (c >= 0 && c < N) ? DSPW_BC_PERIODIC : P.bc[2 * DIR + side];
    T p[5];
    if (kind == DSPW_BC_DIRICHLET) {
#pragma unroll
      for (int v = 0; v < 5; v++) p[v] = T(P.bc_state[2 * DIR + side][v]);
    } else {
      int flip;
      ghost_source(c, N, kind, flip);
      T u[5];
      tile_cons(U, P.nv, q, col, u);
      cons_to_prim<T>(u, G, p);
      if (flip) p[1 + DIR] = -p[1 + DIR];
    }
    T v[5];
    prim_to_ent<T>(p, G, v);
    WarpSmem<T>* sc = sm0 + col;
#pragma unroll
    for (int w = 0; w < 5; w++) { sc->P[w][q] = p[w]; sc->V[w][q] = v[w]; }
  }
}

// Cell epilogue of a block task: residual from the tile R and the warps' face
// fluxes, then either the stored residual or the stage update from the tiles
// U (rows + 2) and Un, with threads laid out as 4 rows x 8 columns per warp
// instruction (coalesced stores).
template <typename T, int DIR, int COLS>
__device__ __forceinline__ void coop_epilogue(const SweepArgs<T>& A, const ProbDev& P, const ProbState& S, WarpSmem<T>* sm0,
                                     const T (*U)[SEG_LOAD][COLS], const T (*Rt)[SEG_CELLS][COLS],
                                     const T (*Unt)[SEG_CELLS][COLS], int i0, int j0, int k0, int c0,
                                     int ncell, int ncols, bool final_sweep, double& smax, double& ent,
                                     unsigned& bad_fin, unsigned& bad_pos) {
  const int tid = threadIdx.x, col = tid % COLS;
  const int nv = P.nv;
  for (int row = tid / COLS; row < ncell && col < ncols; row += 32) {   // COLS warps: 32 rows per pass
    WarpSmem<T>* sc = sm0 + col;
    T R[5], r0[5];
    tile_cons(Rt, nv, row, col, r0);
#pragma unroll
    for (int v = 0; v < 5; v++) R[v] = (r0[v] - sc->F[v][row]) + sc->F[v][row + 1];
    const long long cell = cell_index<DIR>(P, i0 + col, j0, k0, c0 + row);
    if (!final_sweep) {
      store_cons<T>(A.R, A.ctot, cell, nv, R);
    } else {
      T u[5], un[5];
      tile_cons(U, nv, row + 2, col, u);
      tile_cons(Unt, nv, row, col, un);
      update_euler_cell<T>(A, P, S, cell, R, u, un, smax, ent, bad_fin, bad_pos);
    }
  }
}

// Block-cooperative variant for the y and z sweeps: the 8 warps of the block
// hold 8 adjacent x-columns of the same line segment.  The block first issues
// asynchronous row copies (8 adjacent x per row and plane) of the staged cells
// and, as a second group, of the residual and U^n of its cells; it converts the
// staged rows once the first group has landed, evaluates the faces per warp as
// in euler_task while the second group is in flight, and runs the cell
// epilogue from shared memory.  When the rows are not 16-byte aligned in
// global memory (nx, the problem offset or the plane stride not a multiple of
// 16 bytes) the same tiles are filled by plain loads.
// COLS: columns of the block, one warp each (8, or 4 for the narrow tiles of
// k_sweep_narrow); the block has COLS warps.
template <typename T, int DIR, int DIM, typename Sp, int COLS = COOP_COLS>
__device__ void euler_coop_block(const SweepArgs<T>& A, const ProbDev& P, ProbState& S,
                                 WarpSmem<T>* sm0, int lt0, bool group) {
  static_assert(COLS == COOP_COLS || COLS == NARROW_COLS, "column count of a block");
  constexpr int NT = COLS * 32;                       // threads of the block
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int i0, j0, k0, c0, ncell, ncols = COLS;
  // i0 of column 0 (a multiple of COLS); group tasks may end in a partial group
  if (group) decode_group<DIR, COLS>(P, lt0, i0, j0, k0, c0, ncell, ncols);
  else decode_task<DIR>(P, lt0, i0, j0, k0, c0, ncell);
  const int N = dir_len<DIR>(P);
  const int nv = P.nv;
  CoopTiles<T, COLS>& tl = *reinterpret_cast<CoopTiles<T, COLS>*>(sm0 + COLS);
  const bool final_sweep = !A.residual_only && !A.viscous && (DIR == DIM - 1);
  constexpr int VEC = 16 / (int)sizeof(T);           // elements per 16-byte copy
  constexpr int CH = COLS / VEC;                      // copies per row and plane
  static_assert(CH >= 1, "a row of the tile is at least one 16-byte copy");
  const bool aligned = ncols == COLS && (A.ctot % VEC) == 0 && (P.off % VEC) == 0 && (P.nx % VEC) == 0;
  // group 1: staged rows q = 0 .. ncell+3 (cells c0-2 .. c0+ncell+1)
  const int nrow = ncell + 4;
  if (aligned) {
    // one thread per (row, 16-byte chunk): its ghost source is found once and
    // it issues the copies of every component (no division by the row count)
    static_assert((SEG_CELLS + 4) * CH <= NT, "one pass of the block covers the staged rows");
    if (tid < nrow * CH) {
      const int q = tid / CH, ch = tid - q * CH;
      const int c = c0 - 2 + q;
      const int kind = (c >= 0 && c < N) ? DSPW_BC_PERIODIC : P.bc[2 * DIR + (c < 0 ? 0 : 1)];
      if (kind != DSPW_BC_DIRICHLET) {
        int flip;
        const int src = ghost_source(c, N, kind, flip);
        const long long base = cell_index<DIR>(P, i0 + ch * VEC, j0, k0, src);
        for (int comp = 0; comp < nv; comp++) cp_async16(&tl.U[comp][q][ch * VEC], A.Uin + comp * A.ctot + base);
      }
    }
    cp_async_commit();
    // group 2: residual (the previous sweep's) and U^n of the cells
    if (tid < ncell * CH) {
      const int q = tid / CH, ch = tid - q * CH;
      const long long base = cell_index<DIR>(P, i0 + ch * VEC, j0, k0, c0 + q);
      for (int comp = 0; comp < nv; comp++) {
        cp_async16(&tl.R[comp][q][ch * VEC], A.R + comp * A.ctot + base);
        if (final_sweep) cp_async16(&tl.Un[comp][q][ch * VEC], A.Un + comp * A.ctot + base);
      }
    }
    cp_async_commit();
    cp_async_wait<1>();
  } else {
    for (int idx = tid; idx < nv * nrow * COLS; idx += NT) {
      const int comp = idx / (nrow * COLS), rem = idx - comp * nrow * COLS, q = rem / COLS, cc = rem - q * COLS;
      const int c = c0 - 2 + q;
      const int kind = (c >= 0 && c < N) ? DSPW_BC_PERIODIC : P.bc[2 * DIR + (c < 0 ? 0 : 1)];
      if (kind == DSPW_BC_DIRICHLET || cc >= ncols) continue;
      int flip;
      const int src = ghost_source(c, N, kind, flip);
      tl.U[comp][q][cc] = A.Uin[comp * A.ctot + cell_index<DIR>(P, i0 + cc, j0, k0, src)];
    }
    for (int idx = tid; idx < nv * ncell * COLS; idx += NT) {
      const int comp = idx / (ncell * COLS), rem = idx - comp * ncell * COLS, q = rem / COLS, cc = rem - q * COLS;
      if (cc >= ncols) continue;
      const long long off = comp * A.ctot + cell_index<DIR>(P, i0 + cc, j0, k0, c0 + q);
      tl.R[comp][q][cc] = A.R[off];
      if (final_sweep) tl.Un[comp][q][cc] = A.Un[off];
    }
  }
  __syncthreads();
  coop_convert<T, DIR, COLS>(P, sm0, tl.U, c0, nrow, ncols);
  __syncthreads();
  int viol = 0;
  unsigned long long signv = 0;
  unsigned checked = 0;
  if (warp < ncols)   // warp-uniform: the network inside needs every lane of the warp
    euler_faces<T, DIR, DIM, Sp>(A, P, sm0 + warp, lane, ncell, viol, signv, checked, (unsigned)(lt0 + warp));
  if (aligned) cp_async_wait<0>();
  __syncthreads();
  double smax = 0.0;
  double ent = 0.0;
  unsigned bad_fin = 0, bad_pos = 0;
  coop_epilogue<T, DIR, COLS>(A, P, S, sm0, tl.U, tl.R, tl.Un, i0, j0, k0, c0, ncell, ncols, final_sweep, smax,
                              ent, bad_fin, bad_pos);
  if (!final_sweep) { smax = 0.0; ent = 0.0; }
  warp_epilogue<T>(A, A.final_stage && final_sweep, S, lane, smax, ent, bad_fin, bad_pos, signv, viol, checked);
  __syncthreads();
}

// --------------------------------------------------- TMA staging (y / z) --
//
// The specialised y and z sweeps can stage their tiles with the Tensor Memory
// Accelerator instead of per-thread cp.async copies: one thread issues one
// cp.async.bulk.tensor per tile (box of 8 columns x rows x nv planes of this
// GPU's own state, loaded into this block alone) that signals an mbarrier when its bytes have
// landed.  Each block runs its tasks in a loop that prefetches the next task's
// staged rows into a second buffer while the current task's faces are
// evaluated, and loads the residual and U^n of a task at the task's start (they
// are read only by its epilogue).  Rows outside the problem (the two ghost rows
// of a segment at a domain face) are outside the tensor map, so the box fills
// them with zeros; they are then replaced by their boundary-condition source
// rows with plain loads, as the cp.async path stages them.  Every wait on an
// mbarrier is bounded: after TMA_WAIT_LIMIT tries the block records
// DSPW_ERR_TIMEOUT in the status word and leaves the loop.

// byte layout of the TMA region (behind the per-warp scratch, 128-byte
// aligned): three mbarriers, two staged-row tiles, the residual tile, the U^n tile
template <typename T>
struct TmaLayout {
  static constexpr size_t round128(size_t b) { return (b + 127) / 128 * 128; }
  static constexpr size_t u_bytes = round128(sizeof(T) * 5 * SEG_LOAD * COOP_COLS);
  static constexpr size_t r_bytes = round128(sizeof(T) * 5 * SEG_CELLS * COOP_COLS);
  static constexpr size_t bars = 128;
  static constexpr size_t total = bars + 2 * u_bytes + 2 * r_bytes + 128;   // + alignment slack
};

constexpr long long TMA_WAIT_LIMIT = 1LL << 24;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait for the phase of the given parity; false after TMA_WAIT_LIMIT tries
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  for (long long i = 0; i < TMA_WAIT_LIMIT; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// generic-proxy accesses of shared memory before this point are ordered before
// later asynchronous-proxy (TMA) accesses
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// 4-D tiled load (x, y, z, component) of this GPU's global memory into shared
// memory, completion counted on the mbarrier; x is a multiple of 8 elements
// (16-byte aligned), y / z may lie outside the tensor (zero fill)
__device__ __forceinline__ void tma_load_4d(void* dst, const void* map, int x, int y, int z, int c, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
      ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(c), "r"(smem_u32(bar))
      : "memory");
}

// the next task >= g of this block's stride whose problem is stepping (or any
// task for a residual evaluation); A.ntask when none is left
template <typename T>
__device__ __forceinline__ int next_live_task(const SweepArgs<T>& A, int g) {
  for (; g < A.ntask; g += gridDim.x) {
    if (A.residual_only) return g;
    const int p = find_problem(A.task_start, A.nprob, g);
    const int pp = A.pmap ? __ldg(A.pmap + p) : p;
    if (*((volatile int*)&A.st[pp].active)) return g;
  }
  return A.ntask;
}

// coordinates of task g's tile origin: problem (class index), column i0 and
// the (y, z) of its first cell row
template <typename T, int DIR>
__device__ __forceinline__ void tma_task(const SweepArgs<T>& A, int g, int& p, int& i0, int& j0, int& k0, int& c0, int& ncell) {
  p = find_problem(A.task_start, A.nprob, g);
  const int pp = A.pmap ? __ldg(A.pmap + p) : p;
  int ncols;
  decode_group<DIR>(A.prob[pp], g - __ldg(A.task_start + p), i0, j0, k0, c0, ncell, ncols);
}

template <typename T, int DIR>
__device__ __forceinline__ void tma_issue_rows(const SweepArgs<T>& A, int g, unsigned char* ubuf, unsigned long long* bar) {
  int p, i0, j0, k0, c0, ncell;
  tma_task<T, DIR>(A, g, p, i0, j0, k0, c0, ncell);
  const int pp = A.pmap ? __ldg(A.pmap + p) : p;
  const int nv = A.prob[pp].nv;
  const unsigned char* maps = (const unsigned char*)A.tmaps;
  mbar_expect_tx(bar, (unsigned)(sizeof(T) * COOP_COLS * SEG_LOAD * nv));
  const int y = DIR == 1 ? c0 - 2 : j0, z = DIR == 1 ? k0 : c0 - 2;
  tma_load_4d(ubuf, maps + (size_t)TMA_MAP_BYTES * tma_map_index(p, DIR, A.tma_in), i0, y, z, 0, bar);
}

template <typename T, int DIR>
__device__ __forceinline__ void tma_issue_cells(const SweepArgs<T>& A, int g, bool final_sweep, unsigned char* rbuf,
                                       unsigned char* unbuf, unsigned long long* bar) {
  int p, i0, j0, k0, c0, ncell;
  tma_task<T, DIR>(A, g, p, i0, j0, k0, c0, ncell);
  const int pp = A.pmap ? __ldg(A.pmap + p) : p;
  const int nv = A.prob[pp].nv;
  const unsigned char* maps = (const unsigned char*)A.tmaps;
  const unsigned bytes = (unsigned)(sizeof(T) * COOP_COLS * SEG_CELLS * nv);
  mbar_expect_tx(bar, final_sweep ? 2 * bytes : bytes);
  const int y = DIR == 1 ? c0 : j0, z = DIR == 1 ? k0 : c0;
  tma_load_4d(rbuf, maps + (size_t)TMA_MAP_BYTES * tma_map_index(p, DIR, 3), i0, y, z, 0, bar);
  if (final_sweep) tma_load_4d(unbuf, maps + (size_t)TMA_MAP_BYTES * tma_map_index(p, DIR, 4), i0, y, z, 0, bar);
}

// The task loop of a specialised y / z sweep with TMA staging (see above).
// Every problem of the class has nx a multiple of 8 and 16-byte aligned rows
// (the host builds the tensor maps only then), so every task is a full group
// of 8 columns.
template <typename T, int DIR, int DIM, typename Sp>
__device__ __forceinline__ void euler_coop_tma_loop(const SweepArgs<T>& A, WarpSmem<T>* sm0) {
  typedef TmaLayout<T> L;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned char* base = reinterpret_cast<unsigned char*>(sm0 + WARPS_PER_BLOCK);
  base = reinterpret_cast<unsigned char*>(((size_t)base + 127) & ~(size_t)127);
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(base);   // [0], [1]: rows; [2]: cells
  unsigned char* const ubuf0 = base + L::bars;
  unsigned char* const ubuf1 = base + L::bars + L::u_bytes;
  unsigned char* rbuf = base + L::bars + 2 * L::u_bytes;
  unsigned char* unbuf = rbuf + L::r_bytes;
  typedef const T(*UTile)[SEG_LOAD][COOP_COLS];
  typedef const T(*CTile)[SEG_CELLS][COOP_COLS];
  const bool final_sweep = !A.residual_only && !A.viscous && (DIR == DIM - 1);
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init(&bar[2], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fence_proxy_async_smem();
  }
  __syncthreads();
  // mbarrier phases of the two row buffers and of the cell tiles (scalars and
  // selects: an array indexed by the buffer number would live in local memory)
  unsigned ph_u0 = 0u, ph_u1 = 0u, ph_c = 0u;
  int g = next_live_task(A, blockIdx.x);
  if (tid == 0 && g < A.ntask) tma_issue_rows<T, DIR>(A, g, ubuf0, &bar[0]);
  int b = 0;
  bool timed_out = false;
  while (g < A.ntask) {
    const int gn = next_live_task(A, g + gridDim.x);
    int p, i0, j0, k0, c0, ncell;
    tma_task<T, DIR>(A, g, p, i0, j0, k0, c0, ncell);
    const int pp = A.pmap ? __ldg(A.pmap + p) : p;
    const ProbDev& P = A.prob[pp];
    ProbState& S = A.st[pp];
    const int N = dir_len<DIR>(P);
    const int nrow = ncell + 4;
    // the cell tiles of this task (free: the previous task ended at a barrier)
    if (tid == 0) {
      fence_proxy_async_smem();
      tma_issue_cells<T, DIR>(A, g, final_sweep, rbuf, unbuf, &bar[2]);
    }
    // staged rows of this task (prefetched)
    unsigned char* const ucur = b ? ubuf1 : ubuf0;
    unsigned char* const unext = b ? ubuf0 : ubuf1;
    unsigned long long* const bcur = b ? &bar[1] : &bar[0];
    unsigned long long* const bnext = b ? &bar[0] : &bar[1];
    if (!mbar_wait(bcur, b ? ph_u1 : ph_u0)) timed_out = true;
    if (b) ph_u1 ^= 1u; else ph_u0 ^= 1u;
    // rows outside the problem: their boundary-condition source rows
    T(*U)[SEG_LOAD][COOP_COLS] = reinterpret_cast<T(*)[SEG_LOAD][COOP_COLS]>(ucur);
    for (int idx = tid; idx < nrow * COOP_COLS; idx += WARPS_PER_BLOCK * 32) {
      const int q = idx / COOP_COLS, cc = idx - q * COOP_COLS;
      const int c = c0 - 2 + q;
      if (c >= 0 && c < N) continue;
      const int kind = P.bc[2 * DIR + (c < 0 ? 0 : 1)];
      if (kind == DSPW_BC_DIRICHLET) continue;
      int flip;
      const int src = ghost_source(c, N, kind, flip);
      const long long cell = cell_index<DIR>(P, i0 + cc, j0, k0, src);
      for (int comp = 0; comp < P.nv; comp++) U[comp][q][cc] = A.Uin[comp * A.ctot + cell];
    }
    __syncthreads();
    coop_convert<T, DIR, COOP_COLS>(P, sm0, (UTile)U, c0, nrow, COOP_COLS);
    __syncthreads();
    // the next task's rows into the other buffer, behind this task's faces
    if (tid == 0 && gn < A.ntask) {
      fence_proxy_async_smem();
      tma_issue_rows<T, DIR>(A, gn, unext, bnext);
    }
    int viol = 0;
    unsigned long long signv = 0;
    unsigned checked = 0;
    const int lt0 = g - __ldg(A.task_start + p);
    euler_faces<T, DIR, DIM, Sp>(A, P, sm0 + warp, lane, ncell, viol, signv, checked, (unsigned)(lt0 + warp));
    if (!mbar_wait(&bar[2], ph_c)) timed_out = true;
    ph_c ^= 1u;
    __syncthreads();
    double smax = 0.0, ent = 0.0;
    unsigned bad_fin = 0, bad_pos = 0;
    coop_epilogue<T, DIR, COOP_COLS>(A, P, S, sm0, (UTile)U, (CTile)rbuf, (CTile)unbuf, i0, j0, k0, c0, ncell, COOP_COLS,
                          final_sweep, smax, ent, bad_fin, bad_pos);
    if (!final_sweep) { smax = 0.0; ent = 0.0; }
    warp_epilogue<T>(A, A.final_stage && final_sweep, S, lane, smax, ent, bad_fin, bad_pos, signv, viol, checked);
    // this task's shared-memory accesses (the ghost-row stores among them) are
    // ordered before the TMA writes that refill the tiles; the barrier ends
    // the task for every thread
    fence_proxy_async_smem();
    if (__syncthreads_or(timed_out)) {
      // a copy that did not complete: record it and wait (bounded) for the
      // prefetch still in flight before the block leaves
      if (tid == 0) atomicCAS(&A.status->code, 0, DSPW_ERR_TIMEOUT);
      if (gn < A.ntask) mbar_wait(bnext, b ? ph_u0 : ph_u1);
      break;
    }
    g = gn;
    b ^= 1;
  }
}

// scalar laws: lin_/bur_ fluxes (enflo_scalar/src_scalar/num_flux.cc:12-57,
// lin_tecno4.cc:10-31, lin_ec4.cc:10-34, bur_tecno4.cc:10-35, bur_ec4.cc:10-34)
template <typename T, int DIR, typename Sp = SpecGeneric>
__device__ void scalar_task(const SweepArgs<T>& A, const ProbDev& P, ProbState& S,
                            WarpSmem<T>* sm, int lane, int lt) {
  typedef Mth<T> m;
  int i0, j0, k0, c0, ncell;
  decode_task<DIR>(P, lt, i0, j0, k0, c0, ncell);
  const int N = dir_len<DIR>(P);
  const int qb = eno_shift<Sp>(P);
  for (int q = lane; q < ncell + 4 + 2 * qb; q += 32) {
    int c = c0 - 2 - qb + q;
    int side = c < 0 ? 0 : 1;
    int kind = (c >= 0 && c < N) ? DSPW_BC_PERIODIC : P.bc[2 * DIR + side];
    T u;
    if (kind == DSPW_BC_DIRICHLET) u = T(P.bc_state[2 * DIR + side][0]);
    else {
      int flip;
      int src = ghost_source(c, N, kind, flip);
      u = A.Uin[cell_index<DIR>(P, i0, j0, k0, src)];
      if (flip) u = -u;
    }
    sm->P[0][q] = u;
  }
  __syncwarp();
  const bool valid = lane <= ncell;
  const int q = (valid ? lane : 0) + qb;
  T s0 = sm->P[0][q], s1 = sm->P[0][q + 1], s2 = sm->P[0][q + 2], s3 = sm->P[0][q + 3];
  const T vn = T(P.lin_vn[DIR]);
  T flux = T(0);
  const int fl = P.flux;
  if (fl == DSPW_LIN_EC || fl == DSPW_LIN_TECNO) {
    flux = T(0.5) * vn * (s1 + s2);
  } else if (fl == DSPW_LIN_EC4 || fl == DSPW_LIN_TECNO4) {
    flux = T(0.0);
    flux += m::div((T(0.5) * vn * (s1 + s2)) * T(4.0), T(3.0));
    flux += (T(0.5) * vn * (s0 + s2)) * T(-1.0 / 6.0);
    flux += (T(0.5) * vn * (s1 + s3)) * T(-1.0 / 6.0);
  } else if (fl == DSPW_BUR_EC || fl == DSPW_BUR_TECNO) {
    flux = m::div(s1 * s1 + s2 * s2 + s1 * s2, T(6.0));
  } else {
    flux = T(0.0);
    flux += m::div(s1 * s1 + s2 * s2 + s1 * s2, T(6.0)) * T(4.0 / 3.0);
    flux += m::div(s0 * s0 + s2 * s2 + s0 * s2, T(6.0)) * T(-1.0 / 6.0);
    flux += m::div(s1 * s1 + s3 * s3 + s1 * s3, T(6.0)) * T(-1.0 / 6.0);
  }
  int viol = 0;
  unsigned long long signv = 0;
  if (P.tecno) {
    T D = (P.model == DSPW_LINADV) ? m::abs(vn) : T(0.5) * (m::abs(s1) + m::abs(s2));
    T l = T(0), r = T(0);
    if (qb) {
      if (valid) eno3_recon<T>(sm->P[0][q - 1], s0, s1, s2, s3, sm->P[0][q + 4], l, r);
    } else {
      reconstruct_lane<T, Sp>(P, *A.net, sm, lane, valid, s0, s1, s2, s3, l, r, viol, signv);
    }
    if (valid && sign_checked<T, Sp>(P) && sign_violation<T>(s0, s1, s2, s3, l, r)) signv++;
    if (A.collect_buf && valid) collect_pair<T>(A, (unsigned)lt * 32u + (unsigned)lane, s0, s1, s2, s3, l, r);
    flux -= T(0.5) * D * (r - l);
  }
  flux *= T(P.area[DIR]);
  if (valid) sm->F[0][lane] = flux;
  __syncwarp();
  const bool first = (DIR == 0);
  const bool final_sweep = !A.residual_only && (DIR == P.dim - 1);
  double smax = 0.0;
  double ent = 0.0;
  unsigned bad_fin = 0, bad_pos = 0;
  if (lane < ncell) {
    T Fl[5] = {sm->F[0][lane], T(0), T(0), T(0), T(0)};
    T Fr[5] = {sm->F[0][lane + 1], T(0), T(0), T(0), T(0)};
    long long cell = cell_index<DIR>(P, i0, j0, k0, c0 + lane);
    finish_cell<T>(A, P, S, cell, first, final_sweep, Fl, Fr, 1, smax, ent, bad_fin, bad_pos);
  }
  warp_epilogue<T>(A, A.final_stage && final_sweep, S, lane, smax, ent, bad_fin, bad_pos, signv, viol, (P.tecno && valid) ? 1u : 0u);
  __syncwarp();
}

// One sweep of direction DIR over every problem of the batch.  Sp fixes the
// model, dimension and flux structure (SpecHot) or leaves them to ProbDev
// (SpecGeneric); a SpecHot kernel is only launched for directions < its dim.
template <typename T, int DIR, typename Sp>
__global__ void __launch_bounds__(WARPS_PER_BLOCK * 32, MinBlocks<T>::value)
k_sweep(const __grid_constant__ SweepArgs<T> A) {   // grid constant: references to A need no local copy
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSmem<T>* sm0 = reinterpret_cast<WarpSmem<T>*>(smem_raw);
  WarpSmem<T>* sm = sm0 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (!Sp::fixed || Sp::rec == 2) net_frag_stage<T>(*A.net, lane, sm->ns);
  if constexpr (Sp::fixed && DIR >= 1) {
    // specialised y / z sweeps: every task is one block-cooperative column group
    for (int g = blockIdx.x; g < A.ntask; g += gridDim.x) {
      const int p = find_problem(A.task_start, A.nprob, g);
      const int pp = A.pmap ? __ldg(A.pmap + p) : p;
      const ProbDev& P = A.prob[pp];
      ProbState& S = A.st[pp];
      if (!A.residual_only && !*((volatile int*)&S.active)) continue;
      euler_coop_block<T, DIR, Sp::dim, Sp>(A, P, S, sm0, g - __ldg(A.task_start + p), true);
    }
  } else {
    const int stride = gridDim.x * WARPS_PER_BLOCK;
    for (int base = blockIdx.x * WARPS_PER_BLOCK; base < A.ntask; base += stride) {
      if (DIR >= 1 && base + WARPS_PER_BLOCK <= A.ntask) {
        // block-uniform test: 8 tasks of one Euler problem on 8 adjacent columns
        const int p = find_problem(A.task_start, A.nprob, base);
        const int pp = A.pmap ? __ldg(A.pmap + p) : p;
        const int lt0 = base - __ldg(A.task_start + p);
        const ProbDev& P = A.prob[pp];
        if ((Sp::fixed || (!P.is_scalar && P.recon != DSPW_REC_ENO3)) &&
            base + WARPS_PER_BLOCK <= __ldg(A.task_start + p + 1) &&
            (lt0 % P.nx) % COOP_COLS == 0 && (lt0 % P.nx) + COOP_COLS <= P.nx) {
          ProbState& S = A.st[pp];
          if (!A.residual_only && !*((volatile int*)&S.active)) continue;
          if constexpr (Sp::fixed) {
            euler_coop_block<T, DIR, Sp::dim, Sp>(A, P, S, sm0, lt0, false);
          } else if (DIR == 1) {
            if (P.dim == 2) euler_coop_block<T, DIR, 2, Sp>(A, P, S, sm0, lt0, false);
            else euler_coop_block<T, DIR, 3, Sp>(A, P, S, sm0, lt0, false);
          } else {
            euler_coop_block<T, DIR, 3, Sp>(A, P, S, sm0, lt0, false);
          }
          continue;
        }
      }
      const int task = base + (threadIdx.x >> 5);
      if (task >= A.ntask) continue;
      const int p = find_problem(A.task_start, A.nprob, task);
      const int pp = A.pmap ? __ldg(A.pmap + p) : p;
      const ProbDev& P = A.prob[pp];
      ProbState& S = A.st[pp];
      if (!A.residual_only && !*((volatile int*)&S.active)) continue;
      const int lt = task - __ldg(A.task_start + p);
      if constexpr (Sp::fixed) {
        euler_task<T, DIR, Sp::dim, Sp>(A, P, S, sm, lane, lt);
      } else if (P.is_scalar) {
        scalar_task<T, DIR>(A, P, S, sm, lane, lt);
      } else {
        if (DIR == 0) {
          if (P.dim == 1) euler_task<T, DIR, 1, Sp>(A, P, S, sm, lane, lt);
          else if (P.dim == 2) euler_task<T, DIR, 2, Sp>(A, P, S, sm, lane, lt);
          else euler_task<T, DIR, 3, Sp>(A, P, S, sm, lane, lt);
        } else if (DIR == 1) {
          if (P.dim == 2) euler_task<T, DIR, 2, Sp>(A, P, S, sm, lane, lt);
          else euler_task<T, DIR, 3, Sp>(A, P, S, sm, lane, lt);
        } else {
          euler_task<T, DIR, 3, Sp>(A, P, S, sm, lane, lt);
        }
      }
    }
  }
}

// The specialised y / z sweeps with TMA staging (euler_coop_tma_loop): a
// kernel of its own, so that the loop's state does not take registers from the
// cp.async kernel.
template <typename T, int DIR, typename Sp>
__global__ void __launch_bounds__(WARPS_PER_BLOCK * 32, MinBlocks<T>::value)
k_sweep_tma(const __grid_constant__ SweepArgs<T> A) {
  static_assert(Sp::fixed && DIR >= 1, "TMA staging is for the specialised y / z sweeps");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSmem<T>* sm0 = reinterpret_cast<WarpSmem<T>*>(smem_raw);
  const int lane = threadIdx.x & 31;
  if (Sp::rec == 2) net_frag_stage<T>(*A.net, lane, sm0[threadIdx.x >> 5].ns);
  euler_coop_tma_loop<T, DIR, Sp::dim, Sp>(A, sm0);
}

// The specialised y / z sweeps with narrow tiles: blocks of 4 warps on 4
// adjacent columns (16-byte FP32 rows, per-thread cp.async staging), twice the
// resident blocks per SM of k_sweep at the same registers per thread.  Each
// block barrier then waits for 4 warps instead of 8.  The task list of a
// direction that runs it counts groups of 4 columns (decode_group).
template <typename T, int DIR, typename Sp>
__global__ void __launch_bounds__(NARROW_COLS * 32, 2 * MinBlocks<T>::value)
k_sweep_narrow(const __grid_constant__ SweepArgs<T> A) {
  static_assert(Sp::fixed && DIR >= 1, "narrow tiles are for the specialised y / z sweeps");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSmem<T>* sm0 = reinterpret_cast<WarpSmem<T>*>(smem_raw);
  const int lane = threadIdx.x & 31;
  if (Sp::rec == 2) net_frag_stage<T>(*A.net, lane, sm0[threadIdx.x >> 5].ns);
  for (int g = blockIdx.x; g < A.ntask; g += gridDim.x) {
    const int p = find_problem(A.task_start, A.nprob, g);
    const int pp = A.pmap ? __ldg(A.pmap + p) : p;
    const ProbDev& P = A.prob[pp];
    ProbState& S = A.st[pp];
    if (!A.residual_only && !*((volatile int*)&S.active)) continue;
    euler_coop_block<T, DIR, Sp::dim, Sp, NARROW_COLS>(A, P, S, sm0, g - __ldg(A.task_start + p), true);
  }
}

// The x sweep of 1-D scalar problems alone: the reconstruction family fixed at
// compile time (REC 1: SP-WENO, the correction a run-time flag; 2: DSP-WENO),
// none of the Euler code of the generic kernel, and its own register budget.
template <typename T, int REC>
__global__ void __launch_bounds__(WARPS_PER_BLOCK * 32, ScalarMinBlocks<T>::value)
k_sweep_scalar(SweepArgs<T> A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSmem<T>* sm = reinterpret_cast<WarpSmem<T>*>(smem_raw) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (REC == 2) net_frag_stage<T>(*A.net, lane, sm->ns);
  const int stride = gridDim.x * WARPS_PER_BLOCK;
  for (int base = blockIdx.x * WARPS_PER_BLOCK; base < A.ntask; base += stride) {
    const int task = base + (threadIdx.x >> 5);
    if (task >= A.ntask) continue;
    const int p = find_problem(A.task_start, A.nprob, task);
    const int pp = A.pmap ? __ldg(A.pmap + p) : p;
    const ProbDev& P = A.prob[pp];
    ProbState& S = A.st[pp];
    if (!A.residual_only && !*((volatile int*)&S.active)) continue;
    scalar_task<T, 0, SpecHot<1, REC>>(A, P, S, sm, lane, task - __ldg(A.task_start + p));
  }
}

// ----------------------------------------------------------- step control --

// upload: primitive (FP64, staging) -> conserved state, plus the wave speed of
// that primitive state (prim_to_con, enflo/src/fv.cc:405-416) and the sum of
// its entropy (in the state's type, as the steps take it)
template <typename T>
__global__ void k_upload(const ProbDev* prob, ProbState* st, int p, const double* prim, T* U, long long ctot) {
  const ProbDev& P = prob[p];
  ProbState& S = st[p];
  long long n = (long long)P.nx * P.ny * P.nz;
  double smax = 0.0;
  double ent = 0.0;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    if (P.is_scalar) {
      double u = prim[c];
      U[P.off + c] = T(u);
      double sp = (P.model == DSPW_LINADV) ? P.lin_speed : fabs(u);
      if (sp > smax) smax = sp;
      const double ut = (double)T(u);
      ent += 0.5 * ut * ut;
    } else {
      double pd[5];
      for (int v = 0; v < 5; v++) pd[v] = prim[v * n + c];
      T pp[5], u[5];
      for (int v = 0; v < 5; v++) pp[v] = T(pd[v]);
      prim_to_cons<T>(pp, T(P.gamma), u);
      store_cons<T>(U, ctot, P.off + c, P.nv, u);
      double sp = wave_speed<double>(P, pd);
      if (sp > smax) smax = sp;
      const T sT = Mth<T>::log(pp[4]) - T(P.gamma) * Mth<T>::log(pp[0]);
      ent += (double)(-pp[0] * sT / T(P.gamma - 1.0));
    }
  }
  unsigned long long sb = (unsigned long long)__double_as_longlong(smax);
  warp_max_u64_lane0(sb);
  const double es = warp_sum(ent);
  if ((threadIdx.x & 31) == 0) {
    const int sl = blockIdx.x & (EPI_SLOTS - 1);
    atomicMax(&S.smax[sl], sb);
    atomicAdd(&S.ent_acc[sl], es);
  }
}

// wave-speed max of the current state (dspw_compute_dt)
template <typename T>
__global__ void k_speed(const ProbDev* prob, ProbState* st, int p, const T* U, long long ctot, double* out) {
  const ProbDev& P = prob[p];
  long long n = (long long)P.nx * P.ny * P.nz;
  double smax = 0.0;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    T pr[5];
    if (P.is_scalar) { pr[0] = U[P.off + c]; pr[1] = pr[2] = pr[3] = pr[4] = T(0); }
    else {
      T u[5];
      load_cons<T>(U, ctot, P.off + c, P.nv, P.dim, u);
      cons_to_prim<T>(u, T(P.gamma), pr);
    }
    double sp = wave_speed<T>(P, pr);
    if (sp > smax) smax = sp;
  }
  unsigned long long sb = (unsigned long long)__double_as_longlong(smax);
  warp_max_u64_lane0(sb);
  if ((threadIdx.x & 31) == 0) atomicMax((unsigned long long*)out, sb);
  (void)st;
}

// conserved / primitive state of one problem to FP64 staging (download)
template <typename T>
__global__ void k_download(const ProbDev* prob, int p, const T* U, long long ctot, double* out, int prim) {
  const ProbDev& P = prob[p];
  long long n = (long long)P.nx * P.ny * P.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    if (P.is_scalar) { out[c] = (double)U[P.off + c]; continue; }
    T u[5];
    load_cons<T>(U, ctot, P.off + c, P.nv, P.dim, u);
    if (prim) {
      T pr[5];
      cons_to_prim<T>(u, T(P.gamma), pr);
      for (int v = 0; v < 5; v++) out[v * n + c] = (double)pr[v];
    } else {
      for (int v = 0; v < 5; v++) out[v * n + c] = (double)u[v];
    }
  }
}

// FP64 sums for dspw_globals: entropy (enflo/src/compute_global.cc:18-28 /
// enflo_scalar/src_scalar/compute_global.cc:12-21), conserved totals, kinetic energy
// Deterministic FP64 reductions.  Each block reduces its threads' values in a
// fixed order (warp shuffles, then the warps in order) and stores one row of K
// partials per block; k_sum_rows combines the rows in a fixed order.  The
// grid of a launch depends only on the cell count and the device, so a state
// gives the same bits on every call, whatever the scheduling.  Slots whose bit
// is set in MAXMASK are maxima (a NaN wins), the others sums.
template <int K, unsigned MAXMASK>
__device__ inline void block_rows_store(double (&v)[K], double* rows) {
  __shared__ double sh[K][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; k++) {
    if ((MAXMASK >> k) & 1u) {
      for (int o = 16; o > 0; o >>= 1) {
        const double x = __shfl_xor_sync(0xffffffffu, v[k], o);
        v[k] = (x != x || x > v[k]) ? x : v[k];
      }
    } else {
      v[k] = warp_sum(v[k]);
    }
    if (lane == 0) sh[k][w] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < K) {
    const int k = threadIdx.x;
    double s = sh[k][0];
    for (int i = 1; i < nw; i++) {
      const double x = sh[k][i];
      s = ((MAXMASK >> k) & 1u) ? ((x != x || x > s) ? x : s) : s + x;
    }
    rows[(long long)blockIdx.x * K + k] = s;
  }
}

// one block of 256 threads: thread t combines rows t, t + 256, ... in order,
// then a fixed pairwise tree; out[k] receives slot k
template <typename T, int K, unsigned MAXMASK>
__global__ void __launch_bounds__(256) k_sum_rows(const double* rows, int nrows, double* out) {
  __shared__ double sh[K][256];
  const int t = threadIdx.x;
#pragma unroll
  for (int k = 0; k < K; k++) {
    const bool mx = (MAXMASK >> k) & 1u;
    double s = 0.0;
    for (int i = t; i < nrows; i += 256) {
      const double x = rows[(long long)i * K + k];
      s = mx ? ((x != x || x > s) ? x : s) : s + x;
    }
    sh[k][t] = s;
  }
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (t < h) {
#pragma unroll
      for (int k = 0; k < K; k++) {
        const double a = sh[k][t], b = sh[k][t + h];
        sh[k][t] = ((MAXMASK >> k) & 1u) ? ((b != b || b > a) ? b : a) : a + b;
      }
    }
    __syncthreads();
  }
  if (t < K) out[t] = sh[t][0];
}

// total entropy, kinetic energy and conserved totals of problem p: one row of
// 7 partials per block (rows), to be combined by k_sum_rows
template <typename T>
__global__ void __launch_bounds__(256) k_globals(const ProbDev* prob, int p, const T* U, long long ctot,
                                                 double* rows /* 7 per block */) {
  const ProbDev& P = prob[p];
  long long n = (long long)P.nx * P.ny * P.nz;
  double v[7] = {0, 0, 0, 0, 0, 0, 0};   // entropy, ke, conserved 0..4
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    if (P.is_scalar) {
      double u = U[P.off + c];
      v[0] += 0.5 * u * u;
      v[2] += u;
    } else {
      T u[5], pr[5];
      load_cons<T>(U, ctot, P.off + c, P.nv, P.dim, u);
      cons_to_prim<T>(u, T(P.gamma), pr);
      double rho = pr[0], prs = pr[4];
      double s = ::log(prs) - P.gamma * ::log(rho);
      v[0] += -rho * s / (P.gamma - 1.0);
      v[1] += 0.5 * rho * ((double)pr[1] * pr[1] + (double)pr[2] * pr[2] + (double)pr[3] * pr[3]);
      for (int k = 0; k < 5; k++) v[2 + k] += (double)u[k];
    }
  }
  block_rows_store<7, 0u>(v, rows);
}

// L1 / L2^2 / Linf of (component comp of the primitive state) - exact: one row
// of 3 partials per block
template <typename T>
__global__ void __launch_bounds__(256) k_errors(const ProbDev* prob, int p, const T* U, long long ctot, int comp,
                                                const double* exact, double* rows /* 3 per block */) {
  const ProbDev& P = prob[p];
  long long n = (long long)P.nx * P.ny * P.nz;
  double v[3] = {0, 0, 0};
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    double x;
    if (P.is_scalar) x = U[P.off + c];
    else {
      T u[5], pr[5];
      load_cons<T>(U, ctot, P.off + c, P.nv, P.dim, u);
      cons_to_prim<T>(u, T(P.gamma), pr);
      x = pr[comp];
    }
    double d = fabs(exact[c] - x);
    v[0] += d; v[1] += d * d;
    v[2] = (d != d || d > v[2]) ? d : v[2];
  }
  block_rows_store<3, 4u>(v, rows);
}

// ---------------------------------------------------- Navier-Stokes (ES) --

// entropy variables of every cell (input of the node stencil)
template <typename T>
__global__ void k_entvars(const ProbDev* prob, int nprob, const long long* cell_start, const T* U, long long ctot,
                          T* Vout) {
  long long total = cell_start[nprob];
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nprob - 1;
    while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (cell_start[mid] <= g) lo = mid; else hi = mid - 1; }
    const ProbDev& P = prob[lo];
    if (P.model != DSPW_NS_ES && P.model != DSPW_NS_KEP) continue;
    T u[5], pr[5], v[5];
    load_cons<T>(U, ctot, g, P.nv, P.dim, u);
    cons_to_prim<T>(u, T(P.gamma), pr);
    if (P.model == DSPW_NS_KEP) {   // the KE viscous flux works on primitive variables
      for (int c = 0; c < 5; c++) Vout[c * ctot + g] = pr[c];
      continue;
    }
    prim_to_ent<T>(pr, T(P.gamma), v);
    for (int c = 0; c < 5; c++) Vout[c * ctot + g] = v[c];
  }
}

// nodal_vlux_ES (enflo/src/vflux_ES.cc:15-151) for the node between cells
// (i..i+1, j..j+1, k..k+1), periodic; writes 15 values (x, y, z fluxes).
// The y flux keeps only its K22,K23 terms and the z flux only K33 because the
// reference overwrites the earlier accumulations.
// nodal_vlux_KE (enflo/src/vflux_KE.cc:15-96) of the node whose lower cell is
// (i, j, k), from the primitive variables P of the 8 cells around it: node
// average and velocity derivatives as nodal_avg_and_vel_derivatives
// (enflo/src/nodal_avg_and_der.cc:16-82, derivative factor 1/(4 dx)), the
// temperature derivatives with the factor 1/4/dx, stresses and heat flux.
template <typename T>
__device__ inline void visc_node_ke(const ProbDev& P, const T* V, long long ctot, T* node, long long g, int i,
                                    int j, int k, int i1, int j1, int k1) {
  typedef Mth<T> m;
#define VC(c, ii, jj, kk) V[(c) * ctot + P.off + ((long long)(kk) * P.ny + (jj)) * P.nx + (ii)]
  const T f1 = T(1.0 / 8.0);
  T avg[5], Tx[3], Ty[3], Tz[3];
#pragma unroll
  for (int c = 0; c < 5; c++) {
    avg[c] = VC(c, i1, j1, k1) * f1 + VC(c, i, j1, k1) * f1 + VC(c, i1, j, k1) * f1 + VC(c, i1, j1, k) * f1;
    avg[c] += VC(c, i, j, k1) * f1 + VC(c, i, j1, k) * f1 + VC(c, i1, j, k) * f1 + VC(c, i, j, k) * f1;
  }
  const T vx = m::div(T(1.0), T(4.0) * T(P.dx)), vy = m::div(T(1.0), T(4.0) * T(P.dy)),
          vz = m::div(T(1.0), T(4.0) * T(P.dz));
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const int v = 1 + c;
    const T v111 = VC(v, i1, j1, k1), v011 = VC(v, i, j1, k1), v101 = VC(v, i1, j, k1), v110 = VC(v, i1, j1, k);
    const T v001 = VC(v, i, j, k1), v010 = VC(v, i, j1, k), v100 = VC(v, i1, j, k), v000 = VC(v, i, j, k);
    Tx[c] = v111 * vx + v110 * vx + v101 * vx + v100 * vx;
    Tx[c] += v011 * -vx + v010 * -vx + v001 * -vx + v000 * -vx;
    Ty[c] = v111 * vy + v110 * vy + v011 * vy + v010 * vy;
    Ty[c] += v101 * -vy + v100 * -vy + v001 * -vy + v000 * -vy;
    Tz[c] = v111 * vz + v101 * vz + v011 * vz + v001 * vz;
    Tz[c] += v110 * -vz + v100 * -vz + v010 * -vz + v000 * -vz;
  }
  const T Rg = T(P.gas_const);
  auto tmp = [&](int ii, int jj, int kk) { return m::div(VC(4, ii, jj, kk), Rg * VC(0, ii, jj, kk)); };
  const T t111 = tmp(i1, j1, k1), t110 = tmp(i1, j1, k), t101 = tmp(i1, j, k1), t100 = tmp(i1, j, k);
  const T t011 = tmp(i, j1, k1), t010 = tmp(i, j1, k), t001 = tmp(i, j, k1), t000 = tmp(i, j, k);
#undef VC
  const double T_avg = (double)avg[4] / (P.gas_const * (double)avg[0]);
  const T mu = T(viscosity(P, T_avg));
  const T kappa = m::div(mu * T(P.Cp), T(P.prandtl));
  const T fx = m::div(T(1.0 / 4.0), T(P.dx)), fy = m::div(T(1.0 / 4.0), T(P.dy)), fz = m::div(T(1.0 / 4.0), T(P.dz));
  const T Tt_x = fx * (t111 + t110 + t101 + t100 - t011 - t010 - t001 - t000);
  const T Tt_y = fy * (t111 + t110 + t011 + t010 - t101 - t100 - t001 - t000);
  const T Tt_z = fz * (t111 + t101 + t011 + t001 - t110 - t100 - t010 - t000);
  const T grad = Tx[0] + Ty[1] + Tz[2];
  const T txx = mu * (T(2) * Tx[0] - T(2.0 / 3.0) * grad);
  const T tyy = mu * (T(2) * Ty[1] - T(2.0 / 3.0) * grad);
  const T tzz = mu * (T(2) * Tz[2] - T(2.0 / 3.0) * grad);
  const T txy = mu * (Ty[0] + Tx[1]);
  const T txz = mu * (Tx[2] + Tz[0]);
  const T tyz = mu * (Ty[2] + Tz[1]);
  T xf[5], yf[5], zf[5];
  xf[0] = T(0); xf[1] = txx; xf[2] = txy; xf[3] = txz;
  xf[4] = (avg[1] * txx + avg[2] * txy + avg[3] * txz) + kappa * Tt_x;
  yf[0] = T(0); yf[1] = txy; yf[2] = tyy; yf[3] = tyz;
  yf[4] = (avg[1] * txy + avg[2] * tyy + avg[3] * tyz) + kappa * Tt_y;
  zf[0] = T(0); zf[1] = txz; zf[2] = tyz; zf[3] = tzz;
  zf[4] = (avg[1] * txz + avg[2] * tyz + avg[3] * tzz) + kappa * Tt_z;
  const T ax = -(T(P.dy) * T(P.dz)), ay = -(T(P.dx) * T(P.dz)), az = -(T(P.dx) * T(P.dy));
#pragma unroll
  for (int c = 0; c < 5; c++) {
    node[(0 + c) * ctot + g] = xf[c] * ax;
    node[(5 + c) * ctot + g] = yf[c] * ay;
    node[(10 + c) * ctot + g] = zf[c] * az;
  }
}

// (i, j, k) of cell l of a problem (x fastest): 32-bit divisions when the
// problem has fewer than 2^32 cells (every problem that fits in memory)
DSPW_HD void cell_ijk(const ProbDev& P, long long l, int& i, int& j, int& k) {
  const long long nxy = (long long)P.nx * P.ny;
  if (nxy * P.nz <= 0xffffffffLL) {
    const unsigned u = (unsigned)l, nx = (unsigned)P.nx, n2 = (unsigned)nxy;
    const unsigned kk = u / n2, r = u - kk * n2, jj = r / nx;
    i = (int)(r - jj * nx); j = (int)jj; k = (int)kk;
  } else {
    i = (int)(l % P.nx); j = (int)((l / P.nx) % P.ny); k = (int)(l / nxy);
  }
}

template <typename T>
__global__ void k_visc_nodes(const ProbDev* prob, int nprob, const long long* cell_start, const T* V, long long ctot,
                             T* node) {
  typedef Mth<T> m;
  long long total = cell_start[nprob];
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nprob - 1;
    while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (cell_start[mid] <= g) lo = mid; else hi = mid - 1; }
    const ProbDev& P = prob[lo];
    if (P.model != DSPW_NS_ES && P.model != DSPW_NS_KEP) continue;
    int i, j, k;
    cell_ijk(P, g - P.off, i, j, k);
    const int i1 = i + 1 == P.nx ? 0 : i + 1, j1 = j + 1 == P.ny ? 0 : j + 1, k1 = k + 1 == P.nz ? 0 : k + 1;
    if (P.model == DSPW_NS_KEP) {
      visc_node_ke<T>(P, V, ctot, node, g, i, j, k, i1, j1, k1);
      continue;
    }
#define VC(c, ii, jj, kk) V[(c) * ctot + P.off + ((long long)(kk) * P.ny + (jj)) * P.nx + (ii)]
    const T f1 = T(1.0 / 8.0);
    const T fx = m::div(T(1.0 / 4.0), T(P.dx)), fy = m::div(T(1.0 / 4.0), T(P.dy)), fz = m::div(T(1.0 / 4.0), T(P.dz));
    T avg[5], Tx[5], Ty[5], Tz[5];
#pragma unroll
    for (int c = 0; c < 5; c++) {
      T v111 = VC(c, i1, j1, k1), v011 = VC(c, i, j1, k1), v101 = VC(c, i1, j, k1), v110 = VC(c, i1, j1, k);
      T v001 = VC(c, i, j, k1), v010 = VC(c, i, j1, k), v100 = VC(c, i1, j, k), v000 = VC(c, i, j, k);
      avg[c] = v111 * f1 + v011 * f1 + v101 * f1 + v110 * f1;
      avg[c] += v001 * f1 + v010 * f1 + v100 * f1 + v000 * f1;
      Tx[c] = v111 * fx + v110 * fx + v101 * fx + v100 * fx;
      Tx[c] += v011 * -fx + v010 * -fx + v001 * -fx + v000 * -fx;
      Ty[c] = v111 * fy + v110 * fy + v011 * fy + v010 * fy;
      Ty[c] += v101 * -fy + v100 * -fy + v001 * -fy + v000 * -fy;
      Tz[c] = v111 * fz + v101 * fz + v011 * fz + v001 * fz;
      Tz[c] += v110 * -fz + v100 * -fz + v010 * -fz + v000 * -fz;
    }
#undef VC
    double Td = -1 / (double)avg[4] / P.gas_const;
    T mu = T(viscosity(P, Td));
    T kappa = m::div(mu * T(P.Cp), T(P.prandtl));
    T c1 = m::div(T(4.0) * mu, T(3.0)), c2 = m::div(T(-2.0) * mu, T(3.0)), c3 = m::div(kappa, T(P.gas_const));
    T e4 = m::div(T(1.0), avg[4]);
    T e1 = avg[1] * e4, e2 = avg[2] * e4, e3 = avg[3] * e4;
    T xf[5], yf[5], zf[5];
    xf[0] = T(0.0);
    xf[1] = c1 * e4 * (-Tx[1] + e1 * Tx[4]);
    xf[2] = mu * e4 * (-Tx[2] + e2 * Tx[4]);
    xf[3] = mu * e4 * (-Tx[3] + e3 * Tx[4]);
    xf[4] = e4 * (c1 * e1 * Tx[1] + mu * e2 * Tx[2] + mu * e3 * Tx[3] +
                  (-c1 * e1 * e1 - mu * (e2 * e2 + e3 * e3) + c3 * e4) * Tx[4]);
    xf[1] += c2 * e4 * (-Ty[2] + e2 * Ty[4]);
    xf[2] += mu * e4 * (-Ty[1] + e1 * Ty[4]);
    xf[4] += e4 * (mu * e2 * Ty[1] + c2 * e1 * Ty[2] - (mu + c2) * e1 * e2 * Ty[4]);
    xf[1] += c2 * e4 * (-Tz[3] + e3 * Tz[4]);
    xf[3] += mu * e4 * (-Tz[1] + e1 * Tz[4]);
    xf[4] += e4 * (mu * e3 * Tz[1] + c2 * e1 * Tz[3] - (mu + c2) * e1 * e3 * Tz[4]);
    yf[0] = T(0.0);
    yf[1] = mu * e4 * (-Ty[1] + e1 * Ty[4]);
    yf[2] = c1 * e4 * (-Ty[2] + e2 * Ty[4]);
    yf[3] = mu * e4 * (-Ty[3] + e3 * Ty[4]);
    yf[4] = e4 * (mu * e1 * Ty[1] + c1 * e2 * Ty[2] + mu * e3 * Ty[3] +
                  (-c1 * e2 * e2 - mu * (e1 * e1 + e3 * e3) + c3 * e4) * Ty[4]);
    yf[2] += c2 * e4 * (-Tz[3] + e3 * Tz[4]);
    yf[3] += mu * e4 * (-Tz[2] + e2 * Tz[4]);
    yf[4] += e4 * (mu * e3 * Tz[2] + c2 * e2 * Tz[3] - (mu + c2) * e2 * e3 * Tz[4]);
    zf[0] = T(0.0);
    zf[1] = mu * e4 * (-Tz[1] + e1 * Tz[4]);
    zf[2] = mu * e4 * (-Tz[2] + e2 * Tz[4]);
    zf[3] = c1 * e4 * (-Tz[3] + e3 * Tz[4]);
    zf[4] = e4 * (mu * e1 * Tz[1] + mu * e2 * Tz[2] + c1 * e3 * Tz[3] +
                  (-c1 * e3 * e3 - mu * (e1 * e1 + e2 * e2) + c3 * e4) * Tz[4]);
    T ax = -(T(P.dy) * T(P.dz)), ay = -(T(P.dx) * T(P.dz)), az = -(T(P.dx) * T(P.dy));
#pragma unroll
    for (int c = 0; c < 5; c++) {
      node[(0 + c) * ctot + g] = xf[c] * ax;
      node[(5 + c) * ctot + g] = yf[c] * ay;
      node[(10 + c) * ctot + g] = zf[c] * az;
    }
  }
}

// Add the viscous residual of each cell from its 8 corner nodes (scatter of
// compute_visc_residual, enflo/src/fv.cc:786-1157, as a gather) and apply the
// stage update.  Nodes at a domain edge (two coordinates on the boundary
// node layer) are counted twice, as the reference's loops visit them twice.
template <typename T>
__global__ void k_visc_update(SweepArgs<T> A, const long long* cell_start, const T* node) {
  long long total = cell_start[A.nprob];
  double smax = 0.0;
  double ent = 0.0;
  unsigned bad_fin = 0, bad_pos = 0;
  int pcur = -1;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = A.nprob - 1;
    while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (cell_start[mid] <= g) lo = mid; else hi = mid - 1; }
    const ProbDev& P = A.prob[lo];
    if (P.model != DSPW_NS_ES && P.model != DSPW_NS_KEP) continue;
    ProbState& S = A.st[lo];
    if (!A.residual_only && !S.active) continue;
    pcur = lo;
    int I, J, K;
    cell_ijk(P, g - P.off, I, J, K);
    T R[5];
    load_cons<T>(A.R, A.ctot, g, P.nv, P.dim, R);
#pragma unroll
    for (int a = 1; a >= 0; a--)
#pragma unroll
      for (int b = 1; b >= 0; b--)
#pragma unroll
        for (int c = 1; c >= 0; c--) {
          // node position relative to the cell: i = I - 1 + a (a = 1: right node)
          int ni = I - 1 + a, nj = J - 1 + b, nk = K - 1 + c;
          int onb = (ni == -1 || ni == P.nx - 1) + (nj == -1 || nj == P.ny - 1) + (nk == -1 || nk == P.nz - 1);
          int mult = (onb == 2) ? 2 : 1;
          // periodic node index (ni in -1 .. nx-1)
          const int pi = ni < 0 ? ni + P.nx : ni, pj = nj < 0 ? nj + P.ny : nj, pk = nk < 0 ? nk + P.nz : nk;
          long long ng = P.off + ((long long)pk * P.ny + pj) * P.nx + pi;
          const T cx = a ? T(0.25) : T(-0.25), cy = b ? T(0.25) : T(-0.25), cz = c ? T(0.25) : T(-0.25);
          for (int rep = 0; rep < mult; rep++) {
#pragma unroll
            for (int v = 0; v < 5; v++)
              R[v] += node[v * A.ctot + ng] * cx + node[(5 + v) * A.ctot + ng] * cy + node[(10 + v) * A.ctot + ng] * cz;
          }
        }
    if (A.residual_only) { store_cons<T>(A.R, A.ctot, g, P.nv, R); continue; }
    T u[5], un[5];
    load_cons<T>(A.Uin, A.ctot, g, P.nv, P.dim, u);
    load_cons<T>(A.Un, A.ctot, g, P.nv, P.dim, un);
    stage_combine<T>(A, P, S, g, R, u, un);
    store_cons<T>(A.Uout, A.ctot, g, P.nv, u);
    if (A.store_R && A.final_stage) store_cons<T>(A.R, A.ctot, g, P.nv, R);
    if (A.final_stage) {
      T p[5];
      cons_to_prim<T>(u, T(P.gamma), p);
      double sp = wave_speed<T>(P, p);
      if (sp > smax) smax = sp;
      double rho = p[0], pr = p[4];
      if (!(rho > 0.0) || !(pr > 0.0)) bad_pos++;
      if (!isfinite(rho) || !isfinite(pr)) bad_fin++;
      const T sT = Mth<T>::log(p[4]) - T(P.gamma) * Mth<T>::log(p[0]);
      ent += (double)(-p[0] * sT / T(P.gamma - 1.0));
    }
  }
  // one speed-max and entropy flush per thread, warp-aggregated when the warp
  // worked on a single problem
  int p0 = __shfl_sync(0xffffffffu, pcur, 0);
  bool uniform = __all_sync(0xffffffffu, pcur == p0 || pcur < 0);
  if (A.final_stage && !A.residual_only) {
    if (uniform) {
      unsigned long long sb = (unsigned long long)__double_as_longlong(smax);
      warp_max_u64_lane0(sb);
      const double es = warp_sum(ent);
      if ((threadIdx.x & 31) == 0 && p0 >= 0) {
        const int sl = blockIdx.x & (EPI_SLOTS - 1);
        atomicMax(&A.st[p0].smax[sl], sb);
        atomicAdd(&A.st[p0].ent_acc[sl], es);
      }
    } else if (pcur >= 0) {
      const int sl = blockIdx.x & (EPI_SLOTS - 1);
      atomicMax(&A.st[pcur].smax[sl], (unsigned long long)__double_as_longlong(smax));
      atomicAdd(&A.st[pcur].ent_acc[sl], ent);
    }
  }
  if (bad_fin) { atomicAdd(&A.status->nonfinite, (unsigned long long)bad_fin); atomicCAS(&A.status->code, 0, DSPW_ERR_NONFINITE); }
  if (bad_pos) { atomicAdd(&A.status->nonpositive, (unsigned long long)bad_pos); atomicCAS(&A.status->code, 0, DSPW_ERR_NONPOSITIVE); }
}

// Reconstruction of a batch of independent 4-cell stencils with the same
// device code as the sweeps (SP-WENO family or DSP-WENO, FP64 or FP32 with the
// BF16 tensor-core network).  Used to check the reconstruction face by face.
template <typename T>
__global__ void __launch_bounds__(WARPS_PER_BLOCK * 32)
k_recon_batch(const ProbDev* prob, const NetParams* net, const double* u4, long long n, double* l, double* r,
              unsigned long long* acts) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSmem<T>* sm = reinterpret_cast<WarpSmem<T>*>(smem_raw) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  net_frag_stage<T>(*net, lane, sm->ns);
  const long long nchunk = (n + 31) / 32;
  for (long long ch = blockIdx.x * (long long)WARPS_PER_BLOCK + (threadIdx.x >> 5); ch < nchunk;
       ch += (long long)gridDim.x * WARPS_PER_BLOCK) {
    long long i = ch * 32 + lane;
    bool valid = i < n;
    T s0 = valid ? T(u4[4 * i]) : T(0), s1 = valid ? T(u4[4 * i + 1]) : T(1);
    T s2 = valid ? T(u4[4 * i + 2]) : T(2), s3 = valid ? T(u4[4 * i + 3]) : T(3);
    T lo = T(0), ro = T(0);
    int viol = 0;
    unsigned long long signv = 0;   // not reported by this entry point
    reconstruct_lane<T, SpecGeneric>(*prob, *net, sm, lane, valid, s0, s1, s2, s3, lo, ro, viol, signv);
    if (valid) { l[i] = (double)lo; r[i] = (double)ro; }
    unsigned v = __reduce_add_sync(0xffffffffu, (unsigned)viol);
    if (lane == 0 && v) atomicAdd(acts, (unsigned long long)v);
  }
}

}  // namespace dspw

// dspw_diag.cuh -- per-step global diagnostics on the device: the quantities
// the reference's FV::run computes and writes every step, without copying the
// state to the host.
//
//   systems (enflo/src/fv.cc:1276-1307): at stage 0, of U^n at t^n
//     total entropy  sum -rho s / (gamma - 1) * vol      compute_global.cc:18-28,63
//     KE             sum rho |u|^2 * (vol / 2)           compute_global.cc:26,64
//     KE_diss_pr     -sum (|u|^2/2 R_mass + u.R_mom)     fv.cc:756-764 (inviscid residual)
//     KE_diss_stress -sum_nodes (Tx.F_x dx + ..) w       fv.cc:810-814 (NS, viscous node fluxes)
//     enstrophy      sum_nodes rho_avg |curl u|^2 w * (nodal_volume / 2)
//                                                        compute_global.cc:33-65, find_vort.cc:18-28
//   and after the step the residual norm of its last stage, per component
//     sqrt(sum (R / vol)^2) * vol                        fv.cc:1204-1226
//   scalar (enflo_scalar/src_scalar/fv.cc:572-576): after the step, of U^(n+1)
//     total entropy  sum u^2 / 2 * vol, residual norm sqrt(sum R^2)
//
// Every sum is deterministic: each block covers a fixed contiguous range of
// cells (or nodes) and reduces, in a fixed order, one row of partial sums per
// problem it overlaps; a fold kernel adds a problem's rows in block order to
// its FP64 accumulator; a row kernel turns the accumulators into one row per
// problem and step in a device ring that the host drains.  The same state
// gives the same bits on every run.  The summation order differs from the
// reference's sequential loops, so the values agree with the reference's to
// rounding (about 1e-13 relative for FP64 states), not bit for bit.
#pragma once
#include "dspw_kernels.cuh"

namespace dspw {

enum { DIAG_COLS = 12, DIAG_NACC = 10 };
// accumulator slots
enum { DA_ENT = 0, DA_KE = 1, DA_KDP = 2, DA_KDS = 3, DA_ENS = 4, DA_RES = 5 /* 5..9 */ };

struct DiagAcc {
  double v[DIAG_NACC];
  unsigned long long count;   // rows written since the ring was created
  unsigned long long pad;
};

template <typename T>
struct DiagArgs {
  const ProbDev* prob;
  const ProbState* st;
  DiagAcc* acc;
  int nprob;
  const long long* start;   // per problem prefix of cells (k_diag_cells) or nodes (k_diag_nodes)
  const T* U;               // U^n at stage 0, U^(n+1) after the last stage
  const T* R;               // stage-0 inviscid residual, or the last stage's residual
  const T* node;            // stage-0 viscous node fluxes (NS), 15 planes
  long long ctot;
  double* rows;             // ring, slot-major: rows[(slot * nprob + p) * DIAG_COLS]
  int cap;
  // partial sums of one launch, one row of DIAG_NACC per (block b, problem p)
  // the block overlaps, at row b + p (a block's problems are consecutive, so
  // b + p is different for every overlapping pair): (blocks + nprob) rows
  double* part;
};

DSPW_HD int find_problem_ll(const long long* start, int nprob, long long g) {
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// block-wide sum of v[k] in a fixed order (warp shuffles, then the warps in
// order); every thread calls it, thread 0 receives the totals
__device__ inline void block_sum_fixed(double (&v)[DIAG_NACC]) {
  __shared__ double red[DIAG_NACC][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < DIAG_NACC; k++) {
    double s = warp_sum(v[k]);
    if (lane == 0) red[k][warp] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < DIAG_NACC; k++) {
      double s = red[k][0];
      for (int w = 1; w < nw; w++) s += red[k][w];
      v[k] = s;
    }
  }
  __syncthreads();
}

// row b + p of the partial sums: the block total of v (every thread calls it)
__device__ inline void block_store(double (&v)[DIAG_NACC], double* part, int p) {
  block_sum_fixed(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < DIAG_NACC; k++) part[((long long)blockIdx.x + p) * DIAG_NACC + k] = v[k];
  }
}

// the block-contiguous range of block b of a launch of `nblocks` blocks over
// [0, total): tiles of 256 items
DSPW_HD long long diag_chunk(long long total, int nblocks) {
  const long long per = (total + nblocks - 1) / nblocks;
  return ((per + 255) / 256) * 256;
}

// Walk block b's range of the flat index space [0, start[nprob]) in tiles of
// blockDim.x (256); terms(p, g, t) fills the accumulator terms of item g of
// problem p.  The items of one problem accumulate per thread while the tiles
// stay inside it; a tile that straddles problems is split by problem with
// fixed-order block sums.  Every (block, problem) overlap ends in exactly one
// row of partial sums (block_store), zeros included.
template <typename F>
__device__ inline void block_range_sums(const long long* start, int nprob, double* part, F terms) {
  const long long total = start[nprob];
  const long long chunk = diag_chunk(total, gridDim.x);
  const long long begin = (long long)blockIdx.x * chunk;
  const long long end = begin + chunk < total ? begin + chunk : total;
  __shared__ int s_p0, s_pmax;
  int pend = -1;
  double sum[DIAG_NACC];
#pragma unroll
  for (int k = 0; k < DIAG_NACC; k++) sum[k] = 0.0;
  for (long long base = begin; base < end; base += blockDim.x) {
    const long long g = base + threadIdx.x;
    int p = -1;
    double t[DIAG_NACC];
#pragma unroll
    for (int k = 0; k < DIAG_NACC; k++) t[k] = 0.0;
    if (g < end) {
      p = find_problem_ll(start, nprob, g);
      terms(p, g, t);
    }
    if (threadIdx.x == 0) s_p0 = p;
    // the last valid item of the tile has the largest problem
    const long long glast = (base + blockDim.x < end ? base + blockDim.x : end) - 1;
    if (threadIdx.x == (int)(glast - base)) s_pmax = p;
    __syncthreads();
    const int p0 = s_p0, pmax = s_pmax;
    __syncthreads();
    if (p0 == pmax) {   // the tile lies in one problem
      if (p0 != pend) {
        if (pend >= 0) {
          block_store(sum, part, pend);
#pragma unroll
          for (int k = 0; k < DIAG_NACC; k++) sum[k] = 0.0;
        }
        pend = p0;
      }
#pragma unroll
      for (int k = 0; k < DIAG_NACC; k++) sum[k] += t[k];
    } else {
      // problems p0 < ... < pmax (every one of them has items here): all but
      // the last end in this tile.  A pending run of an earlier problem ended
      // with the previous tile.
      if (pend >= 0 && pend != p0) {
        block_store(sum, part, pend);
#pragma unroll
        for (int k = 0; k < DIAG_NACC; k++) sum[k] = 0.0;
        pend = -1;
      }
      for (int q = p0; q <= pmax; q++) {
        double v[DIAG_NACC];
#pragma unroll
        for (int k = 0; k < DIAG_NACC; k++) v[k] = (q == pend ? sum[k] : 0.0) + (p == q ? t[k] : 0.0);
        if (q < pmax) {
          block_store(v, part, q);
        } else {
          // the last problem of the tile stays pending: its per-thread sums
#pragma unroll
          for (int k = 0; k < DIAG_NACC; k++) sum[k] = v[k];
        }
      }
      pend = pmax;
    }
  }
  if (pend >= 0) block_store(sum, part, pend);
}

// fold the partial rows of one launch into each problem's accumulator in a
// fixed order: one block of 256 threads per problem, thread t adds rows
// b0 + t, b0 + t + 256, ..., then the block's fixed-order sum
template <typename T>
__global__ void __launch_bounds__(256) k_diag_fold(const long long* start, int nprob, const double* part, int nblocks,
                                                   DiagAcc* acc) {
  const int p = blockIdx.x;
  if (p >= nprob) return;
  const long long total = start[nprob];
  const long long chunk = diag_chunk(total, nblocks);
  if (start[p + 1] <= start[p]) return;   // block-uniform
  const int b0 = (int)(start[p] / chunk), b1 = (int)((start[p + 1] - 1) / chunk);
  double s[DIAG_NACC];
#pragma unroll
  for (int k = 0; k < DIAG_NACC; k++) s[k] = 0.0;
  for (int b = b0 + (int)threadIdx.x; b <= b1; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < DIAG_NACC; k++) s[k] += part[((long long)b + p) * DIAG_NACC + k];
  block_sum_fixed(s);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < DIAG_NACC; k++) acc[p].v[k] += s[k];
  }
}

// mode 0 (stage 0, systems): entropy, KE and pressure-work KE dissipation of
// U^n with its inviscid residual.  mode 1 (after the last stage, every
// problem): residual norms; scalar energy of U^(n+1).
template <typename T>
__global__ void __launch_bounds__(256) k_diag_cells(DiagArgs<T> A, int mode) {
  block_range_sums(A.start, A.nprob, A.part, [&](int p, long long g, double* t) {
    const ProbDev& P = A.prob[p];
    if (!A.st[p].active) return;
    if (P.is_scalar) {
      if (mode != 1) return;
      const double r = (double)A.R[g], u = (double)A.U[g];
      t[DA_RES] = r * r;
      t[DA_ENT] = 0.5 * (u * u);
      return;
    }
    T uT[5], rT[5];
    if (mode == 1) {
      load_cons<T>(A.R, A.ctot, g, P.nv, P.dim, rT);
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const double x = (double)rT[v] / P.dx / P.dy / P.dz;
        t[DA_RES + v] = x * x;
      }
      return;
    }
    load_cons<T>(A.U, A.ctot, g, P.nv, P.dim, uT);
    load_cons<T>(A.R, A.ctot, g, P.nv, P.dim, rT);
    double u[5], pr[5];
#pragma unroll
    for (int v = 0; v < 5; v++) u[v] = (double)uT[v];
    cons_to_prim<double>(u, P.gamma, pr);
    const double vsq = pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3];
    const double s = ::log(pr[4]) - P.gamma * ::log(pr[0]);
    t[DA_ENT] = -pr[0] * s / (P.gamma - 1.0);
    t[DA_KE] = pr[0] * vsq;
    t[DA_KDP] = -(0.5 * vsq * (double)rT[0] +
                  (pr[1] * (double)rT[1] + pr[2] * (double)rT[2] + pr[3] * (double)rT[3]));
  });
}

// primitive state of cell (ci, cj, ck), each in -1 .. N, with the reference's
// ghost cells: one coordinate outside -> that face's boundary condition
// (periodic copy, wall mirror with the normal velocity negated, neumann copy of
// the first interior cell, dirichlet state); two or three outside -> periodic
// wrap of all of them (the edge and corner fill, enflo/src/fv.cc:317-358)
template <typename T>
__device__ inline void ghost_prim(const DiagArgs<T>& A, const ProbDev& P, int ci, int cj, int ck, double p[5]) {
  const int N[3] = {P.nx, P.ny, P.nz};
  int c[3] = {ci, cj, ck};
  int out = 0, axis = -1;
#pragma unroll
  for (int a = 0; a < 3; a++)
    if (c[a] < 0 || c[a] >= N[a]) { out++; axis = a; }
  int flip = -1;
  if (out >= 2) {
#pragma unroll
    for (int a = 0; a < 3; a++) c[a] = (c[a] + N[a]) % N[a];
  } else if (out == 1) {
    const int face = 2 * axis + (c[axis] < 0 ? 0 : 1);
    const int kind = P.bc[face];
    if (kind == DSPW_BC_DIRICHLET) {
#pragma unroll
      for (int v = 0; v < 5; v++) p[v] = P.bc_state[face][v];
      return;
    }
    int f = 0;
    c[axis] = ghost_source(c[axis], N[axis], kind, f);
    if (f) flip = axis;
  }
  const long long g = P.off + ((long long)c[2] * P.ny + c[1]) * P.nx + c[0];
  T uT[5];
  load_cons<T>(A.U, A.ctot, g, P.nv, P.dim, uT);
  double u[5];
#pragma unroll
  for (int v = 0; v < 5; v++) u[v] = (double)uT[v];
  cons_to_prim<double>(u, P.gamma, p);
  if (flip >= 0) p[1 + flip] = -p[1 + flip];
}

// node weight of find_node_weights (enflo/src/find_node_weights.cc:19-66)
DSPW_HD double node_weight(const ProbDev& P, int a, int b, int c) {
  double w = 1.0;
  if (a == 0 && P.bc[0] == DSPW_BC_PERIODIC) w /= 2.0;
  if (a == P.nx && P.bc[1] == DSPW_BC_PERIODIC) w /= 2.0;
  if (b == 0 && P.bc[2] == DSPW_BC_PERIODIC) w /= 2.0;
  if (b == P.ny && P.bc[3] == DSPW_BC_PERIODIC) w /= 2.0;
  if (c == 0 && P.bc[4] == DSPW_BC_PERIODIC) w /= 2.0;
  if (c == P.nz && P.bc[5] == DSPW_BC_PERIODIC) w /= 2.0;
  return w;
}

// the 8 cells around node (a, b, c) (a in 0..Nx: between cells a-1 and a):
// density average in compute_global's order and the velocity derivatives of
// nodal_avg_and_vel_derivatives (enflo/src/nodal_avg_and_der.cc:37-81)
template <typename T>
__device__ inline void node_state(const DiagArgs<T>& A, const ProbDev& P, int a, int b, int c, double& den,
                                  double Tx[3], double Ty[3], double Tz[3]) {
  double rho[8], vel[8][3];   // index 4*dk + 2*dj + di, d = 1: cell a (b, c), 0: cell a-1
#pragma unroll
  for (int q = 0; q < 8; q++) {
    double p[5];
    ghost_prim<T>(A, P, a - 1 + (q & 1), b - 1 + ((q >> 1) & 1), c - 1 + (q >> 2), p);
    rho[q] = p[0];
    vel[q][0] = p[1]; vel[q][1] = p[2]; vel[q][2] = p[3];
  }
#define Q(i, j, k) ((k) * 4 + (j) * 2 + (i))
  den = (1.0 / 8.0) * (rho[Q(0, 0, 0)] + rho[Q(1, 0, 0)] + rho[Q(0, 1, 0)] + rho[Q(0, 0, 1)] + rho[Q(1, 1, 0)] +
                       rho[Q(1, 0, 1)] + rho[Q(0, 1, 1)] + rho[Q(1, 1, 1)]);
  const double vx = 1.0 / (4.0 * P.dx), vy = 1.0 / (4.0 * P.dy), vz = 1.0 / (4.0 * P.dz);
#pragma unroll
  for (int v = 0; v < 3; v++) {
    Tx[v] = vel[Q(1, 1, 1)][v] * vx + vel[Q(1, 1, 0)][v] * vx + vel[Q(1, 0, 1)][v] * vx + vel[Q(1, 0, 0)][v] * vx;
    Tx[v] += vel[Q(0, 1, 1)][v] * -vx + vel[Q(0, 1, 0)][v] * -vx + vel[Q(0, 0, 1)][v] * -vx + vel[Q(0, 0, 0)][v] * -vx;
    Ty[v] = vel[Q(1, 1, 1)][v] * vy + vel[Q(1, 1, 0)][v] * vy + vel[Q(0, 1, 1)][v] * vy + vel[Q(0, 1, 0)][v] * vy;
    Ty[v] += vel[Q(1, 0, 1)][v] * -vy + vel[Q(1, 0, 0)][v] * -vy + vel[Q(0, 0, 1)][v] * -vy + vel[Q(0, 0, 0)][v] * -vy;
    Tz[v] = vel[Q(1, 1, 1)][v] * vz + vel[Q(1, 0, 1)][v] * vz + vel[Q(0, 1, 1)][v] * vz + vel[Q(0, 0, 1)][v] * vz;
    Tz[v] += vel[Q(1, 1, 0)][v] * -vz + vel[Q(1, 0, 0)][v] * -vz + vel[Q(0, 1, 0)][v] * -vz + vel[Q(0, 0, 0)][v] * -vz;
  }
#undef Q
}

// enstrophy (every system) and viscous-stress KE dissipation (NS) over the
// (Nx+1)(Ny+1)(Nz+1) nodes of each problem, of U^n at stage 0
template <typename T>
__global__ void __launch_bounds__(256) k_diag_nodes(DiagArgs<T> A) {
  block_range_sums(A.start, A.nprob, A.part, [&](int p, long long g, double* t) {
    const ProbDev& P = A.prob[p];
    if (!A.st[p].active || P.is_scalar) return;
    const long long l = g - A.start[p];
    const int a = (int)(l % (P.nx + 1)), b = (int)((l / (P.nx + 1)) % (P.ny + 1));
    const int c = (int)(l / ((long long)(P.nx + 1) * (P.ny + 1)));
    double den, Tx[3], Ty[3], Tz[3];
    node_state<T>(A, P, a, b, c, den, Tx, Ty, Tz);
    const double w = node_weight(P, a, b, c);
    const double wx = Ty[2] - Tz[1], wy = Tz[0] - Tx[2], wz = Tx[1] - Ty[0];
    t[DA_ENS] = den * (wx * wx + wy * wy + wz * wz) * w;
    if (P.model != DSPW_NS_ES && P.model != DSPW_NS_KEP) return;
    // the node flux of reference node (a-1, b-1, c-1): periodic node index of
    // the viscous kernels; edge nodes are visited twice by the reference
    const int pa = (a - 1 + P.nx) % P.nx, pb = (b - 1 + P.ny) % P.ny, pc = (c - 1 + P.nz) % P.nz;
    const long long ng = P.off + ((long long)pc * P.ny + pb) * P.nx + pa;
    const int onb = (a == 0 || a == P.nx) + (b == 0 || b == P.ny) + (c == 0 || c == P.nz);
    double wt = w;
    // corners (0,N,N) and (N,N,N) take derivatives and weight at j = Nz
    // (enflo/src/fv.cc:1141-1150); the same node when Ny == Nz
    if (onb == 3 && b == P.ny && c == P.nz && P.nz < P.ny) {
      node_state<T>(A, P, a, P.nz, P.nz, den, Tx, Ty, Tz);
      wt = node_weight(P, a, P.nz, P.nz);
    }
    double f[3][3];
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
      for (int v = 0; v < 3; v++) f[d][v] = (double)A.node[(5 * d + 1 + v) * A.ctot + ng];
    const double term = (Tx[0] * f[0][0] + Tx[1] * f[0][1] + Tx[2] * f[0][2]) * P.dx +
                        (Ty[0] * f[1][0] + Ty[1] * f[1][1] + Ty[2] * f[1][2]) * P.dy +
                        (Tz[0] * f[2][0] + Tz[1] * f[2][1] + Tz[2] * f[2][2]) * P.dz;
    t[DA_KDS] = -(term * wt) * (onb == 2 ? 2.0 : 1.0);
  });
}

// one row per active problem from its accumulators, then reset them; runs
// after the last stage and before the end-of-step kernel (time and iter are
// still t^n, n)
template <typename T>
__global__ void k_diag_row(DiagArgs<T> A) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= A.nprob) return;
  const ProbState& S = A.st[p];
  if (!S.active) return;
  const ProbDev& P = A.prob[p];
  DiagAcc& acc = A.acc[p];
  double* row = A.rows + ((acc.count % (unsigned long long)A.cap) * A.nprob + p) * DIAG_COLS;
  for (int c = 0; c < DIAG_COLS; c++) row[c] = 0.0;
  if (P.is_scalar) {
    row[0] = S.iter + 1;
    row[1] = S.time + S.dt;
    row[2] = acc.v[DA_ENT] * P.vol;
    row[7] = ::sqrt(acc.v[DA_RES]);
  } else {
    row[0] = S.iter;
    row[1] = S.time;
    row[2] = acc.v[DA_ENT] * P.vol;
    row[3] = acc.v[DA_KE] * (0.5 * P.vol);
    row[4] = acc.v[DA_KDP];
    row[5] = acc.v[DA_KDS];
    row[6] = acc.v[DA_ENS] * (0.5 * P.node_vol);
    for (int v = 0; v < 5; v++) row[7 + v] = ::sqrt(acc.v[DA_RES + v]) * P.vol;
  }
  for (int k = 0; k < DIAG_NACC; k++) acc.v[k] = 0.0;
  acc.count += 1;
}

}  // namespace dspw

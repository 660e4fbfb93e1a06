// dspw_launch.h -- host-side launch interface shared by the precision units
// (dspw_fp64.cu, dspw_fp32.cu) and the C ABI (dspw_capi.cu).
#pragma once
#include <cuda_runtime.h>
#include "dspw_kernels.cuh"
#include "dspw_diag.cuh"
#include "dspw_snap.cuh"

namespace dspw {

template <typename T>
struct Launch {
  static size_t sweep_smem();
  static cudaError_t prepare();   // kernel attributes; call outside stream capture
  // spec: 0 for the generic kernel, spec_code(dim, rec) for a SpecHot kernel
  static cudaError_t sweep(int dir, const SweepArgs<T>& a, int grid, cudaStream_t s, int spec);
  // resident blocks per SM of that sweep kernel (occupancy calculator)
  // narrow: the 4-column tiles of k_sweep_narrow (specialised y / z sweeps)
  static int sweep_blocks_per_sm(int dir, int spec, int narrow = 0);
  static cudaError_t upload(const ProbDev* prob, ProbState* st, int p, const double* prim, T* U, long long ctot,
                            long long ncell, cudaStream_t s);
  static cudaError_t speed(const ProbDev* prob, ProbState* st, int p, const T* U, long long ctot, long long ncell,
                           double* out, cudaStream_t s);
  static cudaError_t download(const ProbDev* prob, int p, const T* U, long long ctot, long long ncell, double* out,
                              int prim, cudaStream_t s);
  // deterministic FP64 sums: block partials in rows (reduce_rows_max() x 8
  // doubles), combined in a fixed order into acc
  static cudaError_t globals(const ProbDev* prob, int p, const T* U, long long ctot, long long ncell, double* rows,
                             double* acc, cudaStream_t s);
  static cudaError_t errors(const ProbDev* prob, int p, const T* U, long long ctot, long long ncell, int comp,
                            const double* exact, double* rows, double* acc, cudaStream_t s);
  static cudaError_t entvars(const ProbDev* prob, int nprob, const long long* cell_start, long long ncell_total,
                             const T* U, long long ctot, T* V, cudaStream_t s);
  static cudaError_t visc_nodes(const ProbDev* prob, int nprob, const long long* cell_start, long long ncell_total,
                                const T* V, long long ctot, T* node, cudaStream_t s);
  static cudaError_t recon_batch(const ProbDev* prob, const NetParams* net, const double* u4, long long n, double* l,
                                 double* r, unsigned long long* acts, cudaStream_t s);
  static cudaError_t visc_update(const SweepArgs<T>& a, const long long* cell_start, long long ncell_total,
                                 const T* node, cudaStream_t s);
  // per-step diagnostics: cell sums (mode 0 at stage 0, mode 1 after the last
  // stage) over `total` cells, node sums over `total` nodes, the row kernel
  static cudaError_t diag_cells(const DiagArgs<T>& a, int mode, long long total, cudaStream_t s);
  static cudaError_t diag_nodes(const DiagArgs<T>& a, long long total, cudaStream_t s);
  static cudaError_t diag_row(const DiagArgs<T>& a, cudaStream_t s);
  // snapshot of the problems that ended the step on a time stamp
  static cudaError_t snap(const SnapArgs<T>& a, long long ncell_total, cudaStream_t s);
};

// streaming multiprocessors of the current device (cached per device; 148
// on a B200), for grid-stride launch sizes
int device_sms();
// most block rows of a deterministic reduction launch (grid_for's cap)
inline long long reduce_rows_max() { return device_sms() * 32LL; }

cudaError_t launch_begin_step(const ProbDev* prob, ProbState* st, int nprob, double fixed_dt, int* nactive,
                              cudaStream_t s);
cudaError_t launch_end_step(const ProbDev* prob, ProbState* st, int nprob, cudaStream_t s);
// host-side construction shared by the C ABI entry points
ProbDev make_prob_public(const dspw_desc& d, long long off);
NetParams make_net_public(const dspw_desc& d);
}  // namespace dspw

struct dspw_handle;
namespace dspw {
// one residual evaluation of the handle's current state with pair collection
// enabled (used by the trainer); returns a dspw status
int handle_collect(dspw_handle* h, float* buf, unsigned long long* count, unsigned long long cap, unsigned stride);
int handle_precision(const dspw_handle* h);

}  // namespace dspw

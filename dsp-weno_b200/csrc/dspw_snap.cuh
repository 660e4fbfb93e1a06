// dspw_snap.cuh -- state snapshots at the output time stamps, taken on the
// device inside the step graph.  FV::run writes the solution whenever a step
// ends on a time stamp (enflo/src/fv.cc:1309-1313,
// enflo_scalar/src_scalar/fv.cc:586-590); the stamp test runs in the
// end-of-step kernel, which marks the problem, and the kernels here copy the
// marked problems' states into a ring of state-shaped slots that the host
// drains between graph launches.
#pragma once
#include "dspw_kernels.cuh"

namespace dspw {

struct SnapMeta {
  double time;
  int iter;
  int pad;
};

template <typename T>
struct SnapArgs {
  const ProbDev* prob;
  ProbState* st;
  int nprob;
  const long long* cell_start;
  const T* U;                     // U^(n+1)
  T* slots;                       // nslots state-shaped buffers (5 planes of ctot each)
  long long ctot;
  int nslots;
  unsigned long long* count;      // snapshots taken per problem
  SnapMeta* meta;                 // nslots * nprob
};

// copy the cells of every problem that ended this step on a time stamp into
// its next slot (a no-op pass when no problem did)
template <typename T>
__global__ void k_snap_copy(SnapArgs<T> A) {
  const long long total = A.cell_start[A.nprob];
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = A.nprob - 1;
    while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (A.cell_start[mid] <= g) lo = mid; else hi = mid - 1; }
    if (!A.st[lo].snap) continue;
    const ProbDev& P = A.prob[lo];
    T* dst = A.slots + (size_t)(A.count[lo] % (unsigned long long)A.nslots) * 5 * A.ctot;
    for (int v = 0; v < P.nv; v++) dst[v * A.ctot + g] = A.U[v * A.ctot + g];
  }
}

// record time and iteration of the new snapshots and clear the marks
template <typename T>
__global__ void k_snap_finish(SnapArgs<T> A) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= A.nprob) return;
  ProbState& S = A.st[p];
  if (!S.snap) return;
  if (A.nslots > 0) {
    const unsigned long long c = A.count[p];
    SnapMeta& m = A.meta[(c % (unsigned long long)A.nslots) * A.nprob + p];
    m.time = S.time;
    m.iter = S.iter;
    A.count[p] = c + 1;
  }
  S.snap = 0;
}

}  // namespace dspw

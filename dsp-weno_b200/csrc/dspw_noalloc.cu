// dspw_noalloc.cu -- global sums of a caller-owned state without any device
// allocation (dspw_globals_noalloc in include/dspw.h).
//
// Why it exists.  dspw_globals needs a handle, and creating a handle allocates
// device memory.  Some callers cannot allocate: a host driver that owns every
// device buffer through its own pool or arena, a library that shares the state
// with another component and may not grow the device footprint, or a loop that
// must not call cudaMalloc between launches because cudaMalloc can synchronise
// the device.  They pass their own state and their own output buffer; the only
// scratch is the file-scope array below.
//
// The scratch.  g_block_sums holds one row of 8 partial sums per thread block
// (NOALLOC_MAX_BLOCKS rows, 256 KiB).  Every GPU that loads the library keeps
// it until the process exits.  Each block covers NOALLOC_CELLS_PER_BLOCK cells,
// so one call handles at most NOALLOC_MAX_BLOCKS * NOALLOC_CELLS_PER_BLOCK
// cells (16,777,216 = 256^3); larger states are rejected with DSPW_ERR_ARG.
// Every block overwrites its own row before the second kernel reads it, so
// nothing needs clearing between calls; the rows keep the last call's values.
// All calls share the one array: calls whose kernels overlap on the GPU (two
// streams, or two host threads) race on it and must be serialised by the
// caller.
//
// Host code may not use the array's name as a device address (in host code it
// names a host-side stand-in).  The device address is obtained once per device
// with cudaGetSymbolAddress, with that device current, on the first call made
// on that device; that first call should therefore not be made while a stream
// is being captured.  The address is kept together with the id of the CUDA
// context it was taken in: after a cudaDeviceReset the device gets a new
// context, where the library's module (and the array) may sit elsewhere, so
// the first call in the new context looks the address up again (and, like the
// very first call, should not be made during stream capture).
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/dspw.h"

namespace {

constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_CELLS_PER_BLOCK = 4096;
constexpr int NOALLOC_MAX_BLOCKS = 4096;
constexpr long long NOALLOC_MAX_CELLS = (long long)NOALLOC_MAX_BLOCKS * NOALLOC_CELLS_PER_BLOCK;
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double g_block_sums[NOALLOC_MAX_BLOCKS][8];

struct SumParams {
  long long ncell;
  long long stride;
  int nv;          // stored components (1 scalar; dim+2 Euler)
  int scalar;
  double gamma;
  double vol;
};

template <typename T>
__device__ inline void cell_sums(const T* U, long long stride, long long c, const SumParams& p, double acc[7]) {
  if (p.scalar) {
    double u = (double)U[c];
    acc[0] += 0.5 * u * u;   // enflo_scalar/src_scalar/compute_global.cc:12-21
    acc[2] += u;
    return;
  }
  double u[5];
  u[0] = U[c];
  u[1] = U[stride + c];
  u[2] = p.nv >= 4 ? (double)U[2 * stride + c] : 0.0;
  u[3] = p.nv == 5 ? (double)U[3 * stride + c] : 0.0;
  u[4] = U[(p.nv - 1) * stride + c];
  double rho = u[0];
  double r = 1.0 / rho;
  double vx = u[1] * r, vy = u[2] * r, vz = u[3] * r;
  double pr = (p.gamma - 1.0) * (u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / rho);
  double s = ::log(pr) - p.gamma * ::log(rho);   // enflo/src/compute_global.cc:18-28
  acc[0] += -rho * s / (p.gamma - 1.0);
  acc[1] += 0.5 * rho * (vx * vx + vy * vy + vz * vz);
  for (int v = 0; v < 5; v++) acc[2 + v] += u[v];
}

// pass 1: each block reduces its NOALLOC_CELLS_PER_BLOCK cells in a fixed
// order and writes its row of the scratch
template <typename T>
__global__ void __launch_bounds__(NOALLOC_THREADS) k_block_sums(const T* U, SumParams p, double (*rows)[8]) {
  __shared__ double red[NOALLOC_THREADS / 32][7];
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  long long first = (long long)blockIdx.x * NOALLOC_CELLS_PER_BLOCK;
  for (int k = threadIdx.x; k < NOALLOC_CELLS_PER_BLOCK; k += NOALLOC_THREADS) {
    long long c = first + k;
    if (c < p.ncell) cell_sums<T>(U, p.stride, c, p, acc);
  }
  for (int v = 0; v < 7; v++)
    for (int o = 16; o > 0; o >>= 1) acc[v] += __shfl_xor_sync(0xffffffffu, acc[v], o);
  if ((threadIdx.x & 31) == 0)
    for (int v = 0; v < 7; v++) red[threadIdx.x >> 5][v] = acc[v];
  __syncthreads();
  if (threadIdx.x < 7) {
    double t = 0.0;
    for (int w = 0; w < NOALLOC_THREADS / 32; w++) t += red[w][threadIdx.x];
    rows[blockIdx.x][threadIdx.x] = t;
  }
}

// pass 2: one block adds the rows in a fixed order and scales by the cell volume
__global__ void __launch_bounds__(NOALLOC_THREADS) k_final_sums(const double (*rows)[8], int nblocks, double vol,
                                                                double* out) {
  __shared__ double red[NOALLOC_THREADS / 32][7];
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += NOALLOC_THREADS)
    for (int v = 0; v < 7; v++) acc[v] += rows[b][v];
  for (int v = 0; v < 7; v++)
    for (int o = 16; o > 0; o >>= 1) acc[v] += __shfl_xor_sync(0xffffffffu, acc[v], o);
  if ((threadIdx.x & 31) == 0)
    for (int v = 0; v < 7; v++) red[threadIdx.x >> 5][v] = acc[v];
  __syncthreads();
  if (threadIdx.x < 7) {
    double t = 0.0;
    for (int w = 0; w < NOALLOC_THREADS / 32; w++) t += red[w][threadIdx.x];
    out[threadIdx.x] = t * vol;
  }
}

std::mutex g_setup_mutex;
void* g_scratch_addr[NOALLOC_MAX_DEVICES] = {};
unsigned long long g_scratch_ctx[NOALLOC_MAX_DEVICES] = {};   // context id the address belongs to

// id of the current CUDA context (driver entry points cuCtxGetCurrent and
// cuCtxGetId, found through the runtime; unique for the life of the process)
int current_context_id(unsigned long long* id) {
  typedef int (*GetCurrentFn)(void**);
  typedef int (*GetIdFn)(void*, unsigned long long*);
  static GetCurrentFn get_current = nullptr;
  static GetIdFn get_id = nullptr;
  if (!get_current || !get_id) {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || !f1)
      return DSPW_ERR_CUDA;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
        q2 != cudaDriverEntryPointSuccess || !f2)
      return DSPW_ERR_CUDA;
    get_current = (GetCurrentFn)f1;
    get_id = (GetIdFn)f2;
  }
  void* ctx = nullptr;
  if (get_current(&ctx) != 0 || !ctx) return DSPW_ERR_CUDA;
  if (get_id(ctx, id) != 0) return DSPW_ERR_CUDA;
  return DSPW_OK;
}

// device address of g_block_sums for the current device, looked up once per
// device and context
int scratch_for_current_device(void** addr) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return DSPW_ERR_CUDA;
  // cudaFree(0) makes the device's primary context current (a no-op when it is)
  if (cudaFree(0) != cudaSuccess) return DSPW_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  unsigned long long ctx = 0;
  int r = current_context_id(&ctx);
  if (r) return r;
  if (!g_scratch_addr[dev] || g_scratch_ctx[dev] != ctx) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_block_sums) != cudaSuccess || !p) return DSPW_ERR_CUDA;
    g_scratch_addr[dev] = p;
    g_scratch_ctx[dev] = ctx;
  }
  *addr = g_scratch_addr[dev];
  return DSPW_OK;
}

}  // namespace

extern "C" DSPW_API int dspw_globals_noalloc(const dspw_desc* desc, const void* d_cons, long long stride,
                                             int elem_bytes, double* d_out, void* stream) {
  if (!desc || !d_cons || !d_out || (elem_bytes != 4 && elem_bytes != 8)) return DSPW_ERR_ARG;
  if (desc->abi_version != DSPW_ABI_VERSION) return DSPW_ERR_ARG;
  if (desc->model < DSPW_LINADV || desc->model > DSPW_NS_KEP) return DSPW_ERR_ARG;
  if (desc->nx < 1 || desc->ny < 1 || desc->nz < 1) return DSPW_ERR_ARG;
  if (!(desc->xmax > desc->xmin) || !(desc->ymax > desc->ymin) || !(desc->zmax > desc->zmin)) return DSPW_ERR_ARG;
  SumParams p;
  p.ncell = (long long)desc->nx * desc->ny * desc->nz;
  if (p.ncell > NOALLOC_MAX_CELLS) return DSPW_ERR_ARG;   // beyond the fixed scratch
  if (stride < p.ncell) return DSPW_ERR_ARG;
  p.stride = stride;
  p.scalar = desc->model == DSPW_LINADV || desc->model == DSPW_BURGERS;
  int dim = desc->nz > 1 ? 3 : (desc->ny > 1 ? 2 : 1);
  p.nv = p.scalar ? 1 : dim + 2;
  p.gamma = desc->gamma;
  if (!p.scalar && !(p.gamma > 1.0)) return DSPW_ERR_ARG;
  // cell sizes as the handle path takes them: a slab of a decomposed domain
  // carries the domain's own in cell_size
  double h[3] = {(desc->xmax - desc->xmin) / desc->nx, (desc->ymax - desc->ymin) / desc->ny,
                 (desc->zmax - desc->zmin) / desc->nz};
  for (int k = 0; k < 3; k++) {
    if (!(desc->cell_size[k] >= 0.0)) return DSPW_ERR_ARG;
    if (desc->cell_size[k] > 0.0) h[k] = desc->cell_size[k];
  }
  p.vol = h[0] * h[1] * h[2];
  void* scratch = nullptr;
  int r = scratch_for_current_device(&scratch);
  if (r) return r;
  double(*rows)[8] = reinterpret_cast<double(*)[8]>(scratch);
  int nblocks = (int)((p.ncell + NOALLOC_CELLS_PER_BLOCK - 1) / NOALLOC_CELLS_PER_BLOCK);
  cudaStream_t s = (cudaStream_t)stream;
  if (elem_bytes == 8)
    k_block_sums<double><<<nblocks, NOALLOC_THREADS, 0, s>>>((const double*)d_cons, p, rows);
  else
    k_block_sums<float><<<nblocks, NOALLOC_THREADS, 0, s>>>((const float*)d_cons, p, rows);
  if (cudaGetLastError() != cudaSuccess) return DSPW_ERR_CUDA;
  k_final_sums<<<1, NOALLOC_THREADS, 0, s>>>(rows, nblocks, p.vol, d_out);
  if (cudaGetLastError() != cudaSuccess) return DSPW_ERR_CUDA;
  return DSPW_OK;
}

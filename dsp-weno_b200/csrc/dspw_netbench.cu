// Measurement kernels for the DSP-WENO network evaluation on the tensor cores.
//
// Two forms of the same 5-5-5-5-5 network (four layers, ReLU between them,
// BF16 operands, FP32 accumulation):
//   * k_net_mma_sync: the sweep kernels' form.  Per warp 32 instances, two
//     m16n8k8 tiles per layer through mlp_warp_tiles, the activations kept in
//     registers from layer to layer, the biases as the C operand.
//   * k_net_tcgen05: the Blackwell tensor-core form.  Per block of 128
//     threads one M = 128 tile per layer: every thread writes its instance's
//     activations as one row of the BF16 A operand in shared memory, one
//     thread issues tcgen05.mma against the layer's weights (the B operand,
//     N = 16, K = 16, zero padded), the FP32 accumulator lands in tensor
//     memory and every warp reads its 32 rows back with tcgen05.ld for the
//     bias and the ReLU of the next layer's operand.
// Both evaluate the same synthetic inputs (a hash of instance, repetition and
// input index) `reps` times per instance and sum the logits over the
// repetitions, so their outputs are comparable with each other and with a CPU
// evaluation.  dspw/netbench.py drives them.
//
// Every wait on the tensor core's mbarrier is bounded; a wait that gives up
// sets the error word, the block leaves its loop and frees its tensor memory.
#include "dspw_kernels.cuh"

#define DSPW_NB_API extern "C" __attribute__((visibility("default")))

namespace dspw {
namespace netbench {

// input k of instance i in repetition r, uniform in [-1, 1)
__device__ __forceinline__ float feat_of(unsigned long long i, int r, int k) {
  unsigned x = (unsigned)i * 0x9E3779B1u ^ (unsigned)(i >> 32) * 0x7FEB352Du ^ (unsigned)r * 0x85EBCA77u ^
               (unsigned)k * 0xC2B2AE3Du;
  x ^= x >> 15;
  x *= 0x2C1B3C6Du;
  x ^= x >> 12;
  x *= 0x297A2D39u;
  x ^= x >> 15;
  return (float)(x >> 8) * (2.0f / 16777216.0f) - 1.0f;
}

constexpr int TILE = 128;   // instances per block and pass, both forms

__global__ void __launch_bounds__(TILE) k_net_mma_sync(const NetParams* np, float* out, long long ntile, int reps,
                                                         long long* cycles) {
  __shared__ __align__(16) NetScratch<float> ns[TILE / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  net_frag_stage<float>(*np, lane, ns[warp]);
  const long long c0 = clock64();
  for (long long t = blockIdx.x; t < ntile; t += gridDim.x) {
    const unsigned long long i = (unsigned long long)t * TILE + threadIdx.x;
    float acc[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    for (int r = 0; r < reps; r++) {
      float in[5], lg[5];
#pragma unroll
      for (int k = 0; k < 5; k++) in[k] = feat_of(i, r, k);
      warp_mlp_bf16(ns[warp], in, lg, lane);
#pragma unroll
      for (int k = 0; k < 5; k++) acc[k] += lg[k];
    }
#pragma unroll
    for (int k = 0; k < 5; k++) out[i * 5 + k] = acc[k];
  }
  if (cycles && threadIdx.x == 0) cycles[blockIdx.x] = clock64() - c0;
}

// ---------------------------------------------------------------- tcgen05 --

// Byte offset of element (row, k) of a 16-wide BF16 operand in the canonical
// K-major layout without swizzle: 8 x 8 core matrices of 128 contiguous bytes
// (8 rows of 16 bytes), the two core matrices of a row group 128 bytes apart
// (leading byte offset), row groups 256 bytes apart (stride byte offset).
__host__ __device__ constexpr unsigned op_off(unsigned row, unsigned k) {
  return (row >> 3) * 256u + (k >> 3) * 128u + (row & 7u) * 16u + (k & 7u) * 2u;
}

struct __align__(1024) TcSmem {
  unsigned char a[TILE * 32];     // A: 128 instances x 16 inputs
  unsigned char b[4][16 * 32];    // B of each layer: 16 outputs x 16 inputs
  float bias[4][8];
  unsigned long long bar;
  unsigned tmem;
};

// shared-memory matrix descriptor: start address, leading byte offset 128,
// stride byte offset 256, descriptor version 1, no swizzle
__device__ __forceinline__ unsigned long long op_desc(const void* p) {
  const unsigned s = smem_u32(p);
  return (unsigned long long)((s & 0x3FFFFu) >> 4) | ((unsigned long long)(128u >> 4) << 16) |
         ((unsigned long long)(256u >> 4) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N = 16, M = 128
constexpr unsigned IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// this thread's row of the A operand: 5 activations rounded to BF16, inputs 5..7 zero
// (inputs 8..15 stay zero from the start)
__device__ __forceinline__ void store_row(unsigned char* a, int row, const float h[5]) {
  uint4 v;
  v.x = pack_bf16(h[0], h[1]);
  v.y = pack_bf16(h[2], h[3]);
  v.z = pack_bf16(h[4], 0.f);
  v.w = 0u;
  *reinterpret_cast<uint4*>(a + op_off(row, 0)) = v;
}

__global__ void __launch_bounds__(TILE) k_net_tcgen05(const float* wts, const float* bias, float* out, long long ntile,
                                                        int reps, long long* cycles, int* err) {
  __shared__ TcSmem S;
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int e = tid; e < TILE * 32 / 16; e += TILE) reinterpret_cast<uint4*>(S.a)[e] = make_uint4(0, 0, 0, 0);
  for (int e = tid; e < 4 * 16 * 16; e += TILE) {
    const int l = e >> 8, n = (e >> 4) & 15, k = e & 15;
    const float w = (n < 5 && k < 5) ? wts[(l * 5 + n) * 5 + k] : 0.f;
    *reinterpret_cast<__nv_bfloat16*>(S.b[l] + op_off(n, k)) = __float2bfloat16_rn(w);
  }
  if (tid < 32) S.bias[tid >> 3][tid & 7] = (tid & 7) < 5 ? bias[(tid >> 3) * 5 + (tid & 7)] : 0.f;
  if (tid == 0) {
    mbar_init(&S.bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                 "r"(32u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_proxy_async_smem();
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  const unsigned tmem = S.tmem;
  const unsigned trow = tmem + ((unsigned)(warp * 32) << 16);   // this warp's 32 lanes
  // layer l's B operand starts 512 bytes (32 address units) after layer 0's
  const unsigned long long bdesc0 = op_desc(S.b[0]);
  const unsigned long long adesc = op_desc(S.a);
  unsigned phase = 0;
  bool bad = false;
  const long long c0 = clock64();
  for (long long t = blockIdx.x; t < ntile && !bad; t += gridDim.x) {
    const unsigned long long i = (unsigned long long)t * TILE + tid;
    float acc[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    for (int r = 0; r < reps && !bad; r++) {
      float h[5];
#pragma unroll
      for (int k = 0; k < 5; k++) h[k] = feat_of(i, r, k);
      store_row(S.a, tid, h);
#pragma unroll 1
      for (int l = 0; l < 4; l++) {
        // the rows written by every thread are visible to the tensor core
        fence_proxy_async_smem();
        tc_before_sync();
        __syncthreads();
        tc_after_sync();
        if (tid == 0) {
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
              ::"r"(tmem), "l"(adesc), "l"(bdesc0 + (unsigned long long)(l * (16 * 32 / 16))), "r"(IDESC), "r"(0)
              : "memory");
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                           smem_u32(&S.bar))
                       : "memory");
        }
        const bool ok = mbar_wait(&S.bar, phase);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
          bad = true;
          break;
        }
        tc_after_sync();
        unsigned d[8];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
            : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7])
            : "r"(trow)
            : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (l < 3) {
#pragma unroll
          for (int k = 0; k < 5; k++) h[k] = fmaxf(__uint_as_float(d[k]) + S.bias[l][k], 0.f);
          store_row(S.a, tid, h);
        } else {
#pragma unroll
          for (int k = 0; k < 5; k++) acc[k] += __uint_as_float(d[k]) + S.bias[3][k];
        }
      }
    }
    if (!bad) {
#pragma unroll
      for (int k = 0; k < 5; k++) out[i * 5 + k] = acc[k];
    }
  }
  const long long c1 = clock64();
  // every tcgen05.ld of the block is complete before the columns are freed
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32u) : "memory");
  if (bad && tid == 0) atomicExch(err, 1);
  if (cycles && tid == 0) cycles[blockIdx.x] = c1 - c0;
}

}  // namespace netbench
}  // namespace dspw

using namespace dspw;
using namespace dspw::netbench;

// Resident blocks per SM of form 0 / 1 (occupancy calculator), and the
// kernel's registers per thread and static shared memory.
DSPW_NB_API int dspw_netbench_occupancy(int form, int* blocks_per_sm, int* regs, int* smem) {
  if (form < 0 || form > 1 || !blocks_per_sm) return 1;
  cudaFuncAttributes fa;
  const void* fn = form == 0 ? (const void*)k_net_mma_sync : (const void*)k_net_tcgen05;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn, TILE, 0) != cudaSuccess ||
      cudaFuncGetAttributes(&fa, fn) != cudaSuccess)
    return 2;
  if (regs) *regs = fa.numRegs;
  if (smem) *smem = (int)fa.sharedSizeBytes;
  return 0;
}

// Evaluates `ntile` x 128 instances `reps` times each with form 0 (mma.sync)
// or 1 (tcgen05) on the current device's default stream.  wts: the four 5 x 5
// weight matrices W[l][out][in]; bias: b[l][out] (device pointers, FP32).
// out: device, 5 floats per instance.  grid 0 takes the occupancy limit times
// the SM count.  cycles (device, optional): clock64 cycles of each block's
// loop.  *ms receives the kernel's device time (CUDA events).  Returns 0, 1
// (bad argument), 2 (CUDA error) or 3 (a tensor-core wait gave up).
DSPW_NB_API int dspw_netbench_run(int form, const float* wts, const float* bias, float* out, long long ntile,
                                  int reps, int grid, long long* cycles, float* ms, int* grid_used) {
  if (form < 0 || form > 1 || !wts || !bias || !out || ntile <= 0 || reps <= 0 || grid < 0) return 1;
  int dev = 0, sms = 0, occ = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 2;
  if (form == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_net_mma_sync, TILE, 0) != cudaSuccess) return 2;
  } else {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_net_tcgen05, TILE, 0) != cudaSuccess) return 2;
    // 32 tensor-memory columns per block: at most 16 blocks of an SM hold
    // columns at once, so no allocation waits on another block
    occ = occ < 16 ? occ : 16;
  }
  if (grid == 0) grid = occ * sms;
  if (form == 1 && grid > 16 * sms) return 1;
  if ((long long)grid > ntile) grid = (int)ntile;
  if (grid_used) *grid_used = grid;
  NetParams* dnp = nullptr;
  int* derr = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int ret = 0;
  if (cudaMalloc(&derr, sizeof(int)) != cudaSuccess) return 2;
  cudaMemset(derr, 0, sizeof(int));
  if (form == 0) {
    // the sweep kernels' parameter block, filled with these weights (no
    // base-2 scaling of the last layer: the logits are compared as they are)
    NetParams np;
    memset(&np, 0, sizeof(np));
    float hw[100], hb[20];
    if (cudaMemcpy(hw, wts, sizeof(hw), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(hb, bias, sizeof(hb), cudaMemcpyDeviceToHost) != cudaSuccess) {
      cudaFree(derr);
      return 2;
    }
    for (int l = 0; l < 4; l++)
      for (int n = 0; n < 5; n++) {
        np.bf[l][n] = hb[l * 5 + n];
        for (int k = 0; k < 5; k++) np.wf[l][n][k] = hw[(l * 5 + n) * 5 + k];
      }
    if (cudaMalloc(&dnp, sizeof(NetParams)) != cudaSuccess ||
        cudaMemcpy(dnp, &np, sizeof(NetParams), cudaMemcpyHostToDevice) != cudaSuccess) {
      ret = 2;
      goto done;
    }
  }
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  if (form == 0)
    k_net_mma_sync<<<grid, TILE>>>(dnp, out, ntile, reps, cycles);
  else
    k_net_tcgen05<<<grid, TILE>>>(wts, bias, out, ntile, reps, cycles, derr);
  cudaEventRecord(e1, 0);
  if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    ret = 2;
    goto done;
  }
  if (ms) cudaEventElapsedTime(ms, e0, e1);
  {
    int herr = 0;
    cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
    if (herr) ret = 3;
  }
done:
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (dnp) cudaFree(dnp);
  cudaFree(derr);
  return ret;
}

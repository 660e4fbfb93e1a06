// dspw_train.cu -- DSP-WENO network training on the GPU.
//
// The reference trains with PyTorch (DSP-WENO_trainer/DSP-WENO_network_trainer.py):
// the 5-5-5-5-5 ReLU MLP (:23-91) maps the features [tanh theta-, tanh theta+,
// d1, d2, d3] to 5 logits, a softmax picks convex weights of 5 feasible-region
// vertices, C1/C2 give the reconstruction weights and inter_evaluation
// (:94-106) the two interface values; the loss is (MSE(left) + MSE(right))/2
// (:404) and the optimiser Adam with L2 weight decay (:353).  Here the same
// model and loss run as CUDA kernels:
//
//   k_prepare      stencil -> features and vertices with the forward's own
//                  preprocessing (neural_network.cc:21-37), once per sample;
//   k_fwd_bwd      one thread per sample of a minibatch: forward, loss,
//                  backward through softmax / ReLU layers; gradients reduced
//                  by warp shuffles, then per block, into an FP64 accumulator;
//   k_adam         one thread per parameter, FP32 master weights (PyTorch
//                  Adam semantics: L2 decay added to the gradient, bias
//                  corrections, eps outside the square root).
//
// compute_bf16 = 1 rounds weights and activations to BF16 before each product
// (FP32 accumulation), the arithmetic of the inference kernels' tensor-core
// layers; compute_bf16 = 0 keeps FP32 throughout (used for the gradient checks).
// The network has 120 parameters, so a minibatch is a few microseconds of
// CUDA-core work; the tensor pipe would stay idle on it.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <algorithm>
#include <random>
#include <vector>

#include "dspw_launch.h"

using namespace dspw;

namespace {

constexpr int NPARAM = 120;   // 4 x 25 weights (out x in), then 4 x 5 biases
constexpr int NCOL = 22;      // feat 5, vx 5, vy 5, u 4, target 2, weight 1
constexpr int TPB = 256;

__device__ __forceinline__ float bfr(float x, int on) {
  return on ? __bfloat162float(__float2bfloat16_rn(x)) : x;
}

// stencil + targets (FP64 host data staged on the device) -> one sample column set
__global__ void k_prepare_f64(const double* st, const double* tg, long long n, float* data, long long cap,
                              long long at) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double u[4] = {st[4 * i], st[4 * i + 1], st[4 * i + 2], st[4 * i + 3]};
  double f[5], vx[5], vy[5];
  nn_features<double>(u[0], u[1], u[2], u[3], f, vx, vy);
  bool ok = fabs(u[2] - u[1]) >= 1e-15;   // the forward is not used below this (reconstruct.cc:152)
  for (int k = 0; k < 5; k++) ok = ok && isfinite(f[k]) && isfinite(vx[k]) && isfinite(vy[k]);
  long long j = at + i;
  for (int k = 0; k < 5; k++) {
    data[(0 + k) * cap + j] = ok ? (float)f[k] : 0.f;
    data[(5 + k) * cap + j] = ok ? (float)vx[k] : 0.f;
    data[(10 + k) * cap + j] = ok ? (float)vy[k] : 0.f;
  }
  for (int k = 0; k < 4; k++) data[(15 + k) * cap + j] = (float)u[k];
  data[19 * cap + j] = (float)tg[2 * i];
  data[20 * cap + j] = (float)tg[2 * i + 1];
  data[21 * cap + j] = ok ? 1.f : 0.f;
}

// collected pairs (6 floats: u0..u3, l, r) -> samples
__global__ void k_prepare_pairs(const float* pairs, long long n, float* data, long long cap, long long at) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* q = pairs + 6 * i;
  double u[4] = {q[0], q[1], q[2], q[3]};
  double f[5], vx[5], vy[5];
  nn_features<double>(u[0], u[1], u[2], u[3], f, vx, vy);
  bool ok = fabs(u[2] - u[1]) >= 1e-15;
  for (int k = 0; k < 5; k++) ok = ok && isfinite(f[k]) && isfinite(vx[k]) && isfinite(vy[k]);
  long long j = at + i;
  for (int k = 0; k < 5; k++) {
    data[(0 + k) * cap + j] = ok ? (float)f[k] : 0.f;
    data[(5 + k) * cap + j] = ok ? (float)vx[k] : 0.f;
    data[(10 + k) * cap + j] = ok ? (float)vy[k] : 0.f;
  }
  for (int k = 0; k < 4; k++) data[(15 + k) * cap + j] = q[k];
  data[19 * cap + j] = q[4];
  data[20 * cap + j] = q[5];
  data[21 * cap + j] = ok ? 1.f : 0.f;
}

// forward + loss + backward of the samples perm[b0 .. b0+B) (perm may be null)
__global__ void __launch_bounds__(TPB) k_fwd_bwd(const float* data, long long cap, const int* perm, long long b0,
                                                 int B, float inv_b, const float* prm, double* grad,
                                                 double* loss, int bf16) {
  __shared__ float sw[NPARAM];
  __shared__ float gsh[NPARAM];
  __shared__ double lsh;
  for (int k = threadIdx.x; k < NPARAM; k += blockDim.x) { sw[k] = prm[k]; gsh[k] = 0.f; }
  if (threadIdx.x == 0) lsh = 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  bool active = t < B;
  float g[NPARAM];
#pragma unroll
  for (int k = 0; k < NPARAM; k++) g[k] = 0.f;
  float lsum = 0.f;
  if (active) {
    long long idx = perm ? (long long)perm[b0 + t] : b0 + t;
    float wgt = data[21 * cap + idx];
    float a[4][5], pre[4][5];
#pragma unroll
    for (int k = 0; k < 5; k++) a[0][k] = bfr(data[k * cap + idx], bf16);
    float z[5];
#pragma unroll
    for (int l = 0; l < 4; l++) {
#pragma unroll
      for (int j = 0; j < 5; j++) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 5; k++) acc += bfr(sw[l * 25 + j * 5 + k], bf16) * a[l][k];
        acc += sw[100 + l * 5 + j];
        if (l < 3) {
          pre[l][j] = acc;
          a[l + 1][j] = bfr(fmaxf(acc, 0.f), bf16);
        } else {
          z[j] = acc;
        }
      }
    }
    // softmax, vertex combination, interface values (trainer :63-106)
    float mx = z[0];
#pragma unroll
    for (int k = 1; k < 5; k++) mx = fmaxf(mx, z[k]);
    float s[5], se = 0.f;
#pragma unroll
    for (int k = 0; k < 5; k++) { s[k] = expf(z[k] - mx); se += s[k]; }
#pragma unroll
    for (int k = 0; k < 5; k++) s[k] /= se;
    float vx[5], vy[5];
#pragma unroll
    for (int k = 0; k < 5; k++) { vx[k] = data[(5 + k) * cap + idx]; vy[k] = data[(10 + k) * cap + idx]; }
    float C1 = 0.f, C2 = 0.f;
#pragma unroll
    for (int k = 0; k < 5; k++) { C1 += s[k] * vx[k]; C2 += s[k] * vy[k]; }
    float u0 = data[15 * cap + idx], u1 = data[16 * cap + idx], u2 = data[17 * cap + idx], u3 = data[18 * cap + idx];
    float c = 0.5f * u1 + 0.5f * u2, bl = -0.5f * u0 + 1.5f * u1, br = 1.5f * u2 - 0.5f * u3;
    float w1 = 0.25f - 2.f * C1, tw0 = 0.25f - 2.f * C2;
    float left = (1.f - w1) * c + w1 * bl;
    float right = tw0 * br + (1.f - tw0) * c;
    float el = left - data[19 * cap + idx], er = right - data[20 * cap + idx];
    lsum = wgt * 0.5f * (el * el + er * er) * inv_b;
    // backward
    float dl = wgt * el * inv_b, dr = wgt * er * inv_b;
    float dC1 = -2.f * dl * (bl - c), dC2 = -2.f * dr * (br - c);
    float ds[5], sds = 0.f;
#pragma unroll
    for (int k = 0; k < 5; k++) { ds[k] = dC1 * vx[k] + dC2 * vy[k]; sds += s[k] * ds[k]; }
    float dpre[5];
#pragma unroll
    for (int k = 0; k < 5; k++) dpre[k] = s[k] * (ds[k] - sds);
#pragma unroll
    for (int l = 3; l >= 0; l--) {
#pragma unroll
      for (int j = 0; j < 5; j++) {
#pragma unroll
        for (int k = 0; k < 5; k++) g[l * 25 + j * 5 + k] += dpre[j] * a[l][k];
        g[100 + l * 5 + j] += dpre[j];
      }
      if (l > 0) {
        float nd[5];
#pragma unroll
        for (int k = 0; k < 5; k++) {
          float acc = 0.f;
#pragma unroll
          for (int j = 0; j < 5; j++) acc += bfr(sw[l * 25 + j * 5 + k], bf16) * dpre[j];
          nd[k] = pre[l - 1][k] > 0.f ? acc : 0.f;
        }
#pragma unroll
        for (int k = 0; k < 5; k++) dpre[k] = nd[k];
      }
    }
  }
  // reduce: warp shuffles, then one shared-memory add per warp, then global
#pragma unroll
  for (int k = 0; k < NPARAM; k++) {
    float v = g[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) atomicAdd(&gsh[k], v);
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if (lane == 0) atomicAdd(&lsh, (double)lsum);
  __syncthreads();
  for (int k = threadIdx.x; k < NPARAM; k += blockDim.x) atomicAdd(&grad[k], (double)gsh[k]);
  if (threadIdx.x == 0) atomicAdd(loss, lsh);
}

// Adam with L2 weight decay (torch.optim.Adam semantics), FP32 master weights
__global__ void k_adam(float* prm, const double* grad, float* m, float* v, int step, float lr, float b1, float b2,
                       float wd, float eps) {
  int k = threadIdx.x;
  if (k >= NPARAM) return;
  float g = (float)grad[k] + wd * prm[k];
  m[k] = b1 * m[k] + (1.f - b1) * g;
  v[k] = b2 * v[k] + (1.f - b2) * g * g;
  float bc1 = 1.f - powf(b1, (float)step);
  float bc2 = 1.f - powf(b2, (float)step);
  float denom = sqrtf(v[k]) / sqrtf(bc2) + eps;
  prm[k] -= (lr / bc1) * m[k] / denom;
}

// max of each feature over the valid samples (the network's training box)
__global__ void k_feature_max(const float* data, long long cap, long long n, unsigned* out /* 5 */) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n || data[21 * cap + i] == 0.f) return;
  for (int k = 0; k < 5; k++) atomicMax(&out[k], __float_as_uint(fabsf(data[k * cap + i])));
}

// order-preserving map of a float onto an unsigned integer (negative values
// reversed below the positive ones), so that unsigned atomicMin / atomicMax
// find the smallest and largest float
__device__ inline unsigned float_key(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
inline float key_float(unsigned k) {
  const unsigned u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  float f;
  memcpy(&f, &u, sizeof(f));
  return f;
}

// smallest and largest value of each feature over the valid samples
// (out[0..4] minima, out[5..9] maxima, as float_key)
__global__ void k_feature_box(const float* data, long long cap, long long n, unsigned* out /* 10 */) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n || data[21 * cap + i] == 0.f) return;
  for (int k = 0; k < 5; k++) {
    const unsigned key = float_key(data[k * cap + i]);
    atomicMin(&out[k], key);
    atomicMax(&out[5 + k], key);
  }
}

// One row of the reference trainer's data file per sample, in the column
// order its reader slices (DSP-WENO_trainer/DSP-WENO_network_trainer.py:305-333
// with tanh_theta: cell values 0-3, theta-, theta+ 4-5, the network inputs
// tanh theta-, tanh theta+, del1..del3 6-10, vertex x 11-15, vertex y 16-20,
// target interface values left, right 21-22), recomputed in FP64 from the
// sample's cell values with the kernels' own feature code.  valid[i] = 0 for
// samples the trainer ignores.
constexpr int EXPORT_COLS = 23;
__global__ void k_export_rows(const float* data, long long cap, long long n, double* out, int* valid) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (data[21 * cap + i] == 0.f) { valid[i] = 0; return; }
  double u[4];
  for (int k = 0; k < 4; k++) u[k] = (double)data[(15 + k) * cap + i];
  double f[5], vx[5], vy[5];
  nn_features<double>(u[0], u[1], u[2], u[3], f, vx, vy);
  // theta of the scaled stencil, as nn_features forms it (neural_network.cc:27-28)
  double mx = 1.0;
  for (int k = 0; k < 4; k++) mx = fmax(mx, fabs(u[k]));
  const double c0 = u[0] / mx, c1 = u[1] / mx, c2 = u[2] / mx, c3 = u[3] / mx;
  double* r = out + (size_t)EXPORT_COLS * i;
  for (int k = 0; k < 4; k++) r[k] = u[k];
  r[4] = (c3 - c2) / (c2 - c1);
  r[5] = (c1 - c0) / (c2 - c1);
  for (int k = 0; k < 5; k++) { r[6 + k] = f[k]; r[11 + k] = vx[k]; r[16 + k] = vy[k]; }
  r[21] = (double)data[19 * cap + i];
  r[22] = (double)data[20 * cap + i];
  valid[i] = 1;
}

}  // namespace

struct dspw_trainer {
  dspw_train_cfg cfg;
  float* prm = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  double* grad = nullptr;
  double* loss = nullptr;
  float* data = nullptr;
  long long n = 0, cap = 0;
  int* perm = nullptr;
  long long perm_cap = 0;
  float* pairs = nullptr;
  unsigned long long* pair_count = nullptr;
  long long pairs_cap = 0;
  int step = 0;
  cudaStream_t stream = nullptr;
  std::mt19937_64 rng;
};

namespace {

#define TK(x)                                \
  do {                                       \
    if ((x) != cudaSuccess) return DSPW_ERR_CUDA; \
  } while (0)

// grow the dataset to hold `need` samples (columns are reallocated and copied)
int ensure_cap(dspw_trainer* t, long long need) {
  if (need <= t->cap) return DSPW_OK;
  long long nc = std::max<long long>(need, t->cap * 2);
  float* nd = nullptr;
  if (cudaMalloc(&nd, sizeof(float) * NCOL * nc) != cudaSuccess) return DSPW_ERR_NOMEM;
  if (t->data && t->n > 0)
    for (int c = 0; c < NCOL; c++)
      TK(cudaMemcpyAsync(nd + c * nc, t->data + c * t->cap, sizeof(float) * t->n, cudaMemcpyDeviceToDevice, t->stream));
  TK(cudaStreamSynchronize(t->stream));
  if (t->data) cudaFree(t->data);
  t->data = nd;
  t->cap = nc;
  return DSPW_OK;
}

int fwd_bwd(dspw_trainer* t, const int* perm, long long b0, int B, const float* prm) {
  TK(cudaMemsetAsync(t->grad, 0, sizeof(double) * NPARAM, t->stream));
  int blocks = (B + TPB - 1) / TPB;
  k_fwd_bwd<<<blocks, TPB, 0, t->stream>>>(t->data, t->cap, perm, b0, B, 1.f / (float)B, prm, t->grad, t->loss,
                                           t->cfg.compute_bf16 ? 1 : 0);
  TK(cudaGetLastError());
  return DSPW_OK;
}

}  // namespace

extern "C" {

int dspw_trainer_create(const dspw_train_cfg* cfg, const double* w_init, const double* b_init, dspw_trainer** out) {
  if (!cfg || !w_init || !b_init || !out || cfg->batch < 1) return DSPW_ERR_ARG;
  dspw_trainer* t = new dspw_trainer;
  t->cfg = *cfg;
  t->rng.seed((unsigned long long)cfg->seed);
  float h[NPARAM];
  for (int k = 0; k < 100; k++) h[k] = (float)w_init[k];
  for (int k = 0; k < 20; k++) h[100 + k] = (float)b_init[k];
  bool ok = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&t->prm, sizeof(float) * NPARAM) == cudaSuccess &&
            cudaMalloc(&t->m, sizeof(float) * NPARAM) == cudaSuccess &&
            cudaMalloc(&t->v, sizeof(float) * NPARAM) == cudaSuccess &&
            cudaMalloc(&t->grad, sizeof(double) * NPARAM) == cudaSuccess &&
            cudaMalloc(&t->loss, sizeof(double)) == cudaSuccess &&
            cudaMemcpy(t->prm, h, sizeof(h), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemset(t->m, 0, sizeof(float) * NPARAM) == cudaSuccess &&
            cudaMemset(t->v, 0, sizeof(float) * NPARAM) == cudaSuccess;
  if (!ok) {
    dspw_trainer_destroy(t);
    return DSPW_ERR_NOMEM;
  }
  *out = t;
  return DSPW_OK;
}

int dspw_trainer_destroy(dspw_trainer* t) {
  if (!t) return DSPW_ERR_ARG;
  if (t->stream) cudaStreamSynchronize(t->stream);
  void* ptrs[] = {t->prm, t->m, t->v, t->grad, t->loss, t->data, t->perm, t->pairs, t->pair_count};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (t->stream) cudaStreamDestroy(t->stream);
  delete t;
  return DSPW_OK;
}

int dspw_trainer_set_data(dspw_trainer* t, const double* stencils, const double* targets, long long n) {
  if (!t || !stencils || !targets || n < 1) return DSPW_ERR_ARG;
  t->n = 0;
  int r = ensure_cap(t, n);
  if (r) return r;
  double *ds = nullptr, *dt = nullptr;
  if (cudaMalloc(&ds, sizeof(double) * 4 * n) != cudaSuccess || cudaMalloc(&dt, sizeof(double) * 2 * n) != cudaSuccess) {
    cudaFree(ds);
    return DSPW_ERR_NOMEM;
  }
  cudaError_t e = cudaMemcpyAsync(ds, stencils, sizeof(double) * 4 * n, cudaMemcpyHostToDevice, t->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dt, targets, sizeof(double) * 2 * n, cudaMemcpyHostToDevice, t->stream);
  if (e == cudaSuccess) {
    k_prepare_f64<<<(int)((n + TPB - 1) / TPB), TPB, 0, t->stream>>>(ds, dt, n, t->data, t->cap, 0);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
  cudaFree(ds);
  cudaFree(dt);
  if (e != cudaSuccess) return DSPW_ERR_CUDA;
  t->n = n;
  return DSPW_OK;
}

int dspw_trainer_collect(dspw_trainer* t, dspw_handle* h, long long max_pairs, long long* added) {
  if (!t || !h || max_pairs < 1) return DSPW_ERR_ARG;
  if (max_pairs > t->pairs_cap) {
    if (t->pairs) cudaFree(t->pairs);
    t->pairs = nullptr;
    if (cudaMalloc(&t->pairs, sizeof(float) * 6 * max_pairs) != cudaSuccess) return DSPW_ERR_NOMEM;
    t->pairs_cap = max_pairs;
  }
  if (!t->pair_count && cudaMalloc(&t->pair_count, sizeof(unsigned long long)) != cudaSuccess) return DSPW_ERR_NOMEM;
  TK(cudaMemset(t->pair_count, 0, sizeof(unsigned long long)));
  // sampling stride: aim at max_pairs reconstructions of the evaluation
  unsigned stride = (unsigned)t->cfg.collect_stride;
  if (stride < 1) stride = 1;
  int r = handle_collect(h, t->pairs, t->pair_count, (unsigned long long)max_pairs, stride);
  if (r) return r;
  unsigned long long cnt = 0;
  TK(cudaMemcpy(&cnt, t->pair_count, sizeof(cnt), cudaMemcpyDeviceToHost));
  long long got = (long long)std::min<unsigned long long>(cnt, (unsigned long long)max_pairs);
  r = ensure_cap(t, t->n + got);
  if (r) return r;
  if (got > 0) {
    k_prepare_pairs<<<(int)((got + TPB - 1) / TPB), TPB, 0, t->stream>>>(t->pairs, got, t->data, t->cap, t->n);
    TK(cudaGetLastError());
    TK(cudaStreamSynchronize(t->stream));
  }
  t->n += got;
  if (added) *added = got;
  return DSPW_OK;
}

int dspw_trainer_epoch(dspw_trainer* t, double* mean_loss) {
  if (!t || t->n < 1) return DSPW_ERR_ARG;
  int B = t->cfg.batch;
  long long nb = t->n / B;
  if (nb < 1) { B = (int)t->n; nb = 1; }
  // random permutation of the samples (DataLoader(shuffle=True) of the trainer)
  std::vector<int> perm(t->n);
  for (long long i = 0; i < t->n; i++) perm[i] = (int)i;
  std::shuffle(perm.begin(), perm.end(), t->rng);
  if (t->perm_cap < t->n) {
    if (t->perm) cudaFree(t->perm);
    if (cudaMalloc(&t->perm, sizeof(int) * t->n) != cudaSuccess) return DSPW_ERR_NOMEM;
    t->perm_cap = t->n;
  }
  TK(cudaMemcpyAsync(t->perm, perm.data(), sizeof(int) * t->n, cudaMemcpyHostToDevice, t->stream));
  TK(cudaMemsetAsync(t->loss, 0, sizeof(double), t->stream));
  const dspw_train_cfg& c = t->cfg;
  for (long long b = 0; b < nb; b++) {
    int r = fwd_bwd(t, t->perm, b * B, B, t->prm);
    if (r) return r;
    t->step++;
    k_adam<<<1, 128, 0, t->stream>>>(t->prm, t->grad, t->m, t->v, t->step, (float)c.lr, (float)c.beta1,
                                     (float)c.beta2, (float)c.weight_decay, (float)c.eps);
    TK(cudaGetLastError());
  }
  double lsum = 0;
  TK(cudaMemcpyAsync(&lsum, t->loss, sizeof(double), cudaMemcpyDeviceToHost, t->stream));
  TK(cudaStreamSynchronize(t->stream));
  if (mean_loss) *mean_loss = lsum / (double)nb;
  return DSPW_OK;
}

int dspw_trainer_loss_grad(dspw_trainer* t, const double* stencils, const double* targets, int n, double* loss,
                           double* grad_w, double* grad_b) {
  if (!t || !stencils || !targets || n < 1 || !loss) return DSPW_ERR_ARG;
  // evaluated on a scratch copy so the training data stays untouched
  long long keep_n = t->n;
  float* keep_data = t->data;
  long long keep_cap = t->cap;
  t->data = nullptr;
  t->cap = 0;
  t->n = 0;
  int r = dspw_trainer_set_data(t, stencils, targets, n);
  if (r == DSPW_OK) {
    cudaMemsetAsync(t->loss, 0, sizeof(double), t->stream);
    r = fwd_bwd(t, nullptr, 0, n, t->prm);
  }
  double g[NPARAM], l = 0;
  if (r == DSPW_OK) {
    if (cudaMemcpyAsync(g, t->grad, sizeof(g), cudaMemcpyDeviceToHost, t->stream) != cudaSuccess ||
        cudaMemcpyAsync(&l, t->loss, sizeof(double), cudaMemcpyDeviceToHost, t->stream) != cudaSuccess ||
        cudaStreamSynchronize(t->stream) != cudaSuccess)
      r = DSPW_ERR_CUDA;
  }
  if (t->data) cudaFree(t->data);
  t->data = keep_data;
  t->cap = keep_cap;
  t->n = keep_n;
  if (r) return r;
  *loss = l;
  if (grad_w) memcpy(grad_w, g, sizeof(double) * 100);
  if (grad_b) memcpy(grad_b, g + 100, sizeof(double) * 20);
  return DSPW_OK;
}

int dspw_trainer_eval(dspw_trainer* t, double* mean_loss) {
  if (!t || !mean_loss || t->n < 1) return DSPW_ERR_ARG;
  int B = (int)std::min<long long>(t->n, 1 << 20);
  long long nb = (t->n + B - 1) / B;
  TK(cudaMemsetAsync(t->loss, 0, sizeof(double), t->stream));
  double total = 0.0;
  for (long long k = 0; k < nb; k++) {
    int Bk = (int)std::min<long long>(B, t->n - k * B);
    TK(cudaMemsetAsync(t->loss, 0, sizeof(double), t->stream));
    int r = fwd_bwd(t, nullptr, k * B, Bk, t->prm);
    if (r) return r;
    double l = 0;
    TK(cudaMemcpyAsync(&l, t->loss, sizeof(double), cudaMemcpyDeviceToHost, t->stream));
    TK(cudaStreamSynchronize(t->stream));
    total += l * Bk;
  }
  *mean_loss = total / (double)t->n;
  return DSPW_OK;
}

int dspw_trainer_get_params(dspw_trainer* t, double* w, double* b) {
  if (!t || !w || !b) return DSPW_ERR_ARG;
  float h[NPARAM];
  if (cudaMemcpy(h, t->prm, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return DSPW_ERR_CUDA;
  for (int k = 0; k < 100; k++) w[k] = h[k];
  for (int k = 0; k < 20; k++) b[k] = h[100 + k];
  return DSPW_OK;
}

int dspw_trainer_export(dspw_trainer* t, double* rows, long long max_rows, long long* nrows) {
  if (!t || !nrows || max_rows < 0 || (max_rows > 0 && !rows)) return DSPW_ERR_ARG;
  *nrows = 0;
  if (t->n == 0) return DSPW_OK;
  double* dout = nullptr;
  int* dvalid = nullptr;
  if (cudaMalloc(&dout, sizeof(double) * EXPORT_COLS * t->n) != cudaSuccess ||
      cudaMalloc(&dvalid, sizeof(int) * t->n) != cudaSuccess) {
    if (dout) cudaFree(dout);
    return DSPW_ERR_CUDA;
  }
  std::vector<double> h((size_t)EXPORT_COLS * t->n);
  std::vector<int> valid(t->n);
  k_export_rows<<<(int)((t->n + TPB - 1) / TPB), TPB, 0, t->stream>>>(t->data, t->cap, t->n, dout, dvalid);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h.data(), dout, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, t->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(valid.data(), dvalid, sizeof(int) * t->n, cudaMemcpyDeviceToHost, t->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
  cudaFree(dout);
  cudaFree(dvalid);
  if (e != cudaSuccess) return DSPW_ERR_CUDA;
  long long k = 0;
  for (long long i = 0; i < t->n; i++) {
    if (!valid[i]) continue;
    if (rows && k < max_rows) memcpy(rows + EXPORT_COLS * k, &h[(size_t)EXPORT_COLS * i], sizeof(double) * EXPORT_COLS);
    k++;
  }
  *nrows = rows ? std::min(k, max_rows) : k;
  return DSPW_OK;
}

int dspw_trainer_info(dspw_trainer* t, long long* nsamples, double* feature_max) {
  if (!t) return DSPW_ERR_ARG;
  if (nsamples) *nsamples = t->n;
  if (feature_max) {
    unsigned* d = nullptr;
    unsigned hmax[5] = {0, 0, 0, 0, 0};
    if (cudaMalloc(&d, sizeof(hmax)) != cudaSuccess) return DSPW_ERR_NOMEM;
    cudaMemset(d, 0, sizeof(hmax));
    if (t->n > 0) k_feature_max<<<(int)((t->n + TPB - 1) / TPB), TPB, 0, t->stream>>>(t->data, t->cap, t->n, d);
    cudaError_t e = cudaMemcpyAsync(hmax, d, sizeof(hmax), cudaMemcpyDeviceToHost, t->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
    cudaFree(d);
    if (e != cudaSuccess) return DSPW_ERR_CUDA;
    for (int k = 0; k < 5; k++) {
      float f;
      memcpy(&f, &hmax[k], sizeof(f));
      feature_max[k] = f;
    }
  }
  return DSPW_OK;
}

int dspw_trainer_box(dspw_trainer* t, double lo[5], double hi[5]) {
  if (!t || !lo || !hi || t->n < 1) return DSPW_ERR_ARG;
  unsigned* d = nullptr;
  unsigned h[10];
  for (int k = 0; k < 5; k++) { h[k] = 0xffffffffu; h[5 + k] = 0u; }
  if (cudaMalloc(&d, sizeof(h)) != cudaSuccess) return DSPW_ERR_NOMEM;
  cudaError_t e = cudaMemcpyAsync(d, h, sizeof(h), cudaMemcpyHostToDevice, t->stream);
  if (e == cudaSuccess) {
    k_feature_box<<<(int)((t->n + TPB - 1) / TPB), TPB, 0, t->stream>>>(t->data, t->cap, t->n, d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, t->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
  cudaFree(d);
  if (e != cudaSuccess) return DSPW_ERR_CUDA;
  if (h[0] == 0xffffffffu) return DSPW_ERR_ARG;   // no valid sample
  for (int k = 0; k < 5; k++) {
    lo[k] = key_float(h[k]);
    hi[k] = key_float(h[5 + k]);
  }
  return DSPW_OK;
}

}  // extern "C"

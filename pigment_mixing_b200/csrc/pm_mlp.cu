// Learned return-map surrogate: a 10 -> 64 -> 64 -> 6 GELU MLP.
//
//   training   FP32 kernels written here: dense forward, backward (input, weight and bias
//              gradients), mean-squared-error loss, Adam.  Inputs and targets are normalised with
//              the training set's mean and standard deviation, which travel with the weights.
//   inference  BF16 tensor cores (mma.sync m16n8k16, FP32 accumulation): one warp per 16
//              samples; layer outputs stay in registers and are re-used directly as the next
//              layer's A fragments.
//
// Parameter vector (float, PM_MLP_NPARAMS entries), the layout every entry point uses:
//   in_mean[10] in_std[10] out_mean[6] out_std[6] W1[64][10] b1[64] W2[64][64] b2[64] W3[6][64] b3[6]
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "pm_internal.cuh"
#include "pm_launch.h"
#include "pm_mlp.h"

namespace pm {

// ------------------------------------------------------------------------------------------
// helpers
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ float gelu(float x) {  // tanh form of GELU
  const float k0 = 0.7978845608028654f, k1 = 0.044715f;
  return 0.5f * x * (1.f + tanhf(k0 * (x + k1 * x * x * x)));
}
// Inference form: the SFU's tanh.approx.f32 (activations are rounded to bf16 right after).
__device__ __forceinline__ float gelu_fast(float x) {
  const float k0 = 0.7978845608028654f, k1 = 0.044715f;
  const float u = k0 * (x + k1 * x * x * x);
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
  return 0.5f * x * (1.f + t);
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float k0 = 0.7978845608028654f, k1 = 0.044715f;
  const float u = k0 * (x + k1 * x * x * x);
  const float t = tanhf(u);
  return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * k0 * (1.f + 3.f * k1 * x * x);
}

// ------------------------------------------------------------------------------------------
// FP32 training kernels
// ------------------------------------------------------------------------------------------
// Z[b][n] = sum_k X[b][k] W[n][k] + bias[n]; H = gelu(Z) when act (Z kept for backward).
__global__ void k_dense_fwd(const float* X, const float* W, const float* bias, float* Z, float* H, int B, int K, int N,
                            int act) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B * N) return;
  const int b = i / N, n = i - b * N;
  const float* x = X + (size_t)b * K;
  const float* w = W + (size_t)n * K;
  float s = bias[n];
  for (int k = 0; k < K; ++k) s += x[k] * w[k];
  Z[i] = s;
  if (H) H[i] = act ? gelu(s) : s;
}

// normalise: Xn = (X - mean) / std
__global__ void k_normalise(const float* X, const float* mean, const float* stdv, float* Xn, int B, int K) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B * K) return;
  const int k = i % K;
  Xn[i] = (X[i] - mean[k]) / stdv[k];
}

// loss = mean over batch and outputs of (Y - T)^2 ; dY = 2 (Y - T) / (B * N); T normalised here
__global__ void k_mse(const float* Y, const float* T, const float* tmean, const float* tstd, float* dY, float* loss,
                      int B, int N) {
  __shared__ float red[256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float v = 0.f;
  if (i < B * N) {
    const int n = i % N;
    const float t = (T[i] - tmean[n]) / tstd[n];
    const float d = Y[i] - t;
    v = d * d;
    dY[i] = 2.f * d / (float)(B * N);
  }
  red[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0] / (float)(B * N));
}

// dZ = dH * gelu'(Z)
__global__ void k_gelu_back(const float* dH, const float* Z, float* dZ, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dZ[i] = dH[i] * gelu_grad(Z[i]);
}

// dX[b][k] = sum_n dZ[b][n] W[n][k]
__global__ void k_dense_bwd_x(const float* dZ, const float* W, float* dX, int B, int K, int N) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B * K) return;
  const int b = i / K, k = i - b * K;
  const float* dz = dZ + (size_t)b * N;
  float s = 0.f;
  for (int n = 0; n < N; ++n) s += dz[n] * W[(size_t)n * K + k];
  dX[i] = s;
}

// dW[n][k] += sum_b dZ[b][n] X[b][k] ; db[n] += sum_b dZ[b][n].  Each block sums a slice of the
// batch in registers and adds its partial once per weight.
constexpr int kRowsPerBlock = 256;
__global__ void k_dense_bwd_w(const float* dZ, const float* X, float* dW, float* db, int B, int K, int N) {
  const int b0 = blockIdx.x * kRowsPerBlock;
  const int b1 = min(b0 + kRowsPerBlock, B);
  for (int e = threadIdx.x; e < N * (K + 1); e += blockDim.x) {
    const int n = e / (K + 1), k = e - n * (K + 1);
    float s = 0.f;
    if (k < K) {
      for (int b = b0; b < b1; ++b) s += dZ[(size_t)b * N + n] * X[(size_t)b * K + k];
      atomicAdd(&dW[(size_t)n * K + k], s);
    } else {
      for (int b = b0; b < b1; ++b) s += dZ[(size_t)b * N + n];
      atomicAdd(&db[n], s);
    }
  }
}

__global__ void k_adam(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  m[i] = b1 * m[i] + (1.f - b1) * gi;
  v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
  p[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}

// ------------------------------------------------------------------------------------------
// BF16 tensor-core inference
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// Shared-memory row strides of the staged weights (bf16 elements).  Rows are padded so that the
// eight rows a B-fragment load touches (lane group g) fall in distinct banks: 24 and 72 elements
// are 12 and 36 words, i.e. 12 g and 4 g (mod 32) for g = 0..7.
constexpr int kW1Ld = 24, kW2Ld = 72, kW3Ld = 72;

// Warp-level forward pass of 16 samples (rows of xs[16][16], bf16, normalised, zero padded)
// producing ys[16][8] (FP32, normalised outputs in columns 0..5).  Weights in shared memory:
// W1s[64][kW1Ld], W2s[64][kW2Ld], W3s[8][kW3Ld] bf16 (row n = output, k contiguous), biases FP32.
__device__ void mlp_warp16(const MlpDev& w, const __nv_bfloat16* xs, float* ys) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  // layer 1 A fragment from xs (row-major 16 x 16)
  uint32_t a[4];
  {
    const uint32_t* x32 = reinterpret_cast<const uint32_t*>(xs);  // 8 words per row
    a[0] = x32[g * 8 + t];
    a[1] = x32[(g + 8) * 8 + t];
    a[2] = x32[g * 8 + 4 + t];
    a[3] = x32[(g + 8) * 8 + 4 + t];
  }
  float h1[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int n = nt * 8 + g;
    const uint32_t* wr = reinterpret_cast<const uint32_t*>(w.W1 + n * kW1Ld);
    const uint32_t b[2] = {wr[t], wr[4 + t]};
    const float bias0 = w.b1[nt * 8 + 2 * t], bias1 = w.b1[nt * 8 + 2 * t + 1];
    h1[nt][0] = bias0; h1[nt][1] = bias1; h1[nt][2] = bias0; h1[nt][3] = bias1;
    mma_bf16(h1[nt], a, b);
#pragma unroll
    for (int r = 0; r < 4; ++r) h1[nt][r] = gelu_fast(h1[nt][r]);
  }
  // layer 2: A fragments of k-step j from h1 tiles 2j and 2j+1
  float h2[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float bias0 = w.b2[nt * 8 + 2 * t], bias1 = w.b2[nt * 8 + 2 * t + 1];
    h2[nt][0] = bias0; h2[nt][1] = bias1; h2[nt][2] = bias0; h2[nt][3] = bias1;
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const uint32_t aj[4] = {pack_bf16(h1[2 * j][0], h1[2 * j][1]), pack_bf16(h1[2 * j][2], h1[2 * j][3]),
                            pack_bf16(h1[2 * j + 1][0], h1[2 * j + 1][1]), pack_bf16(h1[2 * j + 1][2], h1[2 * j + 1][3])};
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const uint32_t* wr = reinterpret_cast<const uint32_t*>(w.W2 + (nt * 8 + g) * kW2Ld + 16 * j);
      const uint32_t b[2] = {wr[t], wr[4 + t]};
      mma_bf16(h2[nt], aj, b);
    }
  }
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int r = 0; r < 4; ++r) h2[nt][r] = gelu_fast(h2[nt][r]);
  // layer 3 (outputs padded to 8)
  float y[4];
  {
    const float bias0 = w.b3[2 * t], bias1 = w.b3[2 * t + 1];
    y[0] = bias0; y[1] = bias1; y[2] = bias0; y[3] = bias1;
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const uint32_t aj[4] = {pack_bf16(h2[2 * j][0], h2[2 * j][1]), pack_bf16(h2[2 * j][2], h2[2 * j][3]),
                            pack_bf16(h2[2 * j + 1][0], h2[2 * j + 1][1]), pack_bf16(h2[2 * j + 1][2], h2[2 * j + 1][3])};
    const uint32_t* wr = reinterpret_cast<const uint32_t*>(w.W3 + g * kW3Ld + 16 * j);
    const uint32_t b[2] = {wr[t], wr[4 + t]};
    mma_bf16(y, aj, b);
  }
  ys[g * 8 + 2 * t] = y[0];
  ys[g * 8 + 2 * t + 1] = y[1];
  ys[(g + 8) * 8 + 2 * t] = y[2];
  ys[(g + 8) * 8 + 2 * t + 1] = y[3];
}

// Copies the inference weights into shared memory (bf16 matrices, FP32 biases and statistics).
__device__ MlpDev mlp_stage(const MlpDev& gw, unsigned char* smem) {
  MlpDev w;
  __nv_bfloat16* W1 = reinterpret_cast<__nv_bfloat16*>(smem);
  __nv_bfloat16* W2 = W1 + 64 * kW1Ld;
  __nv_bfloat16* W3 = W2 + 64 * kW2Ld;
  float* f = reinterpret_cast<float*>(W3 + 8 * kW3Ld);
  for (int i = threadIdx.x; i < 64 * 16; i += blockDim.x) W1[(i >> 4) * kW1Ld + (i & 15)] = gw.W1[i];
  for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x) W2[(i >> 6) * kW2Ld + (i & 63)] = gw.W2[i];
  for (int i = threadIdx.x; i < 8 * 64; i += blockDim.x) W3[(i >> 6) * kW3Ld + (i & 63)] = gw.W3[i];
  float* b1 = f;
  float* b2 = b1 + 64;
  float* b3 = b2 + 64;
  float* st = b3 + 8;
  for (int i = threadIdx.x; i < 64; i += blockDim.x) { b1[i] = gw.b1[i]; b2[i] = gw.b2[i]; }
  for (int i = threadIdx.x; i < 8; i += blockDim.x) b3[i] = gw.b3[i];
  for (int i = threadIdx.x; i < 32; i += blockDim.x) st[i] = gw.stats[i];
  __syncthreads();
  w.W1 = W1; w.W2 = W2; w.W3 = W3; w.b1 = b1; w.b2 = b2; w.b3 = b3; w.stats = st;
  return w;
}

// Inference over rows X[n][10] (raw features) -> Y[n][6] (raw outputs), one warp per 16 rows.
// The row count is read from *n_dev when it is not null (graph-friendly), else n is used.
constexpr int kMlpThreads = 128;
constexpr int kMlpWarps = kMlpThreads / 32;
__host__ __device__ constexpr size_t mlp_weights_smem() {
  return (((64 * kW1Ld + 64 * kW2Ld + 8 * kW3Ld) * 2 + (64 + 64 + 8 + 32) * 4) + 15) / 16 * 16;
}
size_t mlp_stage_bytes() { return mlp_weights_smem(); }
size_t mlp_infer_smem_bytes() { return mlp_weights_smem() + kMlpWarps * (256 * 2 + 128 * 4); }

__device__ __forceinline__ void d_mlp_infer(const MlpDev& gw, const float* X, float* Y, int n, const int blk_,
                                            const int nblk_) {
  extern __shared__ __align__(16) unsigned char smem[];
  MlpDev w = mlp_stage(gw, smem);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __nv_bfloat16* xs = reinterpret_cast<__nv_bfloat16*>(smem + mlp_weights_smem()) + warp * 256;
  float* ys = reinterpret_cast<float*>(smem + mlp_weights_smem() + kMlpWarps * 256 * 2) + warp * 128;
  const float* mean = w.stats;
  const float* sd = w.stats + 10;
  const float* omean = w.stats + 20;
  const float* osd = w.stats + 26;
  const int warps = nblk_ * kMlpWarps;
  for (int r0 = (blk_ * kMlpWarps + warp) * 16; r0 < n; r0 += warps * 16) {
    for (int e = lane; e < 256; e += 32) {
      const int r = e >> 4, k = e & 15;
      float v = 0.f;
      if (k < 10 && r0 + r < n) v = __fdividef(X[(size_t)(r0 + r) * 10 + k] - mean[k], sd[k]);
      xs[e] = __float2bfloat16_rn(v);
    }
    __syncwarp();
    mlp_warp16(w, xs, ys);
    __syncwarp();
    for (int e = lane; e < 96; e += 32) {
      const int r = e / 6, k = e - r * 6;
      if (r0 + r < n) Y[(size_t)(r0 + r) * 6 + k] = ys[r * 8 + k] * osd[k] + omean[k];
    }
    __syncwarp();
  }
}

__global__ void __launch_bounds__(kMlpThreads) k_mlp_infer(MlpDev gw, const float* X, float* Y, int n,
                                                           const uint32_t* n_dev) {
  if (n_dev) n = (int)*n_dev;
  d_mlp_infer(gw, X, Y, n, blockIdx.x, gridDim.x);
}

// Batched form: scene s infers its own queue (row count from its control block).
__global__ void __launch_bounds__(kMlpThreads) kb_mlp_infer(const SceneDev* __restrict__ sd, const int* __restrict__ off,
                                                            int ns) {
  int s_, blk_, nblk_;
  batch_slot(off, ns, s_, blk_, nblk_);
  const SceneDev& d = sd[s_];
  const Bufs& B = d.B[scene_parity(d)];
  const Ctrl* c = B.ctrl;
  if (d.P.return_map != 1 || c->halt || c->idle) return;
  d_mlp_infer(B.mlp, B.qx, B.qy, (int)c->q_n, blk_, nblk_);
}

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
namespace {
constexpr int O_IM = 0, O_IS = 10, O_OM = 20, O_OS = 26, O_W1 = 32, O_B1 = O_W1 + 640, O_W2 = O_B1 + 64,
              O_B2 = O_W2 + 4096, O_W3 = O_B2 + 64, O_B3 = O_W3 + 384;
static_assert(O_B3 + 6 == PM_MLP_NPARAMS_CONST, "parameter layout");

struct TrainBufs {
  float *X = nullptr, *T = nullptr, *Xn = nullptr, *Z1 = nullptr, *H1 = nullptr, *Z2 = nullptr, *H2 = nullptr,
        *Y = nullptr, *dY = nullptr, *dH2 = nullptr, *dZ2 = nullptr, *dH1 = nullptr, *dZ1 = nullptr, *P = nullptr,
        *G = nullptr, *M = nullptr, *V = nullptr, *loss = nullptr;
  ~TrainBufs() {
    float* all[] = {X, T, Xn, Z1, H1, Z2, H2, Y, dY, dH2, dZ2, dH1, dZ1, P, G, M, V, loss};
    for (float* p : all)
      if (p) cudaFree(p);
  }
};

cudaError_t alloc_train(TrainBufs& b, int B) {
  cudaError_t e;
#define A_(ptr, n) if ((e = cudaMalloc(&b.ptr, sizeof(float) * (size_t)(n))) != cudaSuccess) return e
  A_(X, B * 10); A_(T, B * 6); A_(Xn, B * 10); A_(Z1, B * 64); A_(H1, B * 64); A_(Z2, B * 64); A_(H2, B * 64);
  A_(Y, B * 6); A_(dY, B * 6); A_(dH2, B * 64); A_(dZ2, B * 64); A_(dH1, B * 64); A_(dZ1, B * 64);
  A_(P, PM_MLP_NPARAMS_CONST); A_(G, PM_MLP_NPARAMS_CONST); A_(M, PM_MLP_NPARAMS_CONST); A_(V, PM_MLP_NPARAMS_CONST);
  A_(loss, 1);
#undef A_
  return cudaSuccess;
}

// forward + backward of one batch already staged in b.X / b.T; gradient in b.G (zeroed here)
cudaError_t loss_grad_batch(TrainBufs& b, int B, cudaStream_t s) {
  const int T = 256;
  auto g = [&](int n) { return (n + T - 1) / T; };
  const float* P = b.P;
  cudaMemsetAsync(b.G, 0, sizeof(float) * PM_MLP_NPARAMS_CONST, s);
  cudaMemsetAsync(b.loss, 0, sizeof(float), s);
  k_normalise<<<g(B * 10), T, 0, s>>>(b.X, P + O_IM, P + O_IS, b.Xn, B, 10);
  k_dense_fwd<<<g(B * 64), T, 0, s>>>(b.Xn, P + O_W1, P + O_B1, b.Z1, b.H1, B, 10, 64, 1);
  k_dense_fwd<<<g(B * 64), T, 0, s>>>(b.H1, P + O_W2, P + O_B2, b.Z2, b.H2, B, 64, 64, 1);
  k_dense_fwd<<<g(B * 6), T, 0, s>>>(b.H2, P + O_W3, P + O_B3, b.Y, nullptr, B, 64, 6, 0);
  k_mse<<<g(B * 6), T, 0, s>>>(b.Y, b.T, P + O_OM, P + O_OS, b.dY, b.loss, B, 6);
  const int wb = (B + kRowsPerBlock - 1) / kRowsPerBlock;
  k_dense_bwd_w<<<wb, T, 0, s>>>(b.dY, b.H2, b.G + O_W3, b.G + O_B3, B, 64, 6);
  k_dense_bwd_x<<<g(B * 64), T, 0, s>>>(b.dY, P + O_W3, b.dH2, B, 64, 6);
  k_gelu_back<<<g(B * 64), T, 0, s>>>(b.dH2, b.Z2, b.dZ2, B * 64);
  k_dense_bwd_w<<<wb, T, 0, s>>>(b.dZ2, b.H1, b.G + O_W2, b.G + O_B2, B, 64, 64);
  k_dense_bwd_x<<<g(B * 64), T, 0, s>>>(b.dZ2, P + O_W2, b.dH1, B, 64, 64);
  k_gelu_back<<<g(B * 64), T, 0, s>>>(b.dH1, b.Z1, b.dZ1, B * 64);
  k_dense_bwd_w<<<wb, T, 0, s>>>(b.dZ1, b.Xn, b.G + O_W1, b.G + O_B1, B, 10, 64);
  return cudaGetLastError();
}
}  // namespace

cudaError_t mlp_loss_grad(const float* params, const float* x, const float* y, int n, float* loss, float* grad) {
  TrainBufs b;
  cudaError_t e = alloc_train(b, n);
  if (e != cudaSuccess) return e;
  cudaMemcpy(b.P, params, sizeof(float) * PM_MLP_NPARAMS_CONST, cudaMemcpyHostToDevice);
  cudaMemcpy(b.X, x, sizeof(float) * 10 * (size_t)n, cudaMemcpyHostToDevice);
  cudaMemcpy(b.T, y, sizeof(float) * 6 * (size_t)n, cudaMemcpyHostToDevice);
  e = loss_grad_batch(b, n, 0);
  if (e != cudaSuccess) return e;
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return e;
  cudaMemcpy(loss, b.loss, sizeof(float), cudaMemcpyDeviceToHost);
  if (grad) {
    cudaMemcpy(grad, b.G, sizeof(float) * PM_MLP_NPARAMS_CONST, cudaMemcpyDeviceToHost);
    for (int i = 0; i < 32; ++i) grad[i] = 0.f;  // statistics are not trained
  }
  return cudaGetLastError();
}

void mlp_init_params(float* p, const float* x, const float* y, int n, uint64_t seed) {
  std::memset(p, 0, sizeof(float) * PM_MLP_NPARAMS_CONST);
  for (int k = 0; k < 10; ++k) {
    double s = 0, s2 = 0;
    for (int i = 0; i < n; ++i) { s += x[(size_t)i * 10 + k]; s2 += (double)x[(size_t)i * 10 + k] * x[(size_t)i * 10 + k]; }
    const double m = n ? s / n : 0.0, var = n ? s2 / n - m * m : 1.0;
    p[O_IM + k] = (float)m;
    p[O_IS + k] = (float)(var > 1e-20 ? std::sqrt(var) : 1.0);
  }
  for (int k = 0; k < 6; ++k) {
    double s = 0, s2 = 0;
    for (int i = 0; i < n; ++i) { s += y[(size_t)i * 6 + k]; s2 += (double)y[(size_t)i * 6 + k] * y[(size_t)i * 6 + k]; }
    const double m = n ? s / n : 0.0, var = n ? s2 / n - m * m : 1.0;
    p[O_OM + k] = (float)m;
    p[O_OS + k] = (float)(var > 1e-30 ? std::sqrt(var) : 1.0);
  }
  std::mt19937_64 rng(seed);
  auto fill = [&](int off, int fan_in, int count) {
    std::normal_distribution<float> nd(0.f, (float)std::sqrt(2.0 / fan_in));
    for (int i = 0; i < count; ++i) p[off + i] = nd(rng);
  };
  fill(O_W1, 10, 640);
  fill(O_W2, 64, 4096);
  fill(O_W3, 64, 384);
}

cudaError_t mlp_train(const float* x, const float* y, int n, const pm_mlp_train_opts& o, float* params,
                      float* loss_hist, int* steps_done) {
  const int B = std::max(1, std::min(o.batch, n));
  TrainBufs b;
  cudaError_t e = alloc_train(b, B);
  if (e != cudaSuccess) return e;
  float* dX = nullptr;
  float* dT = nullptr;
  if ((e = cudaMalloc(&dX, sizeof(float) * 10 * (size_t)n)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&dT, sizeof(float) * 6 * (size_t)n)) != cudaSuccess) { cudaFree(dX); return e; }
  cudaMemcpy(dX, x, sizeof(float) * 10 * (size_t)n, cudaMemcpyHostToDevice);
  cudaMemcpy(dT, y, sizeof(float) * 6 * (size_t)n, cudaMemcpyHostToDevice);
  if (!o.resume) mlp_init_params(params, x, y, n, o.seed);
  cudaMemcpy(b.P, params, sizeof(float) * PM_MLP_NPARAMS_CONST, cudaMemcpyHostToDevice);
  cudaMemset(b.M, 0, sizeof(float) * PM_MLP_NPARAMS_CONST);
  cudaMemset(b.V, 0, sizeof(float) * PM_MLP_NPARAMS_CONST);
  std::mt19937_64 rng(o.seed ^ 0x9e3779b97f4a7c15ULL);
  const int nb = std::max(1, n / B);
  int step = 0;
  const float b1 = 0.9f, b2 = 0.999f;
  double c1 = 1.0, c2 = 1.0;
  for (int ep = 0; ep < o.epochs; ++ep) {
    const int off0 = (int)(rng() % (uint64_t)std::max(1, n - B + 1));
    double ep_loss = 0.0;
    for (int bi = 0; bi < nb; ++bi) {
      const int off = (off0 + bi * B) % std::max(1, n - B + 1);
      cudaMemcpyAsync(b.X, dX + (size_t)off * 10, sizeof(float) * 10 * B, cudaMemcpyDeviceToDevice, 0);
      cudaMemcpyAsync(b.T, dT + (size_t)off * 6, sizeof(float) * 6 * B, cudaMemcpyDeviceToDevice, 0);
      e = loss_grad_batch(b, B, 0);
      if (e != cudaSuccess) break;
      ++step;
      c1 *= b1;
      c2 *= b2;
      const float lr = o.lr * (float)(0.5 * (1.0 + std::cos(M_PI * (double)step / (double)(o.epochs * nb))));
      // statistics (first 32 entries) are not trained
      k_adam<<<(PM_MLP_NPARAMS_CONST - 32 + 255) / 256, 256>>>(b.P + 32, b.G + 32, b.M + 32, b.V + 32,
                                                               PM_MLP_NPARAMS_CONST - 32, lr, b1, b2, 1e-8f,
                                                               (float)(1.0 - c1), (float)(1.0 - c2));
      float l = 0.f;
      cudaMemcpy(&l, b.loss, sizeof(float), cudaMemcpyDeviceToHost);
      ep_loss += l;
    }
    if (e != cudaSuccess) break;
    if (loss_hist) loss_hist[ep] = (float)(ep_loss / nb);
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaMemcpy(params, b.P, sizeof(float) * PM_MLP_NPARAMS_CONST, cudaMemcpyDeviceToHost);
  cudaFree(dX);
  cudaFree(dT);
  if (steps_done) *steps_done = step;
  return e;
}

cudaError_t mlp_upload(const float* params, MlpDev& dev, void** storage) {
  // device layout: bf16 W1p[64][16], W2[64][64], W3p[8][64] | float b1[64] b2[64] b3[8] stats[32]
  std::vector<__nv_bfloat16> wb(64 * 16 + 64 * 64 + 8 * 64, __float2bfloat16(0.f));
  for (int n = 0; n < 64; ++n)
    for (int k = 0; k < 10; ++k) wb[n * 16 + k] = __float2bfloat16(params[O_W1 + n * 10 + k]);
  for (int i = 0; i < 4096; ++i) wb[64 * 16 + i] = __float2bfloat16(params[O_W2 + i]);
  for (int n = 0; n < 6; ++n)
    for (int k = 0; k < 64; ++k) wb[64 * 16 + 4096 + n * 64 + k] = __float2bfloat16(params[O_W3 + n * 64 + k]);
  std::vector<float> fb(64 + 64 + 8 + 32, 0.f);
  for (int i = 0; i < 64; ++i) { fb[i] = params[O_B1 + i]; fb[64 + i] = params[O_B2 + i]; }
  for (int i = 0; i < 6; ++i) fb[128 + i] = params[O_B3 + i];
  for (int i = 0; i < 32; ++i) fb[136 + i] = params[i];
  const size_t wbytes = wb.size() * sizeof(__nv_bfloat16), fbytes = fb.size() * sizeof(float);
  if (*storage == nullptr) {
    cudaError_t e = cudaMalloc(storage, wbytes + fbytes);
    if (e != cudaSuccess) return e;
  }
  unsigned char* base = static_cast<unsigned char*>(*storage);
  cudaMemcpy(base, wb.data(), wbytes, cudaMemcpyHostToDevice);
  cudaMemcpy(base + wbytes, fb.data(), fbytes, cudaMemcpyHostToDevice);
  dev.W1 = reinterpret_cast<const __nv_bfloat16*>(base);
  dev.W2 = dev.W1 + 64 * 16;
  dev.W3 = dev.W2 + 64 * 64;
  const float* f = reinterpret_cast<const float*>(base + wbytes);
  dev.b1 = f;
  dev.b2 = f + 64;
  dev.b3 = f + 128;
  dev.stats = f + 136;
  return cudaGetLastError();
}

cudaError_t mlp_init() {
  cudaError_t e = cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)mlp_infer_smem_bytes());
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(kb_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp_infer_smem_bytes());
}

void mlp_infer_batched(const SceneDev* sd, const int* off, int ns, int ctas, cudaStream_t s) {
  kb_mlp_infer<<<ctas, kMlpThreads, mlp_infer_smem_bytes(), s>>>(sd, off, ns);
}

cudaError_t mlp_infer(const MlpDev& dev, const float* dX, float* dY, int n, const uint32_t* n_dev, int max_rows,
                      cudaStream_t s) {
  const int rows = n_dev ? max_rows : n;
  if (rows <= 0) return cudaSuccess;
  const int blocks = std::max(1, std::min(148 * 8, (rows + 16 * kMlpWarps - 1) / (16 * kMlpWarps)));
  k_mlp_infer<<<blocks, kMlpThreads, mlp_infer_smem_bytes(), s>>>(dev, dX, dY, n, n_dev);
  return cudaGetLastError();
}

}  // namespace pm

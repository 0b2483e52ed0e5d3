// Return-map surrogate MLP (10 -> 64 -> 64 -> 6, GELU): FP32 training kernels and BF16
// tensor-core inference (pm_mlp.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#define PM_MLP_NPARAMS_CONST 5286

namespace pm {

// Device-side inference weights: bf16 matrices (row = output, padded to 16/64/8), FP32 biases
// and the normalisation statistics (in_mean[10] in_std[10] out_mean[6] out_std[6]).
struct MlpDev {
  const __nv_bfloat16 *W1, *W2, *W3;
  const float *b1, *b2, *b3, *stats;
};

struct pm_mlp_train_opts {
  int epochs;
  int batch;
  float lr;
  uint64_t seed;
  int resume;  // 1: start from the given parameters; 0: initialise (statistics from the data)
};

cudaError_t mlp_loss_grad(const float* params, const float* x, const float* y, int n, float* loss, float* grad);
cudaError_t mlp_train(const float* x, const float* y, int n, const pm_mlp_train_opts& o, float* params,
                      float* loss_hist, int* steps_done);
// One-time kernel attributes (dynamic shared memory of the inference kernel).
cudaError_t mlp_init();
// Converts the parameter vector into the inference layout; allocates *storage on first use.
cudaError_t mlp_upload(const float* params, MlpDev& dev, void** storage);
// Rows X[n][10] -> Y[n][6]; with n_dev the row count is read on the device (max_rows bounds it).
cudaError_t mlp_infer(const MlpDev& dev, const float* dX, float* dY, int n, const uint32_t* n_dev, int max_rows,
                      cudaStream_t s);

}  // namespace pm

// Host-side launchers of the step kernels (pm_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include "pm_internal.cuh"

namespace pm {

cudaError_t launch_init(int device);
int num_sms();
int kernels_per_step(const Params& P);
const char* kernel_name(int i, const Params& P);
size_t p2g_smem_bytes();
size_t g2p_smem_bytes();
// One full step on stream s; with ev, events before and after every kernel (kernels_per_step + 1).
void launch_step(const Params& P, const Bufs& B, cudaStream_t s, cudaEvent_t* ev = nullptr);
void launch_reduce_state(const Params& P, const float* pcur, const uint32_t* meta, Ctrl* ctrl, cudaStream_t s);
void launch_unpermute(const Params& P, const float* pcur, const uint32_t* meta, float* out, uint8_t* active,
                      cudaStream_t s);
void launch_upload(const Params& P, const float* x, const float* lat, const float* v, float* pbuf, uint32_t* meta,
                   cudaStream_t s);
void launch_stats(const Params& P, const float* pcur, const uint32_t* meta, double* acc, cudaStream_t s);

}  // namespace pm

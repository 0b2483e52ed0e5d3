// Headless pigment volume splat: the renderer's two-pass anisotropic bilateral latent splat onto
// a voxel grid four times finer than its density grid (BinaryDensityGrid::fillRenderGrid,
// raytracing/src/raymarch/BinaryDensityGrid.cpp:153-296), computed from the simulation's device
// state.
//
// Pass 1 accumulates every particle's latent with a Gaussian weight of its anisotropic distance to
// each voxel centre, w = exp(-|G (x - c)|^2 / s^2) for |G (x - c)|^2 <= 9 s^2, and normalises
// (latent / weight, then the four pigment concentrations to sum 1).  Pass 2 repeats the splat with
// the weight multiplied by exp(-d^2 / sc^2), d the distance between the particle's and the voxel's
// pass-1 concentrations (first four latent components), and normalises again.
//
// Layout: one warp per particle, lane per voxel of the particle's (2 ext + 1)^3 search box, so the
// 32 atomics of a warp instruction hit 32 different voxels; two red.global.add.v4.f32 per voxel.
// Warps visit the cell-sorted particles in the order i -> i * SplatGeom::order_stride mod np.
#include <cuda_runtime.h>

#include <cstdint>

#include "pm_internal.cuh"
#include "pm_launch.h"

namespace pm {

namespace {

__device__ __forceinline__ void red_add4(float* addr, float a, float b, float c, float d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
               : "memory");
}

__global__ void k_splat(Params P, const float* pcur, const uint32_t* meta, const float* G, SplatGeom g,
                        const float* cvox, float* acc, int phase) {
  const int S = P.np_stride, np = P.np;
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  const int side = 2 * g.ext + 1, box = side * side * side;
  const float inv_s2 = 1.f / g.sig_s2, inv_c2 = 1.f / g.sig_c2, cut = 9.f * g.sig_s2;
  for (int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < np; t += warps) {
    const int i = (int)(((uint64_t)t * g.order_stride) % (uint32_t)np);
    const uint32_t pid = meta[i] & ~kInactiveBit;
    float x[3], lat[7], Gm[9];
#pragma unroll
    for (int d = 0; d < 3; ++d) x[d] = pcur[(F_X + d) * S + i];
#pragma unroll
    for (int k = 0; k < 7; ++k) lat[k] = pcur[(F_LAT + k) * S + i];
    if (G) {
#pragma unroll
      for (int k = 0; k < 9; ++k) Gm[k] = G[(size_t)pid * 9 + k];
    } else {
#pragma unroll
      for (int k = 0; k < 9; ++k) Gm[k] = (k % 4 == 0) ? g.inv_h : 0.f;
    }
    int base[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) base[d] = (int)floorf((x[d] - g.start[d]) / g.v4 - 0.5f);
    for (int k = lane; k < box; k += 32) {
      const int ox = k % side - g.ext, oy = (k / side) % side - g.ext, oz = k / (side * side) - g.ext;
      const int cx = base[0] + ox, cy = base[1] + oy, cz = base[2] + oz;
      if (cx < 0 || cy < 0 || cz < 0 || cx >= g.dims[0] || cy >= g.dims[1] || cz >= g.dims[2]) continue;
      const float diff[3] = {x[0] - (g.start[0] + ((float)cx + 0.5f) * g.v4),
                             x[1] - (g.start[1] + ((float)cy + 0.5f) * g.v4),
                             x[2] - (g.start[2] + ((float)cz + 0.5f) * g.v4)};
      float d2 = 0.f;
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const float l = Gm[3 * r] * diff[0] + Gm[3 * r + 1] * diff[1] + Gm[3 * r + 2] * diff[2];
        d2 += l * l;
      }
      if (d2 > cut) continue;
      float w = expf(-d2 * inv_s2);
      const size_t idx = (((size_t)cz * g.dims[1] + cy) * g.dims[0] + cx) * 8;
      if (phase == 1) {
        const float4 vc = *reinterpret_cast<const float4*>(cvox + idx);
        const float e0 = lat[0] - vc.x, e1 = lat[1] - vc.y, e2 = lat[2] - vc.z, e3 = lat[3] - vc.w;
        w *= expf(-(e0 * e0 + e1 * e1 + e2 * e2 + e3 * e3) * inv_c2);
      }
      red_add4(acc + idx, lat[0] * w, lat[1] * w, lat[2] * w, lat[3] * w);
      red_add4(acc + idx + 4, lat[4] * w, lat[5] * w, lat[6] * w, w);
    }
  }
}

__global__ void k_splat_normalise(float* acc, size_t nvox) {
  for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < nvox; v += (size_t)gridDim.x * blockDim.x) {
    float4* r = reinterpret_cast<float4*>(acc + v * 8);
    float4 a = r[0], b = r[1];
    const float w = b.w;
    if (!(w > 0.f)) continue;
    a.x /= w; a.y /= w; a.z /= w; a.w /= w;
    b.x /= w; b.y /= w; b.z /= w;
    const float ps = a.x + a.y + a.z + a.w;
    if (ps > 1e-6f) { a.x /= ps; a.y /= ps; a.z /= ps; a.w /= ps; }
    r[0] = a;
    r[1] = b;
  }
}

}  // namespace

cudaError_t launch_splat(const Params& P, const float* pcur, const uint32_t* meta, const float* G, const SplatGeom& g,
                         float* tmp, float* out, cudaStream_t s) {
  const size_t nvox = (size_t)g.dims[0] * g.dims[1] * g.dims[2];
  const int sms = num_sms() > 0 ? num_sms() : 148;
  cudaError_t e = cudaMemsetAsync(tmp, 0, nvox * 8 * sizeof(float), s);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(out, 0, nvox * 8 * sizeof(float), s)) != cudaSuccess) return e;
  k_splat<<<sms * 8, 256, 0, s>>>(P, pcur, meta, G, g, nullptr, tmp, 0);
  k_splat_normalise<<<sms * 8, 256, 0, s>>>(tmp, nvox);
  k_splat<<<sms * 8, 256, 0, s>>>(P, pcur, meta, G, g, tmp, out, 1);
  k_splat_normalise<<<sms * 8, 256, 0, s>>>(out, nvox);
  return cudaGetLastError();
}

}  // namespace pm

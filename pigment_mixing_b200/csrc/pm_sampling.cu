// Poisson-disk particle sampling on the GPU: the scene builder of the reference's
// sampleParticles (matter/src/sampling/sampling_particles.hpp:12-70), which draws a Poisson-disk
// set with Bridson's algorithm (tph_poisson 0.3), crops it to a shape and derives dx, the particle
// volume and mass from the sample count.
//
// Parallel dart throwing on a background grid of cells of side r / sqrt(3), so a cell holds at
// most one sample and any sample closer than r to a point lies within two cells of it.  Cells are
// processed in 27 phases (i mod 3, j mod 3, k mod 3): the indices of two cells of one phase
// differ by a multiple of 3 on some axis, so two full cells (2 r / sqrt(3) > r) lie between them
// there, their samples are more than r apart, and a phase needs no synchronisation between cells.
// Each cell of a phase throws up to `attempts` darts (counter-based hash RNG of seed, cell, pass,
// attempt) and keeps the first one with no sample within r in its 5x5x5 neighbourhood.  `passes`
// sweeps over the 27 phases fill the gaps left by earlier rejections.
#include <cuda_runtime.h>

#include <cstdint>

#include "pm_launch.h"

namespace pm {

namespace {

__device__ __forceinline__ uint32_t mix32(uint32_t x) {  // integer avalanche (xorshift-multiply rounds)
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}
__device__ __forceinline__ float unit_rand(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  const uint32_t h = mix32(a ^ mix32(b ^ mix32(c ^ mix32(d + 0x9e3779b9U))));
  return (float)(h >> 8) * (1.0f / 16777216.0f);  // [0, 1)
}

__global__ void k_poisson_phase(float4* cells, int nx, int ny, int nz, float cs, float r2, int px, int py, int pz,
                                uint32_t seed, uint32_t pass, uint32_t attempts) {
  const int mx = (nx - px + 2) / 3, my = (ny - py + 2) / 3, mz = (nz - pz + 2) / 3;
  const long long total = (long long)mx * my * mz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int i = px + 3 * (int)(t % mx), j = py + 3 * (int)((t / mx) % my), k = pz + 3 * (int)(t / ((long long)mx * my));
    const size_t c = ((size_t)k * ny + j) * nx + i;
    if (cells[c].w != 0.f) continue;
    const uint32_t cid = (uint32_t)c;
    for (uint32_t a = 0; a < attempts; ++a) {
      const float x = ((float)i + unit_rand(seed, cid, pass, 3 * a)) * cs;
      const float y = ((float)j + unit_rand(seed, cid, pass, 3 * a + 1)) * cs;
      const float z = ((float)k + unit_rand(seed, cid, pass, 3 * a + 2)) * cs;
      bool ok = true;
      for (int dk = -2; dk <= 2 && ok; ++dk) {
        const int kk = k + dk;
        if (kk < 0 || kk >= nz) continue;
        for (int dj = -2; dj <= 2 && ok; ++dj) {
          const int jj = j + dj;
          if (jj < 0 || jj >= ny) continue;
          for (int di = -2; di <= 2; ++di) {
            const int ii = i + di;
            if (ii < 0 || ii >= nx) continue;
            const float4 s = cells[((size_t)kk * ny + jj) * nx + ii];
            if (s.w == 0.f) continue;
            const float ex = s.x - x, ey = s.y - y, ez = s.z - z;
            if (ex * ex + ey * ey + ez * ez < r2) { ok = false; break; }
          }
        }
      }
      if (ok) {
        cells[c] = make_float4(x, y, z, 1.f);
        break;
      }
    }
  }
}

}  // namespace

cudaError_t poisson_fill(float4* cells, int nx, int ny, int nz, float cs, float r, uint32_t seed, uint32_t passes,
                         uint32_t attempts, cudaStream_t s) {
  const int sms = num_sms() > 0 ? num_sms() : 148;
  cudaError_t e = cudaMemsetAsync(cells, 0, sizeof(float4) * (size_t)nx * ny * nz, s);
  if (e != cudaSuccess) return e;
  for (uint32_t p = 0; p < passes; ++p)
    for (int ph = 0; ph < 27; ++ph)
      k_poisson_phase<<<sms * 8, 128, 0, s>>>(cells, nx, ny, nz, cs, r * r, ph % 3, (ph / 3) % 3, ph / 9, seed, p,
                                               attempts);
  return cudaGetLastError();
}

}  // namespace pm

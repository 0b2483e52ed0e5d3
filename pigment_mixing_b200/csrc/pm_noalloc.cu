// pm_p2g_noalloc: a particle-to-grid transfer that allocates no memory.
//
// Who needs it: callers that cannot call cudaMalloc -- plug-ins whose host application owns every
// device allocation (a caching allocator or a fixed memory budget that a cudaMalloc behind its
// back would break), real-time loops that may not allocate once running, and callers that have no
// pm_sim at all and only hold particle arrays in device memory.
//
// It is the transfer half of the step's P2G kernel (counting sort of particles by cell, then one
// warp per cell accumulating its particles into the cell's 27 stencil nodes) on caller-owned
// device arrays.  All scratch (cell counters, sort keys and ranks, the sorted order and the raw
// node accumulators) lives in one file-scope __device__ array of fixed size, so every GPU that
// loads the library holds those 8 MiB until the process exits.
//
// Limits: at most kNaMaxParticles particles and kNaMaxNodes grid nodes per call; larger inputs
// are rejected with PM_ERR_CAPACITY before any work is queued.  Every particle is scattered (there
// is no active mask, unlike p2g.cpp:22); particles whose stencil leaves the box, and particles with
// a non-finite coordinate, are skipped and counted.
//
// Shared state: every call uses the same array and leaves its contents behind; each call clears
// what must start at zero before using it.  Calls whose work overlaps on the GPU (issued on
// different streams without ordering, or from several host threads at once) race on the
// scratch and give wrong results: serialise them.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/pigment_mpm.h"

namespace {

constexpr uint32_t kNaMaxParticles = 1u << 17;  // 131,072
constexpr uint32_t kNaMaxNodes = 1u << 17;      // 131,072 (e.g. 64 x 64 x 32)
constexpr int kNaCh = 12;                        // sum w, sum w v (3), sum w latent (7), sum w shear

// byte offsets inside the scratch array (all 256-byte aligned)
constexpr size_t kOffKey = 0;
constexpr size_t kOffRank = kOffKey + 4ull * kNaMaxParticles;
constexpr size_t kOffSorted = kOffRank + 4ull * kNaMaxParticles;
constexpr size_t kOffCell = kOffSorted + 4ull * kNaMaxParticles;
constexpr size_t kOffAcc = kOffCell + 4ull * (kNaMaxNodes + 256);
constexpr size_t kOffErr = kOffAcc + 4ull * kNaCh * kNaMaxNodes;
constexpr size_t kScratchBytes = kOffErr + 256;  // 8 MiB + 2 KiB

static __device__ __align__(256) unsigned char g_p2g_scratch[kScratchBytes];

// Per-device address of g_p2g_scratch (host code may not use the symbol itself as a pointer).
std::mutex g_mu;
void* g_scratch_ptr[64] = {nullptr};

struct NaBox {
  float origin[3];
  float dx, inv_dx;
  int dims[3];
  uint32_t n, nodes;
  float mass;
  float apicD;
};

// Position of x in units of dx relative to the stencil base: the base node is floor of it.
__device__ __forceinline__ float na_u(float x, float o, float inv_dx) {
  return __fsub_rn(__fmul_rn(__fsub_rn(x, o), inv_dx), 0.5f);
}
__device__ __forceinline__ float na_node(int g, float o, float dx) { return __fadd_rn(o, __fmul_rn((float)g, dx)); }
__device__ __forceinline__ float na_N(float u) {
  float a = fabsf(u);
  if (a < 0.5f) return 0.75f - a * a;
  if (a < 1.5f) return 0.5f * (1.5f - a) * (1.5f - a);
  return 0.f;
}

__global__ void k_na_clear(NaBox b, unsigned char* s) {
  uint32_t* cell = reinterpret_cast<uint32_t*>(s + kOffCell);
  float* acc = reinterpret_cast<float*>(s + kOffAcc);
  uint32_t* err = reinterpret_cast<uint32_t*>(s + kOffErr);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.nodes + 2; i += stride) cell[i] = 0u;
  // channel k of node i lives at acc[k * kNaMaxNodes + i]: clear the used part of every channel
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.nodes * kNaCh; i += stride)
    acc[(size_t)(i / b.nodes) * kNaMaxNodes + (i % b.nodes)] = 0.f;
  if (blockIdx.x == 0 && threadIdx.x == 0) err[0] = 0u;
}

// key = lattice index (i*Ny + j)*Nz + k of the particle's stencil base node; out-of-box
// particles go to bucket `nodes` and are counted as errors.
__global__ void k_na_count(NaBox b, const float* x, unsigned char* s) {
  uint32_t* key = reinterpret_cast<uint32_t*>(s + kOffKey);
  uint32_t* rank = reinterpret_cast<uint32_t*>(s + kOffRank);
  uint32_t* cell = reinterpret_cast<uint32_t*>(s + kOffCell);
  uint32_t* err = reinterpret_cast<uint32_t*>(s + kOffErr);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < b.n; p += stride) {
    // the box test runs on the float coordinate, before any conversion to int: a NaN fails
    // every comparison and an infinite or huge coordinate fails the upper bound, so no integer
    // overflow can turn an outside particle into an in-box key
    int c[3] = {0, 0, 0};
    bool in = true;
    for (int d = 0; d < 3; ++d) {
      const float u = na_u(x[3 * p + d], b.origin[d], b.inv_dx);
      const bool ok = u >= 0.f && u < (float)(b.dims[d] - 2);  // floor(u) in [0, dims - 3]
      if (ok) c[d] = (int)floorf(u);
      in = in && ok;
    }
    uint32_t k = in ? (uint32_t)((c[0] * b.dims[1] + c[1]) * b.dims[2] + c[2]) : b.nodes;
    if (!in) atomicAdd(err, 1u);
    key[p] = k;
    rank[p] = atomicAdd(&cell[k], 1u);
  }
}

// exclusive scan of cell[0 .. nodes] by one block: each thread scans a contiguous run
__global__ void __launch_bounds__(1024) k_na_scan(NaBox b, unsigned char* s) {
  uint32_t* cell = reinterpret_cast<uint32_t*>(s + kOffCell);
  __shared__ uint32_t part[1024];
  const uint32_t n = b.nodes + 1;
  const uint32_t per = (n + 1023) / 1024;
  const uint32_t i0 = threadIdx.x * per, i1 = min(i0 + per, n);
  uint32_t sum = 0;
  for (uint32_t i = i0; i < i1; ++i) sum += cell[i];
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    uint32_t v = threadIdx.x >= (uint32_t)off ? part[threadIdx.x - off] : 0u;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  uint32_t run = part[threadIdx.x] - sum;
  for (uint32_t i = i0; i < i1; ++i) {
    uint32_t c = cell[i];
    cell[i] = run;
    run += c;
  }
  if (threadIdx.x == 1023) cell[n] = part[1023];
}

__global__ void k_na_scatter(NaBox b, unsigned char* s) {
  const uint32_t* key = reinterpret_cast<const uint32_t*>(s + kOffKey);
  const uint32_t* rank = reinterpret_cast<const uint32_t*>(s + kOffRank);
  const uint32_t* cell = reinterpret_cast<const uint32_t*>(s + kOffCell);
  uint32_t* sorted = reinterpret_cast<uint32_t*>(s + kOffSorted);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < b.n; p += stride) sorted[cell[key[p]] + rank[p]] = p;
}

// One warp per cell, lane l < 27 owns stencil node (l/9, l/3%3, l%3): it accumulates the cell's
// particles in registers and adds them to the node's accumulators once (p2g.cpp:21-77).
__global__ void k_na_p2g(NaBox b, const float* x, const float* v, const float* Bm, const float* lat, const float* diff,
                         unsigned char* s) {
  const uint32_t* cell = reinterpret_cast<const uint32_t*>(s + kOffCell);
  const uint32_t* sorted = reinterpret_cast<const uint32_t*>(s + kOffSorted);
  float* acc = reinterpret_cast<float*>(s + kOffAcc);
  const int lane = threadIdx.x & 31;
  const int la = lane / 9, lb = (lane / 3) % 3, lc = lane % 3;
  const uint32_t warps = gridDim.x * (blockDim.x / 32);
  for (uint32_t c = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); c < b.nodes; c += warps) {
    const uint32_t p0 = cell[c], p1 = cell[c + 1];
    if (p0 == p1 || lane >= 27) continue;
    const int ck = (int)(c % (uint32_t)b.dims[2]);
    const int cj = (int)((c / (uint32_t)b.dims[2]) % (uint32_t)b.dims[1]);
    const int ci = (int)(c / ((uint32_t)b.dims[2] * (uint32_t)b.dims[1]));
    const int gi[3] = {ci + la, cj + lb, ck + lc};
    const float xn[3] = {na_node(gi[0], b.origin[0], b.dx), na_node(gi[1], b.origin[1], b.dx),
                         na_node(gi[2], b.origin[2], b.dx)};
    float a[kNaCh];
#pragma unroll
    for (int k = 0; k < kNaCh; ++k) a[k] = 0.f;
    for (uint32_t q = p0; q < p1; ++q) {
      const uint32_t p = sorted[q];
      float d[3], w = 1.f;
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        d[r] = xn[r] - x[3 * p + r];
        w *= na_N(-d[r] * b.inv_dx);
      }
      if (!(w > 1e-25f)) continue;
      a[0] += w;
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        float t = v[3 * p + r];
        if (Bm) t += b.apicD * (Bm[9 * p + 3 * r] * d[0] + Bm[9 * p + 3 * r + 1] * d[1] + Bm[9 * p + 3 * r + 2] * d[2]);
        a[1 + r] += w * t;
      }
#pragma unroll
      for (int k = 0; k < 7; ++k) a[4 + k] += w * lat[7 * p + k];
      a[11] += w * diff[p];
    }
    const uint32_t node = (uint32_t)((gi[0] * b.dims[1] + gi[1]) * b.dims[2] + gi[2]);
#pragma unroll
    for (int k = 0; k < kNaCh; ++k)
      if (a[k] != 0.f) atomicAdd(&acc[(size_t)k * kNaMaxNodes + node], a[k]);
  }
}

// Normalisation of p2g.cpp:97-124: v /= m, latent /= m with the 4 concentrations renormalised,
// shear /= m, mass *= particle mass.
__global__ void k_na_finalize(NaBox b, const unsigned char* s, float* mass, float* vel, float* latent, float* shear) {
  const float* acc = reinterpret_cast<const float*>(s + kOffAcc);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < b.nodes; n += stride) {
    const float m = acc[n];
    float vv[3] = {0.f, 0.f, 0.f}, l[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, sh = 0.f;
    if (m > 0.f) {
      for (int r = 0; r < 3; ++r) vv[r] = acc[(size_t)(1 + r) * kNaMaxNodes + n] / m;
      for (int k = 0; k < 7; ++k) l[k] = acc[(size_t)(4 + k) * kNaMaxNodes + n] / m;
      sh = acc[(size_t)11 * kNaMaxNodes + n] / m;
      const float ps = l[0] + l[1] + l[2] + l[3];
      if (ps > 1e-6f) for (int k = 0; k < 4; ++k) l[k] /= ps;
    }
    if (mass) mass[n] = m * b.mass;
    if (vel) for (int r = 0; r < 3; ++r) vel[3 * n + r] = vv[r];
    if (latent) for (int k = 0; k < 7; ++k) latent[7 * n + k] = l[k];
    if (shear) shear[n] = sh;
  }
}

}  // namespace

extern "C" {

// See include/pigment_mpm.h.
PM_API pm_status pm_p2g_noalloc(const float* x, const float* v, const float* B, const float* latent,
                                const float* diffusion, uint32_t n, double particle_mass, double dx,
                                const double origin[3], const int32_t dims[3], float* node_mass, float* node_velocity,
                                float* node_latent, float* node_shear, void* stream, uint32_t* outside) {
  // sizes first: anything beyond the fixed scratch is rejected before other checks or work
  if (n > kNaMaxParticles) return PM_ERR_CAPACITY;
  if (!origin || !dims) return PM_ERR_INVALID;
  if (dims[0] < 3 || dims[1] < 3 || dims[2] < 3) return PM_ERR_INVALID;
  const uint64_t nodes = (uint64_t)dims[0] * (uint64_t)dims[1] * (uint64_t)dims[2];
  if (nodes > kNaMaxNodes) return PM_ERR_CAPACITY;
  if ((n > 0 && (!x || !v || !latent || !diffusion)) || !(dx > 0)) return PM_ERR_INVALID;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) return PM_ERR_CUDA;
  void* sp = nullptr;
  {
    // one-time set-up per device, with that device current: the device address of the array
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
      e = cudaGetSymbolAddress(&g_scratch_ptr[dev], g_p2g_scratch);
      if (e != cudaSuccess) {
        g_scratch_ptr[dev] = nullptr;
        return PM_ERR_CUDA;
      }
    }
    sp = g_scratch_ptr[dev];
  }
  unsigned char* s = static_cast<unsigned char*>(sp);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  NaBox b{};
  for (int d = 0; d < 3; ++d) { b.origin[d] = (float)origin[d]; b.dims[d] = dims[d]; }
  b.dx = (float)dx;
  b.inv_dx = (float)(1.0 / dx);
  b.n = n;
  b.nodes = (uint32_t)nodes;
  b.mass = (float)particle_mass;
  b.apicD = (float)(4.0 / (dx * dx));
  k_na_clear<<<256, 256, 0, st>>>(b, s);
  if (n > 0) {
    k_na_count<<<256, 256, 0, st>>>(b, x, s);
    k_na_scan<<<1, 1024, 0, st>>>(b, s);
    k_na_scatter<<<256, 256, 0, st>>>(b, s);
    k_na_p2g<<<512, 256, 0, st>>>(b, x, v, B, latent, diffusion, s);
  }
  k_na_finalize<<<256, 256, 0, st>>>(b, s, node_mass, node_velocity, node_latent, node_shear);
  e = cudaGetLastError();
  if (e != cudaSuccess) return PM_ERR_CUDA;
  if (outside) {
    e = cudaMemcpyAsync(outside, s + kOffErr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return PM_ERR_CUDA;
  }
  return PM_OK;
}

}  // extern "C"

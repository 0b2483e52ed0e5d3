// The renderer's particle-side preprocessing as CUDA kernels, computed from the simulation's
// device state (headless: no GL buffers).
//
// Density voxels (AABBc::fixedAABB, raytracing/src/raymarch/AABBc.cpp:10-25): cubes of the support
// radius h = 2 dx (MPMIntegrationSim.cpp:96-98) over the simulation's grid boundaries.
//
// Particle binning (BinaryDensityGrid::fillCells, BinaryDensityGrid.cpp:22-55): a counting sort of
// the particles by density voxel (voxel id x + X (y + Y z); particles outside are not binned).
//
// Binary density grid (BinaryDensityGrid::generateNc / fillBDG, :57-151): the voxel counts
// filtered separably along x, then y, then z with weight a on the voxel and b on each of its two
// neighbours (indices clamped to the grid); a voxel is occupied when nc * 315 / (64 pi h^3) >= iso
// (or always, in the test-all-filled mode); M2 and M4 OR the occupancy over 2^3 and 4^3 blocks.
//
// Anisotropy (Classification::countMatrix / countCurrDens, Classification.cpp:38-130): for every
// particle, the neighbours within h found through the binning (the 3 x 3 x 3 voxels around its
// own, clamped to the grid) give weights w = (1 - |x_i - x_j| / 2h)^3, their weighted mean and
// covariance C (scaled by s); with fewer than `threshold` neighbours (or no weight) the particle
// keeps the isotropic matrix I / h.  Otherwise C = V diag(l) V^T, the eigenvalues are clamped to at
// least max(l) / k, and G = V diag(1 / sqrt(l)) V^T / h, rescaled (auto-scale) to det G = 1 / h^3.
// The density of a particle is sum_j 315/(64 pi) |det G_j| (1 - |G_j (x_i - x_j)|^2)^3 over the
// neighbours with |G_j (x_i - x_j)| <= 1.
//
// Layout: one thread per density voxel for the occupancy grid.  The anisotropy and density passes
// run one CTA per voxel: the voxel's particles share one neighbourhood, staged once in shared
// memory and tested by all threads in lockstep; particles outside the voxels (not binned) take a
// per-thread path.  The symmetric eigenproblem is solved in FP64 by cyclic Jacobi rotations.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "pm_internal.cuh"
#include "pm_launch.h"

namespace pm {

namespace {

constexpr int kRenderThreads = 256;
constexpr int kRScanPer = 4;
constexpr int kRScanBlock = 1024 * kRScanPer;  // entries per scan block

// density voxel of position x; out-of-range voxels are clamped to -2 / dims + 1 so that the
// clamped 3 x 3 x 3 neighbourhood of a far particle is empty, as it is in the reference's loop
__device__ __forceinline__ bool bdg_voxel(const DensityGeom& g, const float x[3], int c[3]) {
  bool in = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    float f = floorf((x[d] - g.start[d]) / g.h);
    if (!(f >= 0.f && f < (float)g.dims[d])) in = false;
    f = fminf(fmaxf(f, -2.f), (float)(g.dims[d] + 1));  // NaN -> -2
    c[d] = (int)f;
  }
  return in;
}

__device__ __forceinline__ uint32_t bdg_id(const DensityGeom& g, int x, int y, int z) {
  return (uint32_t)x + (uint32_t)g.dims[0] * ((uint32_t)z * (uint32_t)g.dims[1] + (uint32_t)y);
}

__global__ void k_bin_count(Params P, const float* __restrict__ pcur, DensityGeom g, uint32_t* counts,
                            uint32_t* cellid, uint32_t* rank) {
  const int S = P.np_stride, np = P.np;
  const int lane = threadIdx.x & 31;
  for (int base = blockIdx.x * blockDim.x; base < np; base += gridDim.x * blockDim.x) {
    const int i = base + threadIdx.x;
    const bool valid = i < np;
    uint32_t id = 0xffffffffu;
    if (valid) {
      const float x[3] = {pcur[(F_X + 0) * S + i], pcur[(F_X + 1) * S + i], pcur[(F_X + 2) * S + i]};
      int c[3];
      if (bdg_voxel(g, x, c)) id = bdg_id(g, c[0], c[1], c[2]);
    }
    // warp-aggregated ranks: lanes sharing a voxel take consecutive ranks from one atomic
    const unsigned am = __ballot_sync(0xffffffffu, valid && id != 0xffffffffu);
    if (valid && id != 0xffffffffu) {
      const unsigned peers = __match_any_sync(am, id);
      const int leader = __ffs(peers) - 1;
      uint32_t r0 = 0;
      if (lane == leader) r0 = atomicAdd(&counts[id], (uint32_t)__popc(peers));
      r0 = __shfl_sync(peers, r0, leader);
      rank[i] = r0 + (uint32_t)__popc(peers & ((1u << lane) - 1u));
    }
    if (valid) cellid[i] = id;
  }
}

// exclusive scan of v[0..n): per-block local scan with block totals, scan of the totals, add
__device__ __forceinline__ uint32_t block_scan_incl(uint32_t v, uint32_t* wsum) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) wsum[wid] = v;
  __syncthreads();
  if (wid == 0) {
    uint32_t s = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += t;
    }
    wsum[lane] = s;
  }
  __syncthreads();
  const uint32_t r = v + (wid > 0 ? wsum[wid - 1] : 0u);
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(1024) k_rscan_local(const uint32_t* in, uint32_t* out, uint32_t* bsum, uint32_t n) {
  __shared__ uint32_t wsum[32];
  const uint32_t b0 = blockIdx.x * (uint32_t)kRScanBlock + threadIdx.x * kRScanPer;
  uint32_t v[kRScanPer], t = 0;
#pragma unroll
  for (int k = 0; k < kRScanPer; ++k) {
    v[k] = b0 + k < n ? in[b0 + k] : 0u;
    t += v[k];
  }
  const uint32_t incl = block_scan_incl(t, wsum);
  uint32_t run = incl - t;
#pragma unroll
  for (int k = 0; k < kRScanPer; ++k) {
    if (b0 + k < n) out[b0 + k] = run;
    run += v[k];
  }
  if (threadIdx.x == blockDim.x - 1) bsum[blockIdx.x] = incl;
}

__global__ void __launch_bounds__(1024) k_rscan_top(uint32_t* bsum, uint32_t nb, uint32_t* total) {
  __shared__ uint32_t wsum[32];
  const uint32_t b0 = threadIdx.x * kRScanPer;
  uint32_t v[kRScanPer], t = 0;
#pragma unroll
  for (int k = 0; k < kRScanPer; ++k) {
    v[k] = b0 + k < nb ? bsum[b0 + k] : 0u;
    t += v[k];
  }
  const uint32_t incl = block_scan_incl(t, wsum);
  uint32_t run = incl - t;
#pragma unroll
  for (int k = 0; k < kRScanPer; ++k) {
    if (b0 + k < nb) bsum[b0 + k] = run;
    run += v[k];
  }
  if (threadIdx.x == blockDim.x - 1) *total = incl;
}

__global__ void k_rscan_add(uint32_t* out, const uint32_t* bsum, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] += bsum[i / kRScanBlock];
}

__global__ void k_bin_fill(int np, const uint32_t* cellid, const uint32_t* rank, const uint32_t* offsets,
                           uint32_t* ids) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    const uint32_t id = cellid[i];
    if (id != 0xffffffffu) ids[offsets[id] + rank[i]] = (uint32_t)i;
  }
}

// Occupancy of one density voxel; the sums follow the reference's separable passes term by term
// (round-to-nearest products and sums, no fused multiply-add), so M matches a float restatement
// bit for bit.
__global__ void k_bdg_mask(DensityGeom g, const uint32_t* __restrict__ counts, float wa, float wb, float kern,
                           float iso, int test_all, uint32_t* M, uint32_t* M2, uint32_t* M4, uint32_t* occ) {
  const uint32_t nc_all = (uint32_t)g.dims[0] * g.dims[1] * g.dims[2];
  const int X = g.dims[0], Y = g.dims[1], Z = g.dims[2];
  const int X2 = (X + 1) / 2, Y2 = (Y + 1) / 2, X4 = (X + 3) / 4, Y4 = (Y + 3) / 4;
  uint32_t filled = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nc_all; i += gridDim.x * blockDim.x) {
    const int x = (int)(i % (uint32_t)X), y = (int)((i / (uint32_t)X) % (uint32_t)Y), z = (int)(i / ((uint32_t)X * Y));
    float nc = 0.f;
    for (int dz = -1; dz < 2; ++dz) {
      const int zz = min(max(z + dz, 0), Z - 1);
      float ny = 0.f;
      for (int dy = -1; dy < 2; ++dy) {
        const int yy = min(max(y + dy, 0), Y - 1);
        float nx = 0.f;
        for (int dx = -1; dx < 2; ++dx) {
          const int xx = min(max(x + dx, 0), X - 1);
          nx = __fadd_rn(nx, __fmul_rn(dx == 0 ? wa : wb, (float)counts[bdg_id(g, xx, yy, zz)]));
        }
        ny = __fadd_rn(ny, __fmul_rn(dy == 0 ? wa : wb, nx));
      }
      nc = __fadd_rn(nc, __fmul_rn(dz == 0 ? wa : wb, ny));
    }
    const uint32_t num = (__fmul_rn(nc, kern) >= iso || test_all) ? 1u : 0u;
    M[i] = num;
    if (num) {
      ++filled;
      atomicOr(&M2[(uint32_t)(x / 2) + (uint32_t)X2 * ((uint32_t)(y / 2) + (uint32_t)(z / 2) * Y2)], 1u);
      atomicOr(&M4[(uint32_t)(x / 4) + (uint32_t)X4 * ((uint32_t)(y / 4) + (uint32_t)(z / 4) * Y4)], 1u);
    }
  }
  const uint32_t f = __reduce_add_sync(0xffffffffu, filled);
  if ((threadIdx.x & 31) == 0 && f) atomicAdd(occ, f);
}

// Visits the binned neighbours j of sorted particle i within h (|x_i - x_j|^2 <= h^2), in the
// reference's voxel order (z, then y, then x).
template <class Fn>
__device__ __forceinline__ void for_neighbours(const DensityGeom& g, const float* __restrict__ pcur, int S,
                                               const uint32_t* __restrict__ counts,
                                               const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ ids,
                                               const float xi[3], Fn&& fn) {
  int c[3];
  bdg_voxel(g, xi, c);
  const float h2 = g.h * g.h;
  const int x0 = max(0, c[0] - 1), x1 = min(g.dims[0] - 1, c[0] + 1);
  const int y0 = max(0, c[1] - 1), y1 = min(g.dims[1] - 1, c[1] + 1);
  const int z0 = max(0, c[2] - 1), z1 = min(g.dims[2] - 1, c[2] + 1);
  for (int z = z0; z <= z1; ++z)
    for (int y = y0; y <= y1; ++y)
      for (int x = x0; x <= x1; ++x) {
        const uint32_t id = bdg_id(g, x, y, z);
        const uint32_t n = counts[id], o = offsets[id];
        for (uint32_t k = 0; k < n; ++k) {
          const uint32_t j = ids[o + k];
          const float d[3] = {xi[0] - pcur[(F_X + 0) * S + j], xi[1] - pcur[(F_X + 1) * S + j],
                              xi[2] - pcur[(F_X + 2) * S + j]};
          const float dd = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
          if (dd <= h2) fn(j, d, dd);
        }
      }
}

// cyclic Jacobi eigen-decomposition of a symmetric 3x3 (a00 a11 a22 a01 a02 a12) in FP64:
// eigenvalues in l, eigenvectors in the columns of V (row-major)
__device__ void sym_eig3(double a00, double a11, double a22, double a01, double a02, double a12, double l[3],
                         double V[9]) {
  double A[3][3] = {{a00, a01, a02}, {a01, a11, a12}, {a02, a12, a22}};
#pragma unroll
  for (int k = 0; k < 9; ++k) V[k] = (k % 4 == 0) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 16; ++sweep) {
    const double off = fabs(A[0][1]) + fabs(A[0][2]) + fabs(A[1][2]);
    const double dia = fabs(A[0][0]) + fabs(A[1][1]) + fabs(A[2][2]);
    if (off <= 1e-15 * dia || off == 0.0) break;
#pragma unroll
    for (int pq = 0; pq < 3; ++pq) {
      const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2, r = 3 - p - q;
      const double apq = A[p][q];
      if (apq == 0.0) continue;
      const double th = (A[q][q] - A[p][p]) / (2.0 * apq);
      const double t = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
      const double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
      A[p][p] -= t * apq;
      A[q][q] += t * apq;
      A[p][q] = A[q][p] = 0.0;
      const double arp = A[r][p], arq = A[r][q];
      A[r][p] = A[p][r] = cs * arp - sn * arq;
      A[r][q] = A[q][r] = sn * arp + cs * arq;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double vp = V[3 * k + p], vq = V[3 * k + q];
        V[3 * k + p] = cs * vp - sn * vq;
        V[3 * k + q] = sn * vp + cs * vq;
      }
    }
  }
  l[0] = A[0][0];
  l[1] = A[1][1];
  l[2] = A[2][2];
}

// G, |det G| and G^-1 of one particle from its neighbour moments (Classification.cpp:60-100);
// writes the sorted-order copies (Gs, dets) and the original-order outputs.
__device__ void aniso_finish(int i, uint32_t pid, int np, float h, const AnisoParams& ap, uint32_t cnt, float ws,
                             const float su[3], const float suu[6], float* __restrict__ Gs, float* __restrict__ dets,
                             float* G_out, float* Ginv_out, float* det_out) {
  double B[6];  // xx yy zz xy xz yz
  bool iso = cnt < (uint32_t)ap.threshold || ws < 1e-12f;
  if (!iso) {
    const double m[3] = {su[0] / (double)ws, su[1] / (double)ws, su[2] / (double)ws};
    const double sc = ap.s / (double)ws;
    const double c00 = sc * suu[0] - ap.s * m[0] * m[0], c11 = sc * suu[1] - ap.s * m[1] * m[1];
    const double c22 = sc * suu[2] - ap.s * m[2] * m[2], c01 = sc * suu[3] - ap.s * m[0] * m[1];
    const double c02 = sc * suu[4] - ap.s * m[0] * m[2], c12 = sc * suu[5] - ap.s * m[1] * m[2];
    double l[3], V[9];
    sym_eig3(c00, c11, c22, c01, c02, c12, l, V);
    const double lmax = fmax(l[0], fmax(l[1], l[2]));
    if (!(lmax > 0.0)) {
      iso = true;  // no spread among the neighbours: keep the isotropic kernel
    } else {
      double e[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) e[k] = 1.0 / sqrt(fmax(l[k], lmax / ap.k));
      auto Bm = [&](int r, int q) {
        return (V[3 * r] * e[0] * V[3 * q] + V[3 * r + 1] * e[1] * V[3 * q + 1] + V[3 * r + 2] * e[2] * V[3 * q + 2]) / h;
      };
      B[0] = Bm(0, 0); B[1] = Bm(1, 1); B[2] = Bm(2, 2); B[3] = Bm(0, 1); B[4] = Bm(0, 2); B[5] = Bm(1, 2);
      if (ap.auto_scale || !ap.is_ani) {
        const double det = fabs(B[0] * (B[1] * B[2] - B[5] * B[5]) - B[3] * (B[3] * B[2] - B[5] * B[4]) +
                                B[4] * (B[3] * B[5] - B[1] * B[4]));
        if (det > 0.0) {
          const double s3 = cbrt((1.0 / ((double)h * h * h)) / det);
#pragma unroll
          for (int k = 0; k < 6; ++k) B[k] *= s3;
        }
      }
    }
  }
  if (iso) {
    B[0] = B[1] = B[2] = 1.0 / h;
    B[3] = B[4] = B[5] = 0.0;
  }
  float Bf[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) Bf[k] = (float)B[k];
  // determinant and inverse of the rounded matrix
  const double b0 = Bf[0], b1 = Bf[1], b2 = Bf[2], b3 = Bf[3], b4 = Bf[4], b5 = Bf[5];
  const double k00 = b1 * b2 - b5 * b5, k01 = b4 * b5 - b3 * b2, k02 = b3 * b5 - b1 * b4;
  const double det = b0 * k00 + b3 * k01 + b4 * k02;
#pragma unroll
  for (int k = 0; k < 6; ++k) Gs[(size_t)k * np + i] = Bf[k];
  dets[i] = (float)fabs(det);
  if (G_out) {
    float* o = G_out + (size_t)pid * 9;
    o[0] = Bf[0]; o[1] = Bf[3]; o[2] = Bf[4];
    o[3] = Bf[3]; o[4] = Bf[1]; o[5] = Bf[5];
    o[6] = Bf[4]; o[7] = Bf[5]; o[8] = Bf[2];
  }
  if (det_out) det_out[pid] = (float)fabs(det);
  if (Ginv_out) {
    const double id = 1.0 / det;
    const double k11 = b0 * b2 - b4 * b4, k12 = b3 * b4 - b0 * b5, k22 = b0 * b1 - b3 * b3;
    float* o = Ginv_out + (size_t)pid * 9;
    o[0] = (float)(k00 * id); o[1] = (float)(k01 * id); o[2] = (float)(k02 * id);
    o[3] = (float)(k01 * id); o[4] = (float)(k11 * id); o[5] = (float)(k12 * id);
    o[6] = (float)(k02 * id); o[7] = (float)(k12 * id); o[8] = (float)(k22 * id);
  }
}

// neighbour moments: count, weight sum, weighted first and second moments of u = x_j - x_i
struct Moments {
  uint32_t cnt = 0;
  float ws = 0.f, su[3] = {0.f, 0.f, 0.f}, suu[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  __device__ __forceinline__ void add(const float d[3], float dd, float inv_ri) {
    const float q = sqrtf(dd) * inv_ri;
    const float om = 1.f - q;
    const float w = om * om * om;
    const float u[3] = {-d[0], -d[1], -d[2]};
    ++cnt;
    ws += w;
    su[0] += w * u[0]; su[1] += w * u[1]; su[2] += w * u[2];
    suu[0] += w * u[0] * u[0]; suu[1] += w * u[1] * u[1]; suu[2] += w * u[2] * u[2];
    suu[3] += w * u[0] * u[1]; suu[4] += w * u[0] * u[2]; suu[5] += w * u[1] * u[2];
  }
};

// Per-thread form, for the particles outside the density voxels (not binned, so not covered by
// the voxel-parallel kernels): unbinned only.
__global__ void k_aniso(Params P, const float* __restrict__ pcur, const uint32_t* __restrict__ meta, DensityGeom g,
                        const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
                        const uint32_t* __restrict__ ids, const uint32_t* __restrict__ cellid, AnisoParams ap,
                        float* __restrict__ Gs, float* __restrict__ dets, float* G_out, float* Ginv_out,
                        float* det_out) {
  const int S = P.np_stride, np = P.np;
  const float h = g.h, inv_ri = 1.f / (2.f * h);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    if (cellid[i] != 0xffffffffu) continue;
    const float xi[3] = {pcur[(F_X + 0) * S + i], pcur[(F_X + 1) * S + i], pcur[(F_X + 2) * S + i]};
    Moments m;
    for_neighbours(g, pcur, S, counts, offsets, ids, xi, [&](uint32_t, const float d[3], float dd) { m.add(d, dd, inv_ri); });
    aniso_finish(i, meta[i] & ~kInactiveBit, np, h, ap, m.cnt, m.ws, m.su, m.suu, Gs, dets, G_out, Ginv_out, det_out);
  }
}

__device__ __forceinline__ float density_term(const float d[3], float b0, float b1, float b2, float b3, float b4,
                                              float b5, float det, float kern) {
  const float l0 = b0 * d[0] + b3 * d[1] + b4 * d[2];
  const float l1 = b3 * d[0] + b1 * d[1] + b5 * d[2];
  const float l2v = b4 * d[0] + b5 * d[1] + b2 * d[2];
  const float l2 = l0 * l0 + l1 * l1 + l2v * l2v;
  if (l2 > 1.f) return 0.f;
  const float om = 1.f - l2;
  return kern * det * (om * om * om);
}

// Per-thread density for the unbinned particles.
__global__ void k_density(Params P, const float* __restrict__ pcur, const uint32_t* __restrict__ meta, DensityGeom g,
                          const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
                          const uint32_t* __restrict__ ids, const uint32_t* __restrict__ cellid,
                          const float* __restrict__ Gs, const float* __restrict__ dets, float kern, float iso,
                          float* dens_out, uint32_t* n_agg) {
  const int S = P.np_stride, np = P.np;
  uint32_t agg = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    if (cellid[i] != 0xffffffffu) continue;
    const float xi[3] = {pcur[(F_X + 0) * S + i], pcur[(F_X + 1) * S + i], pcur[(F_X + 2) * S + i]};
    float dens = 0.f;
    for_neighbours(g, pcur, S, counts, offsets, ids, xi, [&](uint32_t j, const float d[3], float) {
      dens += density_term(d, Gs[j], Gs[(size_t)np + j], Gs[2 * (size_t)np + j], Gs[3 * (size_t)np + j],
                           Gs[4 * (size_t)np + j], Gs[5 * (size_t)np + j], dets[j], kern);
    });
    if (dens_out) dens_out[meta[i] & ~kInactiveBit] = dens;
    if (dens > iso) ++agg;
  }
  const uint32_t a = __reduce_add_sync(0xffffffffu, agg);
  if ((threadIdx.x & 31) == 0 && a) atomicAdd(n_agg, a);
}


// ---- voxel-parallel forms: one CTA per density voxel.  Its particles share one neighbourhood (the
// 27 voxels around it), so the CTA stages the neighbourhood's candidates in shared memory once
// and every thread tests its particle against the same candidate at the same time (broadcast
// reads, no divergence in the candidate loop).  Candidates keep the reference's order: voxels
// z, then y, then x, and the binning order inside a voxel.
constexpr int kVoxThreads = 64;
constexpr int kCandA = 1024;  // candidates per staged chunk: positions (16 B)
constexpr int kCandD = 448;   // positions + matrices (48 B)

struct VoxSegs {
  int nseg;
  uint32_t off[27];
  uint32_t pre[28];  // exclusive prefix of the segment lengths; pre[nseg] = candidates
};

// warp 0 lists the clamped 27-voxel neighbourhood of voxel (vx, vy, vz) as segments of ids[]
__device__ __forceinline__ void vox_segments(const DensityGeom& g, const uint32_t* __restrict__ counts,
                                             const uint32_t* __restrict__ offsets, int vx, int vy, int vz,
                                             VoxSegs& sg) {
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  const int x0 = max(0, vx - 1), x1 = min(g.dims[0] - 1, vx + 1);
  const int y0 = max(0, vy - 1), y1 = min(g.dims[1] - 1, vy + 1);
  const int z0 = max(0, vz - 1), z1 = min(g.dims[2] - 1, vz + 1);
  const int nx = x1 - x0 + 1, ny = y1 - y0 + 1, nz = z1 - z0 + 1;
  const int nseg = nx * ny * nz;
  uint32_t c = 0;
  if (lane < nseg) {
    const int sx = lane % nx, sy = (lane / nx) % ny, sz = lane / (nx * ny);
    const uint32_t id = bdg_id(g, x0 + sx, y0 + sy, z0 + sz);
    c = counts[id];
    sg.off[lane] = offsets[id];
  }
  uint32_t incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane < nseg) sg.pre[lane + 1] = incl;
  if (lane == 0) {
    sg.pre[0] = 0;
    sg.nseg = nseg;
  }
}

// candidate kk of the staged neighbourhood -> its sorted particle index (s: running segment)
__device__ __forceinline__ uint32_t vox_candidate(const VoxSegs& sg, const uint32_t* __restrict__ ids, uint32_t kk,
                                                  int& s) {
  while (sg.pre[s + 1] <= kk) ++s;
  return ids[sg.off[s] + (kk - sg.pre[s])];
}

__global__ void __launch_bounds__(kVoxThreads) k_aniso_vox(Params P, const float* __restrict__ pcur,
                                                           const uint32_t* __restrict__ meta, DensityGeom g,
                                                           const uint32_t* __restrict__ counts,
                                                           const uint32_t* __restrict__ offsets,
                                                           const uint32_t* __restrict__ ids, AnisoParams ap,
                                                           float* __restrict__ Gs, float* __restrict__ dets,
                                                           float* G_out, float* Ginv_out, float* det_out) {
  __shared__ VoxSegs sg;
  __shared__ float4 cand[kCandA];
  const int S = P.np_stride, np = P.np;
  const float h = g.h, inv_ri = 1.f / (2.f * h), h2 = h * h;
  const uint32_t nvox = (uint32_t)g.dims[0] * g.dims[1] * g.dims[2];
  for (uint32_t v = blockIdx.x; v < nvox; v += gridDim.x) {
    const uint32_t nv = counts[v];
    if (nv == 0) continue;
    const uint32_t ov = offsets[v];
    const int vx = (int)(v % (uint32_t)g.dims[0]), vy = (int)((v / (uint32_t)g.dims[0]) % (uint32_t)g.dims[1]);
    const int vz = (int)(v / ((uint32_t)g.dims[0] * g.dims[1]));
    __syncthreads();  // the previous voxel's readers are done with sg and cand
    vox_segments(g, counts, offsets, vx, vy, vz, sg);
    __syncthreads();
    const uint32_t T = sg.pre[sg.nseg];
    for (uint32_t t0 = 0; t0 < nv; t0 += kVoxThreads) {
      const bool mine = t0 + threadIdx.x < nv;
      const uint32_t i = mine ? ids[ov + t0 + threadIdx.x] : 0u;
      float xi[3] = {0.f, 0.f, 0.f};
      if (mine) { xi[0] = pcur[(F_X + 0) * S + i]; xi[1] = pcur[(F_X + 1) * S + i]; xi[2] = pcur[(F_X + 2) * S + i]; }
      Moments m;
      for (uint32_t c0 = 0; c0 < T; c0 += kCandA) {
        const uint32_t nc = min((uint32_t)kCandA, T - c0);
        const bool staged = t0 > 0 && T <= (uint32_t)kCandA;  // whole neighbourhood still in place
        if (!staged) {
          __syncthreads();
          int sgi = 0;
          for (uint32_t k = threadIdx.x; k < nc; k += kVoxThreads) {
            const uint32_t j = vox_candidate(sg, ids, c0 + k, sgi);
            cand[k] = make_float4(pcur[(F_X + 0) * S + j], pcur[(F_X + 1) * S + j], pcur[(F_X + 2) * S + j], 0.f);
          }
          __syncthreads();
        }
        if (mine) {
#pragma unroll 4
          for (uint32_t k = 0; k < nc; ++k) {
            const float4 c = cand[k];
            const float d[3] = {xi[0] - c.x, xi[1] - c.y, xi[2] - c.z};
            const float dd = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (dd <= h2) m.add(d, dd, inv_ri);
          }
        }
      }
      if (mine) aniso_finish((int)i, meta[i] & ~kInactiveBit, np, h, ap, m.cnt, m.ws, m.su, m.suu, Gs, dets, G_out,
                             Ginv_out, det_out);
    }
  }
}

__global__ void __launch_bounds__(kVoxThreads) k_density_vox(Params P, const float* __restrict__ pcur,
                                                             const uint32_t* __restrict__ meta, DensityGeom g,
                                                             const uint32_t* __restrict__ counts,
                                                             const uint32_t* __restrict__ offsets,
                                                             const uint32_t* __restrict__ ids,
                                                             const float* __restrict__ Gs,
                                                             const float* __restrict__ dets, float kern, float iso,
                                                             float* dens_out, uint32_t* n_agg) {
  __shared__ VoxSegs sg;
  __shared__ float4 cand[3 * kCandD];  // per candidate: x y z |det|, G xx yy zz xy, G xz yz - -
  const int S = P.np_stride, np = P.np;
  const float h2 = g.h * g.h;
  const uint32_t nvox = (uint32_t)g.dims[0] * g.dims[1] * g.dims[2];
  uint32_t agg = 0;
  for (uint32_t v = blockIdx.x; v < nvox; v += gridDim.x) {
    const uint32_t nv = counts[v];
    if (nv == 0) continue;
    const uint32_t ov = offsets[v];
    const int vx = (int)(v % (uint32_t)g.dims[0]), vy = (int)((v / (uint32_t)g.dims[0]) % (uint32_t)g.dims[1]);
    const int vz = (int)(v / ((uint32_t)g.dims[0] * g.dims[1]));
    __syncthreads();
    vox_segments(g, counts, offsets, vx, vy, vz, sg);
    __syncthreads();
    const uint32_t T = sg.pre[sg.nseg];
    for (uint32_t t0 = 0; t0 < nv; t0 += kVoxThreads) {
      const bool mine = t0 + threadIdx.x < nv;
      const uint32_t i = mine ? ids[ov + t0 + threadIdx.x] : 0u;
      float xi[3] = {0.f, 0.f, 0.f};
      if (mine) { xi[0] = pcur[(F_X + 0) * S + i]; xi[1] = pcur[(F_X + 1) * S + i]; xi[2] = pcur[(F_X + 2) * S + i]; }
      float dens = 0.f;
      for (uint32_t c0 = 0; c0 < T; c0 += kCandD) {
        const uint32_t nc = min((uint32_t)kCandD, T - c0);
        const bool staged = t0 > 0 && T <= (uint32_t)kCandD;
        if (!staged) {
          __syncthreads();
          int sgi = 0;
          for (uint32_t k = threadIdx.x; k < nc; k += kVoxThreads) {
            const uint32_t j = vox_candidate(sg, ids, c0 + k, sgi);
            cand[3 * k] = make_float4(pcur[(F_X + 0) * S + j], pcur[(F_X + 1) * S + j], pcur[(F_X + 2) * S + j],
                                      dets[j]);
            cand[3 * k + 1] = make_float4(Gs[j], Gs[(size_t)np + j], Gs[2 * (size_t)np + j], Gs[3 * (size_t)np + j]);
            cand[3 * k + 2] = make_float4(Gs[4 * (size_t)np + j], Gs[5 * (size_t)np + j], 0.f, 0.f);
          }
          __syncthreads();
        }
        if (mine) {
#pragma unroll 4
          for (uint32_t k = 0; k < nc; ++k) {
            const float4 c = cand[3 * k];
            const float d[3] = {xi[0] - c.x, xi[1] - c.y, xi[2] - c.z};
            const float dd = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (dd <= h2) {
              const float4 b = cand[3 * k + 1], e = cand[3 * k + 2];
              dens += density_term(d, b.x, b.y, b.z, b.w, e.x, e.y, c.w, kern);
            }
          }
        }
      }
      if (mine) {
        if (dens_out) dens_out[meta[i] & ~kInactiveBit] = dens;
        if (dens > iso) ++agg;
      }
    }
  }
  const uint32_t a = __reduce_add_sync(0xffffffffu, agg);
  if ((threadIdx.x & 31) == 0 && a) atomicAdd(n_agg, a);
}

__global__ void k_ids_to_pid(const uint32_t* ids, const uint32_t* meta, const uint32_t* total, uint32_t* out, int np) {
  const uint32_t n = min(*total, (uint32_t)np);
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    out[k] = meta[ids[k]] & ~kInactiveBit;
}

int grid_for(long long work, int per_sm) {
  const int sms = num_sms() > 0 ? num_sms() : 148;
  const long long want = (work + kRenderThreads - 1) / kRenderThreads;
  return (int)(want < 1 ? 1 : (want < (long long)sms * per_sm ? want : (long long)sms * per_sm));
}

}  // namespace

size_t render_scratch_bytes(uint32_t np, uint32_t ncell, bool aniso) {
  const size_t nb = (ncell + kRScanBlock - 1) / kRScanBlock;
  size_t b = 4 * ((size_t)2 * ncell + 3 * (size_t)np + nb + 4);
  if (aniso) b += 4 * (size_t)7 * np;
  return (b + 255) / 256 * 256;
}

cudaError_t launch_bin_particles(const Params& P, const float* pcur, const DensityGeom& g, RenderScratch& r,
                                 cudaStream_t s) {
  const uint32_t ncell = (uint32_t)g.dims[0] * g.dims[1] * g.dims[2];
  const uint32_t nb = (ncell + kRScanBlock - 1) / kRScanBlock;
  if (nb > (uint32_t)kRScanBlock) return cudaErrorInvalidValue;  // more voxels than one top scan covers
  cudaError_t e = cudaMemsetAsync(r.counts, 0, sizeof(uint32_t) * ncell, s);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(r.misc, 0, sizeof(uint32_t) * 4, s)) != cudaSuccess) return e;
  if (P.np > 0) k_bin_count<<<grid_for(P.np, 8), kRenderThreads, 0, s>>>(P, pcur, g, r.counts, r.cellid, r.rank);
  k_rscan_local<<<nb, 1024, 0, s>>>(r.counts, r.offsets, r.bsum, ncell);
  k_rscan_top<<<1, 1024, 0, s>>>(r.bsum, nb, r.misc);
  if (nb > 1) k_rscan_add<<<grid_for(ncell, 8), kRenderThreads, 0, s>>>(r.offsets, r.bsum, ncell);
  if (P.np > 0) k_bin_fill<<<grid_for(P.np, 8), kRenderThreads, 0, s>>>(P.np, r.cellid, r.rank, r.offsets, r.ids);
  return cudaGetLastError();
}

cudaError_t launch_density_mask(const DensityGeom& g, const RenderScratch& r, float wa, float wb, float kern, float iso,
                                int test_all, uint32_t* M, uint32_t* M2, uint32_t* M4, cudaStream_t s) {
  const uint32_t X = g.dims[0], Y = g.dims[1], Z = g.dims[2];
  const size_t n2 = (size_t)((X + 1) / 2) * ((Y + 1) / 2) * ((Z + 1) / 2);
  const size_t n4 = (size_t)((X + 3) / 4) * ((Y + 3) / 4) * ((Z + 3) / 4);
  cudaError_t e = cudaMemsetAsync(M2, 0, sizeof(uint32_t) * n2, s);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(M4, 0, sizeof(uint32_t) * n4, s)) != cudaSuccess) return e;
  k_bdg_mask<<<grid_for((long long)X * Y * Z, 8), kRenderThreads, 0, s>>>(g, r.counts, wa, wb, kern, iso, test_all, M,
                                                                          M2, M4, r.misc + 1);
  return cudaGetLastError();
}

cudaError_t launch_ids_to_pid(const uint32_t* ids, const uint32_t* meta, const uint32_t* total, uint32_t* out, int np,
                              cudaStream_t s) {
  if (np <= 0) return cudaSuccess;
  k_ids_to_pid<<<grid_for(np, 8), kRenderThreads, 0, s>>>(ids, meta, total, out, np);
  return cudaGetLastError();
}

cudaError_t launch_anisotropy(const Params& P, const float* pcur, const uint32_t* meta, const DensityGeom& g,
                              const RenderScratch& r, const AnisoParams& ap, float kern, float iso, float* G,
                              float* Ginv, float* det, float* density, cudaStream_t s) {
  if (P.np <= 0) return cudaSuccess;
  const int sms = num_sms() > 0 ? num_sms() : 148;
  const long long nvox = (long long)g.dims[0] * g.dims[1] * g.dims[2];
  const int vgrid = (int)(nvox < (long long)sms * 16 ? nvox : (long long)sms * 16);
  k_aniso_vox<<<vgrid, kVoxThreads, 0, s>>>(P, pcur, meta, g, r.counts, r.offsets, r.ids, ap, r.Gs, r.dets, G, Ginv,
                                            det);
  k_aniso<<<grid_for(P.np, 8), kRenderThreads, 0, s>>>(P, pcur, meta, g, r.counts, r.offsets, r.ids, r.cellid, ap,
                                                      r.Gs, r.dets, G, Ginv, det);
  k_density_vox<<<vgrid, kVoxThreads, 0, s>>>(P, pcur, meta, g, r.counts, r.offsets, r.ids, r.Gs, r.dets, kern, iso,
                                              density, r.misc + 2);
  k_density<<<grid_for(P.np, 8), kRenderThreads, 0, s>>>(P, pcur, meta, g, r.counts, r.offsets, r.ids, r.cellid,
                                                        r.Gs, r.dets, kern, iso, density, r.misc + 2);
  return cudaGetLastError();
}

}  // namespace pm

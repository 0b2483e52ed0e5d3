// Host-side launchers of the step kernels (pm_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include "pm_internal.cuh"

namespace pm {

cudaError_t launch_init(int device);         // once per device; later calls return at once
cudaError_t launch_init_device(int device);  // the set-up itself
int num_sms();
int kernels_per_step(const Params& P);
const char* kernel_name(int i, const Params& P);
size_t p2g_smem_bytes();
size_t g2p_smem_bytes();
// One full step on stream s; with ev, events before and after every kernel (kernels_per_step + 1).
void launch_step(const Params& P, const Bufs& B, cudaStream_t s, cudaEvent_t* ev = nullptr);
void launch_reduce_state(const Params& P, const float* pcur, const uint32_t* meta, Ctrl* ctrl, cudaStream_t s);
// Field groups for launch_unpermute's mask: x, v, B, F, latent, diffusion, plastic, tau.
enum : uint32_t { kGrpX = 1u, kGrpV = 2u, kGrpB = 4u, kGrpF = 8u, kGrpLat = 16u, kGrpDiff = 32u, kGrpPlastic = 64u,
                  kGrpTau = 128u, kGrpAll = 255u };
void launch_unpermute(const Params& P, const float* pcur, const uint32_t* meta, float* out, uint8_t* active,
                      cudaStream_t s, uint32_t group_mask = kGrpAll);
void launch_upload(const Params& P, const float* x, const float* lat, const float* v, float* pbuf, uint32_t* meta,
                   cudaStream_t s);
void launch_stats(const Params& P, const float* pcur, const uint32_t* meta, double* acc, cudaStream_t s, int cyl = 0,
                  float cx = 0.f, float cz = 0.f, float r2 = 0.f);
// The reference's particle PLY row: x y z vx vy vz p q Je eps_pl_vol eps_pl_dev delta_gamma.
constexpr int kPlyFields = 12;
void launch_ply_particles(const Params& P, const float* pcur, const uint32_t* meta, float* out, cudaStream_t s);
// Pigment splat geometry (BinaryDensityGrid::fillRenderGrid): fine-voxel origin and size, voxel
// counts, search half-extent in voxels, squared spatial and colour sigmas, isotropic 1/h.
struct SplatGeom {
  float start[3];
  float v4;
  int dims[3];
  int ext;
  float sig_s2, sig_c2, inv_h;
  uint32_t order_stride;  // particle visiting order i -> i * stride mod np (1: sorted order)
};
// Two-pass splat into out[dims z][y][x][8] (latent 7 + weight); tmp: same size, pass-1 grid.
cudaError_t launch_splat(const Params& P, const float* pcur, const uint32_t* meta, const float* G, const SplatGeom& g,
                         float* tmp, float* out, cudaStream_t s);
// Density voxels of the renderer (AABBc::fixedAABB): origin, side h (the support radius) and counts.
struct DensityGeom {
  float start[3];
  float h;
  int dims[3];
};
// Classification::countMatrix parameters: covariance scale, eigenvalue clamp ratio, minimum
// neighbour count, determinant rescaling (autoScaleS / !isAni).
struct AnisoParams {
  double s, k;
  int threshold;
  int auto_scale, is_ani;
};
// Scratch of the binning and anisotropy passes (render_scratch_bytes bytes, carved by the caller):
// voxel counts and exclusive offsets, scan block sums, misc[0] binned total / [1] occupied voxels /
// [2] aggregate particles, per sorted particle its voxel and rank, the binned sorted indices by
// voxel, and (anisotropy) the symmetric matrices xx yy zz xy xz yz field-major with |det|.
struct RenderScratch {
  uint32_t *counts, *offsets, *bsum, *misc, *cellid, *rank, *ids;
  float *Gs, *dets;
};
size_t render_scratch_bytes(uint32_t np, uint32_t ncell, bool aniso);
cudaError_t launch_bin_particles(const Params& P, const float* pcur, const DensityGeom& g, RenderScratch& r,
                                 cudaStream_t s);
cudaError_t launch_density_mask(const DensityGeom& g, const RenderScratch& r, float wa, float wb, float kern, float iso,
                                int test_all, uint32_t* M, uint32_t* M2, uint32_t* M4, cudaStream_t s);
// ids (binned sorted indices, total[0] of them) -> particle indices
cudaError_t launch_ids_to_pid(const uint32_t* ids, const uint32_t* meta, const uint32_t* total, uint32_t* out, int np,
                              cudaStream_t s);
cudaError_t launch_anisotropy(const Params& P, const float* pcur, const uint32_t* meta, const DensityGeom& g,
                              const RenderScratch& r, const AnisoParams& ap, float kern, float iso, float* G,
                              float* Ginv, float* det, float* density, cudaStream_t s);
// The step's device SVD on n row-major FP64 matrices (self-test entry point).
void launch_svd3_batch(const double* A, int n, float* U, double* S, float* V, cudaStream_t s);
// Poisson-disk dart throwing into a background grid of nx*ny*nz cells of side cs (= r / sqrt(3)):
// cells[c] = (x, y, z, 1) for a cell holding a sample, 0 otherwise.
cudaError_t poisson_fill(float4* cells, int nx, int ny, int nz, float cs, float r, uint32_t seed, uint32_t passes,
                         uint32_t attempts, cudaStream_t s);
// Checkpoint load: grouped host layout of pm_get_particles' unpermute (all F_COUNT fields) -> SoA.
void launch_load_fields(const Params& P, const float* in, const uint8_t* active, float* pbuf, uint32_t* meta,
                        cudaStream_t s);

// Batched scenes: the SceneDev table and, per kernel class, device tables of CTA offsets
// (ns + 1 entries; scene s owns CTAs [off[s], off[s+1])) with their totals.
struct BatchLaunch {
  const SceneDev* sd = nullptr;
  int ns = 0;
  const int* off_unit = nullptr;  // one CTA per scene (prologue, epilogue)
  const int* off_part = nullptr;  // particle-parallel flat kernels (count, scatter)
  const int* off_node = nullptr;  // node-parallel flat kernels (clear, clear_bricks, grid_update)
  const int* off_scan = nullptr;  // scan blocks of each scene's cell array
  const int* off_p2g = nullptr;
  const int* off_g2p = nullptr;
  const int* off_def = nullptr;
  const int* off_sur = nullptr;   // surrogate inference and finish
  int n_part = 0, n_node = 0, n_scan = 0, n_p2g = 0, n_g2p = 0, n_def = 0, n_sur = 0;
  int flat_threads = 256;         // block size of the flat kernels
  bool surrogate = false;         // some scene runs the learned return map
  int defgrad_model = -1;         // plastic model shared by every scene on the plain solver, else -1
  bool g2p_flip = true;           // some scene blends FLIP (flip_ratio >= -1)
};
void launch_step_batched(const BatchLaunch& L, cudaStream_t s, cudaEvent_t* ev = nullptr);
int batched_kernels_per_step(bool surrogate);
const char* batched_kernel_name(int i, bool surrogate);
void batched_occupancy(int& p2g, int& g2p, int& def);
int scan_blocks_for(int node_cap);
// CTAs of the grid-stride scan passes: one per scan block up to max_ctas.
int scan_ctas_for(int node_cap, int max_ctas);
void mlp_infer_batched(const SceneDev* sd, const int* off, int ns, int ctas, cudaStream_t s);

}  // namespace pm

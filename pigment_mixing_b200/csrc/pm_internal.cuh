// Internal device-side data layout of the paint-mixing MPM step.
//
// Layout in HBM (one scene):
//   particles  structure-of-arrays, double-buffered (read "in", write "out" in cell-sorted
//              order; the step's writes are the physical re-sort).  Field f of particle p is
//              at base[f * np_stride + p].
//   grid       dense box of 4x4x4-node bricks covering the step's particle stencils; node n of
//              brick b is record b*64+n.  Main record: 16 floats (64 B):
//                P2G:     [sum w, sum w*(v+APIC) xyz | force xyz, lat0 | lat1..lat4 | lat5, lat6, shear, -]
//                updated: [m,     v xyz              | flip xyz,  lat0 | lat1..lat4 | lat5, lat6, shear, -]
//              MUSL record: float4 [sum w*(v+APIC) xyz, sum w].
//   control    one Ctrl block in device memory: time, dt, frame, the step's grid box, knife
//              pose, reductions.  1-thread kernels update it between steps so a whole step
//              (and many steps) run without host round trips.
#pragma once
#include <cstdint>
#include <cstring>

#include "pm_mlp.h"

namespace pm {

constexpr int kMaxPlates = 8;
constexpr int kMaxObjects = 8;
constexpr int kMaxWaypoints = 16;
constexpr int kBrick = 4;       // nodes per brick edge
constexpr int kBrickNodes = 64;
constexpr int kTile = 6;        // brick + 2-node halo of the 3-node quadratic stencil
constexpr int kTileNodes = 216;

// Particle field offsets (in units of np_stride floats)
enum PField : int {
  F_X = 0,      // 3
  F_V = 3,      // 3
  F_B = 6,      // 9  (APIC B, row-major)
  F_F = 15,     // 9  (deformation gradient, row-major)
  F_LAT = 24,   // 7  (Mixbox latent)
  F_DIFF = 31,  // 1  (diffusion_factor = |sym grad v|)
  F_EPD = 32,   // eps_pl_dev
  F_EPV = 33,   // eps_pl_vol
  F_EPP = 34,   // eps_pl_vol_pradhana
  F_DG = 35,    // delta_gamma
  F_TAU = 36,   // 6  (Kirchhoff stress of F, symmetric: xx yy zz xy xz yz)
  F_COUNT = 42
};

// meta word: bits 0..30 particle id (original order), bit 31 set = inactive
constexpr uint32_t kInactiveBit = 0x80000000u;

enum ErrBits : uint32_t {
  E_NEG_DGAMMA = 0x1u,
  E_NEWTON_NOCONV = 0x2u,
  E_NEWTON_FLAT = 0x4u,
  E_INVALID_BC = 0x8u,
  E_NAN_PARTICLE = 0x10u,
  E_INDEX_RANGE = 0x20u,
  E_CAPACITY = 0x40u,
};

enum ObjKind : int { OBJ_SPATULA = 0, OBJ_BOXKNIFE = 1, OBJ_GROUND = 2, OBJ_CURVE = 3 };
enum PlateT : int { PT_TOP = 0, PT_BOTTOM, PT_LEFT, PT_RIGHT, PT_FRONT, PT_BACK };
enum BCT : int { BC_NOSLIP = 0, BC_SLIPSTICK = 1, BC_SLIPFREE = 2 };
enum PlasticT : int { PL_NONE = 0, PL_VMVISC = 5, PL_DPVISC = 6 };

struct PlateDev {
  int type, bc;
  float friction;
  float vx, vy, vz;        // current velocity (object_plate.hpp: vx_object...)
  float vx0, vy0, vz0;     // original velocity
  float vmin_factor, load_factor;
  double pos, lower, upper;
};

struct ObjDev {
  int kind, bc;
  float friction;
  float y0;                 // ground height
  float Rinv[9];            // world -> local rotation (general inverse of the linear part)
  float tx, ty, tz;         // translation (world position of local origin)
  float vlin[3], omega[3];  // velocity field v = vlin + omega x (X - t)
  float half[3];            // box half extents
  // double-precision pose state advanced by the epilogue kernel
  double t[3];
  double q[4];              // w x y z
  double current_time;      // spatula animation clock
  double s;                 // arc length along the box knife path
  double speed;
  int n_waypoints;
  float waypoints[kMaxWaypoints * 3];
};

// Per-scene constants (set at prepare time, passed by value to kernels)
struct Params {
  int np;                 // particle count
  int np_stride;          // field stride in floats
  float dx, inv_dx;
  double dx_d;
  float anchor[3];        // lattice origin (low_init), node i at anchor + i*dx
  double anchor_d[3];
  float particle_mass, particle_volume;
  float apicD;            // 4/dx^2
  float flip_ratio;
  float gravity[3];
  int use_musl;
  int use_particle_boundaries;
  float pbmin[3], pbmax[3];
  // material
  double mu, lambda, K;
  double E;               // Young's modulus (a surrogate feature)
  double e_mu_prefac, f_mu_prefac, d_prefac;
  double q_max, q_min, p_min, M, q_cohesion, perzyna_exp, perzyna_visc, xi;
  int plastic_model;
  int use_pradhana;
  // pigments (g2p.cpp:103-119)
  float D_max, D_edge0, D_edge1, start_boost, end_boost, boost_factor;
  // time stepping
  double cfl, dt_max, frame_dt, min_dt, final_time;
  // grid capacity
  int brick_cap;
  int node_cap;           // brick_cap * 64
  // spatula animation table
  const float* frames;
  int n_frames;
  int return_map;         // 0 plain, 1 surrogate
  int sur_fallback_plain; // surrogate mode: 1 = failed checks restart Newton from the reference guess
  uint32_t log_cap;       // capacity of the return-map sample log (0 = off)
  uint32_t log_every;     // log about one solve in log_every (hash of slot index and step)
  uint32_t q_cap;         // capacity of the surrogate queue
};

// One particle waiting for the surrogate (the state the return map needs to finish).
struct __align__(16) SurQ {
  float U[9], V[9];       // SVD factors of the trial elastic F (rounded from FP64)
  float h[3], hd[3];      // clamped principal log strains, unit deviatoric direction
  float q_trial, q_y;
  float epd;
  uint32_t i;             // particle slot (sorted order)
  uint32_t vm;            // 1 VMVisc, 0 DPVisc
};

struct Ctrl {
  double time, dt;
  uint32_t step, frame, end_frame;
  uint32_t halt;          // sticky: set by the prologue on capacity overflow
  uint32_t error_flags;
  uint32_t frames_done;
  uint32_t auto_frame;    // 1: epilogue runs frameFinished after every step
  uint32_t need_bricks;   // bricks required when halted
  // grid of this step
  int g0[3];              // lattice index of node (0,0,0)
  int dims[3];            // nodes per axis (multiples of 4)
  int nb[3];              // bricks per axis
  int n_bricks;
  int n_nodes;
  double low[3], high[3];
  double low_init[3], high_init[3], min_init[3], max_init[3];
  // reductions over the particles at the end of the previous step
  uint32_t max_v2;        // float bits of max |v|^2 (non-negative floats order as uints)
  int xmin_key[3], xmax_key[3];
  uint32_t n_active;
  uint32_t plastic_count;
  // return-map statistics of the last step and the sample log fill
  uint32_t q_n;            // particles queued for the surrogate this step
  uint32_t newton_iters;   // Newton updates this step
  uint32_t newton_solves;  // particles that needed the Perzyna consistency solve this step
  uint32_t sur_accept;     // surrogate estimates that passed the consistency check
  uint32_t slog_n;         // samples written to the log (cumulative)
  uint32_t target_step;    // batches: the scene idles once step reaches this (0 = no target)
  uint32_t idle;           // set by the prologue: this round is skipped for the scene
  uint32_t stop_at_end;    // 1: steps idle once frame >= end_frame (the simulate() driver)
  // objects
  int n_plates, n_objects, knife;  // knife: index into objects or -1
  int pad1;
  PlateDev plates[kMaxPlates];
  ObjDev objects[kMaxObjects];
};

struct Bufs {
  const float* pin;       // particle fields, read side
  float* pout;            // particle fields, write side
  const uint32_t* meta_in;
  uint32_t* meta_out;
  float* pic;             // 3 * np_stride, new order (+3 for flip in USL mode)
  uint32_t* key;          // per particle (read order)
  uint32_t* rank;
  uint32_t* sorted;       // new position -> read index
  uint32_t* cell;         // node_cap + 2: counts, then exclusive prefix (cell starts)
  uint32_t* scan_part;    // per scan block partial sums
  uint32_t* scan_occ;     // per scan block (64 bricks): bricks holding particles
  unsigned long long* occ_mask;  // per scan block: bit j set when brick 64 * block + j holds particles
  float4* grid;           // node_cap * 4 float4
  float4* gmusl;          // node_cap float4
  uint8_t* btouch;        // brick_cap: 1 when a particle's stencil reaches the brick this step
  // Brick lists of this step: blist_n[0] bricks holding particles, in ascending order (blist_occ,
  // written by the scan), and blist_n[1] bricks that a particle's stencil reaches (blist_touch,
  // written by k_clear_bricks).  The transfer kernels walk these instead of the whole box, which
  // the knife can stretch to many times the bricks the paint fills.
  uint32_t* blist_n;      // 4 words: counts
  uint4* blist_occ;       // brick_cap: (brick, first particle, end particle, 0) in sorted order
  uint32_t* blist_touch;  // brick_cap
  Ctrl* ctrl;
  // learned return map (optional)
  MlpDev mlp;
  float* slog;            // log_cap x 16: features[10], targets[6]
  SurQ* q;                // q_cap records
  float* qx;              // q_cap x 10 surrogate inputs
  float* qy;              // q_cap x 6 surrogate outputs
};

// One scene of a batch as the batched kernels see it: its constants and both buffer parities.
// The parity of a step is (ctrl->step + par_base) & 1, so scenes that idle or halt for a round
// keep their own parity.
struct SceneDev {
  Params P;
  Bufs B[2];
  uint32_t par_base;
  uint32_t pad[3];
};

__device__ __forceinline__ int scene_parity(const SceneDev& d) {
  return (int)((d.B[0].ctrl->step + d.par_base) & 1u);
}

// Static partition of a batched launch: scene s owns CTAs [off[s], off[s+1]).  Returns the
// scene of this CTA and the CTA's index and count within the scene.
__device__ __forceinline__ void batch_slot(const int* __restrict__ off, int ns, int& s, int& blk, int& nblk) {
  const int b = (int)blockIdx.x;
  int lo = 0, hi = ns;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= b) lo = mid; else hi = mid;
  }
  s = lo;
  blk = b - off[lo];
  nblk = off[lo + 1] - off[lo];
}

// A batched CTA's scene (its constants and this step's buffers) copied into shared memory: the
// kernel bodies then read their parameters from shared memory instead of the scene table in
// global memory, which also frees the registers the compiler would hoist those loads into.
struct SceneShared {
  Params P;
  Bufs B;
};
static_assert(sizeof(Params) % 4 == 0 && sizeof(Bufs) % 4 == 0, "word copy");
__device__ __forceinline__ void load_scene_shared(const SceneDev& d, SceneShared& ss) {
  const int* sp = reinterpret_cast<const int*>(&d.P);
  int* dp = reinterpret_cast<int*>(&ss.P);
  for (int k = threadIdx.x; k < (int)(sizeof(Params) / 4); k += blockDim.x) dp[k] = sp[k];
  const int* sb = reinterpret_cast<const int*>(&d.B[scene_parity(d)]);
  int* db = reinterpret_cast<int*>(&ss.B);
  for (int k = threadIdx.x; k < (int)(sizeof(Bufs) / 4); k += blockDim.x) db[k] = sb[k];
  __syncthreads();
}

// Order-preserving float <-> int key (min/max of floats through integer atomics).
__host__ __device__ inline int fkey(float f) {
  int i;
  memcpy(&i, &f, 4);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__host__ __device__ inline float fkey_inv(int k) {
  int i = k >= 0 ? k : k ^ 0x7fffffff;
  float f;
  memcpy(&f, &i, 4);
  return f;
}

}  // namespace pm

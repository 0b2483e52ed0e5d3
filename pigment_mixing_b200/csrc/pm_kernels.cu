// sm_100a kernels of the paint-mixing MPM step.
//
// One step (the reference's Simulation::advanceStep, matter/src/simulation/simulation.cpp:225-280):
//   k_prologue      dt (update_dt.cpp:5-41) and the step's grid box (remesh.cpp:182-297)
//   k_clear         zero cell counters and the main grid records
//   k_count         per particle: cell key + rank (counting sort, pass 1)
//   k_scan_local,   exclusive prefix of the cell counters -> cell starts (block scans, then the
//   k_scan_add      block offsets, each formed by the CTA that adds it)
//   k_scatter       counting sort, pass 2: new position -> read index
//   k_p2g           P2G + particle half of the explicit update (p2g.cpp:6-126,
//                   explicit_euler_update.cpp:12-55) with the cached Kirchhoff stress
//   k_grid_update   grid half of the explicit update + collisions
//                   (explicit_euler_update.cpp:61-110, boundary_collision.cpp:5-316)
//   k_g2p_musl      G2P + pigment mixing + MUSL velocity update and re-scatter
//                   (g2p.cpp:12-135, musl.cpp:6-98)
//   k_defgrad_head  deformation update: velocity gradient, position update, F_trial, and the
//                   reductions for the next step (deformation_update.cpp, position_update.cpp:6-91)
//   k_defgrad_tail  FP64 SVD, return map and stress cache (plasticity.cpp:18-340,
//                   simulation.hpp:287-294)
//   k_epilogue      moveObjects (simulation.cpp:284-291), time += dt, frame bookkeeping
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cmath>
#include <mutex>
#include <vector>
#include "pm_internal.cuh"
#include "pm_launch.h"

namespace pm {

// ------------------------------------------------------------------------------------------
// helpers
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ int cell_of(float x, float anchor, float inv_dx) {
  // base node of the 3-node quadratic stencil; the exact same float ops everywhere
  return (int)floorf(__fsub_rn(__fmul_rn(__fsub_rn(x, anchor), inv_dx), 0.5f));
}
__device__ __forceinline__ float node_pos(int g, float anchor, float dx) {
  return __fadd_rn(anchor, __fmul_rn((float)g, dx));
}
// quadratic B-spline and derivative, tools.hpp:153-177
__device__ __forceinline__ float bsN(float u) {
  float a = fabsf(u);
  if (a < 0.5f) return 0.75f - a * a;
  if (a < 1.5f) return 0.5f * (1.5f - a) * (1.5f - a);
  return 0.f;
}
__device__ __forceinline__ float bsdN(float u) {
  float a = fabsf(u);
  if (a < 0.5f) return -2.f * u;
  if (a < 1.5f) return u - 1.5f * (float)((0.f < u) - (u < 0.f));
  return 0.f;
}

// 1: the transfer kernels load the next chunk's (or particle's) sorted index during the current
// one and prefetch the particle fields it will read into L2 once that index is known.
#ifndef PM_PREFETCH
#define PM_PREFETCH 1
#endif
// 1: the same for the deformation-update tail's particle loop.
#ifndef PM_PREFETCH_TAIL
#define PM_PREFETCH_TAIL 0
#endif
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
// Asynchronous 4-byte global -> shared copies (cp.async): the copy lands in shared memory without
// passing through registers; a thread waits for its own copies with cp_async_wait_all.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
// 16 bytes, or 16 zero bytes when !valid (no global read then; gmem must still be a valid address)
__device__ __forceinline__ void cp_async16_zfill(void* smem, const void* gmem, bool valid) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Programmatic dependent launch.  The step's kernels are launched with programmatic stream
// serialisation (PM_PDL): the next kernel of the stream is launched while the previous one
// finishes, and each kernel waits for the previous one to complete, with its memory visible,
// before it reads anything (griddepcontrol.wait).  PM_PDL 2 leaves the trigger implicit (the
// previous kernel's completion); PM_PDL 1 also triggers at every CTA's start
// (launch_dependents), so that the next kernel's CTAs take SMs as the previous kernel's last CTAs
// free them.  Measured on the 2M scene (graph-timed steps 5-105, three runs each): 0.929-0.931 ms
// per step with PM_PDL 2, 0.931-0.936 without (the bench's headline measured 0.935 ms both ways,
// so the gain is within its run-to-run spread), 1.016-1.019 with PM_PDL 1.  Launched without the
// attribute (batches, single launches) the instructions return at once.
#ifndef PM_PDL
#define PM_PDL 2
#endif
__device__ __forceinline__ void pdl_enter() {
#if PM_PDL == 1
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
#if PM_PDL
  asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}

__device__ __forceinline__ void red_add_v4(float4* addr, float a, float b, float c, float d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
               : "memory");
}

struct AxisW {
  int base;       // lattice index of the stencil's first node
  float N[3];     // weights at base+0..2
  float dN[3];    // derivative * inv_dx
  float r;        // x - node_pos(base)
};

__device__ __forceinline__ AxisW axis_weights(float x, float anchor, float dx, float inv_dx) {
  AxisW a;
  a.base = cell_of(x, anchor, inv_dx);
  float x0 = node_pos(a.base, anchor, dx);
  a.r = x - x0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float xi = node_pos(a.base + k, anchor, dx);
    float u = (x - xi) * inv_dx;
    a.N[k] = bsN(u);
    a.dN[k] = bsdN(u) * inv_dx;
  }
  return a;
}

__device__ __forceinline__ const Ctrl* C_(const Bufs& B) { return B.ctrl; }

// ------------------------------------------------------------------------------------------
// 1-thread control kernels
// ------------------------------------------------------------------------------------------
__device__ void grid_box_from_aabb(const Params& P, Ctrl* c) {
  // node range covering every particle's stencil, with a 1-node margin
  int lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    float mn = fkey_inv(c->xmin_key[d]), mx = fkey_inv(c->xmax_key[d]);
    if (c->n_active == 0) { mn = mx = P.anchor[d]; }
    lo[d] = cell_of(mn, P.anchor[d], P.inv_dx) - 1;
    hi[d] = cell_of(mx, P.anchor[d], P.inv_dx) + 3;
  }
  long long nbricks = 1;
  for (int d = 0; d < 3; ++d) {
    int n = hi[d] - lo[d] + 1;
    n = (n + kBrick - 1) / kBrick * kBrick;
    c->g0[d] = lo[d];
    c->dims[d] = n;
    c->nb[d] = n / kBrick;
    nbricks *= c->nb[d];
  }
  if (nbricks > P.brick_cap) {
    c->halt = 1;
    c->need_bricks = (uint32_t)(nbricks > 0x7fffffffLL ? 0x7fffffff : nbricks);
    c->error_flags |= E_CAPACITY;
    c->n_bricks = 0;
    c->n_nodes = 0;
    return;
  }
  c->n_bricks = (int)nbricks;
  c->n_nodes = (int)nbricks * kBrickNodes;
}

__device__ __forceinline__ void prologue_body(const Params& P, const Bufs& B, Ctrl* c) {
  if (c->halt) return;
  // a scene of a batch that has reached its target step sits this round out, and so does a
  // simulate() run whose last frame is done (simulation.cpp:170-203 leaves its loop there)
  c->idle = ((c->target_step != 0u && c->step >= c->target_step) || (c->stop_at_end && c->frame >= c->end_frame))
                ? 1u : 0u;
  if (c->idle) return;
  // updateDt (update_dt.cpp:5-41)
  float m2f = __uint_as_float(c->max_v2);
  double ms = sqrt((double)m2f);
  double dt;
  if (fabs(ms) > 1e-10) dt = fmin(P.cfl * P.dx_d / ms, P.dt_max);
  else dt = P.dt_max;
  dt = fmin(dt, P.frame_dt * (double)(c->frame + 1) - c->time);
  dt = fmax(dt, P.min_dt);
  c->dt = dt;
  // reference grid boundaries (remeshFixedCont, remesh.cpp:182-297); step 0 keeps the init box
  if (c->step > 0) {
    for (int d = 0; d < 3; ++d) {
      double mn = fkey_inv(c->xmin_key[d]), mx = fkey_inv(c->xmax_key[d]);
      if (c->n_active == 0) mn = mx = 0.0;
      double dxd = P.dx_d;
      if (mx < c->max_init[d]) {
        double r = floor(fmax(0.0, (c->max_init[d] - mx) / dxd - 1e-8 * dxd));
        c->high[d] = c->high_init[d] - r * dxd;
      } else {
        double e = floor(fmax(0.0, (mx - c->max_init[d]) / dxd - 1e-8 * dxd));
        c->high[d] = c->high_init[d] + e * dxd;
      }
      if (mn > c->min_init[d]) {
        double r = floor(fmax(0.0, (mn - c->min_init[d]) / dxd - 1e-8 * dxd));
        c->low[d] = c->low_init[d] + r * dxd;
      } else {
        double e = floor(fmax(0.0, (c->min_init[d] - mn) / dxd - 1e-8 * dxd));
        c->low[d] = c->low_init[d] - e * dxd;
      }
    }
  }
  grid_box_from_aabb(P, c);
  if (c->halt) return;  // keep the reductions: the host regrows the grid and re-runs this step
  // reset the reductions that this step's deformation update fills
  c->max_v2 = 0u;
  for (int d = 0; d < 3; ++d) { c->xmin_key[d] = 0x7fffffff; c->xmax_key[d] = (int)0x80000000; }
  c->n_active = 0;
  c->plastic_count = 0;
  c->q_n = 0;
  c->newton_iters = 0;
  c->newton_solves = 0;
  c->sur_accept = 0;
  B.blist_n[1] = 0u;  // the touched-brick list that k_clear_bricks fills
}
// (A copy of the control block staged in shared memory for the one thread measured slower:
// 0.9325 against 0.931 ms per step.)
__device__ __forceinline__ void d_prologue(const Params& P, const Bufs& B, const int blk_, const int nblk_) {
  if (threadIdx.x == 0 && blk_ == 0) prologue_body(P, B, B.ctrl);
}
__global__ void k_prologue(Params P, Bufs B) { pdl_enter(); d_prologue(P, B, blockIdx.x, gridDim.x); }
__global__ void kb_prologue(const SceneDev* __restrict__ sd, const int* __restrict__ off, int ns) {
  int s_, blk_, nblk_;
  batch_slot(off, ns, s_, blk_, nblk_);
  const SceneDev& d_ = sd[s_];
  d_prologue(d_.P, d_.B[scene_parity(d_)], blk_, nblk_);
}


// quaternion helpers (w, x, y, z)
__device__ void q_to_rot(const double q[4], double R[9]) {
  double n = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  double w = q[0] / n, x = q[1] / n, y = q[2] / n, z = q[3] / n;
  R[0] = 1 - 2 * (y * y + z * z); R[1] = 2 * (x * y - z * w); R[2] = 2 * (x * z + y * w);
  R[3] = 2 * (x * y + z * w); R[4] = 1 - 2 * (x * x + z * z); R[5] = 2 * (y * z - x * w);
  R[6] = 2 * (x * z - y * w); R[7] = 2 * (y * z + x * w); R[8] = 1 - 2 * (x * x + y * y);
}
__device__ void set_pose(ObjDev& o, const double t[3], const double q[4]) {
  for (int k = 0; k < 3; ++k) o.t[k] = t[k];
  for (int k = 0; k < 4; ++k) o.q[k] = q[k];
  double R[9];
  q_to_rot(q, R);
  double det = R[0] * (R[4] * R[8] - R[5] * R[7]) - R[1] * (R[3] * R[8] - R[5] * R[6]) + R[2] * (R[3] * R[7] - R[4] * R[6]);
  double inv[9];
  inv[0] = (R[4] * R[8] - R[5] * R[7]) / det;
  inv[1] = (R[2] * R[7] - R[1] * R[8]) / det;
  inv[2] = (R[1] * R[5] - R[2] * R[4]) / det;
  inv[3] = (R[5] * R[6] - R[3] * R[8]) / det;
  inv[4] = (R[0] * R[8] - R[2] * R[6]) / det;
  inv[5] = (R[2] * R[3] - R[0] * R[5]) / det;
  inv[6] = (R[3] * R[7] - R[4] * R[6]) / det;
  inv[7] = (R[1] * R[6] - R[0] * R[7]) / det;
  inv[8] = (R[0] * R[4] - R[1] * R[3]) / det;
  for (int k = 0; k < 9; ++k) o.Rinv[k] = (float)inv[k];
  o.tx = (float)t[0]; o.ty = (float)t[1]; o.tz = (float)t[2];
}
__device__ void slerp_d(const double a[4], const double b[4], double t, double out[4]) {
  const double one = 1.0 - 2.220446049250313e-16;
  double d = a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
  double ad = fabs(d), s0, s1;
  if (ad >= one) { s0 = 1.0 - t; s1 = t; }
  else {
    double th = acos(ad), sth = sin(th);
    s0 = sin((1.0 - t) * th) / sth;
    s1 = sin(t * th) / sth;
  }
  if (d < 0) s1 = -s1;
  for (int k = 0; k < 4; ++k) out[k] = s0 * a[k] + s1 * b[k];
}

__device__ void move_knife(const Params& P, ObjDev& o, double dt) {
  if (o.kind == OBJ_SPATULA) {  // object_spatula.hpp:164-233
    o.current_time += dt;
    if (P.n_frames <= 0) {
      for (int k = 0; k < 3; ++k) { o.vlin[k] = 0.f; o.omega[k] = 0.f; }
      return;
    }
    double fi = o.current_time * 60.0;
    int i0u = (int)floor(fi);
    int i0 = min(i0u, P.n_frames - 1), i1 = min(i0u + 1, P.n_frames - 1);
    i0 = max(i0, 0); i1 = max(i1, 0);
    double tt = fi - (double)i0u;
    const float* f0 = P.frames + 7 * i0;
    const float* f1 = P.frames + 7 * i1;
    double pi[3];
    for (int k = 0; k < 3; ++k) pi[k] = (double)f0[k] + tt * ((double)f1[k] - (double)f0[k]);
    double q0[4] = {f0[6], f0[3], f0[4], f0[5]}, q1[4] = {f1[6], f1[3], f1[4], f1[5]};
    double qi[4];
    slerp_d(q0, q1, tt, qi);
    for (int k = 0; k < 3; ++k) o.vlin[k] = (float)((pi[k] - o.t[k]) / dt);
    // relative rotation dq = qi * conj(q_old) -> axis angle (angle in [0, pi])
    const double* a = qi;
    double b[4] = {o.q[0], -o.q[1], -o.q[2], -o.q[3]};
    double dq[4] = {a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3],
                    a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2],
                    a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1],
                    a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0]};
    double n2 = dq[1] * dq[1] + dq[2] * dq[2] + dq[3] * dq[3];
    if (n2 == 0.0) { for (int k = 0; k < 3; ++k) o.omega[k] = 0.f; }
    else {
      double vn = sqrt(n2);
      double ang = 2.0 * atan2(vn, fabs(dq[0]));
      double sg = dq[0] < 0 ? -1.0 : 1.0;
      for (int k = 0; k < 3; ++k) o.omega[k] = (float)(dq[k + 1] * (sg * ang / (vn * dt)));
    }
    set_pose(o, pi, qi);
  } else if (o.kind == OBJ_BOXKNIFE) {
    o.s += o.speed * dt;
    double pn[3] = {o.t[0], o.t[1], o.t[2]};
    if (o.n_waypoints > 0) {
      double acc = 0.0;
      bool found = false;
      for (int i = 0; i + 1 < o.n_waypoints && !found; ++i) {
        double d[3], L = 0.0;
        for (int k = 0; k < 3; ++k) { d[k] = (double)o.waypoints[3 * (i + 1) + k] - (double)o.waypoints[3 * i + k]; L += d[k] * d[k]; }
        L = sqrt(L);
        if (o.s <= acc + L && L > 0) {
          for (int k = 0; k < 3; ++k) pn[k] = (double)o.waypoints[3 * i + k] + d[k] * ((o.s - acc) / L);
          found = true;
        }
        acc += L;
      }
      if (!found) for (int k = 0; k < 3; ++k) pn[k] = (double)o.waypoints[3 * (o.n_waypoints - 1) + k];
    }
    for (int k = 0; k < 3; ++k) { o.vlin[k] = (float)((pn[k] - o.t[k]) / dt); o.omega[k] = 0.f; }
    double q[4] = {o.q[0], o.q[1], o.q[2], o.q[3]};
    set_pose(o, pn, q);
  }
}

__device__ __forceinline__ void epilogue_body(const Params& P, Ctrl* c) {
  if (c->halt || c->idle) return;
  double dt = c->dt;
  // moveObjects (simulation.cpp:284-291): plates, then the spatula
  for (int i = 0; i < c->n_plates; ++i) {  // object_plate.hpp:136-162
    PlateDev& pl = c->plates[i];
    double factor = (c->time < (double)pl.load_factor * P.frame_dt) ? (1.0 / (double)pl.vmin_factor) : 1.0;
    pl.vx = (float)(pl.vx0 * factor); pl.vy = (float)(pl.vy0 * factor); pl.vz = (float)(pl.vz0 * factor);
    if (pl.type == PT_LEFT || pl.type == PT_RIGHT) { pl.pos += dt * pl.vx; pl.upper += dt * pl.vy; pl.lower += dt * pl.vy; }
    else if (pl.type == PT_BOTTOM || pl.type == PT_TOP) { pl.pos += dt * pl.vy; pl.upper += dt * pl.vx; pl.lower += dt * pl.vx; }
    else pl.pos += dt * pl.vz;
  }
  if (c->knife >= 0) move_knife(P, c->objects[c->knife], dt);
  c->time += dt;
  c->step += 1;
  if (c->auto_frame) {  // frameFinished (simulation_units.cpp:235-241)
    if (P.frame_dt * (double)(c->frame + 1) - c->time < P.min_dt * 1.1) { c->frame += 1; c->frames_done += 1; }
  }
}
__device__ __forceinline__ void d_epilogue(const Params& P, const Bufs& B, const int blk_, const int nblk_) {
  if (threadIdx.x == 0 && blk_ == 0) epilogue_body(P, B.ctrl);
}
__global__ void k_epilogue(Params P, Bufs B) { pdl_enter(); d_epilogue(P, B, blockIdx.x, gridDim.x); }
__global__ void kb_epilogue(const SceneDev* __restrict__ sd, const int* __restrict__ off, int ns) {
  int s_, blk_, nblk_;
  batch_slot(off, ns, s_, blk_, nblk_);
  const SceneDev& d_ = sd[s_];
  d_epilogue(d_.P, d_.B[scene_parity(d_)], blk_, nblk_);
}


// ------------------------------------------------------------------------------------------
// counting sort by cell
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void brick_coords(int b, const Ctrl* c, int& bx, int& by, int& bz) {
  const int nyz = c->nb[1] * c->nb[2];
  bx = b / nyz;
  int r = b - bx * nyz;
  by = r / c->nb[2];
  bz = r - by * c->nb[2];
}

// Zeroes the per-node counters of the counting sort (the grid records are cleared per brick by
// k_clear_bricks once the occupied bricks are known).
__device__ __forceinline__ void d_clear(const Params& P, const Bufs& B, const int blk_, const int nblk_) {
  const Ctrl* c = B.ctrl;
  if (c->halt || c->idle) return;
  const int nn = c->n_nodes;
  const int stride = nblk_ * blockDim.x;
  for (int i = blk_ * blockDim.x + threadIdx.x; i < nn + 2; i += stride) B.cell[i] = 0u;
}
__global__ void k_clear(Params P, Bufs B) { pdl_enter(); d_clear(P, B, blockIdx.x, gridDim.x); }
__global__ void kb_clear(const SceneDev* __restrict__ sd, const int* __restrict__ off, int ns) {
  int s_, blk_, nblk_;
  batch_slot(off, ns, s_, blk_, nblk_);
  const SceneDev& d_ = sd[s_];
  d_clear(d_.P, d_.B[scene_parity(d_)], blk_, nblk_);
}


// After the scan: a brick is touched this step when one of the bricks b - d, d in {0,1}^3, holds
// particles (a particle's 3x3x3 stencil spans its own brick and the next one on each axis).
// A warp takes 32 consecutive bricks, lane j testing brick b0 + j: it stores the touch flags,
// appends the touched bricks to this step's list (one atomic per warp) and then zeroes the
// accumulated and MUSL records of each touched brick in turn.  Consecutive groups of 32 bricks go
// to different CTAs, so that a small box still spreads its zeroing over the SMs.  Only touched
// bricks are ever read by the transfers, so untouched ones are left as they are.
__device__ __forceinline__ void d_clear_bricks(const Params& P, const Bufs& B, const int blk_, const int nblk_) {
  const Ctrl* c = B.ctrl;
  if (c->halt || c->idle) return;
  const int nbr = c->n_bricks, lane = threadIdx.x & 31;
  const int wpc = blockDim.x >> 5, warps = nblk_ * wpc;
  const size_t nyz = (size_t)c->nb[1] * c->nb[2], nz = (size_t)c->nb[2];
  const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int b0 = ((threadIdx.x >> 5) * nblk_ + blk_) * 32; b0 < nbr; b0 += warps * 32) {
    const int b = b0 + lane;
    bool touched = false;
    if (b < nbr) {
      int bx, by, bz;
      brick_coords(b, c, bx, by, bz);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int sx = bx - (k >> 2), sy = by - ((k >> 1) & 1), sz = bz - (k & 1);
        if (sx >= 0 && sy >= 0 && sz >= 0) {
          const size_t sb = (size_t)sx * nyz + (size_t)sy * nz + (size_t)sz;
          touched = touched || (B.cell[sb * kBrickNodes] != B.cell[(sb + 1) * kBrickNodes]);
        }
      }
      B.btouch[b] = touched ? 1 : 0;
    }
    const uint32_t mt = __ballot_sync(0xffffffffu, touched);
    uint32_t base = 0u;
    if (lane == 0 && mt) base = atomicAdd(&B.blist_n[1], (uint32_t)__popc(mt));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (touched) B.blist_touch[base + __popc(mt & ((1u << lane) - 1u))] = (uint32_t)b;
    for (uint32_t m = mt; m; m &= m - 1u) {
      const size_t tb = (size_t)(b0 + __ffs(m) - 1);
      float4* rec = B.grid + tb * kBrickNodes * 4;
#pragma unroll
      for (int k = 0; k < 8; ++k) rec[k * 32 + lane] = z;
      if (P.use_musl) {
        float4* mm = B.gmusl + tb * kBrickNodes;
        mm[lane] = z;
        mm[32 + lane] = z;
      }
    }
  }
}
__global__ void k_clear_bricks(Params P, Bufs B) { pdl_enter(); d_clear_bricks(P, B, blockIdx.x, gridDim.x); }
__global__ void kb_clear_bricks(const SceneDev* __restrict__ sd, const int* __restrict__ off, int ns) {
  int s_, blk_, nblk_;
  batch_slot(off, ns, s_, blk_, nblk_);
  const SceneDev& d_ = sd[s_];
  d_clear_bricks(d_.P, d_.B[scene_parity(d_)], blk_, nblk_);
}


__device__ __forceinline__ uint32_t brick_key(const int c[3], const Ctrl* ctrl) {
  int bx = c[0] >> 2, by = c[1] >> 2, bz = c[2] >> 2;
  int lx = c[0] & 3, ly = c[1] & 3, lz = c[2] & 3;
  return (uint32_t)(((bx * ctrl->nb[1] + by) * ctrl->nb[2] + bz) * kBrickNodes + lx * 16 + ly * 4 + lz);
}

__device__ __forceinline__ void d_count(const Params& P, const Bufs& B, const int blk_, const int nblk_) {
  const Ctrl* c = B.ctrl;
  if (c->halt || c->idle) return;
  const int np = P.np, S = P.np_stride;
  const uint32_t inactive_key = (uint32_t)c->n_nodes;
  const int stride = nblk_ * blockDim.x;
  bool range_err = false;
  for (int base = blk_ * blockDim.x; base < np; base += stride) {
    int p = base + threadIdx.x;
    bool valid = p < np;
    uint32_t key = 0xffffffffu;
    if (valid) {
      uint32_t meta = B.meta_in[p];
      if (meta & kInactiveBit) key = inactive_key;
      else {
        int cc[3];
        for (int d = 0; d < 3; ++d) {
          float x = B.pin[(F_X + d) * S + p];
          int g = cell_of(x, P.anchor[d], P.inv_dx) - c->g0[d];
          if (g < 0 || g + 2 >= c->dims[d]) { range_err = true; g = min(max(g, 0), c->dims[d] - 3); }
          cc[d] = g;
        }
        key = brick_key(cc, c);
      }
    }
    // warp-aggregated rank: lanes sharing a key take consecutive ranks from one atomic
    unsigned am = __ballot_sync(0xffffffffu, valid);
    if (valid) {
      unsigned peers = __match_any_sync(am, key);
      int leader = __ffs(peers) - 1;
      int lane = threadIdx.x & 31;
      uint32_t r0 = 0;
      if (lane == leader) r0 = atomicAdd(&B.cell[key], (uint32_t)__popc(peers));
      r0 = __shfl_sync(peers, r0, leader);
      B.key[p] = key;
      B.rank[p] = r0 + __popc(peers & ((1u << lane) - 1u));
    }
  }
  if (range_err) atomicOr(&B.ctrl->error_flags, (uint32_t)E_INDEX_RANGE);
}
__global__ void k_count(Params P, Bufs B) { pdl_enter(); d_count(P, B, blockIdx.x, gridDim.x); }
__global__ void kb_count(const SceneDev* __restrict__ sd, const int* __restrict__ off, int ns) {
  int s_, blk_, nblk_;
  batch_slot(off, ns, s_, blk_, nblk_);
  const SceneDev& d_ = sd[s_];
  d_count(d_.P, d_.B[scene_parity(d_)], blk_, nblk_);
}


// Exclusive scan of cell[0 .. n_nodes+1) in 4096-entry blocks.
constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr int kScanBlock = kScanThreads * kScanPer;

__device__ __forceinline__ uint32_t block_incl_scan(uint32_t v, uint32_t* warp_sums) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) warp_sums[wid] = v;
  __syncthreads();
  if (wid == 0) {
    uint32_t s = warp_sums[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += t;
    }
    warp_sums[lane] = s;
  }
  __syncthreads();
  if (wid > 0) v += warp_sums[wid - 1];
  return v;
}

__device__ __forceinline__ void d_scan_local(const Params& P, const Bufs& B, const int blk_, const int nblk_) {
  const Ctrl* c = B.ctrl;
  if (c->halt || c->idle) return;
  const int n = c->n_nodes + 1;
  __shared__ uint32_t ws[32];
  __shared__ uint32_t occ2[kScanThreads / 32];  // per warp: its two bricks' occupancy bits
  static_assert(kScanBlock == 64 * kBrickNodes && kBrickNodes == 16 * kScanPer, "a scan block is 64 bricks");
  const int lane = threadIdx.x & 31;
  // grid-stride over the 4096-entry scan blocks of this step's box (the launch is sized for a
  // typical box, not for the grid capacity)
  for (int sb = blk_; sb * kScanBlock < n; sb += nblk_) {
    const int b0 = sb * kScanBlock;
    uint32_t v[kScanPer];
    uint32_t tsum = 0;
    const int i0 = b0 + threadIdx.x * kScanPer;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) { v[k] = (i0 + k < n) ? B.cell[i0 + k] : 0u; tsum += v[k]; }
    // 16 threads hold the 64 counters of one brick: warp w covers bricks 2w and 2w + 1 of the block
    const uint32_t nz = __ballot_sync(0xffffffffu, tsum != 0u);
    if (lane == 0) occ2[threadIdx.x >> 5] = ((nz & 0xffffu) ? 1u : 0u) | ((nz >> 16) ? 2u : 0u);
    uint32_t incl = block_incl_scan(tsum, ws);  // its barriers publish occ2
    uint32_t run = incl - tsum;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
      if (i0 + k < n) B.cell[i0 + k] = run;
      run += v[k];
    }
    if (threadIdx.x == kScanThreads - 1) B.scan_part[sb] = incl;
    if (threadIdx.x == 0) {
      // occupied bricks of this block; the inactive-particle counter behind the last brick
      // (entry n_nodes) belongs to no brick
      unsigned long long m = 0ull;
      for (int w = 0; w < kScanThreads / 32; ++w) m |= (unsigned long long)occ2[w] << (2 * w);
      const int first = sb * (kScanBlock / kBrickNodes), valid = c->n_bricks - first;
      if (valid < 64) m &= valid > 0 ? (1ull << valid) - 1ull : 0ull;
      B.occ_mask[sb] = m;
      B.scan_occ[sb] = (uint32_t)__popcll(m);
    }
    __syncthreads();  // ws and occ2 are reused by the next block's scan
  }
}
__global__ void __launch_bounds__(kScanThreads) k_scan_local(Params P, Bufs B) {
  pdl_enter();
  d_scan_local(P, B, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(kScanThreads) kb_scan_local(const SceneDev* __restrict__ sd, const int* __restrict__ off, int ns) {
  int s_, blk_, nblk_;
  batch_slot(off, ns, s_, blk_, nblk_);
  const SceneDev& d_ = sd[s_];
  d_scan_local(d_.P, d_.B[scene_parity(d_)], blk_, nblk_);
}


// Sum of v[a, b) over the block (all threads call it; ws: 33 words of shared memory).
__device__ __forceinline__ uint32_t block_range_sum(const uint32_t* __restrict__ v, int a, int b, uint32_t* ws) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t t = 0;
  for (int j = a + threadIdx.x; j < b; j += blockDim.x) t += v[j];
  t = __reduce_add_sync(0xffffffffu, t);
  if (lane == 0) ws[wid] = t;
  __syncthreads();
  if (wid == 0) {
    uint32_t u = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0u;
    u = __reduce_add_sync(0xffffffffu, u);
    if (lane == 0) ws[32] = u;
  }
  __syncthreads();
  const uint32_t r = ws[32];
  __syncthreads();  // ws is reused by the next call
  return r;
}

// Second scan pass: adds to every scan block the sum of the block totals before it, each CTA
// extending its running prefix over the blocks it skipped (grid-stride), and CTA 0 writes the
// grand total behind the last cell.  Forming the prefixes here replaces a separate one-CTA pass
// over the block totals.
__device__ __forceinline__ void d_scan_add(const Params& P, const Bufs& B, const int blk_, const int nblk_) {
  const Ctrl* c = B.ctrl;
  if (c->halt || c->idle) return;
  const int n = c->n_nodes + 1;
  const int nb = (n + kScanBlock - 1) / kScanBlock;
  __shared__ uint32_t ws[33];
  uint32_t off = 0, off_occ = 0;  // sums of scan_part and scan_occ over [0, upto)
  int upto = 0;
  for (int sb = blk_; sb < nb; sb += nblk_) {
    off += block_range_sum(B.scan_part, upto, sb, ws);
    off_occ += block_range_sum(B.scan_occ, upto, sb, ws);
    upto = sb;
    // this block's occupied bricks with their particle ranges, at their place in the ascending list
    // of occupied bricks: a brick starts at its first counter's block-local prefix plus the block's
    // offset and ends where the next brick starts (the block total for the block's last brick)
    if (threadIdx.x < 64) {
      const unsigned long long m = B.occ_mask[sb];
      if ((m >> threadIdx.x) & 1ull) {
        const uint32_t bi = (uint32_t)(sb * (kScanBlock / kBrickNodes) + threadIdx.x);
        const uint32_t ps = B.cell[(size_t)bi * kBrickNodes] + off;
        const uint32_t pe = (threadIdx.x < 63 ? B.cell[(size_t)(bi + 1) * kBrickNodes] : B.scan_part[sb]) + off;
        B.blist_occ[off_occ + (uint32_t)__popcll(m & ((1ull << threadIdx.x) - 1ull))] = make_uint4(bi, ps, pe, 0u);
      }
    }
    if (sb == 0) continue;  // block 0 needs no offset
    __syncthreads();  // the block-local prefixes above are read before they are offset
    const int b0 = sb * kScanBlock;
    for (int i = b0 + threadIdx.x; i < min(b0 + kScanBlock, n); i += kScanThreads) B.cell[i] += off;
  }
  if (blk_ == 0) {
    const uint32_t total = block_range_sum(B.scan_part, 0, nb, ws);
    const uint32_t occupied = block_range_sum(B.scan_occ, 0, nb, ws);
    if (threadIdx.x == 0) {
      B.cell[n] = total;  // = np
      B.blist_n[0] = occupied;
    }
  }
}
__global__ void __launch_bounds__(kScanThreads) k_scan_add(Params P, Bufs B) {
  pdl_enter();
  d_scan_add(P, B, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(kScanThreads) kb_scan_add(const SceneDev* __restrict__ sd, const int* __restrict__ off, int ns) {
  int s_, blk_, nblk_;
  batch_slot(off, ns, s_, blk_, nblk_);
  const SceneDev& d_ = sd[s_];
  d_scan_add(d_.P, d_.B[scene_parity(d_)], blk_, nblk_);
}


__device__ __forceinline__ void d_scatter(const Params& P, const Bufs& B, const int blk_, const int nblk_) {
  const Ctrl* c = B.ctrl;
  if (c->halt || c->idle) return;
  const int stride = nblk_ * blockDim.x;
  for (int p = blk_ * blockDim.x + threadIdx.x; p < P.np; p += stride)
    B.sorted[B.cell[B.key[p]] + B.rank[p]] = (uint32_t)p;
}
__global__ void k_scatter(Params P, Bufs B) { pdl_enter(); d_scatter(P, B, blockIdx.x, gridDim.x); }
__global__ void kb_scatter(const SceneDev* __restrict__ sd, const int* __restrict__ off, int ns) {
  int s_, blk_, nblk_;
  batch_slot(off, ns, s_, blk_, nblk_);
  const SceneDev& d_ = sd[s_];
  d_scatter(d_.P, d_.B[scene_parity(d_)], blk_, nblk_);
}


// ------------------------------------------------------------------------------------------
// P2G: warp per cell, lane per stencil node, shared 6x6x6 tile per brick
// ------------------------------------------------------------------------------------------
constexpr int kThreads = 128;  // threads per CTA of the brick kernels
// Minimum resident CTAs per SM the register allocation of G2P+MUSL and the deformation update
// is sized for (launch bounds): more CTAs hide more latency, fewer leave registers for the
// FP64 SVD.
#ifndef PM_DEFGRAD_MINB
#define PM_DEFGRAD_MINB 7
#endif
#ifndef PM_HEAD_MINB
#define PM_HEAD_MINB 8
#endif
#ifndef PM_G2P_MINB
#define PM_G2P_MINB 7
#endif
// Unroll factors of the x-layer loop of the 27-node gathers, chosen by measurement on the 2M scene:
// G2P unrolled (0.338 against 0.348 ms rolled), the deformation update rolled (0.373 against
// 0.377 ms unrolled; rolled keeps its code small beside the SVD).
#ifndef PM_G2P_UNROLL_X
#define PM_G2P_UNROLL_X 3
#endif
// 1: the G2P gather forms its B-spline weights where it uses them (fewer live registers).
#ifndef PM_G2P_POLYW
#define PM_G2P_POLYW 1
#endif
// 1: the same in the deformation head's velocity-gradient gather.
#ifndef PM_HEAD_POLYW
#define PM_HEAD_POLYW 1
#endif
// 1: the deformation head loads the next brick's velocity tile and each thread's next particle
// (meta word, position, pic velocity, G2P velocity) with cp.async into double-buffered shared
// slots while the current brick and particle are processed.  Measured on the 2M scene: 88, 90,
// 92, 96 us at steps 1, 20, 100, 500 against 90, 93, 93, 100 us with L2 prefetches.
#ifndef PM_HEAD_ASYNC
#define PM_HEAD_ASYNC 1
#endif
// 1: the G2P gather in two passes over the stencil (velocity, APIC and gradient sums, then latent,
// shear and FLIP sums), so that fewer sums are live at once.
#ifndef PM_G2P_TWOPASS
#define PM_G2P_TWOPASS 0
#endif
// 1: the G2P gather's velocity sums in sum-factorised form (rows, then layers, then the stencil).
#ifndef PM_G2P_FACTORED
#define PM_G2P_FACTORED 0
#endif
#ifndef PM_DEFGRAD_UNROLL_X
#define PM_DEFGRAD_UNROLL_X 1
#endif
constexpr int kG2PUnrollX = PM_G2P_UNROLL_X;
constexpr int kDefgradUnrollX = PM_DEFGRAD_UNROLL_X;
// Unroll factor of the per-run particle loops of the node-parallel scatters (P2G, MUSL) and the
// P2G launch bound (minimum resident CTAs per SM; 0 leaves the register count to the compiler).
#ifndef PM_SCATTER_UNROLL
#define PM_SCATTER_UNROLL 1
#endif
#ifndef PM_P2G_MINB
#define PM_P2G_MINB 6
#endif
constexpr int kScatterUnroll = PM_SCATTER_UNROLL;
constexpr int kWarps = kThreads / 32;
constexpr int kP2GCh = 15;

// Scatter tiles (P2G channels, MUSL channels) are stored with strides (kSX, kSY, 1) instead of
// (36, 6, 1): the 27 offsets a*kSX + b*kSY + c (a, b, c in 0..2) of one stencil are then distinct
// modulo 32, so the 27 lanes of a stencil scatter hit 27 different shared-memory banks.
constexpr int kSX = 43, kSY = 7;
// floats per channel of a padded scatter tile (6 * kSX rounded up to 4 floats, so that the staged
// particle records after the 15 P2G channels stay 16-byte aligned)
constexpr int kTileStride = (6 * kSX + 3) / 4 * 4;
static_assert((15 * kTileStride * 4) % 16 == 0 && 5 * kSX + 5 * kSY + 5 < kTileStride, "scatter tile layout");
__device__ __forceinline__ int tile_pad(int tn) {  // logical node (x*36 + y*6 + z) -> padded offset
  return (tn / 36) * kSX + ((tn / 6) % 6) * kSY + tn % 6;
}


// Per-particle data staged by a warp for its node-parallel scatter: the values every lane reads,
// grouped into float4s (one 128-bit broadcast load each).  The B-spline weights are not staged:
// each lane evaluates the weight of its own stencil node from the particle's position inside its
// base cell (see StencilPoly).  The stage is stored field-major ([8 float4][32 particles] per
// warp): lane i's 128-bit stores of particle i then fall on consecutive banks (a particle-major
// 128-byte record would put the 8 lanes of each store phase on the same four banks).
constexpr int kStageP2G = 8;  // float4s per staged particle:
//   0 f   fx fy fz diff            (f = (x - x_base) / dx, in [0.5, 1.5))
//   1 a   q0 q1 q2 lat0            (q = v - D B r)
//   2 c0  C0x C0y C0z C1x          (C = D dx B, columns)
//   3 c1  C1y C1z C2x C2y
//   4 c2  C2z tau_xx tau_yy tau_zz
//   5 t   tau_xy tau_xz tau_yz lat1
//   6 l0  lat2 lat3 lat4 lat5
//   7 l1  lat6 - - -

// The quadratic B-spline (tools.hpp:153-177) of stencil node k in {0, 1, 2} as a polynomial of the
// position f in [0.5, 1.5) inside the base cell: N0 = (1.5 - f)^2 / 2, N1 = 3/4 - (f - 1)^2,
// N2 = (f - 1/2)^2 / 2, and dN/dx = (f - 1.5, 2 - 2f, f - 0.5) / dx.  A lane keeps the
// coefficients of its node on each axis, so a weight costs three FMAs.
struct StencilPoly {
  float n0, n1, n2, d0, d1;  // N = n0 + n1 f + n2 f^2, dN = d0 + d1 f (times 1/dx)
  __device__ __forceinline__ StencilPoly(int k, float inv_dx) {
    n0 = k == 0 ? 1.125f : (k == 1 ? -0.25f : 0.125f);
    n1 = k == 0 ? -1.5f : (k == 1 ? 2.f : -0.5f);
    n2 = k == 1 ? -1.f : 0.5f;
    d0 = (k == 0 ? -1.5f : (k == 1 ? 2.f : -0.5f)) * inv_dx;
    d1 = (k == 1 ? -2.f : 1.f) * inv_dx;
  }
  __device__ __forceinline__ float N(float f) const { return fmaf(fmaf(n2, f, n1), f, n0); }
  __device__ __forceinline__ float dN(float f) const { return fmaf(d1, f, d0); }
};

// Packed FP32 pairs (sm_100): one instruction performs two multiplies, adds or FMAs, each rounded
// exactly as the scalar instruction, so pair arithmetic gives the bits two scalar instructions give.
// The scatters stage the x and y parts of their per-particle vectors in adjacent float4 slots so that
// they load as register pairs.  PM_PACKED=0 compiles the scalar forms instead.
#ifndef PM_PACKED
#define PM_PACKED 1
#endif
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 lo2(const float4& v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4& v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }

// The x and y axes of a lane's StencilPoly as pairs: N and dN of both axes in one instruction each.
struct StencilPoly2 {
  float2 n0, n1, n2, d0, d1;
  __device__ __forceinline__ StencilPoly2(const StencilPoly& a, const StencilPoly& b)
      : n0{a.n0, b.n0}, n1{a.n1, b.n1}, n2{a.n2, b.n2}, d0{a.d0, b.d0}, d1{a.d1, b.d1} {}
  __device__ __forceinline__ float2 N(float2 f) const { return fma2(fma2(n2, f, n1), f, n0); }
  __device__ __forceinline__ float2 dN(float2 f) const { return fma2(d1, f, d0); }
};

// The quadratic B-spline weight of stencil node k (0, 1, 2) and its derivative (times 1/dx) as
// polynomials of the position f in [0.5, 1.5) inside the base cell (StencilPoly's coefficients),
// for code that forms weights where it uses them instead of keeping all nine per axis live.
__device__ __forceinline__ float bs_n(float f, int k) {
  return k == 0 ? fmaf(fmaf(0.5f, f, -1.5f), f, 1.125f) : (k == 1 ? fmaf(fmaf(-1.f, f, 2.f), f, -0.25f)
                                                                  : fmaf(fmaf(0.5f, f, -0.5f), f, 0.125f));
}
__device__ __forceinline__ float bs_dn(float f, int k, float inv_dx) {
  return (k == 0 ? f - 1.5f : (k == 1 ? fmaf(-2.f, f, 2.f) : f - 0.5f)) * inv_dx;
}

size_t p2g_smem_bytes() { return sizeof(float) * kP2GCh * kTileStride + sizeof(float4) * kStageP2G * kThreads; }


__device__ __forceinline__ int tile_to_node(int tn, int bx, int by, int bz, const Ctrl* c) {
  int tx = tn / 36, ty = (tn / 6) % 6, tz = tn % 6;
  int gx = bx + (tx >> 2), gy = by + (ty >> 2), gz = bz + (tz >> 2);
  if (gx >= c->nb[0] || gy >= c->nb[1] || gz >= c->nb[2]) return -1;
  return ((gx * c->nb[1] + gy) * c->nb[2] + gz) * kBrickNodes + (tx & 3) * 16 + (ty & 3) * 4 + (tz & 3);
}

// Local cell (0..63, lx*16 + ly*4 + lz) of a particle inside brick (bx, by, bz), clamped.
__device__ __forceinline__ int local_cell(const AxisW aw[3], const Ctrl* c, int bx, int by, int bz) {
  const int lx = min(max(aw[0].base - c->g0[0] - bx * 4, 0), 3);
  const int ly = min(max(aw[1].base - c->g0[1] - by * 4, 0), 3);
  const int lz = min(max(aw[2].base - c->g0[2] - bz * 4, 0), 3);
  return lx * 16 + ly * 4 + lz;
}

// One CTA per brick (grid-stride).  Each warp takes 32 consecutive particles of the brick's
// sorted range: lane i stages particle i (weights, APIC terms, stress, latent), then the warp
// walks the runs of equal cells in its 32 particles (found with a ballot) and, for each run,
// lane l < 27 accumulates the run's particles into stencil node l in registers and adds the
// sums once to the brick's shared 6x6x6 tile.  Block barriers only around the tile.
__device__ __forceinline__ void d_p2g(const Params& P, const Bufs& B, const int blk_, const int nblk_) {
  const Ctrl* c = B.ctrl;
  if (c->halt || c->idle) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* tile = reinterpret_cast<float*>(smem_raw);                       // [kP2GCh][216]
  float4* stw = reinterpret_cast<float4*>(tile + kP2GCh * kTileStride);  // [kWarps][kStageP2G][32]
  const int S = P.np_stride;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float4* st = stw + warp * kStageP2G * 32;
  const int la = lane / 9, lb = (lane / 3) % 3, lc = lane % 3;
  const float fa = (float)la, fb = (float)lb, fc = (float)lc;
  const float D = P.apicD, dx = P.dx;
  const bool apic = P.flip_ratio < 0.f;
  const StencilPoly px(la, P.inv_dx), py(lb, P.inv_dx), pz(lc, P.inv_dx);
#if PM_PACKED
  const StencilPoly2 pxy(px, py);
  const float2 fa2 = dup2(fa), fb2 = dup2(fb), fc2 = dup2(fc);
#endif
  // the list length is re-read per brick (one L1 hit) rather than held across the scatter; CTAs take
  // every nblk_-th brick (contiguous runs of bricks per CTA measured slower: 330 against 291 us)
  for (int ib = blk_; ib < (int)B.blist_n[0]; ib += nblk_) {
    const uint4 be = B.blist_occ[ib];
    const int b = (int)be.x;
    const uint32_t ps = be.y, pe = be.z;
    int bx, by, bz;
    brick_coords(b, c, bx, by, bz);
    {
      // the tile is zeroed before every brick (zeroing each node in the flush instead, which
      // saves this barrier, measured 0.937 against 0.936 ms per step)
      float4* t4 = reinterpret_cast<float4*>(tile);  // kP2GCh * kTileStride is a multiple of 4
      for (int i = threadIdx.x; i < kP2GCh * kTileStride / 4; i += kThreads) t4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
#if PM_PREFETCH
    uint32_t o_next = ps + 32u * warp + lane < pe ? B.sorted[ps + 32u * warp + lane] : 0u;
#endif
    for (uint32_t c0 = ps + 32u * warp; c0 < pe; c0 += 32u * kWarps) {
      const int n = (int)min(32u, pe - c0);
      int cl = -1;
#if PM_PREFETCH
      const uint32_t o_cur = o_next, c1 = c0 + 32u * kWarps;
      o_next = c1 + lane < pe ? B.sorted[c1 + lane] : 0u;
#endif
      if (lane < n) {
#if PM_PREFETCH
        const uint32_t o = o_cur;
#else
        const uint32_t o = B.sorted[c0 + lane];
#endif
        AxisW aw[3];
        float r[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          aw[d] = axis_weights(B.pin[(F_X + d) * S + o], P.anchor[d], dx, P.inv_dx);
          r[d] = aw[d].r;
        }
        cl = local_cell(aw, c, bx, by, bz);
        float v[3], Bm[9], q[3], C[9];
#pragma unroll
        for (int d = 0; d < 3; ++d) v[d] = B.pin[(F_V + d) * S + o];
#pragma unroll
        for (int k = 0; k < 9; ++k) Bm[k] = apic ? B.pin[(F_B + k) * S + o] : 0.f;
#pragma unroll
        for (int i = 0; i < 3; ++i) q[i] = v[i] - D * (Bm[3 * i] * r[0] + Bm[3 * i + 1] * r[1] + Bm[3 * i + 2] * r[2]);
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
          for (int i = 0; i < 3; ++i) C[3 * k + i] = D * dx * Bm[3 * i + k];
        float tau[6], lat[7];
#pragma unroll
        for (int k = 0; k < 6; ++k) tau[k] = B.pin[(F_TAU + k) * S + o];
#pragma unroll
        for (int k = 0; k < 7; ++k) lat[k] = B.pin[(F_LAT + k) * S + o];
#if PM_PACKED
        // packed layout: pairs (fx, fy), (q0, q1), (C0x, C0y), (C1x, C1y), (C2x, C2y), (lat0, lat1),
        // (lat2, lat3), (lat4, lat5), (lat6, diffusion) each in one aligned half of a float4
        st[0 * 32 + lane] = make_float4(r[0] * P.inv_dx, r[1] * P.inv_dx, r[2] * P.inv_dx, C[2]);
        st[1 * 32 + lane] = make_float4(q[0], q[1], q[2], C[5]);
        st[2 * 32 + lane] = make_float4(C[0], C[1], C[3], C[4]);
        st[3 * 32 + lane] = make_float4(C[6], C[7], C[8], tau[0]);
        st[4 * 32 + lane] = make_float4(tau[1], tau[2], tau[3], tau[4]);
        st[5 * 32 + lane] = make_float4(tau[5], 0.f, lat[0], lat[1]);
        st[6 * 32 + lane] = make_float4(lat[2], lat[3], lat[4], lat[5]);
        st[7 * 32 + lane] = make_float4(lat[6], B.pin[F_DIFF * S + o], 0.f, 0.f);
#else
        st[0 * 32 + lane] = make_float4(r[0] * P.inv_dx, r[1] * P.inv_dx, r[2] * P.inv_dx, B.pin[F_DIFF * S + o]);
        st[1 * 32 + lane] = make_float4(q[0], q[1], q[2], lat[0]);
        st[2 * 32 + lane] = make_float4(C[0], C[1], C[2], C[3]);
        st[3 * 32 + lane] = make_float4(C[4], C[5], C[6], C[7]);
        st[4 * 32 + lane] = make_float4(C[8], tau[0], tau[1], tau[2]);
        st[5 * 32 + lane] = make_float4(tau[3], tau[4], tau[5], lat[1]);
        st[6 * 32 + lane] = make_float4(lat[2], lat[3], lat[4], lat[5]);
        st[7 * 32 + lane] = make_float4(lat[6], 0.f, 0.f, 0.f);
#endif
      }
#if PM_PREFETCH
      if (c1 + lane < pe) {  // the next chunk's fields, while this chunk scatters
        const float* q = B.pin + o_next;
#pragma unroll
        for (int f = F_X; f < F_F; ++f) prefetch_l2(q + (size_t)f * S);
#pragma unroll
        for (int f = F_LAT; f < F_EPD; ++f) prefetch_l2(q + (size_t)f * S);
#pragma unroll
        for (int f = F_TAU; f < F_COUNT; ++f) prefetch_l2(q + (size_t)f * S);
      }
#endif
      // runs of equal cells among the warp's particles
      const int prev = __shfl_up_sync(0xffffffffu, cl, 1);
      uint32_t heads = __ballot_sync(0xffffffffu, lane < n && (lane == 0 || cl != prev));
      __syncwarp();
      while (heads) {
        const int s0 = __ffs(heads) - 1;
        heads &= heads - 1;
        const int s1 = heads ? __ffs(heads) - 1 : n;
        const int cell = __shfl_sync(0xffffffffu, cl, s0);
        if (lane < 27) {
          float acc[kP2GCh];
#if PM_PACKED
          // A B-spline weight of a stencil node is never below 1e-16 unless it is exactly 0 (the
          // particle's offset f from its base cell is a float in [0.5, 1.5), so (f - 1/2)^2 / 2 is 0
          // or at least about 1.8e-15), so p2g.cpp:39's skip of weights <= 1e-25 only skips terms
          // that are 0 anyway: the weight is used as is.
          float2 a_v = make_float2(0.f, 0.f), a_l01 = a_v, a_l23 = a_v, a_l45 = a_v, a_l6s = a_v;
          float a_m = 0.f, a_vz = 0.f, a_f0 = 0.f, a_f1 = 0.f, a_f2 = 0.f;
#pragma unroll kScatterUnroll
          for (int q = s0; q < s1; ++q) {
            const float4 S0 = st[0 * 32 + q], S1 = st[1 * 32 + q], S2 = st[2 * 32 + q], S3 = st[3 * 32 + q];
            const float4 S4 = st[4 * 32 + q], S5 = st[5 * 32 + q], S6 = st[6 * 32 + q], S7 = st[7 * 32 + q];
            const float2 nxy = pxy.N(lo2(S0)), dxy = pxy.dN(lo2(S0));
            const float nx = nxy.x, ny = nxy.y, nz = pz.N(S0.z);
            const float nyz = ny * nz;
            const float w = nx * nyz;
            const float gx = dxy.x * nyz, gy = nx * dxy.y * nz, gz = nx * ny * pz.dN(S0.z);
            const float2 w2 = dup2(w);
            a_m += w;
            float2 vxy = fma2(fa2, lo2(S2), lo2(S1));
            vxy = fma2(fb2, hi2(S2), vxy);
            vxy = fma2(fc2, lo2(S3), vxy);
            a_v = fma2(w2, vxy, a_v);
            a_vz += w * (S1.z + fa * S0.w + fb * S1.w + fc * S3.z);
            a_f0 += S3.w * gx + S4.z * gy + S4.w * gz;
            a_f1 += S4.z * gx + S4.x * gy + S5.x * gz;
            a_f2 += S4.w * gx + S5.x * gy + S4.y * gz;
            a_l01 = fma2(w2, hi2(S5), a_l01);
            a_l23 = fma2(w2, lo2(S6), a_l23);
            a_l45 = fma2(w2, hi2(S6), a_l45);
            a_l6s = fma2(w2, lo2(S7), a_l6s);
          }
          acc[0] = a_m; acc[1] = a_v.x; acc[2] = a_v.y; acc[3] = a_vz;
          acc[4] = a_f0; acc[5] = a_f1; acc[6] = a_f2;
          acc[7] = a_l01.x; acc[8] = a_l01.y; acc[9] = a_l23.x; acc[10] = a_l23.y;
          acc[11] = a_l45.x; acc[12] = a_l45.y; acc[13] = a_l6s.x; acc[14] = a_l6s.y;
#else
#pragma unroll
          for (int k = 0; k < kP2GCh; ++k) acc[k] = 0.f;
#pragma unroll kScatterUnroll
          for (int q = s0; q < s1; ++q) {
            const float4 Fr = st[0 * 32 + q], A = st[1 * 32 + q], C0 = st[2 * 32 + q], C1 = st[3 * 32 + q];
            const float4 C2 = st[4 * 32 + q], T = st[5 * 32 + q], L0 = st[6 * 32 + q], L1 = st[7 * 32 + q];
            const float nx = px.N(Fr.x), ny = py.N(Fr.y), nz = pz.N(Fr.z);
            const float nyz = ny * nz;
            const float w = nx * nyz;
            const float gx = px.dN(Fr.x) * nyz, gy = nx * py.dN(Fr.y) * nz, gz = nx * ny * pz.dN(Fr.z);
            const float wm = w > 1e-25f ? w : 0.f;  // p2g.cpp:39
            acc[0] += wm;
            acc[1] += wm * (A.x + fa * C0.x + fb * C0.w + fc * C1.z);
            acc[2] += wm * (A.y + fa * C0.y + fb * C1.x + fc * C1.w);
            acc[3] += wm * (A.z + fa * C0.z + fb * C1.y + fc * C2.x);
            acc[4] += C2.y * gx + T.x * gy + T.y * gz;
            acc[5] += T.x * gx + C2.z * gy + T.z * gz;
            acc[6] += T.y * gx + T.z * gy + C2.w * gz;
            acc[7] += wm * A.w;
            acc[8] += wm * T.w;
            acc[9] += wm * L0.x;
            acc[10] += wm * L0.y;
            acc[11] += wm * L0.z;
            acc[12] += wm * L0.w;
            acc[13] += wm * L1.x;
            acc[14] += wm * Fr.w;
          }
#endif
          const int tp = ((cell >> 4) + la) * kSX + (((cell >> 2) & 3) + lb) * kSY + ((cell & 3) + lc);
#pragma unroll
          for (int k = 0; k < kP2GCh; ++k)
            if (acc[k] != 0.f) atomicAdd(&tile[k * kTileStride + tp], acc[k]);
        }
      }
      __syncwarp();
    }
    __syncthreads();
    for (int tn = threadIdx.x; tn < kTileNodes; tn += kThreads) {
      const float* t = tile + tile_pad(tn);
      const float m = t[0];
      const int node = m != 0.f ? tile_to_node(tn, bx, by, bz, c) : -1;  // massless nodes are not flushed
      if (node >= 0) {
        float4* rec = B.grid + (size_t)node * 4;
        red_add_v4(rec + 0, m, t[1 * kTileStride], t[2 * kTileStride], t[3 * kTileStride]);
        red_add_v4(rec + 1, t[4 * kTileStride], t[5 * kTileStride], t[6 * kTileStride], t[7 * kTileStride]);
        red_add_v4(rec + 2, t[8 * kTileStride], t[9 * kTileStride], t[10 * kTileStride], t[11 * kTileStride]);
        red_add_v4(rec + 3, t[12 * kTileStride], t[13 * kTileStride], t[14 * kTileStride], 0.f);
      }
    }
    __syncthreads();
  }
}
#if PM_P2G_MINB > 0
__global__ void __launch_bounds__(kThreads, PM_P2G_MINB) k_p2g(Params P, Bufs B) {
  pdl_enter();
  d_p2g(P, B, blockIdx.x, gridDim.x);
}
#else
__global__ void __launch_bounds__(kThreads) k_p2g(Params P, Bufs B) {
  pdl_enter();
  d_p2g(P, B, blockIdx.x, gridDim.x);
}
#endif
__global__ void __launch_bounds__(kThreads) kb_p2g(const SceneDev* __restrict__ sd, const int* __restrict__ off, int ns) {
  int s_, blk_, nblk_;
  batch_slot(off, ns, s_, blk_, nblk_);
  __shared__ SceneShared ss_;
  load_scene_shared(sd[s_], ss_);
  d_p2g(ss_.P, ss_.B, blk_, nblk_);
}


// ------------------------------------------------------------------------------------------
// grid update with collisions
// ------------------------------------------------------------------------------------------
__device__ float sd_spatula(float px_, float py_, float pz_) {  // object_spatula.hpp:40-82
  const float halfWidth = 0.368f, halfLength = 0.736f, halfThickness = 0.07f, offset = 0.05f;
  float px = fabsf(px_), py = pz_;
  float b1 = halfWidth + offset, b2 = (halfWidth + offset) * 0.25f, he = halfLength + offset;
  float bax = b2 - b1, bay = he - (-he);
  float pax = px - b1, pay = py - (-he);
  float h = fmaxf(0.f, fminf(1.f, (pax * bax + pay * bay) / (bax * bax + bay * bay)));
  float dxs = pax - bax * h, dys = pay - bay * h;
  float d_side = sqrtf(dxs * dxs + dys * dys);
  float inside_x = b1 - (b1 - b2) * (py + he) / (2.f * he);
  float d_inside = px - inside_x;
  float d2 = (px < inside_x) ? d_inside : d_side;
  if (py > he) {
    d2 = sqrtf(px * px + (py - he) * (py - he)) - b2;
  } else if (py < -he) {
    float rx = halfWidth + offset, rz = 1.5f * (halfWidth + offset);
    float qx = px, qz = py + he;
    float k0 = sqrtf((qx / rx) * (qx / rx) + (qz / rz) * (qz / rz));
    float k1 = sqrtf((qx / (rx * rx)) * (qx / (rx * rx)) + (qz / (rz * rz)) * (qz / (rz * rz)));
    d2 = k0 * (k0 - 1.f) / k1;
  }
  float dy = fabsf(py_) - halfThickness;
  float mx = fmaxf(d2, dy);
  float ex = fmaxf(d2, 0.f), ey = fmaxf(dy, 0.f);
  return fminf(mx, 0.f) + sqrtf(ex * ex + ey * ey);
}
__device__ float sd_box(const ObjDev& o, float px, float py, float pz) {
  float qx = fabsf(px) - o.half[0], qy = fabsf(py) - o.half[1], qz = fabsf(pz) - o.half[2];
  float ox = fmaxf(qx, 0.f), oy = fmaxf(qy, 0.f), oz = fmaxf(qz, 0.f);
  return sqrtf(ox * ox + oy * oy + oz * oz) + fminf(fmaxf(qx, fmaxf(qy, qz)), 0.f);
}
__device__ __forceinline__ float sd_local(const ObjDev& o, float x, float y, float z) {
  return o.kind == OBJ_SPATULA ? sd_spatula(x, y, z) : sd_box(o, x, y, z);
}
__device__ __forceinline__ void to_local(const ObjDev& o, const float X[3], float p[3]) {
  float a = X[0] - o.tx, b = X[1] - o.ty, d = X[2] - o.tz;
  p[0] = o.Rinv[0] * a + o.Rinv[1] * b + o.Rinv[2] * d;
  p[1] = o.Rinv[3] * a + o.Rinv[4] * b + o.Rinv[5] * d;
  p[2] = o.Rinv[6] * a + o.Rinv[7] * b + o.Rinv[8] * d;
}
__device__ bool obj_inside(const ObjDev& o, const float X[3]) {
  if (o.kind == OBJ_GROUND) return !(X[1] > o.y0);
  if (o.kind == OBJ_CURVE) return !(X[1] > X[0] * X[0]);
  float p[3];
  to_local(o, X, p);
  return sd_local(o, p[0], p[1], p[2]) < 0.f;
}
__device__ void obj_normal(const ObjDev& o, const float X[3], float n[3]) {
  if (o.kind == OBJ_GROUND) { n[0] = 0.f; n[1] = 1.f; n[2] = 0.f; return; }
  if (o.kind == OBJ_CURVE) {
    float a = -2.f * X[0], b = 1.f;
    float l = sqrtf(a * a + b * b);
    n[0] = a / l; n[1] = b / l; n[2] = 0.f;
    return;
  }
  float p[3];
  to_local(o, X, p);
  const float e = 1e-4f;  // object_spatula.hpp:109-117
  float nl[3] = {sd_local(o, p[0] + e, p[1], p[2]) - sd_local(o, p[0] - e, p[1], p[2]),
                 sd_local(o, p[0], p[1] + e, p[2]) - sd_local(o, p[0], p[1] - e, p[2]),
                 sd_local(o, p[0], p[1], p[2] + e) - sd_local(o, p[0], p[1], p[2] - e)};
  float l = sqrtf(nl[0] * nl[0] + nl[1] * nl[1] + nl[2] * nl[2]);
  if (l > 0.f) { nl[0] /= l; nl[1] /= l; nl[2] /= l; }
  // (linear^-1)^T n = Rinv^T n
  float w[3] = {o.Rinv[0] * nl[0] + o.Rinv[3] * nl[1] + o.Rinv[6] * nl[2],
                o.Rinv[1] * nl[0] + o.Rinv[4] * nl[1] + o.Rinv[7] * nl[2],
                o.Rinv[2] * nl[0] + o.Rinv[5] * nl[1] + o.Rinv[8] * nl[2]};
  float wl = sqrtf(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  if (wl > 0.f) { w[0] /= wl; w[1] /= wl; w[2] /= wl; }
  n[0] = w[0]; n[1] = w[1]; n[2] = w[2];
}
__device__ void obj_velocity(const ObjDev& o, const float X[3], float v[3]) {
  if (o.kind == OBJ_GROUND || o.kind == OBJ_CURVE) { v[0] = v[1] = v[2] = 0.f; return; }
  float r[3] = {X[0] - o.tx, X[1] - o.ty, X[2] - o.tz};
  v[0] = o.vlin[0] + (o.omega[1] * r[2] - o.omega[2] * r[1]);
  v[1] = o.vlin[1] + (o.omega[2] * r[0] - o.omega[0] * r[2]);
  v[2] = o.vlin[2] + (o.omega[0] * r[1] - o.omega[1] * r[0]);
}
__device__ bool plate_inside(const PlateDev& pl, const float X[3]) {  // object_plate.hpp:13-57
  switch (pl.type) {
    case PT_LEFT: return X[1] < pl.upper && X[1] > pl.lower && (X[0] - pl.pos) <= 0;
    case PT_RIGHT: return X[1] < pl.upper && X[1] > pl.lower && (pl.pos - X[0]) <= 0;
    case PT_BOTTOM: return X[0] < pl.upper && X[0] > pl.lower && (X[1] - pl.pos) <= 0;
    case PT_TOP: return X[0] < pl.upper && X[0] > pl.lower && (pl.pos - X[1]) <= 0;
    case PT_BACK: return X[2] - pl.pos <= 0;
    case PT_FRONT: return pl.pos - X[2] <= 0;
  }
  return false;
}

// boundary_collision.cpp:5-316 (3D branch)
__device__ void boundary_collision(const Ctrl* c, float dtf, float dx, float Xi_[3], float vi[3], uint32_t& err) {
  float vo[3] = {vi[0], vi[1], vi[2]};
  float Xi[3] = {Xi_[0] + dtf * vi[0], Xi_[1] + dtf * vi[1], Xi_[2] + dtf * vi[2]};
  bool infl = false;
  const int knife = c->knife;
  if (knife >= 0) {
    const ObjDev& o = c->objects[knife];
    float p[3];
    to_local(o, Xi, p);
    if (sd_local(o, p[0], p[1], p[2]) < 2.f * dx) infl = true;
  }
  for (int oi = 0; oi < c->n_objects; ++oi) {
    const ObjDev& o = c->objects[oi];
    if (!obj_inside(o, Xi)) continue;
    float vobj[3];
    obj_velocity(o, Xi, vobj);
    float vr[3] = {vo[0] - vobj[0], vo[1] - vobj[1], vo[2] - vobj[2]};
    if (o.bc == BC_NOSLIP) { vr[0] = vr[1] = vr[2] = 0.f; }
    else if (o.bc == BC_SLIPFREE) {
      float n[3];
      obj_normal(o, Xi, n);
      float dot = vr[0] * n[0] + vr[1] * n[1] + vr[2] * n[2];
      if (dot < 0.f) {
        float vt[3] = {vr[0] - dot * n[0], vr[1] - dot * n[1], vr[2] - dot * n[2]};
        if (o.friction > 0.f) {
          float vtn = sqrtf(vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2]);
          if (-dot * o.friction < vtn) { float sc = dot * o.friction / vtn; for (int k = 0; k < 3; ++k) vr[k] = vt[k] + vt[k] * sc; }
          else { vr[0] = vr[1] = vr[2] = 0.f; }
        } else { vr[0] = vt[0]; vr[1] = vt[1]; vr[2] = vt[2]; }
      }
    } else if (o.bc == BC_SLIPSTICK) {
      float n[3];
      obj_normal(o, Xi, n);
      float dot = vr[0] * n[0] + vr[1] * n[1] + vr[2] * n[2];
      for (int k = 0; k < 3; ++k) vr[k] -= dot * n[k];
      if (dot < 0.f && o.friction > 0.f) {
        float vtn = sqrtf(vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2]);
        if (-dot * o.friction < vtn) { float sc = dot * o.friction / vtn; for (int k = 0; k < 3; ++k) vr[k] += vr[k] * sc; }
        else { vr[0] = vr[1] = vr[2] = 0.f; }
      }
    } else { err |= E_INVALID_BC; return; }
    for (int k = 0; k < 3; ++k) vi[k] = vr[k] + vobj[k];
    if (oi == knife) {
      infl = true;
      if (Xi[1] < 0.8f * dx) {  // thin-film rule, boundary_collision.cpp:93-111
        float n[3];
        obj_normal(o, Xi, n);
        float t[3] = {-n[1] * n[0], 1.f - n[1] * n[1], -n[1] * n[2]};
        float tn = sqrtf(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        if (tn > 1e-6f) { t[0] /= tn; t[1] /= tn; t[2] /= tn; } else { t[0] = t[1] = t[2] = 0.f; }
        float vn = sqrtf(vobj[0] * vobj[0] + vobj[1] * vobj[1] + vobj[2] * vobj[2]);
        for (int k = 0; k < 3; ++k) vi[k] = vobj[k] + t[k] * (0.2f * vn);
      }
    }
    vo[0] = vi[0]; vo[1] = vi[1]; vo[2] = vi[2];
  }
  for (int pi = 0; pi < c->n_plates; ++pi) {
    const PlateDev& pl = c->plates[pi];
    if (!plate_inside(pl, Xi)) continue;
    if (infl && pl.type == PT_BOTTOM) {
      if (vi[1] < pl.vy) { vi[1] = pl.vy; vo[0] = vi[0]; vo[1] = vi[1]; vo[2] = vi[2]; }
      continue;
    }
    float vr[3] = {vo[0] - pl.vx, vo[1] - pl.vy, vo[2] - pl.vz};
    const int nax = (pl.type == PT_TOP || pl.type == PT_BOTTOM) ? 1 : (pl.type == PT_LEFT || pl.type == PT_RIGHT) ? 0 : 2;
    const int t0 = nax == 0 ? 1 : 0, t1 = nax == 2 ? 1 : 2;
    bool apply;
    if (pl.bc == BC_NOSLIP) { vr[0] = vr[1] = vr[2] = 0.f; apply = false; }
    else if (pl.bc == BC_SLIPSTICK) apply = true;
    else if (pl.bc == BC_SLIPFREE) {
      apply = (pl.type == PT_TOP && vr[1] > 0) || (pl.type == PT_BOTTOM && vr[1] < 0) ||
              (pl.type == PT_LEFT && vr[0] < 0) || (pl.type == PT_RIGHT && vr[0] > 0) ||
              (pl.type == PT_FRONT && vr[2] > 0) || (pl.type == PT_BACK && vr[2] < 0);
    } else { err |= E_INVALID_BC; return; }
    if (apply) {
      float vel_t = sqrtf(vr[t0] * vr[t0] + vr[t1] * vr[t1]);
      float fvn = pl.friction * fabsf(vr[nax]);
      if (pl.friction == 0.f) {
      } else if (vel_t <= fvn) { vr[t0] = 0.f; vr[t1] = 0.f; }
      else { float sc = (vel_t - fvn) / vel_t; vr[t0] *= sc; vr[t1] *= sc; }
      vr[nax] = 0.f;
    }
    vi[0] = vr[0] + pl.vx; vi[1] = vr[1] + pl.vy; vi[2] = vr[2] + pl.vz;
    vo[0] = vi[0]; vo[1] = vi[1]; vo[2] = vi[2];
  }
}

__device__ __forceinline__ void d_grid_update(const Params& P, const Bufs& B, const int blk_, const int nblk_) {
  const Ctrl* c = B.ctrl;
  if (c->halt || c->idle) return;
  const int nt = (int)B.blist_n[1] * kBrickNodes;  // nodes of the bricks a stencil reaches
  const float dtf = (float)c->dt;
  const float dtv = dtf * P.particle_volume;
  const float dtg[3] = {dtf * P.gravity[0], dtf * P.gravity[1], dtf * P.gravity[2]};
  const int stride = nblk_ * blockDim.x;
  uint32_t err = 0;
  for (int t = blk_ * blockDim.x + threadIdx.x; t < nt; t += stride) {
    const int n = (int)B.blist_touch[t >> 6] * kBrickNodes + (t & 63);
    float4* rec = B.grid + (size_t)n * 4;
    float4 r0 = rec[0];
    if (!(r0.x > 0.f)) continue;
    float4 r1 = rec[1], r2 = rec[2], r3 = rec[3];
    const float sw = r0.x;
    const float inv = 1.f / sw;
    // P2G normalisation (p2g.cpp:97-124)
    float v[3] = {r0.y * inv, r0.z * inv, r0.w * inv};
    float lat[7] = {r1.w * inv, r2.x * inv, r2.y * inv, r2.z * inv, r2.w * inv, r3.x * inv, r3.y * inv};
    float shear = r3.z * inv;
    float ps = lat[0] + lat[1] + lat[2] + lat[3];
    if (ps > 1e-6f) { for (int k = 0; k < 4; ++k) lat[k] /= ps; }
    const float mi = sw * P.particle_mass;
    // explicit update (explicit_euler_update.cpp:199-229)
    float nv[3];
    const float fs = -dtv / mi;
    nv[0] = v[0] + (r1.x * fs + dtg[0]);
    nv[1] = v[1] + (r1.y * fs + dtg[1]);
    nv[2] = v[2] + (r1.z * fs + dtg[2]);
    // node position
    const int b = n >> 6, loc = n & 63;
    int bx, by, bz;
    brick_coords(b, c, bx, by, bz);
    const int gi[3] = {c->g0[0] + bx * 4 + (loc >> 4), c->g0[1] + by * 4 + ((loc >> 2) & 3), c->g0[2] + bz * 4 + (loc & 3)};
    float X[3] = {node_pos(gi[0], P.anchor[0], P.dx), node_pos(gi[1], P.anchor[1], P.dx), node_pos(gi[2], P.anchor[2], P.dx)};
    boundary_collision(c, dtf, P.dx, X, nv, err);
    // updated record, laid out as the G2P tile reads it (4 x 16 B per node): the pure-APIC G2P
    // reads the first three, the FLIP velocity change sits in the fourth
    rec[0] = make_float4(nv[0], nv[1], nv[2], lat[0]);
    rec[1] = make_float4(lat[1], lat[2], lat[3], lat[4]);
    rec[2] = make_float4(lat[5], lat[6], shear, mi);
    rec[3] = make_float4(nv[0] - v[0], nv[1] - v[1], nv[2] - v[2], 0.f);
  }
  if (err) atomicOr(&B.ctrl->error_flags, err);
}
__global__ void k_grid_update(Params P, Bufs B) { pdl_enter(); d_grid_update(P, B, blockIdx.x, gridDim.x); }
__global__ void kb_grid_update(const SceneDev* __restrict__ sd, const int* __restrict__ off, int ns) {
  int s_, blk_, nblk_;
  batch_slot(off, ns, s_, blk_, nblk_);
  __shared__ SceneShared ss_;
  load_scene_shared(sd[s_], ss_);
  d_grid_update(ss_.P, ss_.B, blk_, nblk_);
}


// ------------------------------------------------------------------------------------------
// G2P + mixing + MUSL (velocity update and re-scatter)
// ------------------------------------------------------------------------------------------
// The G2P node tile is field-major too: record part k (0..3) of tile node tn at
// tile[k * kG2PTileStride + tn].  The stride 218 = 2 mod 8 puts the four parts of a node on
// different bank groups, so the loads of a brick's tile are conflict-free.
constexpr int kG2PTileStride = 218;
// MUSL stage, field-major like the P2G stage ([4 float4][32 particles] per warp):
constexpr int kStageMUSL = 4;  // float4s per staged particle:
//   0 q   q0 q1 q2 fx  (q = v_new - D B_new r; f = position in the base cell, StencilPoly)
//   1 c0  C0x C0y C0z C1x
//   2 c1  C1y C1z C2x C2y
//   3 c2  C2z fy fz -

// 1: each lane copies its next particle's position and latent into a lane-private shared slot with
// cp.async while the current particle is finished and scattered (replaces the L2 prefetch of those
// fields).  Measured on the 2M scene: G2P 281, 294, 307, 330 us at steps 1, 20, 100, 500 against
// 290, 301, 314, 338 us with the L2 prefetch alone, and 140 -> 104 bytes of spill loads.  Moving
// the deformation head's L2 prefetch ahead of the particle it overlaps gained nothing (92-101 us).
#ifndef PM_G2P_ASYNC
#define PM_G2P_ASYNC 1
#endif
#if PM_G2P_ASYNC && !PM_PREFETCH
#error "PM_G2P_ASYNC uses the next chunk's sorted index that PM_PREFETCH loads"
#endif
constexpr int kG2PAsyncFields = 10;  // x (3), latent (7)
size_t g2p_smem_bytes() {
  return sizeof(float4) * 4 * kG2PTileStride + sizeof(float) * 4 * kTileStride + sizeof(float4) * kStageMUSL * kThreads +
         (PM_G2P_ASYNC ? sizeof(float) * kG2PAsyncFields * kThreads : 0);
}

__device__ __forceinline__ float smooth_step(float e0, float e1, float x) {  // g2p.cpp:7-10
  float t = fmaxf(0.f, fminf(1.f, (x - e0) / (e1 - e0)));
  return t * t * (3.f - 2.f * t);
}

// One CTA per brick.  The brick's 6x6x6 node tile (updated records, 4 x float4 per node) is
// loaded once; each warp then takes 32 consecutive particles of the brick's sorted range: lane i
// gathers G2P for particle i, writes its new state in sorted order and stages its MUSL data; the
// warp then scatters the staged particles run by run of equal cells, lane l < 27 owning stencil
// node l, into the brick's shared MUSL tile, flushed once per brick.
// kFlip: FLIP blending in use (flip_ratio >= -1); false compiles the pure-APIC kernel, which
// neither reads the old particle velocity nor gathers the grid's velocity change.
template <bool kFlip>
__device__ __forceinline__ void d_g2p_musl(const Params& P, const Bufs& B, const int blk_, const int nblk_) {
  const Ctrl* c = B.ctrl;
  if (c->halt || c->idle) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* tile = reinterpret_cast<float4*>(smem_raw);                  // [4][kG2PTileStride]
  float* mtile = reinterpret_cast<float*>(tile + 4 * kG2PTileStride);  // [4][kTileStride], padded layout
  float4* stw = reinterpret_cast<float4*>(mtile + 4 * kTileStride);  // [kWarps][kStageMUSL][32]
  const int S = P.np_stride;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float4* st = stw + warp * kStageMUSL * 32;
#if PM_G2P_ASYNC
  // lane-private slots [field][lane] of this warp: only the owning lane writes and reads them
  float* xs = reinterpret_cast<float*>(stw + kWarps * kStageMUSL * 32) + warp * kG2PAsyncFields * 32;
#endif
  const int la = lane / 9, lb = (lane / 3) % 3, lc = lane % 3;
  const float D = P.apicD, dx = P.dx;
  const float fr = P.flip_ratio;
  const bool apic = fr < 0.f, use_flip = kFlip, musl = P.use_musl != 0;
  const float dtf = (float)c->dt;
  // pigment mixing factor pieces (g2p.cpp:105-119)
  float time_factor = 1.f;
  {
    float ct = (float)c->time;
    if (ct > P.start_boost && P.end_boost > P.start_boost) {
      float t = (ct - P.start_boost) / (P.end_boost - P.start_boost);
      t = fminf(fmaxf(t, 0.f), 1.f);
      time_factor = 1.f + t * (P.boost_factor - 1.f);
    }
  }
  const float dyn = P.D_max * time_factor;
  const int nbr = (int)B.blist_n[0];
  for (int ib = blk_; ib < nbr; ib += nblk_) {
    const uint4 be = B.blist_occ[ib];
    const int b = (int)be.x;
    const uint32_t ps = be.y, pe = be.z;
    int bx, by, bz;
    brick_coords(b, c, bx, by, bz);
    for (int i = threadIdx.x; i < kTileNodes * 4; i += kThreads) {
      if (!kFlip && (i & 3) == 3) continue;  // the velocity change is read by FLIP only
      const int node = tile_to_node(i >> 2, bx, by, bz, c);
      tile[(i & 3) * kG2PTileStride + (i >> 2)] =
          node >= 0 ? B.grid[(size_t)node * 4 + (i & 3)] : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    {
      float4* m4 = reinterpret_cast<float4*>(mtile);
      for (int i = threadIdx.x; i < kTileStride; i += kThreads) m4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
#if PM_PREFETCH
    uint32_t o_next = ps + 32u * warp + lane < pe ? B.sorted[ps + 32u * warp + lane] : 0u;
#endif
#if PM_G2P_ASYNC
    if (ps + 32u * warp + lane < pe) {
#pragma unroll
      for (int f = 0; f < 3; ++f) cp_async4(xs + f * 32 + lane, B.pin + (size_t)(F_X + f) * S + o_next);
#pragma unroll
      for (int f = 0; f < 7; ++f) cp_async4(xs + (3 + f) * 32 + lane, B.pin + (size_t)(F_LAT + f) * S + o_next);
    }
    cp_async_commit();
#endif
    for (uint32_t c0 = ps + 32u * warp; c0 < pe; c0 += 32u * kWarps) {
      const int n = (int)min(32u, pe - c0);
      int cl = -1;
#if PM_PREFETCH
      const uint32_t o_cur = o_next, c1 = c0 + 32u * kWarps;
      o_next = c1 + lane < pe ? B.sorted[c1 + lane] : 0u;
#endif
#if PM_G2P_ASYNC
      cp_async_wait_all();  // this lane's copies of its particle (issued one chunk ahead)
#endif
      if (lane < n) {
        const uint32_t i = c0 + lane;
#if PM_PREFETCH
        const uint32_t o = o_cur;
#else
        const uint32_t o = B.sorted[i];
#endif
        float lat[7];
        AxisW aw[3];
#if PM_G2P_ASYNC
#pragma unroll
        for (int d = 0; d < 3; ++d) aw[d] = axis_weights(xs[d * 32 + lane], P.anchor[d], dx, P.inv_dx);
#else
#pragma unroll
        for (int d = 0; d < 3; ++d) aw[d] = axis_weights(B.pin[(F_X + d) * S + o], P.anchor[d], dx, P.inv_dx);
#endif
        cl = local_cell(aw, c, bx, by, bz);
#if PM_G2P_POLYW
        const float fpos[3] = {aw[0].r * P.inv_dx, aw[1].r * P.inv_dx, aw[2].r * P.inv_dx};
#endif
        const int lx = cl >> 4, ly = (cl >> 2) & 3, lz = cl & 3;
        // Ls: the velocity gradient's symmetric part, accumulated directly (xx, yy, zz and the
        // doubled off-diagonals xy, xz, yz): only |0.5 (L + L^T)|_F is used
        float vp[3] = {0.f, 0.f, 0.f}, fp[3] = {0.f, 0.f, 0.f}, Bp[9], Ls[6], gl[7], gs = 0.f;
#pragma unroll
        for (int k = 0; k < 9; ++k) Bp[k] = 0.f;
#pragma unroll
        for (int k = 0; k < 6; ++k) Ls[k] = 0.f;
#pragma unroll
        for (int k = 0; k < 7; ++k) gl[k] = 0.f;
#if PM_PACKED
        // latent and shear sums on pairs straight from the tile records: (lat1, lat2), (lat3, lat4),
        // (lat5, lat6) and (shear, node mass; the mass sum is not used)
        float2 g12 = make_float2(0.f, 0.f), g34 = g12, g56 = g12, gsm = g12;
#endif
#if PM_G2P_FACTORED
        // Sum factorisation: the weight of node (a, b, c) is Na Nb Nc, so every velocity sum is
        // formed along each row of three nodes (over c), then over the rows of a layer (b), then
        // over the layers (a): per row P = sum_c Nc v, Q = sum_c dNc v and Z = sum_c o_c Nc v (o the
        // node offset -1, 0, 1 from the stencil's middle node); per layer S = sum_b Nb P,
        // Sd = sum_b dNb P, SQ = sum_b Nb Q, Sz = sum_b Nb Z, Sy = sum_b o_b Nb P; finally
        // vp = sum_a Na S, the offset sums of B (sum_a o_a Na S, sum_a Na Sy, sum_a Na Sz) and the
        // velocity gradient's columns L[:, 0] = sum_a dNa S, L[:, 1] = sum_a Na Sd,
        // L[:, 2] = sum_a Na SQ.  Latent, shear and FLIP sums stay node by node.
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const float Na = aw[0].N[a], dNa = aw[0].dN[a];
          float Sv[3] = {0.f, 0.f, 0.f}, Sy[3] = {0.f, 0.f, 0.f}, Sz[3] = {0.f, 0.f, 0.f};
          float Sd[3] = {0.f, 0.f, 0.f}, SQ[3] = {0.f, 0.f, 0.f};
#pragma unroll
          for (int bb = 0; bb < 3; ++bb) {
            const float Nb = aw[1].N[bb], dNb = aw[1].dN[bb];
            const float nxy = Na * Nb;
            float Pv[3] = {0.f, 0.f, 0.f}, Qv[3] = {0.f, 0.f, 0.f}, Zv[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int cz = 0; cz < 3; ++cz) {
              const int tn = ((lx + a) * kTile + (ly + bb)) * kTile + (lz + cz);
              const float Nc = aw[2].N[cz], dNc = aw[2].dN[cz];
              const float4 R0 = tile[tn], R1 = tile[kG2PTileStride + tn], R2 = tile[2 * kG2PTileStride + tn];
              const float gv[3] = {R0.x, R0.y, R0.z};
#pragma unroll
              for (int r = 0; r < 3; ++r) {
                Pv[r] += Nc * gv[r];
                Qv[r] += dNc * gv[r];
                if (cz == 0) Zv[r] -= Nc * gv[r];
                if (cz == 2) Zv[r] += Nc * gv[r];
              }
              const float w = nxy * Nc;
#else
#pragma unroll kG2PUnrollX
        for (int a = 0; a < 3; ++a) {
          const float oa = (float)(a - 1);
#if PM_G2P_POLYW
          // weights formed where they are used, from the position in the base cell
          const float Na = bs_n(fpos[0], a), dNa = bs_dn(fpos[0], a, P.inv_dx);
#define PM_NB(k) bs_n(fpos[1], k)
#define PM_DNB(k) bs_dn(fpos[1], k, P.inv_dx)
#define PM_NC(k) bs_n(fpos[2], k)
#define PM_DNC(k) bs_dn(fpos[2], k, P.inv_dx)
#else
          const float Na = a == 0 ? aw[0].N[0] : (a == 1 ? aw[0].N[1] : aw[0].N[2]);
          const float dNa = a == 0 ? aw[0].dN[0] : (a == 1 ? aw[0].dN[1] : aw[0].dN[2]);
#define PM_NB(k) aw[1].N[k]
#define PM_DNB(k) aw[1].dN[k]
#define PM_NC(k) aw[2].N[k]
#define PM_DNC(k) aw[2].dN[k]
#endif
#pragma unroll
          for (int bb = 0; bb < 3; ++bb) {
            const float nxy = Na * PM_NB(bb);
            const float dnxy = dNa * PM_NB(bb), ndxy = Na * PM_DNB(bb);
#pragma unroll
            for (int cz = 0; cz < 3; ++cz) {
              const int tn = ((lx + a) * kTile + (ly + bb)) * kTile + (lz + cz);
              const float w = nxy * PM_NC(cz);
              const float g0 = dnxy * PM_NC(cz), g1 = ndxy * PM_NC(cz), g2 = nxy * PM_DNC(cz);
              const float4 R0 = tile[tn], R1 = tile[kG2PTileStride + tn], R2 = tile[2 * kG2PTileStride + tn];
              const float gv[3] = {R0.x, R0.y, R0.z};
#pragma unroll
              for (int r = 0; r < 3; ++r) {
                const float wv = gv[r] * w;
                vp[r] += wv;
                Bp[3 * r + 0] += wv * oa;
                if (bb != 1) Bp[3 * r + 1] += bb == 0 ? -wv : wv;
                if (cz != 1) Bp[3 * r + 2] += cz == 0 ? -wv : wv;
              }
              Ls[0] += gv[0] * g0;
              Ls[1] += gv[1] * g1;
              Ls[2] += gv[2] * g2;
              Ls[3] += gv[0] * g1 + gv[1] * g0;
              Ls[4] += gv[0] * g2 + gv[2] * g0;
              Ls[5] += gv[1] * g2 + gv[2] * g1;
#undef PM_NB
#undef PM_DNB
#undef PM_NC
#undef PM_DNC
#endif
              gl[0] += R0.w * w;
#if !PM_G2P_TWOPASS
              if (use_flip) {
                const float4 R3 = tile[3 * kG2PTileStride + tn];
                fp[0] += R3.x * w; fp[1] += R3.y * w; fp[2] += R3.z * w;
              }
#if PM_PACKED
              const float2 w2 = dup2(w);
              g12 = fma2(w2, lo2(R1), g12);
              g34 = fma2(w2, hi2(R1), g34);
              g56 = fma2(w2, lo2(R2), g56);
              gsm = fma2(w2, hi2(R2), gsm);
#else
              gl[1] += R1.x * w; gl[2] += R1.y * w; gl[3] += R1.z * w; gl[4] += R1.w * w;
              gl[5] += R2.x * w; gl[6] += R2.y * w;
              gs += R2.z * w;
#endif
#endif
            }
#if PM_G2P_FACTORED
#pragma unroll
            for (int r = 0; r < 3; ++r) {
              Sv[r] += Nb * Pv[r];
              Sd[r] += dNb * Pv[r];
              SQ[r] += Nb * Qv[r];
              Sz[r] += Nb * Zv[r];
              if (bb == 0) Sy[r] -= Nb * Pv[r];
              if (bb == 2) Sy[r] += Nb * Pv[r];
            }
#endif
          }
#if PM_G2P_FACTORED
#pragma unroll
          for (int r = 0; r < 3; ++r) {
            vp[r] += Na * Sv[r];
            if (a == 0) Bp[3 * r] -= Na * Sv[r];
            if (a == 2) Bp[3 * r] += Na * Sv[r];
            Bp[3 * r + 1] += Na * Sy[r];
            Bp[3 * r + 2] += Na * Sz[r];
          }
          // L[r][k] = sum v_r d_k w: column 0 sum_a dNa S, column 1 sum_a Na Sd, column 2 sum_a Na SQ
          Ls[0] += dNa * Sv[0];
          Ls[1] += Na * Sd[1];
          Ls[2] += Na * SQ[2];
          Ls[3] += dNa * Sv[1] + Na * Sd[0];
          Ls[4] += dNa * Sv[2] + Na * SQ[0];
          Ls[5] += Na * (Sd[2] + SQ[1]);
#endif
        }
#if PM_G2P_TWOPASS
        // second pass over the stencil: latent, shear and the FLIP velocity change, so that these
        // sums are not live together with the velocity, APIC and gradient sums of the first
#pragma unroll kG2PUnrollX
        for (int a = 0; a < 3; ++a) {
#if PM_G2P_POLYW
          const float Na = bs_n(fpos[0], a);
#else
          const float Na = a == 0 ? aw[0].N[0] : (a == 1 ? aw[0].N[1] : aw[0].N[2]);
#endif
#pragma unroll
          for (int bb = 0; bb < 3; ++bb) {
#if PM_G2P_POLYW
            const float nxy = Na * bs_n(fpos[1], bb);
#else
            const float nxy = Na * aw[1].N[bb];
#endif
#pragma unroll
            for (int cz = 0; cz < 3; ++cz) {
              const int tn = ((lx + a) * kTile + (ly + bb)) * kTile + (lz + cz);
#if PM_G2P_POLYW
              const float w = nxy * bs_n(fpos[2], cz);
#else
              const float w = nxy * aw[2].N[cz];
#endif
              const float4 R1 = tile[kG2PTileStride + tn], R2 = tile[2 * kG2PTileStride + tn];
              if (use_flip) {
                const float4 R3 = tile[3 * kG2PTileStride + tn];
                fp[0] += R3.x * w; fp[1] += R3.y * w; fp[2] += R3.z * w;
              }
#if PM_PACKED
              const float2 w2 = dup2(w);
              g12 = fma2(w2, lo2(R1), g12);
              g34 = fma2(w2, hi2(R1), g34);
              g56 = fma2(w2, lo2(R2), g56);
              gsm = fma2(w2, hi2(R2), gsm);
#else
              gl[1] += R1.x * w; gl[2] += R1.y * w; gl[3] += R1.z * w; gl[4] += R1.w * w;
              gl[5] += R2.x * w; gl[6] += R2.y * w;
              gs += R2.z * w;
#endif
            }
          }
        }
#endif
#if PM_PACKED
        gl[1] = g12.x; gl[2] = g12.y; gl[3] = g34.x; gl[4] = g34.y; gl[5] = g56.x; gl[6] = g56.y;
        gs = gsm.x;
#endif
        // B = sum w v (x_i - x_p)^T, accumulated above with the node offsets o in {-1, 0, 1} from
        // the stencil's middle node (x_i - x_p = o dx - (r - dx)): B = dx sum w v o^T - (sum w v)
        // (r - dx)^T.  Centring keeps both terms within half a cell (r - dx is exact), so their
        // difference loses no more than the direct sum would.
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int k = 0; k < 3; ++k) Bp[3 * r + k] = dx * Bp[3 * r + k] - vp[r] * (aw[k].r - dx);
        if (!apic) for (int k = 0; k < 9; ++k) Bp[k] = 0.f;
        // particle state read after the gather (not live across it)
#if PM_G2P_ASYNC
#pragma unroll
        for (int k = 0; k < 7; ++k) lat[k] = xs[(3 + k) * 32 + lane];
#else
#pragma unroll
        for (int k = 0; k < 7; ++k) lat[k] = B.pin[(F_LAT + k) * S + o];
#endif
        float vold[3] = {0.f, 0.f, 0.f};
        if (kFlip || !musl) {
#pragma unroll
          for (int d = 0; d < 3; ++d) vold[d] = B.pin[(F_V + d) * S + o];
        }
        // diffusion factor |0.5 (L + L^T)|_F (g2p.cpp:98-101)
        const float s2 = Ls[0] * Ls[0] + Ls[1] * Ls[1] + Ls[2] * Ls[2] +
                         0.5f * (Ls[3] * Ls[3] + Ls[4] * Ls[4] + Ls[5] * Ls[5]);
        const float diff = sqrtf(s2);
        // mixing (g2p.cpp:105-130)
        const float mixf = smooth_step(P.D_edge0, P.D_edge1, gs);
        const float smix = fminf(fmaxf(dyn * mixf * dtf, 0.f), 1.f);
#pragma unroll
        for (int k = 0; k < 7; ++k) lat[k] = (1.f - smix) * lat[k] + smix * gl[k];
        const float psum = lat[0] + lat[1] + lat[2] + lat[3];
        if (psum > 1e-6f) { for (int k = 0; k < 4; ++k) lat[k] /= psum; }
        // MUSL velocity update (musl.cpp:13-26)
        float vnew[3];
        if (musl) {
          for (int r = 0; r < 3; ++r) {
            if (fr < -1.f) vnew[r] = vp[r];
            else if (fr < 0.f) vnew[r] = (-fr) * (vold[r] + fp[r]) + (1.f - (-fr)) * vp[r];
            else vnew[r] = fr * (vold[r] + fp[r]) + (1.f - fr) * vp[r];
          }
        } else {
          for (int r = 0; r < 3; ++r) vnew[r] = vold[r];
          for (int r = 0; r < 3; ++r) B.pic[(3 + r) * S + i] = fp[r];
        }
        float* po = B.pout;
#pragma unroll
        for (int r = 0; r < 3; ++r) { po[(F_V + r) * S + i] = vnew[r]; B.pic[r * S + i] = vp[r]; }
#pragma unroll
        for (int k = 0; k < 9; ++k) po[(F_B + k) * S + i] = Bp[k];
#pragma unroll
        for (int k = 0; k < 7; ++k) po[(F_LAT + k) * S + i] = lat[k];
        po[F_DIFF * S + i] = diff;
        if (musl) {
          const float r3[3] = {aw[0].r, aw[1].r, aw[2].r};
          float q[3], C[9];
#pragma unroll
          for (int qq = 0; qq < 3; ++qq)
            q[qq] = vnew[qq] - D * (Bp[3 * qq] * r3[0] + Bp[3 * qq + 1] * r3[1] + Bp[3 * qq + 2] * r3[2]);
#pragma unroll
          for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int qq = 0; qq < 3; ++qq) C[3 * k + qq] = D * dx * Bp[3 * qq + k];
#if PM_PACKED
          // packed layout: pairs (fx, fy), (q0, q1), (C0x, C0y), (C1x, C1y), (C2x, C2y)
          st[0 * 32 + lane] = make_float4(r3[0] * P.inv_dx, r3[1] * P.inv_dx, r3[2] * P.inv_dx, q[2]);
          st[1 * 32 + lane] = make_float4(q[0], q[1], C[2], C[5]);
          st[2 * 32 + lane] = make_float4(C[0], C[1], C[3], C[4]);
          st[3 * 32 + lane] = make_float4(C[6], C[7], C[8], 0.f);
#else
          st[0 * 32 + lane] = make_float4(q[0], q[1], q[2], r3[0] * P.inv_dx);
          st[1 * 32 + lane] = make_float4(C[0], C[1], C[2], C[3]);
          st[2 * 32 + lane] = make_float4(C[4], C[5], C[6], C[7]);
          st[3 * 32 + lane] = make_float4(C[8], r3[1] * P.inv_dx, r3[2] * P.inv_dx, 0.f);
#endif
        }
      }
#if PM_G2P_ASYNC
      // the next chunk's position and latent into this lane's slots (read above), while this chunk
      // scatters
      if (c1 + lane < pe) {
#pragma unroll
        for (int f = 0; f < 3; ++f) cp_async4(xs + f * 32 + lane, B.pin + (size_t)(F_X + f) * S + o_next);
#pragma unroll
        for (int f = 0; f < 7; ++f) cp_async4(xs + (3 + f) * 32 + lane, B.pin + (size_t)(F_LAT + f) * S + o_next);
      }
      cp_async_commit();
      if ((kFlip || !musl) && c1 + lane < pe) {
        const float* q = B.pin + o_next;
#pragma unroll
        for (int f = F_V; f < F_V + 3; ++f) prefetch_l2(q + (size_t)f * S);
      }
#elif PM_PREFETCH
      if (c1 + lane < pe) {  // the next chunk's position and latent, while this chunk scatters
        const float* q = B.pin + o_next;
#pragma unroll
        for (int f = F_X; f < F_X + 3; ++f) prefetch_l2(q + (size_t)f * S);
#pragma unroll
        for (int f = F_LAT; f < F_LAT + 7; ++f) prefetch_l2(q + (size_t)f * S);
        if (kFlip || !musl) {
#pragma unroll
          for (int f = F_V; f < F_V + 3; ++f) prefetch_l2(q + (size_t)f * S);
        }
      }
#endif
      if (musl) {
        const int prev = __shfl_up_sync(0xffffffffu, cl, 1);
        uint32_t heads = __ballot_sync(0xffffffffu, lane < n && (lane == 0 || cl != prev));
        __syncwarp();
        while (heads) {
          const int s0 = __ffs(heads) - 1;
          heads &= heads - 1;
          const int s1 = heads ? __ffs(heads) - 1 : n;
          const int cell = __shfl_sync(0xffffffffu, cl, s0);
          if (lane < 27) {
            // the lane's stencil node constants, formed here so that they are not live across the
            // gather above
            const float fa = (float)la, fb = (float)lb, fcc = (float)lc;
            const StencilPoly px(la, P.inv_dx), py(lb, P.inv_dx), pz(lc, P.inv_dx);
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#if PM_PACKED
            const StencilPoly2 pxy(px, py);
            const float2 fa2 = dup2(fa), fb2 = dup2(fb), fc2 = dup2(fcc);
            // weights as in P2G (the skip of weights <= 1e-25, musl.cpp:188, only skips zeros)
            float2 a_v = make_float2(0.f, 0.f);
#pragma unroll kScatterUnroll
            for (int q = s0; q < s1; ++q) {
              const float4 S0 = st[0 * 32 + q], S1 = st[1 * 32 + q], S2 = st[2 * 32 + q], S3 = st[3 * 32 + q];
              const float2 nxy = pxy.N(lo2(S0));
              const float w = nxy.x * (nxy.y * pz.N(S0.z));
              float2 vxy = fma2(fa2, lo2(S2), lo2(S1));
              vxy = fma2(fb2, hi2(S2), vxy);
              vxy = fma2(fc2, lo2(S3), vxy);
              a_v = fma2(dup2(w), vxy, a_v);
              acc[2] += w * (S0.w + fa * S1.z + fb * S1.w + fcc * S3.z);
              acc[3] += w;
            }
            acc[0] = a_v.x;
            acc[1] = a_v.y;
#else
#pragma unroll kScatterUnroll
            for (int q = s0; q < s1; ++q) {
              const float4 Q = st[0 * 32 + q], C0 = st[1 * 32 + q], C1 = st[2 * 32 + q], C2 = st[3 * 32 + q];
              const float w = px.N(Q.w) * (py.N(C2.y) * pz.N(C2.z));
              const float wm = w > 1e-25f ? w : 0.f;  // musl.cpp:188
              acc[0] += wm * (Q.x + fa * C0.x + fb * C0.w + fcc * C1.z);
              acc[1] += wm * (Q.y + fa * C0.y + fb * C1.x + fcc * C1.w);
              acc[2] += wm * (Q.z + fa * C0.z + fb * C1.y + fcc * C2.x);
              acc[3] += wm;
            }
#endif
            const int tp = ((cell >> 4) + la) * kSX + (((cell >> 2) & 3) + lb) * kSY + ((cell & 3) + lc);
#pragma unroll
            for (int k = 0; k < 4; ++k) atomicAdd(&mtile[k * kTileStride + tp], acc[k]);
          }
        }
        __syncwarp();
      }
    }
    __syncthreads();
    if (musl) {
      for (int tn = threadIdx.x; tn < kTileNodes; tn += kThreads) {
        const float* t = mtile + tile_pad(tn);
        const float w = t[3 * kTileStride];
        if (w == 0.f) continue;
        const int node = tile_to_node(tn, bx, by, bz, c);
        if (node < 0) continue;
        red_add_v4(B.gmusl + node, t[0], t[kTileStride], t[2 * kTileStride], w);
      }
    }
    __syncthreads();
  }
}
template <bool kFlip>
__global__ void __launch_bounds__(kThreads, PM_G2P_MINB) k_g2p_musl(Params P, Bufs B) {
  pdl_enter();
  d_g2p_musl<kFlip>(P, B, blockIdx.x, gridDim.x);
}
template <bool kFlip>
__global__ void __launch_bounds__(kThreads, PM_G2P_MINB) kb_g2p_musl(const SceneDev* __restrict__ sd,
                                                                     const int* __restrict__ off, int ns) {
  int s_, blk_, nblk_;
  batch_slot(off, ns, s_, blk_, nblk_);
  __shared__ SceneShared ss_;
  load_scene_shared(sd[s_], ss_);
  d_g2p_musl<kFlip>(ss_.P, ss_.B, blk_, nblk_);
}


// ------------------------------------------------------------------------------------------
// FP64 3x3 SVD (warm-started one-sided Jacobi) -- sigma >= 0, U, V orthogonal
// ------------------------------------------------------------------------------------------

// FP32 cyclic Jacobi rotation of a symmetric 3x3 on pair (p, q); arp, arq are the entries of the
// third row against p and q; V accumulates the rotations.
__device__ __forceinline__ void jrot_f32(float& app, float& aqq, float& apq, float& arp, float& arq, float* V, int p,
                                         int q) {
  if (fabsf(apq) <= 1e-30f || fabsf(apq) <= 1e-9f * (fabsf(app) + fabsf(aqq))) return;
  const float zeta = (aqq - app) / (2.f * apq);
  const float t = copysignf(1.f, zeta) / (fabsf(zeta) + sqrtf(1.f + zeta * zeta));
  const float cs = rsqrtf(1.f + t * t);
  const float sn = t * cs;
  app -= t * apq;
  aqq += t * apq;
  apq = 0.f;
  const float rp = arp, rq = arq;
  arp = cs * rp - sn * rq;
  arq = sn * rp + cs * rq;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float vp = V[3 * k + p], vq = V[3 * k + q];
    V[3 * k + p] = cs * vp - sn * vq;
    V[3 * k + q] = sn * vp + cs * vq;
  }
}

// SVD of a 3x3 with an FP32 warm start: cyclic Jacobi in FP32 on the trace-shifted A^T A gives
// approximate right singular vectors; they are re-orthonormalised in FP64 and one-sided Jacobi
// (Hestenes) sweeps in FP64 run on W = A V until no column pair needs a rotation, so the singular
// values have FP64 accuracy and U, V are orthogonal to FP64 rounding before they are rounded to
// the FP32 factors the rest of the step uses.  Near convergence a rotation angle only has to be
// accurate to first order: (cos, sin) are computed in FP32 from the FP64 column products and
// renormalised in FP64 by one Newton step on cos^2 + sin^2 = 1 (error O(1e-14)), which replaces
// the FP64 divide, square root and reciprocal square root of each rotation.
// At most this many FP32 warm-start sweeps (the FP64 sweeps that follow converge regardless of
// the start; on the 2M scene the tail measured 0.181 ms with 2, 0.187 with 3, 0.194 with 1 or 5).
#ifndef PM_SVD_WARM_SWEEPS
#define PM_SVD_WARM_SWEEPS 2
#endif
__device__ void svd3_warm(const double A[9], float Uf[9], double s[3], float Vf_out[9]) {
  double S[6];
  S[0] = A[0] * A[0] + A[3] * A[3] + A[6] * A[6];
  S[1] = A[1] * A[1] + A[4] * A[4] + A[7] * A[7];
  S[2] = A[2] * A[2] + A[5] * A[5] + A[8] * A[8];
  S[3] = A[0] * A[1] + A[3] * A[4] + A[6] * A[7];
  S[4] = A[0] * A[2] + A[3] * A[5] + A[6] * A[8];
  S[5] = A[1] * A[2] + A[4] * A[5] + A[7] * A[8];
  const double m = (S[0] + S[1] + S[2]) / 3.0;
  float a00 = (float)(S[0] - m), a11 = (float)(S[1] - m), a22 = (float)(S[2] - m);
  float a01 = (float)S[3], a02 = (float)S[4], a12 = (float)S[5];
  float Vf[9] = {1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f};
#pragma unroll 1
  for (int sweep = 0; sweep < PM_SVD_WARM_SWEEPS; ++sweep) {
    jrot_f32(a00, a11, a01, a02, a12, Vf, 0, 1);  // pair (0,1), third index 2
    jrot_f32(a00, a22, a02, a01, a12, Vf, 0, 2);  // pair (0,2), third index 1
    jrot_f32(a11, a22, a12, a01, a02, Vf, 1, 2);  // pair (1,2), third index 0
    const float off = fabsf(a01) + fabsf(a02) + fabsf(a12);
    if (off <= 1e-7f * (fabsf(a00) + fabsf(a11) + fabsf(a22)) + 1e-30f) break;
  }
  // FP64 Gram-Schmidt of the FP32 rotation -> orthonormal V0 (det +1)
  double V[9];
  {
    double v0[3] = {Vf[0], Vf[3], Vf[6]}, v1[3] = {Vf[1], Vf[4], Vf[7]};
    const double n0 = rsqrt(v0[0] * v0[0] + v0[1] * v0[1] + v0[2] * v0[2]);
    for (int k = 0; k < 3; ++k) v0[k] *= n0;
    const double d01 = v0[0] * v1[0] + v0[1] * v1[1] + v0[2] * v1[2];
    for (int k = 0; k < 3; ++k) v1[k] -= d01 * v0[k];
    const double n1 = rsqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]);
    for (int k = 0; k < 3; ++k) v1[k] *= n1;
    const double v2[3] = {v0[1] * v1[2] - v0[2] * v1[1], v0[2] * v1[0] - v0[0] * v1[2], v0[0] * v1[1] - v0[1] * v1[0]};
    for (int k = 0; k < 3; ++k) { V[3 * k] = v0[k]; V[3 * k + 1] = v1[k]; V[3 * k + 2] = v2[k]; }
  }
  double W[9];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int q = 0; q < 3; ++q) W[3 * r + q] = A[3 * r] * V[q] + A[3 * r + 1] * V[3 + q] + A[3 * r + 2] * V[6 + q];
  const double eps2 = 2.220446049250313e-16 * 2.220446049250313e-16;
#pragma unroll 1
  for (int sweep = 0; sweep < 8; ++sweep) {
    bool rotated = false;
#pragma unroll
    for (int pq = 0; pq < 3; ++pq) {
      const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
      const double alpha = W[p] * W[p] + W[3 + p] * W[3 + p] + W[6 + p] * W[6 + p];
      const double beta = W[q] * W[q] + W[3 + q] * W[3 + q] + W[6 + q] * W[6 + q];
      const double gamma = W[p] * W[q] + W[3 + p] * W[3 + q] + W[6 + p] * W[6 + q];
      if (gamma == 0.0 || gamma * gamma <= eps2 * alpha * beta) continue;
      rotated = true;
      const float zeta = (float)(beta - alpha) / (2.f * (float)gamma);
      const float t = copysignf(1.f, zeta) / (fabsf(zeta) + sqrtf(fmaf(zeta, zeta, 1.f)));
      const float csf = rsqrtf(fmaf(t, t, 1.f));
      double cs = csf, sn = (double)(csf * t);
      const double f = 1.5 - 0.5 * (cs * cs + sn * sn);
      cs *= f;
      sn *= f;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double wp = W[3 * k + p], wq = W[3 * k + q];
        W[3 * k + p] = cs * wp - sn * wq;
        W[3 * k + q] = sn * wp + cs * wq;
        const double vp = V[3 * k + p], vq = V[3 * k + q];
        V[3 * k + p] = cs * vp - sn * vq;
        V[3 * k + q] = sn * vp + cs * vq;
      }
    }
    if (!rotated) break;
  }
  // singular values in FP64; U = W diag(1/s) and V rounded to FP32 (fixed indices throughout, so
  // the factors stay in registers).  A column whose singular value is below 1e-6 of the largest
  // carries no reliable direction in W / s; those columns are completed from the others instead
  // (cross product, so that det U = det V = +1), which keeps U orthogonal for (near-)singular A.
#pragma unroll
  for (int j = 0; j < 3; ++j) s[j] = sqrt(W[j] * W[j] + W[3 + j] * W[3 + j] + W[6 + j] * W[6 + j]);
  const double smax = fmax(s[0], fmax(s[1], s[2]));
  bool ok[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    ok[j] = s[j] > 1e-6 * smax && s[j] > 1e-300;
    const float inv = ok[j] ? (float)(1.0 / s[j]) : 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) Uf[3 * k + j] = (float)W[3 * k + j] * inv;
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) Vf_out[k] = (float)V[k];
  const int bad = (!ok[0]) + (!ok[1]) + (!ok[2]);
  auto cross_col = [&](int z, int a, int b) {  // column z = column a x column b
    Uf[0 + z] = Uf[3 + a] * Uf[6 + b] - Uf[6 + a] * Uf[3 + b];
    Uf[3 + z] = Uf[6 + a] * Uf[0 + b] - Uf[0 + a] * Uf[6 + b];
    Uf[6 + z] = Uf[0 + a] * Uf[3 + b] - Uf[3 + a] * Uf[0 + b];
  };
  // column z = the unit vector orthogonal to column g built from the basis axis least aligned with it
  auto perp_col = [&](int z, int g) {
    const float gx = Uf[g], gy = Uf[3 + g], gz = Uf[6 + g];
    float e[3] = {0.f, 0.f, 0.f};
    if (fabsf(gx) <= fabsf(gy) && fabsf(gx) <= fabsf(gz)) e[0] = 1.f;
    else if (fabsf(gy) <= fabsf(gz)) e[1] = 1.f;
    else e[2] = 1.f;
    const float d = e[0] * gx + e[1] * gy + e[2] * gz;
    float p[3] = {e[0] - d * gx, e[1] - d * gy, e[2] - d * gz};
    const float nrm = rsqrtf(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    Uf[z] = p[0] * nrm;
    Uf[3 + z] = p[1] * nrm;
    Uf[6 + z] = p[2] * nrm;
  };
  if (bad == 1) {
    if (!ok[0]) cross_col(0, 1, 2);
    else if (!ok[1]) cross_col(1, 2, 0);
    else cross_col(2, 0, 1);
  } else if (bad == 2) {
    if (ok[0]) { perp_col(1, 0); cross_col(2, 0, 1); }
    else if (ok[1]) { perp_col(2, 1); cross_col(0, 1, 2); }
    else { perp_col(0, 2); cross_col(1, 2, 0); }
  } else if (bad == 3) {
#pragma unroll
    for (int k = 0; k < 9; ++k) Uf[k] = (k % 4 == 0) ? 1.f : 0.f;
  }
}

// ------------------------------------------------------------------------------------------
// deformation update + return map + position update + stress cache + reductions
// ------------------------------------------------------------------------------------------
struct ReturnMapOut {
  float h[3];        // final principal log strains
  bool changed;      // F replaced by U exp(h) V^T
  bool to_rotation;  // capped VM branch: F = U V^T
  bool queued;       // surrogate mode: the consistency solve is left to the surrogate pass
};

// Perzyna consistency solve (plasticity.cpp:194-229 VMVisc, :292-325 DPVisc): Newton on
// r(dg) = (q_trial - f dg) (dt / (eta dg + dt))^m - q_yield(dg) from dg until |r| < 1e-2, at most
// 60 iterations.  iters counts the Newton updates taken.
__device__ double perzyna_newton(const Params& P, bool vm, double q_trial, double q_yield_dp, double epd, double dt,
                                 double dg, uint32_t& iters, uint32_t& err) {
  const double fmu = P.f_mu_prefac, dpre = P.d_prefac;
  for (int it = 0; it < 60; ++it) {
    if (it == 59) err |= E_NEWTON_NOCONV;
    const double tm = P.perzyna_visc * dg + dt;
    const double tmp = dt / tm;
    const double tmp1 = exp(P.perzyna_exp * log(tmp));  // tmp^m; tmp^(m-1) = tmp1 / tmp
    const double tmpm1 = tmp1 / tmp;
    const double q_yield = vm ? P.q_min + (P.q_max - P.q_min) * exp(-P.xi * (epd + dg / dpre)) : q_yield_dp;
    const double res = (q_trial - fmu * dg) * tmp1 - q_yield;
    if (fabs(res) < 1e-2) break;
    const double qyd = vm ? -P.xi / dpre * (P.q_max - P.q_min) * exp(-P.xi * (epd + dg / dpre)) : 0.0;
    const double rd = -fmu * tmp1 + (q_trial - fmu * dg) * P.perzyna_exp * tmpm1 * (-P.perzyna_visc * dt) / (tm * tm) - qyd;
    if (fabs(rd) < 1e-14) err |= E_NEWTON_FLAT;
    dg -= res / rd;
    if (dg < 0) dg = 1e-10;
    ++iters;
  }
  return dg;
}

// The same Perzyna Newton for VMVisc in FP32 (plasticity.cpp:194-229).  The stop test is
// |r| < max(1e-2, 1e-6 q_trial): the reference's 1e-2 Pa unless q_trial exceeds 1e4 Pa, where
// FP32 rounding of q would otherwise keep |r| above 1e-2.
__device__ float perzyna_newton_vm32(const Params& P, float q_trial, float epd, float dt, float dg, uint32_t& iters,
                                     uint32_t& err) {
  const float fmu = (float)P.f_mu_prefac, dpre = (float)P.d_prefac, visc = (float)P.perzyna_visc;
  const float m = (float)P.perzyna_exp, qmin = (float)P.q_min, dq = (float)(P.q_max - P.q_min), xi = (float)P.xi;
  const float tol = fmaxf(1e-2f, 1e-6f * q_trial);
  for (int it = 0; it < 60; ++it) {
    if (it == 59) err |= E_NEWTON_NOCONV;
    const float tm = visc * dg + dt;
    const float tmp = dt / tm;
    const float tmp1 = exp2f(m * log2f(tmp));  // tmp^m; tmp^(m-1) = tmp1 / tmp
    const float tmpm1 = tmp1 / tmp;
    const float soft = xi != 0.f ? expf(-xi * (epd + dg / dpre)) : 1.f;
    const float res = (q_trial - fmu * dg) * tmp1 - (qmin + dq * soft);
    if (fabsf(res) < tol) break;
    const float qyd = -xi / dpre * dq * soft;
    const float rd = -fmu * tmp1 + (q_trial - fmu * dg) * m * tmpm1 * (-visc * dt) / (tm * tm) - qyd;
    if (fabsf(rd) < 1e-14f) err |= E_NEWTON_FLAT;
    dg -= res / rd;
    if (dg < 0.f) dg = 1e-10f;
    ++iters;
  }
  return dg;
}

// Surrogate features of a particle on the Newton path: trial log strains, deviatoric strain
// rate, yield, viscosity, flow index, Young's modulus.
__device__ __forceinline__ void sur_features(const Params& P, const float h[3], float dt, float q_yield, float f[10]) {
  const float m = (h[0] + h[1] + h[2]) / 3.f;
  for (int k = 0; k < 3; ++k) { f[k] = h[k]; f[3 + k] = (h[k] - m) / dt; }
  f[6] = q_yield;
  f[7] = (float)P.perzyna_visc;
  f[8] = (float)P.perzyna_exp;
  f[9] = (float)P.E;
}

// The Newton path of the return map: either queue the particle for the surrogate, or solve
// (VMVisc in FP32, DPVisc in FP64) and, when the sample log is on, record features and the
// projected strains.
// kExtras = false compiles out the surrogate queue and the sample log (plain-solver kernels).
template <bool kExtras>
__device__ bool newton_path(const Params& P, const Bufs& B, uint32_t i, bool vm, double dt, const float h[3],
                            const float hd[3], double q_trial, double q_yield, float epd, const float* U,
                            const float* V, double& dg, uint32_t& iters, uint32_t& err) {
  if (kExtras && P.return_map == 1 && P.q_cap > 0) {
    const uint32_t slot = atomicAdd(&B.ctrl->q_n, 1u);
    if (slot < P.q_cap) {
      SurQ& r = B.q[slot];
      for (int k = 0; k < 9; ++k) { r.U[k] = U[k]; r.V[k] = V[k]; }
      for (int k = 0; k < 3; ++k) { r.h[k] = h[k]; r.hd[k] = hd[k]; }
      r.q_trial = (float)q_trial;
      r.q_y = (float)q_yield;
      r.epd = epd;
      r.i = i;
      r.vm = vm ? 1u : 0u;
      float f[10];
      sur_features(P, h, (float)dt, (float)q_yield, f);
      for (int k = 0; k < 10; ++k) B.qx[(size_t)slot * 10 + k] = f[k];
      return true;
    }
    err |= E_CAPACITY;  // queue full: solve here
  }
  const double guess = 0.01 * (q_trial - q_yield) / P.f_mu_prefac;
  if (vm) dg = perzyna_newton_vm32(P, (float)q_trial, epd, (float)dt, (float)guess, iters, err);
  else dg = perzyna_newton(P, false, q_trial, q_yield, (double)epd, dt, guess, iters, err);
  if (kExtras && P.log_cap > 0 &&
      (P.log_every <= 1 || ((i ^ (B.ctrl->step * 0x9E3779B9u)) * 0x85EBCA6Bu >> 8) % P.log_every == 0)) {
    const uint32_t slot = atomicAdd(&B.ctrl->slog_n, 1u);
    if (slot < P.log_cap) {
      float* o = B.slog + (size_t)slot * 16;
      sur_features(P, h, (float)dt, (float)q_yield, o);
      for (int k = 0; k < 3; ++k) {
        const double d = (dg / P.d_prefac) * hd[k];  // h - h_projected
        o[10 + k] = (float)d;
        o[13 + k] = (float)(d / dt);
      }
    }
  }
  return false;
}

// plasticity.cpp:163-238 (VMVisc, FP32) and :240-340 (DPVisc, FP64: the cone and its apex).
// sg: singular values of the trial elastic F (FP64 SVD); U, V its factors rounded to FP32.
// kModel: the plastic model compiled in (PL_VMVISC, PL_DPVISC), or -1 to branch on P.plastic_model.
template <int kModel, bool kExtras>
__device__ void return_map(const Params& P, const Bufs& B, uint32_t i, double dt, const double sg[3], const float* U,
                           const float* V, float& epd, float& epv, float& epp, float& dgam, uint32_t& plastic,
                           uint32_t& iters, uint32_t& solves, uint32_t& err, ReturnMapOut& out) {
  out.changed = false;
  out.to_rotation = false;
  out.queued = false;
  const int model = kModel >= 0 ? kModel : P.plastic_model;
  if (model == PL_VMVISC) {
    float h[3];
    for (int k = 0; k < 3; ++k) h[k] = logf(fmaxf(fabsf((float)sg[k]), 1e-4f));
    const float htr = h[0] + h[1] + h[2];
    float hd[3] = {h[0] - htr / 3.f, h[1] - htr / 3.f, h[2] - htr / 3.f};
    const float hdn = sqrtf(hd[0] * hd[0] + hd[1] * hd[1] + hd[2] * hd[2]);
    if (hdn > 0.f) for (int k = 0; k < 3; ++k) hd[k] /= hdn;
    for (int k = 0; k < 3; ++k) out.h[k] = h[k];
    const float fmu = (float)P.f_mu_prefac, emu = (float)P.e_mu_prefac, dpre = (float)P.d_prefac, K = (float)P.K;
    const float xi = (float)P.xi;
    const float q_trial = emu * hdn;
    const float q_yield = (float)P.q_min + (float)(P.q_max - P.q_min) * expf(-xi * epd);
    const float p_trial = -K * htr;
    const float dtf = (float)dt;
    if (p_trial < (float)P.p_min * expf(-xi * epv)) {
      const float dg = q_trial / fmu;
      out.to_rotation = true;
      out.changed = true;
      epv += -p_trial / K;
      epd += dg / dpre;
      dgam = dg / dtf;
    } else if (q_trial > q_yield) {
      ++plastic;
      float dg = 0.f;
      if (P.perzyna_exp == 1.0 && P.xi == 0.0) {
        dg = (q_trial - q_yield) / (fmu + q_yield * (float)P.perzyna_visc / dtf);
        if (dg < 0.f) err |= E_NEG_DGAMMA;
      } else {
        ++solves;
        double dgd = 0.0;
        if (newton_path<kExtras>(P, B, i, true, dt, h, hd, q_trial, q_yield, epd, U, V, dgd, iters, err)) {
          out.queued = true;
          return;
        }
        dg = (float)dgd;
      }
      for (int k = 0; k < 3; ++k) out.h[k] = h[k] - (dg / dpre) * hd[k];
      out.changed = true;
      epd += dg / dpre;
      dgam = dg / dtf;
    }
  } else if (model == PL_DPVISC) {
    double h[3];
    for (int k = 0; k < 3; ++k) h[k] = log(fmax(fabs(sg[k]), 1e-4));
    const double htr = h[0] + h[1] + h[2];
    double hd[3] = {h[0] - htr / 3.0, h[1] - htr / 3.0, h[2] - htr / 3.0};
    const double hdn = sqrt(hd[0] * hd[0] + hd[1] * hd[1] + hd[2] * hd[2]);
    if (hdn > 0) for (int k = 0; k < 3; ++k) hd[k] /= hdn;
    for (int k = 0; k < 3; ++k) out.h[k] = (float)h[k];
    const double fmu = P.f_mu_prefac, emu = P.e_mu_prefac, dpre = P.d_prefac;
    const double p_trial = -P.K * htr;
    const double q_trial = emu * hdn;
    const double p_tip = -P.q_cohesion / P.M;
    const double p_shift = P.use_pradhana ? -P.K * (double)epp : 0.0;
    const double q_yield = P.M * (p_trial + p_shift) + P.q_cohesion;
    if ((p_trial + p_shift) < p_tip) {
      const double dg = dpre * hdn;
      const double epv_inst = (p_tip - p_trial) / P.K;
      ++plastic;
      const double hh = -p_tip / (P.K * 3.0);
      for (int k = 0; k < 3; ++k) out.h[k] = (float)hh;
      out.changed = true;
      dgam = (float)(dg / dt);
      epd = (float)((double)epd + dg / dpre);
      epv = (float)((double)epv + epv_inst);
      if (P.use_pradhana) epp = (float)((double)epp + epv_inst);
    } else {
      if (P.use_pradhana) epp = 0.f;
      dgam = 0.f;
    }
    if ((p_trial + p_shift) > p_tip && q_trial > q_yield) {
      ++plastic;
      double dg = 0.0;
      if (P.perzyna_exp == 1.0) {
        dg = (q_trial - q_yield) / (fmu + q_yield * P.perzyna_visc / dt);
        if (dg < 0) err |= E_NEG_DGAMMA;
      } else {
        ++solves;
        const float hf[3] = {(float)h[0], (float)h[1], (float)h[2]};
        const float hdf[3] = {(float)hd[0], (float)hd[1], (float)hd[2]};
        if (newton_path<kExtras>(P, B, i, false, dt, hf, hdf, q_trial, q_yield, epd, U, V, dg, iters, err)) {
          out.queued = true;
          return;
        }
      }
      for (int k = 0; k < 3; ++k) out.h[k] = (float)(h[k] - (dg / dpre) * hd[k]);
      out.changed = true;
      epd = (float)((double)epd + dg / dpre);
      dgam = (float)(dg / dt);
    }
  }
}

// F = U exp(h) V^T and the Kirchhoff stress tau = U diag(2 mu h + lambda tr h) U^T of the final F
// (simulation.hpp:287-294 evaluated on the factors the return map already has), in FP32.
__device__ __forceinline__ void finish_F_tau(const Params& P, const float* U, const float* V, const float hfin[3],
                                             bool rebuild, const float* Ft, float Fout[9], float tau[6]) {
  if (rebuild) {
    const float e[3] = {expf(hfin[0]), expf(hfin[1]), expf(hfin[2])};
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int q = 0; q < 3; ++q)
        Fout[3 * r + q] = U[3 * r] * e[0] * V[3 * q] + U[3 * r + 1] * e[1] * V[3 * q + 1] + U[3 * r + 2] * e[2] * V[3 * q + 2];
  } else if (Ft) {
#pragma unroll
    for (int k = 0; k < 9; ++k) Fout[k] = Ft[k];
  }
  const float tr = hfin[0] + hfin[1] + hfin[2];
  const float mu2 = (float)(2.0 * P.mu), lam = (float)P.lambda;
  float d[3];
  for (int k = 0; k < 3; ++k) d[k] = mu2 * hfin[k] + lam * tr;
  if (!(isfinite(d[0]) && isfinite(d[1]) && isfinite(d[2]))) { d[0] = d[1] = d[2] = 0.f; }
  auto T = [&](int r, int q) { return U[3 * r] * d[0] * U[3 * q] + U[3 * r + 1] * d[1] * U[3 * q + 1] + U[3 * r + 2] * d[2] * U[3 * q + 2]; };
  tau[0] = T(0, 0); tau[1] = T(1, 1); tau[2] = T(2, 2);
  tau[3] = T(0, 1); tau[4] = T(0, 2); tau[5] = T(1, 2);
}

// The update runs as two kernels.  kPart 1, the head, over the bricks: velocity gradient L from
// the brick's MUSL velocity tile (handed to the tail in the output's F field) and the position
// update.  kPart 2, the tail, over the active particles in sorted order: F_trial = F + dt L F in
// FP64, the FP64 SVD, return map and stress.  Split this way the tail is a flat particle-parallel
// kernel with no block barriers and a smaller instruction footprint than the whole update (on the
// 2M scene 0.140 + 0.175 ms against 0.372 ms as one kernel, for 72 B more traffic per particle:
// L out and back).
template <int kModel, bool kExtras, int kPart>
__device__ __forceinline__ void d_defgrad(const Params& P, const Bufs& B, const int blk_, const int nblk_) {
  const int model = kModel >= 0 ? kModel : P.plastic_model;
  const Ctrl* c = B.ctrl;
  if (c->halt || c->idle) return;
  const int S = P.np_stride, np = P.np;
  const double dt = c->dt;
  const float dtf = (float)dt;
  const float dx = P.dx;
  uint32_t err = 0, plastic = 0, nact = 0, niters = 0, nsolves = 0;
  float maxv2 = 0.f;
  int mn[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, mx[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
  const int stride = nblk_ * blockDim.x;
  const float fr = P.flip_ratio;
  // grid velocities of the brick's 6x6x6 stencil tile: the MUSL velocity (normalised once per
  // node here) or, in USL mode, the updated grid velocity
#if PM_HEAD_ASYNC
  __shared__ float4 vt2[2][kTileNodes];
  // per thread, two slots of its particle's staged words: meta, x (3), pic (3), v (3)
  constexpr int kHS = 10;
  __shared__ float hs[2][kHS][kThreads];
  const float4* vt = vt2[0];
  int hslot = 0;
#else
  __shared__ float4 vt[kTileNodes];
#endif
  int bx = 0, by = 0, bz = 0;
  float* po = B.pout;
  const float* pi = B.pin;
  // SVD, return map and stress of sorted particle i (read index o) from its trial F
  auto tail = [&](const int i, const uint32_t o, const double Ft[9]) {
    double sg[3];
    float U[9], V[9];
    svd3_warm(Ft, U, sg, V);
    float epd = pi[F_EPD * S + o], epv = pi[F_EPV * S + o], epp = pi[F_EPP * S + o], dgam = 0.f;
    float hfin[3];
    bool changed = false, queued = false;
    if (model != PL_NONE) {
      ReturnMapOut rm;
      return_map<kModel, kExtras>(P, B, (uint32_t)i, dt, sg, U, V, epd, epv, epp, dgam, plastic, niters, nsolves, err,
                                  rm);
      changed = rm.changed;
      queued = rm.queued;
      if (rm.to_rotation) { hfin[0] = hfin[1] = hfin[2] = 0.f; }
      else for (int k = 0; k < 3; ++k) hfin[k] = rm.h[k];
    }
    if (!changed) for (int k = 0; k < 3; ++k) hfin[k] = logf(fabsf((float)sg[k]));
    if (!queued) {  // queued particles get F, tau, eps_pl_dev and delta_gamma from the surrogate pass
      float Fout[9], tau[6];
      finish_F_tau(P, U, V, hfin, changed, nullptr, Fout, tau);
      if (changed) {
#pragma unroll
        for (int k = 0; k < 9; ++k) po[(F_F + k) * S + i] = Fout[k];
      }
#pragma unroll
      for (int k = 0; k < 6; ++k) po[(F_TAU + k) * S + i] = tau[k];
      po[F_EPD * S + i] = epd;
      po[F_DG * S + i] = dgam;
    }
    po[F_EPV * S + i] = epv;
    po[F_EPP * S + i] = epp;
  };
  auto particle = [&](const int i, const uint32_t o) {
#if PM_HEAD_ASYNC
    const uint32_t meta = __float_as_uint(hs[hslot][0][threadIdx.x]);
#else
    const uint32_t meta = B.meta_in[o];
#endif
    float xp[3];
    AxisW aw[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
#if PM_HEAD_ASYNC
      xp[d] = hs[hslot][1 + d][threadIdx.x];
#else
      xp[d] = pi[(F_X + d) * S + o];
#endif
      aw[d] = axis_weights(xp[d], P.anchor[d], dx, P.inv_dx);
    }
    const int cl = local_cell(aw, c, bx, by, bz);
    const int t0 = ((cl >> 4) * kTile + ((cl >> 2) & 3)) * kTile + (cl & 3);
#if PM_HEAD_POLYW
    const float fpos[3] = {aw[0].r * P.inv_dx, aw[1].r * P.inv_dx, aw[2].r * P.inv_dx};
#endif
    // velocity gradient from the MUSL grid (deformation_update.cpp:26-39)
    float L[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) L[k] = 0.f;
    // the x-layer loop may stay rolled (kDefgradUnrollX) to keep the kernel's code small; its
    // per-layer values are picked with selects, not indexed, so they stay in registers
#pragma unroll kDefgradUnrollX
    for (int a = 0; a < 3; ++a) {
#if PM_HEAD_POLYW
      // weights formed where they are used, from the position in the base cell
      const float Na = bs_n(fpos[0], a), dNa = bs_dn(fpos[0], a, P.inv_dx);
#define PM_HN(d, k) bs_n(fpos[d], k)
#define PM_HDN(d, k) bs_dn(fpos[d], k, P.inv_dx)
#else
      const float Na = a == 0 ? aw[0].N[0] : (a == 1 ? aw[0].N[1] : aw[0].N[2]);
      const float dNa = a == 0 ? aw[0].dN[0] : (a == 1 ? aw[0].dN[1] : aw[0].dN[2]);
#define PM_HN(d, k) aw[d].N[k]
#define PM_HDN(d, k) aw[d].dN[k]
#endif
#pragma unroll
      for (int bb = 0; bb < 3; ++bb)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          const float4 m = vt[t0 + (a * kTile + bb) * kTile + cc];
          const float gv[3] = {m.x, m.y, m.z};
          const float g[3] = {dNa * PM_HN(1, bb) * PM_HN(2, cc), Na * PM_HDN(1, bb) * PM_HN(2, cc),
                              Na * PM_HN(1, bb) * PM_HDN(2, cc)};
#undef PM_HN
#undef PM_HDN
#pragma unroll
          for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int q = 0; q < 3; ++q) L[3 * r + q] += gv[r] * g[q];
        }
    }
    // position update (position_update.cpp:6-91); done before the SVD so that its values are not
    // live across it
    float pic[3], v[3];
#if PM_HEAD_ASYNC
#pragma unroll
    for (int r = 0; r < 3; ++r) { pic[r] = hs[hslot][4 + r][threadIdx.x]; v[r] = hs[hslot][7 + r][threadIdx.x]; }
#else
#pragma unroll
    for (int r = 0; r < 3; ++r) { pic[r] = B.pic[r * S + i]; v[r] = po[(F_V + r) * S + i]; }
#endif
    if (!P.use_musl) {
      for (int r = 0; r < 3; ++r) {
        const float fl = B.pic[(3 + r) * S + i];
        if (fr < -1.f) v[r] = pic[r];
        else if (fr < 0.f) v[r] = (-fr) * (v[r] + fl) + (1.f - (-fr)) * pic[r];
        else v[r] = fr * (v[r] + fl) + (1.f - fr) * pic[r];
      }
    }
    float xn[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) xn[r] = xp[r] + dtf * pic[r];
    bool active = true;
    bool bad = false;
    for (int r = 0; r < 3; ++r)
      if (isnan(xn[r]) || isinf(xn[r]) || isnan(v[r]) || isinf(v[r])) bad = true;
    if (bad) {
      active = false;
      err |= E_NAN_PARTICLE;
      for (int r = 0; r < 3; ++r) { v[r] = 0.f; xn[r] = P.use_particle_boundaries ? P.pbmin[r] : 0.f; }
    } else {
      if (xn[1] < 0.f) { xn[1] = 0.f; if (v[1] < 0.f) v[1] = 0.f; }
      if (P.use_particle_boundaries) {
        for (int r = 0; r < 3; ++r) {
          if (xn[r] < P.pbmin[r]) { xn[r] = P.pbmin[r]; active = false; v[r] = 0.f; }
          else if (xn[r] > P.pbmax[r]) { xn[r] = P.pbmax[r]; active = false; v[r] = 0.f; }
        }
        if (!active) v[0] = v[1] = v[2] = 0.f;
      }
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) { po[(F_X + r) * S + i] = xn[r]; po[(F_V + r) * S + i] = v[r]; }
    B.meta_out[i] = active ? meta : (meta | kInactiveBit);
    if (active) {
      ++nact;
      maxv2 = fmaxf(maxv2, v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      for (int r = 0; r < 3; ++r) { int k = fkey(xn[r]); mn[r] = min(mn[r], k); mx[r] = max(mx[r], k); }
    }
    // the velocity gradient goes to the tail through the output's F field
#pragma unroll
    for (int k = 0; k < 9; ++k) po[(F_F + k) * S + i] = L[k];
  };
  if constexpr (kPart == 2) {
    const int nact_sorted = (int)B.cell[c->n_nodes];
#if PM_PREFETCH_TAIL
    const int i0 = blk_ * blockDim.x + threadIdx.x;
    uint32_t o_next = i0 < nact_sorted ? B.sorted[i0] : 0u;
#endif
    for (int i = blk_ * blockDim.x + threadIdx.x; i < nact_sorted; i += stride) {
#if PM_PREFETCH_TAIL
      // the next particle's sorted index now, its F and plastic state into L2 (below)
      const uint32_t o = o_next;
      const int i2 = i + stride;
      o_next = i2 < nact_sorted ? B.sorted[i2] : 0u;
      if (i2 < nact_sorted) {
#pragma unroll
        for (int f = F_F; f < F_F + 9; ++f) prefetch_l2(pi + (size_t)f * S + o_next);
#pragma unroll
        for (int f = F_EPD; f < F_DG; ++f) prefetch_l2(pi + (size_t)f * S + o_next);
      }
#else
      const uint32_t o = B.sorted[i];
#endif
      // F_trial = F + dt L F (FP64)
      double L[9], F[9], Ft[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        L[k] = (double)po[(F_F + k) * S + i];
        F[k] = (double)pi[(F_F + k) * S + o];
      }
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          double sum = 0.0;
#pragma unroll
          for (int k = 0; k < 3; ++k) sum += L[3 * r + k] * F[3 * k + q];
          Ft[3 * r + q] = F[3 * r + q] + dt * sum;
        }
      // F_trial is the stored F unless the return map changes it (then it is overwritten in the
      // tail; both writes meet in L2), so it need not stay in registers across the SVD
#pragma unroll
      for (int k = 0; k < 9; ++k) po[(F_F + k) * S + i] = (float)Ft[k];
      tail(i, o, Ft);
    }
  }
  const int nbr = kPart == 2 ? 0 : (int)B.blist_n[0];
#if PM_HEAD_ASYNC
  // the velocity tile of brick list entry ib_ into tile slot `slot`, normalised after arrival
  auto issue_tile = [&](const int ib_, const int slot) {
    int qx, qy, qz;
    brick_coords((int)B.blist_occ[ib_].x, c, qx, qy, qz);
    for (int tn = threadIdx.x; tn < kTileNodes; tn += blockDim.x) {
      const int node = tile_to_node(tn, qx, qy, qz, c);
      const float4* src = P.use_musl ? B.gmusl + (node >= 0 ? node : 0) : B.grid + (size_t)(node >= 0 ? node : 0) * 4;
      cp_async16_zfill(&vt2[slot][tn], src, node >= 0);
    }
  };
  // particle i's staged words (read index o) into particle slot `slot`
  auto issue_particle = [&](const int i, const uint32_t o, const int slot) {
    cp_async4(&hs[slot][0][threadIdx.x], B.meta_in + o);
#pragma unroll
    for (int d = 0; d < 3; ++d) cp_async4(&hs[slot][1 + d][threadIdx.x], pi + (size_t)(F_X + d) * S + o);
#pragma unroll
    for (int r = 0; r < 3; ++r) cp_async4(&hs[slot][4 + r][threadIdx.x], B.pic + (size_t)r * S + i);
#pragma unroll
    for (int r = 0; r < 3; ++r) cp_async4(&hs[slot][7 + r][threadIdx.x], po + (size_t)(F_V + r) * S + i);
  };
  if (blk_ < nbr) issue_tile(blk_, 0);
  cp_async_commit();
  int tslot = 0;
  for (int ib = blk_; ib < nbr; ib += nblk_, tslot ^= 1) {
    const uint4 be = B.blist_occ[ib];
    const int b = (int)be.x;
    const uint32_t ps = be.y, pe = be.z;
    brick_coords(b, c, bx, by, bz);
    __syncthreads();  // the brick before the previous one is done with the other tile slot
    if (ib + nblk_ < nbr) issue_tile(ib + nblk_, tslot ^ 1);
    cp_async_commit();
    cp_async_wait_1();  // this brick's tile (all but the group just committed)
    __syncthreads();
    vt = vt2[tslot];
    if (P.use_musl) {
      for (int tn = threadIdx.x; tn < kTileNodes; tn += blockDim.x) {
        const float4 m = vt2[tslot][tn];
        const float inv = m.w > 0.f ? 1.f / m.w : 0.f;
        vt2[tslot][tn] = make_float4(m.x * inv, m.y * inv, m.z * inv, 0.f);
      }
    }
    __syncthreads();
    {
      int i = (int)ps + (int)threadIdx.x;
      if (i < (int)pe) issue_particle(i, B.sorted[i], hslot ^ 1);
      cp_async_commit();
      for (; i < (int)pe; i += blockDim.x) {
        hslot ^= 1;  // the slot the copies above went to
        const uint32_t o = B.sorted[i];
        const int i2 = i + (int)blockDim.x;
        if (i2 < (int)pe) issue_particle(i2, B.sorted[i2], hslot ^ 1);
        cp_async_commit();
        cp_async_wait_1();  // this particle's words
        particle(i, o);
      }
    }
  }
#else
  for (int ib = blk_; ib < nbr; ib += nblk_) {
    const uint4 be = B.blist_occ[ib];
    const int b = (int)be.x;
    const uint32_t ps = be.y, pe = be.z;
    brick_coords(b, c, bx, by, bz);
    __syncthreads();  // the previous brick's readers are done with the tile
    for (int tn = threadIdx.x; tn < kTileNodes; tn += blockDim.x) {
      const int node = tile_to_node(tn, bx, by, bz, c);
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (node >= 0) {
        if (P.use_musl) {
          const float4 m = B.gmusl[node];
          const float inv = m.w > 0.f ? 1.f / m.w : 0.f;
          v = make_float4(m.x * inv, m.y * inv, m.z * inv, 0.f);
        } else {
          const float4 m = B.grid[(size_t)node * 4];
          v = make_float4(m.x, m.y, m.z, 0.f);
        }
      }
      vt[tn] = v;
    }
    __syncthreads();
#if PM_PREFETCH
    uint32_t o_next = (int)ps + (int)threadIdx.x < (int)pe ? B.sorted[ps + threadIdx.x] : 0u;
    for (int i = (int)ps + threadIdx.x; i < (int)pe; i += blockDim.x) {
      const uint32_t o = o_next;
      const int i2 = i + (int)blockDim.x;
      o_next = i2 < (int)pe ? B.sorted[i2] : 0u;
      particle(i, o);
      if (i2 < (int)pe) {  // the next particle's position and meta word
        prefetch_l2(B.meta_in + o_next);
#pragma unroll
        for (int f = F_X; f < F_X + 3; ++f) prefetch_l2(pi + (size_t)f * S + o_next);
      }
    }
#else
    for (int i = (int)ps + threadIdx.x; i < (int)pe; i += blockDim.x) particle(i, B.sorted[i]);
#endif
  }
#endif
  // inactive particles sit behind every brick in the sorted order: carried through unchanged
  // (G2P zeroes B, the deformation update zeroes delta_gamma)
  for (int i = (int)B.cell[c->n_nodes] + blk_ * blockDim.x + threadIdx.x; kPart != 2 && i < np; i += stride) {
    const uint32_t o = B.sorted[i];
    for (int f = 0; f < F_COUNT; ++f) {
      float v = pi[f * S + o];
      if ((f >= F_B && f < F_B + 9) || f == F_DG) v = 0.f;
      po[f * S + i] = v;
    }
    B.meta_out[i] = B.meta_in[o];
  }
  // block reduction, then one set of atomics per block
  __shared__ int red_i[kWarps][8];
  __shared__ uint32_t red_u[kWarps][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t mv = __reduce_max_sync(0xffffffffu, __float_as_uint(maxv2));
  uint32_t na = __reduce_add_sync(0xffffffffu, nact);
  uint32_t pc = __reduce_add_sync(0xffffffffu, plastic);
  uint32_t er = __reduce_or_sync(0xffffffffu, err);
  const uint32_t ni = __reduce_add_sync(0xffffffffu, niters), ns = __reduce_add_sync(0xffffffffu, nsolves);
  int r6[6];
  for (int r = 0; r < 3; ++r) { r6[r] = __reduce_min_sync(0xffffffffu, mn[r]); r6[3 + r] = __reduce_max_sync(0xffffffffu, mx[r]); }
  if (lane == 0) {
    if (ni) atomicAdd(&B.ctrl->newton_iters, ni);
    if (ns) atomicAdd(&B.ctrl->newton_solves, ns);
    red_u[warp][0] = mv; red_u[warp][1] = na; red_u[warp][2] = pc; red_u[warp][3] = er;
    for (int k = 0; k < 6; ++k) red_i[warp][k] = r6[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kWarps; ++w) {
      red_u[0][0] = max(red_u[0][0], red_u[w][0]);
      red_u[0][1] += red_u[w][1];
      red_u[0][2] += red_u[w][2];
      red_u[0][3] |= red_u[w][3];
      for (int r = 0; r < 3; ++r) { red_i[0][r] = min(red_i[0][r], red_i[w][r]); red_i[0][3 + r] = max(red_i[0][3 + r], red_i[w][3 + r]); }
    }
    Ctrl* cw = B.ctrl;
    if (red_u[0][1]) {
      atomicMax(&cw->max_v2, red_u[0][0]);
      atomicAdd(&cw->n_active, red_u[0][1]);
      for (int r = 0; r < 3; ++r) { atomicMin(&cw->xmin_key[r], red_i[0][r]); atomicMax(&cw->xmax_key[r], red_i[0][3 + r]); }
    }
    if (red_u[0][2]) atomicAdd(&cw->plastic_count, red_u[0][2]);
    if (red_u[0][3]) atomicOr(&cw->error_flags, red_u[0][3]);
  }
}
// Plain-solver instantiations per plastic model (kExtras = false) and the generic kernel (model
// and extras chosen at run time) that the surrogate, the sample log and mixed batches use.
__global__ void __launch_bounds__(kThreads, PM_HEAD_MINB) k_defgrad_head(Params P, Bufs B) {
  pdl_enter();
  d_defgrad<PL_NONE, false, 1>(P, B, blockIdx.x, gridDim.x);
}
template <int kModel, bool kExtras>
__global__ void __launch_bounds__(kThreads, PM_DEFGRAD_MINB) k_defgrad_tail(Params P, Bufs B) {
  pdl_enter();
  d_defgrad<kModel, kExtras, 2>(P, B, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(kThreads, PM_HEAD_MINB) kb_defgrad_head(const SceneDev* __restrict__ sd,
                                                               const int* __restrict__ off, int ns) {
  int s_, blk_, nblk_;
  batch_slot(off, ns, s_, blk_, nblk_);
  __shared__ SceneShared ss_;
  load_scene_shared(sd[s_], ss_);
  d_defgrad<PL_NONE, false, 1>(ss_.P, ss_.B, blk_, nblk_);
}
template <int kModel, bool kExtras>
__global__ void __launch_bounds__(kThreads, PM_DEFGRAD_MINB) kb_defgrad_tail(const SceneDev* __restrict__ sd,
                                                                             const int* __restrict__ off, int ns) {
  int s_, blk_, nblk_;
  batch_slot(off, ns, s_, blk_, nblk_);
  __shared__ SceneShared ss_;
  load_scene_shared(sd[s_], ss_);
  d_defgrad<kModel, kExtras, 2>(ss_.P, ss_.B, blk_, nblk_);
}


// Surrogate pass: each queued particle turns the network's plastic strain into an estimate of
// the consistency parameter along its flow direction and checks it against the Perzyna
// consistency condition (|r| < 1e-2 Pa, the reference's Newton tolerance).  Estimates that fail
// drop to the plain Newton solve -- continued from the estimate, or restarted from the
// reference's initial guess when sur_fallback_plain is set.  The final F, stress, eps_pl_dev and
// delta_gamma are written as the plain path writes them.
__device__ __forceinline__ void d_sur_finish(const Params& P, const Bufs& B, const int blk_, const int nblk_) {
  const Ctrl* c = B.ctrl;
  if (c->halt || c->idle) return;
  const uint32_t n = min(c->q_n, P.q_cap);
  const double dt = c->dt;
  const int S = P.np_stride;
  uint32_t err = 0, iters = 0, accepted = 0;
  for (uint32_t k = blk_ * blockDim.x + threadIdx.x; k < n; k += nblk_ * blockDim.x) {
    const SurQ& r = B.q[k];
    const float* y = B.qy + (size_t)k * 6;
    double pd = 0.0, pr = 0.0;
    for (int j = 0; j < 3; ++j) { pd += (double)y[j] * r.hd[j]; pr += (double)y[3 + j] * r.hd[j]; }
    double dg = P.d_prefac * 0.5 * (pd + pr * dt);
    const double dg_max = (double)r.q_trial / P.f_mu_prefac;
    if (!(dg >= 0.0)) dg = 0.0;
    if (dg > dg_max) dg = dg_max;
    uint32_t it = 0;
    const bool vm = r.vm != 0;
    auto solve = [&](double start) -> double {
      if (vm) return perzyna_newton_vm32(P, r.q_trial, r.epd, (float)dt, (float)start, it, err);
      return perzyna_newton(P, false, r.q_trial, r.q_y, (double)r.epd, dt, start, it, err);
    };
    double dgf = solve(dg);
    if (it == 0) ++accepted;
    else if (P.sur_fallback_plain) {
      it = 0;
      dgf = solve(0.01 * ((double)r.q_trial - (double)r.q_y) / P.f_mu_prefac);
    }
    iters += it;
    float hfin[3];
    for (int j = 0; j < 3; ++j) hfin[j] = (float)(r.h[j] - (dgf / P.d_prefac) * r.hd[j]);
    float Fout[9], tau[6];
    finish_F_tau(P, r.U, r.V, hfin, true, nullptr, Fout, tau);
    float* po = B.pout;
    const uint32_t i = r.i;
#pragma unroll
    for (int q = 0; q < 9; ++q) po[(F_F + q) * S + i] = Fout[q];
#pragma unroll
    for (int q = 0; q < 6; ++q) po[(F_TAU + q) * S + i] = tau[q];
    po[F_EPD * S + i] = (float)((double)r.epd + dgf / P.d_prefac);
    po[F_DG * S + i] = (float)(dgf / dt);
  }
  const uint32_t ni = __reduce_add_sync(0xffffffffu, iters), na = __reduce_add_sync(0xffffffffu, accepted);
  const uint32_t er = __reduce_or_sync(0xffffffffu, err);
  if ((threadIdx.x & 31) == 0) {
    if (ni) atomicAdd(&B.ctrl->newton_iters, ni);
    if (na) atomicAdd(&B.ctrl->sur_accept, na);
    if (er) atomicOr(&B.ctrl->error_flags, er);
  }
}
__global__ void __launch_bounds__(128) k_sur_finish(Params P, Bufs B) {
  pdl_enter();
  d_sur_finish(P, B, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(128) kb_sur_finish(const SceneDev* __restrict__ sd, const int* __restrict__ off, int ns) {
  int s_, blk_, nblk_;
  batch_slot(off, ns, s_, blk_, nblk_);
  const SceneDev& d_ = sd[s_];
  d_sur_finish(d_.P, d_.B[scene_parity(d_)], blk_, nblk_);
}


// Reductions over the current particle state (prepare time): max |v|^2, AABB, active count.
__global__ void __launch_bounds__(kThreads) k_reduce_state(Params P, const float* pcur, const uint32_t* meta, Ctrl* cw) {
  const int S = P.np_stride;
  uint32_t nact = 0;
  float maxv2 = 0.f;
  int mn[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, mx[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.np; i += gridDim.x * blockDim.x) {
    if (meta[i] & kInactiveBit) continue;
    ++nact;
    float v2 = 0.f;
    for (int r = 0; r < 3; ++r) {
      float v = pcur[(F_V + r) * S + i];
      v2 += v * v;
      int k = fkey(pcur[(F_X + r) * S + i]);
      mn[r] = min(mn[r], k); mx[r] = max(mx[r], k);
    }
    maxv2 = fmaxf(maxv2, v2);
  }
  uint32_t mv = __reduce_max_sync(0xffffffffu, __float_as_uint(maxv2));
  uint32_t na = __reduce_add_sync(0xffffffffu, nact);
  int r6[6];
  for (int r = 0; r < 3; ++r) { r6[r] = __reduce_min_sync(0xffffffffu, mn[r]); r6[3 + r] = __reduce_max_sync(0xffffffffu, mx[r]); }
  if ((threadIdx.x & 31) == 0 && na) {
    atomicMax(&cw->max_v2, mv);
    atomicAdd(&cw->n_active, na);
    for (int r = 0; r < 3; ++r) { atomicMin(&cw->xmin_key[r], r6[r]); atomicMax(&cw->xmax_key[r], r6[3 + r]); }
  }
}

// Copy particle fields back to the original order, grouped as host arrays: field group g
// (x, v, B, F, latent, diffusion, plastic, tau) of particle pid lands at
// out[g_base * np + pid * g_width + component].
__constant__ int c_group_base[F_COUNT] = {0, 0, 0, 3, 3, 3, 6, 6, 6, 6, 6, 6, 6, 6, 6, 15, 15, 15, 15, 15, 15, 15, 15, 15,
                                          24, 24, 24, 24, 24, 24, 24, 31, 32, 32, 32, 32, 36, 36, 36, 36, 36, 36};
__constant__ int c_group_width[F_COUNT] = {3, 3, 3, 3, 3, 3, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9,
                                           7, 7, 7, 7, 7, 7, 7, 1, 4, 4, 4, 4, 6, 6, 6, 6, 6, 6};
// Field group of each field (x, v, B, F, latent, diffusion, plastic, tau = groups 0..7): k_unpermute
// copies only the groups whose bit is set in group_mask.
__constant__ int c_group_id[F_COUNT] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 2, 2, 2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 3, 3, 3,
                                        4, 4, 4, 4, 4, 4, 4, 5, 6, 6, 6, 6, 7, 7, 7, 7, 7, 7};
__global__ void k_unpermute(Params P, const float* pcur, const uint32_t* meta, float* out, uint8_t* active_out,
                            uint32_t group_mask) {
  const int S = P.np_stride, np = P.np;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    const uint32_t m = meta[i];
    const uint32_t pid = m & ~kInactiveBit;
    if (pid >= (uint32_t)np) continue;
    for (int f = 0; f < F_COUNT; ++f) {
      if (!((group_mask >> c_group_id[f]) & 1u)) continue;
      const int gb = c_group_base[f], gw = c_group_width[f];
      out[(size_t)gb * np + (size_t)pid * gw + (f - gb)] = pcur[f * S + i];
    }
    active_out[pid] = (m & kInactiveBit) ? 0 : 1;
  }
}

// Host arrays (x[n*3], latent[n*7], v[n*3] or null) staged on the device -> SoA state with
// F = I, B = 0 and zero plastic state, meta = particle id.
__global__ void k_upload(Params P, const float* x, const float* lat, const float* v, float* pbuf, uint32_t* meta) {
  const int S = P.np_stride, np = P.np;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < S; p += gridDim.x * blockDim.x) {
    const bool in = p < np;
    for (int f = 0; f < F_COUNT; ++f) pbuf[f * S + p] = 0.f;
    if (in) {
      for (int d = 0; d < 3; ++d) {
        pbuf[(F_X + d) * S + p] = x[3 * p + d];
        pbuf[(F_V + d) * S + p] = v ? v[3 * p + d] : 0.f;
      }
      if (lat) for (int k = 0; k < 7; ++k) pbuf[(F_LAT + k) * S + p] = lat[7 * p + k];
      pbuf[(F_F + 0) * S + p] = 1.f;
      pbuf[(F_F + 4) * S + p] = 1.f;
      pbuf[(F_F + 8) * S + p] = 1.f;
    }
    meta[p] = in ? (uint32_t)p : kInactiveBit;
  }
}

// Inverse of k_unpermute for checkpoints: particle pid's fields from the grouped host layout
// (group base * np + pid * group width + component) into slot pid of the SoA buffer.
__global__ void k_load_fields(Params P, const float* in, const uint8_t* active, float* pbuf, uint32_t* meta) {
  const int S = P.np_stride, np = P.np;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < S; p += gridDim.x * blockDim.x) {
    if (p >= np) {
      for (int f = 0; f < F_COUNT; ++f) pbuf[f * S + p] = 0.f;
      meta[p] = kInactiveBit;
      continue;
    }
    for (int f = 0; f < F_COUNT; ++f) {  // a group's base is the index of its first field
      const int g = c_group_base[f], w = c_group_width[f];
      pbuf[f * S + p] = in[(size_t)g * np + (size_t)p * w + (f - g)];
    }
    meta[p] = (uint32_t)p | (active[p] ? 0u : kInactiveBit);
  }
}

// Diagnostics: mass, momentum, mass-weighted latent sums (double atomics per block).
// With cyl set, only particles inside the vertical cylinder (x - cx)^2 + (z - cz)^2 <= r2 count
// (the sampling region of MPMIntegrationSim::calculateAndPrintFinalColor, MPMIntegrationSim.cpp:48-90).
__global__ void __launch_bounds__(kThreads) k_stats(Params P, const float* pcur, const uint32_t* meta, double* acc,
                                                    int cyl, float cx, float cz, float r2) {
  const int S = P.np_stride;
  double s[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.np; i += gridDim.x * blockDim.x) {
    if (meta[i] & kInactiveBit) continue;
    if (cyl) {
      const float ex = pcur[F_X * S + i] - cx, ez = pcur[(F_X + 2) * S + i] - cz;
      if (ex * ex + ez * ez > r2) continue;
    }
    s[0] += 1.0;
    for (int r = 0; r < 3; ++r) s[1 + r] += pcur[(F_V + r) * S + i];
    for (int k = 0; k < 7; ++k) s[4 + k] += pcur[(F_LAT + k) * S + i];
  }
  for (int k = 0; k < 11; ++k) {
    double v = s[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&acc[k], v);
  }
}

// ------------------------------------------------------------------------------------------
// host-side launchers
// ------------------------------------------------------------------------------------------
static int g_num_sms = 0;
static int g_occ_p2g = 1, g_occ_g2p = 1, g_occ_def = 1;
int scan_ctas_for(int node_cap, int max_ctas);

// Kernel attributes and launch shapes, set once per device (later calls return at once).
cudaError_t launch_init(int device) {
  static std::mutex mu;
  static std::vector<char> done;
  std::lock_guard<std::mutex> lock(mu);
  if (device >= 0 && device < (int)done.size() && done[device]) return cudaSuccess;
  cudaError_t e = launch_init_device(device);
  if (e == cudaSuccess && device >= 0) {
    if ((int)done.size() <= device) done.resize(device + 1, 0);
    done[device] = 1;
  }
  return e;
}

cudaError_t launch_init_device(int device) {
  cudaError_t e = cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_p2g, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p2g_smem_bytes());
  if (e != cudaSuccess) return e;
  for (const void* f : {(const void*)k_g2p_musl<true>, (const void*)k_g2p_musl<false>, (const void*)kb_g2p_musl<true>,
                        (const void*)kb_g2p_musl<false>}) {
    e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g2p_smem_bytes());
    if (e != cudaSuccess) return e;
  }
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_occ_p2g, k_p2g, kThreads, p2g_smem_bytes());
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_occ_g2p, k_g2p_musl<true>, kThreads, g2p_smem_bytes());
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_occ_def, k_defgrad_tail<-1, true>, kThreads, 0);
  e = cudaFuncSetAttribute(kb_p2g, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p2g_smem_bytes());
  if (e != cudaSuccess) return e;

  e = mlp_init();
  if (e != cudaSuccess) return e;
  if (g_occ_p2g < 1) g_occ_p2g = 1;
  if (g_occ_g2p < 1) g_occ_g2p = 1;
  if (g_occ_def < 1) g_occ_def = 1;
  return cudaGetLastError();
}

int num_sms() { return g_num_sms; }

// The kernels of one step in launch order (the surrogate pass adds k_mlp_infer and k_sur_finish).
static const char* kKernelNames[15] = {"k_prologue",     "k_clear",        "k_count",     "k_scan_local",
                                       "k_scan_add",     "k_scatter",      "k_clear_bricks", "k_p2g",
                                       "k_grid_update",  "k_g2p_musl",     "k_defgrad_head", "k_defgrad_tail",
                                       "k_mlp_infer",    "k_sur_finish",   "k_epilogue"};
int kernels_per_step(const Params& P) { return P.return_map == 1 ? 15 : 13; }
const char* kernel_name(int i, const Params& P) {
  if (i < 0 || i >= kernels_per_step(P)) return "";
  if (P.return_map != 1 && i == 12) return kKernelNames[14];
  return kKernelNames[i];
}

// Launches a step kernel with programmatic stream serialisation when PM_PDL is on (see pdl_enter).
template <typename... KArgs>
static void launch_k(void (*kern)(KArgs...), int grid, int block, size_t smem, cudaStream_t s, const Params& P,
                     const Bufs& B) {
#if PM_PDL
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, P, B);
#else
  kern<<<grid, block, smem, s>>>(P, B);
#endif
}

// One step on stream s; when ev is not null an event is recorded before the first kernel and
// after every kernel (ev must hold kernels_per_step + 1 events).
void launch_step(const Params& P, const Bufs& B, cudaStream_t s, cudaEvent_t* ev) {
  const int sms = g_num_sms > 0 ? g_num_sms : 148;
  const int flat_grid = sms * 8;
  const int scan_blocks = scan_ctas_for(P.node_cap, sms * 2);
  int e = 0;
  auto mark = [&]() { if (ev) cudaEventRecord(ev[e++], s); };
  mark();
  launch_k(k_prologue, 1, 32, 0, s, P, B); mark();
  launch_k(k_clear, flat_grid, 256, 0, s, P, B); mark();
  launch_k(k_count, flat_grid, 256, 0, s, P, B); mark();
  launch_k(k_scan_local, scan_blocks, kScanThreads, 0, s, P, B); mark();
  launch_k(k_scan_add, scan_blocks, kScanThreads, 0, s, P, B); mark();
  launch_k(k_scatter, flat_grid, 256, 0, s, P, B); mark();
  launch_k(k_clear_bricks, flat_grid, 256, 0, s, P, B); mark();
  launch_k(k_p2g, sms * g_occ_p2g, kThreads, p2g_smem_bytes(), s, P, B); mark();
  launch_k(k_grid_update, flat_grid, 256, 0, s, P, B); mark();
  if (P.flip_ratio >= -1.f) launch_k(k_g2p_musl<true>, sms * g_occ_g2p, kThreads, g2p_smem_bytes(), s, P, B);
  else launch_k(k_g2p_musl<false>, sms * g_occ_g2p, kThreads, g2p_smem_bytes(), s, P, B);
  mark();
  {
    const int g = sms * g_occ_def;
    const bool extras = P.return_map == 1 || P.log_cap > 0;
    launch_k(k_defgrad_head, sms * PM_HEAD_MINB, kThreads, 0, s, P, B); mark();
    if (!extras && P.plastic_model == PL_VMVISC) launch_k(k_defgrad_tail<PL_VMVISC, false>, g, kThreads, 0, s, P, B);
    else if (!extras && P.plastic_model == PL_DPVISC) launch_k(k_defgrad_tail<PL_DPVISC, false>, g, kThreads, 0, s, P, B);
    else if (!extras && P.plastic_model == PL_NONE) launch_k(k_defgrad_tail<PL_NONE, false>, g, kThreads, 0, s, P, B);
    else launch_k(k_defgrad_tail<-1, true>, g, kThreads, 0, s, P, B);
    mark();
  }
  if (P.return_map == 1) {
    mlp_infer(B.mlp, B.qx, B.qy, 0, &B.ctrl->q_n, (int)P.q_cap, s); mark();
    launch_k(k_sur_finish, sms * 8, 128, 0, s, P, B); mark();
  }
  launch_k(k_epilogue, 1, 32, 0, s, P, B); mark();
}

// ------------------------------------------------------------------------------------------
// batched scenes: every kernel of the step launched once for all scenes
// ------------------------------------------------------------------------------------------
static const char* kBatchKernelNames[15] = {
    "kb_prologue", "kb_clear", "kb_count", "kb_scan_local", "kb_scan_add", "kb_scatter", "kb_clear_bricks",
    "kb_p2g", "kb_grid_update", "kb_g2p_musl", "kb_defgrad_head", "kb_defgrad_tail", "kb_mlp_infer",
    "kb_sur_finish", "kb_epilogue"};
int batched_kernels_per_step(bool surrogate) { return surrogate ? 15 : 13; }
const char* batched_kernel_name(int i, bool surrogate) {
  if (i < 0 || i >= batched_kernels_per_step(surrogate)) return "";
  if (!surrogate && i == 12) return kBatchKernelNames[14];
  return kBatchKernelNames[i];
}
void batched_occupancy(int& p2g, int& g2p, int& def) {
  p2g = g2p = def = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p2g, kb_p2g, kThreads, p2g_smem_bytes());
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g2p, kb_g2p_musl<true>, kThreads, g2p_smem_bytes());
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&def, kb_defgrad_tail<-1, true>, kThreads, 0);
  p2g = p2g < 1 ? 1 : p2g;
  g2p = g2p < 1 ? 1 : g2p;
  def = def < 1 ? 1 : def;
}
int scan_blocks_for(int node_cap) { return (node_cap + 1 + kScanBlock - 1) / kScanBlock; }
int scan_ctas_for(int node_cap, int max_ctas) { return std::max(1, std::min(scan_blocks_for(node_cap), max_ctas)); }

// One round (one step of every scene that has not reached its target) on stream s.  Each launch
// covers all scenes: CTAs are statically partitioned across scenes by the offset tables, and each
// CTA loops over its scene's work with the scene's CTA count as stride.
void launch_step_batched(const BatchLaunch& L, cudaStream_t s, cudaEvent_t* ev) {
  int e = 0;
  auto mark = [&]() { if (ev) cudaEventRecord(ev[e++], s); };
  const SceneDev* sd = L.sd;
  const int ns = L.ns, ft = L.flat_threads;
  mark();
  kb_prologue<<<ns, 32, 0, s>>>(sd, L.off_unit, ns); mark();
  kb_clear<<<L.n_node, ft, 0, s>>>(sd, L.off_node, ns); mark();
  kb_count<<<L.n_part, ft, 0, s>>>(sd, L.off_part, ns); mark();
  kb_scan_local<<<L.n_scan, kScanThreads, 0, s>>>(sd, L.off_scan, ns); mark();
  kb_scan_add<<<L.n_scan, kScanThreads, 0, s>>>(sd, L.off_scan, ns); mark();
  kb_scatter<<<L.n_part, ft, 0, s>>>(sd, L.off_part, ns); mark();
  kb_clear_bricks<<<L.n_node, ft, 0, s>>>(sd, L.off_node, ns); mark();
  kb_p2g<<<L.n_p2g, kThreads, p2g_smem_bytes(), s>>>(sd, L.off_p2g, ns); mark();
  kb_grid_update<<<L.n_node, ft, 0, s>>>(sd, L.off_node, ns); mark();
  if (L.g2p_flip) kb_g2p_musl<true><<<L.n_g2p, kThreads, g2p_smem_bytes(), s>>>(sd, L.off_g2p, ns);
  else kb_g2p_musl<false><<<L.n_g2p, kThreads, g2p_smem_bytes(), s>>>(sd, L.off_g2p, ns);
  mark();
  kb_defgrad_head<<<L.n_def, kThreads, 0, s>>>(sd, L.off_def, ns); mark();
  if (L.defgrad_model == PL_VMVISC) kb_defgrad_tail<PL_VMVISC, false><<<L.n_def, kThreads, 0, s>>>(sd, L.off_def, ns);
  else if (L.defgrad_model == PL_DPVISC)
    kb_defgrad_tail<PL_DPVISC, false><<<L.n_def, kThreads, 0, s>>>(sd, L.off_def, ns);
  else if (L.defgrad_model == PL_NONE) kb_defgrad_tail<PL_NONE, false><<<L.n_def, kThreads, 0, s>>>(sd, L.off_def, ns);
  else kb_defgrad_tail<-1, true><<<L.n_def, kThreads, 0, s>>>(sd, L.off_def, ns);
  mark();
  if (L.surrogate) {
    mlp_infer_batched(sd, L.off_sur, ns, L.n_sur, s); mark();
    kb_sur_finish<<<L.n_sur, 128, 0, s>>>(sd, L.off_sur, ns); mark();
  }
  kb_epilogue<<<ns, 32, 0, s>>>(sd, L.off_unit, ns); mark();
}

void launch_upload(const Params& P, const float* x, const float* lat, const float* v, float* pbuf, uint32_t* meta,
                   cudaStream_t s) {
  const int sms = g_num_sms > 0 ? g_num_sms : 148;
  k_upload<<<sms * 4, 256, 0, s>>>(P, x, lat, v, pbuf, meta);
}

void launch_reduce_state(const Params& P, const float* pcur, const uint32_t* meta, Ctrl* ctrl, cudaStream_t s) {
  const int sms = g_num_sms > 0 ? g_num_sms : 148;
  k_reduce_state<<<sms * 4, kThreads, 0, s>>>(P, pcur, meta, ctrl);
}
void launch_unpermute(const Params& P, const float* pcur, const uint32_t* meta, float* out, uint8_t* active,
                      cudaStream_t s, uint32_t group_mask) {
  const int sms = g_num_sms > 0 ? g_num_sms : 148;
  k_unpermute<<<sms * 4, 256, 0, s>>>(P, pcur, meta, out, active, group_mask);
}
// Per particle, in original order: the reference's PLY vertex row (save_data.cpp:7-166) -- x, v,
// pressure p = -tr(tau)/3, deviatoric stress q = q_prefac |tau + p I|, Je = det F, eps_pl_vol,
// eps_pl_dev, delta_gamma -- from the cached Kirchhoff stress tau of the current F.
__global__ void k_ply_particles(Params P, const float* pcur, const uint32_t* meta, float* out) {
  const int S = P.np_stride, np = P.np;
  const float q_prefac = (float)(1.0 / P.d_prefac);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    const uint32_t pid = meta[i] & ~kInactiveBit;
    if (pid >= (uint32_t)np) continue;
    float* o = out + (size_t)pid * kPlyFields;
    for (int k = 0; k < 3; ++k) { o[k] = pcur[(F_X + k) * S + i]; o[3 + k] = pcur[(F_V + k) * S + i]; }
    float t[6], F[9];
    for (int k = 0; k < 6; ++k) t[k] = pcur[(F_TAU + k) * S + i];
    for (int k = 0; k < 9; ++k) F[k] = pcur[(F_F + k) * S + i];
    const float pr = -(t[0] + t[1] + t[2]) / 3.f;
    const float d0 = t[0] + pr, d1 = t[1] + pr, d2 = t[2] + pr;
    const float dd = d0 * d0 + d1 * d1 + d2 * d2 + 2.f * (t[3] * t[3] + t[4] * t[4] + t[5] * t[5]);
    o[6] = pr;
    o[7] = q_prefac * sqrtf(dd);
    o[8] = F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) + F[2] * (F[3] * F[7] - F[4] * F[6]);
    o[9] = pcur[F_EPV * S + i];
    o[10] = pcur[F_EPD * S + i];
    o[11] = pcur[F_DG * S + i];
  }
}
void launch_load_fields(const Params& P, const float* in, const uint8_t* active, float* pbuf, uint32_t* meta,
                        cudaStream_t s) {
  const int sms = g_num_sms > 0 ? g_num_sms : 148;
  k_load_fields<<<sms * 4, 256, 0, s>>>(P, in, active, pbuf, meta);
}
// Self-test of the device SVD: the step's svd3_warm on n caller matrices (row-major, FP64).
__global__ void k_svd3_batch(const double* __restrict__ A, int n, float* __restrict__ U, double* __restrict__ S,
                             float* __restrict__ V) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double a[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k] = A[(size_t)i * 9 + k];
    float u[9], v[9];
    double sg[3];
    svd3_warm(a, u, sg, v);
#pragma unroll
    for (int k = 0; k < 9; ++k) { U[(size_t)i * 9 + k] = u[k]; V[(size_t)i * 9 + k] = v[k]; }
#pragma unroll
    for (int k = 0; k < 3; ++k) S[(size_t)i * 3 + k] = sg[k];
  }
}
void launch_svd3_batch(const double* A, int n, float* U, double* S, float* V, cudaStream_t s) {
  if (n <= 0) return;
  const int blocks = std::min((n + 127) / 128, (g_num_sms > 0 ? g_num_sms : 148) * 8);
  k_svd3_batch<<<blocks, 128, 0, s>>>(A, n, U, S, V);
}

void launch_ply_particles(const Params& P, const float* pcur, const uint32_t* meta, float* out, cudaStream_t s) {
  const int sms = g_num_sms > 0 ? g_num_sms : 148;
  k_ply_particles<<<sms * 4, 256, 0, s>>>(P, pcur, meta, out);
}

void launch_stats(const Params& P, const float* pcur, const uint32_t* meta, double* acc, cudaStream_t s, int cyl,
                  float cx, float cz, float r2) {
  const int sms = g_num_sms > 0 ? g_num_sms : 148;
  k_stats<<<sms * 4, kThreads, 0, s>>>(P, pcur, meta, acc, cyl, cx, cz, r2);
}

}  // namespace pm

// Host runtime of the C ABI in include/pigment_mpm.h: owns device memory, the stream, the
// CUDA graphs of the step, and the mirror of the reference Simulation's public fields.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/pigment_mpm.h"
#include "pm_internal.cuh"
#include "pm_launch.h"
#include "pm_mlp.h"

using namespace pm;

namespace {

thread_local std::string g_err;

pm_status fail(pm_status s, const std::string& msg) {
  g_err = msg;
  return s;
}

#define CK(call)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return fail(PM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Public fields of Simulation with the reference's defaults (simulation.hpp:38-126).
struct HostParams {
  double fps = 1, cfl = 0.5, cfl_elastic = 1, flip_ratio = -0.95, rho = 1000, E = 1e5, nu = 0.3, min_dt = 1e-14;
  double dx = 0, particle_mass = 0, particle_volume = 0;
  double q_max = 100, q_min = 100, p_min = -1e20, M = 1, q_cohesion = 0, perzyna_exp = 1, perzyna_visc = 0, xi = 0;
  double q_prefac = 1.0 / std::sqrt(2.0);
  double D_max = 10e-2, D_edge0 = 0.5, D_edge1 = 0.8, start_boost = 20, end_boost = 40, boost_factor = 2;
  double end_frame = 10;
  int plastic_model = PM_NO_PLASTICITY;
  int use_pradhana = 1, use_musl = 0, use_particle_boundaries = 0, auto_frame = 0;
  // use_musl as the caller last set it: prepareSimulation turns MUSL on (simulation_units.cpp:
  // 185-186), simulate() keeps the field's own value (false by default, simulation.hpp:49)
  int use_musl_user = 0;
  double gravity[3] = {0, 0, 0};
  double pbmin[3] = {-5, -5, -5}, pbmax[3] = {5, 5, 5};
  double grid_ref[3] = {2e10, 2e10, 2e10};
};

// Minimal reader for a flat JSON object of numbers ({"key": number, ...}).
bool parse_flat_json(const std::string& text, std::map<std::string, double>& out) {
  size_t i = 0, n = text.size();
  auto ws = [&]() { while (i < n && std::isspace((unsigned char)text[i])) ++i; };
  ws();
  if (i >= n || text[i] != '{') return false;
  ++i;
  ws();
  if (i < n && text[i] == '}') return true;
  while (i < n) {
    ws();
    if (i >= n || text[i] != '"') return false;
    size_t j = text.find('"', i + 1);
    if (j == std::string::npos) return false;
    std::string key = text.substr(i + 1, j - i - 1);
    i = j + 1;
    ws();
    if (i >= n || text[i] != ':') return false;
    ++i;
    ws();
    const char* s = text.c_str() + i;
    char* e = nullptr;
    double v = std::strtod(s, &e);
    if (e == s) {
      if (text.compare(i, 4, "true") == 0) { v = 1; e = const_cast<char*>(s) + 4; }
      else if (text.compare(i, 5, "false") == 0) { v = 0; e = const_cast<char*>(s) + 5; }
      else return false;
    }
    i += (size_t)(e - s);
    out[key] = v;
    ws();
    if (i < n && text[i] == ',') { ++i; continue; }
    if (i < n && text[i] == '}') return true;
    return false;
  }
  return false;
}

}  // namespace

// Pinned host mirrors of the control blocks come from a process-wide pool: a page-locked
// allocation costs about a millisecond, a free slot of the pool nothing.  The pool grows by slabs
// of 16 portable pinned blocks, kept until the process exits.
namespace {
std::mutex g_ctrl_mu;
std::vector<Ctrl*> g_ctrl_free;
Ctrl* ctrl_mirror_get() {
  std::lock_guard<std::mutex> lock(g_ctrl_mu);
  if (g_ctrl_free.empty()) {
    void* slab = nullptr;
    if (cudaHostAlloc(&slab, 16 * sizeof(Ctrl), cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    for (int k = 15; k >= 0; --k) g_ctrl_free.push_back(static_cast<Ctrl*>(slab) + k);
  }
  Ctrl* c = g_ctrl_free.back();
  g_ctrl_free.pop_back();
  return c;
}
void ctrl_mirror_put(Ctrl* c) {
  std::lock_guard<std::mutex> lock(g_ctrl_mu);
  g_ctrl_free.push_back(c);
}
}  // namespace

struct pm_sim {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string name;
  HostParams hp;
  std::vector<PlateDev> plates;
  std::vector<ObjDev> objects;
  int knife = -1;
  std::vector<float> frames;
  int return_map = PM_RETURN_MAP_PLAIN;

  uint32_t np = 0;
  int np_stride = 0;
  float* d_pbuf[2] = {nullptr, nullptr};
  uint32_t* d_meta[2] = {nullptr, nullptr};
  int cur = 0;
  float* d_pic = nullptr;
  uint32_t *d_key = nullptr, *d_rank = nullptr, *d_sorted = nullptr;

  int brick_cap = 0;
  uint32_t regrowths = 0;   // grid reallocations so far
  double regrow_ms = 0.0;   // host time spent in them
  uint32_t* d_cell = nullptr;
  uint32_t* d_scan_part = nullptr;
  float4* d_grid = nullptr;
  float4* d_gmusl = nullptr;
  uint8_t* d_btouch = nullptr;
  uint32_t* d_blist = nullptr;  // 4 counts, then the occupied and touched brick lists

  Ctrl* d_ctrl = nullptr;
  Ctrl* h_ctrl = nullptr;  // pinned mirror
  float* d_frames = nullptr;
  float* d_unperm = nullptr;
  uint8_t* d_active = nullptr;
  double* d_stats = nullptr;
  void* d_mlp = nullptr;       // inference weights (bf16 matrices, FP32 biases and statistics)
  MlpDev mlp_dev{};
  bool has_mlp = false;
  int sur_fallback_plain = 0;
  float* d_slog = nullptr;     // return-map sample log: log_cap x 16 floats
  uint32_t log_cap = 0;
  uint32_t log_every = 1;
  SurQ* d_q = nullptr;         // surrogate queue (q_cap records + inputs and outputs)
  float* d_qx = nullptr;
  float* d_qy = nullptr;
  uint32_t q_cap = 0;

  bool prepared = false;
  uint32_t host_step = 0;  // steps completed (mirror of ctrl.step after the last sync)
  // host time spent allocating particle and grid buffers, and capturing and instantiating the
  // step graphs (pm_get_param "alloc_ms", "graph_ms": the fixed costs of a fresh simulation)
  double alloc_ms = 0.0, graph_ms = 0.0;
  Params P{};
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  bool graphs_dirty = true;
  // asynchronous particle readback: copies out of d_unperm run on their own stream
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_unperm = nullptr, ev_copied = nullptr;
  bool copy_pending = false;
  // pigment splat scratch (pass-1 grid, and the output grid of a host-buffer call), kept
  // between calls so that a renderer splatting every frame allocates once
  float* d_splat = nullptr;
  size_t splat_bytes = 0;
  // scratch of the density-grid and anisotropy passes, grown on demand
  void* d_render = nullptr;
  size_t render_bytes = 0;

  ~pm_sim();
  // Waits for an asynchronous readback still copying out of d_unperm / d_active.
  pm_status wait_copy() {
    if (!copy_pending) return PM_OK;
    copy_pending = false;
    const cudaError_t e = cudaEventSynchronize(ev_copied);
    return e == cudaSuccess ? PM_OK : fail(PM_ERR_CUDA, std::string("particle readback: ") + cudaGetErrorString(e));
  }
  void free_grid();
  void free_particles();
  pm_status alloc_grid(int bricks);
  void fill_params();
  Bufs bufs(int parity) const;
  pm_status sync_ctrl();
  pm_status push_ctrl();
  pm_status run_steps(uint32_t n, bool use_graph);
  pm_status capture_graphs();
  void drop_graphs();
  void free_surrogate_queue();
  pm_status ensure_surrogate_queue();
};

// ------------------------------------------------------------------------------------------
// Device memory of the particle and grid buffers comes from one stream-ordered pool per device
// that keeps freed memory for the process (release threshold unlimited), as a caching allocator
// does: a simulation created after another one has been destroyed (or has shrunk) takes its
// buffers from the pool instead of the driver, whose large allocations cost milliseconds per
// gigabyte.  pm_trim_memory returns the cached memory.
// ------------------------------------------------------------------------------------------
namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pool[64] = {};

cudaError_t pool_of(int device, cudaMemPool_t* out) {
  if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (!g_pool[device]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t p = nullptr;
    cudaError_t e = cudaMemPoolCreate(&p, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = UINT64_MAX;
    e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) { cudaMemPoolDestroy(p); return e; }
    g_pool[device] = p;
  }
  *out = g_pool[device];
  return cudaSuccess;
}

// Stream-ordered allocation from the device's pool (usable on `s` at once, on other streams once
// `s` has reached this point).
cudaError_t pool_alloc(void** ptr, size_t bytes, int device, cudaStream_t s) {
  cudaMemPool_t p = nullptr;
  cudaError_t e = pool_of(device, &p);
  if (e != cudaSuccess) return e;
  return cudaMallocFromPoolAsync(ptr, std::max<size_t>(bytes, 256), p, s);
}
template <class T> cudaError_t pool_alloc(T** ptr, size_t bytes, int device, cudaStream_t s) {
  return pool_alloc(reinterpret_cast<void**>(ptr), bytes, device, s);
}
}  // namespace

pm_sim::~pm_sim() {
  if (copy_pending) cudaEventSynchronize(ev_copied);
  if (ev_unperm) cudaEventDestroy(ev_unperm);
  if (ev_copied) cudaEventDestroy(ev_copied);
  if (copy_stream) cudaStreamDestroy(copy_stream);
  drop_graphs();
  free_particles();
  free_grid();
  if (d_ctrl) cudaFree(d_ctrl);  // also holds d_stats
  if (h_ctrl) ctrl_mirror_put(h_ctrl);
  if (d_frames) cudaFree(d_frames);
  if (d_mlp) cudaFree(d_mlp);
  if (d_slog) cudaFree(d_slog);
  if (d_splat) cudaFree(d_splat);
  if (d_render) cudaFree(d_render);
  free_surrogate_queue();
  if (stream) cudaStreamDestroy(stream);
}

void pm_sim::free_surrogate_queue() {
  if (d_q) cudaFree(d_q);
  if (d_qx) cudaFree(d_qx);
  if (d_qy) cudaFree(d_qy);
  d_q = nullptr; d_qx = nullptr; d_qy = nullptr;
  q_cap = 0;
}

pm_status pm_sim::ensure_surrogate_queue() {
  const uint32_t want = (uint32_t)std::max(np_stride, 32);
  if (q_cap >= want && d_q) return PM_OK;
  drop_graphs();
  free_surrogate_queue();
  CK(cudaMalloc(&d_q, (size_t)want * sizeof(SurQ)));
  CK(cudaMalloc(&d_qx, (size_t)want * 10 * sizeof(float)));
  CK(cudaMalloc(&d_qy, (size_t)want * 6 * sizeof(float)));
  q_cap = want;
  return PM_OK;
}

void pm_sim::drop_graphs() {
  for (int k = 0; k < 2; ++k)
    if (gexec[k]) { cudaGraphExecDestroy(gexec[k]); gexec[k] = nullptr; }
  graphs_dirty = true;
}

void pm_sim::free_grid() {
  for (void* p : {(void*)d_cell, (void*)d_scan_part, (void*)d_grid, (void*)d_gmusl, (void*)d_btouch, (void*)d_blist})
    if (p) cudaFreeAsync(p, stream);
  d_cell = nullptr; d_scan_part = nullptr; d_grid = nullptr; d_gmusl = nullptr; d_btouch = nullptr;
  d_blist = nullptr;
  brick_cap = 0;
}

void pm_sim::free_particles() {
  for (int k = 0; k < 2; ++k) {
    if (d_pbuf[k]) cudaFreeAsync(d_pbuf[k], stream);
    if (d_meta[k]) cudaFreeAsync(d_meta[k], stream);
    d_pbuf[k] = nullptr; d_meta[k] = nullptr;
  }
  for (void* p : {(void*)d_pic, (void*)d_key, (void*)d_rank, (void*)d_sorted, (void*)d_unperm, (void*)d_active})
    if (p) cudaFreeAsync(p, stream);
  d_pic = nullptr; d_key = d_rank = d_sorted = nullptr; d_unperm = nullptr; d_active = nullptr;
}

// Adds the host time of its scope to a millisecond counter.
struct ScopeMs {
  double& acc;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  explicit ScopeMs(double& a) : acc(a) {}
  ~ScopeMs() { acc += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); }
};

// Scan blocks (4096 cell counters, 64 bricks each) of a grid of the given brick capacity, plus one.
static size_t scan_blocks_alloc(int bricks) { return ((size_t)bricks * kBrickNodes + 1 + 4095) / 4096 + 1; }

pm_status pm_sim::alloc_grid(int bricks) {
  ScopeMs timer(alloc_ms);
  drop_graphs();
  free_grid();
  const size_t nodes = (size_t)bricks * kBrickNodes;
  if (nodes + 2 > 0x7fffffffULL) return fail(PM_ERR_CAPACITY, "grid capacity exceeds 2^31 nodes");
  CK(pool_alloc(&d_cell, (nodes + 2) * sizeof(uint32_t), device, stream));
  const size_t scan_blocks = scan_blocks_alloc(bricks);
  // per scan block: the partial sum, the count of occupied bricks, the 64-bit occupancy mask
  CK(pool_alloc(&d_scan_part, scan_blocks * 4 * sizeof(uint32_t), device, stream));
  CK(pool_alloc(&d_grid, nodes * 4 * sizeof(float4), device, stream));
  CK(pool_alloc(&d_gmusl, nodes * sizeof(float4), device, stream));
  // grid records need no zeroing here: each step zeroes the bricks it touches (k_clear_bricks)
  // and readers see only touched bricks
  CK(pool_alloc(&d_btouch, (size_t)bricks, device, stream));
  CK(cudaMemsetAsync(d_btouch, 0, (size_t)bricks, stream));
  CK(pool_alloc(&d_blist, (4 + 5 * (size_t)bricks) * sizeof(uint32_t), device, stream));
  CK(cudaMemsetAsync(d_blist, 0, 4 * sizeof(uint32_t), stream));
  CK(cudaStreamSynchronize(stream));  // the buffers are complete for every stream from here
  brick_cap = bricks;
  return PM_OK;
}

Bufs pm_sim::bufs(int parity) const {
  Bufs b{};
  b.pin = d_pbuf[parity];
  b.pout = d_pbuf[parity ^ 1];
  b.meta_in = d_meta[parity];
  b.meta_out = d_meta[parity ^ 1];
  b.pic = d_pic;
  b.key = d_key;
  b.rank = d_rank;
  b.sorted = d_sorted;
  b.cell = d_cell;
  b.scan_part = d_scan_part;
  b.scan_occ = d_scan_part ? d_scan_part + scan_blocks_alloc(brick_cap) : nullptr;
  b.occ_mask = d_scan_part ? reinterpret_cast<unsigned long long*>(d_scan_part + 2 * scan_blocks_alloc(brick_cap))
                           : nullptr;
  b.grid = d_grid;
  b.gmusl = d_gmusl;
  b.btouch = d_btouch;
  b.blist_n = d_blist;
  b.blist_occ = d_blist ? reinterpret_cast<uint4*>(d_blist + 4) : nullptr;
  b.blist_touch = d_blist ? d_blist + 4 + 4 * (size_t)brick_cap : nullptr;
  b.ctrl = d_ctrl;
  b.mlp = mlp_dev;
  b.slog = d_slog;
  b.q = d_q;
  b.qx = d_qx;
  b.qy = d_qy;
  return b;
}

void pm_sim::fill_params() {
  Params& p = P;
  const HostParams& h = hp;
  p.np = (int)np;
  p.np_stride = np_stride;
  p.dx = (float)h.dx;
  p.inv_dx = (float)(1.0 / h.dx);
  p.dx_d = h.dx;
  for (int d = 0; d < 3; ++d) {
    p.anchor_d[d] = h_ctrl->low_init[d];
    p.anchor[d] = (float)h_ctrl->low_init[d];
    p.gravity[d] = (float)h.gravity[d];
    p.pbmin[d] = (float)h.pbmin[d];
    p.pbmax[d] = (float)h.pbmax[d];
  }
  p.particle_mass = (float)h.particle_mass;
  p.particle_volume = (float)h.particle_volume;
  p.apicD = (float)(4.0 / (h.dx * h.dx));
  p.flip_ratio = (float)h.flip_ratio;
  p.use_musl = h.use_musl;
  p.use_particle_boundaries = h.use_particle_boundaries;
  // simulation_units.cpp:167-183
  p.lambda = h.nu * h.E / ((1.0 + h.nu) * (1.0 - 2.0 * h.nu));
  p.mu = h.E / (2.0 * (1.0 + h.nu));
  p.K = p.lambda + 2.0 * p.mu / 3.0;
  p.E = h.E;
  p.d_prefac = 1.0 / h.q_prefac;
  p.e_mu_prefac = 2.0 * h.q_prefac * p.mu;
  p.f_mu_prefac = 2.0 * h.q_prefac * h.q_prefac * p.mu;
  p.q_max = h.q_max; p.q_min = h.q_min; p.p_min = h.p_min; p.M = h.M; p.q_cohesion = h.q_cohesion;
  p.perzyna_exp = h.perzyna_exp; p.perzyna_visc = h.perzyna_visc; p.xi = h.xi;
  p.plastic_model = h.plastic_model;
  p.use_pradhana = h.use_pradhana;
  p.D_max = (float)h.D_max; p.D_edge0 = (float)h.D_edge0; p.D_edge1 = (float)h.D_edge1;
  p.start_boost = (float)h.start_boost; p.end_boost = (float)h.end_boost; p.boost_factor = (float)h.boost_factor;
  p.cfl = h.cfl;
  const double wave_speed = std::sqrt(h.E / h.rho);
  p.dt_max = h.cfl_elastic * h.dx / wave_speed;
  p.frame_dt = 1.0 / h.fps;
  p.min_dt = h.min_dt;
  p.final_time = h.end_frame * p.frame_dt;
  p.brick_cap = brick_cap;
  p.node_cap = brick_cap * kBrickNodes;
  p.frames = d_frames;
  p.n_frames = (int)(frames.size() / 7);
  p.return_map = (return_map == PM_RETURN_MAP_SURROGATE && has_mlp && d_q) ? 1 : 0;
  p.sur_fallback_plain = sur_fallback_plain;
  p.log_cap = d_slog ? log_cap : 0;
  p.log_every = log_every;
  p.q_cap = d_q ? q_cap : 0;
  graphs_dirty = true;
}

pm_status pm_sim::sync_ctrl() {
  CK(cudaMemcpyAsync(h_ctrl, d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  return PM_OK;
}
pm_status pm_sim::push_ctrl() {
  CK(cudaMemcpyAsync(d_ctrl, h_ctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, stream));
  CK(cudaStreamSynchronize(stream));
  return PM_OK;
}

pm_status pm_sim::capture_graphs() {
  ScopeMs timer(graph_ms);
  drop_graphs();
  for (int start = 0; start < 2; ++start) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    launch_step(P, bufs(start), stream, nullptr);
    launch_step(P, bufs(start ^ 1), stream, nullptr);
    cudaError_t e = cudaStreamEndCapture(stream, &g);
    if (e != cudaSuccess) return fail(PM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&gexec[start], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(PM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  }
  graphs_dirty = false;
  return PM_OK;
}

// Runs n steps in chunks of at most kChunkSteps, reading the control block after each chunk.
// The grid box is recomputed on the device every step; when a chunk ends with the box above
// kGrowAt of the capacity, the grid is regrown before the next chunk (and always after a
// capacity halt, which the device raises instead of writing out of bounds), so a halt wastes at
// most one chunk of no-op launches.
pm_status pm_sim::run_steps(uint32_t n, bool use_graph) {
  constexpr uint32_t kChunkSteps = 64;
  constexpr double kGrowAt = 0.8;
  uint32_t remaining = n;
  int guard = 0;
  while (remaining > 0) {
    const uint32_t before = host_step;
    const uint32_t chunk = std::min(remaining, kChunkSteps);
    uint32_t k = 0;
    if (use_graph && chunk >= 2) {
      if (graphs_dirty) { pm_status s = capture_graphs(); if (s != PM_OK) return s; }
      int par = cur;
      for (; k + 2 <= chunk; k += 2) CK(cudaGraphLaunch(gexec[par], stream));
    }
    int par = (cur + (int)k) & 1;
    for (; k < chunk; ++k) { launch_step(P, bufs(par), stream, nullptr); par ^= 1; }
    CK(cudaGetLastError());
    pm_status s = sync_ctrl();
    if (s != PM_OK) return s;
    const uint32_t done = h_ctrl->step - before;
    host_step = h_ctrl->step;
    cur = (cur + (int)done) & 1;
    remaining -= std::min(done, remaining);
    if (done > 0) guard = 0;  // count only regrowths that made no progress
    // a simulate() run ends with its last frame; the steps launched after it idled
    if (h_ctrl->stop_at_end && h_ctrl->frame >= h_ctrl->end_frame && !h_ctrl->halt) return PM_OK;
    if (done == 0 && !h_ctrl->halt)
      return fail(PM_ERR_STATE, "steps made no progress (the control block holds a batch target)");
    long long want = 0;
    if (h_ctrl->halt) {
      if (++guard > 8) return fail(PM_ERR_CAPACITY, "grid keeps overflowing after regrowth");
      want = (long long)h_ctrl->need_bricks * 2 + 64;
    } else if (remaining > 0 && h_ctrl->n_bricks > kGrowAt * brick_cap) {
      want = (long long)h_ctrl->n_bricks * 2 + 64;
    }
    if (want > 0) {
      if (want * kBrickNodes > 0x7ffffff0LL) return fail(PM_ERR_CAPACITY, "grid would exceed 2^31 nodes");
      const auto t0 = std::chrono::steady_clock::now();
      s = alloc_grid((int)want);
      if (s != PM_OK) return s;
      ++regrowths;
      regrow_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      fill_params();
      h_ctrl->halt = 0;
      h_ctrl->error_flags &= ~(uint32_t)E_CAPACITY;
      s = push_ctrl();
      if (s != PM_OK) return s;
    }
  }
  return PM_OK;
}

// ------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------
extern "C" {

const char* pm_last_error_message(void) { return g_err.c_str(); }

pm_status pm_create(int device, pm_sim** out) {
  if (!out) return fail(PM_ERR_INVALID, "out is NULL");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) return fail(PM_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
  if (device < 0 || device >= count) return fail(PM_ERR_INVALID, "device ordinal out of range");
  CK(cudaSetDevice(device));
  int major = 0;  // one attribute query (the full property query costs milliseconds)
  CK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
  if (major < 10) return fail(PM_ERR_UNSUPPORTED, "this library is built for sm_100a (B200) only");
  pm_sim* s = new pm_sim();
  s->device = device;
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) { delete s; return fail(PM_ERR_CUDA, "stream"); }
  // the control block and the statistics accumulators share one device allocation
  const size_t ctrl_bytes = (sizeof(Ctrl) + 255) / 256 * 256;
  if (cudaMalloc(&s->d_ctrl, ctrl_bytes + 16 * sizeof(double)) != cudaSuccess ||
      (s->h_ctrl = ctrl_mirror_get()) == nullptr) {
    delete s;
    return fail(PM_ERR_CUDA, "allocation of the control block failed");
  }
  s->d_stats = reinterpret_cast<double*>(reinterpret_cast<char*>(s->d_ctrl) + ctrl_bytes);
  std::memset(s->h_ctrl, 0, sizeof(Ctrl));
  s->h_ctrl->knife = -1;
  e = launch_init(device);
  if (e != cudaSuccess) { delete s; return fail(PM_ERR_CUDA, std::string("kernel set-up: ") + cudaGetErrorString(e)); }
  *out = s;
  return PM_OK;
}

pm_status pm_destroy(pm_sim* sim) {
  if (!sim) return PM_OK;
  cudaSetDevice(sim->device);
  if (sim->stream) cudaStreamSynchronize(sim->stream);
  delete sim;
  return PM_OK;
}

pm_status pm_trim_memory(int device, uint64_t keep_bytes) {
  cudaMemPool_t p = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (device < 0 || device >= 64) return fail(PM_ERR_INVALID, "device ordinal out of range");
    p = g_pool[device];
  }
  if (!p) return PM_OK;
  CK(cudaSetDevice(device));
  CK(cudaDeviceSynchronize());
  CK(cudaMemPoolTrimTo(p, (size_t)keep_bytes));
  return PM_OK;
}

pm_status pm_initialize_basic(pm_sim* sim, const char* name) {
  if (!sim) return fail(PM_ERR_INVALID, "sim is NULL");
  sim->name = name ? name : "";
  return PM_OK;
}

pm_status pm_set_param(pm_sim* sim, const char* name, double v) {
  if (!sim || !name) return fail(PM_ERR_INVALID, "NULL argument");
  HostParams& h = sim->hp;
  std::string k(name);
  bool ctrl_field = false;
  if (k == "fps") h.fps = v;
  else if (k == "cfl") h.cfl = v;
  else if (k == "cfl_elastic") h.cfl_elastic = v;
  else if (k == "flip_ratio") h.flip_ratio = v;
  else if (k == "rho") h.rho = v;
  else if (k == "E") h.E = v;
  else if (k == "nu") h.nu = v;
  else if (k == "min_dt") h.min_dt = v;
  else if (k == "dx") h.dx = v;
  else if (k == "particle_mass") h.particle_mass = v;
  else if (k == "particle_volume") h.particle_volume = v;
  else if (k == "q_max") h.q_max = v;
  else if (k == "q_min") h.q_min = v;
  else if (k == "p_min") h.p_min = v;
  else if (k == "M") h.M = v;
  else if (k == "q_cohesion") h.q_cohesion = v;
  else if (k == "perzyna_exp") h.perzyna_exp = v;
  else if (k == "perzyna_visc") h.perzyna_visc = v;
  else if (k == "xi") h.xi = v;
  else if (k == "q_prefac") h.q_prefac = v;
  else if (k == "pigment_D_max") h.D_max = v;
  else if (k == "pigment_D_edge0") h.D_edge0 = v;
  else if (k == "pigment_D_edge1") h.D_edge1 = v;
  else if (k == "start_boost_time") h.start_boost = v;
  else if (k == "end_boost_time") h.end_boost = v;
  else if (k == "boost_factor") h.boost_factor = v;
  else if (k == "use_pradhana") h.use_pradhana = v != 0;
  else if (k == "use_musl") h.use_musl = h.use_musl_user = v != 0;
  else if (k == "use_particle_boundaries") h.use_particle_boundaries = v != 0;
  else if (k == "plastic_model") {
    int m = (int)v;
    if (m != PM_NO_PLASTICITY && m != PM_VMVISC && m != PM_DPVISC)
      return fail(PM_ERR_UNSUPPORTED, "plastic_model: this path implements NoPlasticity, VMVisc and DPVisc");
    h.plastic_model = m;
  } else if (k == "end_frame") { h.end_frame = v; ctrl_field = true; }
  else if (k == "frame") { ctrl_field = true; }
  else if (k == "auto_frame") { h.auto_frame = v != 0; ctrl_field = true; }
  else if (k == "surrogate_fallback_plain") { sim->sur_fallback_plain = v != 0; }
  else if (k == "sample_log_every") {
    if (!(v >= 1.0 && v <= 1e6)) return fail(PM_ERR_INVALID, "sample_log_every must be in [1, 1e6]");
    sim->log_every = (uint32_t)v;
  } else return fail(PM_ERR_INVALID, "unknown parameter " + k);
  if (sim->prepared) {
    if (k == "dx") return fail(PM_ERR_STATE, "dx cannot change after prepare");
    if (ctrl_field) {
      pm_status s = sim->sync_ctrl();
      if (s != PM_OK) return s;
      if (k == "frame") sim->h_ctrl->frame = (uint32_t)v;
      if (k == "end_frame") sim->h_ctrl->end_frame = (uint32_t)v;
      if (k == "auto_frame") sim->h_ctrl->auto_frame = (uint32_t)(v != 0);
      s = sim->push_ctrl();
      if (s != PM_OK) return s;
    }
    sim->fill_params();
  }
  return PM_OK;
}

pm_status pm_get_param(pm_sim* sim, const char* name, double* out) {
  if (!sim || !name || !out) return fail(PM_ERR_INVALID, "NULL argument");
  const HostParams& h = sim->hp;
  std::string k(name);
  if (sim->prepared && (k == "time" || k == "dt" || k == "step" || k == "frame" || k == "n_active" ||
                        k == "plastic_count" || k == "grid_nodes")) {
    pm_status s = sim->sync_ctrl();
    if (s != PM_OK) return s;
  }
  const Ctrl* c = sim->h_ctrl;
  if (k == "time") *out = c->time;
  else if (k == "dt") *out = c->dt;
  else if (k == "step") *out = c->step;
  else if (k == "frame") *out = c->frame;
  else if (k == "n_active") *out = c->n_active;
  else if (k == "plastic_count") *out = c->plastic_count;
  else if (k == "grid_nodes") *out = c->n_nodes;
  else if (k == "kernels_per_step") *out = kernels_per_step(sim->P);
  else if (k == "regrowths") *out = sim->regrowths;
  else if (k == "regrow_ms") *out = sim->regrow_ms;
  else if (k == "grid_capacity_nodes") *out = (double)sim->brick_cap * kBrickNodes;
  else if (k == "surrogate_fallback_plain") *out = sim->sur_fallback_plain;
  else if (k == "sample_log_every") *out = sim->log_every;
  else if (k == "Np") *out = sim->np;
  else if (k == "fps") *out = h.fps;
  else if (k == "cfl") *out = h.cfl;
  else if (k == "cfl_elastic") *out = h.cfl_elastic;
  else if (k == "flip_ratio") *out = h.flip_ratio;
  else if (k == "rho") *out = h.rho;
  else if (k == "E") *out = h.E;
  else if (k == "nu") *out = h.nu;
  else if (k == "dx") *out = h.dx;
  else if (k == "particle_mass") *out = h.particle_mass;
  else if (k == "particle_volume") *out = h.particle_volume;
  else if (k == "M") *out = h.M;
  else if (k == "q_cohesion") *out = h.q_cohesion;
  else if (k == "perzyna_exp") *out = h.perzyna_exp;
  else if (k == "perzyna_visc") *out = h.perzyna_visc;
  else if (k == "q_max") *out = h.q_max;
  else if (k == "q_min") *out = h.q_min;
  else if (k == "q_prefac") *out = h.q_prefac;
  else if (k == "plastic_model") *out = h.plastic_model;
  else if (k == "use_musl") *out = h.use_musl;
  else if (k == "use_pradhana") *out = h.use_pradhana;
  else if (k == "end_frame") *out = h.end_frame;
  else if (k == "pigment_D_max") *out = h.D_max;
  else if (k == "pigment_D_edge0") *out = h.D_edge0;
  else if (k == "pigment_D_edge1") *out = h.D_edge1;
  else if (k == "start_boost_time") *out = h.start_boost;
  else if (k == "end_boost_time") *out = h.end_boost;
  else if (k == "boost_factor") *out = h.boost_factor;
  else if (k == "mu") *out = sim->P.mu;
  else if (k == "lambda") *out = sim->P.lambda;
  else if (k == "K") *out = sim->P.K;
  else if (k == "dt_max") *out = sim->P.dt_max;
  else if (k == "frame_dt") *out = sim->P.frame_dt;
  else if (k == "final_time") *out = sim->P.final_time;
  else if (k == "alloc_ms") *out = sim->alloc_ms;
  else if (k == "graph_ms") *out = sim->graph_ms;
  else return fail(PM_ERR_INVALID, "unknown parameter " + k);
  return PM_OK;
}

pm_status pm_set_param3(pm_sim* sim, const char* name, const double v[3]) {
  if (!sim || !name || !v) return fail(PM_ERR_INVALID, "NULL argument");
  std::string k(name);
  double* dst = nullptr;
  if (k == "gravity") dst = sim->hp.gravity;
  else if (k == "particle_boundary_min") dst = sim->hp.pbmin;
  else if (k == "particle_boundary_max") dst = sim->hp.pbmax;
  else if (k == "grid_reference_point") dst = sim->hp.grid_ref;
  else return fail(PM_ERR_INVALID, "unknown vector parameter " + k);
  for (int d = 0; d < 3; ++d) dst[d] = v[d];
  if (sim->prepared) sim->fill_params();
  return PM_OK;
}

static std::string read_file(const char* path, bool& ok) {
  std::ifstream f(path, std::ios::binary);
  ok = (bool)f;
  if (!ok) return std::string();
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

pm_status pm_load_pigment_config(pm_sim* sim, const char* path) {
  if (!sim || !path) return fail(PM_ERR_INVALID, "NULL argument");
  bool ok = false;
  std::string t = read_file(path, ok);
  if (!ok) return PM_OK;  // simulation_units.cpp:46-48: keep current values
  std::map<std::string, double> kv;
  if (!parse_flat_json(t, kv)) return fail(PM_ERR_IO, std::string("parse error in ") + path);
  auto get = [&](const char* key, double def) { auto it = kv.find(key); return it == kv.end() ? def : it->second; };
  HostParams& h = sim->hp;  // simulation_units.cpp:36-41
  h.D_max = get("D_max", 10e-2);
  h.D_edge0 = get("D_edge0", 0.5);
  h.D_edge1 = get("D_edge1", 0.8);
  h.start_boost = get("start_boost_time", 20.0);
  h.end_boost = get("end_boost_time", 40.0);
  h.boost_factor = get("boost_factor", 2.0);
  if (sim->prepared) sim->fill_params();
  return PM_OK;
}

static void sim_config_file_missing_defaults(HostParams& h) {  // simulation_units.cpp:69-80
  h.cfl = 0.2; h.flip_ratio = -0.8; h.E = 5e5; h.nu = 0.3; h.rho = 1000;
  h.M = std::tan(5.0 * M_PI / 180.0); h.q_cohesion = 500; h.perzyna_exp = 1.0; h.perzyna_visc = 0.1;
}

pm_status pm_load_sim_config(pm_sim* sim, const char* path) {
  if (!sim || !path) return fail(PM_ERR_INVALID, "NULL argument");
  bool ok = false;
  std::string t = read_file(path, ok);
  if (!ok) { sim_config_file_missing_defaults(sim->hp); return PM_OK; }
  std::map<std::string, double> kv;
  if (!parse_flat_json(t, kv)) return fail(PM_ERR_IO, std::string("parse error in ") + path);
  auto get = [&](const char* key, double def) { auto it = kv.find(key); return it == kv.end() ? def : it->second; };
  HostParams& h = sim->hp;  // simulation_units.cpp:55-64
  h.cfl = get("cfl", 0.2);
  h.flip_ratio = get("flip_ratio", -0.8);
  h.E = get("E", 500000.0);
  h.nu = get("nu", 0.3);
  h.rho = get("rho", 1000.0);
  h.M = std::tan(get("friction_angle", 5.0) * M_PI / 180.0);
  h.q_cohesion = get("q_cohesion", 500.0);
  h.perzyna_exp = get("perzyna_exp", 1.0);
  h.perzyna_visc = get("perzyna_visc", 0.1);
  if (sim->prepared) sim->fill_params();
  return PM_OK;
}

pm_status pm_set_particles(pm_sim* sim, uint32_t n, const float* x, const float* latent, const float* v) {
  if (sim) { pm_status w = sim->wait_copy(); if (w != PM_OK) return w; }
  if (!sim || (n > 0 && !x)) return fail(PM_ERR_INVALID, "NULL argument");
  if (n >= 0x7fffffffu) return fail(PM_ERR_CAPACITY, "too many particles");
  cudaSetDevice(sim->device);
  sim->drop_graphs();
  sim->free_particles();
  sim->free_surrogate_queue();
  sim->np = n;
  sim->np_stride = (int)((n + 31) / 32 * 32);
  const size_t S = (size_t)std::max(sim->np_stride, 32);
  // stage the host arrays on the device (d_unperm holds n*42 floats >= n*13) and scatter them
  // into the structure-of-arrays state there; the staging buffer comes first so that the copies
  // (asynchronous from pinned host memory) run while the other buffers are allocated
  CK(pool_alloc(&sim->d_unperm, (size_t)std::max(n, 1u) * F_COUNT * sizeof(float), sim->device, sim->stream));
  float* dx_ = sim->d_unperm;
  float* dl_ = dx_ + (size_t)n * 3;
  float* dv_ = dl_ + (size_t)n * 7;
  if (n > 0) {
    CK(cudaMemcpyAsync(dx_, x, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice, sim->stream));
    if (latent) CK(cudaMemcpyAsync(dl_, latent, (size_t)n * 7 * sizeof(float), cudaMemcpyHostToDevice, sim->stream));
    if (v) CK(cudaMemcpyAsync(dv_, v, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice, sim->stream));
  }
  {
    ScopeMs timer(sim->alloc_ms);
    const int dev = sim->device;
    cudaStream_t st = sim->stream;
    for (int k = 0; k < 2; ++k) {
      CK(pool_alloc(&sim->d_pbuf[k], S * F_COUNT * sizeof(float), dev, st));
      CK(pool_alloc(&sim->d_meta[k], S * sizeof(uint32_t), dev, st));
    }
    CK(pool_alloc(&sim->d_pic, S * 6 * sizeof(float), dev, st));
    CK(pool_alloc(&sim->d_key, S * sizeof(uint32_t), dev, st));
    CK(pool_alloc(&sim->d_rank, S * sizeof(uint32_t), dev, st));
    CK(pool_alloc(&sim->d_sorted, S * sizeof(uint32_t), dev, st));
    CK(pool_alloc(&sim->d_active, std::max(n, 1u), dev, st));
  }
  Params up{};
  up.np = (int)n;
  up.np_stride = (int)S;
  launch_upload(up, dx_, latent ? dl_ : nullptr, v ? dv_ : nullptr, sim->d_pbuf[0], sim->d_meta[0], sim->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(sim->stream));
  sim->cur = 0;
  sim->prepared = false;
  sim->host_step = 0;
  std::memset(sim->h_ctrl, 0, sizeof(Ctrl));
  sim->h_ctrl->knife = -1;
  return PM_OK;
}

pm_status pm_get_particles(pm_sim* sim, float* x, float* v, float* latent, float* diffusion, uint8_t* active, float* F,
                           float* Bm, float* plastic) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  const uint32_t n = sim->np;
  if (n == 0) return PM_OK;
  CK(cudaSetDevice(sim->device));
  pm_status w = sim->wait_copy();
  if (w != PM_OK) return w;
  Params p = sim->P;
  p.np = (int)n;
  p.np_stride = sim->np_stride;
  const uint32_t mask = (x ? kGrpX : 0u) | (v ? kGrpV : 0u) | (latent ? kGrpLat : 0u) | (diffusion ? kGrpDiff : 0u) |
                        (F ? kGrpF : 0u) | (Bm ? kGrpB : 0u) | (plastic ? kGrpPlastic : 0u);
  launch_unpermute(p, sim->d_pbuf[sim->cur], sim->d_meta[sim->cur], sim->d_unperm, sim->d_active, sim->stream, mask);
  CK(cudaGetLastError());
  auto fetch = [&](int f0, int nf, float* dst) -> pm_status {
    if (!dst) return PM_OK;
    CK(cudaMemcpyAsync(dst, sim->d_unperm + (size_t)f0 * n, (size_t)n * nf * sizeof(float), cudaMemcpyDeviceToHost,
                       sim->stream));
    return PM_OK;
  };
  pm_status s;
  if ((s = fetch(F_X, 3, x)) != PM_OK) return s;
  if ((s = fetch(F_V, 3, v)) != PM_OK) return s;
  if ((s = fetch(F_LAT, 7, latent)) != PM_OK) return s;
  if ((s = fetch(F_DIFF, 1, diffusion)) != PM_OK) return s;
  if ((s = fetch(F_F, 9, F)) != PM_OK) return s;
  if ((s = fetch(F_B, 9, Bm)) != PM_OK) return s;
  if ((s = fetch(F_EPD, 4, plastic)) != PM_OK) return s;
  if (active) CK(cudaMemcpyAsync(active, sim->d_active, n, cudaMemcpyDeviceToHost, sim->stream));
  CK(cudaStreamSynchronize(sim->stream));
  return PM_OK;
}

pm_status pm_get_particles_async(pm_sim* sim, float* x, float* v, float* latent, float* diffusion, uint8_t* active) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  const uint32_t n = sim->np;
  if (n == 0) return PM_OK;
  CK(cudaSetDevice(sim->device));
  pm_status w = sim->wait_copy();  // the previous readback still owns the staging buffer
  if (w != PM_OK) return w;
  if (!sim->copy_stream) {
    CK(cudaStreamCreateWithFlags(&sim->copy_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&sim->ev_unperm, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&sim->ev_copied, cudaEventDisableTiming));
  }
  Params p = sim->P;
  p.np = (int)n;
  p.np_stride = sim->np_stride;
  const uint32_t mask = (x ? kGrpX : 0u) | (v ? kGrpV : 0u) | (latent ? kGrpLat : 0u) | (diffusion ? kGrpDiff : 0u);
  // the unpermute runs on the step stream (ordered after the steps issued so far); the copies wait
  // for it on the copy stream, so steps issued next overlap them
  launch_unpermute(p, sim->d_pbuf[sim->cur], sim->d_meta[sim->cur], sim->d_unperm, sim->d_active, sim->stream, mask);
  CK(cudaGetLastError());
  CK(cudaEventRecord(sim->ev_unperm, sim->stream));
  CK(cudaStreamWaitEvent(sim->copy_stream, sim->ev_unperm, 0));
  auto fetch = [&](int f0, int nf, float* dst) -> pm_status {
    if (!dst) return PM_OK;
    CK(cudaMemcpyAsync(dst, sim->d_unperm + (size_t)f0 * n, (size_t)n * nf * sizeof(float), cudaMemcpyDeviceToHost,
                       sim->copy_stream));
    return PM_OK;
  };
  pm_status s;
  if ((s = fetch(F_X, 3, x)) != PM_OK) return s;
  if ((s = fetch(F_V, 3, v)) != PM_OK) return s;
  if ((s = fetch(F_LAT, 7, latent)) != PM_OK) return s;
  if ((s = fetch(F_DIFF, 1, diffusion)) != PM_OK) return s;
  if (active) CK(cudaMemcpyAsync(active, sim->d_active, n, cudaMemcpyDeviceToHost, sim->copy_stream));
  CK(cudaEventRecord(sim->ev_copied, sim->copy_stream));
  sim->copy_pending = true;
  return PM_OK;
}

pm_status pm_wait_particles(pm_sim* sim) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  CK(cudaSetDevice(sim->device));
  return sim->wait_copy();
}

pm_status pm_add_plate(pm_sim* sim, double pos, int plate_type, int bc, double friction, double pos_lower,
                       double pos_upper, double vx, double vy, double vz, double vmin_factor, double load_factor) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  if (plate_type < 0 || plate_type > 5) return fail(PM_ERR_INVALID, "plate_type");
  if (bc < 0 || bc > 2) return fail(PM_ERR_INVALID, "bc");
  if ((int)sim->plates.size() >= kMaxPlates) return fail(PM_ERR_CAPACITY, "too many plates");
  PlateDev p{};
  p.type = plate_type; p.bc = bc; p.friction = (float)friction;
  p.pos = pos; p.lower = pos_lower; p.upper = pos_upper;
  p.vx = p.vx0 = (float)vx; p.vy = p.vy0 = (float)vy; p.vz = p.vz0 = (float)vz;
  p.vmin_factor = (float)vmin_factor; p.load_factor = (float)load_factor;
  sim->plates.push_back(p);
  sim->prepared = false;
  return PM_OK;
}

static void pose_from(ObjDev& o, const double t[3], const double q[4]) {
  double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  double w = q[0] / n, x = q[1] / n, y = q[2] / n, z = q[3] / n;
  double R[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
                 2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                 2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)};
  double det = R[0] * (R[4] * R[8] - R[5] * R[7]) - R[1] * (R[3] * R[8] - R[5] * R[6]) + R[2] * (R[3] * R[7] - R[4] * R[6]);
  double inv[9] = {(R[4] * R[8] - R[5] * R[7]) / det, (R[2] * R[7] - R[1] * R[8]) / det, (R[1] * R[5] - R[2] * R[4]) / det,
                   (R[5] * R[6] - R[3] * R[8]) / det, (R[0] * R[8] - R[2] * R[6]) / det, (R[2] * R[3] - R[0] * R[5]) / det,
                   (R[3] * R[7] - R[4] * R[6]) / det, (R[1] * R[6] - R[0] * R[7]) / det, (R[0] * R[4] - R[1] * R[3]) / det};
  for (int k = 0; k < 9; ++k) o.Rinv[k] = (float)inv[k];
  for (int k = 0; k < 3; ++k) o.t[k] = t[k];
  for (int k = 0; k < 4; ++k) o.q[k] = q[k];
  o.tx = (float)t[0]; o.ty = (float)t[1]; o.tz = (float)t[2];
}

pm_status pm_add_spatula(pm_sim* sim, int bc, double friction, const float* frames, uint32_t n) {
  if (!sim || (n > 0 && !frames)) return fail(PM_ERR_INVALID, "NULL argument");
  if (bc < 0 || bc > 2) return fail(PM_ERR_INVALID, "bc");
  if ((int)sim->objects.size() >= kMaxObjects) return fail(PM_ERR_CAPACITY, "too many objects");
  ObjDev o{};
  o.kind = OBJ_SPATULA; o.bc = bc; o.friction = (float)friction;
  double t[3] = {0, 0, 0}, q[4] = {1, 0, 0, 0};
  if (n > 0) {
    for (int k = 0; k < 3; ++k) t[k] = frames[k];
    q[0] = frames[6]; q[1] = frames[3]; q[2] = frames[4]; q[3] = frames[5];
  }
  pose_from(o, t, q);
  sim->frames.assign(frames, frames + (size_t)n * 7);
  sim->objects.push_back(o);
  sim->knife = (int)sim->objects.size() - 1;
  sim->prepared = false;
  return PM_OK;
}

pm_status pm_add_spatula_file(pm_sim* sim, int bc, double friction, const char* anim_path) {
  if (!sim || !anim_path) return fail(PM_ERR_INVALID, "NULL argument");
  std::ifstream f(anim_path, std::ios::binary | std::ios::ate);
  if (!f) return fail(PM_ERR_IO, std::string("cannot open ") + anim_path);
  std::streamsize size = f.tellg();
  f.seekg(0, std::ios::beg);
  std::vector<float> buf((size_t)size / 28 * 7);
  if (!f.read(reinterpret_cast<char*>(buf.data()), (std::streamsize)(buf.size() * sizeof(float))))
    return fail(PM_ERR_IO, std::string("cannot read ") + anim_path);
  return pm_add_spatula(sim, bc, friction, buf.data(), (uint32_t)(buf.size() / 7));
}

pm_status pm_add_box_knife(pm_sim* sim, int bc, double friction, const double half[3], const double* waypoints,
                           uint32_t n, double speed, const double* quat_wxyz) {
  if (!sim || !half || (n > 0 && !waypoints)) return fail(PM_ERR_INVALID, "NULL argument");
  if (bc < 0 || bc > 2) return fail(PM_ERR_INVALID, "bc");
  if (n > (uint32_t)kMaxWaypoints) return fail(PM_ERR_CAPACITY, "too many waypoints");
  if ((int)sim->objects.size() >= kMaxObjects) return fail(PM_ERR_CAPACITY, "too many objects");
  ObjDev o{};
  o.kind = OBJ_BOXKNIFE; o.bc = bc; o.friction = (float)friction;
  for (int k = 0; k < 3; ++k) o.half[k] = (float)half[k];
  o.n_waypoints = (int)n;
  for (uint32_t i = 0; i < n * 3; ++i) o.waypoints[i] = (float)waypoints[i];
  o.speed = speed;
  o.s = 0;
  double t[3] = {0, 0, 0}, q[4] = {1, 0, 0, 0};
  if (n > 0) for (int k = 0; k < 3; ++k) t[k] = waypoints[k];
  if (quat_wxyz) for (int k = 0; k < 4; ++k) q[k] = quat_wxyz[k];
  pose_from(o, t, q);
  sim->objects.push_back(o);
  sim->knife = (int)sim->objects.size() - 1;
  sim->prepared = false;
  return PM_OK;
}

pm_status pm_add_ground(pm_sim* sim, int bc, double friction, double y0) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  if (bc < 0 || bc > 2) return fail(PM_ERR_INVALID, "bc");
  if ((int)sim->objects.size() >= kMaxObjects) return fail(PM_ERR_CAPACITY, "too many objects");
  ObjDev o{};
  o.kind = OBJ_GROUND; o.bc = bc; o.friction = (float)friction; o.y0 = (float)y0;
  double t[3] = {0, 0, 0}, q[4] = {1, 0, 0, 0};
  pose_from(o, t, q);
  sim->objects.push_back(o);
  sim->prepared = false;
  return PM_OK;
}

pm_status pm_add_curve(pm_sim* sim, int bc, double friction) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  if (bc < 0 || bc > 2) return fail(PM_ERR_INVALID, "bc");
  if ((int)sim->objects.size() >= kMaxObjects) return fail(PM_ERR_CAPACITY, "too many objects");
  ObjDev o{};
  o.kind = OBJ_CURVE; o.bc = bc; o.friction = (float)friction;
  double t[3] = {0, 0, 0}, q[4] = {1, 0, 0, 0};
  pose_from(o, t, q);
  sim->objects.push_back(o);
  sim->prepared = false;
  return PM_OK;
}

// Everything of setupScene after the particles exist (simulation_units.cpp:31-131 without blobs()).
static pm_status setup_scene_common(pm_sim* sim, float fps, const char* pigment_config_path,
                                    const char* sim_config_path, const char* anim_path) {
  pm_status s;
  if (pigment_config_path && (s = pm_load_pigment_config(sim, pigment_config_path)) != PM_OK) return s;
  if (sim_config_path && (s = pm_load_sim_config(sim, sim_config_path)) != PM_OK) return s;
  HostParams& h = sim->hp;  // simulation_units.cpp:82-130
  h.end_frame = 1800;
  h.fps = fps;
  h.gravity[0] = 0.0; h.gravity[1] = -9.81; h.gravity[2] = 0.0;
  h.use_particle_boundaries = 1;
  for (int d = 0; d < 3; ++d) { h.pbmin[d] = -2.0; h.pbmax[d] = 2.0; h.grid_ref[d] = 0.0; }
  if ((s = pm_add_plate(sim, 0.0, PM_PLATE_BOTTOM, PM_BC_SLIPSTICK, 1.0, -1e15, 1e15, 0, 0, 0, 1.0, 0.0)) != PM_OK) return s;
  if (anim_path && (s = pm_add_spatula_file(sim, PM_BC_SLIPFREE, 0.0, anim_path)) != PM_OK) return s;
  h.plastic_model = PM_DPVISC;
  h.use_pradhana = 1;
  h.q_prefac = 1.0 / std::sqrt(2.0);
  return PM_OK;
}

pm_status pm_setup_scene(pm_sim* sim, float fps, const char* pigment_config_path, const char* sim_config_path,
                         const char* anim_path) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  if (sim->np == 0) return fail(PM_ERR_STATE, "pm_setup_scene needs particles: call pm_set_particles first");
  return setup_scene_common(sim, fps, pigment_config_path, sim_config_path, anim_path);
}

// ---- Simulation::blobs (simulation_blobs.cpp:7-150) with analytic blobs -----------------------
// The reference morphs pairs of OpenVDB blob level sets to each colour's target volume and samples
// them with sampleParticlesFromVdb; here each blob is the upper half of a superellipsoid
// |dx/R|^p + |y/H|^p + |dz/R|^p <= 1 (p = 2.5, H = 0.55 R) of exactly the target volume, packed by
// the reference's touching arrangements and filled by Poisson-disk sampling of its bounding box.
namespace {
// Volumes of the reference's blob ladder (simulation.hpp:272-279, Blob_01 ... Blob_06).
constexpr double kBlobVolumes[6] = {0.0056, 0.0151, 0.0246, 0.0341, 0.0436, 0.053};
constexpr double kBlobAspect = 0.55, kBlobExp = 2.5;

// Colour ratio -> volume: the ratio clamped to [0.1, 0.9] mapped linearly onto the ladder's
// volume range (simulation_blobs.cpp:11-24).
double blob_volume(double ratio) {
  const double lo = kBlobVolumes[0], hi = kBlobVolumes[5];
  const double r = std::min(0.9, std::max(0.1, ratio));
  return std::min(hi, std::max(lo, lo + (r - 0.1) / 0.8 * (hi - lo)));
}

// Ground-plane offsets of touching blobs of packing radii r (simulation_blobs.cpp:63-116), centred
// on the x / z bounds of the arrangement with y = 0 (:118-140).
std::vector<std::array<double, 3>> blob_offsets(const std::vector<double>& r) {
  const size_t n = r.size();
  std::vector<std::array<double, 3>> o(n, std::array<double, 3>{0.0, 0.0, 0.0});
  auto cz = [](double d, double dist) { return std::sqrt(std::max(0.0, dist * dist - d * d)); };
  if (n == 2) {
    o[0][0] = -r[0]; o[1][0] = r[1];
  } else if (n == 3) {
    o[1][0] = r[0] + r[1];
    const double x1 = o[1][0];
    const double x2 = ((r[0] + r[2]) * (r[0] + r[2]) - (r[1] + r[2]) * (r[1] + r[2]) + x1 * x1) / (2.0 * x1);
    o[2][0] = x2;
    o[2][2] = cz(x2, r[0] + r[2]);
  } else if (n == 4) {
    o[0][0] = -r[0]; o[1][0] = r[1]; o[2][0] = -r[2]; o[3][0] = r[3];
    const double Z = std::max(std::max(cz(o[0][0] - o[2][0], r[0] + r[2]), cz(o[1][0] - o[3][0], r[1] + r[3])),
                              std::max(cz(o[0][0] - o[3][0], r[0] + r[3]), cz(o[1][0] - o[2][0], r[1] + r[2])));
    o[2][2] = o[3][2] = Z;
  } else if (n > 4) {
    double cur = 0.0;
    for (size_t i = 0; i < n; ++i) {
      if (i > 0) cur += r[i - 1] + r[i];
      o[i][0] = cur;
    }
  }
  if (n) {
    double lo[3], hi[3];
    for (int d = 0; d < 3; ++d) { lo[d] = o[0][d] - r[0]; hi[d] = o[0][d] + r[0]; }
    for (size_t i = 1; i < n; ++i)
      for (int d = 0; d < 3; ++d) { lo[d] = std::min(lo[d], o[i][d] - r[i]); hi[d] = std::max(hi[d], o[i][d] + r[i]); }
    for (size_t i = 0; i < n; ++i) {
      o[i][0] -= 0.5 * (lo[0] + hi[0]);
      o[i][2] -= 0.5 * (lo[2] + hi[2]);
    }
  }
  return o;
}
}  // namespace

pm_status pm_setup_scene_blobs(pm_sim* sim, float fps, const float* color_ratios, const float* latents, uint32_t k,
                               const char* pigment_config_path, const char* sim_config_path, const char* anim_path) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  if (k == 0 || !color_ratios || !latents) return fail(PM_ERR_INVALID, "need k >= 1 colour ratios and latents");
  if (k > 1024) return fail(PM_ERR_INVALID, "at most 1024 blobs");
  // the configuration first: the particle mass below uses its density
  pm_status s;
  if (pigment_config_path && (s = pm_load_pigment_config(sim, pigment_config_path)) != PM_OK) return s;
  if (sim_config_path && (s = pm_load_sim_config(sim, sim_config_path)) != PM_OK) return s;
  const double kv = 4.0 * kBlobAspect * std::pow(std::tgamma(1.0 + 1.0 / kBlobExp), 3) / std::tgamma(1.0 + 3.0 / kBlobExp);
  std::vector<double> R(k), H(k);
  for (uint32_t i = 0; i < k; ++i) {
    R[i] = std::cbrt(blob_volume((double)color_ratios[i]) / kv);  // V = kv R^3
    H[i] = kBlobAspect * R[i];
  }
  const auto off = blob_offsets(R);
  // sampleParticlesFromVdb (sampling_particles_vdb.hpp:87-150): radius 0.01, 27 particles per cell
  constexpr double kRadius = 0.01, kPpc = 27.0;
  std::vector<float> x, lat;
  double box_volume = 0.0;
  size_t box_samples = 0;
  for (uint32_t i = 0; i < k; ++i) {
    const double lo[3] = {off[i][0] - R[i], 0.0, off[i][2] - R[i]};
    const double L[3] = {2.0 * R[i], H[i], 2.0 * R[i]};
    uint32_t n = 0;
    if ((s = pm_sample_particles(sim->device, L[0], L[1], L[2], kRadius, kPpc, 0, 30, 2, 42 + i, nullptr, 0, &n,
                                 nullptr, nullptr)) != PM_OK)
      return s;
    std::vector<float> pts((size_t)n * 3);
    if ((s = pm_sample_particles(sim->device, L[0], L[1], L[2], kRadius, kPpc, 0, 30, 2, 42 + i, pts.data(), n, &n,
                                 nullptr, nullptr)) != PM_OK)
      return s;
    box_volume += L[0] * L[1] * L[2];
    box_samples += n;
    for (uint32_t j = 0; j < n; ++j) {
      double p[3], f = 0.0;
      for (int d = 0; d < 3; ++d) p[d] = (double)pts[3 * j + d] + lo[d];
      const double dxr = (p[0] - off[i][0]) / R[i], dy = p[1] / H[i], dzr = (p[2] - off[i][2]) / R[i];
      f = std::pow(std::fabs(dxr), kBlobExp) + std::pow(std::fabs(dy), kBlobExp) + std::pow(std::fabs(dzr), kBlobExp);
      if (!(f <= 1.0 && p[1] >= 0.0)) continue;
      for (int d = 0; d < 3; ++d) x.push_back((float)p[d]);
      for (int c = 0; c < 7; ++c) lat.push_back(latents[7 * i + c]);
    }
  }
  if (x.empty()) return fail(PM_ERR_INVALID, "the blobs hold no particles");
  const double dx = std::cbrt(kPpc / (double)box_samples * box_volume);
  if ((s = pm_set_particles(sim, (uint32_t)(x.size() / 3), x.data(), lat.data(), nullptr)) != PM_OK) return s;
  if ((s = setup_scene_common(sim, fps, nullptr, nullptr, anim_path)) != PM_OK) return s;
  HostParams& h = sim->hp;
  h.dx = dx;
  h.particle_volume = dx * dx * dx / kPpc;
  h.particle_mass = h.rho * h.particle_volume;
  return PM_OK;
}

pm_status pm_prepare(pm_sim* sim) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  if (sim->np == 0) return fail(PM_ERR_STATE, "no particles");
  HostParams& h = sim->hp;
  if (!(h.dx > 0) || !(h.particle_mass > 0) || !(h.particle_volume > 0))
    return fail(PM_ERR_INVALID, "dx, particle_mass and particle_volume must be positive");
  if (h.plastic_model != PM_NO_PLASTICITY && h.plastic_model != PM_VMVISC && h.plastic_model != PM_DPVISC)
    return fail(PM_ERR_UNSUPPORTED, "plastic model");
  CK(cudaSetDevice(sim->device));
  h.use_musl = 1;  // simulation_units.cpp:185-186
  // objects and keyframes
  if (sim->d_frames) { cudaFree(sim->d_frames); sim->d_frames = nullptr; }
  if (!sim->frames.empty()) {
    CK(cudaMalloc(&sim->d_frames, sim->frames.size() * sizeof(float)));
    CK(cudaMemcpy(sim->d_frames, sim->frames.data(), sim->frames.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  Ctrl* c = sim->h_ctrl;
  const bool first = sim->host_step == 0;
  if (first) {
    std::memset(c, 0, sizeof(Ctrl));
    c->n_plates = (int)sim->plates.size();
    for (int i = 0; i < c->n_plates; ++i) c->plates[i] = sim->plates[i];
    c->n_objects = (int)sim->objects.size();
    for (int i = 0; i < c->n_objects; ++i) c->objects[i] = sim->objects[i];
    c->knife = sim->knife;
  } else {
    pm_status s = sim->sync_ctrl();
    if (s != PM_OK) return s;
  }
  // initial reductions over the particles
  c->max_v2 = 0;
  for (int d = 0; d < 3; ++d) { c->xmin_key[d] = 0x7fffffff; c->xmax_key[d] = (int)0x80000000; }
  c->n_active = 0;
  pm_status s = sim->push_ctrl();
  if (s != PM_OK) return s;
  Params tmp{};
  tmp.np = (int)sim->np;
  tmp.np_stride = sim->np_stride;
  launch_reduce_state(tmp, sim->d_pbuf[sim->cur], sim->d_meta[sim->cur], sim->d_ctrl, sim->stream);
  CK(cudaGetLastError());
  if ((s = sim->sync_ctrl()) != PM_OK) return s;
  // remeshFixedInit(2,2,2) (remesh.cpp:45-180), only before the first step
  if (first) {
    double mn[3], mx[3];
    for (int d = 0; d < 3; ++d) {
      if (c->n_active == 0) { mn[d] = mx[d] = 0.0; }
      else { mn[d] = fkey_inv(c->xmin_key[d]); mx[d] = fkey_inv(c->xmax_key[d]); }
    }
    if (h.grid_ref[0] < 1e10) {
      for (int d = 0; d < 3; ++d) {
        if (h.grid_ref[d] < mn[d]) mn[d] = h.grid_ref[d];
        else if (h.grid_ref[d] > mx[d]) mx[d] = h.grid_ref[d];
      }
    }
    for (int d = 0; d < 3; ++d) {
      c->min_init[d] = mn[d]; c->max_init[d] = mx[d];
      c->low_init[d] = mn[d] - 2.0 * h.dx; c->high_init[d] = mx[d] + 2.0 * h.dx;
      c->low[d] = c->low_init[d]; c->high[d] = c->high_init[d];
    }
    c->time = 0; c->frame = 0; c->step = 0;
  } else {
    c->time = 0; c->frame = 0;  // prepareSimulation resets time and frame
  }
  c->end_frame = (uint32_t)h.end_frame;
  c->auto_frame = (uint32_t)h.auto_frame;
  // grid capacity from the initial box with headroom
  {
    long long nb = 1;
    for (int d = 0; d < 3; ++d) {
      double mn = c->n_active ? fkey_inv(c->xmin_key[d]) : c->low_init[d];
      double mx = c->n_active ? fkey_inv(c->xmax_key[d]) : c->low_init[d];
      long long n = (long long)std::ceil((mx - mn) / h.dx) + 8;
      n = (n + 3) / 4 + 1;
      nb *= n;
    }
    long long want = nb * 2 + 64;
    // With particle boundaries the grid box can never outgrow the boundary box: allocate that box
    // once (about 88 B per node) when it takes at most 1/8 of the free device memory, so long runs
    // never stop to regrow.
    if (h.use_particle_boundaries) {
      long long nbb = 1;
      for (int d = 0; d < 3; ++d) {
        const long long n = (long long)std::ceil((h.pbmax[d] - h.pbmin[d]) / h.dx) + 8;
        nbb *= (n + 3) / 4 + 1;
      }
      size_t free_b = 0, total_b = 0;
      if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && nbb > want &&
          (double)nbb * kBrickNodes * 88.0 <= 0.125 * (double)free_b)
        want = nbb;
    }
    if (want * kBrickNodes > 0x7ffffff0LL) want = 0x7ffffff0LL / kBrickNodes;
    if (sim->brick_cap < want) {
      if ((s = sim->alloc_grid((int)want)) != PM_OK) return s;
    }
  }
  if (sim->return_map == PM_RETURN_MAP_SURROGATE && (s = sim->ensure_surrogate_queue()) != PM_OK) return s;
  sim->prepared = true;
  sim->fill_params();
  if ((s = sim->push_ctrl()) != PM_OK) return s;
  return PM_OK;
}

pm_status pm_step(pm_sim* sim) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  if (!sim->prepared) return fail(PM_ERR_STATE, "call pm_prepare first");
  CK(cudaSetDevice(sim->device));
  // one reference step(): no frame bookkeeping even when auto_frame is set
  pm_status s;
  const uint32_t af = sim->h_ctrl->auto_frame;
  if (af) {
    if ((s = sim->sync_ctrl()) != PM_OK) return s;
    sim->h_ctrl->auto_frame = 0;
    if ((s = sim->push_ctrl()) != PM_OK) return s;
  }
  s = sim->run_steps(1, false);
  if (af) {
    sim->h_ctrl->auto_frame = af;
    pm_status s2 = sim->push_ctrl();
    if (s == PM_OK) s = s2;
  }
  return s;
}

pm_status pm_advance(pm_sim* sim, uint32_t nsteps, uint32_t* frames_done) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  if (!sim->prepared) return fail(PM_ERR_STATE, "call pm_prepare first");
  CK(cudaSetDevice(sim->device));
  pm_status s = sim->sync_ctrl();
  if (s != PM_OK) return s;
  const uint32_t fd0 = sim->h_ctrl->frames_done;
  const uint32_t af = sim->h_ctrl->auto_frame;
  if (!af) { sim->h_ctrl->auto_frame = 1; if ((s = sim->push_ctrl()) != PM_OK) return s; }
  s = sim->run_steps(nsteps, true);
  if (!af) { sim->h_ctrl->auto_frame = 0; pm_status s2 = sim->push_ctrl(); if (s == PM_OK) s = s2; }
  if (frames_done) *frames_done = sim->h_ctrl->frames_done - fd0;
  return s;
}

pm_status pm_simulate(pm_sim* sim, uint32_t max_steps, uint32_t* steps_done) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  if (steps_done) *steps_done = 0;
  const int musl = sim->hp.use_musl_user;
  pm_status s = pm_prepare(sim);  // material constants, the initial grid, time = frame = 0
  if (s != PM_OK) return s;
  sim->hp.use_musl = musl;
  sim->fill_params();
  Ctrl* c = sim->h_ctrl;
  const uint32_t step0 = c->step, af = c->auto_frame;
  c->auto_frame = 1;  // the loop's frame test after every step (simulation.cpp:184-193)
  c->stop_at_end = 1;
  if ((s = sim->push_ctrl()) != PM_OK) return s;
  s = sim->run_steps(max_steps ? max_steps : 0xffffffffu, true);
  pm_status s2 = sim->sync_ctrl();
  c->auto_frame = af;
  c->stop_at_end = 0;
  if (s2 == PM_OK) s2 = sim->push_ctrl();
  if (steps_done) *steps_done = c->step - step0;
  if (s != PM_OK) return s;
  if (s2 != PM_OK) return s2;
  if (c->frame < c->end_frame) return fail(PM_ERR_STATE, "simulate: max_steps reached before end_frame");
  return PM_OK;
}

pm_status pm_frame_finished(pm_sim* sim, int* finished) {
  if (!sim || !finished) return fail(PM_ERR_INVALID, "NULL argument");
  pm_status s = sim->sync_ctrl();
  if (s != PM_OK) return s;
  Ctrl* c = sim->h_ctrl;
  const double frame_dt = 1.0 / sim->hp.fps;
  *finished = 0;
  if (frame_dt * (double)(c->frame + 1) - c->time < sim->hp.min_dt * 1.1) {
    c->frame += 1;
    *finished = 1;
    return sim->push_ctrl();
  }
  return PM_OK;
}

pm_status pm_is_finished(pm_sim* sim, int* finished) {
  if (!sim || !finished) return fail(PM_ERR_INVALID, "NULL argument");
  pm_status s = sim->sync_ctrl();
  if (s != PM_OK) return s;
  const double final_time = sim->hp.end_frame / sim->hp.fps;
  *finished = (sim->h_ctrl->frame >= (uint32_t)sim->hp.end_frame || sim->h_ctrl->time >= final_time) ? 1 : 0;
  return PM_OK;
}

pm_status pm_get_grid_boundaries(pm_sim* sim, double lo[3], double hi[3]) {
  if (!sim || !lo || !hi) return fail(PM_ERR_INVALID, "NULL argument");
  if (sim->prepared) { pm_status s = sim->sync_ctrl(); if (s != PM_OK) return s; }
  for (int d = 0; d < 3; ++d) { lo[d] = sim->h_ctrl->low[d]; hi[d] = sim->h_ctrl->high[d]; }
  return PM_OK;
}

pm_status pm_get_knife(pm_sim* sim, int* exists, double inv[16], double half_dims[3]) {
  if (!sim || !exists) return fail(PM_ERR_INVALID, "NULL argument");
  *exists = 0;
  if (sim->knife < 0) return PM_OK;
  const ObjDev* o = &sim->objects[sim->knife];
  if (sim->prepared) {
    pm_status s = sim->sync_ctrl();
    if (s != PM_OK) return s;
    o = &sim->h_ctrl->objects[sim->knife];
  }
  *exists = 1;
  if (inv) {
    double R[9];
    for (int k = 0; k < 9; ++k) R[k] = o->Rinv[k];
    for (int r = 0; r < 3; ++r) {
      for (int q = 0; q < 3; ++q) inv[4 * r + q] = R[3 * r + q];
      inv[4 * r + 3] = -(R[3 * r] * o->t[0] + R[3 * r + 1] * o->t[1] + R[3 * r + 2] * o->t[2]);
    }
    inv[12] = inv[13] = inv[14] = 0; inv[15] = 1;
  }
  if (half_dims) {  // MPMIntegrationSim.cpp:161-168: (halfWidth, halfThickness, halfLength)
    if (o->kind == OBJ_SPATULA) { half_dims[0] = 0.368; half_dims[1] = 0.07; half_dims[2] = 0.736; }
    else for (int k = 0; k < 3; ++k) half_dims[k] = o->half[k];
  }
  return PM_OK;
}

pm_status pm_get_error_flags(pm_sim* sim, uint32_t* flags, int clear) {
  if (!sim || !flags) return fail(PM_ERR_INVALID, "NULL argument");
  pm_status s = sim->sync_ctrl();
  if (s != PM_OK) return s;
  *flags = sim->h_ctrl->error_flags;
  if (clear) { sim->h_ctrl->error_flags = 0; return sim->push_ctrl(); }
  return PM_OK;
}

pm_status pm_get_stats(pm_sim* sim, double* total_mass, double momentum[3], double mean_latent[7], uint32_t* n_active) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  if (sim->np == 0) return PM_OK;
  CK(cudaSetDevice(sim->device));
  CK(cudaMemsetAsync(sim->d_stats, 0, 16 * sizeof(double), sim->stream));
  Params p = sim->P;
  p.np = (int)sim->np;
  p.np_stride = sim->np_stride;
  launch_stats(p, sim->d_pbuf[sim->cur], sim->d_meta[sim->cur], sim->d_stats, sim->stream);
  CK(cudaGetLastError());
  double h[16];
  CK(cudaMemcpyAsync(h, sim->d_stats, sizeof(h), cudaMemcpyDeviceToHost, sim->stream));
  CK(cudaStreamSynchronize(sim->stream));
  const double mp = sim->hp.particle_mass;
  if (total_mass) *total_mass = h[0] * mp;
  if (momentum) for (int d = 0; d < 3; ++d) momentum[d] = h[1 + d] * mp;
  if (mean_latent) for (int k = 0; k < 7; ++k) mean_latent[k] = h[0] > 0 ? h[4 + k] / h[0] : 0.0;
  if (n_active) *n_active = (uint32_t)h[0];
  return PM_OK;
}

pm_status pm_sample_latent_cylinder(pm_sim* sim, double cx, double cz, double radius, double mean_latent[7],
                                    uint32_t* count) {
  if (!sim || !mean_latent) return fail(PM_ERR_INVALID, "NULL argument");
  for (int k = 0; k < 7; ++k) mean_latent[k] = 0.0;
  if (count) *count = 0;
  if (sim->np == 0) return PM_OK;
  CK(cudaSetDevice(sim->device));
  CK(cudaMemsetAsync(sim->d_stats, 0, 16 * sizeof(double), sim->stream));
  Params p = sim->P;
  p.np = (int)sim->np;
  p.np_stride = sim->np_stride;
  launch_stats(p, sim->d_pbuf[sim->cur], sim->d_meta[sim->cur], sim->d_stats, sim->stream, 1, (float)cx, (float)cz,
               (float)(radius * radius));
  CK(cudaGetLastError());
  double h[16];
  CK(cudaMemcpyAsync(h, sim->d_stats, sizeof(h), cudaMemcpyDeviceToHost, sim->stream));
  CK(cudaStreamSynchronize(sim->stream));
  if (h[0] > 0) for (int k = 0; k < 7; ++k) mean_latent[k] = h[4 + k] / h[0];
  if (count) *count = (uint32_t)h[0];
  return PM_OK;
}

pm_status pm_get_grid(pm_sim* sim, double origin[3], uint32_t dims[3], float* mass, float* v_update, float* v_musl,
                      float* flip, float* latent, float* shear) {
  if (!sim || !origin || !dims) return fail(PM_ERR_INVALID, "NULL argument");
  if (!sim->prepared) return fail(PM_ERR_STATE, "not prepared");
  pm_status s = sim->sync_ctrl();
  if (s != PM_OK) return s;
  const Ctrl* c = sim->h_ctrl;
  for (int d = 0; d < 3; ++d) {
    origin[d] = sim->P.anchor_d[d] + (double)c->g0[d] * sim->hp.dx;
    dims[d] = (uint32_t)c->dims[d];
  }
  if (!mass && !v_update && !v_musl && !flip && !latent && !shear) return PM_OK;
  const size_t nn = (size_t)c->n_nodes;
  std::vector<float4> g(nn * 4), m(nn);
  std::vector<uint8_t> touched(nn / kBrickNodes);
  CK(cudaMemcpyAsync(g.data(), sim->d_grid, nn * 4 * sizeof(float4), cudaMemcpyDeviceToHost, sim->stream));
  CK(cudaMemcpyAsync(m.data(), sim->d_gmusl, nn * sizeof(float4), cudaMemcpyDeviceToHost, sim->stream));
  CK(cudaMemcpyAsync(touched.data(), sim->d_btouch, touched.size(), cudaMemcpyDeviceToHost, sim->stream));
  CK(cudaStreamSynchronize(sim->stream));
  // bricks that no particle stencil reached this step hold stale records: report them empty
  for (size_t b = 0; b < touched.size(); ++b)
    if (!touched[b])
      for (size_t n = b * kBrickNodes; n < (b + 1) * kBrickNodes; ++n) {
        for (int q = 0; q < 4; ++q) g[n * 4 + q] = make_float4(0.f, 0.f, 0.f, 0.f);
        m[n] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
  for (int i = 0; i < c->dims[0]; ++i)
    for (int j = 0; j < c->dims[1]; ++j)
      for (int k = 0; k < c->dims[2]; ++k) {
        const size_t l = ((size_t)i * c->dims[1] + j) * c->dims[2] + k;
        const size_t b = ((size_t)(i >> 2) * c->nb[1] + (j >> 2)) * c->nb[2] + (k >> 2);
        const size_t n = b * kBrickNodes + (i & 3) * 16 + (j & 3) * 4 + (k & 3);
        // updated record: [v xyz, lat0 | lat1..lat4 | lat5, lat6, shear, mass | flip xyz, -]
        const float4 r0 = g[n * 4], r1 = g[n * 4 + 1], r2 = g[n * 4 + 2], r3 = g[n * 4 + 3];
        const bool has = r2.w > 0.f;
        if (mass) mass[l] = has ? r2.w : 0.f;
        if (v_update) { v_update[3 * l] = has ? r0.x : 0.f; v_update[3 * l + 1] = has ? r0.y : 0.f; v_update[3 * l + 2] = has ? r0.z : 0.f; }
        if (flip) { flip[3 * l] = has ? r3.x : 0.f; flip[3 * l + 1] = has ? r3.y : 0.f; flip[3 * l + 2] = has ? r3.z : 0.f; }
        if (latent) {
          const float lv[7] = {r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y};
          for (int q = 0; q < 7; ++q) latent[7 * l + q] = has ? lv[q] : 0.f;
        }
        if (shear) shear[l] = has ? r2.z : 0.f;
        if (v_musl) {
          const float4 mm = m[n];
          const float inv = mm.w > 0.f ? 1.f / mm.w : 0.f;
          v_musl[3 * l] = mm.x * inv; v_musl[3 * l + 1] = mm.y * inv; v_musl[3 * l + 2] = mm.z * inv;
        }
      }
  return PM_OK;
}

pm_status pm_set_return_map(pm_sim* sim, int mode) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  if (mode != PM_RETURN_MAP_PLAIN && mode != PM_RETURN_MAP_SURROGATE) return fail(PM_ERR_INVALID, "mode");
  if (mode == PM_RETURN_MAP_SURROGATE && !sim->has_mlp) return fail(PM_ERR_STATE, "no surrogate weights loaded");
  CK(cudaSetDevice(sim->device));
  sim->return_map = mode;
  if (mode == PM_RETURN_MAP_SURROGATE && sim->np > 0) {
    pm_status s = sim->ensure_surrogate_queue();
    if (s != PM_OK) return s;
  }
  if (sim->prepared) sim->fill_params();
  return PM_OK;
}

pm_status pm_set_surrogate(pm_sim* sim, const float* params) {
  if (!sim || !params) return fail(PM_ERR_INVALID, "NULL argument");
  CK(cudaSetDevice(sim->device));
  CK(mlp_upload(params, sim->mlp_dev, &sim->d_mlp));
  sim->has_mlp = true;
  sim->drop_graphs();
  if (sim->prepared) sim->fill_params();
  return PM_OK;
}

pm_status pm_enable_sample_log(pm_sim* sim, uint32_t capacity) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  CK(cudaSetDevice(sim->device));
  sim->drop_graphs();
  if (sim->d_slog) { cudaFree(sim->d_slog); sim->d_slog = nullptr; }
  sim->log_cap = 0;
  if (capacity > 0) {
    CK(cudaMalloc(&sim->d_slog, (size_t)capacity * 16 * sizeof(float)));
    sim->log_cap = capacity;
  }
  if (sim->prepared) {
    pm_status s = sim->sync_ctrl();
    if (s != PM_OK) return s;
    sim->h_ctrl->slog_n = 0;
    if ((s = sim->push_ctrl()) != PM_OK) return s;
    sim->fill_params();
  } else {
    sim->h_ctrl->slog_n = 0;
  }
  return PM_OK;
}

pm_status pm_get_samples(pm_sim* sim, float* features, float* targets, uint32_t max_samples, uint32_t* n) {
  if (!sim || !n) return fail(PM_ERR_INVALID, "NULL argument");
  *n = 0;
  if (!sim->d_slog) return PM_OK;
  pm_status s = sim->sync_ctrl();
  if (s != PM_OK) return s;
  const uint32_t have = std::min(sim->h_ctrl->slog_n, sim->log_cap);
  const uint32_t m = std::min(have, max_samples);
  if (m > 0 && (features || targets)) {
    std::vector<float> tmp((size_t)m * 16);
    CK(cudaMemcpy(tmp.data(), sim->d_slog, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost));
    for (uint32_t r = 0; r < m; ++r) {
      if (features) std::memcpy(features + (size_t)r * 10, &tmp[(size_t)r * 16], 10 * sizeof(float));
      if (targets) std::memcpy(targets + (size_t)r * 6, &tmp[(size_t)r * 16 + 10], 6 * sizeof(float));
    }
  }
  *n = m;
  return PM_OK;
}

pm_status pm_get_return_map_stats(pm_sim* sim, uint32_t stats[5]) {
  if (!sim || !stats) return fail(PM_ERR_INVALID, "NULL argument");
  pm_status s = sim->sync_ctrl();
  if (s != PM_OK) return s;
  const Ctrl* c = sim->h_ctrl;
  stats[0] = c->newton_solves;
  stats[1] = c->newton_iters;
  stats[2] = c->q_n;
  stats[3] = c->sur_accept;
  stats[4] = c->slog_n;
  return PM_OK;
}

pm_status pm_mlp_loss_grad(const float* params, const float* x, const float* y, uint32_t n, float* loss, float* grad) {
  if (!params || !x || !y || !loss || n == 0) return fail(PM_ERR_INVALID, "NULL argument or empty batch");
  CK(mlp_loss_grad(params, x, y, (int)n, loss, grad));
  return PM_OK;
}

pm_status pm_mlp_train(const float* x, const float* y, uint32_t n, uint32_t epochs, uint32_t batch, float lr,
                       uint64_t seed, int resume, float* params, float* loss_history, uint32_t* steps) {
  if (!x || !y || !params || n == 0) return fail(PM_ERR_INVALID, "NULL argument or empty training set");
  pm_mlp_train_opts o{(int)epochs, (int)batch, lr, seed, resume};
  int st = 0;
  CK(mlp_train(x, y, (int)n, o, params, loss_history, &st));
  if (steps) *steps = (uint32_t)st;
  return PM_OK;
}

pm_status pm_mlp_infer(const float* params, const float* x, uint32_t n, float* y) {
  if (!params || !x || !y) return fail(PM_ERR_INVALID, "NULL argument");
  if (n == 0) return PM_OK;
  void* storage = nullptr;
  MlpDev dev{};
  float* dX = nullptr;
  float* dY = nullptr;
  cudaError_t e = mlp_upload(params, dev, &storage);
  if (e == cudaSuccess) e = cudaMalloc(&dX, (size_t)n * 10 * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dY, (size_t)n * 6 * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(dX, x, (size_t)n * 10 * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = mlp_init();
  if (e == cudaSuccess) e = mlp_infer(dev, dX, dY, (int)n, nullptr, 0, 0);
  if (e == cudaSuccess) e = cudaMemcpy(y, dY, (size_t)n * 6 * sizeof(float), cudaMemcpyDeviceToHost);
  if (dX) cudaFree(dX);
  if (dY) cudaFree(dY);
  if (storage) cudaFree(storage);
  if (e != cudaSuccess) return fail(PM_ERR_CUDA, std::string("pm_mlp_infer: ") + cudaGetErrorString(e));
  return PM_OK;
}

pm_status pm_get_stream(pm_sim* sim, void** stream) {
  if (!sim || !stream) return fail(PM_ERR_INVALID, "NULL argument");
  *stream = (void*)sim->stream;
  return PM_OK;
}

const char* pm_kernel_name(pm_sim* sim, int index) { return sim ? kernel_name(index, sim->P) : ""; }

pm_status pm_profile_steps(pm_sim* sim, uint32_t nsteps, float* kernel_ms, uint32_t n_kernels) {
  if (!sim || !kernel_ms) return fail(PM_ERR_INVALID, "NULL argument");
  if (!sim->prepared) return fail(PM_ERR_STATE, "call pm_prepare first");
  const int K = kernels_per_step(sim->P);
  if ((int)n_kernels < K) return fail(PM_ERR_INVALID, "kernel_ms needs kernels_per_step entries");
  CK(cudaSetDevice(sim->device));
  // the steps of pm_advance (frame bookkeeping after every step): without it dt would be clipped
  // to min_dt once the run passes a frame boundary that nothing marks finished
  pm_status st = sim->sync_ctrl();
  if (st != PM_OK) return st;
  const uint32_t af = sim->h_ctrl->auto_frame;
  if (!af) { sim->h_ctrl->auto_frame = 1; if ((st = sim->push_ctrl()) != PM_OK) return st; }
  std::vector<cudaEvent_t> ev(K + 1);
  for (auto& e : ev) CK(cudaEventCreate(&e));
  std::vector<double> acc(K, 0.0);
  uint32_t done_steps = 0;
  for (uint32_t k = 0; k < nsteps && st == PM_OK; ++k) {
    launch_step(sim->P, sim->bufs(sim->cur), sim->stream, ev.data());
    if (cudaStreamSynchronize(sim->stream) != cudaSuccess) { st = fail(PM_ERR_CUDA, "profiled step failed"); break; }
    for (int i = 0; i < K; ++i) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
      acc[i] += ms;
    }
    st = sim->sync_ctrl();
    if (st != PM_OK) break;
    if (sim->h_ctrl->halt) { st = fail(PM_ERR_CAPACITY, "grid capacity reached while profiling"); break; }
    sim->host_step = sim->h_ctrl->step;
    sim->cur ^= 1;
    ++done_steps;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (int i = 0; i < K; ++i) kernel_ms[i] = done_steps ? (float)(acc[i] / done_steps) : 0.f;
  if (!af) {
    pm_status s2 = sim->sync_ctrl();
    if (s2 == PM_OK) { sim->h_ctrl->auto_frame = 0; s2 = sim->push_ctrl(); }
    if (st == PM_OK) st = s2;
  }
  return st;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// batched scenes
// ------------------------------------------------------------------------------------------
struct pm_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<pm_sim*> sims;
  std::vector<SceneDev> h_sd;
  SceneDev* d_sd = nullptr;
  std::vector<int> h_off;
  int* d_off = nullptr;
  std::vector<uint32_t> par_base, target, auto_frame;
  BatchLaunch L;
  pm_batch_tuning tune{};
  int occ_p2g = 1, occ_g2p = 1, occ_def = 1;
  cudaGraphExec_t gexec = nullptr;
  bool graph_dirty = true;

  ~pm_batch() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (d_sd) cudaFree(d_sd);
    if (d_off) cudaFree(d_off);
    if (stream) cudaStreamDestroy(stream);
  }
  int ns() const { return (int)sims.size(); }
  pm_status upload_tables();
  pm_status capture();
  pm_status begin(uint32_t nsteps);
  pm_status poll(bool& all_done, bool& progress, bool allow_regrow);
  pm_status finish();
  pm_status run_rounds(uint32_t n);
};

namespace {
// Splits `total` CTAs over the scenes in proportion to w (at least one each); returns offsets.
void proportional(const std::vector<double>& w, int total, std::vector<int>& off) {
  const int n = (int)w.size();
  double sum = 0.0;
  for (double x : w) sum += x;
  off.assign(n + 1, 0);
  for (int s = 0; s < n; ++s) {
    const int c = std::max(1, (int)std::lround(sum > 0.0 ? total * w[s] / sum : (double)total / n));
    off[s + 1] = off[s] + c;
  }
}
}  // namespace

// Rebuilds the scene table (constants and buffers of both parities) and the CTA partitions,
// uploads them, and marks the graph for recapture when a launch size changed.
pm_status pm_batch::upload_tables() {
  const int n = ns();
  const int sms = num_sms() > 0 ? num_sms() : 148;
  h_sd.assign(n, SceneDev{});
  std::vector<double> wp(n), wn(n);
  std::vector<int> scan(n + 1, 0);
  bool sur = false;
  for (int s = 0; s < n; ++s) {
    pm_sim* m = sims[s];
    m->fill_params();
    h_sd[s].P = m->P;
    h_sd[s].B[0] = m->bufs(0);
    h_sd[s].B[1] = m->bufs(1);
    h_sd[s].par_base = par_base[s];
    wp[s] = (double)std::max<uint32_t>(m->np, 1);
    wn[s] = (double)std::max(m->P.node_cap, 1);
    scan[s + 1] = scan[s] + scan_ctas_for(m->P.node_cap, 16);
    sur = sur || m->P.return_map == 1;
  }
  std::vector<int> unit(n + 1), part, node, p2g, g2p, def, surv;
  for (int s = 0; s <= n; ++s) unit[s] = s;
  proportional(wp, sms * tune.part_ctas_per_sm, part);
  proportional(wn, sms * tune.node_ctas_per_sm, node);
  proportional(wp, sms * tune.p2g_ctas_per_sm, p2g);
  proportional(wp, sms * tune.g2p_ctas_per_sm, g2p);
  proportional(wp, sms * tune.def_ctas_per_sm, def);
  proportional(wp, sms * tune.sur_ctas_per_sm, surv);
  const std::vector<int>* tabs[] = {&unit, &part, &node, &scan, &p2g, &g2p, &def, &surv};
  h_off.clear();
  for (auto* t : tabs) h_off.insert(h_off.end(), t->begin(), t->end());
  if (!d_sd) CK(cudaMalloc(&d_sd, sizeof(SceneDev) * (size_t)n));
  if (!d_off) CK(cudaMalloc(&d_off, sizeof(int) * 8 * (size_t)(n + 1)));
  CK(cudaMemcpyAsync(d_sd, h_sd.data(), sizeof(SceneDev) * (size_t)n, cudaMemcpyHostToDevice, stream));
  CK(cudaMemcpyAsync(d_off, h_off.data(), sizeof(int) * h_off.size(), cudaMemcpyHostToDevice, stream));
  CK(cudaStreamSynchronize(stream));
  BatchLaunch nl;
  nl.sd = d_sd;
  nl.ns = n;
  const int* o = d_off;
  nl.off_unit = o; o += n + 1;
  nl.off_part = o; o += n + 1;
  nl.off_node = o; o += n + 1;
  nl.off_scan = o; o += n + 1;
  nl.off_p2g = o; o += n + 1;
  nl.off_g2p = o; o += n + 1;
  nl.off_def = o; o += n + 1;
  nl.off_sur = o;
  nl.n_part = part[n]; nl.n_node = node[n]; nl.n_scan = scan[n]; nl.n_p2g = p2g[n];
  nl.n_g2p = g2p[n]; nl.n_def = def[n]; nl.n_sur = surv[n];
  nl.flat_threads = tune.flat_threads;
  nl.surrogate = sur;
  // one plain-solver instantiation of the deformation update when every scene shares the model
  nl.g2p_flip = false;
  for (int s = 0; s < n; ++s) nl.g2p_flip = nl.g2p_flip || h_sd[s].P.flip_ratio >= -1.f;
  nl.defgrad_model = h_sd[0].P.plastic_model;
  for (int s = 0; s < n; ++s) {
    const Params& q = h_sd[s].P;
    if (q.plastic_model != nl.defgrad_model || q.return_map == 1 || q.log_cap > 0) nl.defgrad_model = -1;
  }
  if (std::memcmp(&nl, &L, sizeof(BatchLaunch)) != 0) graph_dirty = true;
  L = nl;
  return PM_OK;
}

pm_status pm_batch::capture() {
  if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
  launch_step_batched(L, stream, nullptr);
  cudaError_t e = cudaStreamEndCapture(stream, &g);
  if (e != cudaSuccess) return fail(PM_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(PM_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(e));
  graph_dirty = false;
  return PM_OK;
}

// Sets every scene's target to its current step + nsteps and records its buffer parity.
pm_status pm_batch::begin(uint32_t nsteps) {
  CK(cudaSetDevice(device));
  const int n = ns();
  par_base.assign(n, 0);
  target.assign(n, 0);
  auto_frame.assign(n, 0);
  for (int s = 0; s < n; ++s) {
    pm_sim* m = sims[s];
    if (!m->prepared) return fail(PM_ERR_STATE, "every scene of a batch must be prepared");
    CK(cudaStreamSynchronize(m->stream));
    pm_status st = m->sync_ctrl();
    if (st != PM_OK) return st;
    if (m->h_ctrl->halt) return fail(PM_ERR_STATE, "a scene is halted; step it once on its own first");
    par_base[s] = (uint32_t)(m->cur - (int)(m->h_ctrl->step & 1u)) & 1u;
    target[s] = m->h_ctrl->step + nsteps;
    m->h_ctrl->target_step = target[s];
    // a batch step is an advance(): frame bookkeeping after every step (as pm_advance does)
    auto_frame[s] = m->h_ctrl->auto_frame;
    m->h_ctrl->auto_frame = 1;
    st = m->push_ctrl();
    if (st != PM_OK) return st;
  }
  return upload_tables();
}

// Reads every control block; regrows halted scenes (when allowed).  all_done: every scene at
// its target; progress: some scene advanced since the previous poll.
pm_status pm_batch::poll(bool& all_done, bool& progress, bool allow_regrow) {
  const int n = ns();
  for (int s = 0; s < n; ++s)
    CK(cudaMemcpyAsync(sims[s]->h_ctrl, sims[s]->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  all_done = true;
  progress = false;
  bool regrown = false;
  for (int s = 0; s < n; ++s) {
    pm_sim* m = sims[s];
    if (m->h_ctrl->step != m->host_step) progress = true;
    m->host_step = m->h_ctrl->step;
    if (m->h_ctrl->step < target[s]) all_done = false;
    if (m->h_ctrl->halt) {
      if (!allow_regrow) return fail(PM_ERR_CAPACITY, "grid capacity reached while profiling a batch");
      const long long want = (long long)m->h_ctrl->need_bricks * 2 + 64;
      if (want * kBrickNodes > 0x7ffffff0LL) return fail(PM_ERR_CAPACITY, "grid would exceed 2^31 nodes");
      pm_status st = m->alloc_grid((int)want);
      if (st != PM_OK) return st;
      ++m->regrowths;
      m->h_ctrl->halt = 0;
      m->h_ctrl->error_flags &= ~(uint32_t)E_CAPACITY;
      st = m->push_ctrl();
      if (st != PM_OK) return st;
      regrown = true;
    } else if (!all_done && m->h_ctrl->step < target[s] && m->h_ctrl->n_bricks > 0.8 * m->brick_cap) {
      pm_status st = m->alloc_grid(m->h_ctrl->n_bricks * 2 + 64);
      if (st != PM_OK) return st;
      ++m->regrowths;
      regrown = true;
    }
  }
  if (regrown) return upload_tables();
  return PM_OK;
}

// Leaves every scene ready for per-scene calls: host step and parity mirrored, target cleared.
pm_status pm_batch::finish() {
  for (int s = 0; s < ns(); ++s) {
    pm_sim* m = sims[s];
    pm_status st = m->sync_ctrl();
    if (st != PM_OK) return st;
    m->host_step = m->h_ctrl->step;
    m->cur = (int)((m->h_ctrl->step + par_base[s]) & 1u);
    m->h_ctrl->target_step = 0;
    m->h_ctrl->idle = 0;
    m->h_ctrl->auto_frame = auto_frame[s];
    st = m->push_ctrl();
    if (st != PM_OK) return st;
  }
  return PM_OK;
}

// Replays the one-round graph until every scene has reached its target (at most `n` rounds per
// scene plus the rounds a regrown scene sat out).
pm_status pm_batch::run_rounds(uint32_t n) {
  uint32_t remaining = n;
  int stalls = 0;
  uint64_t launched = 0;
  const uint64_t limit = 4ull * n + 4096;  // regrowth re-runs are rare; anything beyond is a fault
  while (true) {
    if (launched > limit) return fail(PM_ERR_STATE, "batch rounds exceed the expected count");
    if (graph_dirty) { pm_status st = capture(); if (st != PM_OK) return st; }
    const uint32_t r = std::max<uint32_t>(1, std::min<uint32_t>(remaining, (uint32_t)std::max(1, tune.chunk_rounds)));
    for (uint32_t k = 0; k < r; ++k) CK(cudaGraphLaunch(gexec, stream));
    CK(cudaGetLastError());
    launched += r;
    remaining = remaining > r ? remaining - r : 0;
    bool done = false, progress = false;
    pm_status st = poll(done, progress, true);
    if (st != PM_OK) return st;
    if (done) return PM_OK;
    stalls = progress ? 0 : stalls + 1;
    if (stalls > 8) return fail(PM_ERR_CAPACITY, "batch makes no progress after regrowth");
    if (remaining == 0) {  // scenes that sat rounds out still owe steps
      uint32_t owe = 0;
      for (int s = 0; s < ns(); ++s)
        owe = std::max(owe, target[s] > sims[s]->h_ctrl->step ? target[s] - sims[s]->h_ctrl->step : 0u);
      remaining = owe;
    }
  }
}

extern "C" {

pm_status pm_batch_create(pm_sim* const* scenes, uint32_t n, pm_batch** out) {
  if (!scenes || !out || n == 0) return fail(PM_ERR_INVALID, "need at least one scene and an out pointer");
  *out = nullptr;
  const int dev = scenes[0] ? scenes[0]->device : 0;
  for (uint32_t s = 0; s < n; ++s) {
    if (!scenes[s]) return fail(PM_ERR_INVALID, "NULL scene");
    if (scenes[s]->device != dev) return fail(PM_ERR_INVALID, "all scenes of a batch must be on one device");
    if (!scenes[s]->prepared) return fail(PM_ERR_STATE, "every scene of a batch must be prepared");
    for (uint32_t t = 0; t < s; ++t)
      if (scenes[t] == scenes[s]) return fail(PM_ERR_INVALID, "a scene appears twice in the batch");
  }
  CK(cudaSetDevice(dev));
  pm_batch* b = new pm_batch();
  b->device = dev;
  b->sims.assign(scenes, scenes + n);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return fail(PM_ERR_CUDA, "stream");
  }
  batched_occupancy(b->occ_p2g, b->occ_g2p, b->occ_def);
  b->tune.flat_threads = 256;
  b->tune.part_ctas_per_sm = 8;
  b->tune.node_ctas_per_sm = 8;
  // twice the resident CTAs: with static per-scene partitions, finer pieces balance better
  b->tune.p2g_ctas_per_sm = 2 * b->occ_p2g;
  b->tune.g2p_ctas_per_sm = 2 * b->occ_g2p;
  b->tune.def_ctas_per_sm = 2 * b->occ_def;
  b->tune.sur_ctas_per_sm = 8;
  b->tune.chunk_rounds = 64;
  *out = b;
  return PM_OK;
}

pm_status pm_batch_destroy(pm_batch* b) {
  if (!b) return PM_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  delete b;
  return PM_OK;
}

pm_status pm_batch_step(pm_batch* b, uint32_t nsteps) {
  if (!b) return fail(PM_ERR_INVALID, "NULL batch");
  if (nsteps == 0) return PM_OK;
  pm_status st = b->begin(nsteps);
  if (st != PM_OK) return st;
  st = b->run_rounds(nsteps);
  pm_status st2 = b->finish();
  return st != PM_OK ? st : st2;
}

pm_status pm_batch_get_tuning(pm_batch* b, pm_batch_tuning* t) {
  if (!b || !t) return fail(PM_ERR_INVALID, "NULL argument");
  *t = b->tune;
  return PM_OK;
}

pm_status pm_batch_set_tuning(pm_batch* b, const pm_batch_tuning* t) {
  if (!b || !t) return fail(PM_ERR_INVALID, "NULL argument");
  if (t->flat_threads != 128 && t->flat_threads != 256 && t->flat_threads != 512)
    return fail(PM_ERR_INVALID, "flat_threads must be 128, 256 or 512");
  const int32_t v[] = {t->part_ctas_per_sm, t->node_ctas_per_sm, t->p2g_ctas_per_sm, t->g2p_ctas_per_sm,
                       t->def_ctas_per_sm, t->sur_ctas_per_sm};
  for (int32_t x : v)
    if (x < 1 || x > 64) return fail(PM_ERR_INVALID, "CTAs per SM must be in [1, 64]");
  if (t->chunk_rounds < 1 || t->chunk_rounds > 4096) return fail(PM_ERR_INVALID, "chunk_rounds must be in [1, 4096]");
  b->tune = *t;
  b->graph_dirty = true;
  return PM_OK;
}

pm_status pm_batch_get_stream(pm_batch* b, void** stream) {
  if (!b || !stream) return fail(PM_ERR_INVALID, "NULL argument");
  *stream = (void*)b->stream;
  return PM_OK;
}

int32_t pm_batch_kernels_per_round(pm_batch* b) {
  if (!b) return 0;
  bool sur = false;
  for (pm_sim* m : b->sims) sur = sur || (m->return_map == PM_RETURN_MAP_SURROGATE && m->has_mlp && m->d_q);
  return batched_kernels_per_step(sur);
}

const char* pm_batch_kernel_name(pm_batch* b, int index) {
  if (!b) return "";
  bool sur = false;
  for (pm_sim* m : b->sims) sur = sur || (m->return_map == PM_RETURN_MAP_SURROGATE && m->has_mlp && m->d_q);
  return batched_kernel_name(index, sur);
}

pm_status pm_batch_profile(pm_batch* b, uint32_t rounds, float* kernel_ms, uint32_t n_kernels) {
  if (!b || !kernel_ms) return fail(PM_ERR_INVALID, "NULL argument");
  if (rounds == 0) return PM_OK;
  pm_status st = b->begin(rounds);
  if (st != PM_OK) return st;
  const int K = batched_kernels_per_step(b->L.surrogate);
  if ((int)n_kernels < K) { b->finish(); return fail(PM_ERR_INVALID, "kernel_ms needs kernels_per_round entries"); }
  std::vector<cudaEvent_t> ev(K + 1);
  for (auto& e : ev) CK(cudaEventCreate(&e));
  std::vector<double> acc(K, 0.0);
  for (uint32_t r = 0; r < rounds && st == PM_OK; ++r) {
    launch_step_batched(b->L, b->stream, ev.data());
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) { st = fail(PM_ERR_CUDA, "profiled round failed"); break; }
    for (int i = 0; i < K; ++i) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
      acc[i] += ms;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (int i = 0; i < K; ++i) kernel_ms[i] = (float)(acc[i] / rounds);
  if (st == PM_OK) {  // scenes that halted while profiled are regrown and brought to the target
    bool done = false, progress = false;
    st = b->poll(done, progress, true);
    if (st == PM_OK && !done) st = b->run_rounds(0);
  }
  pm_status st2 = b->finish();
  return st != PM_OK ? st : st2;
}

pm_status pm_batch_autotune(pm_batch* b, uint32_t trial_rounds, pm_batch_tuning* best, float* best_ms) {
  if (!b) return fail(PM_ERR_INVALID, "NULL batch");
  if (trial_rounds == 0) trial_rounds = 4;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  auto trial = [&](const pm_batch_tuning& t, float& ms) -> pm_status {
    b->tune = t;
    b->graph_dirty = true;
    pm_status st = b->begin(trial_rounds + 1);
    if (st != PM_OK) return st;
    if ((st = b->capture()) != PM_OK) return st;
    CK(cudaGraphLaunch(b->gexec, b->stream));  // warm-up round
    CK(cudaEventRecord(e0, b->stream));
    for (uint32_t r = 0; r < trial_rounds; ++r) CK(cudaGraphLaunch(b->gexec, b->stream));
    CK(cudaEventRecord(e1, b->stream));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(&ms, e0, e1));
    ms /= (float)trial_rounds;
    bool done = false, progress = false;
    st = b->poll(done, progress, true);
    if (st == PM_OK && !done) st = b->run_rounds(0);
    pm_status st2 = b->finish();
    return st != PM_OK ? st : st2;
  };
  pm_batch_tuning cur = b->tune;
  float cur_ms = 0.f;
  pm_status st = trial(cur, cur_ms);
  // coordinate search: one launch-shape parameter at a time, two passes
  static int32_t pm_batch_tuning::*const kField[7] = {
      &pm_batch_tuning::flat_threads,    &pm_batch_tuning::part_ctas_per_sm, &pm_batch_tuning::node_ctas_per_sm,
      &pm_batch_tuning::p2g_ctas_per_sm, &pm_batch_tuning::g2p_ctas_per_sm, &pm_batch_tuning::def_ctas_per_sm,
      &pm_batch_tuning::sur_ctas_per_sm};
  for (int pass = 0; pass < 2 && st == PM_OK; ++pass) {
    for (int field = 0; field < 7 && st == PM_OK; ++field) {
      std::vector<int32_t> cand;
      switch (field) {
        case 0: cand = {128, 256, 512}; break;
        case 3: cand = {b->occ_p2g, 2 * b->occ_p2g}; break;
        case 4: cand = {b->occ_g2p, 2 * b->occ_g2p}; break;
        case 5: cand = {b->occ_def, 2 * b->occ_def}; break;
        default: cand = {4, 8, 16}; break;
      }
      if (field == 6 && !b->L.surrogate) continue;
      for (int32_t v : cand) {
        if (v == cur.*kField[field] || st != PM_OK) continue;
        pm_batch_tuning tt = cur;
        tt.*kField[field] = v;
        float ms = 0.f;
        st = trial(tt, ms);
        if (st == PM_OK && ms < cur_ms) { cur = tt; cur_ms = ms; }
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->tune = cur;
  b->graph_dirty = true;
  if (best) *best = cur;
  if (best_ms) *best_ms = cur_ms;
  return st;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// output files (save_data.cpp) and checkpoints
// ------------------------------------------------------------------------------------------
namespace {

// Binary little-endian PLY with float32 vertex properties: the format the reference writes through
// tinyply (save_data.cpp:36-162, `file.write(out, true)`).
pm_status write_ply(const std::string& path, const std::vector<std::string>& props, const float* rows, size_t n) {
  std::ofstream f(path, std::ios::binary);
  if (!f) return fail(PM_ERR_IO, "cannot open " + path);
  f << "ply\nformat binary_little_endian 1.0\nelement vertex " << n << "\n";
  for (const std::string& p : props) f << "property float " << p << "\n";
  f << "end_header\n";
  f.write(reinterpret_cast<const char*>(rows), (std::streamsize)(sizeof(float) * props.size() * n));
  if (!f) return fail(PM_ERR_IO, "write failed: " + path);
  return PM_OK;
}

pm_status write_text(const std::string& path, const std::string& text) {
  std::ofstream f(path);
  if (!f) return fail(PM_ERR_IO, "cannot open " + path);
  f << text;
  return f ? PM_OK : fail(PM_ERR_IO, "write failed: " + path);
}

constexpr char kCkptMagic[8] = {'P', 'M', 'C', 'K', 'P', 'T', '0', '1'};
struct CkptHeader {
  char magic[8];
  uint32_t version, np, nfields, ctrl_bytes;
};

}  // namespace

extern "C" {

pm_status pm_save_particle_data(pm_sim* sim, const char* directory, const char* extra) {
  if (!sim || !directory) return fail(PM_ERR_INVALID, "NULL argument");
  if (!sim->prepared) return fail(PM_ERR_STATE, "call pm_prepare first");
  CK(cudaSetDevice(sim->device));
  pm_status s = sim->wait_copy();
  if (s != PM_OK) return s;
  s = sim->sync_ctrl();
  if (s != PM_OK) return s;
  const uint32_t n = sim->np;
  Params p = sim->P;
  launch_ply_particles(p, sim->d_pbuf[sim->cur], sim->d_meta[sim->cur], sim->d_unperm, sim->stream);
  CK(cudaGetLastError());
  std::vector<float> rows((size_t)n * kPlyFields);
  CK(cudaMemcpyAsync(rows.data(), sim->d_unperm, rows.size() * sizeof(float), cudaMemcpyDeviceToHost, sim->stream));
  CK(cudaStreamSynchronize(sim->stream));
  std::vector<std::string> props = {"x", "y", "z", "vx", "vy", "vz", "p", "q", "Je"};
  if (sim->hp.plastic_model != PM_NO_PLASTICITY) {
    props.insert(props.end(), {"eps_pl_vol", "eps_pl_dev", "delta_gamma"});
  } else {  // compact the rows to the 9 written properties
    for (size_t r = 0; r < n; ++r)
      for (int k = 0; k < 9; ++k) rows[r * 9 + k] = rows[r * kPlyFields + k];
  }
  const std::string dir = std::string(directory) + sim->name;
  const std::string frame = std::to_string(sim->h_ctrl->frame);
  s = write_ply(dir + "/particles_f" + (extra ? extra : "") + frame + ".ply", props, rows.data(), n);
  if (s != PM_OK) return s;
  return write_text(dir + "/last_written.txt", frame + "\n");
}

pm_status pm_save_grid_data(pm_sim* sim, const char* directory, const char* extra) {
  if (!sim || !directory) return fail(PM_ERR_INVALID, "NULL argument");
  double origin[3];
  uint32_t dims[3];
  pm_status s = pm_get_grid(sim, origin, dims, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
  if (s != PM_OK) return s;
  const size_t nn = (size_t)dims[0] * dims[1] * dims[2];
  std::vector<float> mass(nn), v(3 * nn);
  // the reference's grid.v after a step is the MUSL velocity (USL: the updated velocity)
  if (sim->hp.use_musl) s = pm_get_grid(sim, origin, dims, mass.data(), nullptr, v.data(), nullptr, nullptr, nullptr);
  else s = pm_get_grid(sim, origin, dims, mass.data(), v.data(), nullptr, nullptr, nullptr, nullptr);
  if (s != PM_OK) return s;
  std::vector<float> rows(7 * nn);
  const double dx = sim->hp.dx;
  for (uint32_t i = 0; i < dims[0]; ++i)
    for (uint32_t j = 0; j < dims[1]; ++j)
      for (uint32_t k = 0; k < dims[2]; ++k) {
        const size_t l = ((size_t)i * dims[1] + j) * dims[2] + k;
        float* r = &rows[7 * l];
        r[0] = (float)(origin[0] + i * dx); r[1] = (float)(origin[1] + j * dx); r[2] = (float)(origin[2] + k * dx);
        r[3] = v[3 * l]; r[4] = v[3 * l + 1]; r[5] = v[3 * l + 2];
        r[6] = mass[l];
      }
  const std::string dir = std::string(directory) + sim->name;
  return write_ply(dir + "/grid_f" + (extra ? extra : "") + std::to_string(sim->h_ctrl->frame) + ".ply",
                   {"x", "y", "z", "vx", "vy", "vz", "mass"}, rows.data(), nn);
}

pm_status pm_save_info(pm_sim* sim, const char* directory) {
  if (!sim || !directory) return fail(PM_ERR_INVALID, "NULL argument");
  std::ostringstream t;  // save_data.cpp:347-356, one value per line
  t << sim->hp.end_frame << "\n" << sim->hp.fps << "\n" << sim->hp.dx << "\n" << sim->np << "\n"
    << sim->hp.particle_volume << "\n";
  return write_text(std::string(directory) + sim->name + "/info.txt", t.str());
}

pm_status pm_save_checkpoint(pm_sim* sim, const char* path) {
  if (!sim || !path) return fail(PM_ERR_INVALID, "NULL argument");
  if (!sim->prepared) return fail(PM_ERR_STATE, "call pm_prepare first");
  CK(cudaSetDevice(sim->device));
  pm_status s = sim->wait_copy();
  if (s != PM_OK) return s;
  s = sim->sync_ctrl();
  if (s != PM_OK) return s;
  const uint32_t n = sim->np;
  Params p = sim->P;
  launch_unpermute(p, sim->d_pbuf[sim->cur], sim->d_meta[sim->cur], sim->d_unperm, sim->d_active, sim->stream);
  CK(cudaGetLastError());
  std::vector<float> fields((size_t)n * F_COUNT);
  std::vector<uint8_t> active(n);
  CK(cudaMemcpyAsync(fields.data(), sim->d_unperm, fields.size() * sizeof(float), cudaMemcpyDeviceToHost, sim->stream));
  CK(cudaMemcpyAsync(active.data(), sim->d_active, n, cudaMemcpyDeviceToHost, sim->stream));
  CK(cudaStreamSynchronize(sim->stream));
  std::ofstream f(path, std::ios::binary);
  if (!f) return fail(PM_ERR_IO, std::string("cannot open ") + path);
  CkptHeader h{};
  std::memcpy(h.magic, kCkptMagic, 8);
  h.version = 1;
  h.np = n;
  h.nfields = F_COUNT;
  h.ctrl_bytes = (uint32_t)sizeof(Ctrl);
  f.write(reinterpret_cast<const char*>(&h), sizeof(h));
  f.write(reinterpret_cast<const char*>(fields.data()), (std::streamsize)(fields.size() * sizeof(float)));
  f.write(reinterpret_cast<const char*>(active.data()), (std::streamsize)active.size());
  f.write(reinterpret_cast<const char*>(sim->h_ctrl), sizeof(Ctrl));
  return f ? PM_OK : fail(PM_ERR_IO, std::string("write failed: ") + path);
}

pm_status pm_load_checkpoint(pm_sim* sim, const char* path) {
  if (!sim || !path) return fail(PM_ERR_INVALID, "NULL argument");
  if (!sim->prepared) return fail(PM_ERR_STATE, "set up the same scene and call pm_prepare before loading");
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(PM_ERR_IO, std::string("cannot open ") + path);
  CkptHeader h{};
  f.read(reinterpret_cast<char*>(&h), sizeof(h));
  if (!f || std::memcmp(h.magic, kCkptMagic, 8) != 0 || h.version != 1)
    return fail(PM_ERR_IO, "not a checkpoint of this library");
  if (h.nfields != F_COUNT || h.ctrl_bytes != sizeof(Ctrl))
    return fail(PM_ERR_UNSUPPORTED, "checkpoint written by a different build of the library");
  if (h.np != sim->np) return fail(PM_ERR_INVALID, "checkpoint particle count differs from the scene's");
  std::vector<float> fields((size_t)h.np * F_COUNT);
  std::vector<uint8_t> active(h.np);
  Ctrl c{};
  f.read(reinterpret_cast<char*>(fields.data()), (std::streamsize)(fields.size() * sizeof(float)));
  f.read(reinterpret_cast<char*>(active.data()), (std::streamsize)active.size());
  f.read(reinterpret_cast<char*>(&c), sizeof(Ctrl));
  if (!f) return fail(PM_ERR_IO, "checkpoint is truncated");
  CK(cudaSetDevice(sim->device));
  CK(cudaStreamSynchronize(sim->stream));
  float* d_in = nullptr;
  uint8_t* d_act = nullptr;
  CK(cudaMalloc(&d_in, fields.size() * sizeof(float)));
  if (cudaMalloc(&d_act, std::max<size_t>(active.size(), 1)) != cudaSuccess) {
    cudaFree(d_in);
    return fail(PM_ERR_CUDA, "allocation for the checkpoint failed");
  }
  cudaMemcpy(d_in, fields.data(), fields.size() * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(d_act, active.data(), active.size(), cudaMemcpyHostToDevice);
  sim->drop_graphs();
  sim->cur = 0;
  Params p = sim->P;
  launch_load_fields(p, d_in, d_act, sim->d_pbuf[0], sim->d_meta[0], sim->stream);
  const cudaError_t e = cudaStreamSynchronize(sim->stream);
  cudaFree(d_in);
  cudaFree(d_act);
  if (e != cudaSuccess) return fail(PM_ERR_CUDA, std::string("checkpoint upload: ") + cudaGetErrorString(e));
  // the control block as saved (time, dt, step, frame, object poses, reference boxes, reductions)
  c.halt = 0;
  c.idle = 0;
  c.target_step = 0;
  *sim->h_ctrl = c;
  sim->host_step = c.step;
  pm_status s = sim->push_ctrl();
  if (s != PM_OK) return s;
  sim->fill_params();
  return PM_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// headless pigment splat (BinaryDensityGrid::fillRenderGrid)
// ------------------------------------------------------------------------------------------
#ifndef PM_SPLAT_SPREAD
#define PM_SPLAT_SPREAD 0
#endif
// Particle visiting order of the splat.  The particles are stored cell-sorted; with
// PM_SPLAT_SPREAD the warps visit particle t * stride mod np instead (stride near the golden
// section of np and coprime to it, so the map is a permutation), which spreads the warps resident
// at one time over the whole body.  On the 2M-particle two-block scene the sorted order measured
// 47.9 ms against 50.1 ms spread (L2 locality of the voxel atomics outweighs their contention),
// so 1 (sorted) is the default stride.
static uint32_t splat_order_stride(uint32_t np) {
  if (!PM_SPLAT_SPREAD || np < 3) return 1;
  uint64_t s = (uint64_t)(0.6180339887498949 * (double)np);
  for (int k = 0; k < 4096; ++k, ++s)
    if (s > 1 && std::gcd(s, (uint64_t)np) == 1) return (uint32_t)s;
  return 1;
}

extern "C" {

pm_status pm_splat_pigments(pm_sim* sim, const float* G, int device_ptrs, float sigma_spatial, float sigma_color,
                            float* voxels, uint32_t dims[3], double origin[3], double* voxel_size) {
  if (!sim || !dims) return fail(PM_ERR_INVALID, "NULL argument");
  if (!sim->prepared) return fail(PM_ERR_STATE, "call pm_prepare first");
  CK(cudaSetDevice(sim->device));
  pm_status s = sim->sync_ctrl();
  if (s != PM_OK) return s;
  // AABBc::fixedAABB (AABBc.cpp:10-25): density voxels of the support radius 2 dx
  // (MPMIntegrationSim.cpp:96-98) over the grid boundaries; the pigment grid is 4x finer
  const float h = (float)(2.0 * sim->hp.dx);
  SplatGeom g{};
  for (int d = 0; d < 3; ++d) {
    const float mn = (float)sim->h_ctrl->low[d], mx = (float)sim->h_ctrl->high[d];
    const float start = std::floor(mn / h) * h;
    const int cells = (int)std::ceil((mx - mn) / h) + 1;
    g.start[d] = start;
    g.dims[d] = 4 * cells;
    dims[d] = (uint32_t)g.dims[d];
    if (origin) origin[d] = start;
  }
  g.v4 = h / 4.0f;
  if (voxel_size) *voxel_size = g.v4;
  if (!voxels) return PM_OK;  // size query
  // BinaryDensityGrid.cpp:162-170: sigmas floored at 0.001, search extent 3 h sigma_s, at most 12
  const float ss = std::max(sigma_spatial, 0.001f), sc = std::max(sigma_color, 0.001f);
  g.ext = std::min(12, (int)std::ceil(h * 3.0f * ss / g.v4));
  g.sig_s2 = ss * ss;
  g.sig_c2 = sc * sc;
  g.inv_h = 1.0f / h;
  const size_t nvox = (size_t)g.dims[0] * g.dims[1] * g.dims[2];
  const size_t bytes = nvox * 8 * sizeof(float);
  g.order_stride = splat_order_stride(sim->np);
  const size_t want = device_ptrs ? bytes : 2 * bytes;
  if (sim->splat_bytes < want) {
    if (sim->d_splat) cudaFree(sim->d_splat);
    sim->d_splat = nullptr;
    sim->splat_bytes = 0;
    if (cudaMalloc(&sim->d_splat, want) != cudaSuccess) {
      cudaGetLastError();
      return fail(PM_ERR_CUDA, "allocation of the splat grids failed");
    }
    sim->splat_bytes = want;
  }
  float* d_tmp = sim->d_splat;
  float* d_out = device_ptrs ? voxels : sim->d_splat + nvox * 8;
  float* d_G = nullptr;
  auto release = [&]() {
    if (d_G) cudaFree(d_G);
  };
  const float* Gd = G;
  if (G && !device_ptrs) {
    if (cudaMalloc(&d_G, (size_t)sim->np * 9 * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      return fail(PM_ERR_CUDA, "allocation of the anisotropy matrices failed");
    }
    cudaMemcpy(d_G, G, (size_t)sim->np * 9 * sizeof(float), cudaMemcpyHostToDevice);
    Gd = d_G;
  }
  Params p = sim->P;
  cudaError_t e = launch_splat(p, sim->d_pbuf[sim->cur], sim->d_meta[sim->cur], Gd, g, d_tmp, d_out, sim->stream);
  if (e == cudaSuccess && !device_ptrs)
    e = cudaMemcpyAsync(voxels, d_out, bytes, cudaMemcpyDeviceToHost, sim->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(sim->stream);
  release();
  if (e != cudaSuccess) return fail(PM_ERR_CUDA, std::string("pigment splat: ") + cudaGetErrorString(e));
  return PM_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// renderer preprocessing: binary density grid (BinaryDensityGrid::fillBDG) and anisotropy
// (Classification::countDensities)
// ------------------------------------------------------------------------------------------
namespace {

// AABBc::fixedAABB (AABBc.cpp:10-25) over the simulation's grid boundaries, in float as there
DensityGeom density_geom(const pm_sim* sim) {
  DensityGeom g{};
  const float h = (float)(2.0 * sim->hp.dx);
  g.h = h;
  for (int d = 0; d < 3; ++d) {
    const float mn = (float)sim->h_ctrl->low[d], mx = (float)sim->h_ctrl->high[d];
    g.start[d] = std::floor(mn / h) * h;
    g.dims[d] = (int)std::ceil((mx - mn) / h) + 1;
  }
  return g;
}

// Grows the render scratch to at least `bytes` and carves the binning / anisotropy arrays.
pm_status render_scratch(pm_sim* sim, uint32_t ncell, bool aniso, size_t extra, RenderScratch& r, char*& tail) {
  const size_t core = render_scratch_bytes(sim->np, ncell, aniso);
  const size_t want = core + (extra + 255) / 256 * 256;
  if (sim->render_bytes < want) {
    if (sim->d_render) cudaFree(sim->d_render);
    sim->d_render = nullptr;
    sim->render_bytes = 0;
    if (cudaMalloc(&sim->d_render, want) != cudaSuccess) {
      cudaGetLastError();
      return fail(PM_ERR_CUDA, "allocation of the density-grid scratch failed");
    }
    sim->render_bytes = want;
  }
  const size_t nb = (ncell + 4095) / 4096;
  uint32_t* u = static_cast<uint32_t*>(sim->d_render);
  r.counts = u; u += ncell;
  r.offsets = u; u += ncell;
  r.bsum = u; u += nb;
  r.misc = u; u += 4;
  r.cellid = u; u += sim->np;
  r.rank = u; u += sim->np;
  r.ids = u; u += sim->np;
  float* f = reinterpret_cast<float*>(u);
  r.Gs = aniso ? f : nullptr;
  r.dets = aniso ? f + (size_t)6 * sim->np : nullptr;
  tail = static_cast<char*>(sim->d_render) + core;
  return PM_OK;
}

}  // namespace

extern "C" {

pm_status pm_density_grid(pm_sim* sim, float a, float b, float iso, int test_all_filled, int device_ptrs,
                          uint32_t* M, uint32_t* M2, uint32_t* M4, uint32_t* cell_count, uint32_t* cell_offset,
                          uint32_t* ids, uint32_t dims[3], double origin[3], double* voxel_size,
                          uint32_t occupancy[2]) {
  if (!sim || !dims) return fail(PM_ERR_INVALID, "NULL argument");
  if (!sim->prepared) return fail(PM_ERR_STATE, "call pm_prepare first");
  CK(cudaSetDevice(sim->device));
  pm_status st = sim->sync_ctrl();
  if (st != PM_OK) return st;
  const DensityGeom g = density_geom(sim);
  for (int d = 0; d < 3; ++d) {
    dims[d] = (uint32_t)g.dims[d];
    if (origin) origin[d] = g.start[d];
  }
  if (voxel_size) *voxel_size = g.h;
  if (!M) return PM_OK;  // size query
  const size_t X = g.dims[0], Y = g.dims[1], Z = g.dims[2];
  const size_t ncell = X * Y * Z;
  if (ncell > (size_t)4096 * 4096) return fail(PM_ERR_CAPACITY, "more density voxels than the binning scan covers");
  const size_t n2 = ((X + 1) / 2) * ((Y + 1) / 2) * ((Z + 1) / 2), n4 = ((X + 3) / 4) * ((Y + 3) / 4) * ((Z + 3) / 4);
  // staging: M2 / M4 always (a caller may not want them), M and ids for host outputs
  const size_t staged = 4 * (n2 + n4) + (device_ptrs ? 0 : 4 * (ncell + (size_t)sim->np));
  RenderScratch r{};
  char* tail = nullptr;
  if ((st = render_scratch(sim, (uint32_t)ncell, false, staged, r, tail)) != PM_OK) return st;
  uint32_t* u = reinterpret_cast<uint32_t*>(tail);
  uint32_t *dM = M, *dM2 = u, *dM4 = u + n2, *dids = ids;
  if (device_ptrs) {
    if (M2) dM2 = M2;
    if (M4) dM4 = M4;
  } else {
    dM = u + n2 + n4;
    dids = u + n2 + n4 + ncell;
  }
  Params p = sim->P;
  cudaError_t e = launch_bin_particles(p, sim->d_pbuf[sim->cur], g, r, sim->stream);
  const float kern = (float)(315.0 / (64.0 * M_PI * std::pow((double)g.h, 3)));  // BinaryDensityGrid.cpp:117
  if (e == cudaSuccess)
    e = launch_density_mask(g, r, a, b, kern, iso, test_all_filled, dM, dM2, dM4, sim->stream);
  if (e == cudaSuccess && ids) e = launch_ids_to_pid(r.ids, sim->d_meta[sim->cur], r.misc, dids, (int)sim->np, sim->stream);
  uint32_t misc[4] = {0, 0, 0, 0};
  const cudaMemcpyKind k = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (e == cudaSuccess && cell_count) e = cudaMemcpyAsync(cell_count, r.counts, 4 * ncell, k, sim->stream);
  if (e == cudaSuccess && cell_offset) e = cudaMemcpyAsync(cell_offset, r.offsets, 4 * ncell, k, sim->stream);
  if (e == cudaSuccess && !device_ptrs) {
    e = cudaMemcpyAsync(M, dM, 4 * ncell, cudaMemcpyDeviceToHost, sim->stream);
    if (e == cudaSuccess && M2) e = cudaMemcpyAsync(M2, dM2, 4 * n2, cudaMemcpyDeviceToHost, sim->stream);
    if (e == cudaSuccess && M4) e = cudaMemcpyAsync(M4, dM4, 4 * n4, cudaMemcpyDeviceToHost, sim->stream);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(misc, r.misc, sizeof(misc), cudaMemcpyDeviceToHost, sim->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(sim->stream);
  if (e != cudaSuccess) return fail(PM_ERR_CUDA, std::string("density grid: ") + cudaGetErrorString(e));
  if (ids && !device_ptrs) {
    CK(cudaMemcpy(ids, dids, 4 * (size_t)misc[0], cudaMemcpyDeviceToHost));
  }
  if (occupancy) {
    occupancy[0] = (uint32_t)(ncell - misc[1]);
    occupancy[1] = misc[1];
  }
  return PM_OK;
}

pm_status pm_anisotropy(pm_sim* sim, float s, float k, int threshold, int auto_scale, int is_ani, float iso,
                        int device_ptrs, float* G, float* G_inv, float* det, float* density, uint32_t* n_aggregate) {
  if (!sim) return fail(PM_ERR_INVALID, "NULL sim");
  if (!sim->prepared) return fail(PM_ERR_STATE, "call pm_prepare first");
  if (!(k > 0.f)) return fail(PM_ERR_INVALID, "k must be positive");
  CK(cudaSetDevice(sim->device));
  pm_status st = sim->sync_ctrl();
  if (st != PM_OK) return st;
  const DensityGeom g = density_geom(sim);
  const size_t ncell = (size_t)g.dims[0] * g.dims[1] * g.dims[2];
  if (ncell > (size_t)4096 * 4096) return fail(PM_ERR_CAPACITY, "more density voxels than the binning scan covers");
  const size_t np = sim->np;
  const size_t staged = device_ptrs ? 0 : 4 * np * ((G ? 9 : 0) + (G_inv ? 9 : 0) + (det ? 1 : 0) + (density ? 1 : 0));
  RenderScratch r{};
  char* tail = nullptr;
  if ((st = render_scratch(sim, (uint32_t)ncell, true, staged, r, tail)) != PM_OK) return st;
  float *dG = G, *dGi = G_inv, *dD = det, *dR = density;
  if (!device_ptrs) {
    float* f = reinterpret_cast<float*>(tail);
    if (G) { dG = f; f += 9 * np; }
    if (G_inv) { dGi = f; f += 9 * np; }
    if (det) { dD = f; f += np; }
    if (density) { dR = f; f += np; }
  }
  AnisoParams ap{};
  ap.s = s;
  ap.k = k;
  ap.threshold = threshold;
  ap.auto_scale = auto_scale;
  ap.is_ani = is_ani;
  const float kern = 315.0f / (64.0f * (float)M_PI);  // state.h:36
  Params p = sim->P;
  cudaError_t e = launch_bin_particles(p, sim->d_pbuf[sim->cur], g, r, sim->stream);
  if (e == cudaSuccess)
    e = launch_anisotropy(p, sim->d_pbuf[sim->cur], sim->d_meta[sim->cur], g, r, ap, kern, iso, dG, dGi, dD, dR,
                          sim->stream);
  if (e == cudaSuccess && !device_ptrs) {
    if (G) e = cudaMemcpyAsync(G, dG, 36 * np, cudaMemcpyDeviceToHost, sim->stream);
    if (e == cudaSuccess && G_inv) e = cudaMemcpyAsync(G_inv, dGi, 36 * np, cudaMemcpyDeviceToHost, sim->stream);
    if (e == cudaSuccess && det) e = cudaMemcpyAsync(det, dD, 4 * np, cudaMemcpyDeviceToHost, sim->stream);
    if (e == cudaSuccess && density) e = cudaMemcpyAsync(density, dR, 4 * np, cudaMemcpyDeviceToHost, sim->stream);
  }
  uint32_t misc[4] = {0, 0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(misc, r.misc, sizeof(misc), cudaMemcpyDeviceToHost, sim->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(sim->stream);
  if (e != cudaSuccess) return fail(PM_ERR_CUDA, std::string("anisotropy: ") + cudaGetErrorString(e));
  if (n_aggregate) *n_aggregate = misc[2];
  return PM_OK;
}

}  // extern "C"

extern "C" pm_status pm_svd3_batch(int device, const double* A, uint32_t n, float* U, double* S, float* V) {
  if (!A || !U || !S || !V) return fail(PM_ERR_INVALID, "NULL argument");
  CK(cudaSetDevice(device));
  cudaError_t e = cudaSuccess;
  if (num_sms() <= 0 && (e = launch_init(device)) != cudaSuccess)
    return fail(PM_ERR_CUDA, std::string("kernel set-up: ") + cudaGetErrorString(e));
  if (n == 0) return PM_OK;
  double *dA = nullptr, *dS = nullptr;
  float *dU = nullptr, *dV = nullptr;
  auto release = [&]() { cudaFree(dA); cudaFree(dS); cudaFree(dU); cudaFree(dV); };
  if (cudaMalloc(&dA, 72ull * n) != cudaSuccess || cudaMalloc(&dS, 24ull * n) != cudaSuccess ||
      cudaMalloc(&dU, 36ull * n) != cudaSuccess || cudaMalloc(&dV, 36ull * n) != cudaSuccess) {
    release();
    cudaGetLastError();
    return fail(PM_ERR_CUDA, "allocation failed");
  }
  e = cudaMemcpy(dA, A, 72ull * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    launch_svd3_batch(dA, (int)n, dU, dS, dV, nullptr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(U, dU, 36ull * n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(S, dS, 24ull * n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(V, dV, 36ull * n, cudaMemcpyDeviceToHost);
  release();
  if (e != cudaSuccess) return fail(PM_ERR_CUDA, std::string("svd self-test: ") + cudaGetErrorString(e));
  return PM_OK;
}

// ------------------------------------------------------------------------------------------
// Poisson-disk particle sampling (sampleParticles, sampling_particles.hpp:12-70)
// ------------------------------------------------------------------------------------------
extern "C" {

pm_status pm_sample_particles(int device, double Lx, double Ly, double Lz, double radius, double ppc,
                              int crop_to_shape, uint32_t attempts, uint32_t passes, uint32_t seed, float* x,
                              uint32_t capacity, uint32_t* n, double* dx, double* particle_volume) {
  if (!n) return fail(PM_ERR_INVALID, "NULL count pointer");
  if (!(radius > 0.0) || !(Lx > 0.0) || !(Ly > 0.0) || !(Lz > 0.0) || !(ppc > 0.0))
    return fail(PM_ERR_INVALID, "radius, box sides and ppc must be positive");
  if (crop_to_shape < 0 || crop_to_shape > 2) return fail(PM_ERR_INVALID, "crop_to_shape: 0 box, 1 cylinder, 2 silo");
  const double cs = radius / std::sqrt(3.0);
  const long long nx = (long long)std::ceil(Lx / cs), ny = (long long)std::ceil(Ly / cs), nz = (long long)std::ceil(Lz / cs);
  const long long ncell = nx * ny * nz;
  if (ncell > (1ll << 31)) return fail(PM_ERR_CAPACITY, "box too large for the sampling grid");
  CK(cudaSetDevice(device));
  cudaError_t e = cudaSuccess;
  if (num_sms() <= 0 && (e = launch_init(device)) != cudaSuccess)
    return fail(PM_ERR_CUDA, std::string("kernel set-up: ") + cudaGetErrorString(e));
  float4* d_cells = nullptr;
  CK(cudaMalloc(&d_cells, sizeof(float4) * (size_t)ncell));
  e = poisson_fill(d_cells, (int)nx, (int)ny, (int)nz, (float)cs, (float)radius, seed, std::max(passes, 1u),
                   attempts ? attempts : 30u, 0);
  std::vector<float4> cells(e == cudaSuccess ? (size_t)ncell : 0);
  if (e == cudaSuccess) e = cudaMemcpy(cells.data(), d_cells, sizeof(float4) * (size_t)ncell, cudaMemcpyDeviceToHost);
  cudaFree(d_cells);
  if (e != cudaSuccess) return fail(PM_ERR_CUDA, std::string("Poisson sampling: ") + cudaGetErrorString(e));
  // samples inside the box, in cell order; dx and the particle volume from the uncropped count
  std::vector<float> pts;
  size_t square = 0;
  for (const float4& c : cells) {
    if (c.w == 0.f || c.x >= Lx || c.y >= Ly || c.z >= Lz) continue;
    ++square;
    const double px = c.x - Lx / 2.0, py = c.y, pz = c.z - Lz / 2.0;
    if (crop_to_shape == 1 && !(px * px + pz * pz < (Lx / 2.0) * (Lx / 2.0))) continue;
    if (crop_to_shape == 2) {
      const double rs = std::tanh(py) + 1.0;
      if (!(px * px + pz * pz < rs * rs)) continue;
    }
    pts.insert(pts.end(), {c.x, c.y, c.z});
  }
  const double d = std::cbrt(ppc / (double)std::max<size_t>(square, 1) * Lx * Ly * Lz);
  if (dx) *dx = d;
  if (particle_volume) *particle_volume = d * d * d / ppc;
  *n = (uint32_t)(pts.size() / 3);
  if (x) {
    if (capacity < *n) return fail(PM_ERR_CAPACITY, "output array holds fewer particles than were sampled");
    std::memcpy(x, pts.data(), pts.size() * sizeof(float));
  }
  return PM_OK;
}

}  // extern "C"

/*
 * pigment_mpm.h -- C ABI of the B200 paint-mixing MPM step (drop-in for the reference's
 * `Simulation` setup/step API, Natashaaak/pigment_mixing matter/src/simulation/simulation.hpp:25-186).
 *
 * One `pm_sim` is one `Simulation`.  All particle and grid state lives in GPU memory; host
 * buffers passed to the calls below are copied in or out.  Every call returns a pm_status.
 * Plain C types only: the library can be bound from C, C++, ctypes, cgo, JNI or N-API.
 *
 * Each declaration names the reference interface it replaces (file:line in the reference
 * repository).  Enumerations keep the reference's numeric values (matter/src/tools.hpp:55-59).
 */
#ifndef PIGMENT_MPM_H
#define PIGMENT_MPM_H

#include <stddef.h>
#include <stdint.h>

#if defined(_WIN32)
#define PM_API __declspec(dllexport)
#else
#define PM_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pm_sim pm_sim;

typedef enum pm_status {
  PM_OK = 0,
  PM_ERR_INVALID = 1,      /* bad argument or unknown parameter name */
  PM_ERR_STATE = 2,        /* call out of order (e.g. step before prepare) */
  PM_ERR_CUDA = 3,         /* a CUDA call failed; pm_last_error_message() has the text */
  PM_ERR_IO = 4,           /* a file could not be read */
  PM_ERR_UNSUPPORTED = 5,  /* model or option not implemented on this path */
  PM_ERR_CAPACITY = 6      /* a size limit was exceeded */
} pm_status;

/* matter/src/tools.hpp:55 */
typedef enum pm_plate_type { PM_PLATE_TOP = 0, PM_PLATE_BOTTOM, PM_PLATE_LEFT, PM_PLATE_RIGHT, PM_PLATE_FRONT,
                             PM_PLATE_BACK } pm_plate_type;
/* matter/src/tools.hpp:59 */
typedef enum pm_bc { PM_BC_NOSLIP = 0, PM_BC_SLIPSTICK = 1, PM_BC_SLIPFREE = 2 } pm_bc;
/* matter/src/tools.hpp:57; this path implements NoPlasticity, VMVisc and DPVisc */
typedef enum pm_plastic_model { PM_NO_PLASTICITY = 0, PM_VM = 1, PM_DP = 2, PM_DPSOFT = 3, PM_MCC = 4,
                                PM_VMVISC = 5, PM_DPVISC = 6, PM_MCCVISC = 7, PM_DPMUI = 8,
                                PM_MCCMUI = 9 } pm_plastic_model;
/* Return-map implementation (no reference counterpart: the learned surrogate is new). */
typedef enum pm_return_map { PM_RETURN_MAP_PLAIN = 0, PM_RETURN_MAP_SURROGATE = 1 } pm_return_map;

/* Device error bits read by pm_get_error_flags (the reference's `int exit`, simulation.hpp:30). */
#define PM_FLAG_NEG_DGAMMA 0x1u    /* plasticity.cpp:186-192, 286-289 */
#define PM_FLAG_NEWTON_NOCONV 0x2u /* plasticity.cpp:200-203, 298-301 */
#define PM_FLAG_NEWTON_FLAT 0x4u   /* plasticity.cpp:219-222, 314-317 */
#define PM_FLAG_INVALID_BC 0x8u    /* boundary_collision.cpp:84-88 */
#define PM_FLAG_NAN_PARTICLE 0x10u /* position_update.cpp:311-327: a particle was deactivated */
#define PM_FLAG_INDEX_RANGE 0x20u  /* a particle fell outside the step's grid (never expected) */
#define PM_FLAG_CAPACITY 0x40u     /* grid capacity exceeded; the host regrows and resumes */

/* ---- lifetime ---------------------------------------------------------------------------- */
/* Simulation::Simulation() (simulation.cpp:3-22).  device: CUDA ordinal. */
PM_API pm_status pm_create(int device, pm_sim** out);
/* ~Simulation() */
PM_API pm_status pm_destroy(pm_sim* sim);
/* The particle and grid buffers of every simulation on a device come from one pool that keeps
 * freed memory for the process (as a caching allocator does), so that a later simulation reuses
 * it without driver allocations.  This hands cached memory above keep_bytes back to the driver
 * (no counterpart in the reference, which allocates host vectors). */
PM_API pm_status pm_trim_memory(int device, uint64_t keep_bytes);
/* Text of the last error on this thread (static storage, never NULL). */
PM_API const char* pm_last_error_message(void);

/* Simulation::initializeBasic(name) (simulation_units.cpp:9-26). */
PM_API pm_status pm_initialize_basic(pm_sim* sim, const char* name);

/* ---- parameters: the public fields of Simulation (simulation.hpp:38-126) ---------------- */
/* Scalar fields by name: "cfl", "cfl_elastic", "flip_ratio", "rho", "E", "nu", "fps", "end_frame",
 * "min_dt", "dx", "particle_mass", "particle_volume", "plastic_model", "use_pradhana", "use_musl",
 * "use_particle_boundaries", "q_max", "q_min", "p_min", "M", "q_cohesion", "perzyna_exp",
 * "perzyna_visc", "xi", "q_prefac", "pigment_D_max", "pigment_D_edge0", "pigment_D_edge1",
 * "start_boost_time", "end_boost_time", "boost_factor", "frame", "auto_frame"; and (no reference
 * counterpart) "surrogate_fallback_plain", "sample_log_every".
 * Read-only extras for pm_get_param: "time", "dt", "step", "Np", "mu", "lambda", "K", "dt_max",
 * "frame_dt", "final_time", "n_active", "plastic_count", "grid_nodes", "kernels_per_step",
 * "regrowths", "regrow_ms", "grid_capacity_nodes", and the host time of a simulation's fixed costs so
 * far, "alloc_ms" (particle and grid buffer allocation) and "graph_ms" (step-graph capture and
 * instantiation). */
PM_API pm_status pm_set_param(pm_sim* sim, const char* name, double value);
PM_API pm_status pm_get_param(pm_sim* sim, const char* name, double* value);
/* Vector fields: "gravity", "particle_boundary_min", "particle_boundary_max", "grid_reference_point". */
PM_API pm_status pm_set_param3(pm_sim* sim, const char* name, const double value[3]);

/* The JSON readers of Simulation::setupScene (simulation_units.cpp:31-80): same keys, same
 * defaults when a key is absent; a missing file leaves the fields as set (the reference's
 * file-missing defaults are applied by pm_setup_scene).  Returns PM_ERR_IO on a parse error. */
PM_API pm_status pm_load_pigment_config(pm_sim* sim, const char* path);
PM_API pm_status pm_load_sim_config(pm_sim* sim, const char* path);

/* ---- particles (Simulation::particles / Np, data_structures.hpp:9-50) --------------------- */
/* Host arrays, row-major: x[n*3], latent[n*7] (Mixbox latent: 4 concentrations + 3 RGB
 * residuals), v[n*3] or NULL for zero.  Resets F to identity and all plastic state to zero. */
PM_API pm_status pm_set_particles(pm_sim* sim, uint32_t n, const float* x, const float* latent, const float* v);
/* Copies particle state back to host arrays in the original particle order.  Any pointer may
 * be NULL.  F and B: n*9 row-major; plastic: n*4 (eps_pl_dev, eps_pl_vol, eps_pl_vol_pradhana,
 * delta_gamma); active: n bytes (0/1). */
PM_API pm_status pm_get_particles(pm_sim* sim, float* x, float* v, float* latent, float* diffusion, uint8_t* active,
                           float* F, float* B, float* plastic);
/* The per-frame readback of MPMIntegrationSim::recountParticles (MPMIntegrationSim.cpp:100-116)
 * without waiting for it: the fields are gathered into original order behind the steps issued so
 * far and copied to the host on a separate stream, so steps issued afterwards overlap the copy.
 * The host arrays must stay valid (and should be pinned: pageable memory makes the copy
 * synchronous) until pm_wait_particles returns; any other readback call waits first. */
PM_API pm_status pm_get_particles_async(pm_sim* sim, float* x, float* v, float* latent, float* diffusion,
                                        uint8_t* active);
/* Waits for the last pm_get_particles_async to land in its host arrays. */
PM_API pm_status pm_wait_particles(pm_sim* sim);

/* ---- object plugins --------------------------------------------------------------------- */
/* ObjectPlate(pos, type, bc, friction, pos_lower, pos_upper, vx, vy, vz, vmin_factor,
 * load_factor) (object_plate.hpp:13-28). */
PM_API pm_status pm_add_plate(pm_sim* sim, double pos, int plate_type, int bc, double friction, double pos_lower,
                       double pos_upper, double vx, double vy, double vz, double vmin_factor, double load_factor);
/* ObjectSpatula(bc, friction, name, anim_path) (object_spatula.hpp:16-37) with the keyframes
 * given in memory: frames[n*7] = position xyz, quaternion xyzw at 60 frames/s. */
PM_API pm_status pm_add_spatula(pm_sim* sim, int bc, double friction, const float* frames, uint32_t n);
/* Same, reading a spatula_motion.bin file (ObjectSpatula::loadAnimation, object_spatula.hpp:235-250). */
PM_API pm_status pm_add_spatula_file(pm_sim* sim, int bc, double friction, const char* anim_path);
/* Box knife (no reference counterpart; the synthetic workloads' knife): a box SDF with the given
 * half extents, fixed orientation quat_wxyz (NULL = identity), centre moving along the polyline
 * waypoints[n*3] at `speed` units/s.  Like the spatula it is the scene's knife
 * (spatula_ptr, simulation.hpp:131) and takes the knife-specific collision rules. */
PM_API pm_status pm_add_box_knife(pm_sim* sim, int bc, double friction, const double half[3], const double* waypoints,
                           uint32_t n, double speed, const double* quat_wxyz);
/* ObjectGround(bc, friction, name, y) (object_ground.hpp:14) and ObjectCurve(bc, friction)
 * (object_curve.hpp:13), the analytic colliders of the reference's tests. */
PM_API pm_status pm_add_ground(pm_sim* sim, int bc, double friction, double y0);
PM_API pm_status pm_add_curve(pm_sim* sim, int bc, double friction);

/* ---- scene set-up and stepping ------------------------------------------------------------ */
/* Simulation::setupScene(fps, colorRatios, pigments, anim_path) (simulation_units.cpp:28-131)
 * without the OpenVDB blob sampling: the particles come from a prior pm_set_particles call.
 * Reads the two JSON files (NULL = skip), sets gravity, particle boundaries [-2, 2]^3, the grid
 * reference point (0,0,0), the bottom floor plate (SlipStick, friction 1), the spatula from
 * anim_path (NULL = none), DPVisc with Pradhana correction and q_prefac = 1/sqrt(2). */
PM_API pm_status pm_setup_scene(pm_sim* sim, float fps, const char* pigment_config_path, const char* sim_config_path,
                         const char* anim_path);
/* Simulation::setupScene(fps, colorRatios, pigments, anim_path) (simulation_units.cpp:28-131) in the
 * reference's own shape, with its blob scene (Simulation::blobs, simulation_blobs.cpp:7-150): one
 * paint blob per colour ratio, k blobs, latents[k*7] the Mixbox latent of each colour.  A ratio
 * clamped to [0.1, 0.9] sets the blob's volume on the reference's blob ladder (0.0056-0.053); the
 * blobs are packed touching as the reference packs them, centred on the origin, and filled by
 * Poisson-disk sampling (radius 0.01, 30 attempts, seed 42 + blob index) with dx = cbrt(27 x box
 * volume / box samples) and particle volume dx^3 / 27 (sampleParticlesFromVdb).  The blob shape is
 * analytic (the upper half of the superellipsoid |x/R|^2.5 + |y/H|^2.5 + |z/R|^2.5 <= 1, H = 0.55 R)
 * instead of the reference's OpenVDB level sets.  Then everything pm_setup_scene does. */
PM_API pm_status pm_setup_scene_blobs(pm_sim* sim, float fps, const float* color_ratios, const float* latents, uint32_t k,
                                      const char* pigment_config_path, const char* sim_config_path,
                                      const char* anim_path);
/* Simulation::prepareSimulation() (simulation_units.cpp:133-215): material constants, MUSL on,
 * the initial grid (remeshFixedInit(2,2,2)), time = frame = 0.  Uploads objects. */
PM_API pm_status pm_prepare(pm_sim* sim);
/* Simulation::step() (simulation_units.cpp:217-233): one advanceStep, time += dt. */
PM_API pm_status pm_step(pm_sim* sim);
/* nsteps of { step(); frameFinished(); } -- the render loop's idiom (raytracing/src/main.cpp:
 * 270-285) -- on the device without host round trips (CUDA graph replay).  *frames_done, if not
 * NULL, receives the number of frame boundaries crossed. */
PM_API pm_status pm_advance(pm_sim* sim, uint32_t nsteps, uint32_t* frames_done);
/* Simulation::simulate() (simulation.cpp:86-222), the reference's offline driver used by its tests:
 * prepares the scene (material constants, the initial grid, time = frame = 0) and steps until
 * end_frame frames are done, with simulate()'s frame test after every step, on the device (the
 * steps issued after the last frame idle).  The update is USL unless use_musl was set to 1 (the
 * field's own default, simulation.hpp:49; pm_prepare turns MUSL on as prepareSimulation does).
 * max_steps > 0 bounds the run (PM_ERR_STATE when end_frame was not reached); *steps_done, if not
 * NULL, receives the steps taken. */
PM_API pm_status pm_simulate(pm_sim* sim, uint32_t max_steps, uint32_t* steps_done);
/* Simulation::frameFinished() (simulation_units.cpp:235-241): mutates `frame`. */
PM_API pm_status pm_frame_finished(pm_sim* sim, int* finished);
/* Simulation::isFinished() (simulation_units.cpp:243-245). */
PM_API pm_status pm_is_finished(pm_sim* sim, int* finished);
/* Simulation::getGridBoundaries() (simulation_units.cpp:247-255). */
PM_API pm_status pm_get_grid_boundaries(pm_sim* sim, double lo[3], double hi[3]);
/* Simulation::getSpatulaObject() (simulation.hpp:186) as read by the renderer
 * (MPMIntegrationSim.cpp:144-167): world->local transform (row-major 4x4) and the spatula's
 * half width, half thickness, half length.  *exists = 0 when the scene has no knife. */
PM_API pm_status pm_get_knife(pm_sim* sim, int* exists, double inv_transform[16], double half_dims[3]);
/* Device error bits (PM_FLAG_*), accumulated since creation; clear = 1 resets them. */
PM_API pm_status pm_get_error_flags(pm_sim* sim, uint32_t* flags, int clear);
/* Conservation and mixing diagnostics over active particles (simulation.cpp:302-348,
 * MPMIntegrationSim.cpp:48-90): total mass, momentum, mass-weighted mean latent. */
PM_API pm_status pm_get_stats(pm_sim* sim, double* total_mass, double momentum[3], double mean_latent[7],
                       uint32_t* n_active);
/* Grid after the last step in lattice order (debug / parity): origin of node (0,0,0), dims, and
 * per node mass, velocity after the grid update, MUSL velocity, flip, latent[7], shear.  Arrays
 * have dims[0]*dims[1]*dims[2] entries; pass NULL arrays to query origin and dims only. */
PM_API pm_status pm_get_grid(pm_sim* sim, double origin[3], uint32_t dims[3], float* mass, float* v_update,
                      float* v_musl, float* flip, float* latent, float* shear);

/* ---- learned return map (no reference counterpart) -----------------------------------------
 * A 10 -> 64 -> 64 -> 6 GELU MLP predicts the viscoplastic projection of the Perzyna return map
 * (plasticity.cpp:194-229 VMVisc, :292-325 DPVisc) for particles that would need the Newton
 * solve.  Features: trial principal log strains (3), deviatoric strain rate dev(h)/dt (3), yield
 * stress, Perzyna viscosity, flow index, Young's modulus.  Targets: plastic strain h_trial - h (3)
 * and its rate (3).  Parameter vector (PM_MLP_NPARAMS floats): in_mean[10] in_std[10]
 * out_mean[6] out_std[6] W1[64][10] b1[64] W2[64][64] b2[64] W3[6][64] b3[6]. */
#define PM_MLP_NPARAMS 5286
/* Selects the return-map implementation used by pm_step/pm_advance: PM_RETURN_MAP_SURROGATE
 * needs weights from pm_set_surrogate.  Every surrogate estimate is checked against the Perzyna
 * consistency condition (|r| < 1e-2 Pa, the reference's tolerance); estimates that fail drop to
 * the Newton solve (continued from the estimate, or from the reference's initial guess when the
 * parameter "surrogate_fallback_plain" is 1). */
PM_API pm_status pm_set_return_map(pm_sim* sim, int mode);
/* Loads surrogate weights (host array, PM_MLP_NPARAMS floats) for BF16 tensor-core inference. */
PM_API pm_status pm_set_surrogate(pm_sim* sim, const float* params);
/* Turns on logging of (features, targets) for every particle the plain return map solves with
 * Newton, up to `capacity` samples (0 turns it off; the buffer is device memory). */
PM_API pm_status pm_enable_sample_log(pm_sim* sim, uint32_t capacity);
/* Copies up to max_samples logged samples: features[n*10], targets[n*6]; *n = number copied. */
PM_API pm_status pm_get_samples(pm_sim* sim, float* features, float* targets, uint32_t max_samples, uint32_t* n);
/* Return-map statistics of the last step: [0] particles needing the consistency solve,
 * [1] Newton updates taken, [2] particles sent to the surrogate, [3] surrogate estimates that
 * passed the check, [4] samples logged so far. */
PM_API pm_status pm_get_return_map_stats(pm_sim* sim, uint32_t stats[5]);
/* Trains the MLP on the current device with the library's FP32 forward/backward kernels and
 * Adam (cosine learning-rate decay).  x[n*10], y[n*6] host arrays; params (in/out) receives the
 * trained vector (resume = 1 starts from its content, 0 initialises it and the normalisation
 * statistics from the data); loss_history[epochs] (may be NULL) the mean normalised MSE per epoch. */
PM_API pm_status pm_mlp_train(const float* x, const float* y, uint32_t n, uint32_t epochs, uint32_t batch, float lr,
                              uint64_t seed, int resume, float* params, float* loss_history, uint32_t* steps);
/* Normalised mean-squared-error loss and its gradient (grad[PM_MLP_NPARAMS], statistics entries
 * zero) of one batch, computed by the training kernels (for gradient checks). */
PM_API pm_status pm_mlp_loss_grad(const float* params, const float* x, const float* y, uint32_t n, float* loss,
                                  float* grad);
/* Inference through the BF16 tensor-core kernel: x[n*10] -> y[n*6], host arrays. */
PM_API pm_status pm_mlp_infer(const float* params, const float* x, uint32_t n, float* y);

/* ---- diagnostics (no reference counterpart; the reference times phases with gettimeofday,
 * simulation.cpp:247-274) -------------------------------------------------------------------- */
/* The cudaStream_t all of this simulation's work is issued on (for CUDA event timing). */
PM_API pm_status pm_get_stream(pm_sim* sim, void** stream);
/* Name of the i-th kernel of this simulation's step (launch order), "" when out of range. */
PM_API const char* pm_kernel_name(pm_sim* sim, int index);
/* Runs nsteps steps of pm_advance (frame bookkeeping after each) without graphs, timing every
 * kernel with CUDA events on the stream;
 * kernel_ms[i] receives the mean duration of kernel i.  n_kernels must be >= the kernels per
 * step (pm_get_param "kernels_per_step"). */
PM_API pm_status pm_profile_steps(pm_sim* sim, uint32_t nsteps, float* kernel_ms, uint32_t n_kernels);

/* ---- output files and checkpoints -------------------------------------------------------------
 * Simulation::saveParticleData(extra) (save_data.cpp:7-166): binary little-endian PLY
 * `<directory><name>/particles_f<extra><frame>.ply` with float32 vertex properties x y z vx vy vz
 * p q Je, plus eps_pl_vol eps_pl_dev delta_gamma when a plastic model is set (p = -tr(tau)/3,
 * q = q_prefac |dev tau|, Je = det F, tau the Kirchhoff stress of F), and `last_written.txt` with the
 * frame.  <name> is the pm_initialize_basic name; the directory must exist (as in the reference). */
PM_API pm_status pm_save_particle_data(pm_sim* sim, const char* directory, const char* extra);
/* Simulation::saveGridData(extra) (save_data.cpp:168-254): `<directory><name>/grid_f<extra><frame>.ply`
 * with x y z vx vy vz mass for every node of the step's grid box (v: the MUSL velocity). */
PM_API pm_status pm_save_grid_data(pm_sim* sim, const char* directory, const char* extra);
/* Simulation::saveInfo() (save_data.cpp:347-356): `<directory><name>/info.txt`. */
PM_API pm_status pm_save_info(pm_sim* sim, const char* directory);
/* Checkpoints (no reference counterpart): the full particle state (all fields, original order,
 * active flags) and the device control block (time, dt, step, frame, object poses, grid reference
 * box).  Load into a simulation set up like the saved one and prepared; the run then continues as
 * the saved one would.  A checkpoint is tied to the library build that wrote it. */
PM_API pm_status pm_save_checkpoint(pm_sim* sim, const char* path);
PM_API pm_status pm_load_checkpoint(pm_sim* sim, const char* path);

/* Mean latent of the active particles inside the vertical cylinder (x - cx)^2 + (z - cz)^2 <=
 * radius^2 and their count: the sampling of MPMIntegrationSim::calculateAndPrintFinalColor
 * (MPMIntegrationSim.cpp:48-90, centre (0, 0.1, 0) and radius 0.2 there), reduced on the device.
 * The caller turns the mean latent into a colour with Mixbox's latent-to-RGB. */
PM_API pm_status pm_sample_latent_cylinder(pm_sim* sim, double cx, double cz, double radius, double mean_latent[7],
                                           uint32_t* count);

/* ---- scene builder -----------------------------------------------------------------------------
 * sampleParticles (matter/src/sampling/sampling_particles.hpp:12-70) on the GPU: a Poisson-disk set
 * of minimum distance `radius` in [0, Lx] x [0, Ly] x [0, Lz] (parallel dart throwing on a grid of
 * cells of side radius / sqrt(3), 27 independent phases, `attempts` darts per cell and `passes`
 * sweeps; deterministic for a seed), cropped like the reference (0 box, 1 cylinder of diameter Lx
 * around the y axis through the box centre, 2 the silo r = tanh(y) + 1), with dx =
 * cbrt(ppc / N_box * Lx Ly Lz) and particle volume dx^3 / ppc.  x: n*3 floats or NULL to only count. */
PM_API pm_status pm_sample_particles(int device, double Lx, double Ly, double Lz, double radius, double ppc,
                                     int crop_to_shape, uint32_t attempts, uint32_t passes, uint32_t seed, float* x,
                                     uint32_t capacity, uint32_t* n, double* dx, double* particle_volume);

/* ---- self-test of the device SVD --------------------------------------------------------------
 * No counterpart in the reference (it calls Eigen's JacobiSVD, plasticity.cpp:18).  Runs the step's
 * warm-started FP64 SVD on n host matrices A (row-major 3x3, FP64): A = U diag(S) V^T with S >= 0
 * in FP64 and U, V rounded to FP32, as the return map uses them. */
PM_API pm_status pm_svd3_batch(int device, const double* A, uint32_t n, float* U, double* S, float* V);

/* ---- headless pigment splat --------------------------------------------------------------------
 * BinaryDensityGrid::fillRenderGrid (raytracing/src/raymarch/BinaryDensityGrid.cpp:153-296) without
 * the GL upload: the two-pass anisotropic bilateral splat of the particle latents onto the pigment
 * grid, whose voxels are a quarter of the density voxel (the support radius 2 dx,
 * MPMIntegrationSim.cpp:96-98) over the grid boundaries (AABBc.cpp:10-25).  voxels[dims z][y][x][8]
 * receives latent 7 + weight per voxel; NULL only fills dims, origin and voxel_size.  G: per-particle
 * 3x3 anisotropy matrices (row-major, original particle order) or NULL for the isotropic I / h the
 * reference uses for sparse neighbourhoods.  device_ptrs: G and voxels are device pointers. */
PM_API pm_status pm_splat_pigments(pm_sim* sim, const float* G, int device_ptrs, float sigma_spatial,
                                   float sigma_color, float* voxels, uint32_t dims[3], double origin[3],
                                   double* voxel_size);

/* ---- renderer preprocessing: binary density grid and anisotropy ---------------------------------
 * BinaryDensityGrid::fillCells / generateNc / fillBDG (raytracing/src/raymarch/BinaryDensityGrid.cpp:
 * 22-151) on the density voxels of AABBc::fixedAABB (side h = 2 dx over the grid boundaries):
 * particle counts per voxel, the separable neighbour filter with weights a (voxel) and b (each
 * neighbour; the reference's state.params 0.75, 0.74), occupancy M = (nc 315/(64 pi h^3) >= iso)
 * (reference iso 9285; test_all_filled sets every voxel), and M2 / M4, the OR of M over 2^3 and
 * 4^3 blocks.  Voxel v = x + X (y + Y z); M2 and M4 have ceil(X/2) x ceil(Y/2) x ceil(Z/2) and
 * ceil(X/4) x ... entries.  cell_count / cell_offset (per voxel) and ids (particle indices of the
 * binned particles, grouped by voxel; order inside a voxel unspecified) are the binning itself;
 * each output may be NULL.  M == NULL only fills dims, origin and voxel_size.  occupancy[2]
 * receives the counts of empty and occupied voxels (state.count).  device_ptrs: the arrays are
 * device pointers. */
PM_API pm_status pm_density_grid(pm_sim* sim, float a, float b, float iso, int test_all_filled, int device_ptrs,
                                 uint32_t* M, uint32_t* M2, uint32_t* M4, uint32_t* cell_count,
                                 uint32_t* cell_offset, uint32_t* ids, uint32_t dims[3], double origin[3],
                                 double* voxel_size, uint32_t occupancy[2]);
/* Classification::countMatrix / countCurrDens (raytracing/src/raymarch/Classification.cpp:38-130):
 * per particle (original order) the anisotropy matrix G (3x3, row-major, symmetric), its inverse,
 * |det G| and the anisotropic density, from the neighbours within h found through the binning.
 * Parameters are the reference's state.s (1400), state.k (4), state.aniso_threshold (15),
 * state.autoScaleS (1) and state.isAni (1); iso (9285) counts the aggregate particles
 * (density > iso) into n_aggregate.  Outputs may be NULL.  device_ptrs: the arrays are device
 * pointers; G from here feeds pm_splat_pigments. */
PM_API pm_status pm_anisotropy(pm_sim* sim, float s, float k, int threshold, int auto_scale, int is_ani, float iso,
                               int device_ptrs, float* G, float* G_inv, float* det, float* density,
                               uint32_t* n_aggregate);

/* ---- batched scenes --------------------------------------------------------------------------
 * No counterpart in the reference, which runs one Simulation per process
 * (R/src/mpm/MPMIntegrationSim.cpp:16-38 creates one).  A batch steps many independent, prepared
 * simulations on one GPU together: every kernel of the step is launched once for all scenes,
 * its CTAs statically partitioned across the scenes in proportion to their work and looping over
 * their scene's particles, bricks or nodes; one round (one step of every scene) is captured as a
 * CUDA graph and replayed.  Scenes keep their own dt, time, frame, grid box and capacity; a scene
 * whose grid overflows sits rounds out until the host has regrown it, so pm_batch_step(n) ends
 * with every scene exactly n steps further.  A batch step is an advance (frame bookkeeping after
 * every step, as pm_advance).  The batch references the simulations (it does not
 * own them): destroy the batch first.  While a batch step runs, the member simulations must not
 * be used on other threads; between batch steps every per-scene call works as usual. */
typedef struct pm_batch pm_batch;

/* Launch shapes of the batched kernels (what pm_batch_autotune picks). */
typedef struct pm_batch_tuning {
  int32_t flat_threads;      /* block size of the flat kernels: 128, 256 or 512 */
  int32_t part_ctas_per_sm;  /* CTAs per SM, particle-parallel flat kernels (count, scatter) */
  int32_t node_ctas_per_sm;  /* CTAs per SM, node-parallel flat kernels (clear, grid update) */
  int32_t p2g_ctas_per_sm;   /* CTAs per SM of P2G, G2P+MUSL, deformation update, surrogate */
  int32_t g2p_ctas_per_sm;
  int32_t def_ctas_per_sm;
  int32_t sur_ctas_per_sm;
  int32_t chunk_rounds;      /* rounds replayed between host checks of the control blocks */
} pm_batch_tuning;

PM_API pm_status pm_batch_create(pm_sim* const* scenes, uint32_t n, pm_batch** out);
PM_API pm_status pm_batch_destroy(pm_batch* batch);
/* Advances every scene by nsteps steps. */
PM_API pm_status pm_batch_step(pm_batch* batch, uint32_t nsteps);
PM_API pm_status pm_batch_get_tuning(pm_batch* batch, pm_batch_tuning* tuning);
PM_API pm_status pm_batch_set_tuning(pm_batch* batch, const pm_batch_tuning* tuning);
/* Coordinate search over the launch shapes: each candidate is timed with CUDA events over
 * trial_rounds rounds (which advance the scenes like pm_batch_step), the fastest is kept and
 * returned in best (may be NULL) with its time per round in best_ms (may be NULL). */
PM_API pm_status pm_batch_autotune(pm_batch* batch, uint32_t trial_rounds, pm_batch_tuning* best, float* best_ms);
/* The stream the batch issues its work on, for CUDA event timing. */
PM_API pm_status pm_batch_get_stream(pm_batch* batch, void** stream);
/* Kernels per round and their names in launch order. */
PM_API int32_t pm_batch_kernels_per_round(pm_batch* batch);
PM_API const char* pm_batch_kernel_name(pm_batch* batch, int index);
/* Runs `rounds` rounds without the graph, timing every kernel with CUDA events; kernel_ms[i]
 * receives the mean duration of kernel i (n_kernels >= pm_batch_kernels_per_round). */
PM_API pm_status pm_batch_profile(pm_batch* batch, uint32_t rounds, float* kernel_ms, uint32_t n_kernels);

/* ---- particle-to-grid transfer that allocates nothing --------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc: plug-ins whose host
 * application owns every device allocation (a caching allocator or a fixed memory budget), loops
 * that may not allocate once running, callers holding only raw device arrays.
 * It scatters caller-owned particle arrays onto a caller-described node box with the step's
 * P2G transfer (quadratic B-splines, counting sort by cell, one warp per cell) and the
 * reference's normalisation (p2g.cpp:97-124).  Inputs and outputs are device pointers:
 * x[n*3], v[n*3], B[n*9] (APIC matrix, NULL = none), latent[n*7], diffusion[n]; node (i,j,k) sits
 * at origin + (i,j,k)*dx and is entry (i*dims[1] + j)*dims[2] + k of node_mass[nodes],
 * node_velocity[nodes*3], node_latent[nodes*7], node_shear[nodes] (any output may be NULL).
 * All n particles are treated as active (no active mask, unlike p2g.cpp:22).
 * Scratch is one fixed 8 MiB __device__ array inside the library (held by every GPU that loads
 * it until exit): at most 131072 particles and 131072 nodes per call, PM_ERR_CAPACITY beyond.
 * The first call on a device looks up that array's device address (a synchronous runtime query).
 * All calls share the array: calls whose work overlaps on the GPU race.  Work is queued on
 * `stream` (NULL = default stream).  When `outside` is not NULL the call synchronises `stream`
 * and stores the number of particles skipped because their stencil left the box or a coordinate
 * was not finite. */
PM_API pm_status pm_p2g_noalloc(const float* x, const float* v, const float* B, const float* latent,
                                const float* diffusion, uint32_t n, double particle_mass, double dx,
                                const double origin[3], const int32_t dims[3], float* node_mass,
                                float* node_velocity, float* node_latent, float* node_shear, void* stream,
                                uint32_t* outside);

#ifdef __cplusplus
}
#endif

#endif /* PIGMENT_MPM_H */

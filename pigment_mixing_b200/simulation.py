"""Python mirror of the reference ``Simulation`` class (matter/src/simulation/simulation.hpp:25-186)
on top of the C ABI.  Method names follow the reference; public fields are properties that set
the same-named parameters through ``pm_set_param``.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from ._lib import call

# matter/src/tools.hpp:55-59
PLATE_TOP, PLATE_BOTTOM, PLATE_LEFT, PLATE_RIGHT, PLATE_FRONT, PLATE_BACK = range(6)
BC_NOSLIP, BC_SLIPSTICK, BC_SLIPFREE = range(3)
NO_PLASTICITY, VM, DP, DPSOFT, MCC, VMVISC, DPVISC, MCCVISC, DPMUI, MCCMUI = range(10)
RETURN_MAP_PLAIN, RETURN_MAP_SURROGATE = 0, 1

_SCALARS = ("cfl", "cfl_elastic", "flip_ratio", "rho", "E", "nu", "fps", "end_frame", "min_dt", "dx",
            "particle_mass", "particle_volume", "plastic_model", "use_pradhana", "use_musl",
            "use_particle_boundaries", "q_max", "q_min", "p_min", "M", "q_cohesion", "perzyna_exp",
            "perzyna_visc", "xi", "q_prefac", "pigment_D_max", "pigment_D_edge0", "pigment_D_edge1",
            "start_boost_time", "end_boost_time", "boost_factor", "auto_frame", "surrogate_fallback_plain",
            "sample_log_every")
_READONLY = ("time", "dt", "step", "Np", "mu", "lambda", "K", "dt_max", "frame_dt", "final_time",
             "n_active", "plastic_count", "grid_nodes", "frame", "kernels_per_step", "regrowths", "regrow_ms",
             "grid_capacity_nodes", "alloc_ms", "graph_ms")
_VECTORS = ("gravity", "particle_boundary_min", "particle_boundary_max", "grid_reference_point")


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def _fp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


class Particles:
    """Host copy of the particle state in the original particle order (data_structures.hpp:9-50)."""

    def __init__(self, d: dict):
        self.__dict__.update(d)


class Simulation:
    """One MPM scene on one GPU.  Mirrors ``Simulation`` (simulation.hpp:25-186)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        call("pm_create", device, C.byref(h))
        self._h = h
        self._np = 0
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            call("pm_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- public fields ---------------------------------------------------------------------
    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        if name in _SCALARS or name in _READONLY:
            out = C.c_double()
            call("pm_get_param", self._h, name.encode(), C.byref(out))
            return out.value
        raise AttributeError(name)

    def param(self, name: str) -> float:
        """Any scalar of pm_get_param by name (e.g. "step", which the step() method shadows)."""
        out = C.c_double()
        call("pm_get_param", self._h, name.encode(), C.byref(out))
        return out.value

    @property
    def steps_done(self) -> int:
        """Steps completed so far (the control block's step counter)."""
        return int(self.param("step"))

    def __setattr__(self, name, value):
        if name.startswith("_"):
            object.__setattr__(self, name, value)
        elif name in _SCALARS or name == "frame":
            call("pm_set_param", self._h, name.encode(), float(value))
        elif name in _VECTORS:
            v = np.ascontiguousarray(value, dtype=np.float64).reshape(3)
            call("pm_set_param3", self._h, name.encode(), _dp(v))
        else:
            object.__setattr__(self, name, value)

    def set(self, **kw) -> "Simulation":
        for k, v in kw.items():
            setattr(self, k, v)
        return self

    @property
    def Np(self) -> int:
        return self._np

    # ---- reference API -----------------------------------------------------------------------
    def initializeBasic(self, name: str) -> None:  # simulation_units.cpp:9-26
        call("pm_initialize_basic", self._h, name.encode())

    def loadPigmentConfig(self, path: str) -> None:  # simulation_units.cpp:31-48
        call("pm_load_pigment_config", self._h, path.encode())

    def loadSimConfig(self, path: str) -> None:  # simulation_units.cpp:50-80
        call("pm_load_sim_config", self._h, path.encode())

    def setParticles(self, x, latent=None, v=None) -> None:
        x = _f32(x).reshape(-1, 3)
        n = x.shape[0]
        lat = None if latent is None else _f32(latent).reshape(n, 7)
        vv = None if v is None else _f32(v).reshape(n, 3)
        call("pm_set_particles", self._h, n, _fp(x), _fp(lat), _fp(vv))
        self._np = n

    def setupScene(self, fps: float, pigment_config: Optional[str] = None, sim_config: Optional[str] = None,
                   anim_path: Optional[str] = None) -> None:  # simulation_units.cpp:28-131
        enc = lambda s: None if s is None else s.encode()
        call("pm_setup_scene", self._h, float(fps), enc(pigment_config), enc(sim_config), enc(anim_path))

    def setupSceneBlobs(self, fps: float, color_ratios, latents, pigment_config: Optional[str] = None,
                        sim_config: Optional[str] = None, anim_path: Optional[str] = None) -> None:
        """setupScene(fps, colorRatios, pigments, anim_path) with the blob scene built by the library
        (pm_setup_scene_blobs): one blob per colour ratio, latents[k, 7] their Mixbox latents."""
        r = _f32(color_ratios).reshape(-1)
        lat = _f32(latents).reshape(len(r), 7)
        enc = lambda s: None if s is None else s.encode()  # noqa: E731
        call("pm_setup_scene_blobs", self._h, float(fps), _fp(r), _fp(lat), len(r), enc(pigment_config),
             enc(sim_config), enc(anim_path))
        n = C.c_double()
        call("pm_get_param", self._h, b"Np", C.byref(n))
        self._np = int(n.value)

    def prepareSimulation(self) -> None:  # simulation_units.cpp:133-215
        call("pm_prepare", self._h)

    def step(self) -> None:  # simulation_units.cpp:217-233
        call("pm_step", self._h)

    def advance(self, nsteps: int) -> int:
        """nsteps of step() + frameFinished() on the device; returns frames finished."""
        fd = C.c_uint32()
        call("pm_advance", self._h, int(nsteps), C.byref(fd))
        return fd.value

    def simulate(self, max_steps: int = 0) -> int:  # simulation.cpp:86-222
        """The reference's offline driver: prepare, then step until end_frame frames are done
        (USL unless use_musl was set to 1).  max_steps > 0 bounds the run.  Returns the steps taken."""
        n = C.c_uint32()
        call("pm_simulate", self._h, int(max_steps), C.byref(n))
        return n.value

    def frameFinished(self) -> bool:  # simulation_units.cpp:235-241
        o = C.c_int()
        call("pm_frame_finished", self._h, C.byref(o))
        return bool(o.value)

    def isFinished(self) -> bool:  # simulation_units.cpp:243-245
        o = C.c_int()
        call("pm_is_finished", self._h, C.byref(o))
        return bool(o.value)

    def getGridBoundaries(self):  # simulation_units.cpp:247-255
        lo, hi = np.zeros(3), np.zeros(3)
        call("pm_get_grid_boundaries", self._h, _dp(lo), _dp(hi))
        return lo, hi

    def getSpatulaObject(self):  # simulation.hpp:186 as read in MPMIntegrationSim.cpp:144-167
        ex = C.c_int()
        inv, half = np.zeros(16), np.zeros(3)
        call("pm_get_knife", self._h, C.byref(ex), _dp(inv), _dp(half))
        if not ex.value:
            return None
        return inv.reshape(4, 4), half

    # ---- objects -----------------------------------------------------------------------------
    def addPlate(self, pos, plate_type, bc=BC_NOSLIP, friction=0.0, pos_lower=-1e15, pos_upper=1e15, vx=0.0,
                 vy=0.0, vz=0.0, vmin_factor=1.0, load_factor=0.0) -> None:  # object_plate.hpp:13-28
        call("pm_add_plate", self._h, float(pos), int(plate_type), int(bc), float(friction), float(pos_lower),
             float(pos_upper), float(vx), float(vy), float(vz), float(vmin_factor), float(load_factor))

    def addSpatula(self, bc, friction, frames=None, anim_path: Optional[str] = None) -> None:
        if anim_path is not None:
            call("pm_add_spatula_file", self._h, int(bc), float(friction), anim_path.encode())
        else:
            fr = _f32(frames).reshape(-1, 7)
            call("pm_add_spatula", self._h, int(bc), float(friction), _fp(fr), fr.shape[0])

    def addBoxKnife(self, bc, friction, half, waypoints, speed, quat_wxyz=None) -> None:
        h = np.ascontiguousarray(half, dtype=np.float64)
        w = np.ascontiguousarray(waypoints, dtype=np.float64).reshape(-1, 3)
        q = None if quat_wxyz is None else np.ascontiguousarray(quat_wxyz, dtype=np.float64)
        call("pm_add_box_knife", self._h, int(bc), float(friction), _dp(h), _dp(w), w.shape[0], float(speed), _dp(q))

    def addGround(self, bc, friction, y0=0.0) -> None:  # object_ground.hpp:14
        call("pm_add_ground", self._h, int(bc), float(friction), float(y0))

    def addCurve(self, bc, friction) -> None:  # object_curve.hpp:13
        call("pm_add_curve", self._h, int(bc), float(friction))

    def setReturnMap(self, mode: int) -> None:
        call("pm_set_return_map", self._h, int(mode))

    def setSurrogate(self, params) -> None:
        """Load surrogate MLP weights (PM_MLP_NPARAMS floats, see pigment_mixing_b200.surrogate)."""
        p = _f32(params).reshape(-1)
        call("pm_set_surrogate", self._h, _fp(p))

    def enableSampleLog(self, capacity: int) -> None:
        call("pm_enable_sample_log", self._h, int(capacity))

    def samples(self, max_samples: int = 1 << 26):
        """(features[n,10], targets[n,6]) logged by the plain return map."""
        st = self.returnMapStats()
        m = min(int(st["logged"]), int(max_samples))
        x = np.zeros((max(m, 1), 10), np.float32)
        y = np.zeros((max(m, 1), 6), np.float32)
        n = C.c_uint32()
        call("pm_get_samples", self._h, _fp(x), _fp(y), m, C.byref(n))
        return x[: n.value], y[: n.value]

    def returnMapStats(self) -> dict:
        a = np.zeros(5, np.uint32)
        call("pm_get_return_map_stats", self._h, a.ctypes.data_as(C.POINTER(C.c_uint32)))
        return dict(solves=int(a[0]), newton_iters=int(a[1]), queued=int(a[2]), accepted=int(a[3]), logged=int(a[4]))

    # ---- readback ------------------------------------------------------------------------------
    def getParticles(self, fields=("x", "v", "latent", "diffusion", "active")) -> Particles:
        n = self._np
        shapes = dict(x=(n, 3), v=(n, 3), latent=(n, 7), diffusion=(n,), F=(n, 3, 3), B=(n, 3, 3), plastic=(n, 4))
        arrs = {k: np.zeros(shapes[k], np.float32) for k in shapes if k in fields}
        act = np.zeros(n, np.uint8) if "active" in fields else None
        call("pm_get_particles", self._h, _fp(arrs.get("x")), _fp(arrs.get("v")), _fp(arrs.get("latent")),
             _fp(arrs.get("diffusion")), None if act is None else act.ctypes.data_as(C.POINTER(C.c_uint8)),
             _fp(arrs.get("F")), _fp(arrs.get("B")), _fp(arrs.get("plastic")))
        if act is not None:
            arrs["active"] = act
        return Particles(arrs)

    def readInto(self, x=None, latent=None, diffusion=None, v=None) -> None:
        """Copy particle fields into caller-owned float32 arrays (e.g. pinned host buffers)."""
        call("pm_get_particles", self._h, _fp(x), _fp(v), _fp(latent), _fp(diffusion), None, None, None, None)

    def readIntoAsync(self, x=None, latent=None, diffusion=None, v=None) -> None:
        """Start copying particle fields into caller-owned (pinned) float32 arrays; steps issued
        afterwards overlap the copy.  Call waitReadback() before using the arrays."""
        call("pm_get_particles_async", self._h, _fp(x), _fp(v), _fp(latent), _fp(diffusion), None)

    def waitReadback(self) -> None:
        call("pm_wait_particles", self._h)

    @property
    def particles(self) -> Particles:
        return self.getParticles()

    def stream(self) -> int:
        """cudaStream_t (as an integer) on which all of this simulation's kernels run."""
        p = C.c_void_p()
        call("pm_get_stream", self._h, C.byref(p))
        return p.value or 0

    def profileSteps(self, nsteps: int) -> dict:
        """Mean CUDA-event duration (ms) of every kernel of a step over nsteps steps."""
        from ._lib import lib
        k = int(self.kernels_per_step)
        ms = np.zeros(k, np.float32)
        call("pm_profile_steps", self._h, int(nsteps), _fp(ms), k)
        return {lib().pm_kernel_name(self._h, i).decode(): float(ms[i]) for i in range(k)}

    # ---- output files (save_data.cpp) and checkpoints ----------------------------------------
    def saveParticleData(self, directory: str, extra: str = "") -> None:
        """Binary PLY `<directory><name>/particles_f<extra><frame>.ply` (save_data.cpp:7-166)."""
        call("pm_save_particle_data", self._h, directory.encode(), extra.encode())

    def saveGridData(self, directory: str, extra: str = "") -> None:
        """Binary PLY `<directory><name>/grid_f<extra><frame>.ply` (save_data.cpp:168-254)."""
        call("pm_save_grid_data", self._h, directory.encode(), extra.encode())

    def saveInfo(self, directory: str) -> None:
        call("pm_save_info", self._h, directory.encode())

    def sampleLatentCylinder(self, cx: float = 0.0, cz: float = 0.0, radius: float = 0.2):
        """(mean latent[7], count) of the active particles in a vertical cylinder (the final-colour
        sampling of MPMIntegrationSim.cpp:48-90)."""
        m = np.zeros(7)
        n = C.c_uint32()
        call("pm_sample_latent_cylinder", self._h, float(cx), float(cz), float(radius), _dp(m), C.byref(n))
        return m, n.value

    def splatPigments(self, sigma_spatial: float = 0.5, sigma_color: float = 0.2, G=None, out=None):
        """The renderer's pigment volume (BinaryDensityGrid::fillRenderGrid) without GL.  Returns
        (voxels[z][y][x][8] float32: latent 7 + weight, origin[3], voxel size).  G: optional
        per-particle 3x3 anisotropy matrices (n x 3 x 3, original order); out: optional device
        tensor (torch, float32, contiguous) to fill in place instead of a host array."""
        dims = np.zeros(3, np.uint32)
        origin = np.zeros(3)
        vs = C.c_double()
        up = dims.ctypes.data_as(C.POINTER(C.c_uint32))
        call("pm_splat_pigments", self._h, None, 0, sigma_spatial, sigma_color, None, up, _dp(origin), C.byref(vs))
        shape = (int(dims[2]), int(dims[1]), int(dims[0]), 8)
        if out is not None:
            assert tuple(out.shape) == shape and out.is_cuda and out.is_contiguous()
            gptr = None
            if G is not None:
                gptr = C.c_void_p(G.data_ptr())
            call("pm_splat_pigments", self._h, gptr, 1, sigma_spatial, sigma_color, C.c_void_p(out.data_ptr()), up,
                 _dp(origin), C.byref(vs))
            return out, origin, vs.value
        vox = np.zeros(shape, np.float32)
        g = None if G is None else np.ascontiguousarray(G, np.float32).reshape(-1, 9)
        call("pm_splat_pigments", self._h, None if g is None else g.ctypes.data_as(C.c_void_p), 0, sigma_spatial,
             sigma_color, vox.ctypes.data_as(C.c_void_p), up, _dp(origin), C.byref(vs))
        return vox, origin, vs.value

    def densityGrid(self, a: float = 0.75, b: float = 0.74, iso: float = 9285.0, test_all_filled: bool = False,
                    device: bool = False) -> dict:
        """The renderer's binary density grid (BinaryDensityGrid::fillBDG) over the density voxels
        (side 2 dx): occupancy M and its 2^3 / 4^3 ORs M2 / M4 (voxel order x + X (y + Y z)), the
        per-voxel particle counts and offsets, the binned particle indices grouped by voxel, and
        the (empty, occupied) voxel counts.  device=True returns M, M2, M4 as torch tensors on
        the simulation's GPU and skips the binning arrays."""
        dims = np.zeros(3, np.uint32)
        origin = np.zeros(3)
        vs = C.c_double()
        up = dims.ctypes.data_as(C.POINTER(C.c_uint32))
        call("pm_density_grid", self._h, a, b, iso, int(test_all_filled), 0, None, None, None, None, None, None, up,
             _dp(origin), C.byref(vs), None)
        X, Y, Z = (int(v) for v in dims)
        n = X * Y * Z
        if device:
            import torch
            dev = f"cuda:{self.device}"
            M = torch.empty(n, dtype=torch.int32, device=dev)
            M2 = torch.empty(((X + 1) // 2) * ((Y + 1) // 2) * ((Z + 1) // 2), dtype=torch.int32, device=dev)
            M4 = torch.empty(((X + 3) // 4) * ((Y + 3) // 4) * ((Z + 3) // 4), dtype=torch.int32, device=dev)
            occ = np.zeros(2, np.uint32)
            ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
            call("pm_density_grid", self._h, a, b, iso, int(test_all_filled), 1, ptr(M), ptr(M2), ptr(M4), None, None,
                 None, up, _dp(origin), C.byref(vs), occ.ctypes.data_as(C.POINTER(C.c_uint32)))
            return dict(M=M, M2=M2, M4=M4, dims=dims.copy(), origin=origin, voxel_size=vs.value,
                        occupancy=(int(occ[0]), int(occ[1])))
        M = np.zeros(n, np.uint32)
        M2 = np.zeros(((X + 1) // 2) * ((Y + 1) // 2) * ((Z + 1) // 2), np.uint32)
        M4 = np.zeros(((X + 3) // 4) * ((Y + 3) // 4) * ((Z + 3) // 4), np.uint32)
        counts, offsets = np.zeros(n, np.uint32), np.zeros(n, np.uint32)
        ids = np.zeros(self.Np, np.uint32)
        occ = np.zeros(2, np.uint32)
        vp = lambda a_: a_.ctypes.data_as(C.c_void_p)  # noqa: E731
        call("pm_density_grid", self._h, a, b, iso, int(test_all_filled), 0, vp(M), vp(M2), vp(M4), vp(counts),
             vp(offsets), vp(ids), up, _dp(origin), C.byref(vs), occ.ctypes.data_as(C.POINTER(C.c_uint32)))
        return dict(M=M, M2=M2, M4=M4, counts=counts, offsets=offsets, ids=ids[:int(counts.sum())], dims=dims.copy(),
                    origin=origin, voxel_size=vs.value, occupancy=(int(occ[0]), int(occ[1])))

    def anisotropy(self, s: float = 1400.0, k: float = 4.0, threshold: int = 15, auto_scale: bool = True,
                   is_ani: bool = True, iso: float = 9285.0, device: bool = False) -> dict:
        """The renderer's per-particle anisotropy matrices G (n x 3 x 3, symmetric), their inverses,
        |det G| and anisotropic densities (Classification::countDensities), original particle
        order, and the count of aggregate particles (density > iso).  device=True returns torch
        tensors on the simulation's GPU (G ready for splatPigments(G=..., out=...))."""
        n = self.Np
        agg = C.c_uint32()
        if device:
            import torch
            dev = f"cuda:{self.device}"
            G = torch.empty((n, 3, 3), dtype=torch.float32, device=dev)
            Gi = torch.empty((n, 3, 3), dtype=torch.float32, device=dev)
            det = torch.empty(n, dtype=torch.float32, device=dev)
            dens = torch.empty(n, dtype=torch.float32, device=dev)
            ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
            call("pm_anisotropy", self._h, s, k, threshold, int(auto_scale), int(is_ani), iso, 1, ptr(G), ptr(Gi),
                 ptr(det), ptr(dens), C.byref(agg))
        else:
            G = np.zeros((n, 3, 3), np.float32)
            Gi = np.zeros((n, 3, 3), np.float32)
            det = np.zeros(n, np.float32)
            dens = np.zeros(n, np.float32)
            ptr = lambda a_: a_.ctypes.data_as(C.c_void_p)  # noqa: E731
            call("pm_anisotropy", self._h, s, k, threshold, int(auto_scale), int(is_ani), iso, 0, ptr(G), ptr(Gi),
                 ptr(det), ptr(dens), C.byref(agg))
        return dict(G=G, G_inv=Gi, det=det, density=dens, n_aggregate=int(agg.value))

    def saveCheckpoint(self, path: str) -> None:
        call("pm_save_checkpoint", self._h, path.encode())

    def loadCheckpoint(self, path: str) -> None:
        """Restore a checkpoint into this (identically set up, prepared) simulation."""
        call("pm_load_checkpoint", self._h, path.encode())

    def errorFlags(self, clear: bool = False) -> int:
        f = C.c_uint32()
        call("pm_get_error_flags", self._h, C.byref(f), int(clear))
        return f.value

    def stats(self) -> dict:
        m = C.c_double()
        mom, lat = np.zeros(3), np.zeros(7)
        na = C.c_uint32()
        call("pm_get_stats", self._h, C.byref(m), _dp(mom), _dp(lat), C.byref(na))
        return dict(mass=m.value, momentum=mom, mean_latent=lat, n_active=na.value)

    def grid(self) -> dict:
        origin = np.zeros(3)
        dims = np.zeros(3, np.uint32)
        call("pm_get_grid", self._h, _dp(origin), dims.ctypes.data_as(C.POINTER(C.c_uint32)), None, None, None, None,
             None, None)
        n = int(np.prod(dims.astype(np.int64)))
        out = dict(origin=origin, dims=dims.astype(int), mass=np.zeros(n, np.float32),
                   v_update=np.zeros((n, 3), np.float32), v_musl=np.zeros((n, 3), np.float32),
                   flip=np.zeros((n, 3), np.float32), latent=np.zeros((n, 7), np.float32),
                   shear=np.zeros(n, np.float32))
        call("pm_get_grid", self._h, _dp(origin), dims.ctypes.data_as(C.POINTER(C.c_uint32)), _fp(out["mass"]),
             _fp(out["v_update"]), _fp(out["v_musl"]), _fp(out["flip"]), _fp(out["latent"]), _fp(out["shear"]))
        return out


class Batch:
    """Independent prepared scenes stepped together on one GPU (``pm_batch_*``): every kernel of
    the step is launched once for all scenes, one round is a CUDA graph.  The batch references the
    simulations; close it before them."""

    def __init__(self, sims):
        self._sims = list(sims)
        arr = (C.c_void_p * len(self._sims))(*[s._h.value for s in self._sims])
        h = C.c_void_p()
        call("pm_batch_create", arr, len(self._sims), C.byref(h))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            call("pm_batch_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def scenes(self):
        return list(self._sims)

    def step(self, nsteps: int) -> None:
        """Advance every scene by nsteps steps."""
        call("pm_batch_step", self._h, int(nsteps))

    def tuning(self) -> dict:
        from ._lib import BatchTuning
        t = BatchTuning()
        call("pm_batch_get_tuning", self._h, C.byref(t))
        return t.as_dict()

    def setTuning(self, **kw) -> None:
        from ._lib import BatchTuning
        t = BatchTuning()
        call("pm_batch_get_tuning", self._h, C.byref(t))
        for k, v in kw.items():
            setattr(t, k, int(v))
        call("pm_batch_set_tuning", self._h, C.byref(t))

    def autotune(self, trial_rounds: int = 4):
        """Search the launch shapes (advances the scenes); returns (tuning, ms per round)."""
        from ._lib import BatchTuning
        t = BatchTuning()
        ms = C.c_float()
        call("pm_batch_autotune", self._h, int(trial_rounds), C.byref(t), C.byref(ms))
        return t.as_dict(), float(ms.value)

    def stream(self) -> int:
        p = C.c_void_p()
        call("pm_batch_get_stream", self._h, C.byref(p))
        return p.value or 0

    @property
    def kernels_per_round(self) -> int:
        from ._lib import lib
        return int(lib().pm_batch_kernels_per_round(self._h))

    def profile(self, rounds: int) -> dict:
        """Mean CUDA-event duration (ms) of every batched kernel over `rounds` rounds."""
        from ._lib import lib
        k = self.kernels_per_round
        ms = np.zeros(k, np.float32)
        call("pm_batch_profile", self._h, int(rounds), _fp(ms), k)
        return {lib().pm_batch_kernel_name(self._h, i).decode(): float(ms[i]) for i in range(k)}

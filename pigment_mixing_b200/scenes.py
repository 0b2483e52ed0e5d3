"""Seeded synthetic palette scenes (the workloads the step is measured and checked on).

The reference builds its paint scene from OpenVDB blob level sets with Poisson-disk sampling
(matter/src/simulation/simulation_blobs.cpp:7-150, 27 particles per cell); those assets and
libraries are not used here.  The measured workloads place cuboid paint blocks of 8 jittered
particles per cell (2 x 2 x 2 sub-cells, uniform jitter inside each), all from a seed;
``blob_scene`` restates the reference's blob recipe with analytic dome-shaped blobs.

A scene is a plain dict that ``apply(scene, sim)`` loads into any object with the Simulation
call surface (the product :class:`Simulation` or the CPU oracle).
"""
from __future__ import annotations

import numpy as np

# Mixbox latents (rgb -> 7-float latent: 4 pigment concentrations + 3 RGB residuals) of the scene
# colours, as computed by Mixbox's float_rgb_to_latent for these sRGB triples.
MIXBOX_LATENTS = {
    (0.99, 0.86, 0.08): [0.003921568393707275, 0.8289437890052795, 0.0, 0.16713464260101318,
                         0.02399754524230957, 0.03179413080215454, -0.01334661990404129],
    (0.10, 0.20, 0.60): [0.7396079301834106, 0.02299606241285801, 0.07450980693101883, 0.16288620233535767,
                         0.0012317672371864319, -0.0003674924373626709, -0.0024244189262390137],
    (0.80, 0.10, 0.12): [0.002337253885343671, 0.0262086670845747, 0.8995293974876404, 0.07192468643188477,
                         0.003439664840698242, -0.0034313425421714783, 0.0016628801822662354],
    (0.05, 0.45, 0.25): [0.5207844376564026, 0.42559564113616943, 0.0, 0.05361992120742798,
                         -0.03620488569140434, 0.015082001686096191, 0.0036397576332092285],
    (0.95, 0.95, 0.93): [0.02470589615404606, 0.02636185847222805, 0.01235294807702303, 0.9365792870521545,
                         0.0021063685417175293, 0.00013774633407592773, -0.0014260411262512207],
    (0.45, 0.25, 0.05): [0.26009073853492737, 0.280588299036026, 0.45912498235702515, 0.00019598007202148438,
                         -0.0287514328956604, 0.02641358971595764, -0.08001551032066345],
}

RGB_SEEDS = list(MIXBOX_LATENTS)

# pigment_config.json of the reference (matter/pigment_config.json)
PIGMENT_CONFIG = dict(pigment_D_max=50.0, pigment_D_edge0=1.5, pigment_D_edge1=7.0, start_boost_time=15.0,
                      end_boost_time=30.0, boost_factor=3.0)


def jittered_block(lo, ncells, dx, rng, per_axis=2):
    """Particles at per_axis^3 sub-cells of every cell of a box, uniformly jittered inside each."""
    n = np.asarray(ncells, dtype=np.int64)
    sub = dx / per_axis
    idx = np.stack(np.meshgrid(*[np.arange(k * per_axis) for k in n], indexing="ij"), -1).reshape(-1, 3)
    return (np.asarray(lo, np.float64) + (idx + rng.uniform(0.0, 1.0, idx.shape)) * sub).astype(np.float32)


def knife_path(rng, x_mid, y_c, z_lo, z_hi, segments=3, drift=0.1):
    """A seeded piecewise-linear knife path sweeping back and forth through the paint along z."""
    pts = []
    for i in range(segments + 1):
        z = z_lo if i % 2 == 0 else z_hi
        pts.append([x_mid + rng.uniform(-drift, drift), y_c, z])
    return np.asarray(pts, np.float64)


def two_block_scene(dx: float, block_cells=(16, 16, 8), seed: int = 0, steps: int = 500, knife: bool = True,
                    material: str = "vmvisc") -> dict:
    """Two x-adjacent paint blocks resting on y = 0 in the unit cube, a box knife on a seeded
    3-segment path at 0.5 units/s (friction 0.3), floor plate SlipStick with friction 1."""
    rng = np.random.default_rng(seed)
    bc = np.asarray(block_cells, np.int64)
    size = bc * dx
    x0 = 0.5 - size[0]
    z0 = 0.5 - 0.5 * size[2]
    a = jittered_block([x0, 0.0, z0], bc, dx, rng)
    b = jittered_block([x0 + size[0], 0.0, z0], bc, dx, rng)
    x = np.concatenate([a, b])
    lat = np.concatenate([np.tile(MIXBOX_LATENTS[RGB_SEEDS[0]], (len(a), 1)),
                          np.tile(MIXBOX_LATENTS[RGB_SEEDS[1]], (len(b), 1))]).astype(np.float32)
    params = dict(rho=1300.0, E=5e4, nu=0.3, cfl=0.5, cfl_elastic=1.0, flip_ratio=-1.5, fps=60.0, end_frame=100000,
                  dx=dx, particle_volume=dx ** 3 / 8.0, particle_mass=1300.0 * dx ** 3 / 8.0,
                  use_particle_boundaries=1, q_prefac=1.0 / np.sqrt(2.0), **PIGMENT_CONFIG)
    if material == "vmvisc":
        # von Mises / Herschel-Bulkley: yield 100 Pa, consistency 10 Pa s^n, flow index 0.6.  The
        # Perzyna residual q = q_y (1 + eta*gamma_dot)^n (plasticity.cpp:211) gives
        # eta = (k / q_y)^(1/n).
        params.update(plastic_model=5, q_max=100.0, q_min=100.0, xi=0.0, perzyna_exp=0.6,
                      perzyna_visc=(10.0 / 100.0) ** (1.0 / 0.6))
    elif material == "dpvisc":
        # matter/sim_config.json: E 5e5, nu 0.2, rho 1000, friction angle 5 deg, cohesion 500,
        # Perzyna exponent 1, viscosity 0.4; Pradhana correction on.
        params.update(plastic_model=6, E=5e5, nu=0.2, rho=1000.0, particle_mass=1000.0 * dx ** 3 / 8.0,
                      M=float(np.tan(np.deg2rad(5.0))), q_cohesion=500.0, perzyna_exp=1.0, perzyna_visc=0.4,
                      use_pradhana=1)
    vectors = dict(gravity=[0.0, -9.81, 0.0], grid_reference_point=[0.0, 0.0, 0.0],
                   particle_boundary_min=[0.0, 0.0, 0.0], particle_boundary_max=[1.0, 1.0, 1.0])
    objects = [("plate", dict(pos=0.0, plate_type=1, bc=1, friction=1.0))]
    if knife:
        half = [0.2, 0.1, 0.005]
        yk = half[1] + 0.5 * dx
        path = knife_path(rng, 0.5, yk, z0 - 0.05, z0 + size[2] + 0.05)
        objects.append(("box_knife", dict(bc=2, friction=0.3, half=half, waypoints=path, speed=0.5)))
    return dict(x=x, latent=lat, params=params, vectors=vectors, objects=objects, steps=steps,
                name=f"two_blocks_dx{1.0 / dx:.0f}")


def config1(seed: int = 0) -> dict:
    """64^3 grid, dx = 1/64, two 16x16x8-cell blocks: 32,768 particles, 500 steps."""
    return two_block_scene(1.0 / 64, (16, 16, 8), seed, 500)


def config2(seed: int = 0) -> dict:
    """256^3 grid, dx = 1/256, two 64x64x32-cell blocks: 2,097,152 particles, 1000 steps."""
    return two_block_scene(1.0 / 256, (64, 64, 32), seed, 1000)


def four_block_scene(dx: float, block_cells=(64, 64, 64), seed: int = 0, steps: int = 2000) -> dict:
    """2 x 2 blocks (in x and z) of four pigments on the floor, box knife through the middle."""
    rng = np.random.default_rng(seed)
    bc = np.asarray(block_cells, np.int64)
    size = bc * dx
    x0 = 0.5 - size[0]
    z0 = 0.5 - size[2]
    xs, lats = [], []
    for k, (ix, iz) in enumerate([(0, 0), (1, 0), (0, 1), (1, 1)]):
        blk = jittered_block([x0 + ix * size[0], 0.0, z0 + iz * size[2]], bc, dx, rng)
        xs.append(blk)
        lats.append(np.tile(MIXBOX_LATENTS[RGB_SEEDS[k]], (len(blk), 1)))
    sc = two_block_scene(dx, block_cells, seed, steps)
    sc["x"] = np.concatenate(xs)
    sc["latent"] = np.concatenate(lats).astype(np.float32)
    half = [0.2, 0.1, 0.005]
    path = knife_path(rng, 0.5, half[1] + 0.5 * dx, z0 - 0.05, z0 + 2 * size[2] + 0.05)
    sc["objects"] = [sc["objects"][0], ("box_knife", dict(bc=2, friction=0.3, half=half, waypoints=path, speed=0.5))]
    sc["name"] = f"four_blocks_dx{1.0 / dx:.0f}"
    return sc


def config3(seed: int = 0) -> dict:
    """384^3 grid, dx = 1/384, four 64^3-cell blocks of four pigments: 8,388,608 particles."""
    return four_block_scene(1.0 / 384, (64, 64, 64), seed, 2000)


def six_block_scene(dx: float, block_cells=(87, 87, 87), seed: int = 0, steps: int = 4000) -> dict:
    """3 x 2 blocks (x by z) of six pigments on the floor and a box knife making four
    back-and-forth strokes through them along z."""
    rng = np.random.default_rng(seed)
    bc = np.asarray(block_cells, np.int64)
    size = bc * dx
    x0 = 0.5 - 1.5 * size[0]
    z0 = 0.5 - size[2]
    xs, lats = [], []
    for k, (ix, iz) in enumerate([(i, j) for j in range(2) for i in range(3)]):
        blk = jittered_block([x0 + ix * size[0], 0.0, z0 + iz * size[2]], bc, dx, rng)
        xs.append(blk)
        lats.append(np.tile(MIXBOX_LATENTS[RGB_SEEDS[k]], (len(blk), 1)))
    sc = two_block_scene(dx, block_cells, seed, steps)
    sc["x"] = np.concatenate(xs)
    sc["latent"] = np.concatenate(lats).astype(np.float32)
    half = [0.2, 0.1, 0.005]
    path = knife_path(rng, 0.5, half[1] + 0.5 * dx, z0 - 0.05, z0 + 2 * size[2] + 0.05, segments=8)
    sc["objects"] = [sc["objects"][0], ("box_knife", dict(bc=2, friction=0.3, half=half, waypoints=path, speed=0.5))]
    sc["name"] = f"six_blocks_dx{1.0 / dx:.0f}"
    return sc


def config5(seed: int = 0) -> dict:
    """512^3 grid, dx = 1/512, six 87^3-cell blocks in a 3 x 2 arrangement: 31,608,144 particles,
    a knife making four back-and-forth strokes, 4000 steps."""
    return six_block_scene(1.0 / 512, (87, 87, 87), seed, 4000)


def palette_scene(n_particles: int, grid_res: int, pair=(0, 1), yield_pa: float = 100.0, seed: int = 0,
                  steps: int = 500) -> dict:
    """One palette scene of the batched workload: the two-block recipe at dx = 1/grid_res with
    blocks of (2c, 2c, c) cells, c chosen so that 64 c^3 is close to n_particles (and the blocks
    fit the domain), pigments RGB_SEEDS[pair[0]] and RGB_SEEDS[pair[1]], and von Mises /
    Herschel-Bulkley paint of the given yield stress (consistency 10 Pa s^0.6 kept)."""
    c = max(2, int(round((n_particles / 64.0) ** (1.0 / 3.0))))
    c = min(c, grid_res // 5)
    sc = two_block_scene(1.0 / grid_res, (2 * c, 2 * c, c), seed, steps)
    half = len(sc["x"]) // 2
    sc["latent"] = np.concatenate([np.tile(MIXBOX_LATENTS[RGB_SEEDS[pair[0]]], (half, 1)),
                                   np.tile(MIXBOX_LATENTS[RGB_SEEDS[pair[1]]], (len(sc["x"]) - half, 1))]
                                  ).astype(np.float32)
    sc["params"].update(q_max=float(yield_pa), q_min=float(yield_pa),
                        perzyna_visc=(10.0 / float(yield_pa)) ** (1.0 / 0.6))
    sc["name"] = f"palette_{grid_res}_{len(sc['x'])}"
    return sc


def batch_scenes(n: int = 64, seed: int = 0, min_particles: int = 20000, max_particles: int = 400000,
                 min_grid: int = 64, max_grid: int = 160, steps: int = 500) -> list:
    """The batched workload: n independent palette scenes, particle counts log-uniform in
    [min_particles, max_particles], grids min_grid^3 .. max_grid^3 (at least large enough for the
    blocks), a random pigment pair of the six RGB seeds, yield stress uniform in [50, 200] Pa and a
    random 3-segment knife path per scene, all from one seed."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        npart = int(np.exp(rng.uniform(np.log(min_particles), np.log(max_particles))))
        c = max(2, int(round((npart / 64.0) ** (1.0 / 3.0))))
        g = int(rng.integers(max(min_grid, 5 * c), max(max_grid, 5 * c) + 1))
        pair = tuple(int(v) for v in rng.choice(len(RGB_SEEDS), size=2, replace=False))
        y = float(rng.uniform(50.0, 200.0))
        out.append(palette_scene(npart, g, pair, y, seed=int(rng.integers(1 << 30)), steps=steps))
    return out


def sample_particles(Lx: float, Ly: float, Lz: float, radius: float, ppc: float = 8.0, crop_to_shape: int = 0,
                     attempts: int = 30, passes: int = 2, seed: int = 42, device: int = 0):
    """Poisson-disk particles on the GPU (pm_sample_particles, the reference's sampleParticles):
    returns (x[n, 3] float32, dx, particle_volume)."""
    import ctypes as C
    from ._lib import call
    n = C.c_uint32()
    dx, vol = C.c_double(), C.c_double()
    call("pm_sample_particles", device, Lx, Ly, Lz, radius, ppc, crop_to_shape, attempts, passes, seed, None, 0,
         C.byref(n), C.byref(dx), C.byref(vol))
    x = np.zeros((n.value, 3), np.float32)
    call("pm_sample_particles", device, Lx, Ly, Lz, radius, ppc, crop_to_shape, attempts, passes, seed,
         x.ctypes.data_as(C.POINTER(C.c_float)), n.value, C.byref(n), C.byref(dx), C.byref(vol))
    return x, dx.value, vol.value


# ---- blob scenes (Simulation::blobs, matter/src/simulation/simulation_blobs.cpp:7-150) ---------------
# Volumes of the reference's blob ladder (simulation.hpp:272-279: Blob_01 ... Blob_06).
BLOB_VOLUMES = (0.0056, 0.0151, 0.0246, 0.0341, 0.0436, 0.053)


class DomeBlob:
    """An analytic paint dab standing in for the reference's VDB blobs: the upper half of a
    superellipsoid |dx/R|^p + |y/H|^p + |dz/R|^p <= 1 resting on y = 0, centred at (cx, cz)."""

    def __init__(self, volume: float, aspect: float = 0.55, exponent: float = 2.5):
        from math import gamma
        self.p = float(exponent)
        self.k = 4.0 * aspect * gamma(1.0 + 1.0 / self.p) ** 3 / gamma(1.0 + 3.0 / self.p)  # V = k R^3
        self.R = (volume / self.k) ** (1.0 / 3.0)
        self.H = aspect * self.R
        self.c = np.zeros(3)

    @property
    def volume(self) -> float:
        return self.k * self.R ** 3

    def bounds(self):
        lo = self.c + np.array([-self.R, 0.0, -self.R])
        hi = self.c + np.array([self.R, self.H, self.R])
        return lo, hi

    def inside(self, x) -> np.ndarray:
        d = np.asarray(x, np.float64) - self.c
        f = (np.abs(d[:, 0]) / self.R) ** self.p + (np.abs(d[:, 1]) / self.H) ** self.p + \
            (np.abs(d[:, 2]) / self.R) ** self.p
        return (f <= 1.0) & (d[:, 1] >= 0.0)


def blob_target_volume(ratio: float) -> float:
    """Colour ratio -> blob volume: the ratio clamped to [0.1, 0.9] mapped linearly onto the
    ladder's volume range (simulation_blobs.cpp:11-24)."""
    lo, hi = BLOB_VOLUMES[0], BLOB_VOLUMES[-1]
    r = min(0.9, max(0.1, float(ratio)))
    return min(hi, max(lo, lo + (r - 0.1) / 0.8 * (hi - lo)))


def blob_offsets(radii) -> np.ndarray:
    """Ground-plane placement of n blobs of the given packing radii so that neighbours touch
    (simulation_blobs.cpp:63-116): one at the origin; two side by side on x; three with the third
    touching both; four in two rows of two; more in a row along x.  Returns n x 3 offsets (y 0),
    centred on the x / z bounds of the arrangement (:118-140)."""
    r = [float(v) for v in radii]
    n = len(r)
    o = np.zeros((n, 3))
    if n == 2:
        o[0, 0], o[1, 0] = -r[0], r[1]
    elif n == 3:
        o[1, 0] = r[0] + r[1]
        x1 = o[1, 0]
        x2 = ((r[0] + r[2]) ** 2 - (r[1] + r[2]) ** 2 + x1 * x1) / (2.0 * x1)
        o[2, 0] = x2
        o[2, 2] = np.sqrt(max(0.0, (r[0] + r[2]) ** 2 - x2 * x2))
    elif n == 4:
        o[0, 0], o[1, 0], o[2, 0], o[3, 0] = -r[0], r[1], -r[2], r[3]

        def cz(d, dist):
            return np.sqrt(max(0.0, dist * dist - d * d))
        Z = max(cz(o[0, 0] - o[2, 0], r[0] + r[2]), cz(o[1, 0] - o[3, 0], r[1] + r[3]),
                cz(o[0, 0] - o[3, 0], r[0] + r[3]), cz(o[1, 0] - o[2, 0], r[1] + r[2]))
        o[2, 2] = o[3, 2] = Z
    elif n > 4:
        cur = 0.0
        for i in range(n):
            if i > 0:
                cur += r[i - 1] + r[i]
            o[i, 0] = cur
    if n:
        rr = np.asarray(r)
        lo = np.min(o - rr[:, None], axis=0)
        hi = np.max(o + rr[:, None], axis=0)
        centre = 0.5 * (lo + hi)
        centre[1] = 0.0
        o = o - centre
    return o


def blob_scene(color_ratios, latents=None, radius: float = 0.01, ppc: float = 27.0, seed: int = 42,
               aspect: float = 0.55, exponent: float = 2.5, material: str = "dpvisc", knife: bool = True,
               steps: int = 500, device: int = 0) -> dict:
    """The reference's paint scene (Simulation::blobs): one blob per colour ratio, sized by
    blob_target_volume, packed by blob_offsets around (0.5, 0, 0.5), filled by Poisson-disk
    sampling of each blob's bounding box (pm_sample_particles, radius `radius`, 30 attempts, seed
    seed + i) kept inside the blob, and dx = cbrt(ppc * sum of box volumes / sum of box samples)
    (sampleParticlesFromVdb, sampling_particles_vdb.hpp:87-150).  The blobs are analytic domes
    (DomeBlob) instead of the reference's VDB level sets; their packing radius is the exact
    footprint radius, where the reference subtracts 0.055 from its padded VDB bounds."""
    n = len(color_ratios)
    if latents is None:
        latents = [MIXBOX_LATENTS[RGB_SEEDS[i % len(RGB_SEEDS)]] for i in range(n)]
    blobs = [DomeBlob(blob_target_volume(c), aspect, exponent) for c in color_ratios]
    off = blob_offsets([b.R for b in blobs])
    for b, o in zip(blobs, off):
        b.c = o + np.array([0.5, 0.0, 0.5])
    xs, lats = [], []
    total_vol, total_samples = 0.0, 0
    for i, b in enumerate(blobs):
        lo, hi = b.bounds()
        L = hi - lo
        pts, _, _ = sample_particles(L[0], L[1], L[2], radius, ppc, 0, 30, 2, seed + i, device)
        pts = pts.astype(np.float64) + lo
        total_vol += float(np.prod(L))
        total_samples += len(pts)
        keep = pts[b.inside(pts)]
        xs.append(keep.astype(np.float32))
        lats.append(np.tile(np.asarray(latents[i % len(latents)], np.float32), (len(keep), 1)))
    x = np.concatenate(xs)
    dx = float(np.cbrt(ppc / total_samples * total_vol))
    sc = two_block_scene(dx, (1, 1, 1), seed=seed, steps=steps, knife=False, material=material)
    sc["x"], sc["latent"] = x, np.concatenate(lats)
    p = sc["params"]
    p["dx"] = dx
    p["particle_volume"] = dx ** 3 / ppc
    p["particle_mass"] = p["rho"] * p["particle_volume"]
    lo = np.min([b.bounds()[0] for b in blobs], axis=0)
    hi = np.max([b.bounds()[1] for b in blobs], axis=0)
    margin = 0.25
    sc["vectors"]["particle_boundary_min"] = [float(lo[0] - margin), 0.0, float(lo[2] - margin)]
    sc["vectors"]["particle_boundary_max"] = [float(hi[0] + margin), float(hi[1] + margin), float(hi[2] + margin)]
    if knife:
        rng = np.random.default_rng(seed)
        half = [0.2, 0.1, 0.005]
        path = knife_path(rng, 0.5, half[1] + 0.5 * dx, lo[2] - 0.05, hi[2] + 0.05)
        sc["objects"].append(("box_knife", dict(bc=2, friction=0.3, half=half, waypoints=path, speed=0.5)))
    sc["blobs"] = [dict(centre=b.c.tolist(), R=b.R, H=b.H, volume=b.volume, particles=len(xx))
                   for b, xx in zip(blobs, xs)]
    sc["name"] = f"blobs_{n}"
    return sc


def apply(scene: dict, sim) -> None:
    """Load a scene into a Simulation-like object (product Simulation or the oracle wrapper)."""
    if hasattr(sim, "setParticles"):  # product API
        sim.setParticles(scene["x"], scene["latent"])
        sim.set(**scene["params"])
        for k, v in scene["vectors"].items():
            setattr(sim, k, v)
        for kind, kw in scene["objects"]:
            if kind == "plate":
                sim.addPlate(kw["pos"], kw["plate_type"], kw["bc"], kw["friction"])
            elif kind == "box_knife":
                sim.addBoxKnife(kw["bc"], kw["friction"], kw["half"], kw["waypoints"], kw["speed"])
            elif kind == "spatula":
                sim.addSpatula(kw["bc"], kw["friction"], frames=kw["frames"])
    else:  # oracle wrapper
        sim.set_particles(scene["x"], scene["latent"])
        sim.set(**scene["params"])
        sim.set(**scene["vectors"])
        for kind, kw in scene["objects"]:
            if kind == "plate":
                sim.add_plate(kw["pos"], kw["plate_type"], kw["bc"], kw["friction"])
            elif kind == "box_knife":
                sim.add_box_knife(kw["bc"], kw["friction"], kw["half"], kw["waypoints"], kw["speed"])
            elif kind == "spatula":
                sim.add_spatula(kw["bc"], kw["friction"], kw["frames"])

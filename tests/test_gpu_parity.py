"""GPU path (through the C ABI) against the FP64 CPU oracle on identical seeded scenes.

Tolerances: after one step the GPU (FP32 transfers, FP64 SVD) agrees with the FP64 oracle to
FP32 rounding (1e-5 relative); after 50 steps per-particle position error <= 1e-3 of the domain
size (1) and latent error <= 1e-3, the bar the workload sets for the plain FP32 path.
"""
import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _pair(scene, oracle_threads=8):
    from oracle.oracle import OracleSim
    from pigment_mixing_b200 import Simulation, scenes
    g = Simulation(0)
    scenes.apply(scene, g)
    g.prepareSimulation()
    o = OracleSim(64)
    o.set(n_threads=oracle_threads)
    scenes.apply(scene, o)
    o.prepare()
    return g, o


def _fields(g, o, n):
    pg = g.getParticles(fields=("x", "v", "latent", "diffusion", "active", "F", "B", "plastic"))
    po = o.particles()
    return pg, po


def _grid_maps(gr, dx, key):
    d = gr["dims"]
    m = gr["mass"].reshape(d)
    idx = np.argwhere(m > 0)
    base = np.round(gr["origin"] / dx).astype(int)
    vals = gr[key].reshape(list(d) + [-1])
    return {tuple(i + base): vals[tuple(i)].astype(np.float64) for i in idx}


@pytest.fixture(scope="module")
def small_scene():
    from pigment_mixing_b200 import scenes
    return scenes.two_block_scene(1.0 / 32, (8, 8, 4), seed=0, steps=20)


def test_one_step_particles_and_grid(small_scene):
    g, o = _pair(small_scene)
    g.advance(1)
    o.advance(1)
    assert g.time == pytest.approx(o.get("time"), rel=1e-12)
    n = len(small_scene["x"])
    pg, po = _fields(g, o, n)
    for k, tol in (("x", 1e-6), ("v", 1e-6), ("latent", 1e-6), ("F", 1e-6), ("B", 1e-7), ("diffusion", 1e-5)):
        a = getattr(pg, k).reshape(n, -1).astype(np.float64)
        b = po[k].reshape(n, -1).astype(np.float64)
        assert np.abs(a - b).max() <= tol * max(1.0, np.abs(b).max()), k
    assert np.array_equal(pg.active, po["active"])
    # grid node by node on the shared lattice
    dx = small_scene["params"]["dx"]
    gg, og = g.grid(), o.grid()
    for kg, ko, tol in (("mass", "mass", 1e-6), ("v_update", "v_update", 1e-6), ("flip", "flip", 1e-6),
                        ("latent", "latent", 1e-6), ("shear", "shear", 1e-5), ("v_musl", "v", 1e-6)):
        mg, mo = _grid_maps(gg, dx, kg), _grid_maps(og, dx, ko)
        assert set(mg) == set(mo), kg
        scale = max(1e-12, max(np.abs(v).max() for v in mo.values()))
        err = max(np.abs(mg[k] - mo[k]).max() for k in mo)
        assert err <= tol * max(1.0, scale), (kg, err)


def _mixing_fired(latent0, latent, thresh=1e-3):
    """Particles whose latent moved by more than thresh from its initial value (g2p.cpp:103-126)."""
    return int((np.abs(latent.astype(np.float64) - latent0).max(1) > thresh).sum())


def test_config1_fifty_steps_within_tolerance():
    """32,768-particle scene (dx = 1/64): 50 steps against the FP64 oracle.  The workload's bar is
    1e-3 of the domain for positions and 1e-3 for latents; the observed errors are 6.3e-7 and 7e-6,
    so the test holds them to 1e-5 and 1e-4 (a regression of more than about 15x fails).  The knife
    has started mixing: some latents moved by more than 1e-3, identically in both."""
    from pigment_mixing_b200 import scenes
    sc = scenes.config1(seed=0)
    g, o = _pair(sc)
    g.advance(50)
    o.advance(50)
    n = len(sc["x"])
    pg = g.getParticles(fields=("x", "v", "latent", "active"))
    po = o.particles_f64()
    dxp = np.linalg.norm(pg.x.astype(np.float64) - po["x"], axis=1)
    dl = np.abs(pg.latent.astype(np.float64) - po["latent"]).max(1)
    print(f"config1 50 steps: max |dx| {dxp.max():.3e}, max |dlatent| {dl.max():.3e}, "
          f"mixed {_mixing_fired(sc['latent'], pg.latent)} (oracle {_mixing_fired(sc['latent'], po['latent'])})")
    assert dxp.max() <= 1e-5, dxp.max()
    assert dl.max() <= 1e-4, dl.max()
    mixed = _mixing_fired(sc["latent"], po["latent"])
    assert mixed > 0
    assert abs(_mixing_fired(sc["latent"], pg.latent) - mixed) <= max(2, mixed // 100)
    st = g.stats()
    mp = sc["params"]["particle_mass"]
    assert st["mass"] == pytest.approx(mp * n, rel=1e-12)
    mom_o = mp * po["v"].sum(0)
    assert np.allclose(st["momentum"], mom_o, atol=1e-4 * max(1e-6, np.abs(mom_o).max()) + 1e-9)
    assert np.allclose(st["mean_latent"], po["latent"].mean(0), atol=1e-5)


def test_paint_default_scene_with_reference_spatula():
    """DPVisc paint (matter/sim_config.json values) with the reference knife keyframes."""
    import os
    from pigment_mixing_b200 import scenes
    frames = np.load(os.path.join(GOLDEN, "spatula_frames_head.npy"))
    sc = scenes.two_block_scene(1.0 / 48, (12, 12, 6), seed=2, steps=10, knife=False, material="dpvisc")
    # place the paint under the knife's start pose so it is touched within a few steps
    f0 = frames[0]
    sc["x"] = sc["x"] + np.asarray([f0[0] - 0.5, 0.0, f0[2] - 0.5], np.float32)
    sc["objects"].append(("spatula", dict(bc=2, friction=0.0, frames=frames)))
    g, o = _pair(sc)
    for _ in range(3):
        g.advance(5)
        o.advance(5)
    n = len(sc["x"])
    pg = g.getParticles(fields=("x", "v", "latent", "active", "plastic"))
    po = o.particles_f64()
    assert np.abs(pg.x.astype(np.float64) - po["x"]).max() <= 1e-4
    assert np.abs(pg.latent.astype(np.float64) - po["latent"]).max() <= 1e-4
    print(f"paint scene: mixed {_mixing_fired(sc['latent'], pg.latent)} of {n}")
    kg, ko = g.getSpatulaObject(), o.knife()
    assert np.allclose(kg[0], ko[0], atol=1e-5)


def test_noslip_colliders_and_moving_plates_match_oracle():
    """NoSlip on a general object (boundary_collision.cpp:36-38) and on plates, plates moving with
    the first-frame slow-down of vmin_factor / load_factor (object_plate.hpp:136-162): a block
    squeezed by a descending top plate and pushed by a left wall, on a NoSlip ground object."""
    import sys
    sys.path.insert(0, GOLDEN.rsplit("/", 1)[0])
    import reference_kats as K
    from oracle.oracle import OracleSim
    from pigment_mixing_b200 import Simulation, scenes
    base = scenes.two_block_scene(1.0 / 32, (4, 4, 4), seed=4, steps=10, knife=False, material="vmvisc")
    dx = base["params"]["dx"]
    x = base["x"].astype(np.float64)
    top = float(x[:, 1].max()) + 0.5 * dx
    left = float(x[:, 0].min()) - 0.5 * dx
    params = dict(base["params"], fps=20.0, end_frame=1000)
    params.pop("use_particle_boundaries")
    sc = dict(name="squeeze", x=x, v=None, params=params, vectors=dict(gravity=[0.0, -9.81, 0.0]),
              objects=[("ground", dict(bc=K.BC_NOSLIP, friction=0.0, y0=0.0)),
                       ("plate", dict(pos=top, plate_type=K.PLATE_TOP, bc=K.BC_NOSLIP, friction=0.0, vy=-0.3,
                                      vmin_factor=4.0, load_factor=1.0)),
                       ("plate", dict(pos=left, plate_type=K.PLATE_LEFT, bc=K.BC_SLIPSTICK, friction=0.4, vx=0.2,
                                      vmin_factor=2.0, load_factor=2.0))])
    g = Simulation(0)
    K.apply(sc, g)
    g.prepareSimulation()
    o = OracleSim(64)
    o.set(n_threads=8)
    K.apply(sc, o)
    o.prepare()
    for _ in range(4):
        g.advance(10)
        o.advance(10)
    assert g.frame == o.get("frame") and g.frame >= 1  # the slow first frames are over
    pg = g.getParticles(fields=("x", "v", "active"))
    po = o.particles_f64()
    assert np.abs(pg.x - po["x"]).max() <= 1e-5
    assert np.abs(pg.v - po["v"]).max() <= 1e-4 * max(1.0, np.abs(po["v"]).max())
    # the plates did squeeze and push the block
    assert po["x"][:, 1].max() < top - 0.5 * dx - 1e-3
    assert po["x"][:, 0].min() > left + 0.5 * dx + 1e-4


def test_usl_mode_matches_oracle(small_scene):
    """use_musl = 0 after prepare gives the reference's USL update (simulate(), simulation.cpp:524)."""
    g, o = _pair(small_scene)
    g.use_musl = 0
    o.set(use_musl=0)
    g.advance(4)
    o.advance(4)
    n = len(small_scene["x"])
    pg = g.getParticles(fields=("x", "v", "F"))
    po = o.particles()
    assert np.abs(pg.x - po["x"]).max() <= 1e-5
    assert np.abs(pg.v - po["v"]).max() <= 1e-4 * max(1.0, np.abs(po["v"]).max())


def test_grid_capacity_regrowth():
    """A block expanding radially to several times its size outgrows the initial grid capacity:
    the device halts, the host regrows the grid and resumes; results still match the oracle."""
    from oracle.oracle import OracleSim
    from pigment_mixing_b200 import Simulation, scenes
    sc = scenes.two_block_scene(1.0 / 32, (4, 4, 4), seed=5, steps=10, knife=False, material="vmvisc")
    sc["params"].update(plastic_model=0, E=1.0, rho=1000.0, particle_mass=1000.0 * (1.0 / 32) ** 3 / 8.0)
    sc["vectors"]["gravity"] = [0.0, 0.0, 0.0]
    sc["params"]["use_particle_boundaries"] = 0  # unbounded: the grid is sized from the blocks and must grow
    c = sc["x"].mean(0)
    c[1] = 0.0
    v = (3.0 * (sc["x"] - c)).astype(np.float32)
    g = Simulation(0)
    scenes.apply(sc, g)
    g.setParticles(sc["x"], sc["latent"], v)
    g.prepareSimulation()
    o = OracleSim(64)
    o.set(n_threads=4)
    scenes.apply(sc, o)
    o.set_particles(sc["x"], sc["latent"], v)
    o.prepare()
    g.advance(2)
    o.advance(2)
    nodes0 = g.grid_nodes
    for _ in range(8):
        g.advance(10)
        o.advance(10)
    assert g.grid_nodes > 4 * nodes0
    assert int(g.regrowths) >= 1
    pg = g.getParticles(fields=("x", "active"))
    po = o.particles()
    assert np.array_equal(pg.active, po["active"])
    assert np.abs(pg.x - po["x"]).max() <= 1e-4
    assert g.errorFlags() & 0x40 == 0  # capacity flag cleared after regrowth


def test_particle_boundaries_deactivate_like_reference():
    """position_update.cpp:74-89: particles leaving [min, max] are clamped and deactivated."""
    from pigment_mixing_b200 import scenes
    sc = scenes.two_block_scene(1.0 / 32, (4, 4, 4), seed=6, steps=5, knife=False)
    sc["params"]["use_particle_boundaries"] = 1
    sc["vectors"]["particle_boundary_max"] = [0.6, 2.0, 2.0]
    from oracle.oracle import OracleSim
    from pigment_mixing_b200 import Simulation
    v = np.zeros_like(sc["x"])
    v[:, 0] = 2.0
    g = Simulation(0)
    scenes.apply(sc, g)
    g.setParticles(sc["x"], sc["latent"], v)
    g.prepareSimulation()
    o = OracleSim(64)
    scenes.apply(sc, o)
    o.set_particles(sc["x"], sc["latent"], v)
    o.prepare()
    g.advance(20)
    o.advance(20)
    pg = g.getParticles(fields=("x", "v", "active"))
    po = o.particles()
    assert po["active"].sum() < len(sc["x"])
    assert np.array_equal(pg.active, po["active"])
    assert np.abs(pg.x - po["x"]).max() <= 1e-4


def test_async_readback_matches_sync_readback(small_scene):
    """pm_get_particles_async into pinned buffers, overlapped with further steps, delivers the
    state of the moment it was issued (the render loop's per-frame readback)."""
    import torch
    from pigment_mixing_b200 import Simulation, scenes
    g = Simulation(0)
    scenes.apply(small_scene, g)
    g.prepareSimulation()
    g.advance(3)
    ref = g.getParticles(fields=("x", "latent", "diffusion"))
    n = len(small_scene["x"])
    ox = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    ol = torch.empty((n, 7), dtype=torch.float32).pin_memory()
    od = torch.empty((n,), dtype=torch.float32).pin_memory()
    g.readIntoAsync(x=ox.numpy(), latent=ol.numpy(), diffusion=od.numpy())
    g.advance(4)  # overlaps the copy; must not change what it delivers
    g.waitReadback()
    assert np.array_equal(ox.numpy(), ref.x)
    assert np.array_equal(ol.numpy(), ref.latent)
    assert np.array_equal(od.numpy(), ref.diffusion)
    now = g.getParticles(fields=("x",))  # a sync readback after an async one
    assert not np.array_equal(now.x, ref.x)


def test_sparse_box_with_outliers_matches_oracle():
    """Four particles far from the paint stretch the grid box to dozens of times the bricks that hold
    particles, as the knife's splashes do: the occupied- and touched-brick lists must still reach
    every brick, so after one step the grid holds the oracle's nodes with the oracle's values, and
    after ten steps the particles match."""
    from pigment_mixing_b200 import scenes
    sc = scenes.two_block_scene(1.0 / 32, (4, 4, 4), seed=11, steps=10)
    far = np.float32([[0.05, 0.9, 0.05], [0.95, 0.9, 0.95], [0.05, 0.6, 0.95], [0.95, 0.02, 0.05]])
    sc["x"] = np.concatenate([sc["x"], far]).astype(np.float32)
    sc["latent"] = np.concatenate([sc["latent"], sc["latent"][:4]]).astype(np.float32)
    g, o = _pair(sc)
    g.advance(1)
    o.advance(1)
    dx = sc["params"]["dx"]
    gg, og = g.grid(), o.grid()
    box_bricks = int(np.prod(gg["dims"])) // 64
    mg, mo = _grid_maps(gg, dx, "mass"), _grid_maps(og, dx, "mass")
    assert set(mg) == set(mo)
    assert box_bricks > 20 * (len(mo) // 64 + 1)  # the box is mostly empty bricks
    for kg, ko in (("mass", "mass"), ("v_update", "v_update"), ("latent", "latent")):
        a, b = _grid_maps(gg, dx, kg), _grid_maps(og, dx, ko)
        scale = max(1.0, max(np.abs(v).max() for v in b.values()))
        assert max(np.abs(a[k] - b[k]).max() for k in b) <= 1e-6 * scale, kg
    g.advance(9)
    o.advance(9)
    pg = g.getParticles(fields=("x", "latent", "active"))
    po = o.particles_f64()
    assert np.array_equal(pg.active, o.particles()["active"])
    assert np.abs(pg.x - po["x"]).max() <= 1e-5
    assert np.abs(pg.latent - po["latent"]).max() <= 1e-5
    assert g.errorFlags() == 0


@pytest.mark.parametrize("count", [1, 7, 33, 1000])
def test_ragged_particle_counts_match_oracle(count):
    """Particle counts that fill no warp, CTA or brick evenly (a single particle, 7, 33, 1000 drawn
    from a block) step like the oracle: free fall, the floor, the knife and the return map."""
    from pigment_mixing_b200 import scenes
    sc = scenes.two_block_scene(1.0 / 32, (4, 4, 4), seed=9, steps=10)
    rng = np.random.default_rng(count)
    keep = np.sort(rng.choice(len(sc["x"]), size=count, replace=False))
    sc["x"] = sc["x"][keep]
    sc["latent"] = sc["latent"][keep]
    g, o = _pair(sc)
    g.advance(12)
    o.advance(12)
    pg = g.getParticles(fields=("x", "v", "latent", "active"))
    po = o.particles_f64()
    assert len(pg.x) == count
    # a few isolated particles amplify FP32 rounding more than a dense block (observed 1.3e-5)
    assert np.abs(pg.x - po["x"]).max() <= 1e-4
    assert np.abs(pg.latent - po["latent"]).max() <= 1e-5
    # velocities: the 33 scattered particles are thrown by the knife to |v| = 8.5 and their largest
    # error measured 6.5e-3 to 8.8e-3 over ten GPU runs (0.8e-3 to 1.03e-3 of |v|max); the GPU runs
    # differ among themselves by up to 6.5e-4 (the order of FP32 atomic adds between CTAs), so the
    # bar is 2e-3 of |v|max; the other counts stay below 7e-5 of it
    assert np.abs(pg.v - po["v"]).max() <= 2e-3 * max(1.0, np.abs(po["v"]).max())
    assert g.errorFlags() == 0


@pytest.mark.gpu
def test_device_svd_on_hard_matrices():
    """The step's device SVD (FP32 warm start, FP64 one-sided Jacobi) on matrices that stress
    it: random, near-identity, repeated and clustered singular values, large condition numbers,
    large rotations, a reflection, rank-deficient.  A = U diag(s) V^T to FP32 factor rounding,
    s equal to numpy's singular values in FP64."""
    import ctypes as C
    from pigment_mixing_b200._lib import call
    rng = np.random.default_rng(7)

    def rot(rng):
        q, r = np.linalg.qr(rng.normal(size=(3, 3)))
        q *= np.sign(np.diag(r))
        return q if np.linalg.det(q) > 0 else -q

    mats = [rng.normal(size=(3, 3)) for _ in range(200)]
    mats += [np.eye(3) + 1e-4 * rng.normal(size=(3, 3)) for _ in range(100)]
    for s in ([1, 1, 1], [2, 2, 0.5], [1, 1 + 1e-9, 3], [1e4, 1, 1e-4], [5, 1e-3, 1e-3], [1, 0.5, 0.0],
              [1, 0.0, 0.0], [0.3, 0.3, 0.3 + 1e-12]):
        for _ in range(20):
            mats.append(rot(rng) @ np.diag(s) @ rot(rng).T)
    mats.append(np.diag([1.0, 1.0, -1.0]))
    mats.append(np.zeros((3, 3)))
    A = np.ascontiguousarray(np.array(mats, np.float64))
    n = len(A)
    U = np.zeros((n, 3, 3), np.float32)
    V = np.zeros((n, 3, 3), np.float32)
    S = np.zeros((n, 3), np.float64)
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    call("pm_svd3_batch", 0, ptr(A), n, ptr(U), ptr(S), ptr(V))
    ref = np.linalg.svd(A, compute_uv=False)
    scale = np.maximum(ref[:, :1], 1e-300)
    assert np.all(S >= 0.0)
    assert np.abs(np.sort(S, 1)[:, ::-1] - ref).max(initial=0.0) <= 1e-12 * max(1.0, ref.max())
    rec = np.einsum("nij,nj,nkj->nik", U.astype(np.float64), S, V.astype(np.float64))
    assert (np.abs(rec - A).max(axis=(1, 2)) / scale[:, 0]).max() <= 2e-6
    eye = np.eye(3)
    for Q in (U, V):
        Qd = Q.astype(np.float64)
        assert np.abs(np.einsum("nji,njk->nik", Qd, Qd) - eye).max() <= 2e-6

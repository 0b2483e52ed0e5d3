"""pm_p2g_noalloc -- the particle-to-grid transfer for callers that cannot allocate device memory.

Plug-ins whose host application owns every device allocation (a caching allocator, a fixed
memory budget) cannot call cudaMalloc behind its back; this entry point runs the step's P2G
transfer with all scratch in a fixed array inside the library.  The tests drive it through the C
ABI on two calls in a row and check both against the grid the existing stepping entry point
produced from the same particle state (mass, latent, shear) and against a numpy restatement of the
reference's P2G (p2g.cpp:21-124) for the APIC velocity, with the particles' own B matrices.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind():
    from pigment_mixing_b200._lib import lib
    f = lib().pm_p2g_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p] * 5 + [C.c_uint32, C.c_double, C.c_double, C.POINTER(C.c_double),
                                     C.POINTER(C.c_int32)] + [C.c_void_p] * 5 + [C.POINTER(C.c_uint32)]
    return f


def _p2g_numpy(x, v, B, lat, dif, mp, dx, origin, dims):
    """The reference's P2G (p2g.cpp:21-124) in float64: quadratic B-spline weights on the 3-node
    stencil, momentum with the APIC term B (x_i - x_p) 4 / dx^2, latent and shear averaged, the four
    concentrations renormalised."""
    x = x.astype(np.float64)
    u = (x - origin) / dx - 0.5
    base = np.floor(u).astype(np.int64)
    nodes = int(np.prod(dims))
    m = np.zeros(nodes)
    mom = np.zeros((nodes, 3))
    la = np.zeros((nodes, 7))
    sh = np.zeros(nodes)

    def N(t):
        a = np.abs(t)
        return np.where(a < 0.5, 0.75 - a * a, np.where(a < 1.5, 0.5 * (1.5 - a) ** 2, 0.0))

    for a in range(3):
        for b in range(3):
            for c in range(3):
                g = base + np.array([a, b, c])
                xi = origin + g * dx
                d = xi - x
                w = N(d[:, 0] / dx) * N(d[:, 1] / dx) * N(d[:, 2] / dx)
                idx = (g[:, 0] * dims[1] + g[:, 1]) * dims[2] + g[:, 2]
                np.add.at(m, idx, w)
                t = v.astype(np.float64) + 4.0 / dx ** 2 * np.einsum("nij,nj->ni", B.astype(np.float64), d)
                np.add.at(mom, idx, w[:, None] * t)
                np.add.at(la, idx, w[:, None] * lat)
                np.add.at(sh, idx, w * dif)
    has = m > 0
    vel = np.zeros_like(mom)
    vel[has] = mom[has] / m[has, None]
    la[has] /= m[has, None]
    sh[has] /= m[has]
    ps = la[:, :4].sum(1)
    ok = ps > 1e-6
    la[ok, :4] /= ps[ok, None]
    return m * mp, vel, la, sh


def test_p2g_noalloc_matches_step_grid_on_two_calls():
    import torch
    from pigment_mixing_b200 import Simulation, scenes
    p2g = _bind()
    sc = scenes.two_block_scene(1.0 / 32, (8, 8, 4), seed=3, steps=4)
    sim = Simulation(0)
    scenes.apply(sc, sim)
    sim.prepareSimulation()
    sim.advance(3)
    p = sim.getParticles(fields=("x", "v", "latent", "diffusion", "active", "B"))
    assert p.active.all()
    assert np.abs(p.B).max() > 0  # pure APIC scene: the B term is exercised
    # The existing entry point: this step's P2G runs on exactly the state read above; the grid
    # update then changes only velocities, so mass, latent and shear are the P2G results.
    sim.advance(1)
    ref = sim.grid()
    dims = np.asarray(ref["dims"], np.int32)
    nodes = int(np.prod(dims.astype(np.int64)))
    origin = np.ascontiguousarray(ref["origin"], np.float64)
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(np.ascontiguousarray(p.x)).to(dev)
    v = torch.from_numpy(np.ascontiguousarray(p.v)).to(dev)
    lat = torch.from_numpy(np.ascontiguousarray(p.latent)).to(dev)
    dif = torch.from_numpy(np.ascontiguousarray(p.diffusion)).to(dev)
    Bm = torch.from_numpy(np.ascontiguousarray(p.B.reshape(-1, 9))).to(dev)
    n = x.shape[0]
    mp = sc["params"]["particle_mass"]
    dx = sc["params"]["dx"]
    _, vel_np, _, _ = _p2g_numpy(p.x, p.v, p.B, p.latent, p.diffusion, mp, dx, origin, dims.astype(np.int64))
    vscale = np.abs(vel_np).max()
    for call in range(2):
        mass = torch.full((nodes,), float("nan"), device=dev)
        vel = torch.full((nodes, 3), float("nan"), device=dev)
        latn = torch.full((nodes, 7), float("nan"), device=dev)
        shear = torch.full((nodes,), float("nan"), device=dev)
        outside = C.c_uint32(123)
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = p2g(x.data_ptr(), v.data_ptr(), Bm.data_ptr(), lat.data_ptr(), dif.data_ptr(), n, mp, dx,
                 origin.ctypes.data_as(C.POINTER(C.c_double)), dims.ctypes.data_as(C.POINTER(C.c_int32)),
                 mass.data_ptr(), vel.data_ptr(), latn.data_ptr(), shear.data_ptr(), stream, C.byref(outside))
        torch.cuda.synchronize(dev)
        assert rc == 0, f"call {call}: status {rc}"
        assert outside.value == 0
        m = mass.cpu().numpy()
        assert np.isfinite(m).all() and np.isfinite(vel.cpu().numpy()).all()
        # same tolerances as the one-step grid parity test
        assert np.abs(m - ref["mass"]).max() <= 1e-6 * max(1.0, np.abs(ref["mass"]).max()), call
        assert np.abs(latn.cpu().numpy() - ref["latent"]).max() <= 1e-6, call
        assert np.abs(shear.cpu().numpy() - ref["shear"]).max() <= 1e-5 * max(1.0, np.abs(ref["shear"]).max()), call
        assert (m > 0).sum() == (ref["mass"] > 0).sum()
        assert m.sum() == pytest.approx(mp * n, rel=1e-5)
        # APIC velocity, normalised by the node mass (p2g.cpp:21-77, 97-124)
        assert np.abs(vel.cpu().numpy() - vel_np).max() <= 1e-5 * max(1.0, vscale), call
    sim.close()


def test_p2g_noalloc_skips_and_counts_nonfinite_and_far_particles():
    """Particles with a NaN, an infinite or a huge coordinate, or whose stencil leaves the box, are
    skipped and counted in `outside`; the others scatter exactly as without them."""
    import torch
    p2g = _bind()
    rng = np.random.default_rng(11)
    dx = 1.0 / 32
    dims = np.asarray([20, 20, 20], np.int32)
    origin = np.zeros(3)
    n = 5000
    x = rng.uniform(0.1, 0.5, size=(n, 3)).astype(np.float32)
    bad = np.array([[np.nan, 0.3, 0.3], [np.inf, 0.3, 0.3], [-np.inf, 0.3, 0.3], [0.3, 1e30, 0.3],
                    [0.3, 0.3, -1e30], [0.3, 3e9, 0.3], [0.3, 0.3, 0.61], [-0.001, 0.3, 0.3]], np.float32)
    xa = np.concatenate([x, bad])
    na = len(xa)
    v = rng.normal(size=(na, 3)).astype(np.float32)
    B = (0.1 * rng.normal(size=(na, 3, 3))).astype(np.float32)
    lat = rng.uniform(size=(na, 7)).astype(np.float32)
    dif = rng.uniform(size=na).astype(np.float32)
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a.reshape(na, -1))).to(dev)  # noqa: E731
    nodes = int(np.prod(dims.astype(np.int64)))
    mass = torch.zeros(nodes, device=dev)
    vel = torch.zeros((nodes, 3), device=dev)
    outside = C.c_uint32(0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    arrs = [t(a) for a in (xa, v, B, lat, dif)]  # held until the call has run
    rc = p2g(*[a.data_ptr() for a in arrs], na, 1.0, dx,
             origin.ctypes.data_as(C.POINTER(C.c_double)), dims.ctypes.data_as(C.POINTER(C.c_int32)), mass.data_ptr(),
             vel.data_ptr(), None, None, stream, C.byref(outside))
    torch.cuda.synchronize(dev)
    assert rc == 0
    assert outside.value == len(bad)
    m_np, v_np, _, _ = _p2g_numpy(x, v[:n], B[:n], lat[:n], dif[:n], 1.0, dx, origin, dims.astype(np.int64))
    assert np.abs(mass.cpu().numpy() - m_np).max() <= 1e-5 * m_np.max()
    assert np.abs(vel.cpu().numpy() - v_np).max() <= 1e-4 * np.abs(v_np).max()


def test_p2g_noalloc_rejects_sizes_beyond_its_scratch():
    p2g = _bind()
    origin = np.zeros(3)
    dims = np.asarray([128, 128, 16], np.int32)  # 262144 nodes > 131072
    rc = p2g(None, None, None, None, None, 0, 1.0, 0.01, origin.ctypes.data_as(C.POINTER(C.c_double)),
             dims.ctypes.data_as(C.POINTER(C.c_int32)), None, None, None, None, None, None)
    assert rc == 6  # PM_ERR_CAPACITY
    dims = np.asarray([8, 8, 8], np.int32)
    rc = p2g(None, None, None, None, None, (1 << 17) + 1, 1.0, 0.01, origin.ctypes.data_as(C.POINTER(C.c_double)),
             dims.ctypes.data_as(C.POINTER(C.c_int32)), None, None, None, None, None, None)
    assert rc == 6

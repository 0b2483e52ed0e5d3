"""pm_p2g_noalloc -- the particle-to-grid transfer for callers that cannot allocate device memory.

Callers inside CUDA graph capture, or plug-ins whose host owns every allocation, cannot call
cudaMalloc; this entry point runs the step's P2G transfer with all scratch in a fixed array
inside the library.  The test drives it through the C ABI on two calls in a row and checks both
against the grid the existing stepping entry point produced from the same particle state.
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


def test_p2g_noalloc_matches_step_grid_on_two_calls():
    import torch
    from pigment_mixing_b200 import Simulation, scenes
    p2g = _bind()
    sc = scenes.two_block_scene(1.0 / 32, (8, 8, 4), seed=3, steps=4)
    sim = Simulation(0)
    scenes.apply(sc, sim)
    sim.prepareSimulation()
    sim.advance(3)
    p = sim.getParticles(fields=("x", "v", "latent", "diffusion", "active"))
    assert p.active.all()
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
    n = x.shape[0]
    mp = sc["params"]["particle_mass"]
    dx = sc["params"]["dx"]
    for call in range(2):
        mass = torch.full((nodes,), float("nan"), device=dev)
        vel = torch.full((nodes, 3), float("nan"), device=dev)
        latn = torch.full((nodes, 7), float("nan"), device=dev)
        shear = torch.full((nodes,), float("nan"), device=dev)
        outside = C.c_uint32(123)
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = p2g(x.data_ptr(), v.data_ptr(), None, lat.data_ptr(), dif.data_ptr(), n, mp, dx,
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
    sim.close()


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

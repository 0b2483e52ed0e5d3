"""Headless pigment volume splat (pm_splat_pigments) against the numpy restatement of the
renderer's BinaryDensityGrid::fillRenderGrid, isotropic and with anisotropy matrices."""
import numpy as np
import pytest

from conftest import ROOT  # noqa: F401


def test_splat_oracle_properties():
    """The restatement alone: normalised voxels carry pigments summing to 1 and a weight."""
    from oracle import splat_ref
    rng = np.random.default_rng(0)
    x = rng.uniform(0.4, 0.6, size=(300, 3))
    lat = np.zeros((300, 7))
    lat[:150, 0] = 1.0
    lat[150:, 1] = 1.0
    vox, start, v4 = splat_ref.splat(x, lat, [0.38] * 3, [0.62] * 3, 1.0 / 32)
    w = vox[..., 7]
    assert (w > 0).sum() > 100
    s = vox[..., :4].sum(-1)[w > 0]
    assert np.allclose(s, 1.0, atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("aniso", [False, True])
def test_splat_matches_oracle(aniso):
    from oracle import splat_ref
    from pigment_mixing_b200 import Simulation, scenes
    sc = scenes.two_block_scene(1.0 / 32, (6, 6, 3), seed=7, steps=10)
    g = Simulation(0)
    scenes.apply(sc, g)
    g.prepareSimulation()
    g.advance(6)
    st = g.getParticles(fields=("x", "latent"))
    n = len(st.x)
    G = None
    if aniso:
        rng = np.random.default_rng(1)
        h = 2.0 / 32
        A = rng.normal(scale=0.3, size=(n, 3, 3))
        G = ((np.eye(3) + 0.5 * (A + A.transpose(0, 2, 1))) / h).astype(np.float32)
    vox, origin, vs = g.splatPigments(0.5, 0.2, G=G)
    lo, hi = g.getGridBoundaries()
    ref, start, v4 = splat_ref.splat(st.x, st.latent, lo, hi, sc["params"]["dx"], 0.5, 0.2, G=G)
    assert vox.shape == ref.shape
    assert np.allclose(origin, start) and vs == pytest.approx(v4)
    w, wr = vox[..., 7], ref[..., 7]
    assert np.abs(w - wr).max() <= 1e-4 * wr.max()
    both = (w > 1e-3 * wr.max()) & (wr > 1e-3 * wr.max())
    assert both.sum() > 100
    assert np.abs(vox[both, :7] - ref[both, :7]).max() <= 2e-4


@pytest.mark.gpu
def test_cylinder_latent_sample_matches_particles():
    """The final-colour sampling (MPMIntegrationSim.cpp:48-90) reduced on the device equals the
    same average over the particles read back."""
    from pigment_mixing_b200 import Simulation, scenes
    sc = scenes.two_block_scene(1.0 / 32, (6, 6, 3), seed=8, steps=10)
    g = Simulation(0)
    scenes.apply(sc, g)
    g.prepareSimulation()
    g.advance(5)
    st = g.getParticles(fields=("x", "latent", "active"))
    for cx, cz, r in ((0.5, 0.5, 0.2), (0.45, 0.5, 0.05), (0.0, 0.1, 0.2)):
        m, n = g.sampleLatentCylinder(cx, cz, r)
        sel = (st.active > 0) & ((st.x[:, 0] - cx) ** 2 + (st.x[:, 2] - cz) ** 2 <= r * r)
        assert n == int(sel.sum())
        if n:
            assert np.allclose(m, st.latent[sel].astype(np.float64).mean(0), atol=1e-6)
        else:
            assert np.all(m == 0)

"""GPU Poisson-disk scene builder (pm_sample_particles, the reference's sampleParticles): the
Poisson-disk property, near-maximal coverage, density, determinism, the crop shapes and the
derived dx / particle volume (sampling_particles.hpp:26-29)."""
import numpy as np
import pytest

from conftest import ROOT  # noqa: F401


@pytest.mark.gpu
def test_poisson_disk_properties():
    from scipy.spatial import cKDTree
    from pigment_mixing_b200 import scenes
    L = (0.3, 0.2, 0.25)
    r = 0.01
    x, dx, vol = scenes.sample_particles(*L, r, ppc=8, seed=3)
    n = len(x)
    assert n > 1000
    assert x.min() >= 0.0 and np.all(x.max(0) < np.array(L))
    tree = cKDTree(x.astype(np.float64))
    assert not tree.query_pairs(r * (1 - 1e-6)), "two samples closer than the radius"
    frac = n * (4.0 / 3.0) * np.pi * (r / 2) ** 3 / np.prod(L)
    assert 0.30 < frac < 0.60, frac
    probes = np.random.default_rng(0).uniform([2 * r] * 3, np.array(L) - 2 * r, size=(20000, 3))
    d, _ = tree.query(probes)
    assert np.mean(d < 2 * r) > 0.999  # no holes wider than the next dart would fill
    assert dx == pytest.approx(np.cbrt(8 / n * np.prod(L)), rel=1e-9)
    assert vol == pytest.approx(dx ** 3 / 8, rel=1e-9)
    x2, _, _ = scenes.sample_particles(*L, r, ppc=8, seed=3)
    assert np.array_equal(x, x2)
    x3, _, _ = scenes.sample_particles(*L, r, ppc=8, seed=4)
    assert len(x3) != n or not np.array_equal(x, x3)


@pytest.mark.gpu
def test_poisson_crop_shapes():
    from pigment_mixing_b200 import scenes
    L = (0.4, 0.3, 0.4)
    box, dxb, _ = scenes.sample_particles(*L, 0.015, seed=1)
    cyl, dxc, _ = scenes.sample_particles(*L, 0.015, crop_to_shape=1, seed=1)
    silo, dxs, _ = scenes.sample_particles(*L, 0.015, crop_to_shape=2, seed=1)
    assert dxb == dxc == dxs  # dx comes from the uncropped count
    rc = (cyl[:, 0] - L[0] / 2) ** 2 + (cyl[:, 2] - L[2] / 2) ** 2
    assert np.all(rc < (L[0] / 2) ** 2) and len(cyl) < len(box)
    inside = ((box[:, 0] - L[0] / 2) ** 2 + (box[:, 2] - L[2] / 2) ** 2) < (L[0] / 2) ** 2
    assert len(cyl) == int(inside.sum())
    rs = np.tanh(silo[:, 1].astype(np.float64)) + 1
    assert np.all((silo[:, 0] - L[0] / 2) ** 2 + (silo[:, 2] - L[2] / 2) ** 2 < rs ** 2)


def test_blob_recipe_geometry():
    """Simulation::blobs' recipe (simulation_blobs.cpp): ratio -> volume on the blob ladder,
    touching packings for 1..5 blobs, dome volumes."""
    from pigment_mixing_b200 import scenes
    assert scenes.blob_target_volume(0.0) == scenes.BLOB_VOLUMES[0]
    assert scenes.blob_target_volume(1.0) == scenes.BLOB_VOLUMES[-1]
    assert abs(scenes.blob_target_volume(0.5) - 0.5 * (scenes.BLOB_VOLUMES[0] + scenes.BLOB_VOLUMES[-1])) < 1e-12
    r = [0.2, 0.25, 0.3, 0.22, 0.18]
    for n in range(1, 6):
        o = scenes.blob_offsets(r[:n])
        assert np.all(o[:, 1] == 0.0)
        gaps = [np.linalg.norm(o[i] - o[j]) - r[i] - r[j] for i in range(n) for j in range(i + 1, n)]
        assert all(g > -1e-12 for g in gaps)  # no overlap
        if n in (2, 3):
            assert max(abs(g) for g in gaps) < 1e-12  # every pair touches
        if n == 5:
            assert all(abs(np.linalg.norm(o[i + 1] - o[i]) - r[i] - r[i + 1]) < 1e-12 for i in range(4))
        if n:
            lo = np.min(o - np.array(r[:n])[:, None], 0)
            hi = np.max(o + np.array(r[:n])[:, None], 0)
            assert np.allclose((lo + hi)[[0, 2]], 0.0)  # centred on x and z
    rng = np.random.default_rng(0)
    for v in (scenes.BLOB_VOLUMES[0], scenes.BLOB_VOLUMES[-1]):
        b = scenes.DomeBlob(v)
        lo, hi = b.bounds()
        pts = rng.uniform(lo, hi, (200000, 3))
        mc = b.inside(pts).mean() * np.prod(hi - lo)
        assert abs(mc / v - 1.0) < 0.02


@pytest.mark.gpu
def test_blob_scene_samples_and_steps():
    from pigment_mixing_b200 import Simulation, scenes
    sc = scenes.blob_scene([0.3, 0.8, 0.5], radius=0.012, steps=20)
    assert len(sc["blobs"]) == 3
    # particles sit inside their own blobs, above the floor, with their blob's latent
    start = 0
    for i, b in enumerate(sc["blobs"]):
        xb = sc["x"][start:start + b["particles"]]
        blob = scenes.DomeBlob(b["volume"])
        blob.c = np.asarray(b["centre"])
        assert blob.inside(xb).all() and (xb[:, 1] >= 0).all()
        assert np.allclose(sc["latent"][start:start + b["particles"]],
                           scenes.MIXBOX_LATENTS[scenes.RGB_SEEDS[i]], atol=1e-7)
        # the sampled mass matches the blob's volume (Poisson density -> dx as in the reference)
        vol = b["particles"] * sc["params"]["particle_volume"]
        assert abs(vol / b["volume"] - 1.0) < 0.15, (vol, b["volume"])
        start += b["particles"]
    assert start == len(sc["x"])
    g = Simulation(0)
    scenes.apply(sc, g)
    g.prepareSimulation()
    g.advance(10)
    assert g.errorFlags() == 0
    st = g.getParticles(fields=("x", "active"))
    assert st.active.all() and np.isfinite(st.x).all()
    g.close()

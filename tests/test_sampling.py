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

"""The renderer's particle-side preprocessing: the binary density grid (BinaryDensityGrid::fillBDG)
and the anisotropy classification (Classification::countDensities).  CPU tests pin the numpy
restatement (the checker) on cases with known answers; GPU tests compare pm_density_grid and
pm_anisotropy with it on a stepped scene, and the splat fed with the kernel's matrices with the
splat restatement fed with the checker's."""
import numpy as np
import pytest

from conftest import ROOT  # noqa: F401


def _lattice(n, dx, origin=(0.3, 0.0, 0.3), ppc=2, jitter=0.0, seed=0):
    """n^3 cells of ppc^3 particles each (spacing dx / ppc), optionally jittered."""
    rng = np.random.default_rng(seed)
    s = dx / ppc
    g = (np.arange(n * ppc) + 0.5) * s
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) + np.asarray(origin)
    if jitter:
        x += rng.uniform(-jitter * s, jitter * s, x.shape)
    return x.astype(np.float32)


def test_density_grid_filter_is_the_separable_triple_sum():
    from oracle import density_ref as D
    dx = 1.0 / 64
    x = _lattice(6, dx, jitter=0.4)
    lo, hi = x.min(0) - 2 * dx, x.max(0) + 2 * dx
    r = D.density_grid(x, lo, hi, dx)
    X, Y, Z = (int(v) for v in r["dims"])
    c = r["counts"].reshape(Z, Y, X).astype(np.float64)
    w = {-1: 0.74, 0: 0.75, 1: 0.74}
    direct = np.zeros_like(c)
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for ddx in (-1, 0, 1):
                sh = c[np.clip(np.arange(Z) + dz, 0, Z - 1)][:, np.clip(np.arange(Y) + dy, 0, Y - 1)][
                    :, :, np.clip(np.arange(X) + ddx, 0, X - 1)]
                direct += w[dz] * w[dy] * w[ddx] * sh
    assert np.allclose(r["nc"].reshape(Z, Y, X), direct, rtol=1e-5, atol=1e-5)
    assert int(r["counts"].sum()) == len(x)
    # occupancy ORs: every occupied voxel's 2^3 and 4^3 block is set, and nothing else
    M = r["M"].reshape(Z, Y, X)
    zz, yy, xx = np.nonzero(M)
    M2 = r["M2"].reshape((Z + 1) // 2, (Y + 1) // 2, (X + 1) // 2)
    assert M2.sum() == len({(a // 2, b // 2, e // 2) for a, b, e in zip(zz, yy, xx)})
    assert np.all(M2[zz // 2, yy // 2, xx // 2] == 1)
    assert r["occupancy"][1] == int(M.sum()) and sum(r["occupancy"]) == M.size
    # test-all-filled mode
    assert D.density_grid(x, lo, hi, dx, test_all_filled=True)["M"].all()


def test_anisotropy_known_cases():
    from oracle import density_ref as D
    dx = 1.0 / 64
    h = 2 * dx
    # a dense, regular interior: isotropic spread, det G = 1 / h^3 (auto-scale)
    x = _lattice(6, dx, ppc=4)
    lo, hi = x.min(0) - 2 * dx, x.max(0) + 2 * dx
    r = D.anisotropy(x, lo, hi, dx)
    centre = np.argmin(((x - x.mean(0)) ** 2).sum(1))
    G = r["G"][centre].astype(np.float64)
    assert np.allclose(G, G.T)
    assert abs(r["det"][centre] * h ** 3 - 1.0) < 1e-4
    ev = np.linalg.eigvalsh(G)
    assert ev.max() / ev.min() < 1.05  # cubic lattice: nearly isotropic
    assert r["density"][centre] > 0.0
    assert np.allclose(r["G_inv"][centre] @ G, np.eye(3), atol=1e-4)
    # a thin sheet (one particle layer in y): strongly anisotropic, shortest axis ... longest along y
    s = dx / 4
    g = (np.arange(24) + 0.5) * s
    sheet = np.stack(np.meshgrid(g, [0.01], g, indexing="ij"), -1).reshape(-1, 3) + np.array([0.3, 0.0, 0.3])
    sheet = sheet.astype(np.float32)
    rs = D.anisotropy(sheet, sheet.min(0) - 2 * dx, sheet.max(0) + 2 * dx, dx)
    c = np.argmin(((sheet - sheet.mean(0)) ** 2).sum(1))
    lam, V = np.linalg.eigh(rs["G"][c].astype(np.float64))
    assert abs(abs(V[1, np.argmax(lam)]) - 1.0) < 1e-3  # largest G eigenvalue (thinnest kernel) along y
    assert lam.max() / lam.min() > 1.9  # clamped at k = 4 on the covariance: sqrt(4) = 2
    # a lone pair: fewer than 15 neighbours -> isotropic I / h
    pair = np.array([[0.5, 0.1, 0.5], [0.5 + dx / 2, 0.1, 0.5]], np.float32)
    rp = D.anisotropy(pair, pair.min(0) - 2 * dx, pair.max(0) + 2 * dx, dx)
    assert np.allclose(rp["G"][0], np.eye(3) / h, rtol=1e-6)
    assert np.all(rp["n_neighbours"] == 2)


def _stepped_scene(steps=6):
    from pigment_mixing_b200 import Simulation, scenes
    sc = scenes.two_block_scene(1.0 / 32, (4, 4, 4), seed=4, steps=20)
    g = Simulation(0)
    scenes.apply(sc, g)
    g.prepareSimulation()
    g.advance(steps)
    return g, sc


@pytest.mark.gpu
def test_density_grid_matches_restatement():
    from oracle import density_ref as D
    g, sc = _stepped_scene()
    x = g.getParticles(fields=("x",)).x
    lo, hi = g.getGridBoundaries()
    dx = sc["params"]["dx"]
    ref = D.density_grid(x, lo, hi, dx)
    got = g.densityGrid()
    assert np.array_equal(got["dims"], ref["dims"])
    assert np.allclose(got["origin"], ref["start"])
    assert np.array_equal(got["counts"], ref["counts"])
    assert np.array_equal(got["offsets"], ref["offsets"])
    assert np.array_equal(got["M"], ref["M"])
    assert np.array_equal(got["M2"], ref["M2"]) and np.array_equal(got["M4"], ref["M4"])
    assert got["occupancy"] == ref["occupancy"]
    # ids: the same particles per voxel (order inside a voxel is free)
    for v in np.nonzero(ref["counts"])[0][:200]:
        o, n = ref["offsets"][v], ref["counts"][v]
        assert set(got["ids"][o:o + n]) == set(ref["ids"][o:o + n])
    dev = g.densityGrid(device=True)
    assert np.array_equal(dev["M"].cpu().numpy().astype(np.uint32), ref["M"])
    assert np.array_equal(dev["M4"].cpu().numpy().astype(np.uint32), ref["M4"])
    # a lower iso threshold occupies more voxels; test-all-filled occupies all
    assert g.densityGrid(iso=1.0)["occupancy"][1] >= got["occupancy"][1]
    assert g.densityGrid(test_all_filled=True)["M"].all()
    g.close()


@pytest.mark.gpu
def test_anisotropy_matches_restatement_and_feeds_the_splat():
    import torch
    from oracle import density_ref as D
    from oracle import splat_ref
    g, sc = _stepped_scene()
    pg = g.getParticles(fields=("x", "latent"))
    lo, hi = g.getGridBoundaries()
    dx = sc["params"]["dx"]
    h = 2 * dx
    ref = D.anisotropy(pg.x, lo, hi, dx)
    got = g.anisotropy()
    # FP32 neighbour sums in a different order: the matrices agree to ~1e-5 of their scale 1/h
    assert np.abs(got["G"] - ref["G"]).max() <= 1e-4 / h
    assert np.abs(got["G_inv"] - ref["G_inv"]).max() <= 1e-4 * h
    assert np.allclose(got["det"], ref["det"], rtol=1e-4)
    assert np.allclose(got["density"], ref["density"], rtol=1e-3, atol=1e-3 * ref["density"].max())
    assert abs(got["n_aggregate"] - ref["n_aggregate"]) <= max(1, len(pg.x) // 200)
    # device outputs: the same numbers up to the order of the neighbour sums (the order of the
    # particles inside a voxel follows the binning's atomics), and they drive the splat
    dev = g.anisotropy(device=True)
    assert np.abs(dev["G"].cpu().numpy() - got["G"]).max() <= 1e-5 / h
    vox0, origin, vs = g.splatPigments(0.5, 0.2)
    out = torch.empty(vox0.shape, dtype=torch.float32, device="cuda:0")
    g.splatPigments(0.5, 0.2, G=dev["G"], out=out)
    mine = out.cpu().numpy()
    chk, _, _ = splat_ref.splat(pg.x, pg.latent, lo, hi, dx, 0.5, 0.2, G=ref["G"])
    w = chk[..., 7]
    assert np.abs(mine[..., 7] - w).max() <= 1e-3 * max(1.0, w.max())
    filled = w > 1e-3 * w.max()
    assert np.abs(mine[..., :7][filled] - chk[..., :7][filled]).max() <= 2e-3
    g.close()

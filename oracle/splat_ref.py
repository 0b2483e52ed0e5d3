"""TEST INFRASTRUCTURE ONLY -- numpy restatement of the renderer's pigment volume splat
(BinaryDensityGrid::fillRenderGrid, raytracing/src/raymarch/BinaryDensityGrid.cpp:153-296) and of
its grid geometry (AABBc::fixedAABB, AABBc.cpp:10-25; support radius 2 dx,
MPMIntegrationSim.cpp:96-98).  Checks the library's pm_splat_pigments on small scenes.
Parity unpinned against the reference itself (its renderer needs OpenGL, glm and Eigen, none of
which are here); the restatement follows the source line by line.
"""
from __future__ import annotations

import numpy as np


def geometry(lo, hi, dx):
    """Fine-voxel origin, size and counts (x, y, z) of the pigment grid."""
    h = np.float32(2.0 * dx)
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)
    start = np.floor(lo / h) * h
    cells = np.ceil((hi - lo) / h).astype(np.int64) + 1
    return start.astype(np.float64), float(h) / 4.0, 4 * cells, float(h)


def _pass(x, lat, G, start, v4, dims, ext, ss, sc, cvox=None):
    n = len(x)
    acc = np.zeros((dims[2], dims[1], dims[0], 8))
    base = np.floor((x - start) / v4 - 0.5).astype(np.int64)
    rng = np.arange(-ext, ext + 1)
    for oz in rng:
        for oy in rng:
            for ox in rng:
                cell = base + np.array([ox, oy, oz])
                ok = np.all((cell >= 0) & (cell < dims), axis=1)
                if not ok.any():
                    continue
                c = cell[ok]
                diff = x[ok] - (start + (c + 0.5) * v4)
                l = np.einsum("nij,nj->ni", G[ok], diff)
                d2 = (l * l).sum(1)
                near = d2 <= 9.0 * ss * ss
                if not near.any():
                    continue
                c, d2 = c[near], d2[near]
                p = lat[ok][near]
                w = np.exp(-d2 / (ss * ss))
                if cvox is not None:
                    vc = cvox[c[:, 2], c[:, 1], c[:, 0], :4]
                    w = w * np.exp(-((p[:, :4] - vc) ** 2).sum(1) / (sc * sc))
                vals = np.concatenate([p * w[:, None], w[:, None]], 1)
                np.add.at(acc, (c[:, 2], c[:, 1], c[:, 0]), vals)
    return acc


def _normalise(acc):
    w = acc[..., 7]
    m = w > 0
    acc[m, :7] /= w[m, None]
    ps = acc[..., :4].sum(-1)
    m2 = m & (ps > 1e-6)
    acc[m2, :4] /= ps[m2, None]
    return acc


def splat(x, lat, lo, hi, dx, sigma_spatial=0.5, sigma_color=0.2, G=None):
    """voxels[z][y][x][8] (latent 7 + weight), origin, fine voxel size."""
    x = np.asarray(x, np.float64)
    lat = np.asarray(lat, np.float64)
    start, v4, dims, h = geometry(lo, hi, dx)
    ss = max(sigma_spatial, 0.001)
    sc = max(sigma_color, 0.001)
    ext = min(12, int(np.ceil(np.float32(h) * np.float32(3.0) * np.float32(ss) / np.float32(v4))))
    if G is None:
        G = np.broadcast_to(np.eye(3) / h, (len(x), 3, 3))
    G = np.asarray(G, np.float64).reshape(-1, 3, 3)
    tmp = _normalise(_pass(x, lat, G, start, v4, dims, ext, ss, sc))
    out = _normalise(_pass(x, lat, G, start, v4, dims, ext, ss, sc, cvox=tmp))
    return out, start, v4

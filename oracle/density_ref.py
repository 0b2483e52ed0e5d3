"""TEST INFRASTRUCTURE ONLY -- numpy restatement of the renderer's particle-side preprocessing,
the checker of the library's pm_density_grid and pm_anisotropy:

* density voxels, AABBc::fixedAABB (raytracing/src/raymarch/AABBc.cpp:10-25): side h = 2 dx
  (MPMIntegrationSim.cpp:96-98), origin floor(lo / h) h, ceil((hi - lo) / h) + 1 voxels per axis;
* particle binning, BinaryDensityGrid::fillCells (BinaryDensityGrid.cpp:22-55);
* the binary density grid, generateNc / fillBDG (:57-151): separable x, y, z filter with weight a
  on the voxel and b on its clamped neighbours, occupancy nc * 315 / (64 pi h^3) >= iso, M2 / M4;
* anisotropy and density, Classification::countMatrix / countCurrDens (Classification.cpp:38-130),
  with the neighbour search of MPMIntegrationSim::neighborsByIndex (MPMIntegrationSim.cpp:182-224).

The arithmetic is float32 where the reference's is float (positions, voxel assignment, the filter
sums in the reference's order), and float64 for the covariance eigenproblem (the reference calls
Eigen's float SelfAdjointEigenSolver, absent here; the matrix it builds, V diag V^T, does not
depend on the eigenvector signs or order).  Parity unpinned against the reference itself: its
renderer needs OpenGL, glm and Eigen, none of which are here.
"""
from __future__ import annotations

import numpy as np

F = np.float32


def geometry(lo, hi, dx):
    """(origin[3] float32, h float32, dims[3] int) of the density voxels."""
    h = F(2.0 * dx)
    lo = np.asarray(lo, np.float64).astype(F)
    hi = np.asarray(hi, np.float64).astype(F)
    start = (np.floor(lo / h) * h).astype(F)
    dims = (np.ceil((hi - lo) / h)).astype(np.int64) + 1
    return start, h, dims


def voxels(x, start, h, dims):
    """Voxel coordinates (int, n x 3) and whether each particle is inside the voxel grid."""
    c = np.floor((np.asarray(x, F) - start) / h)
    inside = np.all((c >= 0) & (c < dims), axis=1)
    return c.astype(np.int64), inside


def bin_particles(x, lo, hi, dx):
    """fillCells: per-voxel counts and exclusive offsets, ids grouped by voxel (ascending inside
    a voxel here; the reference's order inside a voxel is that of its OpenMP threads)."""
    start, h, dims = geometry(lo, hi, dx)
    c, inside = voxels(x, start, h, dims)
    vid = c[:, 0] + dims[0] * (c[:, 2] * dims[1] + c[:, 1])
    n = int(np.prod(dims))
    counts = np.bincount(vid[inside], minlength=n).astype(np.uint32)
    offsets = np.zeros(n, np.uint32)
    offsets[1:] = np.cumsum(counts)[:-1]
    idx = np.nonzero(inside)[0]
    ids = idx[np.argsort(vid[inside], kind="stable")].astype(np.uint32)
    return dict(start=start, h=h, dims=dims, counts=counts, offsets=offsets, ids=ids, vid=vid, inside=inside)


def density_grid(x, lo, hi, dx, a=0.75, b=0.74, iso=9285.0, test_all_filled=False):
    """generateNc + fillBDG: M, M2, M4 (uint32, voxel order x + X (y + Y z)), occupancy[2], nc."""
    bn = bin_particles(x, lo, hi, dx)
    X, Y, Z = (int(v) for v in bn["dims"])
    cnt = bn["counts"].reshape(Z, Y, X).astype(F)  # [z][y][x]
    a, b = F(a), F(b)
    xi = np.arange(X)
    yi = np.arange(Y)
    zi = np.arange(Z)
    nx = np.zeros_like(cnt)
    for d in (-1, 0, 1):  # x pass, generateNc :63-73
        k = a if d == 0 else b
        nx = (nx + k * cnt[:, :, np.clip(xi + d, 0, X - 1)]).astype(F)
    ny = np.zeros_like(cnt)
    for d in (-1, 0, 1):  # y pass :75-86
        k = a if d == 0 else b
        ny = (ny + k * nx[:, np.clip(yi + d, 0, Y - 1), :]).astype(F)
    nc = np.zeros_like(cnt)
    for d in (-1, 0, 1):  # z pass :88-99
        k = a if d == 0 else b
        nc = (nc + k * ny[np.clip(zi + d, 0, Z - 1), :, :]).astype(F)
    kern = F(315.0 / (64.0 * np.pi * float(bn["h"]) ** 3))  # fillBDG :117
    M = ((nc * kern >= F(iso)) | bool(test_all_filled)).astype(np.uint32)
    X2, Y2, Z2 = (X + 1) // 2, (Y + 1) // 2, (Z + 1) // 2
    X4, Y4, Z4 = (X + 3) // 4, (Y + 3) // 4, (Z + 3) // 4
    M2 = np.zeros((Z2, Y2, X2), np.uint32)
    M4 = np.zeros((Z4, Y4, X4), np.uint32)
    zz, yy, xx = np.nonzero(M)
    M2[zz // 2, yy // 2, xx // 2] = 1
    M4[zz // 4, yy // 4, xx // 4] = 1
    occ = int(M.sum())
    return dict(M=M.reshape(-1), M2=M2.reshape(-1), M4=M4.reshape(-1), occupancy=(M.size - occ, occ),
                nc=nc.reshape(-1), **{k: bn[k] for k in ("start", "h", "dims", "counts", "offsets", "ids")})


def neighbours(x, bn):
    """neighborsByIndex: for each particle, the binned particles in the 3 x 3 x 3 voxels around
    its own (clamped to the grid) with |x_i - x_j|^2 <= h^2 (float32)."""
    x = np.asarray(x, F)
    start, h, dims = bn["start"], bn["h"], bn["dims"]
    c, _ = voxels(x, start, h, dims)
    h2 = F(h * h)
    out = []
    for i in range(len(x)):
        lo = np.maximum(c[i] - 1, 0)
        hi = np.minimum(c[i] + 1, dims - 1)
        cand = []
        for z in range(lo[2], hi[2] + 1):
            for y in range(lo[1], hi[1] + 1):
                for xx in range(lo[0], hi[0] + 1):
                    v = xx + dims[0] * (z * dims[1] + y)
                    o, n = bn["offsets"][v], bn["counts"][v]
                    cand.append(bn["ids"][o:o + n])
        cand = np.concatenate(cand) if cand else np.zeros(0, np.uint32)
        d = (x[i] - x[cand]).astype(F)
        dd = (d * d).sum(1, dtype=F)
        out.append(cand[dd <= h2])
    return out


def anisotropy(x, lo, hi, dx, s=1400.0, k=4.0, threshold=15, auto_scale=True, is_ani=True, iso=9285.0):
    """countMatrix + countCurrDens: G (n x 3 x 3), G_inv, |det G|, density, n_aggregate."""
    x = np.asarray(x, F)
    bn = bin_particles(x, lo, hi, dx)
    nb = neighbours(x, bn)
    h = float(bn["h"])
    n = len(x)
    G = np.zeros((n, 3, 3))
    for i in range(n):
        js = nb[i]
        d = x[js].astype(np.float64) - x[i].astype(np.float64)
        l = np.sqrt((d * d).sum(1))
        w = (1.0 - l / (2.0 * h)) ** 3  # (1 - q)^3, q = l / 2h (:50-55)
        ws = w.sum()
        if len(js) < threshold or ws < 1e-12:  # :60-67
            G[i] = np.eye(3) / h
            continue
        xc = (w[:, None] * x[js]).sum(0) / ws  # :58, 68
        dc = x[js] - xc
        C = s * np.einsum("n,ni,nj->ij", w / ws, dc, dc)  # :69-76
        lam, V = np.linalg.eigh(C)  # :78-80
        lmax = lam.max()
        if not lmax > 0.0:
            G[i] = np.eye(3) / h
            continue
        e = 1.0 / np.sqrt(np.maximum(lam, lmax / k))  # :82-86
        B = (V * e) @ V.T / h
        det = abs(np.linalg.det(B))
        if (auto_scale or not is_ani) and det > 0.0:  # :88-93
            B *= np.cbrt((1.0 / h ** 3) / det)
        G[i] = B
    Gf = G.astype(F)
    det = np.abs(np.linalg.det(Gf.astype(np.float64)))
    Ginv = np.linalg.inv(Gf.astype(np.float64))
    kern = F(315.0) / (F(64.0) * F(np.pi))  # state.h:36
    dens = np.zeros(n)
    for i in range(n):  # countCurrDens :113-126
        js = nb[i]
        d = (x[i] - x[js]).astype(np.float64)
        lv = np.einsum("nij,nj->ni", Gf[js].astype(np.float64), d)
        l2 = (lv * lv).sum(1)
        keep = l2 <= 1.0
        dens[i] = (float(kern) * det[js][keep] * (1.0 - l2[keep]) ** 3).sum()
    return dict(G=Gf, G_inv=Ginv, det=det, density=dens, n_aggregate=int((dens > iso).sum()),
                n_neighbours=np.array([len(v) for v in nb]))

"""Seeded sparse least-squares systems shaped like DAzi's G matrix: rows of
ray-path weights over a band of neighbouring cells, times the depth kernels
of the layers under them (a few hundred non-zeros per row), then one
Tikhonov smoothing row per parameter (the cell and its lateral neighbours),
as TikhRegul.f90 appends them.  Values real*4, 1-based triplets (the
reference's iw/rw layout)."""
import numpy as np


def g_like_system(nvx=30, nvz=24, nz=8, nrays=6000, smooth=0.3, seed=0):
    rng = np.random.default_rng(seed)
    ncell = nvx * nvz
    n = ncell * nz
    rows, cols, vals = [], [], []
    kern = np.exp(-np.arange(nz) / 3.0)
    for r in range(nrays):
        x0, z0 = rng.uniform(0, nvx), rng.uniform(0, nvz)
        x1, z1 = rng.uniform(0, nvx), rng.uniform(0, nvz)
        t = np.linspace(0.0, 1.0, 60)
        cx = np.clip((x0 + t * (x1 - x0)).astype(int), 0, nvx - 1)
        cz = np.clip((z0 + t * (z1 - z0)).astype(int), 0, nvz - 1)
        cells = np.unique(cz * nvx + cx)
        w = rng.uniform(0.5, 1.5, cells.size)
        depth = kern * rng.uniform(0.5, 1.0)
        c = (np.arange(nz)[:, None] * ncell + cells[None, :]).ravel()
        v = (depth[:, None] * w[None, :]).ravel()
        rows.append(np.full(c.size, r))
        cols.append(c)
        vals.append(v)
    m = nrays
    # smoothing rows: 4 p - neighbours (lateral), one per parameter
    p = np.arange(n)
    cell = p % ncell
    ix, iz = cell % nvx, cell // nvx
    for dx, dz in ((1, 0), (-1, 0), (0, 1), (0, -1)):
        ok = (ix + dx >= 0) & (ix + dx < nvx) & (iz + dz >= 0) & (iz + dz < nvz)
        rows.append(m + p[ok])
        cols.append(p[ok] + dx + dz * nvx)
        vals.append(np.full(int(ok.sum()), -smooth))
    rows.append(m + p)
    cols.append(p)
    vals.append(np.full(n, 4.0 * smooth))
    m += n
    row = np.concatenate(rows).astype(np.int32) + 1
    col = np.concatenate(cols).astype(np.int32) + 1
    val = np.concatenate(vals).astype(np.float32)
    x_true = rng.standard_normal(n) * 0.05
    A_x = np.zeros(m)
    np.add.at(A_x, row - 1, val.astype(np.float64) * x_true[col - 1])
    b = A_x + 0.01 * rng.standard_normal(m)
    b[nrays:] = 0.0
    return row, col, val, b, m, n

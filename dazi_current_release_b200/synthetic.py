"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference measures on no public dataset; these generators produce inputs
with the sizes and value distributions of the five benchmark configurations
(all values float32, like the reference's real*4 model arrays; periods
ascending, as the period continuation of surfdisp96.f:262-265 expects).

grid configurations (one depth grid shared by every column, the reference's
`depthkernel(nx,ny,nz,vel,...)` interface):
    config0  16x16 columns, 21 nodes every 3 km, 10 periods 5-40 s, minthk 4,
             Vp = 1.75 Vs, rho = Brocher(Vp)  (explicit vp/rho entry)
    config1  60x50 columns, 31 nodes (30 layers, 1 km growing geometrically
             to 90 km in total), smooth 6 % random field, 25 periods 3-50 s
    config2  100x100 columns, config-1 recipe (seed 2), 30 periods 3-60 s,
             plus a 3 %-perturbed "observed" model (seed 3) and azimuths
    config4  200x200 columns, 41 nodes to 150 km, clipped 5 % noise,
             40 periods 2-80 s, anisotropy amplitudes for the epilogue
ragged configuration (per-column node grids and period lists):
    config3  realisations x 2500 columns, 10-60 layers, sediments, 20 % LVZ,
             8-40 periods in 3-60 s, minthk 2
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class GridCase:
    name: str
    vel: np.ndarray            # (nx, ny, nz) float32, Fortran order
    depz: np.ndarray           # (nz,) float32
    periods: np.ndarray        # (K,) float64
    minthk: float
    vp: np.ndarray | None = None
    rho: np.ndarray | None = None
    extra: dict = field(default_factory=dict)

    @property
    def shape(self):
        return self.vel.shape


def brocher_rho(vp):
    """rho(Vp), the density half of depthkernel_empirical_vp_rho
    (DepthKernel1D.f90:187-200), in float32."""
    p = np.asarray(vp, np.float32)
    p2 = p * p
    p3 = p2 * p
    p4 = p2 * p2
    p5 = p3 * p2
    r = np.float32(1.6612) * p - np.float32(0.4721) * p2
    r = r + np.float32(0.0671) * p3
    r = r - np.float32(0.0043) * p4
    r = r + np.float32(0.000106) * p5
    return r.astype(np.float32)


def geometric_thicknesses(h1: float, total: float, n: int) -> np.ndarray:
    """n thicknesses h1*r**i summing to `total` (ratio by bisection)."""
    lo, hi = 1.0 + 1e-9, 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        s = h1 * (r ** n - 1.0) / (r - 1.0)
        if s > total:
            hi = r
        else:
            lo = r
    r = 0.5 * (lo + hi)
    return h1 * r ** np.arange(n)


def smooth_field(shape, spacing, corr_len, rng):
    """Unit-std Gaussian-correlated random field by FFT filtering of white
    noise (Gaussian spectrum, correlation length corr_len)."""
    noise = rng.standard_normal(shape)
    f = np.fft.fftn(noise)
    k2 = np.zeros(shape)
    for ax, (n, dx) in enumerate(zip(shape, spacing)):
        k = np.fft.fftfreq(n, d=dx) * 2 * np.pi
        sh = [1] * len(shape)
        sh[ax] = n
        k2 = k2 + (k.reshape(sh)) ** 2
    filt = np.exp(-0.25 * k2 * corr_len ** 2)
    g = np.real(np.fft.ifftn(f * filt))
    g -= g.mean()
    g /= g.std()
    return g


def config0(seed: int = 0) -> GridCase:
    nx = ny = 16
    nz = 21
    rng = np.random.default_rng(seed)
    depz = (3.0 * np.arange(nz)).astype(np.float32)
    k = np.arange(nz)
    grad = 2.6 + 2.0 * k / 20.0
    vs = grad[None, None, :] * (1.0 + 0.05 * rng.standard_normal((nx, ny, nz)))
    vs = np.asfortranarray(vs.astype(np.float32))
    vp = np.asfortranarray((np.float32(1.75) * vs).astype(np.float32))
    rho = np.asfortranarray(brocher_rho(vp))
    per = np.geomspace(5.0, 40.0, 10)
    return GridCase("config0", vs, depz, per, 4.0, vp=vp, rho=rho)


def _regional(nx, ny, seed, n_layers=30, total=90.0, h1=1.0, std=0.06):
    rng = np.random.default_rng(seed)
    thk = geometric_thicknesses(h1, total, n_layers)
    depz = np.concatenate([[0.0], np.cumsum(thk)]).astype(np.float32)
    depz[-1] = np.float32(total)
    nz = depz.size
    grad = 2.6 + 2.0 * depz.astype(np.float64) / total
    # 3-D correlated field on a regular grid (10 km lateral, 3 km vertical),
    # sampled at the node depths
    nzr = int(np.ceil(total / 3.0)) + 1
    g = smooth_field((nx, ny, nzr), (10.0, 10.0, 3.0), 50.0, rng)
    iz = np.clip(np.rint(depz / 3.0).astype(int), 0, nzr - 1)
    vs = grad[None, None, :] * (1.0 + std * g[:, :, iz])
    return np.asfortranarray(vs.astype(np.float32)), depz


def config1(seed: int = 1) -> GridCase:
    vs, depz = _regional(60, 50, seed)
    return GridCase("config1", vs, depz, np.geomspace(3.0, 50.0, 25), 4.0)


def config2(seed_a: int = 2, seed_b: int = 3, seed_psi: int = 4) -> GridCase:
    vs, depz = _regional(100, 100, seed_a)
    rng = np.random.default_rng(seed_b)
    vs_b = np.asfortranarray((vs * (1.0 + 0.03 * rng.standard_normal(vs.shape))).astype(np.float32))
    per = np.geomspace(3.0, 60.0, 30)
    psi = np.random.default_rng(seed_psi).uniform(0.0, np.pi, (100 * 100, per.size))
    return GridCase("config2", vs, depz, per, 4.0, extra={"vs_obs": vs_b, "psi": psi})


def config4(seed: int = 5, seed_ani: int = 6) -> GridCase:
    nx = ny = 200
    rng = np.random.default_rng(seed)
    thk = geometric_thicknesses(1.0, 150.0, 40)
    depz = np.concatenate([[0.0], np.cumsum(thk)]).astype(np.float32)
    depz[-1] = np.float32(150.0)
    grad = 2.6 + 2.0 * depz.astype(np.float64) / 150.0
    pert = np.clip(0.05 * rng.standard_normal((nx, ny, depz.size)), -0.15, 0.15)
    vs = np.asfortranarray((grad[None, None, :] * (1.0 + pert)).astype(np.float32))
    ra = np.random.default_rng(seed_ani)
    amp = ra.uniform(0.02, 0.06, (nx * ny, depz.size - 1))
    phi0 = ra.uniform(0.0, np.pi)
    return GridCase("config4", vs, depz, np.geomspace(2.0, 80.0, 40), 3.0,
                    extra={"gc": amp * np.cos(2 * phi0), "gs": amp * np.sin(2 * phi0),
                           "phi0": phi0})


GRID_CONFIGS = {"config0": config0, "config1": config1, "config2": config2, "config4": config4}


@dataclass
class RaggedBatch:
    """Columns with their own node grids and period lists (CSR layout)."""
    node_off: np.ndarray     # (ncol+1,) int64 offsets into depz/vs
    depz: np.ndarray         # (sum nz,) float32
    vs: np.ndarray           # (sum nz,) float32
    per_off: np.ndarray      # (ncol+1,) int64 offsets into periods
    periods: np.ndarray      # (sum K,) float64
    minthk: float

    @property
    def ncol(self):
        return self.node_off.size - 1

    @property
    def column_periods(self):
        return int(self.per_off[-1])

    def column(self, c):
        a, b = self.node_off[c], self.node_off[c + 1]
        p, q = self.per_off[c], self.per_off[c + 1]
        return self.depz[a:b], self.vs[a:b], self.periods[p:q]


def config3(realisations: int = 100, columns: int = 2500, base_seed: int = 1000) -> RaggedBatch:
    """Per realisation r (seed base_seed + r), per column: L ~ U{10..60}
    layers; 1-3 sediment layers of total thickness U(0.3, 3) km with
    Vs ~ U(0.8, 1.5) (increasing), each at least 50 m thick; the remaining
    thicknesses a Dirichlet split of 100 km minus the sediment, each at least
    200 m; Vs at the other nodes the 2.6-4.6
    km/s gradient x (1 + 0.05 N(0,1)); in 20 % of the columns a -8 % low-
    velocity zone at 15-25 km; n ~ U{8..40} periods log-uniform in 3-60 s,
    sorted.  Vectorised over the columns of a realisation."""
    deps, vss, pers, nn, npers = [], [], [], [], []
    for r in range(realisations):
        rng = np.random.default_rng(base_seed + r)
        C = columns
        L = rng.integers(10, 61, C)
        ns = rng.integers(1, 4, C)
        sed = rng.uniform(0.3, 3.0, C)
        nper = rng.integers(8, 41, C)
        # thicknesses: gamma variates normalised per segment (a Dirichlet split)
        g_sed = rng.gamma(1.0, 1.0, (C, 3))
        g_rest = rng.gamma(2.0, 1.0, (C, 60))
        jj = np.arange(3)[None, :]
        g_sed = np.where(jj < ns[:, None], g_sed, 0.0)
        g_sed /= g_sed.sum(axis=1, keepdims=True)
        kk = np.arange(60)[None, :]
        nrest = (L - ns)[:, None]
        g_rest = np.where(kk < nrest, g_rest, 0.0)
        g_rest /= g_rest.sum(axis=1, keepdims=True)
        noise = rng.standard_normal((C, 61))
        vsed = np.sort(rng.uniform(0.8, 1.5, (C, 3)), axis=1)
        lvz = rng.random(C) < 0.2
        praw = np.exp(rng.uniform(np.log(3.0), np.log(60.0), (C, 40)))
        for c in range(C):
            nsc, Lc = ns[c], L[c]
            # floors of 50 m (sediments) and 200 m: no sliver layers
            ts = 0.05 + (sed[c] - 0.05 * nsc) * g_sed[c, :nsc]
            tr = 0.2 + (100.0 - sed[c] - 0.2 * (Lc - nsc)) * g_rest[c, :Lc - nsc]
            thk = np.concatenate([ts, tr])
            z = np.concatenate([[0.0], np.cumsum(thk)])
            z[-1] = 100.0
            vs = (2.6 + 2.0 * z / 100.0) * (1.0 + 0.05 * noise[c, :Lc + 1])
            vs[:nsc] = vsed[c, 3 - nsc:] if nsc < 3 else vsed[c]
            if lvz[c]:
                vs[(z >= 15.0) & (z <= 25.0)] *= 0.92
            deps.append(z.astype(np.float32))
            vss.append(vs.astype(np.float32))
            pers.append(np.sort(np.round(praw[c, :nper[c]], 6)))
        nn.append(L + 1)
        npers.append(nper)
    nn = np.concatenate(nn)
    npers = np.concatenate(npers)
    node_off = np.concatenate([[0], np.cumsum(nn)]).astype(np.int64)
    per_off = np.concatenate([[0], np.cumsum(npers)]).astype(np.int64)
    return RaggedBatch(node_off, np.concatenate(deps), np.concatenate(vss), per_off,
                       np.concatenate(pers), 2.0)


def subgrid(case: GridCase, nx: int, ny: int) -> GridCase:
    """The first nx x ny columns of a grid case (for quick parity runs)."""
    sl = (slice(0, nx), slice(0, ny), slice(None))
    f = lambda a: None if a is None else np.asfortranarray(a[sl])  # noqa: E731
    return GridCase(case.name + f"_{nx}x{ny}", f(case.vel), case.depz, case.periods,
                    case.minthk, vp=f(case.vp), rho=f(case.rho), extra={})


# ---------------------------------------------------------------------------
# Sparse least-squares systems shaped like DAzi's G matrix (the LSMR input):
# rows of ray-path weights over a band of neighbouring cells, times the depth
# kernels of the layers under them (a few hundred non-zeros per row), then
# one Tikhonov smoothing row per parameter (the cell and its lateral
# neighbours), as TikhRegul.f90 appends them.  Values real*4, 1-based
# triplets (the reference's iw/rw layout).

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

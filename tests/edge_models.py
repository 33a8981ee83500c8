"""Column models for the edge-case tests (CPU and GPU)."""
import numpy as np


def _batch(cols):
    """cols: list of (depz, vs, periods) -> CSR arrays."""
    if not cols:
        z = np.zeros(1, np.int64)
        return z, np.zeros(0, np.float32), np.zeros(0, np.float32), z.copy(), np.zeros(0)
    node_off = np.concatenate([[0], np.cumsum([c[0].size for c in cols])]).astype(np.int64)
    per_off = np.concatenate([[0], np.cumsum([c[2].size for c in cols])]).astype(np.int64)
    depz = np.concatenate([c[0] for c in cols]).astype(np.float32)
    vs = np.concatenate([c[1] for c in cols]).astype(np.float32)
    per = np.concatenate([c[2] for c in cols]).astype(np.float64)
    return node_off, depz, vs, per_off, per


def _random_columns(n, seed=7):
    """Seeded random 2-12 node models, half of them over a slow half-space
    (about one in ten has a period without a root)."""
    rng = np.random.default_rng(seed)
    cols = []
    for _ in range(n):
        nz = int(rng.integers(3, 12))
        dep = np.concatenate([[0.0], np.cumsum(rng.uniform(0.5, 20.0, nz - 1))]).astype(np.float32)
        vs = rng.uniform(0.5, 5.0, nz).astype(np.float32)
        if rng.random() < 0.5:
            vs[-1] = np.float32(rng.uniform(0.5, 2.0))
        per = np.sort(rng.uniform(0.2, 150.0, int(rng.integers(3, 12))))
        cols.append((dep, vs, per))
    return cols


def leaky_periods(pv, vs_halfspace, brocher):
    """Periods whose phase velocity is at or above 0.97 x the half-space P
    speed: both of the half-space's vertical wavenumbers are imaginary, and
    tregn96 picks their sign through signed-zero rounding in its complex
    arithmetic, so Lsen_Gsc is not comparable there (the library takes the
    principal branch +i).  The 3 % margin covers the Earth flattening."""
    vp_hs = brocher(np.asarray([vs_halfspace], np.float32))[0][0]
    return np.asarray(pv) >= 0.97 * vp_hs

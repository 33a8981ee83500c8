"""Checker of the GPU LSMR (test infrastructure only): the reference's SciPy
backend of its LSMR call, restated.

code/depthkernel_lab/scipy_lsmr_triplet_solver.py:60-90 builds
coo_matrix((data, (row - base, col - base)), shape=(m, n)).tocsr() from the
triplets (float64 with --float-dtype float64) and calls
scipy.sparse.linalg.lsmr(matrix, rhs, damp, atol, btol, conlim, maxiter);
the Fortran driver selects it with DAZI_LSMR_BACKEND=scipy
(code/src_inv_iso_joint/Main_Jt.f90:1163-1171).  The algorithm is SciPy's
implementation of LSMR (Fong & Saunders, SIAM J. Sci. Comput. 33, 2011),
a third-party dependency the reference does not vendor; it runs with the
SciPy of this image (1.18)."""
from __future__ import annotations

import numpy as np


def lsmr(row, col, val, b, m, n, *, damp=0.0, atol=1e-6, btol=1e-6, conlim=1e8, maxiter=None,
         index_base=1):
    """(x, istop, itn, normr, normar, norma, conda, normx) as SciPy returns
    them, for the triplets (row, col, val) with the given index base."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.linalg import lsmr as sp_lsmr
    r = np.asarray(row, np.int64) - index_base
    c = np.asarray(col, np.int64) - index_base
    a = coo_matrix((np.asarray(val, np.float64), (r, c)), shape=(m, n)).tocsr()
    out = sp_lsmr(a, np.asarray(b, np.float64), damp=damp, atol=atol, btol=btol, conlim=conlim,
                  maxiter=maxiter, show=False)
    return out[:8]

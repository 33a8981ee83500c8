"""Generate tests/golden/pdsurf_fd.npz: phase velocities and finite-difference
kernels dc/dVs, dc/dVp, dc/drho produced by the reference's own pDSurf tile
backend of depthkernel (code/depthkernel_lab/pdsurf_tile_senk_solver.py:
make_jobs :104-122, run_pdsurf_batch :125-175, process_tile :184-245, on
top of the Numba surf96 of code/pDSurfTomo-main/bin/surf96_disba.py:
surf96_batch :907), with the settings its command line defaults to (dln =
0.01, dc = dt = 0.005, iflsph = 1, FP64 model and output, the "default"
engine).  The reference's A/B script compares this backend against the
Fortran default_fortran_fd within fixed gates
(code/depthkernel_lab/run_iso_depthkernel_ab.py:324-336), so these vectors
pin the kernels of a reference run.

Columns: every 53rd column of examples/test4_Yunnan/voro/MOD (18 nodes,
depths 0-120 km, minthk = 4) as in tests/golden/yunnan_pv.npz, 36 periods
5..40 s.  Both modules are executed from their source text (not imported),
with numba's jit and guvectorize forced to cache=False and the tile solver's
`from surf96_disba import surf96_batch` served by the source-executed
module, so nothing precompiled that ships beside them is loaded.  The wall
time of process_tile on those columns (numba threads = all host cores, after
one warm-up call that compiles) is stored as well.

Usage: python tests/golden/make_pdsurf_fd.py REFERENCE_ROOT
"""
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

if len(sys.argv) != 2:
    sys.exit(__doc__)
ref = sys.argv[1]   # the reference checkout (the root of the DAzi project)
surf_src = os.path.join(ref, "code", "pDSurfTomo-main", "bin", "surf96_disba.py")
tile_src = os.path.join(ref, "code", "depthkernel_lab", "pdsurf_tile_senk_solver.py")


def exec_source(name, path):
    mod = types.ModuleType(name)
    mod.__file__ = path
    with open(path) as f:
        code = compile(f.read(), path, "exec")
    exec(code, mod.__dict__)
    return mod


def load_modules():
    import numba

    def nocache(deco):
        def wrapped(*args, **kwargs):
            kwargs["cache"] = False
            return deco(*args, **kwargs)
        return wrapped

    saved = numba.jit, numba.guvectorize
    numba.jit, numba.guvectorize = nocache(numba.jit), nocache(numba.guvectorize)
    sys.dont_write_bytecode = True
    try:
        surf = exec_source("surf96_disba", surf_src)
        sys.modules["surf96_disba"] = surf
        tile = exec_source("pdsurf_tile_senk_solver_src", tile_src)
    finally:
        numba.jit, numba.guvectorize = saved
    return surf, tile


def main():
    import numba
    g = np.load(os.path.join(HERE, "yunnan_pv.npz"))
    vel, depz, minthk = g["vel"], g["depz"], float(g["minthk"])
    nx, ny, nz = vel.shape
    cols = vel.reshape(nx * ny, nz, order="F")
    periods = np.arange(5.0, 41.0)
    picks = np.arange(0, nx * ny, 53)
    _, tile = load_modules()
    items = [(int(c), cols[c].astype(np.float64)) for c in picks]
    dep = depz.astype(np.float64)
    args = (dep, periods, minthk, 2, 0, 0.01, 0.005, 0.005)
    tile.process_tile(items[:1], *args)          # compile
    t0 = time.perf_counter()
    pv, svs, svp, srh, batch_s, njobs = tile.process_tile(items, *args)
    wall = time.perf_counter() - t0
    np.savez_compressed(os.path.join(HERE, "pdsurf_fd.npz"), columns=picks, periods=periods,
                        pv=pv, sen_vs=svs, sen_vp=svp, sen_rho=srh,
                        wall_seconds=wall, threads=numba.get_num_threads(), jobs=njobs)
    print(f"wrote pdsurf_fd.npz: {picks.size} columns x {periods.size} periods, {njobs} "
          f"surf96 jobs, {wall:.2f} s on {numba.get_num_threads()} threads "
          f"({picks.size * periods.size / wall:.1f} column-periods/s)")


if __name__ == "__main__":
    main()

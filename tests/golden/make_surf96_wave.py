"""Generate tests/golden/surf96_wave.npz: Love / Rayleigh phase and group
velocities from the reference's own Python surf96 (pDSurfTomo's Numba
translation, code/pDSurfTomo-main/bin/surf96_disba.py: surf96(), with
iflsph = 1, mode = 0, dc = 0.005 and dt = 0.005, the settings
code/depthkernel_lab/batch_pdsurf_numba_fd.py:54-66 runs it with), on
layered models built from the reference's Yunnan example.

Models: every 37th column of examples/test4_Yunnan/voro/MOD (18 nodes, Vs),
Brocher Vp/rho and the sublayer split with minthk = 4 (the oracle's
or_brocher / or_refine, both pinned to the golden phase-velocity maps),
stored as the real*4 layer arrays surfdisp96 receives.  Periods 5..40 s.

The module is executed from its source text (not imported), with numba's
jit and guvectorize forced to cache=False, so nothing precompiled that ships
beside it is loaded.

Usage: python tests/golden/make_surf96_wave.py REFERENCE_ROOT
"""
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

if len(sys.argv) != 2:
    sys.exit(__doc__)
ref = sys.argv[1]   # the reference checkout (the root of the DAzi project)
src_path = os.path.join(ref, "code", "pDSurfTomo-main", "bin", "surf96_disba.py")


def load_surf96():
    import numba

    def nocache(deco):
        def wrapped(*args, **kwargs):
            kwargs["cache"] = False
            return deco(*args, **kwargs)
        return wrapped

    saved = numba.jit, numba.guvectorize
    numba.jit, numba.guvectorize = nocache(numba.jit), nocache(numba.guvectorize)
    try:
        mod = types.ModuleType("surf96_disba_src")
        mod.__file__ = src_path
        with open(src_path) as f:
            code = compile(f.read(), src_path, "exec")
        exec(code, mod.__dict__)
    finally:
        numba.jit, numba.guvectorize = saved
    return mod


def main():
    from oracle import oracle as O
    g = np.load(os.path.join(HERE, "yunnan_pv.npz"))
    vel, depz, minthk = g["vel"], g["depz"], float(g["minthk"])
    nx, ny, nz = vel.shape
    cols = vel.reshape(nx * ny, nz, order="F")
    periods = np.arange(5.0, 41.0)
    picks = np.arange(0, nx * ny, 37)
    layers = []
    for c in picks:
        vs = cols[c].astype(np.float32)
        vp, rho = O.brocher(vs)
        thk, rvp, rvs, rrho, _ = O.refine(minthk, depz, vp, vs, rho)
        layers.append(np.stack([thk, rvp, rvs, rrho]))
    nl = np.array([L.shape[1] for L in layers])
    off = np.concatenate([[0], np.cumsum(nl)])
    flat = np.concatenate(layers, axis=1).astype(np.float32)

    S = load_surf96()
    out = {}
    for ifunc in (1, 2):
        for itype in (0, 1):
            cg = np.zeros((picks.size, periods.size))
            for j in range(picks.size):
                d, a, b, r = (flat[q, off[j]:off[j + 1]].astype(np.float64) for q in range(4))
                cg[j] = S.surf96(periods, d, a, b, r, 1, 0, itype, ifunc, 0.005, 0.005)
            out[f"cg_ifunc{ifunc}_itype{itype}"] = cg
            print(f"ifunc {ifunc} itype {itype}: {np.count_nonzero(cg)} nonzero of {cg.size}")
    np.savez_compressed(os.path.join(HERE, "surf96_wave.npz"), columns=picks, layer_off=off,
                        layers=flat, periods=periods, **out)
    print("wrote surf96_wave.npz")


if __name__ == "__main__":
    main()

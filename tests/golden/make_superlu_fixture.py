"""Site fields of a direct solve on the 32x32x24 mesh, the reference's production-solver stand-in.

The reference's production solver is MKL PARDISO (a closed binary, absent
here); its stand-in is SciPy's SuperLU (complex128, symmetric minimum-degree
ordering on A^T + A), run on the oracle's assembly of the seeded 32x32x24
log-normal model (147,456 tetrahedra, 179,800 edges).  One factorisation takes
minutes on a CPU, so the site fields are committed here and the GPU test
compares the device's batched solve against them without running SuperLU.

Systems: the 16-system batch of the batched workload on this mesh, with system
0 at the M2 period: system 0 (M2, velocity pattern 1) and system 12 (23.9345 h,
pattern 2) are solved directly.

Usage: python tests/golden/make_superlu_fixture.py
"""
import dataclasses
import os
import sys
import time

import numpy as np
import scipy.sparse.linalg as sla

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from actfemtide_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def batch_freqs(m):
    """The batch's frequencies: the 8 tidal periods twice (two velocity patterns), system 0 at M2."""
    freqs = 1.0 / (3600.0 * np.array(synth.BATCH_PERIODS_H))
    freqs[0] = m.freqs[0]
    return np.concatenate([freqs, freqs]), np.repeat([0, 1], 8).astype(np.int32)


def models():
    m = synth.tidal_box(32, 32, 24, seed=3, grf=True, block=False, name="box32x32x24")
    m2 = synth.tidal_box(32, 32, 24, seed=1003, grf=True, block=False, name="box32x32x24")
    return m, m2


def main():
    m, m2 = models()
    f, src = batch_freqs(m)
    of = O.OracleForward(m)
    out = {}
    for k in (0, 12):
        mk = m if src[k] == 0 else dataclasses.replace(m, F=m2.F, v=m2.v)
        A = O.forward_assemble(mk, of.line, of.n6line, of.pat, f[k], of.sigma_tet)
        t0 = time.time()
        lu = sla.splu(A.to_scipy().tocsc(), permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.0,
                      options=dict(SymmetricMode=True))
        x = lu.solve(A.b)
        tr = O.true_residual(A, x)
        fields, _, _ = of.sites(x, f[k])
        print(f"system {k}: f={f[k]:.6e} Hz, SuperLU {time.time() - t0:.0f} s, true residual {tr:.2e}")
        out[f"sites_{k}"] = fields[0]
        out[f"resid_{k}"] = tr
        out[f"freq_{k}"] = f[k]
    np.savez_compressed(os.path.join(HERE, "box32x32x24_superlu.npz"), sites=m.sites, **out)


if __name__ == "__main__":
    main()

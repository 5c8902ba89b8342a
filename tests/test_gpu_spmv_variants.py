"""The SpMV variants of a 16-system batch solve the same systems.

Each variant is pinned in turn (one row per warp, two systems per lane, and the tiled
kernel that stages a tile's distinct p rows in shared memory); the 16-system hybrid
solve on the 32x32x24 model must reach an FP64 true residual <= 1e-8 with each, in
FP64 and with the FP32 preconditioner, take the same iteration count within 2, and
give site fields within 1e-6 relative of the one-row-per-warp variant.  The tiled
variant sums a row in the two-systems-per-lane variant's order, so its q is the same;
only p^T q's partial sums are grouped differently.
"""
import numpy as np
import pytest

from actfemtide_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch_model():
    m = synth.tidal_box(32, 32, 24, seed=5, grf=True, block=False, name="box32x32x24")
    m2 = synth.tidal_box(32, 32, 24, seed=1005, grf=True, block=False, name="box32x32x24")
    freqs = 1.0 / (3600.0 * np.array(synth.BATCH_PERIODS_H))
    f = np.concatenate([freqs, freqs])
    src = np.repeat([0, 1], 8).astype(np.int32)
    return m, m2, f, src


@pytest.mark.parametrize("precision", ["fp64", "pc32"])
def test_spmv_variants_agree(gpulib, batch_model, precision):
    from actfemtide_b200.forward import Forward
    m, m2, f, src = batch_model
    out, its = {}, {}
    with Forward(0) as fw:
        fw.load_model(m, sources=[(m.F, m.v), (m2.F, m2.v)])
        fw.assemble()
        for rpw in (1, 8, 16):
            fw.set_spmv_rows_per_warp(rpw)
            r = fw.solve(f, srcs=src, precond="HYBRID", precision=precision, tol=1e-8)
            assert r.ok and r.resid_true <= 1e-8, (rpw, r)
            its[rpw] = r.iterations
            out[rpw] = fw.sites(m.sites, nsys=16)
    for rpw in (8, 16):
        assert abs(its[rpw] - its[1]) <= 2, its
        rel = np.abs(out[rpw] - out[1]).max() / np.abs(out[1]).max()
        assert rel <= 1e-6, (rpw, rel)


def test_tiled_pin_on_a_small_batch_falls_back(gpulib, batch_model):
    """Pinning the tiled variant on a batch it does not serve (fewer than 16 systems)
    falls back to one row per warp and still solves."""
    from actfemtide_b200.forward import Forward
    m, m2, f, src = batch_model
    with Forward(0) as fw:
        fw.load_model(m, sources=[(m.F, m.v), (m2.F, m2.v)])
        fw.assemble()
        fw.set_spmv_rows_per_warp(16)
        r = fw.solve(f[:4], srcs=src[:4], precond="HYBRID", precision="fp64", tol=1e-8)
        assert r.ok and r.resid_true <= 1e-8, r

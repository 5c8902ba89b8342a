"""The allocation-free site evaluation (afem_sites_noalloc) against afem_sites (GPU).

Collected last on purpose: it must pass on its own and after every other
test.  Two calls in a row must give afem_sites' values exactly (same kernels,
same order), and sizes over the scratch's limits must be refused.
"""
import numpy as np
import pytest

from actfemtide_b200 import synth
from actfemtide_b200.capi import AfemError

pytestmark = pytest.mark.gpu


def test_sites_noalloc_matches_sites_twice(gpulib):
    from actfemtide_b200.forward import Forward
    m = synth.tidal_box(6, 6, 8, seed=2, half_km=12.0)
    with Forward(0) as fw:
        fw.load_model(m, sources=[(m.F, m.v), (m.F, 0.5j * m.v)])
        fw.assemble()
        freqs = 1.0 / (3600.0 * np.array(synth.BATCH_PERIODS_H[:2]))
        assert fw.solve(freqs, [0, 1], precond="SSOR", tol=1e-8).ok
        rng = np.random.default_rng(9)
        pts = np.stack([rng.uniform(-11, 11, 300), rng.uniform(-11, 11, 300), rng.uniform(-11, 11, 300)], 1)
        ref = fw.sites(pts)
        first = fw.sites_noalloc(pts)
        second = fw.sites_noalloc(pts[::-1].copy())
        assert np.array_equal(first, ref)
        assert np.array_equal(second, ref[:, :, ::-1])
        with pytest.raises(AfemError):
            fw.sites_noalloc(np.zeros((1025, 3)))

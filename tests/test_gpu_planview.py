"""Plan-view element search on the GPU (FINDELEWITHGRID order) against the oracle, bit for bit.

The points are PREPOBSCOEFF_XY's cell centres; on the Kuhn box meshes many of
them lie on shared faces, where the grid list's order (not the tetrahedron
id) decides the element.  Elements, the sorted edge ids and the coefficient
rows must equal the oracle's restatement exactly.
"""
import numpy as np
import pytest

from actfemtide_b200 import capi, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fw(gpulib):
    from actfemtide_b200.forward import Forward
    f = Forward(0)
    yield f
    f.close()


@pytest.mark.parametrize("dims,half,depth", [((6, 6, 8), 12.0, -5.0), ((12, 12, 9), 50.0, -5.001),
                                             ((8, 8, 6), 50.0, -2.5)])
def test_grid_search_matches_oracle(fw, oracle, dims, half, depth):
    m = synth.tidal_box(*dims, seed=2, half_km=half)
    fw.load_model(m)
    line, n6 = fw.lines()
    pts = capi.xy_points(-half + 1.0, half - 1.0, -half + 1.0, half - 1.0, 2 * dims[0], 2 * dims[1], depth)
    item, ve, vf, iele = fw.site_coeffs_grid(pts)
    oi, ove, ovf, oiele = oracle.prepobscoeff_grid(m, n6, pts)
    assert np.array_equal(iele, oiele)
    assert np.array_equal(item, oi)
    assert np.array_equal(ve, ove) and np.array_equal(vf, ovf)


def test_grid_sites_equal_brute_force_fields_inside_elements(fw):
    """Away from shared faces both searches find the same tetrahedron, so the fields agree."""
    m = synth.tidal_box(6, 6, 8, seed=2, half_km=12.0)
    fw.load_model(m)
    fw.assemble()
    assert fw.solve(m.freqs[0], precond="SSOR", tol=1e-8).ok
    rng = np.random.default_rng(5)
    pts = np.stack([rng.uniform(-10, 10, 64), rng.uniform(-10, 10, 64), rng.uniform(-10, 10, 64)], 1)
    a = fw.sites(pts)
    b = fw.sites_grid(pts)
    assert np.array_equal(a, b)

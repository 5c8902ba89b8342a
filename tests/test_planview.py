"""Plan-view sites (PREPOBSCOEFF_XY), host side: point layout, SORT_INDEX and the grid-list search.

The grid list orders tetrahedra by the box of their centroid with SORT_INDEX,
a heapsort, so equal keys leave in the heapsort's own order and
FINDELEWITHGRID returns the first holder of a site in that order.  The
product's heapsort is checked against the oracle's on keys with many ties;
the oracle's grid search is checked against the brute-force FINDELEMENT0
wherever one tetrahedron alone holds the site.
"""
import numpy as np

from actfemtide_b200 import capi, synth


def test_xy_points_layout():
    p = capi.xy_points(-50.0, 50.0, -40.0, 40.0, 4, 5, -5.001)
    assert p.shape == (20, 3)
    dx, dy = 100.0 / 4, 80.0 / 5
    for j in range(1, 5):
        for i in range(1, 6):
            ii = (j - 1) * 5 + i - 1
            assert p[ii, 0] == (j - 1) * dx + -50.0 + dx / 2.0
            assert p[ii, 1] == (i - 1) * dy + -40.0 + dy / 2.0
            assert p[ii, 2] == -5.001


def test_sort_index_equal_keys_match_oracle(oracle):
    import ctypes as C
    L = capi.lib()
    rng = np.random.default_rng(1)
    for n in (1, 2, 3, 17, 100, 1000):
        keys = rng.integers(0, max(2, n // 7), size=n).astype(np.float64)
        na = np.arange(1, n + 1, dtype=np.int32); ra = keys.copy()
        assert L.afem_sort_index(n, na.ctypes.data_as(C.c_void_p), ra.ctypes.data_as(C.c_void_p)) == 0
        on, orr = oracle.sort_index(np.arange(1, n + 1), keys)
        assert np.array_equal(ra, orr) and np.array_equal(na, on)


def test_grid_search_agrees_with_brute_force(oracle):
    m = synth.tidal_box(6, 6, 8, seed=1, half_km=12.0)
    line, n6 = oracle.mkline(m.node, m.n4)
    rng = np.random.default_rng(3)
    pts = np.stack([rng.uniform(-11.0, 11.0, 200), rng.uniform(-11.0, 11.0, 200), rng.uniform(-11.0, 11.0, 200)], 1)
    _, _, _, ig = oracle.prepobscoeff_grid(m, n6, pts)
    _, _, _, ib = oracle.prepobscoeff(m, n6, pts)
    # random points lie strictly inside one tetrahedron: both searches find it
    assert np.array_equal(ig, ib)

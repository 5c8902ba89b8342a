"""The 3-D MT forward on the device against the CPU oracle (oracle/afem_oracle_mt.cpp).

Reference: src/src_3DMT/n_ebfem_3DMT.f90:38-113, forward_3DMT.f90 (GENBCMT, GENMAT_MT,
SET_BC_3DJoint), src/src_2D/forward_2DTM.f90 (the 2-D TM boundary solves) and
src/src_2D/m_surface_type.f90 (EXTRACT6SURFACES, COND3DTO2D, the triangle element).
Tolerances: the 2-D systems (matrix and lifted right-hand side) bit for bit; the
2-D solutions by their residual (1e-14) and within 1e-6 of SciPy's SuperLU, the
stand-in for PARDISO (both are backward stable; the resistive air leaves their
solutions 1e-8 apart at 0.01 Hz); the 3-D matrix within 1e-12 of each row's largest
entry; impedances within 1e-6 of the oracle's direct solve.
"""
import numpy as np
import pytest

from actfemtide_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    from actfemtide_b200.forward import MTForward
    m = synth.mt_box(6, 5, 4, 6, grf=True, seed=3, block_sigma=0.5, freqs=[0.1, 0.01, 0.001])
    fw = MTForward(0)
    fw.load_mt_model(m)
    fw._sizes()
    import ctypes as C
    line = np.zeros((fw.nline, 2), np.int32)
    n6 = np.zeros((m.ntet, 6), np.int32)
    fw._check(fw._L.afem_get_lines(fw.ctx, C.byref(C.c_int()), line.ctypes.data, n6.ctypes.data))
    mt = O.MTOracle(m, line, n6)
    yield m, fw, mt, line, n6
    fw.close()


def _by_line3d(A, line3d):
    """Dense copy of a surface system indexed by the position of each line in 3-D id order."""
    order = np.argsort(line3d)
    return A.toarray()[np.ix_(order, order)], order


def test_face_systems_bit_exact(small):
    m, fw, mt, _, _ = small
    for f in m.freqs:
        for j in (2, 3, 4, 5):
            d = fw.mt_face(j, f)
            F = mt.face(j, f)
            assert np.array_equal(np.sort(d["line3d"]), F.line3d)
            Ad, order = _by_line3d(d["A"], d["line3d"])
            Ao = F.A.to_scipy().toarray()  # surface lines are numbered in 3-D order
            np.testing.assert_array_equal(Ad.real, Ao.real)
            np.testing.assert_array_equal(Ad.imag, Ao.imag)
            np.testing.assert_array_equal(d["rhs"][order], F.rf)
            # the band L D L^T solution: residual and agreement with a pivoted sparse LU
            x = d["bs"]
            res = np.linalg.norm(d["A"] @ x - d["rhs"]) / np.linalg.norm(d["rhs"])
            assert res <= 1e-14, (j, f, res)
            xo = F.solve()
            if f >= 0.01:
                assert np.abs(x[order] - xo).max() <= 1e-6 * np.abs(xo).max(), (j, f)


def test_boundary_values_match_the_oracle(small):
    m, fw, mt, _, _ = small
    f = 0.01
    av, bc = fw.mt_boundary(f)
    avo, bco, bs = mt.boundary(f)
    np.testing.assert_array_equal(bc, bco)
    # the same values up to the 2-D solutions' agreement; the top lines exactly
    top = np.zeros(fw.nline, bool)
    top[mt.surface(1)["line3d"] - 1] = True
    for j in (2, 3, 4, 5):
        top[mt.surface(j)["line3d"] - 1] = False
    np.testing.assert_array_equal(av[:, top], avo[:, top])
    assert np.abs(av - avo).max() <= 1e-6 * np.abs(avo).max()


def test_mt_system_matches_the_oracle(small):
    m, fw, mt, _, _ = small
    f = m.freqs[:1]
    fw.mt_forward(f, m.sites, tol=1e-8)
    av, bc = fw.mt_boundary(f[0])
    A, rf = mt.system(f[0], av, bc)   # the oracle's GENMAT_MT + SET_BC_3DJoint on the device's values
    amax = max(np.abs(A.D).max(), np.abs(A.AU).max())
    for pol in range(2):
        e = fw.export_system(f[0], pol)
        np.testing.assert_array_equal(e["bc"], bc)
        np.testing.assert_array_equal(e["IAU"], A.IAU)
        np.testing.assert_array_equal(e["D"].real, A.D.real)       # curl-curl and the identity rows
        np.testing.assert_array_equal(e["AU"].real, A.AU.real)
        assert np.abs(e["D"] - A.D).max() <= 1e-12 * amax
        assert np.abs(e["AU"] - A.AU).max() <= 1e-12 * amax
        assert np.abs(e["b"] - rf[pol]).max() <= 1e-12 * np.abs(rf[pol]).max(), pol


def test_halfspace_apparent_resistivity_on_device():
    """MT over a 10 Ohm m half-space on the device: 10 Ohm m and 45 / -135 degrees within the
    mesh's discretisation error, and the oracle's direct-solve impedances within 1e-6."""
    from actfemtide_b200.forward import MTForward
    m = synth.mt_box(10, 10, 6, 12, sigma=0.1, freqs=[0.01], site_grid=(-20.0, 0.0, 20.0))
    with MTForward(0) as fw:
        fw.load_mt_model(m)
        r = fw.mt_forward(m.freqs, m.sites, tol=1e-9)
        assert r.solve.ok and r.solve.resid_true <= 1e-9, r.solve
        np.testing.assert_allclose(r.rho[0, 1], 10.0, rtol=0.025)
        np.testing.assert_allclose(r.rho[0, 2], 10.0, rtol=0.025)
        np.testing.assert_allclose(r.pha[0, 1], -135.0, atol=2.5)
        np.testing.assert_allclose(r.pha[0, 2], 45.0, atol=2.5)
        line, n6 = O.mkline(m.node, m.n4)
        ro = O.MTOracle(m, line, n6).forward(m.freqs, m.sites)
        zs = np.abs(ro["z"][0]).max()
        assert np.abs(r.z[0] - ro["z"][0]).max() <= 1e-6 * zs
        assert np.abs(r.be - ro["be"]).max() <= 1e-6 * np.abs(ro["be"]).max()


def test_three_frequencies_in_two_batches(small):
    """Three frequencies = six systems, solved as a batch of 4 and one of 2; the conductive block
    and the random field make every impedance component non-trivial."""
    m, fw, mt, _, _ = small
    r = fw.mt_forward(m.freqs, m.sites, tol=1e-9)
    assert r.solve.ok and r.solve.resid_true <= 1e-9, r.solve
    ro = mt.forward(m.freqs, m.sites)
    for k in range(len(m.freqs)):
        zs = np.abs(ro["z"][k]).max()
        assert np.abs(r.z[k] - ro["z"][k]).max() <= 1e-6 * zs, k
        np.testing.assert_allclose(r.rho[k], ro["rho"][k], rtol=1e-5)


def test_mt_rejects_bad_conductivity(small):
    from actfemtide_b200.capi import AfemError
    m, fw, _, _, _ = small
    with pytest.raises(AfemError):
        fw.set_mt_cond(m.sigma_air, 1, sigma_file=m.sigma_land[:-1])  # one value short
        fw.mt_forward(m.freqs[:1], m.sites)
    fw.set_mt_cond(m.sigma_air, 1, sigma_file=m.sigma_land)

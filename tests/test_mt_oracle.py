"""The CPU oracle of the 3-D MT forward (oracle/afem_oracle_mt.cpp) against what it must satisfy.

The reference ships no MT data and cannot be compiled here, so the MT oracle is
pinned by: the surface extraction's counts on a box (EXTRACT6SURFACES,
src/src_2D/m_surface_type.f90:189-502), the identities of the 2-D TM element
(its curl-curl annihilates discrete gradients, its mass matrix is SPD;
GENMAT2DTM, src/src_2D/forward_2DTM.f90:253-363), GENBCMT's assignment order
(src/src_3DMT/forward_3DMT.f90:92-177) and the known answers of MT over a uniform
half-space: apparent resistivity 1/sigma and phase 45 degrees (mod 180) where the skin
depth is well above the bottom boundary, and the 1-D answer of a layer over a perfect
conductor (the E = 0 bottom) where it is not.
"""
import numpy as np
import pytest

from actfemtide_b200 import synth
from oracle import oracle as O


@pytest.fixture(scope="module")
def box():
    m = synth.mt_box(6, 5, 4, 6, sigma=0.1, freqs=[0.01])
    line, n6 = O.mkline(m.node, m.n4)
    return m, line, n6, O.MTOracle(m, line, n6)


def test_surfaces_of_a_box(box):
    m, line, _, mt = box
    nx, ny, nz = m.dims
    dims = {1: (nx, ny), 2: (nx, nz), 3: (ny, nz), 4: (nx, nz), 5: (ny, nz), 6: (nx, ny)}
    for j, (a, b) in dims.items():
        s = mt.surface(j)
        assert s["x1x2"].shape[0] == (a + 1) * (b + 1)
        assert s["n3"].shape[0] == 2 * a * b
        assert s["line3d"].shape[0] == a * (b + 1) + b * (a + 1) + a * b
        # FINDBOUNDARYLINE: a top and a bottom run of a lines, left and right runs of b lines
        assert np.bincount(s["flag"], minlength=5)[1:].tolist() == [a, a, b, b]
        xy = s["x1x2"]
        n3 = s["n3"] - 1
        assert (n3[:, 0] < n3[:, 1]).all() and (n3[:, 0] < n3[:, 2]).all()  # smallest node first
        e1 = xy[n3[:, 1]] - xy[n3[:, 0]]
        e2 = xy[n3[:, 2]] - xy[n3[:, 0]]
        assert (e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0] > 0).all()  # anticlockwise
        # n3line(t, l) runs from n3(t, l) to n3(t, l+1) with the sign of the 3-D line's direction
        ln = s["line"] - 1
        for t in range(n3.shape[0]):
            for l in range(3):
                e = s["n3line"][t, l]
                a0, b0 = ln[abs(e) - 1]
                p, q = n3[t, l], n3[t, (l + 1) % 3]
                assert (a0, b0) == ((p, q) if e > 0 else (q, p))
        # surface lines are 3-D lines, in 3-D order, with both nodes on the plane
        assert (np.diff(s["line3d"]) > 0).all()
    # the triangle's tetrahedron holds all three of its nodes
    for j in (1, 3, 6):
        s = mt.surface(j)
        onnodes = np.nonzero(np.isin(np.arange(1, m.node + 1), np.unique(m.n4)))[0]
        assert onnodes.size == m.node
        xyz = m.xyz
        face_nodes = []
        for t in range(s["n3"].shape[0]):
            tet = m.n4[s["tet"][t] - 1]
            tri = [int(np.nonzero((xyz == p).all(axis=1))[0][0]) + 1 for p in
                   _lift(j, s["x1x2"][s["n3"][t] - 1], mt.minmax())]
            assert set(tri) <= set(tet.tolist())
            face_nodes.append(tri)


def _lift(j, yz, mm):
    """Surface-plane coordinates back to 3-D points on surface j."""
    out = np.zeros((yz.shape[0], 3))
    plane = {1: (2, mm[5]), 2: (1, mm[3]), 3: (0, mm[0]), 4: (1, mm[2]), 5: (0, mm[1]), 6: (2, mm[4])}[j]
    free = {1: (0, 1), 6: (0, 1), 2: (0, 2), 4: (0, 2), 3: (1, 2), 5: (1, 2)}[j]
    out[:, free[0]] = yz[:, 0]
    out[:, free[1]] = yz[:, 1]
    out[:, plane[0]] = plane[1]
    return out


def test_face_element_identities(box):
    _, _, _, mt = box
    for j in (2, 3):
        s = mt.surface(j)
        K = mt.face(j, 0.0, apply_bc=False).A.to_scipy().toarray()
        f = 0.01
        A = mt.face(j, f, apply_bc=False).A.to_scipy().toarray()
        assert np.array_equal(A.real, K.real)  # the curl-curl part does not depend on the frequency
        M = A.imag / (2 * np.pi * f)
        # curl-curl annihilates the discrete gradients: G = +1 at line(2), -1 at line(1)
        n, nn = s["line"].shape[0], s["x1x2"].shape[0]
        G = np.zeros((n, nn))
        G[np.arange(n), s["line"][:, 1] - 1] = 1.0
        G[np.arange(n), s["line"][:, 0] - 1] = -1.0
        assert np.abs(K.real @ G).max() <= 1e-12 * np.abs(K).max() * np.abs(G).sum(axis=0).max()
        np.testing.assert_allclose(M, M.T, rtol=0, atol=1e-15 * np.abs(M).max())
        assert np.linalg.eigvalsh(M).min() > 0.0


def test_face_dirichlet_rows(box):
    _, _, _, mt = box
    s = mt.surface(2)
    F = mt.face(2, 0.01)
    top = s["flag"] == 1
    # GENBC2D: the top run carries El = (y2 - y1) * 1 mV/km, the other runs 0
    y = s["x1x2"][:, 0]
    np.testing.assert_array_equal(F.gval[top].real, y[s["line"][top, 1] - 1] - y[s["line"][top, 0] - 1])
    assert (F.gval[~top] == 0).all()
    assert F.A.bc.sum() == (s["flag"] > 0).sum()
    x = F.solve()
    np.testing.assert_array_equal(x[F.A.bc == 1], F.gval[F.A.bc == 1])


def test_genbcmt_assignment_order(box):
    m, line, _, mt = box
    f = 0.01
    om = 2 * np.pi * f
    av, bc, bs = mt.boundary(f)
    # every line with both nodes on one of the six planes is Dirichlet
    mm = mt.minmax()
    lo, hi = mm[0::2] + np.float32(0.1), mm[1::2] - np.float32(0.1)
    p = m.xyz[line - 1]  # (nline, 2, 3)
    onplane = np.zeros(len(line), bool)
    for c in range(3):
        onplane |= (p[:, :, c] <= lo[c]).all(axis=1) | (p[:, :, c] >= hi[c]).all(axis=1)
    np.testing.assert_array_equal(bc.astype(bool), onplane)
    # top lines: i/omega * dx and i/omega * dy; side lines of north/south set Ex, of west/east Ey
    s1 = mt.surface(1)
    d = m.xyz[line[s1["line3d"] - 1, 1] - 1] - m.xyz[line[s1["line3d"] - 1, 0] - 1]
    side = np.zeros(len(line), bool)
    for j in (2, 3, 4, 5):
        side[mt.surface(j)["line3d"] - 1] = True
    top_only = ~side[s1["line3d"] - 1]
    np.testing.assert_array_equal(av[0, s1["line3d"] - 1][top_only], (1j / om * d[:, 0])[top_only])
    np.testing.assert_array_equal(av[1, s1["line3d"] - 1][top_only], (1j / om * d[:, 1])[top_only])
    bottom = mt.surface(6)["line3d"] - 1
    for j, col in ((2, 0), (3, 1), (4, 0), (5, 1)):
        s = mt.surface(j)
        keep = ~np.isin(s["line3d"] - 1, bottom) if col == 1 else np.ones(len(s["line3d"]), bool)
        np.testing.assert_array_equal(av[col, s["line3d"] - 1][keep], (1j / om * bs[j - 2])[keep])
    # the bottom loop resets only the column the side loop left behind (Ey)
    assert (av[1, bottom] == 0).all()


def test_halfspace_apparent_resistivity():
    """MT over a 10 Ohm m half-space: rho_a = 10 Ohm m and |phase| = 45 / 135 degrees at every site,
    Zxx = Zyy = 0, to the discretisation error of a 10 x 10 x (6 + 12) graded mesh (measured: 1.5 %,
    1.6 degrees, |Zxx|, |Zyy| up to 1.1 % of |Zxy| from the Kuhn split's directional bias)."""
    m = synth.mt_box(10, 10, 6, 12, sigma=0.1, freqs=[0.01], site_grid=(-20.0, 0.0, 20.0))
    line, n6 = O.mkline(m.node, m.n4)
    r = O.MTOracle(m, line, n6).forward(m.freqs, m.sites)
    assert max(np.max(x) for x in r["resid"]) < 1e-12
    rho, pha, z = r["rho"][0], r["pha"][0], r["z"][0]
    np.testing.assert_allclose(rho[1], 10.0, rtol=0.025)
    np.testing.assert_allclose(rho[2], 10.0, rtol=0.025)
    np.testing.assert_allclose(pha[1], -135.0, atol=2.5)
    np.testing.assert_allclose(pha[2], 45.0, atol=2.5)
    assert np.abs(z[[0, 3]]).max() < 2e-2 * np.abs(z[[1, 2]]).min()


def _z1d_over_conductor(f, sigma, depth_km):
    """Impedance (SI, E/H) of a uniform earth of `depth_km` over a perfect conductor (E = 0), the
    textbook 1-D layer recursion with a zero impedance below: Z = Z_i tanh(k h), k = sqrt(i w mu sigma)."""
    mu = 4e-7 * np.pi
    w = 2 * np.pi * f
    k = np.sqrt(1j * w * mu * sigma)
    return 1j * w * mu / k * np.tanh(k * depth_km * 1e3)


def test_halfspace_over_the_bottom_boundary():
    """At 1 mHz a 10 Ohm m earth's skin depth (50 km) reaches the E = 0 bottom at -50 km, so the
    answer is that of a 50 km layer over a perfect conductor: rho_a = 12.44 Ohm m, phase 59.3
    degrees, not 10 and 45.  The oracle's chain on a 10 x 10 x (6 + 18) mesh with 1.3 km surface
    cells reproduces it (measured: 0.46 % and 1.0 degree)."""
    f = 0.001
    m = synth.mt_box(10, 10, 6, 18, ratio_earth=1.08, sigma=0.1, freqs=[f], site_grid=(-20.0, 0.0, 20.0))
    line, n6 = O.mkline(m.node, m.n4)
    r = O.MTOracle(m, line, n6).forward(m.freqs, m.sites)
    Z = _z1d_over_conductor(f, 0.1, 50.0)
    rho = abs(Z) ** 2 / (2 * np.pi * f * 4e-7 * np.pi)
    pha = np.degrees(np.angle(Z))
    assert abs(rho - 12.44) < 0.01 and abs(pha - 59.34) < 0.01
    np.testing.assert_allclose(r["rho"][0][1:3], rho, rtol=0.01)
    np.testing.assert_allclose(r["pha"][0][1] + 180.0, pha, atol=1.5)
    np.testing.assert_allclose(r["pha"][0][2], pha, atol=1.5)


def test_layered_earth_converges_with_the_surface_cells():
    """10 Ohm m over 100 Ohm m (below the mesh level near 9 km) at 0.01 Hz over the E = 0 bottom:
    the oracle's apparent resistivity approaches the 1-D layered answer as the first cell under
    the surface thins, about in proportion to it (B = curl A is constant in a tetrahedron, so a
    site 1 m deep sees the top cell's average; measured 15.3, 8.2, 4.3 % for 1.34, 0.66, 0.32 km)."""
    f = 0.01
    mu = 4e-7 * np.pi
    w = 2 * np.pi * f
    errs, firsts = [], []
    for ratio in (1.08, 1.15, 1.22):
        m = synth.mt_box(10, 10, 6, 18, ratio_earth=ratio, sigma=0.1, freqs=[f], site_grid=(0.0,))
        z = np.unique(m.xyz[:, 2])
        zl = z[z < 0]
        d = float(-zl[np.argmin(np.abs(zl + 10.0))])
        cen = m.xyz[m.n4[m.nphys1:] - 1].mean(axis=1)
        m.sigma_land = np.where(cen[:, 2] < -d, 0.01, m.sigma_land)
        line, n6 = O.mkline(m.node, m.n4)
        r = O.MTOracle(m, line, n6).forward(m.freqs, m.sites)
        # the 1-D recursion: 100 Ohm m from -d to -50 km over the conductor, 10 Ohm m above
        k = np.sqrt(1j * w * mu * np.array([0.1, 0.01]))
        zi = 1j * w * mu / k
        Z = zi[1] * np.tanh(k[1] * (50.0 - d) * 1e3)
        t = np.tanh(k[0] * d * 1e3)
        Z = zi[0] * (Z + zi[0] * t) / (zi[0] + Z * t)
        rho = abs(Z) ** 2 / (w * mu)
        errs.append(abs(r["rho"][0][1][0] / rho - 1.0))
        firsts.append(-zl[-1])
    assert firsts[0] > firsts[1] > firsts[2]
    assert errs[0] > errs[1] > errs[2] and errs[2] < 0.06, errs
    # first order: the error per km of the first cell stays within a factor 1.5
    per_km = np.array(errs) / np.array(firsts)
    assert per_km.max() <= 1.5 * per_km.min(), per_km


def test_mt_box_layout():
    """The synthetic MT model: graded levels finest at the surface, air (tag 1) above and earth
    (tag 3, 4 in the block) below z = 0 by centroid, the earth tetrahedra last with one
    conductivity each, and each region's first cell set by its ratio."""
    m = synth.mt_box(6, 5, 4, 6, ratio_air=1.3, ratio_earth=1.1, block_sigma=0.5, half_km=20.0)
    z = np.unique(m.xyz[:, 2])
    assert z[0] == -50.0 and z[-1] == 50.0 and 0.0 in z and z.size == 4 + 6 + 1
    dz = np.diff(z)
    i0 = int(np.searchsorted(z, 0.0))
    assert np.all(np.diff(dz[i0:]) > 0) and np.all(np.diff(dz[:i0]) < 0)  # thicker away from 0
    np.testing.assert_allclose(dz[i0 + 1] / dz[i0], 1.3)
    np.testing.assert_allclose(dz[i0 - 2] / dz[i0 - 1], 1.1)
    cz = m.xyz[m.n4 - 1].mean(axis=1)[:, 2]
    assert np.all(m.tag[cz > 0] == 1) and np.all(m.tag[cz < 0] >= 3)
    assert np.all(np.diff(m.tag >= 3) >= 0)  # earth last
    assert m.sigma_land.shape[0] == int((m.tag >= 3).sum()) == m.ntet - m.nphys1
    assert set(np.unique(m.sigma_land)) == {0.1, 0.5} and np.all(m.sigma_land[m.tag[m.nphys1:] == 4] == 0.5)

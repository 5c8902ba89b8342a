"""CPU oracle checks: known answers from the reference sources, counts, identities, direct solves.

The reference ships no tests or golden data for this path (it has no tests/
directory and no CI), so the oracle is pinned by (i) the two known-answer examples written
in the reference's own sources, (ii) structural counts of the Kuhn meshes,
(iii) mathematical identities of the edge-element system, (iv) a direct
solve, and (v) the committed golden fixtures (regression).
"""
import os

import numpy as np
import pytest

from actfemtide_b200 import synth

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_sort_index_known_answer(oracle):
    # src/solver/sort_index.f90:3-10: n4 = (5,10,1,20), r4 = (3,2,1,4) sorted by r4
    na, ra = oracle.sort_index([5, 10, 1, 20], [3.0, 2.0, 1.0, 4.0])
    assert list(ra) == [1.0, 2.0, 3.0, 4.0]
    assert list(na) == [1, 10, 5, 20]


def test_sort_index_heap_sort_matches_argsort(oracle):
    rng = np.random.default_rng(0)
    for n in range(1, 40):
        r = rng.permutation(n).astype(np.float64) + 1.0
        na, ra = oracle.sort_index(np.arange(1, n + 1), r)
        assert np.array_equal(ra, np.sort(r))
        assert np.array_equal(na, np.argsort(r) + 1)


def test_crs_matvec_known_answer(oracle):
    # src/common/test.f90:5-20: A1 (3x5) times B (5x5) = A*B, column by column through mul_matcrs_cv
    A1 = np.array([[1, 0, 1, 0, 0], [2, 1, 3, 0, 0], [0, 1, 0, 1, 0]], dtype=np.float64)
    B = np.array([[1, 3, 1, 0, 0], [1, 0, 0, 2, 0], [2, 0, 3, 1, 0], [0, 1, 2, 4, 0], [0, 0, 0, 0, 0]], dtype=float)
    AB = np.array([[3, 3, 4, 1, 0], [9, 6, 11, 5, 0], [1, 1, 2, 6, 0]], dtype=np.float64)
    stack = [0]; item = []; val = []
    for r in range(3):
        for c in range(5):
            if A1[r, c] != 0:
                item.append(c + 1); val.append(A1[r, c])
        stack.append(len(item))
    for j in range(5):
        out = oracle.mul_matcrs_cv(stack, item, val, B[:, j].astype(np.complex128))
        assert np.array_equal(out.real, AB[:, j])


def test_mesh_counts_box20(oracle):
    m = synth.small_model()
    line, n6 = oracle.mkline(m.node, m.n4)
    assert m.ntet == 48000 and m.node == 9261
    assert line.shape[0] == 59660
    INU, IAU, INL, IAL = oracle.pattern(line.shape[0], n6)
    assert line.shape[0] + len(IAU) + len(IAL) == 938060


def test_numbering_rules(oracle):
    m = synth.tiny_model()
    line, n6 = oracle.mkline(m.node, m.n4)
    # line(1,:) < line(2,:), groups by the smaller node ascending
    assert np.all(line[:, 0] < line[:, 1])
    assert np.all(np.diff(line[:, 0]) >= 0)
    # n6line sign = orientation of kl(j) against the (n1 < n2) edge
    kl = [(0, 1), (1, 2), (0, 2), (0, 3), (1, 3), (2, 3)]
    for t in range(m.ntet):
        for j, (a, b) in enumerate(kl):
            na, nb = m.n4[t, a], m.n4[t, b]
            e = abs(n6[t, j]) - 1
            assert set(line[e]) == {na, nb}
            assert (n6[t, j] > 0) == (na < nb)


def test_pattern_is_symmetric_and_sorted(oracle):
    m = synth.tiny_model()
    line, n6 = oracle.mkline(m.node, m.n4)
    INU, IAU, INL, IAL = oracle.pattern(line.shape[0], n6)
    n = line.shape[0]
    up = {(i, IAU[k] - 1) for i in range(n) for k in range(INU[i], INU[i + 1])}
    lo = {(IAL[k] - 1, i) for i in range(n) for k in range(INL[i], INL[i + 1])}
    assert up == lo
    for i in range(n):
        assert np.all(np.diff(IAU[INU[i]:INU[i + 1]]) > 0) and np.all(IAU[INU[i]:INU[i + 1]] > i + 1)
        assert np.all(np.diff(IAL[INL[i]:INL[i + 1]]) > 0) and np.all(IAL[INL[i]:INL[i + 1]] < i + 1)


def _gradient_matrix(line, node):
    n = line.shape[0]
    G = np.zeros((n, node))
    G[np.arange(n), line[:, 1] - 1] = 1.0
    G[np.arange(n), line[:, 0] - 1] = -1.0
    return G


def test_curl_curl_annihilates_gradients(oracle):
    # discrete de Rham property of first-order Nedelec elements: K G = 0
    m = synth.tiny_model()
    of = oracle.OracleForward(m)
    Kd, Ku, Md, Mu = oracle.assemble_split(m, of.n6line, of.pat, of.sigma_tet)
    n = of.line.shape[0]
    INU, IAU = of.pat[0], of.pat[1]
    K = np.diag(Kd)
    for i in range(n):
        for k in range(INU[i], INU[i + 1]):
            K[i, IAU[k] - 1] = Ku[k]; K[IAU[k] - 1, i] = Ku[k]
    G = _gradient_matrix(of.line, m.node)
    assert np.abs(K @ G).max() < 1e-12 * np.abs(K).max()
    # mass matrix: symmetric positive definite
    M = np.diag(Md)
    for i in range(n):
        for k in range(INU[i], INU[i + 1]):
            M[i, IAU[k] - 1] = Mu[k]; M[IAU[k] - 1, i] = Mu[k]
    assert np.linalg.eigvalsh(M).min() > 0


def test_split_assembly_equals_complex_assembly(oracle):
    m = synth.tiny_model()
    of = oracle.OracleForward(m)
    A = of.assemble(m.freqs[0], apply_bc=False)
    Kd, Ku, Md, Mu = oracle.assemble_split(m, of.n6line, of.pat, of.sigma_tet)
    om = 2 * np.pi * m.freqs[0]
    assert np.array_equal(A.D.real, Kd) and np.array_equal(A.AU.real, Ku)
    np.testing.assert_allclose(A.D.imag, om * Md, rtol=1e-14, atol=0)
    np.testing.assert_allclose(A.AU.imag, om * Mu, rtol=1e-14, atol=1e-300)


def test_dirichlet_rows(oracle):
    m = synth.tiny_model()
    of = oracle.OracleForward(m)
    A = of.assemble(m.freqs[0])
    bc = A.bc.astype(bool)
    assert bc.sum() > 0
    assert np.all(A.D[bc] == 1.0) and np.all(A.b[bc] == 0.0)
    S = A.to_scipy().toarray()
    off = S - np.diag(np.diag(S))
    assert np.all(off[bc, :] == 0) and np.all(off[:, bc] == 0)


def test_cocg_matches_direct_solve(oracle):
    import scipy.sparse.linalg as spla
    m = synth.tiny_model()
    of = oracle.OracleForward(m)
    A = of.assemble(m.freqs[0])
    xd = spla.spsolve(A.to_scipy().tocsc(), A.b)
    r = oracle.cocg13_single(A, precond="SSOR", resid=1e-13, maxit=100000)
    assert r["error"] == 0
    assert oracle.true_residual(A, r["x"]) < 1e-12
    # the curl-curl null space in the resistive air leaves x loosely determined;
    # the site fields (B = curl A, E in the conductors) are not
    o1, _, _ = of.sites(r["x"], m.freqs[0])
    o2, _, _ = of.sites(xd, m.freqs[0])
    assert np.abs(o1 - o2).max() <= 1e-8 * np.abs(o2).max()


def test_cocg_reference_semantics(oracle):
    m = synth.tiny_model()
    of = oracle.OracleForward(m)
    A = of.assemble(m.freqs[0])
    # NSET = 0 on first use -> ERROR 101
    assert oracle.cocg13_single(A, nset=0)["error"] == 101
    # iteration cap -> ERROR -100, ITER = MAXIT + 1 is the Fortran DO-variable value; here the count
    r = oracle.cocg13_single(A, precond="IC", resid=1e-30, maxit=3)
    assert r["error"] == -100
    # zero right-hand side -> x = 0, ITER = 0
    z = oracle.cocg13_single(A, b=np.zeros(A.n, np.complex128))
    assert z["iter"] == 0 and np.all(z["x"] == 0)


@pytest.mark.parametrize("name", ["tiny_2x2x4", "box4x4x6"])
def test_golden_fixture_regression(oracle, name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    line, n6 = oracle.mkline(int(g["xyz"].shape[0]), g["n4"])
    assert np.array_equal(line, g["line"]) and np.array_equal(n6, g["n6line"])
    INU, IAU, INL, IAL = oracle.pattern(line.shape[0], n6)
    for a, k in ((INU, "INU"), (IAU, "IAU"), (INL, "INL"), (IAL, "IAL")):
        assert np.array_equal(a, g[k])
    m = fixture_model(g)
    A = oracle.forward_assemble(m, line, n6, (INU, IAU, INL, IAL), float(g["freq"]), m.sigma_per_tet())
    for k in ("D", "AU", "AL", "b"):
        assert np.array_equal(getattr(A, k), g[k])
    item, ve, vf, iele = oracle.prepobscoeff(m, n6, g["sites"])
    assert np.array_equal(item, g["item"]) and np.array_equal(ve, g["val_e"]) and np.array_equal(vf, g["val_f"])


def fixture_model(g):
    b = g["bounds"]
    return synth.TidalModel(name="fixture", xyz=g["xyz"], n4=g["n4"], tag=g["tag"], sigma_land=g["sigma_land"],
                            nodes=int(g["nodes"]), F=g["F"], v=g["v"], freqs=np.array([float(g["freq"])]),
                            sites=g["sites"], bounds=dict(zmin=b[0], zmax=b[1], xout=b[2], yout=b[3]),
                            sigma_air=float(g["sigma_air"]), sigma_ocean=float(g["sigma_ocean"]))

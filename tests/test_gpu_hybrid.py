"""Gradient-space (nodal) correction of the COCG preconditioner on the GPU.

The nodal matrix must be the Galerkin product G^T P A P G of the assembled
edge matrix (G the edge-node incidence, P dropping Dirichlet edges), checked
against a scipy product of the exported system within 1e-12 of the sum of
the magnitudes of each entry's terms (the curl-curl part cancels to roundoff).  Solves with AFEM_PRECOND_HYBRID must reach an FP64 true
residual <= 1e-8 (single and batched), give site
fields within 1e-6 relative of the oracle's own SSOR-COCG solve, and need far
fewer iterations than SSOR alone.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from actfemtide_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fw(gpulib):
    from actfemtide_b200.forward import Forward
    f = Forward(0)
    yield f
    f.close()


@pytest.fixture(scope="module")
def grf_model(oracle):
    """A 12x12x9 log-normal model with the oracle's 1e-11 SSOR-COCG site fields."""
    m = synth.tidal_box(12, 12, 9, seed=3, field_seed=7, grf=True, block=False)
    of = oracle.OracleForward(m)
    A = of.assemble(m.freqs[0])
    r = oracle.cocg13_single(A, precond="SSOR", resid=1e-11, maxit=200000)
    ref, _, _ = of.sites(r["x"], m.freqs[0])
    return m, of, ref


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def _split(sysd, om):
    n = len(sysd["D"])
    INU, IAU, INL, IAL = sysd["INU"], sysd["IAU"], sysd["INL"], sysd["IAL"]
    rows = np.concatenate([np.arange(n), np.repeat(np.arange(n), np.diff(INU)), np.repeat(np.arange(n), np.diff(INL))])
    cols = np.concatenate([np.arange(n), IAU - 1, IAL - 1])
    vals = np.concatenate([sysd["D"], sysd["AU"], sysd["AL"]])
    K = sp.csr_matrix((vals.real, (rows, cols)), shape=(n, n))
    M = sp.csr_matrix((vals.imag / om, (rows, cols)), shape=(n, n))
    return K, M


def test_nodal_matrix_is_the_galerkin_product(fw, grf_model):
    m, of, _ = grf_model
    fw.load_model(m)
    fw.assemble()
    f = m.freqs[0]
    sysd = fw.export_system(f)
    K, M = _split(sysd, 2 * np.pi * f)
    line, _ = fw.lines()
    n = len(sysd["D"])
    free = sysd["bc"] == 0
    G = sp.csr_matrix((np.concatenate([np.ones(n), -np.ones(n)]),
                       (np.concatenate([np.arange(n)] * 2), np.concatenate([line[:, 1] - 1, line[:, 0] - 1]))),
                      shape=(n, m.node))
    PG = sp.diags(free.astype(float)) @ G
    KG = (PG.T @ K @ PG).tocsr()
    MG = (PG.T @ M @ PG).tocsr()
    rp, col, kg, mg = fw.hybrid_matrix()
    assert rp[-1] == len(col)
    # pattern: each row is the node and its edge neighbours, ascending
    adj = sp.csr_matrix((np.ones(2 * n), (np.concatenate([line[:, 0], line[:, 1]]) - 1,
                                          np.concatenate([line[:, 1], line[:, 0]]) - 1)), shape=(m.node, m.node))
    adj = (adj + sp.identity(m.node)).tocsr()
    adj.sort_indices()
    assert np.array_equal(rp, adj.indptr) and np.array_equal(col, adj.indices)
    dev_K = sp.csr_matrix((kg, col, rp), shape=(m.node, m.node)).toarray()
    dev_M = sp.csr_matrix((mg, col, rp), shape=(m.node, m.node)).toarray()
    aG = abs(PG)
    for X, ref, dev in ((K, KG.toarray(), dev_K), (M, MG.toarray(), dev_M)):
        # the entries are sums of +-X terms (the curl-curl part cancels to roundoff inside the
        # mesh): compare within 1e-12 of the sum of the terms' magnitudes
        bound = (aG.T @ abs(X) @ aG).toarray()
        assert np.all(np.abs(dev - ref) <= 1e-12 * bound)


@pytest.mark.parametrize("precision", ["fp64", "pc32"])
def test_hybrid_cocg_matches_oracle(fw, grf_model, precision):
    m, of, ref = grf_model
    fw.load_model(m)
    fw.assemble()
    f = m.freqs[0]
    r_h = fw.solve(f, precond="HYBRID", precision=precision, tol=1e-8, maxit=20000)
    assert r_h.ok and r_h.resid_true <= 1e-8, r_h
    out = fw.sites(m.sites)[0]
    assert _rel(out, ref) <= 1e-6
    if precision == "fp64":
        r_s = fw.solve(f, precond="SSOR", tol=1e-8, maxit=50000)
        assert r_s.ok
        assert r_h.iterations * 5 < r_s.iterations, (r_h.iterations, r_s.iterations)


def test_hybrid_batched_matches_single(fw, grf_model):
    m, _, _ = grf_model
    fw.load_model(m, sources=[(m.F, m.v), (m.F, 0.5j * m.v)])
    fw.assemble()
    freqs = 1.0 / (3600.0 * np.array(synth.BATCH_PERIODS_H[:4]))
    srcs = np.array([0, 1, 0, 1])
    rb = fw.solve(freqs, srcs, precond="HYBRID", tol=1e-8, maxit=20000)
    assert rb.ok and rb.resid_true <= 1e-8, rb
    outb = fw.sites(m.sites, nsys=4)
    for k in range(4):
        r1 = fw.solve(freqs[k], [srcs[k]], precond="HYBRID", tol=1e-8, maxit=20000)
        assert r1.ok
        assert _rel(outb[k], fw.sites(m.sites)[0]) <= 1e-6


@pytest.fixture(scope="module")
def box20_ref(oracle):
    """The 20x20x20 model and the oracle's SSOR-COCG (the reference's own solver) at 1e-10."""
    m = synth.small_model()
    of = oracle.OracleForward(m)
    A = of.assemble(m.freqs[0])
    r = oracle.cocg13_single(A, precond="SSOR", resid=1e-10, maxit=100000)
    assert r["error"] == 0
    ref, _, _ = of.sites(r["x"], m.freqs[0])
    return m, A, ref[0]


@pytest.mark.parametrize("precision", ["fp64", "pc32"])
def test_hybrid_box20_sites(fw, oracle, box20_ref, precision):
    """SSOR-COCG needs ~2,550 iterations on the 20x20x20 model; the corrected COCG several-fold fewer,
    and its site fields match the reference solver's to 1e-6 (FP64 preconditioner and FP32 one)."""
    m, A, ref = box20_ref
    fw.load_model(m)
    fw.assemble()
    r = fw.solve(m.freqs[0], precond="HYBRID", precision=precision, tol=1e-8, maxit=20000)
    assert r.ok and r.resid_true <= 1e-8, r
    assert r.iterations < 1000, r.iterations
    assert oracle.true_residual(A, fw.solution(0)) <= 1.01e-8
    assert _rel(fw.sites(m.sites)[0], ref) <= 1e-6


@pytest.mark.parametrize("precision", ["fp64", "pc32"])
def test_hybrid_box20_batch_of_16_sites(fw, oracle, box20_ref, precision):
    """The benchmark's batch shape (8 periods x 2 source patterns) on the 20x20x20 model, with system 0
    at the M2 period of the reference solve: its site fields within 1e-6 of the reference solver's."""
    m, A, ref = box20_ref
    m2 = synth.tidal_box(20, 20, 20, seed=1000, name="box20")
    fw.load_model(m, sources=[(m.F, m.v), (m2.F, m2.v)])
    fw.assemble()
    freqs = 1.0 / (3600.0 * np.array(synth.BATCH_PERIODS_H))
    freqs[0] = m.freqs[0]
    f = np.concatenate([freqs, freqs])
    src = np.repeat([0, 1], 8).astype(np.int32)
    r = fw.solve(f, srcs=src, precond="HYBRID", precision=precision, tol=1e-8, maxit=20000)
    assert r.ok and r.resid_true <= 1e-8, r
    assert oracle.true_residual(A, fw.solution(0)) <= 1.01e-8
    assert _rel(fw.sites(m.sites, nsys=16)[0], ref) <= 1e-6


@pytest.mark.parametrize("precision", ["fp64", "pc32"])
def test_batched_hybrid_matches_direct_solve_32x32x24(fw, precision):
    """The batched gradient-corrected solve (16 systems, 8 periods x 2 velocity patterns) on the 32x32x24 mesh
    (179,800 edges): the site fields of systems 0 and 12 within 1e-6 of a direct solve (SciPy SuperLU, the
    stand-in for the reference's PARDISO) of the oracle's assembly, committed by
    tests/golden/make_superlu_fixture.py."""
    import os
    import sys
    here = os.path.join(os.path.dirname(__file__), "golden")
    sys.path.insert(0, here)
    import make_superlu_fixture as msf
    g = np.load(os.path.join(here, "box32x32x24_superlu.npz"))
    m, m2 = msf.models()
    f, src = msf.batch_freqs(m)
    assert np.array_equal(g["sites"], m.sites)
    fw.load_model(m, sources=[(m.F, m.v), (m2.F, m2.v)])
    fw.assemble()
    r = fw.solve(f, srcs=src, precond="HYBRID", precision=precision, tol=1e-8, maxit=20000)
    assert r.ok and r.resid_true <= 1e-8, r
    out = fw.sites(m.sites, nsys=16)
    for k in (0, 12):
        assert float(g[f"freq_{k}"]) == f[k]
        assert float(g[f"resid_{k}"]) <= 1e-10
        assert _rel(out[k], g[f"sites_{k}"]) <= 1e-6, (k, _rel(out[k], g[f"sites_{k}"]))

"""Packed batches of uneven meshes on the GPU, through the C ABI.

One solve runs every mesh of the batch, each with its own COCG scalars.
Checked against (i) the same meshes loaded one at a time on the device
(union assembly bit-exact, site fields within 1e-9 relative) and (ii) the
oracle's own solve of each mesh (site fields within 1e-6 relative), with an
FP64 true residual <= 1e-8 for every mesh.
"""
import numpy as np
import pytest

from actfemtide_b200 import synth
from actfemtide_b200.capi import AfemError

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fw(gpulib):
    from actfemtide_b200.forward import Forward
    f = Forward(0)
    yield f
    f.close()


@pytest.fixture(scope="module")
def parts():
    # n >= 8 keeps the 5 km sea layer resolved (cells of at most 100/6 km), so every mesh has a source
    return synth.uneven_models(5, seed=2, nmin=8, nmax=11)


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_packed_assembly_equals_separate(fw, parts):
    pk = synth.pack(parts)
    fw.load_packed(pk)
    rp, tp = fw.segment_info()
    assert np.array_equal(tp, pk.tet_ptr)
    fw.assemble()
    f = parts[0].freqs[0]
    su = fw.export_system(f)
    for k, m in enumerate(parts):
        fw.load_model(m)
        fw.assemble()
        s = fw.export_system(f)
        r0, r1 = rp[k], rp[k + 1]
        assert r1 - r0 == fw.nline
        assert np.array_equal(su["D"][r0:r1], s["D"])
        assert np.array_equal(su["b"][r0:r1], s["b"])
        assert np.array_equal(su["bc"][r0:r1], s["bc"])
        u0, u1 = su["INU"][r0], su["INU"][r1]
        assert np.array_equal(su["AU"][u0:u1], s["AU"])
        assert np.array_equal(su["IAU"][u0:u1] - r0, s["IAU"])
        l0, l1 = su["INL"][r0], su["INL"][r1]
        assert np.array_equal(su["AL"][l0:l1], s["AL"])


@pytest.mark.parametrize("precond,precision", [("SSOR", "fp64"), ("HYBRID", "fp64")])
def test_packed_solve_matches_separate_and_oracle(fw, oracle, parts, precond, precision):
    nseg = len(parts)
    freqs = np.array([m.freqs[0] for m in parts])
    sites = parts[0].sites
    # separate device solves, one mesh at a time
    sep = []
    for m in parts:
        fw.load_model(m)
        fw.assemble()
        r = fw.solve(m.freqs[0], precond="SSOR", tol=1e-8, maxit=50000)
        assert r.ok and r.resid_true <= 1e-8
        sep.append(fw.sites(sites)[0])
    pk = synth.pack(parts)
    fw.load_packed(pk)
    fw.assemble()
    res = fw.solve(freqs, np.zeros(nseg, int), precond=precond, precision=precision, tol=1e-8, maxit=50000)
    assert res.ok and res.resid_true <= 1e-8, res
    out = fw.sites(sites, nsys=nseg)
    for k, m in enumerate(parts):
        # every mesh's own true residual, from its rows of the union
        x = fw.solution(k)
        assert x.shape[0] == fw.row_ptr[k + 1] - fw.row_ptr[k]
        assert _rel(out[k], sep[k]) <= 1e-6
        of = oracle.OracleForward(m)
        A = of.assemble(m.freqs[0])
        assert oracle.true_residual(A, x) <= 1e-8
        ro = oracle.cocg13_single(A, precond="SSOR", resid=1e-10, maxit=100000)
        ref, _, _ = of.sites(ro["x"], m.freqs[0])
        assert _rel(out[k], ref) <= 1e-6


def test_packed_each_mesh_converges_on_its_own(fw, parts):
    """A mesh with a zero source finishes at once; the others still converge."""
    pk = synth.pack(parts)
    pk.F[pk.node_ptr[1]:pk.node_ptr[2]] = 0.0  # mesh 1: no source
    fw.load_packed(pk)
    fw.assemble()
    nseg = len(parts)
    res = fw.solve(np.full(nseg, parts[0].freqs[0]), np.zeros(nseg, int), precond="SSOR", tol=1e-8, maxit=50000)
    assert res.ok and res.resid_true <= 1e-8
    assert np.all(fw.solution(1) == 0)
    assert np.abs(fw.solution(0)).max() > 0


def test_packed_errors(fw, parts):
    pk = synth.pack(parts)
    fw.load_packed(pk)
    fw.assemble()
    nseg = len(parts)
    with pytest.raises(AfemError):  # one system per mesh
        fw.solve(parts[0].freqs[0], precond="SSOR")
    with pytest.raises(AfemError):  # no learned preconditioner on packed batches
        fw.solve(np.full(nseg, parts[0].freqs[0]), np.zeros(nseg, int), precond="LEARNED")
    bad = pk.node_ptr.copy()
    bad[1] += 1  # a node range that splits a mesh
    with pytest.raises(AfemError):
        fw.set_segments(bad)
    with pytest.raises(AfemError):
        fw.set_segments(np.arange(40, dtype=np.int32))  # more than 32 meshes / wrong end
    # clearing the declaration returns to a single system
    fw.set_segments(None)
    assert fw.segment_info()[0].shape == (1,)


@pytest.mark.parametrize("precision", ["fp64", "pc32"])
def test_packed_24_uneven_meshes_full_size(fw, oracle, precision):
    """The batched workload's second batch at its stated size: 24 meshes of n x n x round(3n/4) cells,
    n uniform in 8..32, each with its own seeded log-normal subsurface, in one packed solve.  Every
    mesh's solution is checked by the oracle's FP64 true residual of that mesh's own assembly, and its
    site fields against a separate device solve of the mesh alone (1e-6)."""
    parts = synth.uneven_models(24, seed=0)
    ns_ = sorted(m.dims[0] for m in parts)
    assert len(parts) == 24 and ns_[0] >= 8 and ns_[-1] <= 32
    sites = parts[0].sites
    sep = []
    for m in parts:
        fw.load_model(m)
        fw.assemble()
        r = fw.solve(m.freqs[0], precond="HYBRID", tol=1e-8, maxit=20000)
        assert r.ok and r.resid_true <= 1e-8, (m.name, r)
        sep.append(fw.sites(sites)[0])
    pk = synth.pack(parts)
    fw.load_packed(pk)
    fw.assemble()
    freqs = np.array([m.freqs[0] for m in parts])
    res = fw.solve(freqs, np.zeros(24, int), precond="HYBRID", precision=precision, tol=1e-8, maxit=20000)
    assert res.ok and res.resid_true <= 1e-8, res
    out = fw.sites(sites, nsys=24)
    for k, m in enumerate(parts):
        A = oracle.OracleForward(m).assemble(m.freqs[0])
        assert oracle.true_residual(A, fw.solution(k)) <= 1.01e-8, m.name
        assert _rel(out[k], sep[k]) <= 1e-6, m.name

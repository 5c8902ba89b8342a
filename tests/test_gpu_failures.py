"""Failure statuses of the device solve, each made on the host, none by faulting or hanging the GPU.

* a wait bound of one poll makes the sync-free sweeps' bounded waits run out:
  the kernel records the timeout, every waiting row gives up and returns, and
  the solve reports AFEM_ETIMEOUT; the context then solves normally again;
* a NaN conductivity gives NaN matrix entries: AFEM_ENONFINITE at the start of
  the solve (the reference would iterate on NaN until its cap);
* a right-hand side with r^T r = 0 (b = e_i + i e_j, unconjugated product
  1 + i^2) makes rho vanish in the first COCG iteration: AFEM_EBREAKDOWN.
"""
import numpy as np
import pytest

from actfemtide_b200 import capi, synth
from actfemtide_b200.capi import AfemError

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fw(gpulib):
    from actfemtide_b200.forward import Forward
    f = Forward(0)
    yield f
    f.close()


@pytest.fixture(scope="module")
def box20():
    return synth.small_model()


def test_wait_bound_expires_with_status_and_context_survives(fw, box20):
    m = box20
    fw.load_model(m)
    fw.assemble()
    ref = fw.solve(m.freqs[0], precond="SSOR", tol=1e-8)
    assert ref.ok
    out_ref = fw.sites(m.sites)
    fw.set_wait_limit(1)
    try:
        with pytest.raises(AfemError) as e:
            fw.solve(m.freqs[0], precond="SSOR", tol=1e-8, maxit=64, use_graph=False)
        assert e.value.code == capi.STATUS_CODE["AFEM_ETIMEOUT"], e.value
    finally:
        fw.set_wait_limit(0)
    again = fw.solve(m.freqs[0], precond="SSOR", tol=1e-8)
    assert again.ok and again.resid_true <= 1e-8
    assert again.iterations == ref.iterations
    assert np.array_equal(fw.sites(m.sites), out_ref)


@pytest.mark.parametrize("precond", ["SSOR", "HYBRID"])
def test_nan_conductivity_is_reported_non_finite(fw, box20, precond):
    m = box20
    fw.load_model(m)
    sig = m.sigma_per_tet().copy()
    sig[m.nphys1 + 17] = np.nan  # one land tetrahedron
    fw.set_sigma(sig)
    fw.assemble()
    with pytest.raises(AfemError) as e:
        fw.solve(m.freqs[0], precond=precond, tol=1e-8, maxit=200)
    assert e.value.code == capi.STATUS_CODE["AFEM_ENONFINITE"], e.value
    fw.set_sigma(m.sigma_per_tet())
    fw.assemble()
    r = fw.solve(m.freqs[0], precond=precond, tol=1e-8)
    assert r.ok and r.resid_true <= 1e-8


def test_vanishing_rho_is_reported_as_breakdown(fw, box20):
    m = box20
    fw.load_model(m)
    fw.assemble()
    b = np.zeros(fw.nline, np.complex128)
    b[100] = 1.0
    b[200] = 1.0j  # b^T b = 1 + i^2 = 0 exactly, ||b|| = sqrt(2)
    with pytest.raises(AfemError) as e:
        fw.solve_rhs(m.freqs[0], b[:, None], precond="NONE", tol=1e-8, maxit=100)
    assert e.value.code == capi.STATUS_CODE["AFEM_EBREAKDOWN"], e.value
    r = fw.solve(m.freqs[0], precond="SSOR", tol=1e-8)
    assert r.ok

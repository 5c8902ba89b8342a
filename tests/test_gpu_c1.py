"""Parity on the 96x96x64 model, the configuration the headline solve time is measured on.

3,538,944 tetrahedra, 4,193,536 edges, nnz 68,152,576, log-normal subsurface,
400 sites.  Against the CPU oracle (the statement-by-statement restatement of
the reference's routines):

* the device edge numbering (MKLINE_V2/MKN6) and CSR pattern (C_set_dof2)
  bit-exact, the Dirichlet flags bit-exact, and the assembled system (GENMAT +
  COPY_UL_ICCG12 + SET_BC_ICCG) within 1e-12 of each row's largest entry, the
  curl-curl part bit-exact, at two tidal frequencies;
* the batched solve the benchmark times (8 tidal periods x 2 source patterns =
  16 systems, gradient-corrected COCG): each sampled system's solution checked
  by the oracle's own FP64 true residual ||b - A x|| / ||b|| of the oracle's
  assembly (an independent check of the answer the benchmark times), for the
  FP64 preconditioner and the FP32 one, and the site fields of the two within
  1e-6 of each other.
"""
import dataclasses

import numpy as np
import pytest

from actfemtide_b200 import synth
from parity_util import assert_system_close, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fw(gpulib):
    from actfemtide_b200.forward import Forward
    f = Forward(0)
    yield f
    f.close()


@pytest.fixture(scope="module")
def c1(oracle):
    m = synth.large_model(seed=0)
    of = oracle.OracleForward(m)
    return m, of


@pytest.fixture(scope="module")
def batch(c1):
    """The benchmark's batch: 8 periods for each of two seeded velocity patterns."""
    m, _ = c1
    m2 = synth.large_model(seed=1000)
    freqs = 1.0 / (3600.0 * np.array(synth.BATCH_PERIODS_H))
    f = np.concatenate([freqs, freqs])
    src = np.repeat([0, 1], 8).astype(np.int32)
    return f, src, [(m.F, m.v), (m2.F, m2.v)]


def test_c1_numbering_pattern_assembly(fw, oracle, c1):
    m, of = c1
    fw.load_model(m)  # numbering built on the device
    line, n6 = fw.lines()
    assert np.array_equal(line, of.line)
    assert np.array_equal(n6, of.n6line)
    INU, IAU, INL, IAL = fw.export_pattern()
    for a, b in zip((INU, IAU, INL, IAL), of.pat):
        assert np.array_equal(a, b)
    fw.assemble()
    for period_h in (12.4206, 25.8193):
        f = 1.0 / (3600.0 * period_h)
        A = of.assemble(f)
        sg = fw.export_system(f)
        assert np.array_equal(sg["bc"], A.bc)
        assert_system_close(sg, A, rtol=1e-12)
        del A, sg


def test_c1_batched_hybrid_oracle_true_residual(fw, oracle, c1, batch):
    m, of = c1
    f, src, sources = batch
    fw.load_model(m, with_lines=(of.line, of.n6line), sources=sources)
    fw.assemble()
    sites = {}
    for precision in ("fp64", "pc32"):
        res = fw.solve(f, srcs=src, precond="HYBRID", precision=precision, tol=1e-8, maxit=20000)
        assert res.ok and res.resid_true <= 1e-8, (precision, res)
        sites[precision] = fw.sites(m.sites, nsys=len(f))
        # systems 0 (12.42 h, pattern 1) and 13 (24.07 h, pattern 2): the oracle's own assembly
        # of A(omega_k) and b_k, and its FP64 residual of the device solution
        for k in (0, 13):
            F, v = sources[src[k]]
            mk = dataclasses.replace(m, F=F, v=v)
            A = oracle.forward_assemble(mk, of.line, of.n6line, of.pat, f[k], of.sigma_tet)
            x = fw.solution(k)
            tr = oracle.true_residual(A, x)
            assert tr <= 1.01e-8, (precision, k, tr)
            del A, x
    # both reach a 1e-8 true residual; their site fields agree to 1e-6
    err = max(rel_err(sites["pc32"][k], sites["fp64"][k]) for k in range(len(f)))
    assert err <= 1e-6, err

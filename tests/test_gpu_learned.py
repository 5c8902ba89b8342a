"""Learned preconditioner on the GPU: network parity with the CPU reference, gradients, training, flexible COCG.

Tolerances: the device network runs BF16 weights/activations with FP32
accumulation; its forward output is compared with the CPU reference that
emulates the same BF16 roundings (relative 2e-2 of the output norm), its
gradient by cosine similarity (>= 0.99) and norm ratio (within 5 %).  The
CPU reference's own gradient is checked by central finite differences.
"""
import numpy as np
import pytest

from actfemtide_b200 import learned, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fw(gpulib):
    from actfemtide_b200.forward import Forward
    f = Forward(0)
    yield f
    f.close()


def ref_graph(fw, m, freq):
    from oracle import mpnn_ref as R
    n = fw.nline
    s = fw.export_system(freq)
    INU, IAU, INL, IAL = s["INU"], s["IAU"], s["INL"], s["IAL"]
    om = 2 * np.pi * freq
    rows, cols, kv, mv = [], [], [], []
    for i in range(n):
        for k in range(INL[i], INL[i + 1]):
            rows.append(i); cols.append(IAL[k] - 1); kv.append(s["AL"][k].real); mv.append(s["AL"][k].imag / om)
        rows.append(i); cols.append(i); kv.append(s["D"][i].real); mv.append(s["D"][i].imag / om)
        for k in range(INU[i], INU[i + 1]):
            rows.append(i); cols.append(IAU[k] - 1); kv.append(s["AU"][k].real); mv.append(s["AU"][k].imag / om)
    rowptr = np.zeros(n + 1, np.int64)
    np.add.at(rowptr, np.array(rows) + 1, 1)
    rowptr = np.cumsum(rowptr)
    col = np.array(cols); K = np.array(kv); M = np.array(mv)
    diagpos = np.array([rowptr[i] + np.nonzero(col[rowptr[i]:rowptr[i + 1]] == i)[0][0] for i in range(n)])
    return R.Graph(rowptr, col, K, M, diagpos, om, s["bc"])


def test_network_forward_and_gradient_match_cpu(fw):
    from oracle import mpnn_ref as R
    m = synth.tidal_box(4, 4, 6, seed=3, site_grid=(-6.0, 0.0, 6.0), half_km=12.0)
    fw.load_model(m)
    fw.assemble()
    f = m.freqs[0]
    g = ref_graph(fw, m, f)
    rng = np.random.default_rng(0)
    p = learned.init_params(1)
    p[-2 * learned.H:] = rng.standard_normal(2 * learned.H) * 0.1  # non-zero W_out to exercise every layer
    P = learned.unflatten(p)
    fw.mpnn_set_params(p)
    r = rng.standard_normal(fw.nline) + 1j * rng.standard_normal(fw.nline)
    z = fw.mpnn_forward(f, r)
    zr, _ = R.forward(P, g, r, bf16=True)
    assert np.linalg.norm(z - zr) <= 2e-2 * np.linalg.norm(zr)
    loss, grad = fw.mpnn_loss_grad(f, r[None, :])
    lr_, G = R.grad(P, g, r, bf16=True)
    assert abs(loss - lr_) <= 2e-2 * lr_
    gref = learned.flatten(G).astype(np.float64)
    cos = float(grad @ gref / (np.linalg.norm(grad) * np.linalg.norm(gref)))
    assert cos >= 0.99, cos
    assert abs(np.linalg.norm(grad) / np.linalg.norm(gref) - 1.0) <= 0.05


def test_training_lowers_the_loss(fw):
    m = learned.training_model(0, 8, 8, 6)
    fw.load_model(m)
    fw.assemble()
    f = m.freqs[0]
    fw.mpnn_set_params(learned.init_params(0))
    R = learned.collect_residuals(fw, f)
    hist = fw.mpnn_train(f, R, steps=60, lr=2e-3)
    assert hist[-1] < 0.8 * hist[0], hist[[0, -1]]


def test_flexible_cocg_learned_reaches_tolerance(fw):
    """Flexible COCG with the trained network reaches an FP64 true residual of 1e-8 and beats no preconditioner."""
    m = learned.training_model(7, 8, 8, 6)
    fw.load_model(m)
    fw.assemble()
    f = m.freqs[0]
    fw.mpnn_set_params(learned.init_params(0))
    for k in range(6):
        mk = learned.training_model(k, 8, 8, 6)
        fw.set_cond(mk.sigma_air, mk.sigma_ocean, 1, sigma_file=mk.sigma_land)
        fw.assemble()
        fw.mpnn_train(f, learned.collect_residuals(fw, f), steps=20, lr=2e-3)
    fw.set_cond(m.sigma_air, m.sigma_ocean, 1, sigma_file=m.sigma_land)
    fw.assemble()
    res_l = fw.solve(f, precond="LEARNED", tol=1e-8, maxit=20000)
    assert res_l.ok and res_l.resid_true <= 1e-8
    res_n = fw.solve(f, precond="NONE", tol=1e-8, maxit=20000)
    assert res_l.iterations < res_n.iterations


def test_hybrid_base_adds_the_same_correction(fw):
    """With the hybrid base the network's output is H(r) plus the correction it gives over the Jacobi base."""
    m = synth.tidal_box(4, 4, 6, seed=3, site_grid=(-6.0, 0.0, 6.0), half_km=12.0)
    fw.load_model(m)
    fw.assemble()
    f = m.freqs[0]
    rng = np.random.default_rng(4)
    p = learned.init_params(2)
    p[-2 * learned.H:] = rng.standard_normal(2 * learned.H) * 0.1
    p0 = p.copy()
    p0[-2 * learned.H:] = 0.0  # no correction: the base alone
    r = rng.standard_normal(fw.nline) + 1j * rng.standard_normal(fw.nline)
    out = {}
    for base in (False, True):
        fw.mpnn_set_base(base)
        fw.mpnn_set_params(p)
        z = fw.mpnn_forward(f, r)
        fw.mpnn_set_params(p0)
        z0 = fw.mpnn_forward(f, r)
        out[base] = (z, z0)
    fw.mpnn_set_base(False)
    h = fw.precond_apply(f, r)
    assert np.array_equal(out[True][1], h)
    corr_j = out[False][0] - out[False][1]
    corr_h = out[True][0] - out[True][1]
    # the Jacobi base adds r/|A_ii| and the correction in one FP32 sum, the hybrid base adds the
    # correction to H(r) in FP64, and H(r) reaches ~1e11 on air edges: each difference carries
    # the rounding of its own sums, FP32 of the Jacobi terms and FP64 of the hybrid ones
    terms_j = np.abs(out[False][0]) + np.abs(out[False][1]) + np.abs(corr_j)
    terms_h = np.abs(out[True][0]) + np.abs(out[True][1])
    assert np.all(np.abs(corr_h - corr_j) <= 4 * 2.0 ** -24 * terms_j + 4 * 2.0 ** -53 * terms_h + 1e-12)
    assert np.abs(corr_j).max() > 0


def test_learned_over_hybrid_falls_back_and_reaches_tolerance(fw):
    """Flexible COCG with z = H(r) + N(r), trained briefly, reaches 1e-8.

    This claims no gain: the trained correction costs iterations on these systems
    (measured: about twice H's on held-out 32x32x24 models, recorded in the
    checkpoint's JSON), and how many varies with the training run (its gradient sums
    use atomics: 127 to 300 iterations against H's 55 here).  The bound is what the
    stall detector guarantees: after at most a few windows of 128 iterations without
    progress the solve falls back to H alone, so the cost stays within 3 H + 4 windows."""
    m = learned.training_model(7, 8, 8, 6)
    fw.load_model(m)
    fw.assemble()
    f = m.freqs[0]
    fw.mpnn_set_params(learned.init_params(0))
    fw.mpnn_set_base(True)
    for k in range(4):
        mk = learned.training_model(k, 8, 8, 6)
        fw.set_cond(mk.sigma_air, mk.sigma_ocean, 1, sigma_file=mk.sigma_land)
        fw.assemble()
        hist = fw.mpnn_train(f, learned.collect_residuals(fw, f, precond="HYBRID"), steps=20, lr=1e-3)
        assert np.all(np.isfinite(hist))
    fw.set_cond(m.sigma_air, m.sigma_ocean, 1, sigma_file=m.sigma_land)
    fw.assemble()
    r_l = fw.solve(f, precond="LEARNED", tol=1e-8, maxit=5000)
    r_h = fw.solve(f, precond="HYBRID", tol=1e-8, maxit=5000)
    fw.mpnn_set_base(False)
    assert r_l.ok and r_l.resid_true <= 1e-8, r_l
    assert r_h.ok
    assert r_l.iterations <= 3 * r_h.iterations + 4 * 128, (r_l.iterations, r_h.iterations)

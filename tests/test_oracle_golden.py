"""The CPU oracle against golden vectors produced by the reference package's
own code (tests/golden/make_golden.py): per-event |A|^2, NLL and its
GradientTape gradient on identical events and parameters."""
import numpy as np
import pytest

from common import golden_data, load_golden, load_model
from oracle.pwa_oracle import OracleModel, OracleNLL

CASES = ["d2kpipi", "d2kpipi_float", "lc2pkpi", "toy_vvp", "b2dstkpi", "d2kpipi_shapes",
         "dp2kpipi_ident", "ident_fermions", "epem_cp", "lc2pkpi_cc", "b2dstkpi_cc",
         "lc2pkpi_pol", "epem_pol", "ident3_fermions", "lc2pkpi_pol_lab",
         "lc2pkpi_cp"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference(name):
    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    assert plan.fields == meta["fields"]
    m = OracleModel(dc.decay_group, plan)
    vals = meta["variables"]
    fd = m.pdf(g["fields_data"], vals)
    fm = m.pdf(g["fields_mc"], vals)
    np.testing.assert_allclose(fd, g["f_data"], rtol=1e-12)
    np.testing.assert_allclose(fm, g["f_mc"], rtol=1e-12)
    x, w = golden_data(g, meta)
    np.testing.assert_allclose(w, g["weight_data"], rtol=1e-15)
    o = OracleNLL(m, x, w, g["fields_mc"], np.ones(g["fields_mc"].shape[1]),
                  meta["trainable"], {}, vals)
    p = [vals[k] for k in meta["trainable"]]
    assert abs(o.nll(p) - g["nll"]) <= 1e-12 * abs(g["nll"])
    gr = o.grad(p)
    # couplings exact; masses/widths by 4-point differences
    np.testing.assert_allclose(gr, g["grad"], rtol=1e-8, atol=1e-8 * np.abs(g["grad"]).max())


def test_reference_gradient_is_a_derivative():
    """The golden gradient (reference autodiff through the TF stand-in) agrees
    with central differences of the oracle NLL."""
    g, meta = load_golden("d2kpipi_float")
    dc, vm, plan = load_model(meta["config"])
    m = OracleModel(dc.decay_group, plan)
    vals = meta["variables"]
    x, w = golden_data(g, meta)
    o = OracleNLL(m, x, w, g["fields_mc"], np.ones(g["fields_mc"].shape[1]),
                  meta["trainable"], {}, vals)
    p = np.array([vals[k] for k in meta["trainable"]])
    for k in range(len(p)):
        h = 1e-6 * max(abs(p[k]), 1.0)
        q1, q2 = p.copy(), p.copy()
        q1[k] += h
        q2[k] -= h
        fd = (o.nll(q1) - o.nll(q2)) / (2 * h)
        assert abs(fd - g["grad"][k]) <= 1e-5 * max(1.0, abs(g["grad"][k]))


def test_known_answers():
    """Reference unit-test known answers (tf_pwa/tests/test_amp.py:294-305,
    94-113; test_model_new.py-style sums)."""
    from oracle.pwa_oracle import bw, clip_log, rel_p, rel_p2, small_d

    # BW at m=[1,2], m0=g0=2 times -1 -> [-0.12-0.16j, -0.25j]
    r = -bw(np.array([1.0, 2.0]), 2.0, 2.0)
    np.testing.assert_allclose(r, [-0.12 - 0.16j, -0.25j], atol=1e-15)
    m0 = np.linspace(1.0, 3.0, 11)
    np.testing.assert_allclose(rel_p2(m0, 0.4, 0.3), rel_p(m0, 0.4, 0.3) ** 2, rtol=1e-12)
    b = np.linspace(0, np.pi, 7)
    np.testing.assert_allclose(small_d(b, 2)[:, 1, 1], np.cos(b), atol=1e-15)  # d^1_00
    np.testing.assert_allclose(small_d(b, 1)[:, 0, 0], np.cos(b / 2), atol=1e-15)
    # unitarity of d^{3/2}
    d = small_d(b, 3)
    for k in range(len(b)):
        np.testing.assert_allclose(d[k] @ d[k].T, np.eye(4), atol=1e-14)
    assert clip_log(np.array([1.0]))[0] == 0.0
    x = np.array([0.5e-6])
    assert np.isfinite(clip_log(x)).all()


@pytest.mark.parametrize("name", ["d2kpipi", "lc2pkpi", "dp2kpipi_ident", "b2dstkpi"])
def test_oracle_one_pass_gradient(name):
    """The oracle's one-pass form (partial-wave columns, then every coupling
    derivative from the same pass -- the CPU baseline's formulation) equals
    the reference's NLL and GradientTape gradient."""
    from common import golden_data, load_golden, load_model
    from oracle.pwa_oracle import OracleModel, column_sums, nll_grad_from_sums

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    vals = meta["variables"]
    x, w = golden_data(g, meta)
    xm = g["fields_mc"]
    wm = np.ones(xm.shape[1]) / xm.shape[1]
    m = OracleModel(dc.decay_group, plan)
    names = m.columns(x[:, :2], vals, {})[1]
    sd, gd = column_sums(m, x, w, vals, {}, True)
    sm, gm = column_sums(m, xm, wm, vals, {}, False)
    tr = [t for t in meta["trainable"] if "_g_ls_" in t or "_total_" in t]
    nll, grad = nll_grad_from_sums(names, vals, {}, tr, sd, gd, sm, gm, w.sum())
    idx = [meta["trainable"].index(t) for t in tr]
    assert abs(nll - float(g["nll"])) <= 1e-12 * abs(float(g["nll"]))
    np.testing.assert_allclose(grad, g["grad"][idx], rtol=0,
                               atol=1e-10 * np.abs(g["grad"]).max())


@pytest.mark.parametrize("name", ["d2kpipi", "lc2pkpi", "dp2kpipi_ident", "ident_fermions",
                                  "toy_vvp", "b2dstkpi"])
def test_oracle_exact_coupling_hessian(name):
    """The closed-form second derivatives in the couplings (two weighted
    Gram-type sums over the data, the MC Gram matrix and the derivatives
    of the column couplings) equal the reference's nested-GradientTape
    Hessian (FCN.nll_grad_hessian) on the golden events."""
    from common import golden_data, load_golden, load_model
    from oracle.pwa_oracle import (OracleModel, gram_matrix, hessian_sums,
                                   nll_grad_hessian_from_sums)

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    vals = meta["variables"]
    x, w = golden_data(g, meta)
    xm = g["fields_mc"]
    wm = np.ones(xm.shape[1]) / xm.shape[1]
    m = OracleModel(dc.decay_group, plan)
    S0, S1, H1, H2, names = hessian_sums(m, x, w, vals, {})
    M, _ = gram_matrix(m, xm, wm, vals, {})
    nll, grad, H = nll_grad_hessian_from_sums(names, vals, {}, meta["trainable"],
                                              (S0, S1, H1, H2), M, w.sum())
    assert abs(nll - float(g["hess_nll"])) <= 1e-12 * abs(float(g["hess_nll"]))
    np.testing.assert_allclose(grad, g["hess_grad"], rtol=0,
                               atol=1e-12 * np.abs(g["hess_grad"]).max())
    np.testing.assert_allclose(H, g["hess"], rtol=0, atol=1e-12 * np.abs(g["hess"]).max())

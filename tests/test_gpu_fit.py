"""Hessian, parameter errors and fits through the reference-facing API.

* FCN.nll_grad_hessian (central differences of the adjoint gradient) against
  the reference's exact Hessian (nested GradientTape) on golden events.
* A BFGS fit of a toy in plain FP64 and in the mixed form lands on the same
  minimum: parameters within 0.01 sigma and |dNLL| < 1e-3.
"""
import numpy as np
import pytest

from common import CONFIGS, golden_data, load_golden

pytestmark = pytest.mark.gpu


def _fcn(name, precision="plain"):
    import os

    from tf_pwa_b200.api import FCN, ConfigLoader, EventData

    g, meta = load_golden(name)
    cl = ConfigLoader(os.path.join(CONFIGS, meta["config"]))
    cl.vm.set_all(meta["variables"])
    x, w = golden_data(g, meta)
    alpha = w.sum() / (w * w).sum()
    fcn = FCN(cl, EventData(x, w / alpha), EventData(g["fields_mc"]), precision=precision)
    return cl, fcn, g, meta


@pytest.mark.parametrize("name", ["d2kpipi", "d2kpipi_float", "d2kpipi_shapes"])
def test_hessian_matches_reference(name):
    cl, fcn, g, meta = _fcn(name)
    nll, grad, H = fcn.nll_grad_hessian()
    assert abs(nll - g["hess_nll"]) <= 1e-9 * abs(g["hess_nll"])
    np.testing.assert_allclose(grad, g["hess_grad"], rtol=1e-7,
                               atol=1e-7 * np.abs(g["hess_grad"]).max())
    Href = g["hess"]
    np.testing.assert_allclose(H, Href, rtol=2e-5, atol=2e-5 * np.abs(Href).max())
    fcn.eng.close()


def test_fit_plain_vs_mixed_same_minimum():
    """The mixed form moves the fitted parameters by less than 0.01 sigma:
    at the plain-FP64 minimum x*, the shift of the minimum caused by the
    mixed form's gradient error is dx = -H^-1 (g_mixed(x*) - g_plain(x*)).
    Both fits also reach the same minimum NLL within 1e-3."""
    from tf_pwa_b200.api import FCN
    from tf_pwa_b200.workload import make_dataset

    cl, data, bg, mc = make_dataset("lc2pkpi.yml", 20000, 60000, n_bg=2000, seed=7)
    truth = list(cl.vm.get_all_val())
    fp = FCN(cl, data, mc, bg=bg, precision="plain")
    fr_p = cl.fit(fcn=fp, gtol=1e-6)
    xstar = np.array(cl.vm.get_all_val())
    nll_p, g_p, H = fp.nll_grad_hessian(xstar)
    # directions the data do not constrain (Hessian eigenvalues below 1e-8 of
    # the largest, e.g. phase degeneracies of this model) have no finite
    # sigma; the criterion applies to the constrained subspace
    cov = np.linalg.pinv(H, rcond=1e-8, hermitian=True)
    sig = np.sqrt(np.abs(np.diag(cov)))
    fm = FCN(cl, data, mc, bg=bg, precision="mixed")
    assert fm.use_gram
    nll_m, g_m = fm.nll_grad(xstar)
    assert abs(nll_m - nll_p) < 1e-3
    dx = -cov @ (g_m - g_p)
    assert np.all(np.abs(dx) < 0.01 * sig), np.max(np.abs(dx) / sig)
    cl.vm.set_all(truth)
    fr_m = cl.fit(fcn=fm, gtol=1e-6)
    assert abs(fr_p.min_nll - fr_m.min_nll) < 1e-3
    fp.eng.close()
    fm.eng.close()


def test_autograd_function_matches_finite_differences():
    """FCN.torch_nll: a torch.autograd.Function whose backward is the
    adjoint gradient; checked against central finite differences with
    h = 1e-6 of the same FP64 NLL (masses and widths floating)."""
    import torch

    cl, fcn, g, meta = _fcn("d2kpipi_float")
    x0 = np.array(cl.vm.get_all_val())
    x = torch.tensor(x0, dtype=torch.float64, requires_grad=True)
    nll = fcn.torch_nll(x)
    nll.backward()
    assert float(nll) == pytest.approx(float(g["nll"]), rel=1e-9)
    fd = np.zeros_like(x0)
    for i in range(len(x0)):
        h = 1e-6 * max(abs(x0[i]), 1.0)
        xp, xm = x0.copy(), x0.copy()
        xp[i] += h
        xm[i] -= h
        fd[i] = (fcn(xp) - fcn(xm)) / (2 * h)
    fcn._set(x0)
    np.testing.assert_allclose(x.grad.numpy(), fd, rtol=1e-5, atol=1e-5 * np.abs(fd).max())
    np.testing.assert_allclose(x.grad.numpy(), g["grad"], rtol=1e-7,
                               atol=1e-7 * np.abs(g["grad"]).max())
    fcn.eng.close()


def test_native_hessian_equals_python_stencil():
    """pwa_hessian_cached (the 4P stencil points in one multi-point pass with
    FP32 amplitudes) agrees with the same 4-point stencil of FCN gradients
    driven from Python (FP64 amplitudes) to 1e-5 of the largest element,
    and with the plain-FP64 Hessian of the reference-parity path to 1e-4
    (cached form: step 1e-2, see FCN.nll_grad_hessian)."""
    cl, fm, g, meta = _fcn("lc2pkpi", "mixed")
    assert fm.use_gram
    x0 = np.array(cl.vm.get_all_val())
    nll_c, g_c, H_c = fm.nll_grad_hessian(x0, step=1e-2)
    P = len(x0)
    H = np.zeros((P, P))
    for i in range(P):
        h = 1e-2 * max(abs(x0[i]), 1e-2)
        gs = []
        for s in (-2, -1, 1, 2):
            xs = x0.copy()
            xs[i] += s * h
            gs.append(fm.get_nll_grad(xs)[1])
        H[i] = (gs[0] - 8 * gs[1] + 8 * gs[2] - gs[3]) / (12 * h)
    fm._set(x0)
    H = 0.5 * (H + H.T)
    np.testing.assert_allclose(H_c, H, rtol=0, atol=1e-5 * np.abs(H).max())
    assert np.array_equal(H_c, H_c.T)
    _, fp, _, _ = _fcn("lc2pkpi", "plain")
    _, _, H_p = fp.nll_grad_hessian()
    np.testing.assert_allclose(H_c, H_p, rtol=0, atol=1e-4 * np.abs(H_p).max())
    fm.eng.close()
    fp.eng.close()


def test_bounded_fit_stays_inside_bounds(tmp_path):
    """A fit with a floating mass bounded to a window that excludes the
    generated value ends on the window's edge (the transform keeps it
    inside), with the gradient chain rule through dy/dx."""
    import os

    import yaml

    from tf_pwa_b200.api import FCN, ConfigLoader
    from tf_pwa_b200.workload import make_dataset

    cl0, data, _, mc = make_dataset("d2kpipi_float.yml", 20000, 40000, seed=9)
    dic = yaml.safe_load(open(os.path.join(CONFIGS, "d2kpipi_float.yml")))
    m_true = float(cl0.vm.get("R1_mass"))
    dic["particle"]["R1"].update({"mass_min": m_true + 0.01, "mass_max": m_true + 0.05})
    f = tmp_path / "c.yml"
    f.write_text(yaml.safe_dump(dic))
    cl = ConfigLoader(str(f))
    cl.vm.set_all(cl0.vm.get_all_dic())
    cl.vm.set_all({"R1_mass": m_true + 0.03})
    fcn = FCN(cl, data, mc, precision="plain")
    r = cl.fit(fcn=fcn, gtol=1e-4, maxiter=400)
    m_fit = float(cl.vm.get("R1_mass"))
    assert m_true + 0.01 - 1e-12 <= m_fit <= m_true + 0.05 + 1e-12
    assert abs(m_fit - (m_true + 0.01)) < 2e-3  # pushed to the lower edge
    assert np.isfinite(r.min_nll)
    fcn.eng.close()


@pytest.mark.parametrize("name", ["lc2pkpi", "b2dstkpi"])
def test_multi_point_pass_matches_single_points(name):
    """pwa_pieces_points (every point on one pass over the column cache, FP32
    amplitudes) against one FP64-amplitude evaluation per point: NLL within
    1e-3, gradient within 1e-5 of its largest entry, for more points than
    one launch holds (the four-body model's limit is about 25)."""
    from tf_pwa_b200.engine import combine_pieces

    cl, fm, g, meta = _fcn(name, "mixed")
    assert fm.use_gram
    base = np.array([fm.vm.variables[k] for k in fm._var_names])
    rng = np.random.default_rng(4)
    idx = [fm._var_names.index(k) for k in fm.vm.trainable_vars]
    rows = np.repeat(base[None], 40, 0)
    rows[:, idx] += rng.normal(0, 0.02, (40, len(idx)))
    pts = fm.eng.pieces_points(rows)
    P = len(idx)
    for m in range(len(rows)):
        n1, g1 = combine_pieces(pts[m], P)
        n0, g0 = fm.eng.nll_grad_cached(rows[m])
        assert abs(n1 - n0) < 1e-3, (m, n1, n0)
        assert np.max(np.abs(g1 - g0)) <= 1e-5 * np.max(np.abs(g0)), m
    fm.eng.close()


EXACT_CASES = ["d2kpipi", "lc2pkpi", "dp2kpipi_ident", "ident_fermions", "b2dstkpi"]


@pytest.mark.parametrize("name", EXACT_CASES)
def test_exact_hessian_sums_match_oracle(name):
    """The Hessian-sums kernel (pwa_hess_sums_cached) against the oracle's
    FP64 sums from the FP64 columns: S0 to 1e-7 (the cached columns are FP32,
    as in the mixed form's NLL), the gradient sum and both 2K x 2K sums to
    1e-5 of their largest entry (FP32 products, FP64 across tiles)."""
    from oracle.pwa_oracle import OracleModel, hessian_sums
    from common import load_model

    cl, fm, g, meta = _fcn(name, "mixed")
    assert fm.use_gram
    v = fm.vm.variables
    hs = fm.eng.hess_sums_cached([v[k] for k in fm._var_names])
    dc, vm, plan = load_model(meta["config"])
    x, w = golden_data(g, meta)
    S0, S1, H1, H2, names = hessian_sums(OracleModel(dc.decay_group, plan), x, fm.weight,
                                         meta["variables"], {})
    K = len(S1)
    W = 2 * K
    assert abs(hs[0] - S0) <= 1e-7 * abs(S0)
    s1 = hs[1:1 + W].reshape(K, 2)
    ref1 = np.stack([S1.real, S1.imag], 1)
    np.testing.assert_allclose(s1, ref1, rtol=0, atol=1e-5 * np.abs(ref1).max())
    iu = np.triu_indices(W)
    G1 = np.zeros((W, W))
    G1[iu] = hs[1 + W:1 + W + len(iu[0])]
    G1 = G1 + np.triu(G1, 1).T
    G2 = np.zeros((W, W))
    G2[iu] = hs[1 + W + len(iu[0]):]
    G2 = G2 + np.triu(G2, 1).T
    H1g = (G1[:K, :K] + G1[K:, K:]) + 1j * (G1[:K, K:] - G1[K:, :K])
    np.testing.assert_allclose(H1g, H1, rtol=0, atol=1e-5 * np.abs(H1).max())
    np.testing.assert_allclose(G2, H2, rtol=0, atol=1e-5 * np.abs(H2).max())
    fm.eng.close()


@pytest.mark.parametrize("name", EXACT_CASES)
def test_exact_hessian_matches_reference(name):
    """FCN.nll_grad_hessian in the cached form (exact Hessian in the
    couplings, one pass) against the reference's nested-tape Hessian on the
    golden events: NLL 1e-7 relative, gradient and Hessian 1e-5 of their
    largest entry (FP32 columns)."""
    cl, fm, g, meta = _fcn(name, "mixed")
    assert fm.use_gram
    nll, grad, H = fm.nll_grad_hessian()
    assert abs(nll - g["hess_nll"]) <= 1e-7 * abs(g["hess_nll"])
    np.testing.assert_allclose(grad, g["hess_grad"], rtol=0,
                               atol=1e-5 * np.abs(g["hess_grad"]).max())
    np.testing.assert_allclose(H, g["hess"], rtol=0, atol=1e-5 * np.abs(g["hess"]).max())
    assert np.array_equal(H, H.T)
    fm.eng.close()


def test_exact_hessian_large_matches_plain_stencil():
    """At 2.2e5 data rows (with background) and 2e5 MC events the exact
    cached-form Hessian agrees with the plain-FP64 4-point-stencil Hessian
    to 1e-4 of its largest element, and its NLL and gradient with the
    cached form's own evaluation."""
    from tf_pwa_b200.api import FCN
    from tf_pwa_b200.workload import make_dataset

    cl, data, bg, mc = make_dataset("lc2pkpi.yml", 200000, 200000, n_bg=20000, seed=9)
    fm = FCN(cl, data, mc, bg=bg, precision="mixed")
    fp = FCN(cl, data, mc, bg=bg, precision="plain")
    x0 = np.array(cl.vm.get_all_val())
    nll, grad, H = fm.nll_grad_hessian(x0)
    nll_m, g_m = fm.nll_grad(x0)
    assert abs(nll - nll_m) <= 1e-9 * abs(nll_m)
    np.testing.assert_allclose(grad, g_m, rtol=0, atol=1e-6 * np.abs(g_m).max())
    _, _, H_p = fp.nll_grad_hessian(x0)
    np.testing.assert_allclose(H, H_p, rtol=0, atol=1e-4 * np.abs(H_p).max())
    fm.eng.close()
    fp.eng.close()


def test_wide_model_hessian_falls_back_to_stencil():
    """toy_vvp (spin-1 finals: 18 columns x 18 helicity outputs) has per-tile
    rows larger than a block's shared memory: the exact-sums kernel refuses
    with PWA_ERR_STATE, the cached form's evaluation runs the non-ring
    variants, and FCN.nll_grad_hessian falls back to the 4-point stencil,
    which matches the reference's Hessian to 1e-4 of its largest entry."""
    from tf_pwa_b200.engine import PWAError

    cl, fm, g, meta = _fcn("toy_vvp", "mixed")
    assert fm.use_gram
    v = fm.vm.variables
    with pytest.raises(PWAError, match="shared memory"):
        fm.eng.hess_sums_cached([v[k] for k in fm._var_names])
    nll, grad, H = fm.nll_grad_hessian()
    assert abs(nll - g["hess_nll"]) < 1e-3
    np.testing.assert_allclose(grad, g["hess_grad"], rtol=0,
                               atol=1e-4 * np.abs(g["hess_grad"]).max())
    np.testing.assert_allclose(H, g["hess"], rtol=0, atol=1e-4 * np.abs(g["hess"]).max())
    fm.eng.close()


def test_fit_floating_shapes_cache_vs_plain_same_minimum():
    """Masses and widths floating: the mixed form (floating-shape column
    cache) and the plain FP64 form reach the same minimum -- at the plain
    minimum x*, the shift dx = -H^-1 (g_mixed(x*) - g_plain(x*)) is below
    0.01 sigma in every constrained direction, and both fits end within
    1e-3 of each other in NLL."""
    from tf_pwa_b200.api import FCN
    from tf_pwa_b200.workload import make_dataset

    cl, data, bg, mc = make_dataset("d2kpipi_float.yml", 20000, 60000, seed=11)
    truth = list(cl.vm.get_all_val())
    fp = FCN(cl, data, mc, precision="plain")
    fr_p = cl.fit(fcn=fp, gtol=1e-6)
    xstar = np.array(cl.vm.get_all_val())
    _, g_p, H = fp.nll_grad_hessian(xstar)
    cov = np.linalg.pinv(H, rcond=1e-8, hermitian=True)
    sig = np.sqrt(np.abs(np.diag(cov)))
    fm = FCN(cl, data, mc, precision="mixed")
    assert fm.use_shape_cache and not fm.use_gram
    _, g_m = fm.nll_grad(xstar)
    dx = -cov @ (g_m - g_p)
    assert np.all(np.abs(dx) < 0.01 * sig), np.max(np.abs(dx) / sig)
    cl.vm.set_all(truth)
    fr_m = cl.fit(fcn=fm, gtol=1e-6)
    assert abs(fr_p.min_nll - fr_m.min_nll) < 1e-3
    fp.eng.close()
    fm.eng.close()

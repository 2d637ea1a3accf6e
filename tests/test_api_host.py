"""The reference-facing API (ConfigLoader.get_data -> get_fcn -> fit ->
get_params_error -> cal_fitfractions) end to end on the CPU: the engine's
device calls are replaced by the generated kernel code run on the host
(tests/hostexec.py), so the host logic of the API -- data and weights,
parameter transforms, BFGS driver, Hessian from differenced gradients,
error propagation, fit fractions -- is exercised without a GPU."""
import os

import numpy as np
import pytest
import yaml

from common import CONFIGS, load_golden
from hostexec import HostModel


def _config(tmp_path, name):
    """The golden events written as the reference's data files."""
    g, meta = load_golden(name)
    dic = yaml.safe_load(open(os.path.join(CONFIGS, meta["config"])))
    for kind, key in (("data", "p4_data"), ("phsp", "p4_mc")):
        f = tmp_path / f"{kind}.dat"
        np.savetxt(f, g[key].reshape(-1, 4), fmt="%.17g")
        dic["data"][kind] = [str(f)]
    cfg = tmp_path / "config.yml"
    cfg.write_text(yaml.safe_dump(dic))
    return str(cfg), g, meta


@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_fit_errors_fractions(host_engine, tmp_path, precision):
    from tf_pwa_b200.api import ConfigLoader

    cfg, g, meta = _config(tmp_path, "d2kpipi_float")
    cl = ConfigLoader(cfg, precision=precision)
    cl.set_params(meta["variables"])
    fcn = cl.get_fcn()
    assert not fcn.use_gram  # floating masses and widths: no column cache
    nll0, g0 = fcn.nll_grad()
    # same events, same parameters as the reference's golden NLL (the
    # mixed form here is the FP32-recompute kernel loop)
    tol = 1e-9 * abs(g["nll"]) if precision == "plain" else 1e-3
    assert abs(nll0 - g["nll"]) <= tol
    # the FP32 form's gradient carries ~1e-6 relative rounding noise: BFGS
    # ends at the reference fit's tolerance (max |g| < 1e-3) or, stalled at
    # that noise level, with a gradient of the same size
    fr = cl.fit(fcn=fcn, gtol=1e-4 if precision == "plain" else 1e-3)
    assert fr.min_nll <= nll0
    _, gmin = fcn.nll_grad()
    if precision == "plain":
        assert fr.success and np.max(np.abs(gmin)) < 1e-3
    else:
        assert np.max(np.abs(gmin)) < 1e-2, (fr.message, gmin)
    err = cl.get_params_error(fr, fcn=fcn)
    assert set(err) == set(cl.vm.trainable_vars)
    assert all(np.isfinite(v) and v > 0 for v in err.values())
    frac, err_frac = cl.cal_fitfractions(fcn=fcn)
    singles = [v for k, v in frac.items() if isinstance(k, str)]
    inter = [v for k, v in frac.items() if not isinstance(k, str)]
    assert abs(sum(singles) + sum(inter) - 1.0) < 1e-9
    assert all(np.isfinite(e) for e in err_frac.values())


def test_fit_arguments_as_reference(host_engine, tmp_path, capsys):
    """ConfigLoader.fit takes the reference's arguments: the initial NLL is
    printed, callback sees every iteration, grad_scale changes the
    minimiser's scale but not the minimum reported, jac=False differences
    the NLL, inmc / reweight are refused."""
    from tf_pwa_b200.api import ConfigLoader

    cfg, g, meta = _config(tmp_path, "d2kpipi")
    cl = ConfigLoader(cfg)
    cl.set_params(meta["variables"])
    fcn = cl.get_fcn()
    x0 = list(cl.vm.get_all_val())
    seen = []
    fr = cl.fit(fcn=fcn, callback=lambda xk: seen.append(np.array(xk)))
    assert "initial NLL" in capsys.readouterr().out
    assert seen and fr.success
    cl.vm.set_all(x0)
    fr2 = cl.fit(fcn=fcn, grad_scale=10.0, print_init_nll=False)
    assert abs(fr2.min_nll - fr.min_nll) < 1e-6
    cl.vm.set_all(x0)
    fr3 = cl.fit(fcn=fcn, jac=False, print_init_nll=False)
    assert abs(fr3.min_nll - fr.min_nll) < 1e-4
    with pytest.raises(NotImplementedError):
        cl.fit(fcn=fcn, reweight=True)


def test_force_pos_def():
    """Inverse of a positive-definite Hessian unchanged; a small negative
    eigenvalue (rounding) lifted to positive; a strongly indefinite matrix
    turned into a positive-definite error matrix."""
    from tf_pwa_b200.api import force_pos_def

    rng = np.random.default_rng(3)
    q, _ = np.linalg.qr(rng.normal(size=(5, 5)))
    h = q @ np.diag([5.0, 3.0, 2.0, 1.0, 0.5]) @ q.T
    np.testing.assert_allclose(force_pos_def(h), np.linalg.inv(h), rtol=1e-10, atol=1e-12)
    h2 = q @ np.diag([5.0, 3.0, 2.0, 1.0, -1e-7]) @ q.T
    assert np.all(np.linalg.eigvalsh(force_pos_def(h2)) > 0)
    h3 = q @ np.diag([5.0, 3.0, 2.0, 1.0, -2.0]) @ q.T
    v3 = force_pos_def(h3)
    assert np.all(np.diag(v3) > 0)
    d = np.sqrt(np.diag(v3))
    assert np.all(np.linalg.eigvalsh(v3 / np.outer(d, d)) > 0)


def test_params_error_arguments(host_engine, tmp_path):
    """get_params_error with the reference's arguments: errors stored on the
    fit result, using_cached reuses the inverse Hessian."""
    from tf_pwa_b200.api import ConfigLoader

    cfg, g, meta = _config(tmp_path, "d2kpipi")
    cl = ConfigLoader(cfg)
    cl.set_params(meta["variables"])
    fcn = cl.get_fcn()
    fr = cl.fit(fcn=fcn, print_init_nll=False)
    err = cl.get_params_error(fr, fcn=fcn)
    assert fr.error == err
    assert cl.get_params_error(using_cached=True) == err
    err2 = cl.get_params_error(fcn=fcn, force_pos=False)
    for k in err:
        assert err2[k] == pytest.approx(err[k], rel=1e-6)


def test_params_files(tmp_path):
    """save_params / set_params round trip (the fit result's "value" layout
    too), with neglect_params left untouched."""
    import json

    from tf_pwa_b200.api import ConfigLoader

    cl = ConfigLoader(os.path.join(CONFIGS, "d2kpipi.yml"))
    vals = cl.get_params()
    f = tmp_path / "p.json"
    cl.save_params(str(f))
    k0, k1 = list(cl.vm.trainable_vars)[:2]
    cl.vm.set(k0, 0.123)
    cl.vm.set(k1, 0.456)
    cl.set_params(str(f), neglect_params=[k1])
    assert cl.vm.get(k0) == vals[k0] and cl.vm.get(k1) == 0.456
    g = tmp_path / "fit.json"
    g.write_text(json.dumps({"value": {k0: 0.789}, "error": {}}))
    cl.set_params(str(g))
    assert cl.vm.get(k0) == 0.789


def test_fcn_derivative_methods(host_engine, tmp_path):
    """FCN.get_nll / get_grad / grad_hessp agree with nll_grad and the
    differenced Hessian (Hessian-vector product within 1e-6 of H p)."""
    from tf_pwa_b200.api import ConfigLoader

    cfg, g, meta = _config(tmp_path, "d2kpipi_float")
    cl = ConfigLoader(cfg)
    cl.set_params(meta["variables"])
    fcn = cl.get_fcn()
    x = np.array(cl.vm.get_all_val())
    nll, grad = fcn.nll_grad(x)
    assert fcn.get_nll(x) == nll
    np.testing.assert_array_equal(fcn.get_grad(x), grad)
    _, _, H = fcn.nll_grad_hessian(x)
    p = np.random.default_rng(2).normal(size=len(x))
    g0, hp = fcn.grad_hessp(x, p)
    np.testing.assert_array_equal(g0, grad)
    np.testing.assert_allclose(hp, H @ p, rtol=1e-6, atol=1e-6 * np.abs(H @ p).max())
    np.testing.assert_array_equal(np.array(cl.vm.get_all_val()), x)


def test_refresh_vars_ranges():
    """VarsManager.refresh_vars draws free couplings in their ranges, keeps
    fixed ones, sets init values, and draws bounded parameters inside the
    bounds (``tf_pwa/variable.py:329-420``)."""
    from tf_pwa_b200.variables import VarsManager

    vm = VarsManager(rng=np.random.default_rng(5))
    vm.add_complex_var("a")
    vm.add_complex_var("b", polar=False)
    vm.add_complex_var("c", trainable=False)
    vm.add_real_var("m", value=1.0)
    vm.add_real_var("g", value=0.1)
    vm.add_real_var("h", value=0.2)
    vm.add_real_var("k", value=0.3)
    vm.set_fix("k")
    bounds = {"g": (0.05, 0.2), "h": (0.1, None), "k": (0.0, 1.0)}
    for _ in range(50):
        vm.refresh_vars(init_val={"m": [1.0, 0.01]}, bound_dic=bounds)
        v = vm.variables
        assert 0 <= v["ar"] <= 2 and -np.pi <= v["ai"] <= np.pi
        assert -1 <= v["br"] <= 1 and -1 <= v["bi"] <= 1
        assert (v["cr"], v["ci"]) == (1.0, 0.0)
        assert 0.9 < v["m"] < 1.1 and 0.05 <= v["g"] <= 0.2 and v["h"] >= 0.1
        assert v["k"] == 0.3
    vm.refresh_vars(init_val={"m": 2.5}, bound_dic={})
    assert vm.variables["m"] == 2.5


def test_loader_fit_helpers(host_engine, tmp_path):
    """get_ndf, reinit_params, get_phsp_noeff, cal_signal_yields and
    likelihood_profile of the loader (``tf_pwa/config_loader/
    config_loader.py:180-188,722-725,803-812,918-993``)."""
    import warnings

    from tf_pwa_b200.api import ConfigLoader

    cfg, g, meta = _config(tmp_path, "d2kpipi_float")
    cl = ConfigLoader(cfg, seed=3)
    cl.set_params(meta["variables"])
    assert cl.get_ndf() == len(cl.vm.trainable_vars)
    # floated masses/widths keep their configured values, couplings move
    floated = dict(cl.init_value)
    assert floated
    before = cl.get_params()
    cl.reinit_params()
    after = cl.get_params()
    for k, v in floated.items():
        assert after[k] == v
    assert any(after[k] != before[k] for k in cl.vm.trainable_vars if k not in floated)
    cl.set_params(before)
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        ph = cl.get_phsp_noeff()
    assert ph.n == g["fields_mc"].shape[1] and w
    cl.fit(print_init_nll=False)
    cl.get_params_error()
    frac, err = cl.cal_fitfractions()
    (ys,) = cl.cal_signal_yields()
    n = g["p4_data"].shape[0]
    for k, f in frac.items():
        assert ys[k][0] == pytest.approx(f * n, rel=1e-12)
        assert ys[k][1] == pytest.approx(np.hypot(n * err[k], np.sqrt(n) * f), rel=1e-12)
    # profile in one coupling magnitude: the fitted point is the lowest
    p0 = cl.get_params()
    var = next(k for k in cl.vm.trainable_vars if k.endswith("r") and k not in floated)
    v0 = p0[var]
    vals, nlls = cl.likelihood_profile(var, v0 - 0.1 * abs(v0), v0 + 0.1 * abs(v0), N=2)
    assert len(vals) == len(nlls) >= 2 and np.all(np.diff(vals) > 0)
    assert min(nlls) == pytest.approx(nlls[vals.index(v0)], abs=1e-4)
    assert var in cl.vm.trainable_vars
    assert cl.get_params()[var] == v0


def test_attach_fix_params_error(host_engine, tmp_path):
    """attach_fix_params_error: V_a = J V_b J^T with J = da/db of the
    minimum; J checked against refits with the fixed parameter moved."""
    from tf_pwa_b200.api import ConfigLoader

    cfg, g, meta = _config(tmp_path, "d2kpipi_float")
    cl = ConfigLoader(cfg)
    cl.set_params(meta["variables"])
    b = "R2_width"
    # a well-conditioned free set on this small sample: R2's coupling and mass
    for n in (b, "R1_mass", "R1_width"):
        cl.vm.set_fix(n)
    cl.fit(print_init_nll=False, gtol=1e-9)
    cl.get_params_error()
    inv0 = cl.inv_he.copy()
    free = list(cl.vm.trainable_vars)
    a0 = np.array(cl.vm.get_all_val())
    b0 = cl.vm.variables[b]
    err_b = 1e-3
    V = cl.attach_fix_params_error({b: err_b})
    assert list(cl.vm.trainable_vars) == free and cl.vm.is_fixed(b)
    np.testing.assert_allclose(cl.inv_he, inv0 + V, rtol=0, atol=0)
    assert np.all(np.linalg.eigvalsh(V) > -1e-12 * np.abs(V).max())
    # the slope of the refitted minimum in b
    shifts = []
    for d in (-1e-4, 1e-4):
        cl.vm.set_all(list(a0))
        cl.vm.variables[b] = b0 + d
        cl.fit(print_init_nll=False, gtol=1e-9)
        shifts.append(np.array(cl.vm.get_all_val()))
    slope = (shifts[1] - shifts[0]) / 2e-4
    # V = (slope err_b)(slope err_b)^T up to the sign of the slope
    np.testing.assert_allclose(np.sqrt(np.diag(V)), np.abs(slope) * err_b,
                               rtol=2e-2, atol=1e-3 * np.abs(slope).max() * err_b)


def test_eval_amplitude_inputs(tmp_path, monkeypatch):
    """eval_amplitude accepts per-final arrays (decay order), a dict and a
    dat_order array, and hands the amplitude the same event fields."""
    from tf_pwa_b200.api import ConfigLoader

    cfg, g, meta = _config(tmp_path, "lc2pkpi")
    cl = ConfigLoader(cfg)
    seen = []
    monkeypatch.setattr(cl, "get_amplitude", lambda *a, **k: (lambda d: seen.append(d.fields)))
    p4 = g["p4_data"][:50]
    order = cl.get_dat_order()
    outs = [str(o) for o in cl.decay_group.outs]
    cl.eval_amplitude(p4)
    cl.eval_amplitude({n: p4[:, i] for i, n in enumerate(order)})
    cl.eval_amplitude(*[p4[:, order.index(n)] for n in outs])
    ref = cl.data_from_p4(p4).fields
    assert len(seen) == 3
    for f in seen:
        np.testing.assert_array_equal(f, ref)
    with pytest.raises(NotImplementedError):
        cl.eval_amplitude(p4, extra={"center_mass": True})


def test_get_chain(tmp_path):
    """get_chain by index and by particle names (``tf_pwa/particle.py:
    888-956``)."""
    from tf_pwa_b200.api import ConfigLoader

    cfg, g, meta = _config(tmp_path, "d2kpipi_float")
    cl = ConfigLoader(cfg)
    c0, c1 = cl.decay_group.chains[:2]
    assert cl.get_chain(1) is c1
    r = [p for p in c1.inner][0]
    assert cl.get_chain(str(r)) is c1 and cl.get_chain([r]) is c1
    assert cl.get_chain(str(c0.top)) is c0
    with pytest.raises(ValueError):
        cl.get_chain("no_such_particle")


def test_fcn_hessian_argument_order(host_engine, tmp_path):
    """nll_grad_hessian(x, batch) as the reference: a positional batch
    leaves the difference step at its default."""
    from tf_pwa_b200.api import ConfigLoader

    cfg, g, meta = _config(tmp_path, "d2kpipi_float")
    cl = ConfigLoader(cfg)
    cl.set_params(meta["variables"])
    fcn = cl.get_fcn()
    x = np.array(cl.vm.get_all_val())
    _, _, H1 = fcn.nll_grad_hessian(x)
    _, _, H2 = fcn.nll_grad_hessian(x, 65000)
    np.testing.assert_array_equal(H1, H2)


def test_fcn_positional_order(host_engine, tmp_path):
    """FCN(model, data, mcdata, bg, batch) as the reference: a positional
    batch does not change the likelihood; inmc samples are refused."""
    from tf_pwa_b200.api import FCN, ConfigLoader

    cfg, g, meta = _config(tmp_path, "d2kpipi_float")
    cl = ConfigLoader(cfg)
    cl.set_params(meta["variables"])
    data, phsp, _, _ = cl.get_all_data()
    a = FCN(cl, data[0], phsp[0]).nll_grad()
    b = FCN(cl, data[0], phsp[0], None, 1000).nll_grad()
    assert a[0] == b[0]
    np.testing.assert_array_equal(a[1], b[1])
    with pytest.raises(NotImplementedError):
        FCN(cl, data[0], phsp[0], None, 1000, phsp[0])

"""Fit fractions and their gradients (error propagation) against the FP64
oracle on the golden events.

* Gram path (fixed masses/widths: sub-blocks of the MC Gram matrix) and MC
  path (restricted FP64 MC pass) give the oracle's fractions within 1e-9
  relative and the same gradients within 1e-8.
* Gradients equal central finite differences (h = 1e-6) of the oracle's
  fractions, including mass and width parameters (floating-shape model).
"""
import numpy as np
import pytest

from common import golden_data, load_golden, load_model

pytestmark = pytest.mark.gpu


def _fcn(name, precision):
    from tf_pwa_b200.api import FCN, EventData

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])

    class _Cfg:
        pass

    cfg = _Cfg()
    cfg.vm, cfg.decay_group, cfg.plan = vm, dc.decay_group, plan
    x, w = golden_data(g, meta)
    fcn = FCN(cfg, EventData(x, w / (w.sum() / (w * w).sum())), EventData(g["fields_mc"]),
              precision=precision)
    return fcn, dc, vm, plan, g, meta


def _oracle_ff(dc, plan, vals, xm, res):
    from oracle.pwa_oracle import OracleModel

    m = OracleModel(dc.decay_group, plan)
    group = dc.decay_group
    tot = [c.params_head + "_total_0" for c in group]

    def integral(chains):
        v = dict(vals)
        for ci, t in enumerate(tot):
            if ci not in chains:
                v[t + "r"] = 0.0
                v[t + "i"] = 0.0
        A = m.amp(xm, v).reshape(xm.shape[1], -1)
        return float(np.sum(np.abs(A) ** 2))

    sets = [{ci for ci, c in enumerate(group) if any(str(p) == r for p in c.inner)} for r in res]
    I_all = integral(set(range(len(group))))
    out = {}
    for i, r in enumerate(res):
        for j in range(i, -1, -1):
            if i == j:
                out[r] = integral(sets[i]) / I_all
            else:
                out[(res[i], res[j])] = (integral(sets[i] | sets[j]) / I_all
                                         - out[res[i]] - out[res[j]])
    return out


@pytest.mark.parametrize("name", ["lc2pkpi", "b2dstkpi"])
def test_fit_fractions_gram_and_mc_paths(name):
    from tf_pwa_b200.fitfractions import fit_fractions

    fm, dc, vm, plan, g, meta = _fcn(name, "mixed")
    assert fm.use_gram
    res = sorted(str(p) for p in dc.decay_group.resonances)
    f_gram, _, g_gram = fit_fractions(fm.eng, vm, res, use_gram=True)
    f_mc, _, g_mc = fit_fractions(fm.eng, vm, res, use_gram=False)
    ref = _oracle_ff(dc, plan, meta["variables"], g["fields_mc"], res)
    assert set(f_gram) == set(ref)
    for k in ref:
        assert abs(f_gram[k] - ref[k]) <= 1e-9 * max(abs(ref[k]), 1e-3), (k, f_gram[k], ref[k])
        assert abs(f_mc[k] - ref[k]) <= 1e-9 * max(abs(ref[k]), 1e-3), (k, f_mc[k], ref[k])
        np.testing.assert_allclose(g_gram[k], g_mc[k], rtol=1e-8,
                                   atol=1e-8 * max(np.abs(g_mc[k]).max(), 1e-12))
    # error propagation with a given covariance
    V = np.eye(len(vm.trainable_vars)) * 1e-4
    _, err, _ = fit_fractions(fm.eng, vm, res, inv_he=V, use_gram=True)
    for k in ref:
        assert err[k] == pytest.approx(np.sqrt(1e-4 * np.sum(g_gram[k] ** 2)), rel=1e-12)
    fm.eng.close()


@pytest.mark.parametrize("name", ["lc2pkpi", "d2kpipi_float"])
def test_fit_fraction_gradients_finite_differences(name):
    from tf_pwa_b200.fitfractions import fit_fractions

    fp, dc, vm, plan, g, meta = _fcn(name, "plain")
    res = sorted(str(p) for p in dc.decay_group.resonances)
    frac, _, grad = fit_fractions(fp.eng, vm, res, use_gram=False)
    names = list(vm.trainable_vars)
    vals = dict(meta["variables"])
    xm = g["fields_mc"]
    for pi, n in enumerate(names):
        h = 1e-6 * max(abs(vals[n]), 1.0)
        vp, vmn = dict(vals), dict(vals)
        vp[n] += h
        vmn[n] -= h
        fp_, fm_ = _oracle_ff(dc, plan, vp, xm, res), _oracle_ff(dc, plan, vmn, xm, res)
        for k in frac:
            fd = (fp_[k] - fm_[k]) / (2 * h)
            scale = max(np.abs(grad[k]).max(), 1e-8)
            assert abs(grad[k][pi] - fd) <= 2e-6 * scale, (n, k, grad[k][pi], fd)
    fp.eng.close()

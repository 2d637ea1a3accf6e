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


@pytest.mark.parametrize("name", ["d2kpipi", "d2kpipi_float"])
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
    from tf_pwa_b200.api import FCN
    from tf_pwa_b200.workload import make_dataset

    cl, data, bg, mc = make_dataset("lc2pkpi.yml", 20000, 60000, n_bg=2000, seed=7)
    truth = cl.vm.get_all_val()
    res = {}
    for prec in ("plain", "mixed"):
        cl.vm.set_all(list(truth))
        fcn = FCN(cl, data, mc, bg=bg, precision=prec)
        fr = cl.fit(fcn=fcn, gtol=1e-6)
        res[prec] = (fr, np.array(cl.vm.get_all_val()))
        if prec == "plain":
            err = cl.get_params_error(fcn=fcn)
            sig = np.array([err[k] for k in cl.vm.trainable_vars])
        fcn.eng.close()
    (fp, xp), (fm, xm) = res["plain"], res["mixed"]
    assert fp.success or fp.min_nll < 0
    assert abs(fp.min_nll - fm.min_nll) < 1e-3
    # polar phases: compare modulo 2 pi
    d = xp - xm
    names = cl.vm.trainable_vars
    for i, n in enumerate(names):
        if n.endswith("i"):
            d[i] = (d[i] + np.pi) % (2 * np.pi) - np.pi
    assert np.all(np.abs(d) < 0.01 * sig), np.max(np.abs(d) / sig)

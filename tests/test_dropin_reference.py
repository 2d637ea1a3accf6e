"""The engine behind the reference package's own NLL-model registry.

The reference's ``ConfigLoader`` (run over the torch-backed TF-API stand-in
in tests/golden/tfshim) loads a config with ``data: {model: b200}``; its
``get_fcn().nll_grad()`` then goes through ``tf_pwa_b200.tfpwa_plugin``'s
``B200Model.nll_grad_batch`` and must reproduce the reference's own NLL
and GradientTape gradient recorded in the golden files (plain FP64: 1e-9
relative NLL, 1e-7 of the largest gradient entry; mixed form: |dNLL| <
1e-3, 1e-4).  On the CPU the engine's device calls run as the generated
kernel code on the host (``host_engine``); under ``-m gpu`` the real
library runs.  The reference package comes from ``baseline/_ref`` (an
installed copy) or, on the CPU only, from the checkout named by
``PWA_REFERENCE``.
"""
import os
import sys
import warnings

import numpy as np
import pytest
import yaml

from common import CONFIGS, GOLDEN, ROOT, load_golden


def _reference_path(gpu):
    cands = [os.path.join(ROOT, "baseline", "_ref")]
    if not gpu and os.environ.get("PWA_REFERENCE"):
        cands.append(os.environ["PWA_REFERENCE"])
    for c in cands:
        if os.path.isdir(os.path.join(c, "tf_pwa")):
            return c
    return None


def _import_reference(gpu):
    ref = _reference_path(gpu)
    if ref is None:
        pytest.skip("the reference package is not installed (baseline/_ref)")
    shim = os.path.join(GOLDEN, "tfshim")
    for p in (ref, shim):
        if p not in sys.path:
            sys.path.insert(0, p)
    warnings.filterwarnings("ignore")
    import tf_pwa  # noqa: F401


def _config(tmp_path, name, precision, device):
    g, meta = load_golden(name)
    dic = yaml.safe_load(open(os.path.join(CONFIGS, meta["config"])))
    for kind, key in (("data", "p4_data"), ("phsp", "p4_mc"), ("bg", "p4_bg")):
        if key in g:
            f = tmp_path / f"{kind}.dat"
            np.savetxt(f, g[key].reshape(-1, 4), fmt="%.17g")
            dic["data"][kind] = [str(f)]
    dic["data"].update(meta.get("extra_data", {}))
    cfg = tmp_path / "config.yml"
    dic["data"]["model"] = "b200"
    dic["nll_model"] = {"config_file": str(cfg), "precision": precision, "device": device}
    cfg.write_text(yaml.safe_dump(dic))
    return str(cfg), g, meta


def _run(cfg, meta):
    from tf_pwa.config_loader import ConfigLoader as RefConfigLoader

    from tf_pwa_b200.tfpwa_plugin import register

    cls = register()
    ref = RefConfigLoader(cfg)
    ref.set_params(meta["variables"])
    fcn = ref.get_fcn()
    assert isinstance(fcn.model, cls)
    assert list(ref.get_amplitude().vm.trainable_vars) == meta["trainable"]
    nll, grad = fcn.nll_grad()
    return float(nll), np.asarray(grad, np.float64)


@pytest.mark.parametrize("name", ["d2kpipi", "lc2pkpi"])
def test_registry_model_host(host_engine, tmp_path, name):
    _import_reference(gpu=False)
    cfg, g, meta = _config(tmp_path, name, "plain", "cpu")
    nll, grad = _run(cfg, meta)
    assert abs(nll - float(g["nll"])) <= 1e-9 * abs(float(g["nll"])), (nll, g["nll"])
    assert np.max(np.abs(grad - g["grad"])) <= 1e-7 * np.max(np.abs(g["grad"]))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_registry_model_gpu(tmp_path, precision):
    _import_reference(gpu=True)
    cfg, g, meta = _config(tmp_path, "lc2pkpi", precision, "cuda")
    nll, grad = _run(cfg, meta)
    if precision == "plain":
        assert abs(nll - float(g["nll"])) <= 1e-9 * abs(float(g["nll"]))
        assert np.max(np.abs(grad - g["grad"])) <= 1e-7 * np.max(np.abs(g["grad"]))
    else:
        assert abs(nll - float(g["nll"])) < 1e-3
        assert np.max(np.abs(grad - g["grad"])) <= 1e-4 * np.max(np.abs(g["grad"]))

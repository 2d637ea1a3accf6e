"""Test configuration: registers the ``gpu`` marker and makes the engine
package importable as ``tf_pwa_b200`` from its ``tf-pwa_b200`` directory."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _load_pkg():
    if "tf_pwa_b200" in sys.modules:
        return
    d = os.path.join(ROOT, "tf-pwa_b200")
    spec = importlib.util.spec_from_file_location(
        "tf_pwa_b200", os.path.join(d, "__init__.py"), submodule_search_locations=[d])
    m = importlib.util.module_from_spec(spec)
    sys.modules["tf_pwa_b200"] = m
    spec.loader.exec_module(m)


_load_pkg()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture()
def host_engine(monkeypatch, tmp_path):
    """Engine whose plan creation, upload and evaluation run on the host:
    the generated kernel code compiled with g++ (tests/hostexec.py)."""
    import numpy as np

    import tf_pwa_b200.engine as E
    from hostexec import HostModel

    built = {}

    def _create(self):
        self.h = None
        key = self.src
        if key not in built:
            built[key] = HostModel(self.code, str(tmp_path))
        self._host = built[key]

    def upload(self, x_data, w_data, x_mc=None, w_mc=None, stream=None):
        xd = np.asarray(x_data, np.float64)
        wd = np.asarray(w_data, np.float64)
        xm = np.asarray(x_mc, np.float64)
        wm = np.ones(xm.shape[1]) if w_mc is None else np.asarray(w_mc, np.float64)
        self._hx = (np.concatenate([xd, xm], 1), np.concatenate([wd, wm / wm.sum()]),
                    xd.shape[1])
        self._n_data, self._n_mc = xd.shape[1], xm.shape[1]
        self._sw = float(wd.sum())
        self._gram = None

    def eval_sums(self, C, precision=E.PLAIN_F64, mc=True, stream=None):
        x, w, nd = self._hx
        return self._host.sums(C, x, w, nd, f32=precision == E.MIXED_F32)

    # the native host program runs as in the product; only the kernels'
    # sums come from the host-compiled model code
    def set_host_program(self, var_names, train_names):
        self._hp = self.host_program(var_names, train_names)
        self._hp_train = len(train_names)

    def pieces_vars(self, var_values, form, mc_share=None, stream=None):
        v = np.asarray(var_values, np.float64)
        C = self._hp.consts(v)
        sd, sm = self.eval_sums(C, E.PLAIN_F64 if form == E.FORM_PLAIN_F64 else E.MIXED_F32)
        share = self.mc_share if mc_share is None else mc_share
        return self._hp.pieces(v, sd, sm, self._sw, share)

    def nll_grad_vars(self, var_values, form, stream=None):
        vec = self.pieces_vars(var_values, form, stream=stream)
        if self.dist_reduce is not None:
            vec = self.dist_reduce(vec)
        return E.combine_pieces(vec, self._hp_train)

    monkeypatch.setattr(E.Engine, "set_host_program", set_host_program)
    monkeypatch.setattr(E.Engine, "pieces_vars", pieces_vars)
    monkeypatch.setattr(E.Engine, "nll_grad_vars", nll_grad_vars)
    monkeypatch.setattr(E.Engine, "_create", _create)
    monkeypatch.setattr(E.Engine, "upload", upload)
    monkeypatch.setattr(E.Engine, "eval_sums", eval_sums)
    monkeypatch.setattr(E.Engine, "close", lambda self: None)
    return E

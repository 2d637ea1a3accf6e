"""Host logic of the reference-named generators on ConfigLoader
(``generate_phsp``, ``generate_phsp_p``, ``generate_toy``;
``tf_pwa/config_loader/sample.py``): chunked candidate loop, accept-reject
maximum kept and reused, seeds.  The engine's toy kernels are replaced by
the generator and amplitude oracles on the CPU (the kernels themselves are
checked against the same oracles in the GPU tests)."""
import numpy as np
import pytest
import torch

from common import CONFIGS


class OracleToyEngine:
    """Stand-in for the toy kernels of ``Engine`` (same call signatures)."""

    device = "cpu"
    toy_chunk = 4096

    def __init__(self, cl):
        from oracle.pwa_oracle import OracleModel
        from tf_pwa_b200.engine import Engine

        self.real = Engine(cl.decay_group, cl.plan, cl.vm, compile=False)
        self.plan, self.code = cl.plan, self.real.code
        self.model = OracleModel(cl.decay_group, cl.plan)
        self.cl = cl
        self.calls = []

    def consts(self, vals):
        self.vals = dict(vals)
        return self.real.consts(vals)

    def _events(self, seed, idx):
        from oracle.toy_oracle import genbod_levels, uniforms

        kin = self.code.kin
        U = uniforms(seed, np.asarray(idx), kin.ndraw)
        p, wps = genbod_levels(U, kin.levels, kin.nfin)
        return U, p, wps

    def _fields(self, p):
        from tf_pwa_b200.kinematics import event_fields, p4_dict

        return event_fields(self.plan, p4_dict(np.transpose(p, (2, 0, 1)), self.plan.order))

    def toy_select(self, C, seed, first, n, fmax, flat, out):
        from oracle.toy_oracle import select

        kin = self.code.kin
        self.calls.append((first, n, fmax, flat))
        pdf = None
        if not flat:
            pdf = lambda p4: self.model.pdf(  # noqa: E731
                self._fields(np.transpose(p4, (1, 2, 0))).numpy(), self.vals)
        res, _ = select(seed, first, n, kin.levels, kin.nfin, pdf=pdf, fmax=fmax)
        out[:n] = torch.as_tensor(res)

    def toy_fields(self, seed, idx, with_p4=False):
        _, p, _ = self._events(seed, idx.numpy())
        x = self._fields(p)
        if with_p4:
            return x, torch.as_tensor(np.transpose(p, (2, 0, 1)))
        return x

    def close(self):
        pass


@pytest.fixture()
def loader(monkeypatch):
    import os

    from tf_pwa_b200.api import ConfigLoader

    cl = ConfigLoader(os.path.join(CONFIGS, "d2kpipi.yml"), seed=3)
    engines = []

    def make():
        engines.append(OracleToyEngine(cl))
        return engines[-1]

    monkeypatch.setattr(cl, "_toy_engine", make)
    cl._engines = engines
    return cl


def test_phase_space_events_and_momenta(loader):
    from tf_pwa_b200.kinematics import event_fields, p4_dict

    d = loader.generate_phsp(1500, seed=11)
    assert d.fields.shape == (loader.plan.n_fields, 1500)
    assert np.all(np.asarray(d.weight) == 1.0)
    p4 = loader.generate_phsp_p(1500, seed=11)
    assert tuple(p4.shape) == (1500, 3, 4)
    x = event_fields(loader.plan, p4_dict(p4.numpy(), loader.get_dat_order())).numpy()
    np.testing.assert_array_equal(x, d.fields.numpy())
    # a fresh seed per call when none is given
    a = loader.generate_phsp(10).fields.numpy()
    b = loader.generate_phsp(10).fields.numpy()
    assert not np.array_equal(a, b)
    assert loader.generate_phsp(0).fields.shape == (loader.plan.n_fields, 0)


def test_toy_accept_reject_and_max_reused(loader):
    from oracle.pwa_oracle import OracleModel

    n = 800
    toy = loader.generate_toy(n, seed=5)
    assert toy.fields.shape[1] == n
    fmax = loader.max_amplitude
    assert fmax is not None and fmax > 0
    first = loader._engines[-1].calls[0]
    assert first[2] == 0.0 and first[3] == 0  # the phase-space pass that finds the maximum
    m = OracleModel(loader.decay_group, loader.plan)
    vals = loader.vm.get_all_dic()
    f_toy = m.pdf(toy.fields.numpy(), vals)
    f_phsp = m.pdf(loader.generate_phsp(n, seed=6).fields.numpy(), vals)
    assert np.all(f_toy <= fmax)
    assert f_toy.mean() > 1.2 * f_phsp.mean()  # accept-reject favours large |A|^2
    loader.generate_toy(100, seed=7)
    assert all(c[2] > 0 for c in loader._engines[-1].calls)  # the kept maximum is reused

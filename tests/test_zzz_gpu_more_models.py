"""GPU checks of the later model options, collected after the rest of the
GPU suite (so that under ``-x`` a failure here does not stop the others):

* per-event charges (parity transform under cp_trans; helicity-coupling
  reversal without it), vector-polarised spin-1/2 and spin-1 parents,
  CP-violating chain totals:
  plain FP64 NLL within 1e-9 and gradient within 1e-7 of the reference's
  values, the FP32 form within |dNLL| < 1e-3 and 1e-4 of the largest
  gradient component, per-event |A|^2 within 1e-11 (FP64) / 2e-4 (FP32);
* device kinematics of charged and lab-frame events against the
  reference's fields (1e-11 absolute);
* ConfigLoader.generate_phsp / generate_phsp_p / generate_toy.

The same models are checked on the CPU by the oracle and by the generated
kernel code run on the host (tests/test_hostexec_codegen.py)."""
import numpy as np
import pytest

from common import golden_data, load_golden, load_model

pytestmark = pytest.mark.gpu

TOL_FIELD = 1e-11
MODELS = ["lc2pkpi_cc", "b2dstkpi_cc", "lc2pkpi_pol", "epem_pol", "lc2pkpi_cp"]


def _engine(name):
    from tf_pwa_b200.engine import Engine

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])
    eng = Engine(dc.decay_group, plan, vm)
    x, w = golden_data(g, meta)
    eng.upload(x, w, g["fields_mc"], np.ones(g["fields_mc"].shape[1]))
    return eng, g, meta


@pytest.mark.parametrize("name", MODELS)
def test_plain_and_fp32_forms(name):
    import torch

    from tf_pwa_b200.engine import MIXED_F32, PLAIN_F64

    eng, g, meta = _engine(name)
    scale = np.abs(g["grad"]).max()
    nll, grad = eng.nll_grad(meta["variables"], meta["trainable"], PLAIN_F64)
    assert abs(nll - g["nll"]) <= 1e-9 * abs(g["nll"]), (nll, g["nll"])
    np.testing.assert_allclose(grad, g["grad"], rtol=1e-7, atol=1e-7 * scale)
    nll, grad = eng.nll_grad(meta["variables"], meta["trainable"], MIXED_F32)
    assert abs(nll - g["nll"]) < 1e-3
    assert np.max(np.abs(grad - g["grad"])) <= 1e-4 * scale
    C = eng.consts(meta["variables"])
    nd = g["fields_data"].shape[1]
    out = torch.empty(nd, dtype=torch.float64, device="cuda")
    eng.pdf_device(C, 0, nd, out.data_ptr(), PLAIN_F64)
    np.testing.assert_allclose(out.cpu().numpy(), g["f_data"], rtol=1e-11)
    eng.pdf_device(C, 0, nd, out.data_ptr(), MIXED_F32)
    np.testing.assert_allclose(out.cpu().numpy(), g["f_data"], rtol=2e-4)
    eng.close()


@pytest.mark.parametrize("name", ["lc2pkpi_cc", "b2dstkpi_cc", "lc2pkpi_pol_lab"])
def test_device_kinematics(name):
    import torch

    from tf_pwa_b200.engine import Engine

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    eng = Engine(dc.decay_group, plan, vm)
    for kind in ("data", "mc"):
        p4 = torch.as_tensor(g["p4_" + kind], device="cuda")
        ch = g.get("charge_" + kind)
        x = eng.fields_from_p4(p4, charge=None if ch is None else
                               torch.as_tensor(ch, device="cuda")).cpu().numpy()
        np.testing.assert_allclose(x, g["fields_" + kind], rtol=0, atol=TOL_FIELD)
    eng.close()


def test_config_loader_generators():
    """ConfigLoader.generate_phsp / generate_phsp_p / generate_toy on the
    toy kernels: the phase-space fields are the kinematics of the returned
    momenta; the toy keeps its accept-reject maximum."""
    import os

    from common import CONFIGS
    from tf_pwa_b200.api import ConfigLoader
    from tf_pwa_b200.kinematics import event_fields, p4_dict

    cl = ConfigLoader(os.path.join(CONFIGS, "lc2pkpi.yml"), seed=2)
    d = cl.generate_phsp(3000, seed=21)
    p4 = cl.generate_phsp_p(3000, seed=21)
    assert tuple(p4.shape) == (3000, 3, 4)
    x = event_fields(cl.plan, p4_dict(p4.cpu().numpy(), cl.get_dat_order())).numpy()
    np.testing.assert_allclose(d.fields.cpu().numpy(), x, rtol=0, atol=TOL_FIELD)
    toy = cl.generate_toy(2000, seed=22)
    assert toy.fields.shape == (cl.plan.n_fields, 2000)
    assert cl.max_amplitude is not None and cl.max_amplitude > 0

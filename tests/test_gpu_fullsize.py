"""Parity against the reference at the workloads' own sizes (through the C ABI).

D -> K pi pi with 1e4 data / 1e5 MC events, and Lambda_c -> p K pi with 1e5
signal + 1e4 background rows (weight -0.1) / 1e6 MC events; the signal
data are drawn from the model by accept-reject on |A|^2, as the workloads
define them.  The golden
files (``tests/golden/make_golden.py``, cases ``d2kpipi_1e4`` and
``lc2pkpi_full``) hold the reference's own NLL and GradientTape gradient
over all events, its fields and |A|^2 at seeded subsets of the events, and
the generator seeds; the events are regenerated here with the same seeded
generator, their fields formed on the GPU.

Tolerances (written in the assertions):
  * fields: 1e-11 absolute; |A|^2: 1e-10 relative per event;
  * plain FP64 form: NLL 1e-9 relative, gradient 1e-7 of its largest entry;
  * mixed form (FP32 column cache + FP64 Gram) and FP32-amplitude
    recompute form: |dNLL| < 1e-3, gradient 1e-4 of its largest entry --
    both against the reference, not against the plain GPU path.
"""
import numpy as np
import pytest

from common import load_golden, load_model

pytestmark = pytest.mark.gpu


class _Cfg:
    pass


def _events(meta, g, dc, plan):
    """Momenta (n, n_final, 4) of every set, regenerated from the seeds; the
    signal data are the stored accept-reject survivors among their flat
    candidates."""
    from tf_pwa_b200.decay_config import load_yaml
    from tf_pwa_b200.phasespace import generate_phsp

    import os
    from common import CONFIGS

    dic = load_yaml(os.path.join(CONFIGS, meta["config"]))
    order = dic["data"]["dat_order"]
    masses = [dc.particle_property[o]["mass"] for o in order]
    M = dc.particle_property[str(dc.decay_group.top)]["mass"]
    ev = meta["events"]
    out = {}
    for tag in ("data", "bg", "mc"):
        n = ev["sizes"][tag]
        if not n:
            continue
        if tag == "data" and ev.get("data_candidates"):
            cand = np.stack(generate_phsp(M, masses, ev["data_candidates"],
                                          seed=ev["seeds"][tag]), 1)
            out[tag] = cand[g["data_kept"]]
            assert out[tag].shape[0] == n
        else:
            out[tag] = np.stack(generate_phsp(M, masses, n, seed=ev["seeds"][tag]), 1)
    return out


@pytest.fixture(scope="module", params=["d2kpipi_1e4", "lc2pkpi_full"])
def case(request):
    import torch

    from tf_pwa_b200.api import EventData
    from tf_pwa_b200.engine import Engine

    g, meta = load_golden(request.param)
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])
    p4 = _events(meta, g, dc, plan)
    eng = Engine(dc.decay_group, plan, vm)
    fields = {t: eng.fields_from_p4(torch.as_tensor(a, device="cuda")) for t, a in p4.items()}
    cfg = _Cfg()
    cfg.vm, cfg.decay_group, cfg.plan = vm, dc.decay_group, plan
    data = EventData(fields["data"], np.ones(fields["data"].shape[1]))
    bg = None
    if "bg" in fields:
        bg = EventData(fields["bg"], -meta["extra_data"]["bg_weight"] * np.ones(fields["bg"].shape[1]))
    mc = EventData(fields["mc"])
    yield dict(g=g, meta=meta, vm=vm, eng=eng, fields=fields, cfg=cfg, data=data, bg=bg, mc=mc)
    eng.close()


def test_fields_and_amplitudes(case):
    import torch

    g, eng, vm = case["g"], case["eng"], case["vm"]
    C = eng.consts(vm.get_all_dic())
    for tag, x in case["fields"].items():
        i_f = g[f"idx_fields_{tag}"]
        got = x[:, torch.as_tensor(i_f, device="cuda")].cpu().numpy()
        np.testing.assert_allclose(got, g[f"fields_{tag}"], rtol=0, atol=1e-11)
        n = x.shape[1]
        assert n == int(g[f"n_{tag}"])
        xc = x.cpu().numpy()
        eng.upload(xc, np.ones(n))
        f = torch.empty(n, dtype=torch.float64, device="cuda")
        eng.pdf_device(C, 0, n, f.data_ptr())
        f = f.cpu().numpy()
        i_a = g[f"idx_f_{tag}"]
        np.testing.assert_allclose(f[i_a], g[f"f_{tag}"], rtol=1e-10)
        assert abs(f.sum() - float(g[f"sum_f_{tag}"])) <= 1e-10 * abs(float(g[f"sum_f_{tag}"]))


def _fcn(case, precision, gram=None):
    from tf_pwa_b200.api import FCN

    return FCN(case["cfg"], case["data"], case["mc"], bg=case["bg"], precision=precision,
               gram=gram)


def test_plain_nll_grad(case):
    g = case["g"]
    fcn = _fcn(case, "plain")
    nll, grad = fcn.nll_grad()
    fcn.eng.close()
    ref_nll, ref_g = float(g["nll"]), g["grad"]
    assert abs(nll - ref_nll) <= 1e-9 * abs(ref_nll), (nll, ref_nll)
    assert np.max(np.abs(grad - ref_g)) <= 1e-7 * np.max(np.abs(ref_g)), (grad, ref_g)
    assert abs(float(np.sum(fcn.weight)) - float(g["sum_w"])) <= 1e-12 * abs(float(g["sum_w"]))


@pytest.mark.parametrize("form", ["mixed_gram", "fp32_recompute"])
def test_chosen_forms_against_reference(case, form):
    g = case["g"]
    fcn = _fcn(case, "mixed", gram=(form == "mixed_gram"))
    assert fcn.use_gram == (form == "mixed_gram")
    nll, grad = fcn.nll_grad()
    fcn.eng.close()
    ref_nll, ref_g = float(g["nll"]), g["grad"]
    assert abs(nll - ref_nll) < 1e-3, (form, nll, ref_nll)
    assert np.max(np.abs(grad - ref_g)) <= 1e-4 * np.max(np.abs(ref_g)), (form, grad, ref_g)

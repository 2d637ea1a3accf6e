"""Dataset step on the GPU: kinematics and toy generation kernels.

* pwa_fields_from_p4 on the golden momenta reproduces the fields that the
  reference's cal_angle produced (1e-11 absolute), including the proton
  alignment angles of the Lambda_c model and the four-body topologies.
* pwa_toy_select keeps exactly the candidates the CPU generator oracle
  keeps (same Philox stream, GENBOD, |A|^2 from the FP64 amplitude oracle),
  flat and with accept-reject; kept |A|^2 agree to 1e-10 relative.
* pwa_toy_fields regenerates the kept events: momenta equal the oracle's,
  fields equal the host kinematics of those momenta.
"""
import numpy as np
import pytest

from common import load_golden, load_model

pytestmark = pytest.mark.gpu

TOL_FIELD = 1e-11


def _engine(cfg, variables=None):
    from tf_pwa_b200.engine import Engine

    dc, vm, plan = load_model(cfg)
    if variables is not None:
        vm.set_all(variables)
    return Engine(dc.decay_group, plan, vm), dc, vm, plan


@pytest.mark.parametrize("name", ["d2kpipi", "lc2pkpi", "b2dstkpi", "dp2kpipi_ident", "ident_fermions",
                                  "epem_cp"])
def test_fields_from_p4_match_reference(name):
    import torch

    g, meta = load_golden(name)
    eng, dc, vm, plan = _engine(meta["config"])
    for kind in ("data", "mc"):
        p4 = torch.as_tensor(g["p4_" + kind], device="cuda")
        ch = g.get("charge_" + kind)
        x = eng.fields_from_p4(p4, charge=None if ch is None else
                               torch.as_tensor(ch, device="cuda")).cpu().numpy()
        np.testing.assert_allclose(x, g["fields_" + kind], rtol=0, atol=TOL_FIELD)
    eng.close()


def _oracle_pdf(dc, plan, vals):
    from oracle.pwa_oracle import OracleModel
    from tf_pwa_b200.kinematics import event_fields, p4_dict

    m = OracleModel(dc.decay_group, plan)

    def pdf(p4):
        x = event_fields(plan, p4_dict(p4, plan.order)).numpy()
        return np.sum(np.abs(m.amp(x, vals).reshape(x.shape[1], -1)) ** 2, 1)

    return pdf


@pytest.mark.parametrize("name", ["lc2pkpi", "b2dstkpi"])
def test_toy_select_matches_oracle(name):
    import torch

    from oracle.toy_oracle import select

    g, meta = load_golden(name)
    eng, dc, vm, plan = _engine(meta["config"], meta["variables"])
    kin = eng.code.kin
    seed, first, n = 0x1234ABCD5678, 1 << 33, 20000
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    # flat phase space
    eng.toy_select(None, seed, first, n, 0.0, 1, out)
    ref, _ = select(seed, first, n, kin.levels, kin.nfin)
    np.testing.assert_array_equal(out.cpu().numpy(), ref)
    # signal: phase-space step alone, then accept-reject against fmax
    C = eng.consts(meta["variables"])
    pdf = _oracle_pdf(dc, plan, meta["variables"])
    eng.toy_select(C, seed, first, n, 0.0, 0, out)
    f0 = out.cpu().numpy()
    ref0, _ = select(seed, first, n, kin.levels, kin.nfin, pdf=pdf)
    np.testing.assert_array_equal(f0 >= 0, ref0 >= 0)
    np.testing.assert_allclose(f0, ref0, rtol=1e-10)
    fmax = 0.3 * float(ref0.max())   # a low bound, so that many candidates are kept
    eng.toy_select(C, seed, first, n, fmax, 0, out)
    f1 = out.cpu().numpy()
    ref1, _ = select(seed, first, n, kin.levels, kin.nfin, pdf=pdf, fmax=fmax)
    np.testing.assert_array_equal(f1 >= 0, ref1 >= 0)
    assert 0 < (f1 >= 0).sum() < (f0 >= 0).sum()
    eng.close()


@pytest.mark.parametrize("name", ["lc2pkpi", "b2dstkpi"])
def test_toy_fields_regenerate_events(name):
    import torch

    from oracle.toy_oracle import select
    from tf_pwa_b200.kinematics import event_fields, p4_dict

    g, meta = load_golden(name)
    eng, dc, vm, plan = _engine(meta["config"])
    kin = eng.code.kin
    seed, n = 77, 4096
    ref, p = select(seed, 0, n, kin.levels, kin.nfin)
    keep = np.nonzero(ref >= 0)[0]
    idx = torch.as_tensor(keep, dtype=torch.int64, device="cuda")
    x, p4 = eng.toy_fields(seed, idx, with_p4=True)
    p_ref = np.transpose(p[:, :, keep], (2, 0, 1))
    np.testing.assert_allclose(p4.cpu().numpy(), p_ref, rtol=0, atol=1e-13)
    x_ref = event_fields(plan, p4_dict(p_ref, plan.order)).numpy()
    np.testing.assert_allclose(x.cpu().numpy(), x_ref, rtol=0, atol=TOL_FIELD)
    eng.close()


def test_generated_dataset_statistics():
    """make_dataset on the device: requested sizes, finite fields, unit
    weights, and the flat MC's first invariant mass moment equal to the
    oracle generator's within 5 sigma."""
    import torch

    from oracle.toy_oracle import select
    from tf_pwa_b200.workload import make_dataset

    cl, data, bg, mc = make_dataset("lc2pkpi.yml", 20000, 50000, n_bg=2000, seed=3)
    assert data.n == 20000 and mc.n == 50000 and bg.n == 2000
    for d in (data, mc, bg):
        assert bool(torch.isfinite(d.fields).all())
    from tf_pwa_b200.kincode import KinCode
    from tf_pwa_b200.kinematics import event_fields, p4_dict

    plan = cl.plan
    j = plan.fields.index(next(f for f in plan.fields if f.startswith("m/")))
    kin = KinCode(plan, plan.order)
    ref, p = select(11, 0, 200000, kin.levels, kin.nfin)
    keep = ref >= 0
    xr = event_fields(plan, p4_dict(np.transpose(p[:, :, keep], (2, 0, 1)), plan.order)).numpy()[j]
    xm = mc.fields[j].cpu().numpy()
    err = np.sqrt(xr.var() / len(xr) + xm.var() / len(xm))
    assert abs(xr.mean() - xm.mean()) < 5 * err


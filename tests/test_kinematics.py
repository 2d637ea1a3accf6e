"""Dataset kinematics (four-momenta -> masses, helicity and alignment
angles) against the fields the reference's cal_angle produced for the same
momenta (golden vectors)."""
import numpy as np
import pytest

from common import load_golden, load_model


@pytest.mark.parametrize("name", ["d2kpipi", "lc2pkpi", "toy_vvp", "b2dstkpi", "dp2kpipi_ident",
                                  "ident_fermions", "epem_cp", "lc2pkpi_cc", "b2dstkpi_cc",
                                  "ident3_fermions", "lc2pkpi_pol_lab"])
@pytest.mark.parametrize("kind", ["data", "mc"])
def test_fields_match_reference_cal_angle(name, kind):
    """(with per-event charges: parity transform of charge -1 momenta under
    cp_trans, or the charge field without it; lc2pkpi_pol_lab: momenta out
    of the parent rest frame, its flight direction as z)"""
    from tf_pwa_b200.kinematics import event_fields, p4_dict

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    x = event_fields(plan, p4_dict(g["p4_" + kind], dc.data_config["dat_order"]),
                     charge=g.get("charge_" + kind)).numpy()
    np.testing.assert_allclose(x, g["fields_" + kind], rtol=0, atol=1e-11)


def test_phase_space_conservation():
    """Generated momenta conserve four-momentum and have the final masses
    (tf_pwa/tests/test_phasespace.py:7-30)."""
    from tf_pwa_b200.phasespace import generate_phsp

    ms = [0.938272, 0.493677, 0.13957]
    ps = generate_phsp(2.28646, ms, 5000, seed=3)
    tot = sum(ps)
    np.testing.assert_allclose(tot[:, 0], 2.28646, atol=1e-12)
    np.testing.assert_allclose(tot[:, 1:], 0.0, atol=1e-12)
    for p, m in zip(ps, ms):
        np.testing.assert_allclose(np.sqrt(p[:, 0] ** 2 - (p[:, 1:] ** 2).sum(1)), m, atol=1e-10)


def test_helicity_gamma_zero_and_ranges():
    """Helicity angles: beta in [0, pi], alpha in the reference's range
    (tf_pwa/tests/test_cal_angle.py)."""
    from tf_pwa_b200.kinematics import event_fields, p4_dict
    from tf_pwa_b200.phasespace import generate_phsp

    dc, vm, plan = load_model("lc2pkpi.yml")
    ps = generate_phsp(2.28646, [0.938272, 0.493677, 0.13957], 2000, seed=4)
    x = event_fields(plan, p4_dict(np.stack(ps, 1), ["p", "K", "pi"])).numpy()
    for f, col in zip(plan.fields, x):
        if f.endswith("/beta"):
            assert col.min() >= 0 and col.max() <= np.pi
        if f.endswith("/alpha") and "aligned" not in f:
            assert col.min() >= -2 * np.pi - 1e-12 and col.max() <= np.pi + 1e-12

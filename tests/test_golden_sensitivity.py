"""The golden comparisons have teeth: a deliberate mistake planted in the
oracle (on the CPU) -- a wrong swap sign, no helicity-coupling reversal for
charge -1 events, an unpolarised density matrix, BWR in place of BWR2, CP
asymmetries of the chain totals dropped -- moves
sum |A|^2 far outside the parity tolerance against the reference's values."""
import copy

import numpy as np
import pytest

from common import load_golden, load_model


def _max_rel(m, g, meta):
    return np.max(np.abs(m.pdf(g["fields_data"], meta["variables"]) / g["f_data"] - 1))


def _setup(name):
    from oracle.pwa_oracle import OracleModel

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    m = OracleModel(dc.decay_group, plan)
    assert _max_rel(m, g, meta) < 1e-10
    return g, meta, dc, plan, m


def test_swap_sign():
    g, meta, dc, plan, m = _setup("ident_fermions")
    plan.swaps = copy.deepcopy(plan.swaps)
    plan.swaps[0]["factor"] *= -1
    assert _max_rel(m, g, meta) > 1e-3


def test_swap_axis_order():
    g, meta, dc, plan, m = _setup("ident_fermions")
    plan.swaps = copy.deepcopy(plan.swaps)
    plan.swaps[0]["trans"] = list(range(len(plan.swaps[0]["trans"])))
    assert _max_rel(m, g, meta) > 1e-3


def test_charge_reversal():
    g, meta, dc, plan, m = _setup("b2dstkpi_cc")
    plan.charge_index = None
    assert _max_rel(m, g, meta) > 1e-3


def test_cp_conjugate_flip():
    g, meta, dc, plan, m = _setup("epem_cp")
    plan.swaps = copy.deepcopy(plan.swaps)
    plan.swaps[0]["flip"] = False
    assert _max_rel(m, g, meta) > 1e-3


def test_density_matrix():
    g, meta, dc, plan, m = _setup("lc2pkpi_pol")
    m.density = lambda vals: None
    assert _max_rel(m, g, meta) > 1e-3


@pytest.mark.parametrize("what", ["bwr2", "width_norm"])
def test_lineshape_options(what, monkeypatch):
    from tf_pwa_b200.particles import Particle

    g, meta, dc, plan, m = _setup("d2kpipi_shapes")
    if what == "bwr2":
        orig = Particle.lineshape_kind
        monkeypatch.setattr(Particle, "lineshape_kind",
                            lambda self: "BWR" if orig(self) == "BWR2" else orig(self))
    else:
        monkeypatch.setattr(Particle, "width_norm_applies", lambda self: False)
    assert _max_rel(m, g, meta) > 1e-3


def test_cp_violating_totals():
    g, meta, dc, plan, m = _setup("lc2pkpi_cp")
    v = {k: (0.0 if k.endswith(("deltar", "deltai")) else x) for k, x in meta["variables"].items()}
    assert np.max(np.abs(m.pdf(g["fields_data"], v) / g["f_data"] - 1)) > 1e-3

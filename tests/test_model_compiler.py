"""Model compiler against the reference: parameter names and order, chain
order, LS lists and CG matrices recorded from the reference package."""
import numpy as np
import pytest

from common import load_golden, load_model

CASES = ["d2kpipi", "d2kpipi_float", "lc2pkpi", "toy_vvp", "b2dstkpi", "d2kpipi_shapes",
         "dp2kpipi_ident", "ident_fermions", "epem_cp", "lc2pkpi_cc", "b2dstkpi_cc",
         "lc2pkpi_pol", "epem_pol", "ident3_fermions", "lc2pkpi_cp"]


@pytest.mark.parametrize("name", CASES)
def test_params_chains_ls_cg(name):
    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    assert vm.trainable_vars == meta["trainable"]
    assert list(vm.variables.keys()) == list(meta["variables"].keys())
    assert [str(c) for c in dc.decay_group] == meta["chains"]
    for c, ls_ref, cg_ref in zip(dc.decay_group, meta["ls"], meta["cg"]):
        for d, l1, c1 in zip(c, ls_ref, cg_ref):
            assert [list(x) for x in d.get_ls_list()] == l1
            np.testing.assert_allclose(d.cg(), np.array(c1), atol=1e-14)


def test_cg_against_sympy():
    from sympy import Rational
    from sympy.physics.quantum.cg import CG

    from tf_pwa_b200.particles import clebsch_gordan, spin_range, two

    for j1 in (0, 0.5, 1, 1.5, 2):
        for j2 in (0, 0.5, 1, 1.5):
            for j in spin_range(abs(j1 - j2), j1 + j2):
                for m1 in spin_range(-j1, j1):
                    for m2 in spin_range(-j2, j2):
                        if abs(m1 + m2) > j:
                            continue
                        r = lambda x: Rational(two(x), 2)  # noqa: E731
                        ref = float(CG(r(j1), r(m1), r(j2), r(m2), r(j), r(m1 + m2)).doit().evalf())
                        assert abs(clebsch_gordan(j1, m1, j2, m2, j, m1 + m2) - ref) < 1e-14


def test_bprime_coefficients():
    from tf_pwa_b200.particles import bprime_coeff

    assert bprime_coeff(2) == [1.0, 3.0, 9.0]
    assert bprime_coeff(5) == [1.0, 15.0, 315.0, 6300.0, 99225.0, 893025.0]


def test_unsupported_options_raise():
    """Options the engine does not compile fail loudly instead of being
    ignored: other decay_chain options, non-default kinematics options,
    unknown lineshape models."""
    import os

    from common import CONFIGS
    from tf_pwa_b200.codegen import ModelCode
    from tf_pwa_b200.decay_config import DecayConfig, load_yaml
    from tf_pwa_b200.plan import Plan

    dic = load_yaml(os.path.join(CONFIGS, "d2kpipi.yml"))
    dic["decay_chain"] = {"$all": {"aligned": True}}
    with pytest.raises(NotImplementedError):
        DecayConfig(dic)
    dic = load_yaml(os.path.join(CONFIGS, "d2kpipi.yml"))
    dic["data"]["align_ref"] = "center_mass"
    with pytest.raises(NotImplementedError):
        DecayConfig(dic)
    dic = load_yaml(os.path.join(CONFIGS, "d2kpipi.yml"))
    dic["particle"]["R1"]["model"] = "Flatte"
    dc = DecayConfig(dic)
    with pytest.raises(NotImplementedError):
        ModelCode(dc.decay_group, Plan(dc.decay_group))


@pytest.mark.parametrize("cfg", ["lc2pkpi_cp.yml", "lc2pkpi_pol.yml", "d2kpipi_shapes.yml",
                                 "lc2pkpi_cc.yml"])
def test_plan_accumulator_count(cfg):
    """The accumulator count the engine hands the native plan (1 + 2*ncol +
    nshape argument) equals the generated source's PWA_NACC, charge -1 and
    polarisation sums included."""
    import re

    from tf_pwa_b200.engine import Engine

    dc, vm, plan = load_model(cfg)
    eng = Engine(dc.decay_group, plan, vm, compile=False)
    c = eng.code
    nacc = int(re.search(r"#define PWA_NACC (\d+)", eng.src).group(1))
    assert nacc == 1 + 2 * c.ncol + c.nshape + c.nrho + c.ncp
    if cfg == "lc2pkpi_cp.yml":
        assert c.ncp > 0


def test_small_d_weights_match_reference_table():
    """The Wigner small-d coefficient tables (spinor-polynomial derivation)
    equal the reference's own tables (tests/golden/small_d.json, recorded
    from tf_pwa.dfun.small_d_weight) for 2j = 0 .. 10, and the matrices
    they give are orthogonal with d(0) = 1 and d^{1/2}(b) the rotation by
    b/2."""
    import json
    import os

    from common import GOLDEN
    from oracle.pwa_oracle import d_weight
    from tf_pwa_b200.particles import small_d_weight

    with open(os.path.join(GOLDEN, "small_d.json")) as f:
        ref = json.load(f)
    for j2s, table in ref.items():
        j2 = int(j2s)
        w = small_d_weight(j2)
        t = np.array(table)
        np.testing.assert_allclose(w, t, rtol=1e-14, atol=1e-14 * max(1.0, np.abs(t).max()))
        # the oracle's table (Wigner's explicit sum) as well
        np.testing.assert_allclose(d_weight(j2), t, rtol=1e-14,
                                   atol=1e-14 * max(1.0, np.abs(t).max()))
        for beta in (0.0, 0.37, 1.9, 3.0):
            x, y = np.sin(beta / 2), np.cos(beta / 2)
            powers = np.array([x ** l * y ** (j2 - l) for l in range(j2 + 1)])
            d = np.einsum("l,lab->ab", powers, w)
            np.testing.assert_allclose(d @ d.T, np.eye(j2 + 1), atol=1e-12)
            if beta == 0.0:
                np.testing.assert_allclose(d, np.eye(j2 + 1), atol=1e-15)
            if j2 == 1:
                # rows/columns m = -1/2, +1/2: d_{1/2,-1/2} = -sin(b/2)
                np.testing.assert_allclose(d, [[y, x], [-x, y]], atol=1e-15)

"""The native host program (pwa_hostprog_*) against the engine's Python host
code, on the host alone (no device): the constant block, the Jacobian of the
column couplings with every mass and width trainable (with the charge -1
couplings of CP-violating totals and the density matrix of a polarised
parent), the piece vector of the chain rule, the columns'
barrier-normalisation products, the cache of the shape part, and malformed
programs.

The Python host code is the one the parity tests pin against the oracle
(test_oracle_golden.py, test_gpu_parity.py); here the native restatement is
held to it: constants to 1e-12 relative (complex-step derivatives and the C
library's pow / sqrt round differently from numpy's in the last bits), the
Jacobian and the pieces to 1e-12 of their largest entry."""
import numpy as np
import pytest

from common import load_golden, load_model

CASES = ["d2kpipi", "d2kpipi_float", "d2kpipi_shapes", "lc2pkpi", "lc2pkpi_cc", "b2dstkpi",
         "b2dstkpi_cc", "toy_vvp", "dp2kpipi_ident", "ident_fermions", "ident3_fermions",
         "lc2pkpi_pol", "lc2pkpi_cp", "epem_pol", "epem_cp"]


def _setup(name):
    from tf_pwa_b200.engine import Engine

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])
    eng = Engine(dc.decay_group, plan, vm, compile=False)
    names = list(vm.variables)
    mw = [n for n in names if n.endswith(("_mass", "_width"))]
    train = list(vm.trainable_vars) + [n for n in mw if n not in vm.trainable_vars]
    return eng, vm, names, train


def _shifted(vm, f_m=1.004, f_g=1.07):
    v = dict(vm.get_all_dic())
    for n in v:
        if n.endswith("_mass"):
            v[n] *= f_m
        elif n.endswith("_width"):
            v[n] *= f_g
    return v


def _close(a, b, rtol):
    a, b = np.asarray(a), np.asarray(b)
    np.testing.assert_allclose(a, b, rtol=rtol, atol=rtol * max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", CASES)
def test_consts_and_jacobian_match_python(name):
    eng, vm, names, train = _setup(name)
    hp = eng.host_program(names, train)
    for vals in (vm.get_all_dic(), _shifted(vm), vm.get_all_dic()):
        v = np.array([vals[k] for k in names])
        C_py = eng.consts(vals)
        C_nat = hp.consts(v)
        np.testing.assert_allclose(C_nat, C_py, rtol=1e-12, atol=0)
        J_py, D_py = eng.jacobian(vals, train)
        J_nat, D_nat, Jm_nat = hp.jacobian(v)
        _close(J_nat, J_py, 1e-12)
        ns = eng.code.nshape + eng.code.nrho
        np.testing.assert_allclose(D_nat[:, :ns], D_py[:, :ns], rtol=1e-15, atol=0)
        assert not np.any(D_nat[:, ns:])  # the charge -1 sums enter through Jm
        if eng.code.cp_cols:
            _close(Jm_nat, eng._Jm, 1e-12)
        else:
            assert Jm_nat.size == 0


@pytest.mark.parametrize("name", CASES)
def test_pieces_match_python_chain_rule(name):
    eng, vm, names, train = _setup(name)
    hp = eng.host_program(names, train)
    rng = np.random.default_rng(7)
    vals = _shifted(vm)
    v = np.array([vals[k] for k in names])
    nacc = eng.code.nacc
    sd, sm = rng.normal(size=nacc), rng.normal(size=nacc)
    sm[0] = abs(sm[0]) + 1.0
    C = eng.consts(vals)
    J, D = eng.jacobian(vals, train)
    f, sw = 0.37, 1234.5
    ref = np.concatenate([[sd[0], sm[0] * f, sw], eng.grad_from_sums(J, D, sd),
                          eng.grad_from_sums(J, D, sm) * f])
    _close(hp.pieces(v, sd, sm, sw, f), ref, 1e-12)
    del C


@pytest.mark.parametrize("name", ["d2kpipi_float", "d2kpipi_shapes", "lc2pkpi", "b2dstkpi"])
def test_column_rho_matches_python(name):
    from tf_pwa_b200.engine import PWAError

    eng, vm, names, train = _setup(name)
    hp = eng.host_program(names, train)
    for vals in (vm.get_all_dic(), _shifted(vm)):
        C = eng.consts(vals)
        try:
            ref = eng._column_rho(C)
        except PWAError:
            with pytest.raises(PWAError, match="non-positive"):
                hp.column_rho(C)
            continue
        np.testing.assert_allclose(hp.column_rho(C), ref, rtol=1e-13)


def test_shape_part_follows_the_masses():
    """The shape part is cached per mass/width setting: a changed width or
    mass gives the constants of the new setting, the old setting its own
    again, and coupling-only changes keep it."""
    eng, vm, names, train = _setup("d2kpipi_float")
    hp = eng.host_program(names, train)
    base = vm.get_all_dic()
    pts = [base, _shifted(vm), _shifted(vm, 0.997, 0.9), base]
    coupling = next(n for n in names if n.endswith("r") and "_total_" in n)
    for vals in pts + [dict(base, **{coupling: base[coupling] * 1.3})]:
        v = np.array([vals[k] for k in names])
        np.testing.assert_allclose(hp.consts(v), eng.consts(vals), rtol=1e-12, atol=0)


def test_below_threshold_resonance_mass():
    """A resonance mass below its decay threshold: the BWR q0 is clamped
    (useq = 0) and the vertex barrier constants take |q0^2|; native and
    Python agree there too."""
    eng, vm, names, train = _setup("d2kpipi_float")
    hp = eng.host_program(names, train)
    vals = vm.get_all_dic()
    m = next(n for n in names if n.endswith("_mass"))
    vals[m] = 0.5  # below K pi / pi pi thresholds of the resonances of this model
    v = np.array([vals[k] for k in names])
    np.testing.assert_allclose(hp.consts(v), eng.consts(vals), rtol=1e-12, atol=0)
    J_py, _ = eng.jacobian(vals, train)
    J_nat, _, _ = hp.jacobian(v)
    _close(J_nat, J_py, 1e-12)


def test_trainable_without_a_role():
    from tf_pwa_b200.engine import PWAError

    eng, vm, names, train = _setup("d2kpipi")
    with pytest.raises(PWAError, match="no role"):
        eng.host_program(names, train + ["not_a_variable"])


def test_malformed_programs_are_rejected():
    from tf_pwa_b200.engine import HostProgram, PWAError

    eng, vm, names, train = _setup("lc2pkpi")
    ip, dp = eng.host_program_arrays(names, train)
    sizes = (eng.code.ncol, len(eng.code.consts), eng.code.nshape, len(train))
    HostProgram(ip, dp, *sizes).close()
    with pytest.raises(PWAError, match="truncated|trailing"):
        HostProgram(ip[:-5], dp, *sizes)
    with pytest.raises(PWAError, match="truncated|trailing"):
        HostProgram(ip, dp[:-1], *sizes)
    with pytest.raises(PWAError, match="trailing"):
        HostProgram(np.append(ip, 0), dp, *sizes)
    bad = ip.copy()
    bad[1] = 1  # the layout before polarisation and CP sections
    with pytest.raises(PWAError, match="magic or version"):
        HostProgram(bad, dp, *sizes)
    # a coupling's variable index past the variables
    bad = ip.copy()
    bad[9] = len(names)
    with pytest.raises(PWAError, match="coupling index"):
        HostProgram(bad, dp, *sizes)
    # a constant-block slot past the block (first vertex coupling's re slot)
    ncoup, nfac, K = ip[7], ip[8], ip[2]
    o = 9 + 3 * ncoup + K * nfac + len(train)
    assert ip[o] > 0
    bad = ip.copy()
    bad[o + 2] = len(eng.code.consts)
    with pytest.raises(PWAError, match="vertex coupling slot"):
        HostProgram(bad, dp, *sizes)
    # a list count larger than the program itself is refused before anything
    # of that size is allocated
    bad = ip.copy()
    bad[o] = 1 << 20
    with pytest.raises(PWAError, match="truncated"):
        HostProgram(bad, dp, *sizes)

"""The generated model code, compiled for the host with g++ (the same text
the library hands to NVRTC, after host stand-ins of the CUDA built-ins), run
event by event on the golden events, against the reference's numbers.

This checks the code generator's arithmetic without a GPU, at the
tolerances the GPU parity tests use:

* sum |A|^2 per event from ``model_amp`` vs the reference's |A|^2 (1e-10;
  2e-4 in the FP32 form);
* the plain kernel's per-event loop (forward, clip_log / MC weight,
  adjoint with and without the half-angle stash) summed on the host and fed
  to the engine's host-side chain rule: NLL within 1e-9 relative and
  gradient within 1e-7 relative of the reference's GradientTape values; the
  FP32 form of the same loop within |dNLL| < 1e-3 and 1e-4 of the largest
  gradient component;
* ``model_columns``: sum_k c_k F_k reproduces the amplitude (1e-12);
* ``model_kin``: momenta -> fields equal the reference's cal_angle fields
  (1e-11 absolute);
* ``model_genbod`` + Philox: momenta, phase-space weights and acceptance
  uniforms equal the generator oracle's; sum |A|^2 of the generated events
  equals the amplitude oracle's (1e-10).
"""
import numpy as np
import pytest

from common import golden_data, load_golden, load_model
from hostexec import HostModel

CASES = ["d2kpipi", "d2kpipi_float", "lc2pkpi", "toy_vvp", "b2dstkpi", "d2kpipi_shapes",
         "dp2kpipi_ident", "ident_fermions", "epem_cp", "lc2pkpi_cc", "b2dstkpi_cc",
         "lc2pkpi_pol", "epem_pol", "ident3_fermions", "lc2pkpi_pol_lab",
         "lc2pkpi_cp"]

_CACHE = {}


@pytest.fixture(scope="module")
def build_dir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("hostexec"))


def _setup(name, build_dir):
    if name in _CACHE:
        return _CACHE[name]
    from tf_pwa_b200.engine import Engine

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])
    eng = Engine(dc.decay_group, plan, vm, compile=False)
    hm = HostModel(eng.code, build_dir)
    _CACHE[name] = (eng, hm, g, meta, dc, plan)
    return _CACHE[name]


@pytest.mark.parametrize("name", CASES)
def test_pdf_matches_reference(name, build_dir):
    eng, hm, g, meta, _, _ = _setup(name, build_dir)
    C = eng.consts(meta["variables"])
    for kind in ("data", "mc"):
        np.testing.assert_allclose(hm.pdf(C, g["fields_" + kind]), g["f_" + kind], rtol=1e-10)
        np.testing.assert_allclose(hm.pdf(C, g["fields_" + kind], f32=True), g["f_" + kind],
                                   rtol=2e-4)


@pytest.mark.parametrize("stash", [False, True])
@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("name", CASES)
def test_kernel_loop_nll_grad(name, f32, stash, build_dir):
    from tf_pwa_b200.engine import MIXED_F32, PLAIN_F64

    eng, hm, g, meta, _, _ = _setup(name, build_dir)
    x, w = golden_data(g, meta)
    xm = g["fields_mc"]
    xall = np.concatenate([x, xm], 1)
    wall = np.concatenate([w, np.ones(xm.shape[1]) / xm.shape[1]])
    n_data = x.shape[1]
    eng._sw = float(w.sum())
    eng.eval_sums = lambda C, precision=PLAIN_F64, mc=True, stream=None: hm.sums(
        C, xall, wall, n_data, f32=precision == MIXED_F32, stash=stash)
    prec = MIXED_F32 if f32 else PLAIN_F64
    nll, grad = eng.nll_grad(meta["variables"], meta["trainable"], prec)
    scale = np.abs(g["grad"]).max()
    if f32:
        assert abs(nll - g["nll"]) < 1e-3
        assert np.max(np.abs(grad - g["grad"])) <= 1e-4 * scale
    else:
        assert abs(nll - g["nll"]) <= 1e-9 * abs(g["nll"]), (nll, g["nll"])
        np.testing.assert_allclose(grad, g["grad"], rtol=1e-7, atol=1e-7 * scale)


@pytest.mark.parametrize("name", CASES)
def test_columns_rebuild_amplitude(name, build_dir):
    eng, hm, g, meta, _, plan = _setup(name, build_dir)
    C = eng.consts(meta["variables"])
    x = g["fields_data"][:, :200]
    A = hm.amp(C, x)
    F = hm.columns(C, x)
    ck = np.tile(eng._ck, (x.shape[1], 1))
    if eng.code.ncp:  # CP-violating totals: charge -1 events take c_k^-
        minus = x[plan.charge_index] < 0
        ck[np.ix_(minus, eng._cp_cols)] = eng._ck_m[eng._cp_cols]
    A2 = np.einsum("nk,nko->no", ck, F)
    np.testing.assert_allclose(A2, A, rtol=1e-12, atol=1e-12 * np.abs(A).max())


@pytest.mark.parametrize("name", ["d2kpipi", "lc2pkpi", "toy_vvp", "b2dstkpi", "dp2kpipi_ident",
                                  "ident_fermions", "epem_cp", "lc2pkpi_pol_lab"])
def test_kinematics_match_reference(name, build_dir):
    eng, hm, g, meta, _, _ = _setup(name, build_dir)
    for kind in ("data", "mc"):
        np.testing.assert_allclose(hm.kin(g["p4_" + kind]), g["fields_" + kind], rtol=0,
                                   atol=1e-11)


@pytest.mark.parametrize("name", ["lc2pkpi", "b2dstkpi", "ident_fermions", "epem_cp"])
def test_generator_matches_oracle(name, build_dir):
    from oracle.pwa_oracle import OracleModel
    from oracle.toy_oracle import genbod_levels, uniforms
    from tf_pwa_b200.kinematics import event_fields, p4_dict

    eng, hm, g, meta, dc, plan = _setup(name, build_dir)
    if not hm.has_toy:
        pytest.skip("model without a phase-space generator")
    kin = eng.code.kin
    seed, first, n = 1234567, 5000, 2000
    t = hm.toy(eng.consts(meta["variables"]), seed, first, n)
    ndraw = sum(3 * len(b) - 4 for _, b in kin.levels) + 2
    U = uniforms(seed, np.arange(first, first + n), ndraw)
    p, wps = genbod_levels(U, kin.levels, kin.nfin)
    np.testing.assert_array_equal(t["u_ps"], U[ndraw - 2])
    np.testing.assert_array_equal(t["u_amp"], U[ndraw - 1])
    np.testing.assert_allclose(t["wps"], wps, rtol=1e-12)
    np.testing.assert_allclose(t["p4"], np.transpose(p, (2, 0, 1)), rtol=0, atol=1e-13)
    x_ref = event_fields(plan, p4_dict(t["p4"], plan.order)).numpy()
    np.testing.assert_allclose(t["fields"], x_ref, rtol=0, atol=1e-11)
    f_ref = OracleModel(dc.decay_group, plan).pdf(x_ref, meta["variables"])
    np.testing.assert_allclose(t["f"], f_ref, rtol=1e-10)


@pytest.mark.parametrize("name", ["d2kpipi", "d2kpipi_float", "d2kpipi_shapes", "dp2kpipi_ident"])
def test_hessian_from_kernel_loop(name, build_dir):
    """Differenced adjoint gradients of the host-run kernel loop against the
    reference's nested-tape Hessian (same tolerance as the GPU test)."""
    from tf_pwa_b200.api import hessian_from_gradient
    from tf_pwa_b200.engine import PLAIN_F64

    eng, hm, g, meta, _, _ = _setup(name, build_dir)
    x, w = golden_data(g, meta)
    xm = g["fields_mc"]
    xall = np.concatenate([x, xm], 1)
    wall = np.concatenate([w, np.ones(xm.shape[1]) / xm.shape[1]])
    eng._sw = float(w.sum())
    eng.eval_sums = lambda C, precision=PLAIN_F64, mc=True, stream=None: hm.sums(
        C, xall, wall, x.shape[1])
    names = meta["trainable"]
    base = dict(meta["variables"])

    def nll_grad(p):
        v = dict(base)
        v.update(zip(names, p))
        return eng.nll_grad(v, names, PLAIN_F64)

    nll, grad, H = hessian_from_gradient(nll_grad, [base[k] for k in names], 1e-4)
    assert abs(nll - g["hess_nll"]) <= 1e-9 * abs(g["hess_nll"])
    Href = g["hess"]
    np.testing.assert_allclose(H, Href, rtol=2e-5, atol=2e-5 * np.abs(Href).max())

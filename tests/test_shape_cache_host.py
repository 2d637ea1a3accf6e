"""The floating-shape column cache, checked on the host with the generated
code compiled by g++ (tests/hostexec.py):

* factorisation: with the shape-free columns Fhat of model_columns_ns built
  at one shape setting, the lineshapes of model_shapes at another, and the
  columns' barrier-normalisation ratios r_k (Engine._column_rho),
  A_o = sum_k c_k r_k BW_ch(k) Fhat_k,o equals model_amp's amplitude at the
  second setting (1e-12);
* the evaluation kernel's sums, restated in numpy from those pieces (the
  same formulas as pwa_eval_shapecache), equal the plain kernel's per-event
  loop (hx_sums) at the second setting: NLL term, column sums and lineshape
  sums to 1e-10 of their largest entry.
"""
import numpy as np
import pytest

from common import golden_data, load_golden, load_model
from hostexec import HostModel

CASES = ["d2kpipi_float", "d2kpipi_shapes", "lc2pkpi", "b2dstkpi", "lc2pkpi_cc"]


@pytest.fixture(scope="module")
def build_dir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("hostexec_sc"))


def _shifted(vals):
    """The same parameters with every resonance mass +0.5 % and width +8 %."""
    v = dict(vals)
    for n in list(v):
        if n.endswith("_mass"):
            v[n] = v[n] * 1.005
        elif n.endswith("_width"):
            v[n] = v[n] * 1.08
    return v


def _pieces(name, build_dir):
    from tf_pwa_b200.engine import Engine

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])
    eng = Engine(dc.decay_group, plan, vm, compile=False)
    assert eng.code.shape_cache_ok
    hm = HostModel(eng.code, build_dir)
    return eng, hm, g, meta, plan, dict(vm.get_all_dic())


def _amp_from_cache(eng, hm, x, C_cache, C_new):
    Fhat = hm.columns_ns(C_cache, x)
    BW, DM, DG = hm.shapes(C_new, x)
    ratio = eng._column_rho(C_new) / eng._column_rho(C_cache)
    chain = np.array([ci for ci, _ in eng.code.columns])
    ck = np.array([C_new[2 * k] + 1j * C_new[2 * k + 1] for k in range(eng.code.ncol)])
    S = ratio[None, :] * BW[:, chain]                      # (n, K)
    A = np.einsum("k,nk,nko->no", ck, S, Fhat)
    return A, Fhat, S, ck, DM, DG


@pytest.mark.parametrize("name", CASES)
def test_shape_free_columns_factorise(name, build_dir):
    eng, hm, g, meta, plan, vals = _pieces(name, build_dir)
    x = g["fields_data"][:, :300]
    C0 = eng.consts(vals)
    C1 = eng.consts(_shifted(vals))
    try:
        A, *_ = _amp_from_cache(eng, hm, x, C0, C1)
    except Exception as e:  # a barrier normalisation <= 0: the engine recomputes
        assert "barrier normalisation" in str(e)
        pytest.skip(str(e))
    A_ref = hm.amp(C1, x)
    np.testing.assert_allclose(A, A_ref, rtol=0, atol=1e-12 * np.abs(A_ref).max())


@pytest.mark.parametrize("name", CASES)
def test_shape_cache_sums_equal_plain_loop(name, build_dir):
    """pwa_eval_shapecache's per-event formulas in numpy against the plain
    kernel's loop on the host, data and MC, at a shifted shape setting."""
    from oracle.pwa_oracle import clip_log

    eng, hm, g, meta, plan, vals = _pieces(name, build_dir)
    x_d, w_d = golden_data(g, meta)
    x_m = g["fields_mc"]
    w_m = np.ones(x_m.shape[1]) / x_m.shape[1]
    C0 = eng.consts(vals)
    C1 = eng.consts(_shifted(vals))
    try:
        eng._column_rho(C0), eng._column_rho(C1)
    except Exception as e:
        pytest.skip(str(e))
    code = eng.code
    K, nsr = code.ncol, len(code.shape_res)
    chain = np.array([ci for ci, _ in code.columns])
    in_chain = np.array([[p in c.inner for c in code.group] for p in code.shape_res],
                        bool).reshape(nsr, len(code.group))
    out = []
    for x, w, data in ((x_d, w_d, True), (x_m, w_m, False)):
        A, Fhat, S, ck, DM, DG = _amp_from_cache(eng, hm, x, C0, C1)
        f = np.sum(np.abs(A) ** 2, 1)
        if data:
            s0 = np.sum(w * clip_log(f))
            eps = 1e-6
            fac = w * np.where(f > eps, 1.0 / np.where(f > eps, f, 1.0), 1.0 / eps - (f - eps) / eps ** 2)
        else:
            s0 = np.sum(w * f)
            fac = w
        h = np.einsum("no,nko->nk", np.conj(A), Fhat)
        gk = fac[:, None] * S * h                          # (n, K)
        acc = np.zeros(code.nacc)
        acc[0] = s0
        G = gk.sum(0)
        acc[1:1 + 2 * K:2], acc[2:2 + 2 * K:2] = G.real, G.imag
        cg = ck[None, :] * gk
        for q in range(nsr):
            SR = cg[:, in_chain[q][chain]].sum(1)
            acc[1 + 2 * K + 2 * q] = np.sum(2.0 * (SR * DM[:, q]).real)
            acc[2 + 2 * K + 2 * q] = np.sum(2.0 * (SR * DG[:, q]).real)
        out.append(acc)
    x = np.concatenate([x_d, x_m], 1)
    w = np.concatenate([w_d, w_m])
    sd, sm = hm.sums(C1, x, w, x_d.shape[1])
    for mine, ref in ((out[0], sd), (out[1], sm)):
        n = 1 + 2 * K + 2 * nsr
        np.testing.assert_allclose(mine[:n], ref[:n], rtol=0, atol=1e-10 * np.abs(ref[:n]).max())

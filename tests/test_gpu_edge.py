"""Edge cases of the GPU paths (through the C ABI), against the FP64 oracle:
single events, ragged tile counts (1, 127, 128, 129 data events in the
column cache), and the error codes of calls made out of order or with bad
sizes (rejected on the host before any launch)."""
import ctypes

import numpy as np
import pytest

from common import golden_data, load_golden, load_model

pytestmark = pytest.mark.gpu


def _oracle_nll(dc, plan, vals, xd, wd, xm):
    from oracle.pwa_oracle import OracleModel, nll_value

    m = OracleModel(dc.decay_group, plan)
    fd = m.pdf(xd, vals)
    fm = m.pdf(xm, vals)
    return nll_value(fd, wd, fm, np.ones(xm.shape[1]) / xm.shape[1])


@pytest.mark.parametrize("nd,nm", [(1, 1), (1, 300), (127, 129), (128, 128), (129, 1)])
def test_small_and_ragged_sets(nd, nm):
    from tf_pwa_b200.api import FCN, EventData
    from tf_pwa_b200.engine import PLAIN_F64, Engine

    g, meta = load_golden("lc2pkpi")
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])
    vals = meta["variables"]
    xd = g["fields_data"][:, :nd]
    xm = g["fields_mc"][:, :nm]
    wd = np.ones(nd)
    ref = _oracle_nll(dc, plan, vals, xd, wd, xm)
    eng = Engine(dc.decay_group, plan, vm)
    eng.upload(xd, wd, xm, np.ones(nm))
    nll, _ = eng.nll_grad(vals, meta["trainable"], PLAIN_F64)
    assert abs(nll - ref) <= 1e-10 * max(abs(ref), 1.0), (nll, ref)
    eng.close()

    class _Cfg:
        pass

    cfg = _Cfg()
    cfg.vm, cfg.decay_group, cfg.plan = vm, dc.decay_group, plan
    fcn = FCN(cfg, EventData(xd, wd), EventData(xm), precision="mixed")
    assert fcn.use_gram
    for var in (0, 1, 2, 3, 4, 5):
        fcn.eng.set_cached_variant(var)
        nll_m, _ = fcn.nll_grad()
        assert abs(nll_m - ref) <= 1e-6 * max(abs(ref), 1.0), (var, nll_m, ref)
    fcn.eng.close()


def test_error_codes_before_launch():
    from tf_pwa_b200.engine import Engine, load_library

    ARG, STATE, OOM = 1, 4, 5  # PWA_ERR_* of include/pwa_b200.h
    lib = load_library()
    g, meta = load_golden("d2kpipi")
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])
    eng = Engine(dc.decay_group, plan, vm)
    h = eng.h
    C = np.ascontiguousarray(eng.consts(meta["variables"]))
    cp = C.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    out = np.zeros(2 * eng.code.nacc)
    op = out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    # nothing uploaded yet
    assert lib.pwa_eval(h, cp, 0, 1, None, op) == STATE
    assert lib.pwa_eval_cached_enqueue(h, cp, None) == STATE
    assert lib.pwa_set_cached_variant(h, 7) == ARG
    # uploads with bad sizes
    assert lib.pwa_upload_events(h, None, None, None, 0, 0, 0, None) == ARG
    x, w = golden_data(g, meta)
    eng.upload(x, w, g["fields_mc"], np.ones(g["fields_mc"].shape[1]))
    assert lib.pwa_eval(h, cp, 5, 1, None, op) == ARG  # unknown precision
    # pool before reservation, fill of an unallocated run
    a, b = ctypes.c_longlong(), ctypes.c_longlong()
    assert lib.pwa_pool_alloc(h, 10, ctypes.byref(a), ctypes.byref(b)) == STATE
    eng.pool_reserve(4)
    assert lib.pwa_pool_alloc(h, 10 ** 6, ctypes.byref(a), ctypes.byref(b)) == OOM
    assert lib.pwa_pool_fill(h, 2, cp, None, None, None, 10, 10, None) == ARG
    # dataset-step calls: empty and inconsistent sizes
    assert lib.pwa_toy_select(h, cp, 1, 0, 0, 0.0, 0, None, None) == 0
    assert lib.pwa_fields_from_p4(h, None, 5, 4, None, 5, None) == ARG
    # server needs a parameter layout and a Gram matrix
    srv = ctypes.c_void_p()
    base = np.zeros(len(vm.variables))
    assert lib.pwa_server_create(h, base.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cp,
                                 4, 1e-3, 10, ctypes.byref(srv)) == STATE
    assert lib.pwa_last_error(h)
    eng.close()

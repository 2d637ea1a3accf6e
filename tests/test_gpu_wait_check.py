"""Failure detection of the cached evaluation without a GPU fault.

A one-block kernel arms a barrier for bytes that no copy brings; its wait
gives up after a few polls, it drains the one bulk copy it did issue and
publishes the error flag: the host must get PWA_ERR_CUDA ("a barrier wait
timed out").  With nothing launched at all, the host's poll of the mapped
result must give up after its (shortened) limit: PWA_ERR_CUDA ("stale
result").  After either, the plan evaluates the NLL and gradient exactly
as before."""
import time

import numpy as np
import pytest

from common import golden_data, load_golden, load_model

pytestmark = pytest.mark.gpu

CUDA_ERR = 3  # PWA_ERR_CUDA


def test_bounded_waits_report_and_recover():
    from tf_pwa_b200.api import FCN, EventData
    from tf_pwa_b200.engine import load_library

    g, meta = load_golden("lc2pkpi")
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])

    class _Cfg:
        pass

    cfg = _Cfg()
    cfg.vm, cfg.decay_group, cfg.plan = vm, dc.decay_group, plan
    x, w = golden_data(g, meta)
    fcn = FCN(cfg, EventData(x, w), EventData(g["fields_mc"]), precision="mixed")
    vals = [vm.variables[k] for k in fcn._var_names]
    ref = fcn.eng.nll_grad_cached(vals)
    lib = load_library()
    h = fcn.eng.h

    rc = lib.pwa_wait_check(h, 0, 2000, 1.0, None)
    assert rc == CUDA_ERR
    assert "timed out" in lib.pwa_last_error(h).decode()
    n1, g1 = fcn.eng.nll_grad_cached(vals)
    assert n1 == ref[0] and np.array_equal(g1, ref[1])

    t0 = time.perf_counter()
    rc = lib.pwa_wait_check(h, 1, 1, 0.05, None)
    dt = time.perf_counter() - t0
    assert rc == CUDA_ERR
    assert "stale" in lib.pwa_last_error(h).decode()
    assert 0.05 <= dt < 1.0, dt
    n2, g2 = fcn.eng.nll_grad_cached(vals)
    assert n2 == ref[0] and np.array_equal(g2, ref[1])
    fcn.eng.close()

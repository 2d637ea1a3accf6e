"""The allocation-free entry point ``pwa_eval_noalloc``.

Some callers cannot call cudaMalloc while they run -- for example a host
framework that hands out all device memory from its own arena, or a loop
that must not take the allocator's locks.  ``pwa_eval_noalloc`` evaluates
the fused FP64 kernels on events the caller already holds on the device and
writes the sums into a caller-provided device buffer, keeping its block
partials in a fixed device array inside the library instead of allocating.

This test calls it through the C ABI twice in a row and checks both results
against the regular entry point ``pwa_eval`` on the same events (relative
tolerance 1e-12: identical FP64 arithmetic, only the block split differs).
It lives in its own file, collected last, so a failure here does not hide
the other tests.
"""
import numpy as np
import pytest

from common import golden_data, load_golden, load_model

pytestmark = pytest.mark.gpu


def test_noalloc_matches_pwa_eval_twice():
    import torch

    from tf_pwa_b200.engine import PLAIN_F64, Engine, _dptr, load_library

    g, meta = load_golden("lc2pkpi")
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])
    eng = Engine(dc.decay_group, plan, vm)
    xd, wd = golden_data(g, meta)
    xmc = g["fields_mc"]
    eng.upload(xd, wd, xmc, np.ones(xmc.shape[1]))
    C = np.ascontiguousarray(eng.consts(meta["variables"]))
    ref_d, ref_m = eng.eval_sums(C, PLAIN_F64, mc=True)
    ref = np.concatenate([ref_d, ref_m])

    # caller-owned device inputs in the C-ABI layout, data rows then MC rows
    nd, nm = xd.shape[1], xmc.shape[1]
    x = np.concatenate([xd, xmc], 1)
    xm, xa = eng.split_fields(x)
    w = np.concatenate([wd, np.ones(nm) / nm])
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    txm, txa, tw = dev(xm), dev(xa), dev(w)
    out = torch.full((2 * eng.code.nacc,), np.nan, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()

    lib = load_library()
    for _ in range(2):
        rc = lib.pwa_eval_noalloc(eng.h, _dptr(C), txm.data_ptr(), txa.data_ptr(), tw.data_ptr(),
                                  nd, nm, nd + nm, out.data_ptr(), None)
        assert rc == 0, lib.pwa_last_error(eng.h).decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
        out.fill_(np.nan)
    eng.close()


def test_noalloc_rejects_bad_sizes():
    import torch

    from tf_pwa_b200.engine import Engine, _dptr, load_library

    g, meta = load_golden("d2kpipi")
    dc, vm, plan = load_model(meta["config"])
    eng = Engine(dc.decay_group, plan, vm)
    C = np.zeros(len(eng.code.consts))
    lib = load_library()
    buf = torch.zeros(4096, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    # a leading dimension below the event count is refused before any launch
    rc = lib.pwa_eval_noalloc(eng.h, _dptr(C), p, p, p, 10, 10, 5, p, None)
    assert rc != 0
    assert "leading dimension" in lib.pwa_last_error(eng.h).decode()
    eng.close()

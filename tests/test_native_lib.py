"""The C-ABI library loads on a machine without a GPU, exports every symbol
include/pwa_b200.h declares, and the generated model sources compile for
sm_100a (NVRTC, no device needed)."""
import os
import re

import numpy as np
import pytest

from common import ROOT, load_model


def _declared():
    txt = open(os.path.join(ROOT, "include", "pwa_b200.h")).read()
    return sorted(set(re.findall(r"\b(pwa_[a-z_]+)\s*\(", txt)))


def test_library_exports_header_symbols():
    from tf_pwa_b200.engine import load_library

    lib = load_library()
    for name in _declared():
        assert hasattr(lib, name), name


@pytest.mark.parametrize("cfg", ["d2kpipi.yml", "lc2pkpi.yml"])
def test_generated_model_compiles_for_sm100a(cfg):
    from tf_pwa_b200.engine import Engine

    dc, vm, plan = load_model(cfg)
    eng = Engine(dc.decay_group, plan, vm, compile=False)
    log = eng.compile_check("sm_100a")
    assert "pwa_eval_f64" in log and "pwa_eval_f32" in log


def test_read_dat_matches_numpy(tmp_path):
    """pwa_read_dat (multithreaded text ingest) returns numpy.loadtxt's
    numbers in file order, comments skipped; bad tokens are errors."""
    from tf_pwa_b200.api import load_dat_file
    from tf_pwa_b200.engine import PWAError, read_dat

    rng = np.random.default_rng(3)
    a = rng.normal(size=(300000, 4)) * np.array([1.0, 1e-3, 1e3, 1e-12])
    f = tmp_path / "p4.dat"
    with open(f, "w") as fh:
        fh.write("# E px py pz\n")
        np.savetxt(fh, a, fmt="%.17g")
    x = read_dat(str(f))
    np.testing.assert_array_equal(x, a.reshape(-1))
    np.testing.assert_array_equal(load_dat_file(str(f), 3)[:, 0, :], a[:100000 * 3:3])
    bad = tmp_path / "bad.dat"
    bad.write_text("1.0 2.0 x3\n")
    with pytest.raises(PWAError):
        read_dat(str(bad))


def test_argument_errors_without_a_device():
    """Bad arguments come back as PWA_ERR_ARG with a message, before any
    device call (so also on a machine without a GPU); calls on a null
    handle are refused."""
    import ctypes

    from tf_pwa_b200.engine import load_library

    lib = load_library()
    h = ctypes.c_void_p()
    src = b"// empty"
    # ncol = 0 is invalid
    rc = lib.pwa_plan_create(src, len(src), 1, 1, 0, 1, 0, 1, 1, 128, ctypes.byref(h))
    assert rc == 1
    assert len(lib.pwa_last_error(h)) > 0
    lib.pwa_plan_destroy(h)
    # threads per block must be a multiple of 32
    h = ctypes.c_void_p()
    rc = lib.pwa_plan_create(src, len(src), 1, 1, 1, 1, 0, 1, 1, 100, ctypes.byref(h))
    assert rc == 1
    lib.pwa_plan_destroy(h)
    # the accumulator count must equal the source's PWA_NACC (1 + 2*2 + 3 = 8)
    src = b"#define PWA_NACC 9\n"
    h = ctypes.c_void_p()
    rc = lib.pwa_plan_create(src, len(src), 1, 1, 2, 2, 3, 1, 1, 128, ctypes.byref(h))
    assert rc == 1
    assert b"PWA_NACC" in lib.pwa_last_error(h)
    lib.pwa_plan_destroy(h)
    out = (ctypes.c_double * 4)()
    assert lib.pwa_hessian_cached(None, out, 1.0, 1e-3, None, out, out, out) == 1
    assert lib.pwa_last_error(None)

"""The C-ABI library loads on a machine without a GPU, exports every symbol
include/pwa_b200.h declares, and the generated model sources compile for
sm_100a (NVRTC, no device needed)."""
import os
import re

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

"""Ahead-of-time model builds (pwa_precompile): NVRTC runs without a device
and the cubin lands in the on-disk cache that pwa_plan_create reads."""
import os

import pytest

from common import load_model


def _engine():
    from tf_pwa_b200.engine import Engine

    dc, vm, plan = load_model("d2kpipi.yml")
    return Engine(dc.decay_group, plan, vm, compile=False)


def test_precompile_stores_cubin(tmp_path, monkeypatch):
    monkeypatch.setenv("PWA_CUBIN_CACHE", str(tmp_path))
    eng = _engine()
    eng.precompile("sm_100a")
    files = [f for f in os.listdir(tmp_path) if f.endswith(".cubin")]
    assert len(files) == 1 and os.path.getsize(tmp_path / files[0]) > 0
    eng.precompile("sm_100a")  # same source: the same single entry
    assert [f for f in os.listdir(tmp_path) if f.endswith(".cubin")] == files


def test_precompile_needs_cache_dir(monkeypatch):
    from tf_pwa_b200.engine import PWAError

    eng = _engine()
    monkeypatch.setenv("PWA_CUBIN_CACHE", "")
    with pytest.raises(PWAError, match="PWA_CUBIN_CACHE"):
        eng.precompile("sm_100a")


def test_default_cache_dir_is_the_package(monkeypatch):
    from tf_pwa_b200 import engine

    monkeypatch.delenv("PWA_CUBIN_CACHE", raising=False)
    engine._default_cubin_cache()
    assert os.environ["PWA_CUBIN_CACHE"] == engine.CUBIN_DIR
    monkeypatch.setenv("PWA_CUBIN_CACHE", "/nonexistent-choice")
    engine._default_cubin_cache()  # an explicit setting is kept
    assert os.environ["PWA_CUBIN_CACHE"] == "/nonexistent-choice"


def test_floating_shapes_share_the_kernels():
    """Floating a model's masses and widths changes its trainable set, not
    its kernels: the floating-shape Lambda_c config compiles to the same
    source (and cubin) as the fixed one, so the plain and FP32 kernels'
    measured operation counts apply to both."""
    from tf_pwa_b200.engine import Engine

    srcs = []
    for cfg in ("lc2pkpi.yml", "lc2pkpi_float.yml"):
        dc, vm, plan = load_model(cfg)
        srcs.append(Engine(dc.decay_group, plan, vm, compile=False).src)
        if cfg == "lc2pkpi_float.yml":
            assert sum(n.endswith(("_mass", "_width")) for n in vm.trainable_vars) == 6
    assert srcs[0] == srcs[1]


def test_plain_kernel_occupancy_by_model_size():
    """The model source sets the plain kernels' blocks per SM: 4 for the
    Lambda_c model (23 accumulators), 3 for the four-body model (85)."""
    import re

    from tf_pwa_b200.engine import Engine

    for cfg, want in (("lc2pkpi.yml", 4), ("b2dstkpi.yml", 3)):
        dc, vm, plan = load_model(cfg)
        src = Engine(dc.decay_group, plan, vm, compile=False).src
        assert re.search(r"#define PWA_EVAL_MINB (\d+)", src).group(1) == str(want)

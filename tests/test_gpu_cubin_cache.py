"""On-disk cubin cache (PWA_CUBIN_CACHE): the first process compiles the
model with NVRTC and stores the cubin; a second process loads it from the
cache and computes the same NLL bit for bit."""
import os
import subprocess
import sys

import pytest

from common import ROOT

pytestmark = pytest.mark.gpu

SCRIPT = r"""
import sys, time
sys.path[:0] = [{root!r}, {tests!r}]
import conftest
from common import golden_data, load_golden, load_model
from tf_pwa_b200.engine import PLAIN_F64, Engine
g, meta = load_golden("d2kpipi")
dc, vm, plan = load_model(meta["config"])
vm.set_all(meta["variables"])
t = time.time()
eng = Engine(dc.decay_group, plan, vm)
dt = time.time() - t
x, w = golden_data(g, meta)
eng.upload(x, w, g["fields_mc"], [1.0] * g["fields_mc"].shape[1])
nll, _ = eng.nll_grad(meta["variables"], meta["trainable"], PLAIN_F64)
print(repr(nll), dt)
"""


def test_disk_cache_roundtrip(tmp_path):
    env = dict(os.environ, PWA_CUBIN_CACHE=str(tmp_path))
    code = SCRIPT.format(root=ROOT, tests=os.path.join(ROOT, "tests"))
    out1 = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                          timeout=600)
    assert out1.returncode == 0, out1.stderr[-2000:]
    files = [f for f in os.listdir(tmp_path) if f.endswith(".cubin")]
    assert len(files) == 1
    out2 = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                          timeout=600)
    assert out2.returncode == 0, out2.stderr[-2000:]
    nll1, _ = out1.stdout.split()[-2:]
    nll2, _ = out2.stdout.split()[-2:]
    assert nll1 == nll2

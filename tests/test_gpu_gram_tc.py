"""The MC Gram matrix on the tensor cores (tcgen05 int8 MMAs on exact slices,
int32 accumulation, FP64 recombination) against the FP64 CUDA-core Gram,
through the C ABI.

Tolerances: every entry within 1e-12 of the largest entry, and the
normalisation integral I = c^H M c within 1e-12 relative on the golden
models; at the four-body workload's own size (4e6 MC events, 30 columns)
|dI / I| <= 1e-9 (the bound under which the MC term moves the NLL of 1e6
data events by less than 1e-3).
"""
import numpy as np
import pytest

from common import load_golden, load_model

pytestmark = pytest.mark.gpu


def _grams(eng, vals):
    out = {}
    for method in (0, 1):
        eng.set_gram_method(method)
        out[method] = eng.set_gram(vals).copy()
    return out


def _integral(eng, M, vals):
    eng.consts(vals)
    c = eng._ck
    return float(np.real(np.conj(c) @ M @ c))


@pytest.mark.parametrize("name", ["d2kpipi", "lc2pkpi", "b2dstkpi", "dp2kpipi_ident",
                                  "toy_vvp"])
def test_tensor_core_gram_matches_fp64(name):
    from tf_pwa_b200.engine import Engine

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])
    vals = meta["variables"]
    eng = Engine(dc.decay_group, plan, vm)
    xm = g["fields_mc"]
    wm = np.random.default_rng(3).uniform(0.5, 1.5, xm.shape[1])  # uneven weights
    eng.upload(g["fields_data"], np.ones(g["fields_data"].shape[1]), xm, wm)
    M = _grams(eng, vals)
    scale = np.abs(M[0]).max()
    assert np.max(np.abs(M[1] - M[0])) <= 1e-12 * scale, np.max(np.abs(M[1] - M[0])) / scale
    np.testing.assert_allclose(M[1], np.conj(M[1]).T, rtol=0, atol=1e-13 * scale)  # Hermitian
    i0, i1 = _integral(eng, M[0], vals), _integral(eng, M[1], vals)
    assert abs(i1 - i0) <= 1e-12 * abs(i0)
    eng.close()


def test_tensor_core_gram_four_body_full_size():
    """B -> D* K pi, 12 resonances, 30 columns, 4e6 flat MC events."""
    import torch

    from tf_pwa_b200.engine import Engine
    from tf_pwa_b200.workload import make_dataset

    cl, data, bg, mc = make_dataset("b2dstkpi.yml", 1000, 4_000_000, seed=7)
    eng = Engine(cl.decay_group, cl.plan, cl.vm)
    c = eng.code
    x = torch.cat([data.fields, mc.fields], 1)
    xm = x[c.mass_fields].contiguous()
    xa = x[c.angle_fields].contiguous()
    w = torch.as_tensor(np.concatenate([np.ones(data.n), np.ones(mc.n) / mc.n]), device="cuda")
    eng.upload_device(xm.data_ptr(), xa.data_ptr(), w.data_ptr(), data.n, mc.n, float(data.n))
    torch.cuda.synchronize()
    vals = cl.vm.get_all_dic()
    M = _grams(eng, vals)
    i0, i1 = _integral(eng, M[0], vals), _integral(eng, M[1], vals)
    assert abs(i1 - i0) <= 1e-9 * abs(i0), (i0, i1)
    scale = np.abs(M[0]).max()
    assert np.max(np.abs(M[1] - M[0])) <= 1e-11 * scale
    eng.close()

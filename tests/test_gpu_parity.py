"""GPU parity: the CUDA engine (through the C ABI) against the reference's
golden vectors and the FP64 oracle.

Tolerances (stated by the workload definition):
  plain FP64 path: NLL within 1e-9 relative, gradient within 1e-7 relative;
  mixed path (FP32 amplitudes, FP64 sums): |dNLL| < 1e-3, gradient within
  1e-4 relative to its largest component.
"""
import numpy as np
import pytest

from common import golden_data, load_golden, load_model

pytestmark = pytest.mark.gpu

CASES = ["d2kpipi", "d2kpipi_float", "lc2pkpi", "b2dstkpi", "d2kpipi_shapes", "dp2kpipi_ident",
         "ident_fermions", "epem_cp", "toy_vvp", "ident3_fermions"]


def _engine(name):
    from tf_pwa_b200.engine import Engine

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])
    eng = Engine(dc.decay_group, plan, vm)
    x, w = golden_data(g, meta)
    eng.upload(x, w, g["fields_mc"], np.ones(g["fields_mc"].shape[1]))
    return eng, g, meta, vm


@pytest.mark.parametrize("name", CASES)
def test_plain_f64_matches_reference(name):
    from tf_pwa_b200.engine import PLAIN_F64

    eng, g, meta, vm = _engine(name)
    nll, grad = eng.nll_grad(meta["variables"], meta["trainable"], PLAIN_F64)
    assert abs(nll - g["nll"]) <= 1e-9 * abs(g["nll"]), (nll, g["nll"])
    scale = np.abs(g["grad"]).max()
    np.testing.assert_allclose(grad, g["grad"], rtol=1e-7, atol=1e-7 * scale)
    eng.close()


@pytest.mark.parametrize("name", CASES)
def test_mixed_f32_within_tolerance(name):
    from tf_pwa_b200.engine import MIXED_F32

    eng, g, meta, vm = _engine(name)
    nll, grad = eng.nll_grad(meta["variables"], meta["trainable"], MIXED_F32)
    assert abs(nll - g["nll"]) < 1e-3
    scale = np.abs(g["grad"]).max()
    assert np.max(np.abs(grad - g["grad"])) <= 1e-4 * scale
    eng.close()


@pytest.mark.parametrize("name", CASES)
def test_pdf_matches_reference(name):
    import torch

    from tf_pwa_b200.engine import MIXED_F32, PLAIN_F64

    eng, g, meta, vm = _engine(name)
    C = eng.consts(meta["variables"])
    nd = g["fields_data"].shape[1]
    out = torch.empty(nd, dtype=torch.float64, device="cuda")
    eng.pdf_device(C, 0, nd, out.data_ptr(), PLAIN_F64)
    np.testing.assert_allclose(out.cpu().numpy(), g["f_data"], rtol=1e-11)
    eng.pdf_device(C, 0, nd, out.data_ptr(), MIXED_F32)
    np.testing.assert_allclose(out.cpu().numpy(), g["f_data"], rtol=2e-4)
    eng.close()


@pytest.mark.parametrize("name", ["d2kpipi", "lc2pkpi", "b2dstkpi"])
def test_gram_mc_term(name):
    """Cached MC integral I = c^H M c and its gradient equal the direct sums."""
    from tf_pwa_b200.engine import PLAIN_F64

    eng, g, meta, vm = _engine(name)
    eng.set_gram(meta["variables"])
    nll_g, grad_g = eng.nll_grad(meta["variables"], meta["trainable"], PLAIN_F64, use_gram=True)
    nll_d, grad_d = eng.nll_grad(meta["variables"], meta["trainable"], PLAIN_F64)
    assert abs(nll_g - nll_d) <= 1e-10 * abs(nll_d)
    np.testing.assert_allclose(grad_g, grad_d, rtol=1e-9, atol=1e-9 * np.abs(grad_d).max())
    eng.close()


def test_reproducible_bitwise():
    from tf_pwa_b200.engine import PLAIN_F64

    eng, g, meta, vm = _engine("lc2pkpi")
    a = eng.nll_grad(meta["variables"], meta["trainable"], PLAIN_F64)
    b = eng.nll_grad(meta["variables"], meta["trainable"], PLAIN_F64)
    assert a[0] == b[0] and np.array_equal(a[1], b[1])
    eng.close()


@pytest.mark.parametrize("name", ["d2kpipi", "lc2pkpi", "b2dstkpi", "dp2kpipi_ident", "ident_fermions",
                                  "epem_cp"])
def test_cached_columns_fcn(name):
    """Mixed form with fixed masses/widths: FP32 column cache + FP64 Gram,
    NLL/gradient from the C-side chain rule, against the reference."""
    from tf_pwa_b200.api import FCN, EventData

    g, meta = load_golden(name)
    from common import load_model as lm

    dc, vm, plan = lm(meta["config"])
    vm.set_all(meta["variables"])

    class _Cfg:
        pass

    cfg = _Cfg()
    cfg.vm, cfg.decay_group, cfg.plan = vm, dc.decay_group, plan
    x, w = golden_data(g, meta)
    data = EventData(x, w / (w.sum() / (w * w).sum()))
    fcn = FCN(cfg, data, EventData(g["fields_mc"]), precision="mixed")
    assert fcn.use_gram
    nll, grad = fcn.nll_grad()
    assert abs(nll - g["nll"]) < 1e-5 * abs(g["nll"])
    np.testing.assert_allclose(grad, g["grad"], rtol=1e-4, atol=1e-5 * np.abs(g["grad"]).max())
    # C-side pieces recombine to the same answer
    from tf_pwa_b200.engine import combine_pieces

    v = fcn.eng.pieces_cached([vm.variables[k] for k in fcn._var_names])
    n2, g2 = combine_pieces(v, len(meta["trainable"]))
    assert n2 == pytest.approx(nll, rel=1e-14)
    fcn.eng.close()


@pytest.mark.parametrize("name", ["lc2pkpi", "b2dstkpi"])
def test_cached_kernel_variants_agree(name):
    """The six data-term kernels on the column cache (shared-memory ring,
    per-thread FP64 column sums, warp reduce-scatter of FP32 column sums,
    ring with reduce-scatter consumers, one block per SM with contiguous
    warp runs, one block per SM with a producer warp and a deep bulk-copy
    ring) give the same NLL (FP64 amplitude and log in all of them) and
    gradients that differ only by FP32 rounding of per-event / per-warp
    sums."""
    from tf_pwa_b200.api import FCN, EventData
    from common import load_model as lm

    g, meta = load_golden(name)
    dc, vm, plan = lm(meta["config"])
    vm.set_all(meta["variables"])

    class _Cfg:
        pass

    cfg = _Cfg()
    cfg.vm, cfg.decay_group, cfg.plan = vm, dc.decay_group, plan
    x, w = golden_data(g, meta)
    fcn = FCN(cfg, EventData(x, w / (w.sum() / (w * w).sum())), EventData(g["fields_mc"]),
              precision="mixed")
    vals = [vm.variables[k] for k in fcn._var_names]
    res = {}
    from tf_pwa_b200.engine import PWAError

    with pytest.raises(PWAError):  # the ring's two consumer groups need an even depth
        fcn.eng.set_cached_config(5, 3)
    for var in (0, 1, 2, 3, 4, 5):
        fcn.eng.set_cached_variant(var)
        res[var] = fcn.eng.nll_grad_cached(vals)
        # a second call reuses the ticket counters the first one reset
        n_again, g_again = fcn.eng.nll_grad_cached(vals)
        assert n_again == res[var][0] and np.array_equal(g_again, res[var][1])
    fcn.eng.close()
    n1, g1 = res[1]
    for var in (0, 2, 3, 4, 5):
        n, gr = res[var]
        assert abs(n - n1) <= 1e-12 * abs(n1)
        np.testing.assert_allclose(gr, g1, rtol=1e-5, atol=1e-6 * np.abs(g1).max())


@pytest.mark.parametrize("name", ["d2kpipi_float", "d2kpipi_shapes"])
def test_shape_cache_fcn(name):
    """Floating masses/widths in the mixed form: FCN evaluates from the
    shape-free column cache (FP32 columns, FP64 lineshapes, amplitude and
    sums).  At the golden point: NLL and gradient against the reference
    (|dNLL| < 1e-4, gradient 1e-5 of its largest entry); at a shifted shape
    setting (masses +0.5 %, widths +8 %): against the plain FP64 form."""
    import os

    from common import CONFIGS
    from tf_pwa_b200.api import FCN, ConfigLoader, EventData

    g, meta = load_golden(name)
    cl = ConfigLoader(os.path.join(CONFIGS, meta["config"]))
    cl.vm.set_all(meta["variables"])
    x, w = golden_data(g, meta)
    alpha = w.sum() / (w * w).sum()
    fm = FCN(cl, EventData(x, w / alpha), EventData(g["fields_mc"]), precision="mixed")
    fp = FCN(cl, EventData(x, w / alpha), EventData(g["fields_mc"]), precision="plain")
    assert fm.use_shape_cache and not fm.use_gram
    nll, grad = fm.nll_grad()
    scale = np.abs(g["grad"]).max()
    assert abs(nll - float(g["nll"])) < 1e-4
    np.testing.assert_allclose(grad, g["grad"], rtol=0, atol=1e-5 * scale)
    x0 = np.array(cl.vm.get_all_val())
    names = list(cl.vm.trainable_vars)
    x1 = x0.copy()
    for i, n in enumerate(names):
        if n.endswith("_mass"):
            x1[i] *= 1.005
        elif n.endswith("_width"):
            x1[i] *= 1.08
    n_m, g_m = fm.nll_grad(x1)
    n_p, g_p = fp.nll_grad(x1)
    assert abs(n_m - n_p) < 1e-4
    np.testing.assert_allclose(g_m, g_p, rtol=0, atol=1e-5 * np.abs(g_p).max())
    fm.eng.close()
    fp.eng.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["d2kpipi_float", "d2kpipi_shapes", "lc2pkpi", "b2dstkpi",
                                  "dp2kpipi_ident", "toy_vvp", "lc2pkpi_pol", "lc2pkpi_cp",
                                  "epem_pol"])
@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_native_host_matches_python_host(name, precision):
    """FCN's evaluations with the host side in native code (pwa_nll_grad_vars:
    constants, Jacobian and chain rule of the host program) against the
    engine's Python host code on the same device sums: NLL to 1e-12
    relative, gradient to 1e-10 of its largest entry, at the golden point
    and at a shifted shape setting; every mass and width trainable."""
    import os

    from common import CONFIGS
    from tf_pwa_b200.api import FCN, ConfigLoader, EventData

    g, meta = load_golden(name)
    cl = ConfigLoader(os.path.join(CONFIGS, meta["config"]))
    cl.vm.set_all(meta["variables"])
    vm = cl.vm
    for n in list(vm.variables):
        if n.endswith(("_mass", "_width")) and n not in vm.trainable_vars:
            vm.set_fix(n, unfix=True)
    x, w = golden_data(g, meta)
    alpha = w.sum() / (w * w).sum()
    f = FCN(cl, EventData(x, w / alpha), EventData(g["fields_mc"]), precision=precision,
            shape_cache=False)
    assert f.native_host and not f.use_gram
    names = list(vm.trainable_vars)
    x0 = np.array(vm.get_all_val())
    x1 = x0.copy()
    for i, n in enumerate(names):
        if n.endswith("_mass"):
            x1[i] *= 1.003
        elif n.endswith("_width"):
            x1[i] *= 1.05
    for xv in (x0, x1):
        nll, grad = f.nll_grad(xv)
        ref_n, ref_g = f.eng.nll_grad(vm.get_all_dic(), names, f.precision)
        assert abs(nll - ref_n) <= 1e-12 * abs(ref_n)
        np.testing.assert_allclose(grad, ref_g, rtol=0, atol=1e-10 * np.abs(ref_g).max())
    f.eng.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["d2kpipi_float", "d2kpipi_shapes"])
def test_native_host_shape_cache(name):
    """The floating-shape column cache through the native host side
    (pwa_pieces_vars with the shape-cache form) against the Python host
    side's shape-cache evaluation: same NLL and gradient to 1e-12 / 1e-10."""
    import os

    from common import CONFIGS
    from tf_pwa_b200.api import FCN, ConfigLoader, EventData

    g, meta = load_golden(name)
    cl = ConfigLoader(os.path.join(CONFIGS, meta["config"]))
    cl.vm.set_all(meta["variables"])
    x, w = golden_data(g, meta)
    alpha = w.sum() / (w * w).sum()
    f = FCN(cl, EventData(x, w / alpha), EventData(g["fields_mc"]), precision="mixed")
    assert f.native_host and f.use_shape_cache
    names = list(cl.vm.trainable_vars)
    x1 = np.array(cl.vm.get_all_val())
    for i, n in enumerate(names):
        if n.endswith("_mass"):
            x1[i] *= 1.005
        elif n.endswith("_width"):
            x1[i] *= 1.08
    nll, grad = f.nll_grad(x1)
    ref_n, ref_g = f.eng.nll_grad(cl.vm.get_all_dic(), names, f.precision)
    assert abs(nll - ref_n) <= 1e-12 * abs(ref_n)
    np.testing.assert_allclose(grad, ref_g, rtol=0, atol=1e-10 * np.abs(ref_g).max())
    f.eng.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n_data,n_mc", [(1, 1), (31, 33), (129, 95), (397, 1499)])
def test_shape_cache_ragged_sizes(n_data, n_mc):
    """The floating-shape evaluation at set sizes that end inside a 32-event
    segment and a 128-event tile, and a data/MC boundary inside one: NLL and
    gradient against the plain FP64 form on the same events."""
    import os

    from common import CONFIGS
    from tf_pwa_b200.api import FCN, ConfigLoader, EventData

    g, meta = load_golden("d2kpipi_float")
    cl = ConfigLoader(os.path.join(CONFIGS, meta["config"]))
    cl.vm.set_all(meta["variables"])
    xd = g["fields_data"][:, :n_data]
    xm = g["fields_mc"][:, :n_mc]
    assert xd.shape[1] == n_data and xm.shape[1] == n_mc
    fm = FCN(cl, EventData(xd), EventData(xm), precision="mixed")
    fp = FCN(cl, EventData(xd), EventData(xm), precision="plain")
    assert fm.use_shape_cache
    x1 = np.array(cl.vm.get_all_val())
    for i, n in enumerate(cl.vm.trainable_vars):
        if n.endswith(("_mass", "_width")):
            x1[i] *= 1.01
    n_m, g_m = fm.nll_grad(x1)
    n_p, g_p = fp.nll_grad(x1)
    assert abs(n_m - n_p) < 1e-6 * max(1.0, abs(n_p))
    np.testing.assert_allclose(g_m, g_p, rtol=0, atol=1e-6 * np.abs(g_p).max())
    fm.eng.close()
    fp.eng.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["lc2pkpi", "lc2pkpi_cc", "b2dstkpi", "b2dstkpi_cc", "toy_vvp"])
def test_shape_cache_models_with_floating_shapes(name):
    """Every resonance mass and width of a fixed-shape golden model set
    free: FCN's mixed form then evaluates from the floating-shape column
    cache (staged kernel, in-launch reduction, native host side); at the
    golden point and at masses +0.3 % / widths +5 %, NLL and gradient
    against the plain FP64 form on the same events (|dNLL| < 1e-4, gradient
    1e-5 of its largest entry)."""
    import os

    from common import CONFIGS
    from tf_pwa_b200.api import FCN, ConfigLoader, EventData

    g, meta = load_golden(name)
    cl = ConfigLoader(os.path.join(CONFIGS, meta["config"]))
    cl.vm.set_all(meta["variables"])
    vm = cl.vm
    for n in list(vm.variables):
        if n.endswith(("_mass", "_width")) and n not in vm.trainable_vars:
            vm.set_fix(n, unfix=True)
    x, w = golden_data(g, meta)
    alpha = w.sum() / (w * w).sum()
    fm = FCN(cl, EventData(x, w / alpha), EventData(g["fields_mc"]), precision="mixed")
    fp = FCN(cl, EventData(x, w / alpha), EventData(g["fields_mc"]), precision="plain")
    assert fm.use_shape_cache and fm.native_host and not fm.use_gram
    names = list(vm.trainable_vars)
    x0 = np.array(vm.get_all_val())
    x1 = x0.copy()
    for i, n in enumerate(names):
        if n.endswith("_mass"):
            x1[i] *= 1.003
        elif n.endswith("_width"):
            x1[i] *= 1.05
    for xv in (x0, x1):
        n_m, g_m = fm.nll_grad(xv)
        n_p, g_p = fp.nll_grad(xv)
        assert abs(n_m - n_p) < 1e-4
        np.testing.assert_allclose(g_m, g_p, rtol=0, atol=1e-5 * np.abs(g_p).max())
    fm.eng.close()
    fp.eng.close()

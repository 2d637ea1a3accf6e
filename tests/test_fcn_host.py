"""Host side of FCN.nll_grad in the cached form and with the native host
program: the parameter vector, the variable buffer handed to the library,
the trainable order of the returned gradient, the variables left in the
VarsManager and a trainable set changed after construction.  The library call is
replaced by a stand-in that reads and writes the same buffers (the device
evaluation itself is covered by the GPU tests)."""
import ctypes

import numpy as np

from common import load_golden, load_model


class _FakeCachedLib:
    """pwa_nll_grad_cached stand-in: nll = sw * sum(vars), grad_i =
    2 * vars[train_i]; everything else from the real library."""

    def __init__(self, lib, nvars, train_pos):
        self.lib, self.nvars, self.train_pos = lib, nvars, train_pos
        self.calls = 0
        self.forms = []

    def __getattr__(self, name):
        return getattr(self.lib, name)

    def pwa_nll_grad_vars(self, h, pv, form, sw, stream, pn, pg):
        self.forms.append(form)
        return self.pwa_nll_grad_cached(h, pv, sw, stream, pn, pg)

    def pwa_nll_grad_cached(self, h, pv, sw, stream, pn, pg):
        self.calls += 1
        v = np.frombuffer((ctypes.c_double * self.nvars).from_address(pv))
        g = np.frombuffer((ctypes.c_double * len(self.train_pos)).from_address(pg))
        ctypes.c_double.from_address(pn).value = sw * float(v.sum())
        g[:] = 2.0 * v[self.train_pos]
        return 0


def test_cached_call_buffers(monkeypatch):
    import tf_pwa_b200.engine as E
    from tf_pwa_b200.api import FCN

    g, meta = load_golden("lc2pkpi")
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])
    names = list(vm.variables.keys())
    train_pos = np.array([names.index(n) for n in vm.trainable_vars])

    class HostFCN(FCN):
        def __init__(self):
            self.vm, self.use_gram, self.n_call = vm, True, 0
            self.native_host = False
            self.eng = E.Engine(dc.decay_group, plan, vm, compile=False)
            self._var_names = names
            self._train = list(vm.trainable_vars)
            self.eng._sw = 3.0
            # the buffers set_param_layout allocates
            eng = self.eng
            eng._n_train = len(train_pos)
            eng._vbuf, eng._gbuf, eng._nbuf = np.zeros(len(names)), np.zeros(len(train_pos)), np.zeros(1)
            eng._vbuf_p, eng._gbuf_p, eng._nbuf_p = (eng._vbuf.ctypes.data, eng._gbuf.ctypes.data,
                                                     eng._nbuf.ctypes.data)

    fake = _FakeCachedLib(E.load_library(), len(names), train_pos)
    monkeypatch.setattr(E, "load_library", lambda path=None: fake)
    f = HostFCN()
    rng = np.random.default_rng(1)
    for x in (rng.normal(size=len(train_pos)), list(rng.normal(size=len(train_pos)))):
        nll, grad = f.nll_grad(x)
        full = np.array([vm.variables[n] for n in names])
        np.testing.assert_array_equal(full[train_pos], np.asarray(x, float))
        assert nll == 3.0 * full.sum()
        np.testing.assert_array_equal(grad, 2.0 * np.asarray(x, float))
        # the returned gradient is a copy, not the library's buffer
        grad[:] = 0.0
        assert np.all(f.eng._gbuf == 2.0 * np.asarray(x, float))
    assert fake.calls == 2
    # dict input and no input leave the values / reuse them
    nll2, _ = f.nll_grad()
    assert nll2 == nll
    f.nll_grad({vm.trainable_vars[0]: 0.5})
    assert vm.variables[vm.trainable_vars[0]] == 0.5


def test_real_library_takes_buffer_addresses():
    """The library's argument conversion accepts the buffer addresses (a
    null plan handle is refused before any memory is touched)."""
    from tf_pwa_b200.engine import load_library

    lib = load_library()
    buf = np.zeros(4)
    p = buf.ctypes.data
    assert lib.pwa_nll_grad_cached(None, p, 1.0, None, p, p) == 1


def test_native_host_call_buffers(monkeypatch):
    """FCN with the native host program (not the cached form): the full
    variable vector goes to pwa_nll_grad_vars with the FCN's form, the
    gradient comes back in trainable order, and a set_fix after
    construction re-lays the program out before the next call."""
    import tf_pwa_b200.engine as E
    from tf_pwa_b200.api import FCN

    g, meta = load_golden("d2kpipi_float")
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])
    names = list(vm.variables.keys())

    class HostFCN(FCN):
        def __init__(self):
            self.vm, self.use_gram, self.n_call = vm, False, 0
            self.precision, self.native_host, self._form = E.MIXED_F32, True, E.FORM_SHAPE_CACHE
            self.eng = E.Engine(dc.decay_group, plan, vm, compile=False)
            self.eng._sw = 2.0
            self._var_names = names
            self._train = list(vm.trainable_vars)
            self.layouts = []
            self.eng.set_host_program = self._set_hp
            self._set_hp(names, self._train)

        def _set_hp(self, var_names, train_names):
            # what Engine.set_host_program leaves behind, without a plan
            self.layouts.append(list(train_names))
            self.eng.host_program(var_names, train_names).close()
            eng = self.eng
            eng._hp_train = len(train_names)
            eng._hp_vbuf, eng._hp_gbuf, eng._hp_nbuf = (np.zeros(len(var_names)),
                                                        np.zeros(len(train_names)), np.zeros(1))
            eng._hp_ptrs = (eng._hp_vbuf.ctypes.data, eng._hp_gbuf.ctypes.data,
                            eng._hp_nbuf.ctypes.data)
            self.fake.train_pos = np.array([names.index(n) for n in train_names])

    train_pos = np.array([names.index(n) for n in vm.trainable_vars])
    fake = _FakeCachedLib(E.load_library(), len(names), train_pos)
    monkeypatch.setattr(E, "load_library", lambda path=None: fake)
    HostFCN.fake = fake
    f = HostFCN()
    x = np.random.default_rng(2).normal(size=len(train_pos))
    nll, grad = f.nll_grad(x)
    full = np.array([vm.variables[n] for n in names])
    assert nll == 2.0 * full.sum()
    np.testing.assert_array_equal(grad, 2.0 * x)
    assert fake.forms == [E.FORM_SHAPE_CACHE]
    # a parameter fixed after construction: new layout, shorter gradient
    fixed = vm.trainable_vars[0]
    vm.set_fix(fixed)
    nll, grad = f.nll_grad()
    assert f.layouts[-1] == vm.trainable_vars and fixed not in f.layouts[-1]
    assert len(grad) == len(train_pos) - 1
    full = np.array([vm.variables[n] for n in names])
    np.testing.assert_array_equal(grad, 2.0 * full[fake.train_pos])

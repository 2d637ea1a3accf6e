"""Reference-facing API: ConfigLoader, amplitude, FCN and fit.

Mirrors the public surface of TF-PWA that callers of the amplitude-fit hot
path use, with the same names, arguments and parameter conventions:

* ``ConfigLoader(file)``: ``tf_pwa/config_loader/config_loader.py:62-104``;
  ``get_amplitude`` (:210-237), ``get_data``/``get_all_data`` (:130-200),
  ``get_fcn`` (:659-720), ``fit`` (:744-801), ``get_params_error``
  (:814-874), ``set_params``/``get_params``/``save_params`` (:995-1040).
* ``FCN``: ``tf_pwa/model/model.py:1115-1285`` -- ``__call__``, ``grad``,
  ``nll_grad`` (float NLL and gradient list in ``vm.trainable_vars`` order),
  ``nll_grad_hessian``.
* ``FitResult``: ``tf_pwa/fit.py:497-536``.

Data: the reference's ``E px py pz`` text files or ``.npy`` arrays, grouped
per event in ``dat_order`` (``tf_pwa/data.py:300-365``); an index matching
``negtive_idx`` (default ``bg*``) enters with weight ``-<idx>_weight``
(``config_loader/data.py:149-169,215-232``).
Every evaluation runs on the CUDA engine; there is no CPU path.
"""
import json
import os
import re
import time
import warnings

import numpy as np

from .decay_config import DecayConfig, float_particles, init_params, load_yaml
from .engine import (FORM_MIXED_F32, FORM_PLAIN_F64, FORM_SHAPE_CACHE, MIXED_F32, PLAIN_F64,
                     Engine, PWAError, read_dat)
from .kinematics import event_fields, p4_dict
from .plan import Plan
from .variables import Bound, VarsManager

PRECISIONS = {"plain": PLAIN_F64, "f64": PLAIN_F64, "mixed": MIXED_F32, "chosen": MIXED_F32}


class EventData:
    """One dataset: plan-ordered (n_fields, N) FP64 columns and weights."""

    def __init__(self, fields, weight=None):
        self.fields = fields
        n = fields.shape[1]
        self.weight = np.ones(n) if weight is None else np.asarray(weight, np.float64)
        self.n = n

    def __len__(self):
        return self.n

    def numpy_fields(self):
        f = self.fields
        return f.detach().cpu().numpy() if hasattr(f, "detach") else np.asarray(f)


def load_dat_file(fnames, n_particles):
    """(N, n_particles, 4) momenta from ``.dat``/``.npy``/``.npz`` files
    (``tf_pwa/data.py:300-365``): the files of one list hold the same N
    events split by particle -- file i has N x n_i rows, event by event, for
    the next n_i particles of ``dat_order`` -- so a single file holds all
    particles of each event in turn."""
    if isinstance(fnames, str):
        fnames = [fnames]
    datas = []
    for fn in fnames:
        if fn.endswith(".npz"):
            a = np.load(fn)["arr_0"]
        elif fn.endswith(".npy"):
            a = np.load(fn)
        else:
            a = read_dat(fn)
        datas.append(np.reshape(a, (-1, 4)))
    n_total = sum(d.shape[0] for d in datas)
    if n_total % n_particles != 0:
        raise ValueError(f"number of data find {n_total}/{n_particles}")
    n_data = n_total // n_particles
    parts = [d.reshape(n_data, d.shape[0] // n_data, 4) for d in datas]
    out = np.concatenate(parts, 1)
    if out.shape[1] != n_particles:
        raise ValueError(f"files hold {out.shape[1]} particles per event, expected {n_particles}")
    return out


def force_pos_def(h):
    """Inverse of the Hessian ``h``, made positive definite where rounding
    or a poorly constrained direction left it indefinite
    (``tf_pwa/applications.py:206-276``): a small negative eigenvalue
    (above -1e-5 of the largest) is lifted by 1.1 times its size before
    inverting; a strongly indefinite matrix gets the diagonal correction of
    Minuit2's MnPosDef on its pseudo-inverse (error diagonal raised to be
    positive, then scaled until the correlation matrix is positive
    definite)."""
    h = np.asarray(h, np.float64)
    e, v = np.linalg.eig(h)
    inv = np.linalg.pinv(h)
    e_min, e_max = float(np.min(e.real)), float(np.max(np.abs(e)))
    if e_min > 0:
        return inv
    if e_min > -1e-5 * e_max:
        e2 = np.where(e.real < 0, e - 1.1 * e_min, e)
        return np.linalg.inv(np.real(v @ np.diag(e2) @ np.linalg.inv(v)))
    eps2 = max(1e-6, 2.0 * np.sqrt(np.finfo(np.float64).eps))
    err = inv.copy()
    d = np.diag(err)
    if d.min() <= 0:
        err = err + np.eye(len(d)) * (0.5 + eps2 - d.min())
    d = np.diag(err)
    w = np.linalg.eigvalsh(err / np.sqrt(np.outer(d, d)))
    pmin, pmax = float(w.min()), max(float(np.abs(w).max()), 1.0)
    if pmin > eps2 * pmax:
        return err
    return err + np.diag(d * (0.001 * pmax - pmin))


class AmplitudeModel:
    """sum |A|^2 of the model per event (``AbsPDF.__call__``)."""

    def __init__(self, config, precision="plain"):
        self.config = config
        self.vm = config.vm
        self.decay_group = config.decay_group
        self.precision = PRECISIONS[precision]
        self._eng = None
        self._cached = None

    @property
    def trainable_variables(self):
        return list(self.vm.trainable_vars)

    def get_params(self, trainable_only=False):
        return self.vm.get_all_dic(trainable_only)

    def set_params(self, var):
        self.vm.set_all(var)

    def _engine(self):
        if self._eng is None:
            self._eng = Engine(self.decay_group, self.config.plan, self.vm)
        return self._eng

    def __call__(self, data):
        self._engine()
        if self._cached is not data:
            x = data.numpy_fields()
            self._eng.upload(x, np.ones(x.shape[1]))
            self._cached = data
        import torch

        out = torch.empty(data.n, dtype=torch.float64, device="cuda")
        C = self._eng.consts(self.vm.get_all_dic())
        self._eng.pdf_device(C, 0, data.n, out.data_ptr(), self.precision)
        return out.cpu().numpy()


class FCN:
    """Negative log-likelihood of data against the MC-normalised amplitude.

    ``precision``: "plain" (FP64 throughout) or "mixed" (FP32 amplitudes,
    FP64 sums; with ``gram=True`` and fixed masses/widths the MC integral
    uses the cached Gram matrix; with floating masses/widths and
    ``shape_cache`` (default where the columns factorise) every evaluation
    reads the cached shape-free columns and recomputes only the lineshapes).  ``bg``, ``batch`` take the reference's
    positions; ``w_bkg`` (weight of bg rows without their own weights),
    ``precision`` and ``gram`` are passed by keyword."""

    def __init__(self, config, data, mcdata, bg=None, batch=65000, inmc=None, gauss_constr=None,
                 w_bkg=1.0, precision="plain", gram=None, shape_cache=None):
        # positional order of tf_pwa/model/model.py:1126-1135
        if inmc is not None or gauss_constr:
            raise NotImplementedError("inmc samples / Gaussian constraints")
        self.config = config
        self.vm = config.vm
        self.precision = PRECISIONS[precision]
        self.n_call = 0
        self.cached_nll = None
        wd = list(data.weight)
        xd = [data.numpy_fields()] if not hasattr(data.fields, "data_ptr") else None
        if bg is not None:
            wb = bg.weight if bg.weight is not None else -w_bkg * np.ones(bg.n)
            w = np.concatenate([data.weight, wb])
        else:
            w = np.asarray(data.weight)
        self.alpha = w.sum() / (w * w).sum()
        self.weight = self.alpha * w
        self.eng = Engine(config.decay_group, config.plan, self.vm)
        self._upload(data, bg, mcdata)
        shape_free = any(n.endswith(("_mass", "_width")) for n in self.vm.trainable_vars)
        # a polarised parent weights the helicity products with its density
        # matrix, CP-violating totals differ per event charge: the column
        # cache / Gram form does not apply
        polarised = self.eng.code.nrho > 0 or bool(self.eng.code.cp_chains)
        self.use_gram = (self.precision == MIXED_F32 and not shape_free and not polarised) \
            if gram is None else gram
        if self.use_gram and (shape_free or polarised):
            raise ValueError("the Gram cache needs fixed masses and widths, no polarisation "
                             "and no CP-violating totals")
        self.tune = None
        # floating masses/widths in the mixed form: the shape-free column
        # cache where the columns factorise (else the FP32 recompute form)
        self.use_shape_cache = (self.precision == MIXED_F32 and shape_free
                                and self.eng.code.shape_cache_ok) \
            if shape_cache is None else shape_cache
        if self.use_shape_cache:
            try:
                self.eng.shape_cache(self.vm.get_all_dic())
                self.eng.use_shape_cache = True
            except PWAError as e:
                if shape_cache:
                    raise
                warnings.warn(f"floating-shape column cache not used: {e}")
                self.use_shape_cache = False
        self._var_names = list(self.vm.variables.keys())
        self._train = list(self.vm.trainable_vars)
        # the host side of each evaluation (constants, Jacobian, chain rule)
        # in native code where the host program covers the model (no
        # CP-violating totals, no polarised parent); else the Python host code
        self.native_host = False
        if not self.use_gram:
            self._form = (FORM_PLAIN_F64 if self.precision == PLAIN_F64 else
                          FORM_SHAPE_CACHE if self.use_shape_cache else FORM_MIXED_F32)
            try:
                self.eng.set_host_program(self._var_names, self._train)
                self.native_host = True
            except PWAError:
                pass
        if self.use_gram:
            vals = self.vm.get_all_dic()
            self.eng.set_gram(vals)
            self.eng.cache_data(vals)
            self.eng.set_param_layout(self._var_names, self._train)
            # pick the fastest configuration of the cached data-term kernel
            # for this model and event count (PWA_AUTOTUNE=0: keep the default;
            # PWA_CACHED_CONFIG="variant,ring_depth,blocks_per_sm": pin one)
            pin = os.environ.get("PWA_CACHED_CONFIG")
            if pin:
                parts = [int(v) for v in pin.split(",")]
                self.eng.set_cached_config(*(parts + [0, 0])[:3])
                self.tune = (None, self.eng.cached_config(), None)
            elif os.environ.get("PWA_AUTOTUNE", "1") != "0":
                self.eng.consts(vals)
                try:
                    self.tune = self.eng.autotune_cached()
                except PWAError as e:  # keep the default configuration
                    warnings.warn(f"cached-kernel autotuning failed, default kept: {e}")
                    self.tune = (None, None, str(e))
                    self.eng.set_cached_config(-1)

    def _upload(self, data, bg, mcdata):
        import torch

        parts = [data] + ([bg] if bg is not None else [])
        if all(hasattr(p.fields, "data_ptr") and p.fields.is_cuda for p in parts + [mcdata]):
            x = torch.cat([p.fields for p in parts] + [mcdata.fields], 1)
            c = self.eng.code
            xm = x[c.mass_fields].contiguous() if c.mass_fields else x[:1].contiguous()
            xa = x[c.angle_fields].contiguous() if c.angle_fields else x[:1].contiguous()
            wm = np.asarray(mcdata.weight, np.float64)
            wm = wm / wm.sum()
            w = torch.as_tensor(np.concatenate([self.weight, wm]), device="cuda")
            nd = sum(p.n for p in parts)
            self.eng.upload_device(xm.data_ptr(), xa.data_ptr(), w.data_ptr(), nd, mcdata.n,
                                   float(self.weight.sum()))
            torch.cuda.synchronize()
        else:
            xd = np.concatenate([p.numpy_fields() for p in parts], 1)
            self.eng.upload(xd, self.weight, mcdata.numpy_fields(), mcdata.weight)

    # -- reference API -----------------------------------------------------
    def get_params(self, trainable_only=False):
        return self.vm.get_all_dic(trainable_only)

    def _set(self, x):
        if x is None:
            return
        if isinstance(x, dict):
            if x:
                self.vm.set_all(x)
        elif isinstance(x, np.ndarray):
            if x.size:
                self.vm.set_all(x)
        elif len(x):
            self.vm.set_all(list(x))

    def get_nll_grad(self, x=None):
        self._set(x)
        if self.vm.trainable_vars != self._train:
            self._relayout()
        if self.use_gram:
            v = self.vm.variables
            nll, g = self.eng.nll_grad_cached([v[k] for k in self._var_names])
        elif self.native_host:
            v = self.vm.variables
            nll, g = self.eng.nll_grad_vars([v[k] for k in self._var_names], self._form)
        else:
            nll, g = self.eng.nll_grad(self.vm.get_all_dic(), self.vm.trainable_vars,
                                       self.precision)
        self.n_call += 1
        return nll, g

    def _relayout(self):
        """The trainable set changed (set_fix after construction): new
        gradient layout for the native chain rules."""
        self._train = list(self.vm.trainable_vars)
        if self.use_gram:
            self.eng.set_param_layout(self._var_names, self._train)
        elif self.native_host:
            self.eng.set_host_program(self._var_names, self._train)

    def nll_grad(self, x=None):
        nll, g = self.get_nll_grad(x)
        self.cached_nll = nll
        return float(nll), g

    def get_nll(self, x=None):
        return self.get_nll_grad(x)[0]

    def get_grad(self, x=None):
        return self.get_nll_grad(x)[1]

    def grad_hessp(self, x, p, batch=None, step=None):
        """(gradient at x, Hessian times p) (``tf_pwa/model/model.py:
        1268-1275``): the product by a 4-point central difference of the
        adjoint gradient along p; the step along p moves no parameter by
        more than ``step * max(|x_i|, 1e-2)``, the per-parameter step of
        ``nll_grad_hessian``."""
        x0 = np.array(x if x is not None else self.vm.get_all_val(), dtype=np.float64)
        p = np.asarray(p, dtype=np.float64)
        if step is None:
            step = 1e-4 if self.precision == PLAIN_F64 else 1e-2
        pn = float(np.max(np.abs(p) / np.maximum(np.abs(x0), 1e-2)))
        _, g0 = self.get_nll_grad(x0)
        if pn == 0.0:
            return g0, np.zeros_like(g0)
        eps = step / pn
        gs = [np.asarray(self.get_nll_grad(x0 + s_ * eps * p)[1]) for s_ in (-2, -1, 1, 2)]
        self._set(x0)
        return g0, (gs[0] - 8 * gs[1] + 8 * gs[2] - gs[3]) / (12 * eps)

    def __call__(self, x=None):
        nll, _ = self.get_nll_grad(x)
        self.cached_nll = nll
        return nll

    def grad(self, x=None):
        return self.get_nll_grad(x)[1]

    def torch_nll(self, x):
        """NLL(x) as a torch scalar whose backward is the engine's adjoint
        gradient (``NLLFunction``)."""
        return NLLFunction.apply(x, self)

    def nll_grad_hessian(self, x=None, batch=None, step=None):
        """NLL, gradient and Hessian.  In the cached form (fixed masses and
        widths) with no ``step``: the exact Hessian in the couplings from
        one pass over the column cache (``pwa_hessian_cached_exact``; the
        reference's nested-tape Hessian, ``tf_pwa/model/model.py:513-561``).
        (Models whose per-tile rows do not fit in a block's shared memory,
        e.g. 18 columns x 18 helicity outputs, fall back to the stencil.)
        Otherwise by differencing the adjoint gradient: 4-point central
        stencil per parameter, h_i = step * max(|x_i|, 1e-2) (error O(h^4)),
        symmetrised.  Default step: 1e-4 in the plain form; 1e-2 in the
        mixed forms, whose FP32 per-event (or per-warp) values put 1e-7 to
        1e-6 relative rounding noise on the gradient (noise / h must stay
        small); in the cached form the stencil loop runs in the native
        library.  ``batch`` is accepted in the reference's position
        (``tf_pwa/model/model.py:1258``); the engine does not batch."""
        self._set(x)
        if self.use_gram and step is None and self.eng.dist_reduce is None:
            v = self.vm.variables
            try:
                return self.eng.hessian_cached_exact([v[k] for k in self._var_names])
            except PWAError as e:
                # models whose per-tile rows (2 x columns x helicity outputs)
                # exceed a block's shared memory take the stencil below
                if "shared memory" not in str(e):
                    raise
        if step is None:
            step = 1e-4 if self.precision == PLAIN_F64 else 1e-2
        if self.use_gram:
            v = self.vm.variables
            return self.eng.hessian_cached([v[k] for k in self._var_names], step)
        x0 = np.array(self.vm.get_all_val())
        nll, g0, H = hessian_from_gradient(self.get_nll_grad, x0, step)
        self._set(x0)
        return nll, g0, H


def hessian_from_gradient(nll_grad, x0, step):
    """(f, g, H) at ``x0`` from a function returning (f, gradient): row i of
    H is the 4-point central difference (g(x-2h) - 8g(x-h) + 8g(x+h) -
    g(x+2h)) / 12h along parameter i, h = step * max(|x0_i|, 1e-2), exact
    for gradients polynomial up to degree 4; the result is symmetrised.
    Stands in for the reference's nested-tape ``sum_hessian``
    (``tf_pwa/model/model.py:97-140``)."""
    x0 = np.asarray(x0, dtype=np.float64)
    f0, g0 = nll_grad(x0)
    P = len(x0)
    H = np.zeros((P, P))
    for i in range(P):
        h = step * max(abs(x0[i]), 1e-2)
        gs = []
        for s in (-2, -1, 1, 2):
            xs = x0.copy()
            xs[i] += s * h
            gs.append(np.asarray(nll_grad(xs)[1], dtype=np.float64))
        H[i] = (gs[0] - 8 * gs[1] + 8 * gs[2] - gs[3]) / (12 * h)
    return f0, np.asarray(g0, dtype=np.float64), 0.5 * (H + H.T)


class NLLFunction:
    """The NLL as a differentiable torch operation: forward runs the engine
    (NLL and adjoint gradient in one evaluation), backward returns the
    stored gradient times the incoming one.  ``NLLFunction.apply(x, fcn)``
    with x a float64 tensor of the trainable parameters (vm order)."""

    _fn = None

    @classmethod
    def apply(cls, x, fcn):
        if cls._fn is None:
            import torch

            class _F(torch.autograd.Function):
                @staticmethod
                def forward(ctx, xx, f):
                    nll, g = f.get_nll_grad(xx.detach().cpu().numpy())
                    ctx.save_for_backward(torch.as_tensor(g, dtype=xx.dtype, device=xx.device))
                    return xx.new_tensor(float(nll))

                @staticmethod
                def backward(ctx, gout):
                    (g,) = ctx.saved_tensors
                    return gout * g, None

            cls._fn = _F
        return cls._fn.apply(x, fcn)


class FitResult:
    def __init__(self, params, fcn, min_nll, ndf=0, success=True, message="", hess_inv=None,
                 n_call=0):
        self.params = params
        self.error = {}
        self.fcn = fcn
        self.min_nll = float(min_nll)
        self.ndf = int(ndf)
        self.success = success
        self.message = message
        self.hess_inv = hess_inv
        self.n_call = n_call

    def save_as(self, file_name, save_hess=False):
        s = {"value": self.params, "error": self.error, "status": {
            "success": self.success, "NLL": self.min_nll, "Ndf": self.ndf}}
        with open(file_name, "w") as f:
            json.dump(s, f, indent=2)

    def set_error(self, error):
        self.error = dict(error)


class ConfigLoader:
    """config.yml -> model, data, FCN and fit (reference-compatible)."""

    def __init__(self, file_name, vm=None, share_dict=None, precision="plain", seed=None):
        self.config_file = file_name
        self.config = load_yaml(file_name, share_dict)
        base = os.path.dirname(os.path.abspath(file_name)) if isinstance(file_name, str) else "."
        self.base_dir = base
        self.decay_config = DecayConfig(self.config, base_dir=base, share_dict=share_dict)
        self.decay_group = self.decay_config.decay_group
        self.full_decay = self.decay_group
        self.vm = vm if vm is not None else VarsManager(
            rng=np.random.default_rng(seed))
        self._names = init_params(self.decay_group, self.vm, self.config.get("constrains"))
        self.bound_dic = float_particles(self.decay_group, self.vm, self._names,
                                         self.decay_config.particle_property)
        self.plan = Plan(self.decay_group, self.config.get("data", {}).get("dat_order"))
        # configured values of the floated masses/widths: kept by reinit_params
        self.init_value = {n: self.vm.variables[n] for kind in ("mass", "width")
                           for n in self._names.get(kind, {}).values()
                           if n in self.vm.trainable_vars}
        self.precision = precision
        self._amp = None
        self._data = {}
        self._toy_seed = 0 if seed is None else int(seed)
        self._toy_calls = 0
        self.max_amplitude = None

    # -- model --------------------------------------------------------------
    def get_decay(self, full=True):
        return self.decay_group

    def get_amplitude(self, vm=None, name=""):
        if self._amp is None:
            self._amp = AmplitudeModel(self, self.precision)
        return self._amp

    def get_dat_order(self):
        order = self.config.get("data", {}).get("dat_order")
        return order if order is not None else [str(o) for o in self.decay_group.outs]

    # -- data ---------------------------------------------------------------
    def _path(self, f):
        return f if os.path.isabs(f) else os.path.join(self.base_dir, f)

    def load_p4(self, files):
        files = [self._path(f) for f in (files if isinstance(files, list) else [files])]
        return load_dat_file(files, len(self.get_dat_order()))

    def data_from_p4(self, p4, weight=None, device=None, charge=None):
        """EventData from (N, n_final, 4) momenta in dat_order.  With
        ``device="cuda"`` the engine's kinematics kernel computes the fields
        on the GPU (one thread per event); otherwise the host code does.
        ``charge``: per-event charge_conjugation (+1 / -1) for models whose
        data carry charges."""
        if device is not None and str(device).startswith("cuda"):
            import torch

            eng = self.get_amplitude()._engine()
            x = eng.fields_from_p4(torch.as_tensor(p4, dtype=torch.float64, device=device),
                                   charge=charge)
            return EventData(x, weight)
        x = event_fields(self.plan, p4_dict(p4, self.get_dat_order()), device=device,
                         charge=charge)
        return EventData(x, weight)

    def eval_amplitude(self, *p, extra=None):
        """sum |A|^2 per event from momenta (``config_loader.py:239-249``):
        one (N, 4) array per final particle in the decay's final-state order,
        or one argument -- a {particle name: (N, 4)} dict or an
        (N, n_final, 4) array in dat_order.  ``extra`` may hold the events'
        ``charge``."""
        extra = dict(extra or {})
        charge = extra.pop("charge", extra.pop("charge_conjugation", None))
        if extra:
            raise NotImplementedError(f"eval_amplitude options {sorted(extra)}")
        order = self.get_dat_order()
        outs = [str(o) for o in self.decay_group.outs]
        if len(p) == len(outs) and len(outs) > 1 or (len(p) == 1 and len(outs) == 1
                                                     and np.ndim(p[0]) == 2):
            p = (dict(zip(outs, p)),)
        if len(p) != 1:
            raise ValueError("eval_amplitude: give every final momentum, a dict or one array")
        p4 = p[0]
        if isinstance(p4, dict):
            p4 = np.stack([np.asarray(p4[n], dtype=np.float64) for n in order], 1)
        return self.get_amplitude()(self.data_from_p4(np.asarray(p4, dtype=np.float64),
                                                      charge=charge))

    def get_data(self, idx):
        if idx in self._data:
            return self._data[idx]
        dcfg = self.config.get("data", {})
        files = dcfg.get(idx)
        if files is None:
            return None
        if isinstance(files, str):
            files = [files]
        # a list of files is one sample split by particle; a list of lists,
        # one sample per inner list (tf_pwa/config_loader/data.py:415-421)
        groups = files if files and isinstance(files[0], (list, tuple)) else [files]
        # weight = sign * (scalar ``<idx>_weight`` or the concatenated weight
        # files cut to the events read), sign -1 for indices matching
        # ``negtive_idx`` (default "bg*")
        wkey = dcfg.get(idx + "_weight")
        wfile = None
        if wkey is not None and not isinstance(wkey, (int, float)):
            wfile = np.concatenate([np.loadtxt(self._path(x)).reshape(-1)
                                    for x in (wkey if isinstance(wkey, list) else [wkey])])
        sign = -1.0 if any(re.match(pat, idx) for pat in dcfg.get("negtive_idx", ["bg*"])) else 1.0
        # per-event charges (``<idx>_charge``: a number or files, default +1)
        ckey = dcfg.get(idx + "_charge")
        cfile = None
        if ckey is not None and not isinstance(ckey, (int, float)):
            cfile = np.concatenate([np.loadtxt(self._path(x)).reshape(-1)
                                    for x in (ckey if isinstance(ckey, list) else [ckey])])
        ret, off = [], 0
        for grp in groups:
            p4 = self.load_p4(list(grp))
            n = p4.shape[0]
            if wfile is not None:
                w = wfile[off:off + n]
                if w.shape[0] != n:
                    raise ValueError(f"{idx}_weight holds {wfile.shape[0]} values for more events")
            else:
                w = np.full(n, 1.0 if wkey is None else float(wkey))
            ch = None
            if self.plan.use_charge:
                ch = cfile[off:off + n] if cfile is not None else \
                    np.full(n, 1.0 if ckey is None else float(ckey))
                if ch.shape[0] != n:
                    raise ValueError(f"{idx}_charge holds {cfile.shape[0]} values for more events")
            off += n
            ret.append(self.data_from_p4(p4, sign * w, charge=ch))
        self._data[idx] = ret
        return ret

    def get_all_data(self):
        return [self.get_data(k) for k in ("data", "phsp", "bg", "inmc")]

    @staticmethod
    def _merge(lst):
        if lst is None:
            return None
        if len(lst) == 1:
            return lst[0]
        import torch

        if hasattr(lst[0].fields, "data_ptr"):
            f = torch.cat([d.fields for d in lst], 1)
        else:
            f = np.concatenate([d.fields for d in lst], 1)
        return EventData(f, np.concatenate([d.weight for d in lst]))

    def get_fcn(self, all_data=None, batch=65000, vm=None, name="", precision=None, gram=None):
        """FCN of the config's (or the given) data, phsp, bg samples
        (``config_loader.py:659-720``); ``vm`` and ``name`` are accepted as in
        the reference (the loader's own parameters are used)."""
        if all_data is None:
            data, phsp, bg, _ = self.get_all_data()
        else:
            data, phsp, bg = all_data[:3]
        data = self._merge(data if isinstance(data, list) else [data])
        phsp = self._merge(phsp if isinstance(phsp, list) else [phsp])
        if bg is not None:
            bg = self._merge(bg if isinstance(bg, list) else [bg])
        return FCN(self, data, phsp, bg=bg, precision=precision or self.precision, gram=gram,
                   batch=batch)

    # -- parameters ---------------------------------------------------------
    def get_params(self, trainable_only=False):
        return self.vm.get_all_dic(trainable_only)

    def set_params(self, params, neglect_params=None):
        if isinstance(params, str):
            with open(params) as f:
                params = json.load(f)
            params = params.get("value", params)
        skip = set(neglect_params or [])
        self.vm.set_all({k: v for k, v in params.items()
                         if k in self.vm.variables and k not in skip})
        return True

    def save_params(self, file_name):
        with open(file_name, "w") as f:
            json.dump(self.get_params(), f, indent=2)

    # -- fit ----------------------------------------------------------------
    def fit(self, data=None, phsp=None, bg=None, inmc=None, batch=65000, method="BFGS",
            check_grad=False, improve=False, reweight=False, maxiter=None, jac=True,
            print_init_nll=True, callback=None, grad_scale=1.0, gtol=1e-3, fcn=None,
            precision=None):
        """BFGS on FCN.nll_grad (``config_loader.py:745-801``,
        ``tf_pwa/fit.py:189-419``): same arguments; the objective and its
        gradient are multiplied by ``grad_scale`` for the minimiser (gtol
        too), ``jac=False`` lets scipy difference the NLL, ``callback`` goes
        to scipy.  ``inmc`` samples and ``reweight`` are not supported;
        ``check_grad`` and ``improve`` are accepted and have no effect."""
        from scipy.optimize import minimize

        if inmc is not None or reweight:
            raise NotImplementedError("inmc samples / reweight")
        if fcn is None:
            fcn = self.get_fcn(None if data is None else [data, phsp, bg], batch,
                               precision=precision)
        if print_init_nll:
            print("initial NLL: ", fcn.nll_grad()[0])
        y0 = np.array(self.vm.get_all_val())
        maxiter = maxiter or max(100 * len(y0), 2000)
        # bounded variables are fitted through their transform
        # (tf_pwa/fit.py:270-280, vm.trans_fcn_grad)
        names = list(self.vm.trainable_vars)
        bounds = {i: Bound(*self.bound_dic[n]) for i, n in enumerate(names)
                  if n in getattr(self, "bound_dic", {})}

        def to_y(x):
            y = np.array(x, dtype=float)
            for i, b in bounds.items():
                y[i] = b.x2y(x[i])
            return y

        def fg(x):
            nll, g = fcn.nll_grad(to_y(x))
            g = np.array(g, dtype=float)
            for i, b in bounds.items():
                g[i] *= b.dydx(x[i])
            return grad_scale * nll, grad_scale * g

        x0 = y0.copy()
        for i, b in bounds.items():
            x0[i] = b.y2x(y0[i])
        t0 = time.time()
        opts = {"maxiter": maxiter, "gtol": gtol * grad_scale}
        if jac:
            res = minimize(fg, x0, jac=True, method=method, options=opts, callback=callback)
        else:
            res = minimize(lambda x: fg(x)[0], x0, method=method, options=opts,
                           callback=callback)
        self.vm.set_all(list(to_y(res.x)))
        self.vm.std_polar_all()
        hess_inv = getattr(res, "hess_inv", None)
        if hess_inv is not None and not isinstance(hess_inv, np.ndarray):
            hess_inv = None  # (L-BFGS-B returns an operator)
        fr = FitResult(self.get_params(), fcn, res.fun / grad_scale, ndf=len(x0),
                       success=bool(res.success), message=str(res.message),
                       hess_inv=None if hess_inv is None else hess_inv * grad_scale,
                       n_call=fcn.n_call)
        fr.time = time.time() - t0
        self._fcn = fcn
        self.fit_params = fr
        return fr

    def get_chain(self, idx):
        """``config_loader.py:889-891``: a chain by index or particle names."""
        return self.full_decay.get_decay_chain(idx)

    def get_ndf(self):
        """Number of free parameters (``config_loader.py:722-725``)."""
        return len(self.vm.trainable_vars)

    def reinit_params(self):
        """New random starting point (``config_loader.py:803-805``)."""
        self.vm.refresh_vars(init_val=self.init_value, bound_dic=self.bound_dic)

    def fitNtimes(self, N, *args, **kwargs):
        """N fits from random starting points, each result's parameters
        printed as JSON (``config_loader.py:807-812``); returns the results."""
        out = []
        for _ in range(N):
            self.reinit_params()
            fr = self.fit(*args, **kwargs)
            print(json.dumps(fr.params, indent=2), flush=True)
            out.append(fr)
        return out

    def likelihood_profile(self, var, var_min, var_max, N=100):
        """Profile of the minimum NLL in ``var`` (``config_loader.py:
        964-993``): ``var`` fixed at steps of (var_max - var_min)/N upward
        from its current value to var_max, then downward to var_min, a fit
        of the other parameters at each; returns (values, NLLs) in
        ascending order and restores the parameters and the free flag."""
        params = self.get_params()
        delta = (var_max - var_min) / N
        unfix = var in self.vm.trainable_vars
        up_v, up_n, down_v, down_n = [], [], [], []
        v = params[var]
        while v <= var_max:
            self.vm.set_fix(var, v)
            up_v.append(v)
            up_n.append(self.fit(print_init_nll=False).min_nll)
            v += delta
        self.set_params(params)
        v = params[var] - delta
        while v >= var_min:
            self.vm.set_fix(var, v)
            down_v.append(v)
            down_n.append(self.fit(print_init_nll=False).min_nll)
            v -= delta
        self.set_params(params)
        self.vm.set_fix(var, params[var], unfix=unfix)
        return down_v[::-1] + up_v, down_n[::-1] + up_n

    def get_params_error(self, params=None, data=None, phsp=None, bg=None, inmc=None,
                         batch=10000, using_cached=False, method=None, force_pos=True,
                         correct_params=None, fcn=None):
        """Errors from the inverse Hessian in FP64 (``config_loader.py:814-873``,
        ``applications.py:249-309``): with ``using_cached`` the last inverse
        Hessian is reused; otherwise the Hessian of ``FCN.nll_grad_hessian``
        (exact in the cached form, differenced adjoint gradients otherwise)
        is inverted -- made positive definite first with
        ``force_pos`` (``force_pos_def``), else by pseudo-inverse.  The
        errors are also stored on the last fit's result."""
        if inmc is not None or correct_params:
            raise NotImplementedError("inmc samples / corrected parameters")
        if params is not None:
            self.set_params(params.params if isinstance(params, FitResult) else params)
        if using_cached and getattr(self, "inv_he", None) is not None:
            inv = self.inv_he
        else:
            fcn = fcn or getattr(self, "_fcn", None) or self.get_fcn(
                None if data is None else [data, phsp, bg])
            _, _, H = fcn.nll_grad_hessian()
            inv = force_pos_def(H) if force_pos else np.linalg.pinv(H)
            self.inv_he = inv
        err = dict(zip(self.vm.trainable_vars, np.sqrt(np.abs(np.diag(inv)))))
        if getattr(self, "fit_params", None) is not None:
            self.fit_params.set_error(err)
        return err

    def attach_fix_params_error(self, params, V_b=None):
        """Propagate the errors of fixed parameters b into the free ones a
        (``config_loader.py:1049-1100``): with a(b) the minimum, da/db =
        H_aa^-1 H_ab from the FP64 Hessian over a and b (b freed for the
        Hessian, fixed again after); V_a = (da/db) V_b (da/db)^T, V_b by
        default diag(error_b^2) from ``params`` {name: error}.  V_a is added
        to ``self.inv_he`` and returned."""
        new = list(params)
        for n in new:
            self.vm.set_fix(n, unfix=True)
        all_params = list(self.vm.trainable_vars)
        try:
            fcn = self.get_fcn(precision="plain")
            try:
                _, _, hess = fcn.nll_grad_hessian()
            finally:
                fcn.eng.close()
        finally:
            for n in new:
                self.vm.set_fix(n)
        old = [n for n in all_params if n not in new]
        ia = np.array([all_params.index(n) for n in old])
        ib = np.array([all_params.index(n) for n in new])
        grad = np.linalg.inv(hess[np.ix_(ia, ia)]) @ hess[np.ix_(ia, ib)]
        if V_b is None:
            V_b = np.diag([float(params[n]) for n in new]) ** 2
        V = grad @ np.asarray(V_b, dtype=np.float64) @ grad.T
        inv = getattr(self, "inv_he", None)
        self.inv_he = V if inv is None else inv + V
        return V

    # -- toys and phase space (``tf_pwa/config_loader/sample.py``) ------------
    def _toy_engine(self):
        from .engine import Engine

        return Engine(self.decay_group, self.plan, self.vm)

    def _next_seed(self, seed):
        """64-bit key of one generator call: the given seed, else the
        loader's seed and a per-call counter (successive calls differ)."""
        from .workload import _seed

        if seed is not None:
            return _seed(seed, 0)
        self._toy_calls += 1
        return _seed(self._toy_seed, 2 + self._toy_calls)

    def generate_phsp(self, N=1000, include_charge=False, cal_max=False, seed=None):
        """N flat phase-space events (``sample.py:254-260``) as device
        EventData with unit weights: GENBOD candidates accepted on their
        phase-space weight and their fields computed, in the engine's toy
        kernels."""
        from .workload import generate

        if include_charge:
            raise NotImplementedError("charge-conjugated events")
        eng = self._toy_engine()
        try:
            x, _ = generate(eng, int(N), self._next_seed(seed))
        finally:
            eng.close()
        return EventData(x, np.ones(int(N)))

    def generate_phsp_p(self, N=1000, cal_max=False, seed=None):
        """Momenta (N, n_final, 4) of N flat phase-space events in
        ``dat_order`` (``sample.py:224-229``), on the device."""
        from .workload import generate

        eng = self._toy_engine()
        try:
            _, _, p4 = generate(eng, int(N), self._next_seed(seed), with_p4=True)
        finally:
            eng.close()
        return p4

    def generate_toy(self, N=1000, force=True, gen=None, gen_p=None, importance_f=None,
                     max_N=100000, include_charge=False, cal_phsp_max=False, seed=None):
        """N events of the current model by accept-reject on sum |A|^2
        (``sample.py:75-141``, ``applications.py:394-487``) as device
        EventData with unit weights.  The maximum found is kept in
        ``self.max_amplitude`` and reused by later calls, as the reference
        does; a candidate above it raises it and restarts the sample."""
        from .workload import generate

        if gen is not None or gen_p is not None or importance_f is not None or include_charge:
            raise NotImplementedError("custom generators, importance functions or charges")
        eng = self._toy_engine()
        try:
            C = eng.consts(self.vm.get_all_dic())
            x, fmax = generate(eng, int(N), self._next_seed(seed), consts=C,
                               fmax=self.max_amplitude)
        finally:
            eng.close()
        self.max_amplitude = fmax
        return EventData(x, np.ones(int(N)))

    def cal_fitfractions(self, params={}, mcdata=None, res=None, exclude_res=[], batch=25000,
                         method="old", fcn=None):
        """Fit fractions and errors (``config_loader.py:893-916`` ->
        ``applications.fit_fractions``): (frac, err_frac), keyed by resonance
        name and by (name_i, name_j) pairs for interference terms.  The MC
        sample is that of ``fcn`` (default: the last fitted FCN, else the
        config's phsp); errors use ``self.inv_he`` from get_params_error."""
        from .fitfractions import fit_fractions

        if hasattr(params, "params"):
            params = params.params
        if params:
            self.set_params(params)
        if fcn is None:
            fcn = getattr(self, "_fcn", None) or self.get_fcn(
                None if mcdata is None else [self._merge(self.get_data("data")), mcdata, None])
        if res is None:
            res = sorted(set(str(p) for p in self.decay_group.resonances) - set(exclude_res))
        frac, err, _ = fit_fractions(fcn.eng, self.vm, res, getattr(self, "inv_he", None),
                                     use_gram=fcn.use_gram)
        return frac, err

    def get_phsp_noeff(self):
        """The ``phsp_noeff`` sample, else the first ``phsp`` one
        (``config_loader.py:180-188``)."""
        if "phsp_noeff" in self.config.get("data", {}):
            d = self.get_data("phsp_noeff")
            assert len(d) == 1
            return d[0]
        warnings.warn("No data file as 'phsp_noeff', using the first 'phsp' file instead.")
        return self.get_data("phsp")[0]

    def cal_signal_yields(self, params={}, mcdata=None, batch=25000):
        """Signal yield of each fit-fraction term, with error
        (``config_loader.py:918-962``): N = data events - bg_weight * bg
        events, error sqrt(N_data + bg_weight^2 N_bg) (sqrt(N_data) without
        background; 0 for ``extended`` fits; per-event bg weights summed); yield_i = frac_i N, error
        sqrt((N err_frac_i)^2 + (err_N frac_i)^2).  One dict per data
        sample."""
        frac, err = self.cal_fitfractions(params, mcdata, batch=batch)
        dcfg = self.config.get("data", {})
        data, bg = self.get_data("data"), self.get_data("bg")
        out = []
        for k, d in enumerate(data):
            n_data = d.n
            if bg is None:
                n, n_err = float(n_data), float(np.sqrt(n_data))
            else:
                # bg rows carry weight -bg_weight: N_data - w N_bg, N_data + w^2 N_bg
                wb = np.asarray(bg[k].weight, dtype=np.float64)
                n, n_err = n_data + float(wb.sum()), float(np.sqrt(n_data + float(wb @ wb)))
            if dcfg.get("extended", False):
                n_err = 0.0
            out.append({key: (f * n, float(np.sqrt((n * err.get(key, 0.0)) ** 2
                                                   + (n_err * f) ** 2)))
                        for key, f in frac.items()})
        return out

"""A small TensorFlow-2 stand-in on top of torch (CPU, float64), used ONLY by
``tests/golden/make_golden.py`` to execute the reference package's own Python
code (its ConfigLoader, amplitude, NLL and GradientTape gradient) in a
container where TensorFlow is not installed.  It is test infrastructure for
generating golden vectors; nothing in the product imports it.

Only the subset of the TF API that the reference's hot path touches is
provided.  Semantics follow the public TF documentation of each op; the one
deliberate difference is that Python floats become float64 tensors (the
reference configures float64 everywhere, so this matches its intent).
GradientTape maps to torch.autograd.
"""
import builtins
import contextlib
import functools
import math as _pymath
import types

import numpy as np
import torch

torch.set_default_dtype(torch.float64)
torch.backends.opt_einsum.enabled = False

# the reference predates NumPy 2; restore the aliases it still names
for _n, _v in (("Inf", np.inf), ("NaN", np.nan), ("float_", np.float64), ("complex_", np.complex128)):
    if not hasattr(np, _n):
        setattr(np, _n, _v)

__version__ = "2.99.0-torchshim"

float64 = torch.float64
float32 = torch.float32
complex128 = torch.complex128
complex64 = torch.complex64
int64 = torch.int64
int32 = torch.int32
bool = torch.bool  # noqa: A001  (mirrors tf.bool)

_NP2T = {
    np.dtype("float64"): torch.float64,
    np.dtype("float32"): torch.float32,
    np.dtype("complex128"): torch.complex128,
    np.dtype("complex64"): torch.complex64,
    np.dtype("int64"): torch.int64,
    np.dtype("int32"): torch.int32,
    np.dtype("bool"): torch.bool,
}


def as_dtype(d):
    if isinstance(d, torch.dtype):
        return d
    if d is None:
        return None
    if isinstance(d, str):
        return {
            "float64": torch.float64,
            "float32": torch.float32,
            "complex128": torch.complex128,
            "complex64": torch.complex64,
            "int64": torch.int64,
            "int32": torch.int32,
            "bool": torch.bool,
        }[d]
    return _NP2T[np.dtype(d)]


class TensorShape(tuple):
    def as_list(self):
        return list(self)

    @property
    def rank(self):
        return len(self)

    @property
    def ndims(self):
        return len(self)


class Tensor(torch.Tensor):
    """torch tensor with the few TF Tensor behaviours the reference uses."""

    @classmethod
    def __torch_function__(cls, func, types, args=(), kwargs=None):
        kwargs = kwargs or {}
        return super().__torch_function__(func, types, args, kwargs)

    def numpy(self):
        t = torch.Tensor.detach(self)
        return torch.Tensor.numpy(t.as_subclass(torch.Tensor))

    def __array__(self, dtype=None, copy=None):
        a = self.numpy()
        if dtype is not None:
            a = a.astype(dtype)
        return a

    @property
    def shape(self):
        return TensorShape(torch.Tensor.size(self))

    def get_shape(self):
        return self.shape

    def __getitem__(self, idx):
        # TF reads a list of slices / Ellipsis as a tuple of slice specs
        if isinstance(idx, list) and any(isinstance(s, slice) or s is Ellipsis for s in idx):
            idx = tuple(idx)
        idx_t = idx if isinstance(idx, tuple) else (idx,)
        flips = []
        new_idx = []
        ell = None
        for k, s in enumerate(idx_t):
            if isinstance(s, slice) and s.step is not None and s.step < 0:
                if s.start is not None or s.stop is not None or s.step != -1:
                    raise NotImplementedError("only [::-1] slices")
                flips.append(len(new_idx))
                new_idx.append(slice(None))
            else:
                new_idx.append(s)
        base = torch.Tensor.__getitem__(self, tuple(new_idx))
        if not flips:
            return base
        # resolve flipped dims against the result's rank
        n_before_ell = None
        for k, s in enumerate(new_idx):
            if s is Ellipsis:
                n_before_ell = k
        dims = []
        nd = base.dim()
        for f in flips:
            if n_before_ell is not None and f > n_before_ell:
                dims.append(f - len(new_idx) + nd)
            else:
                dims.append(f)
        return torch.flip(base, dims)

    def __hash__(self):
        return id(self)

    # numpy operands on either side become tensors (TF converts them too)
    def _np(self, o):
        if isinstance(o, (np.ndarray, np.generic)):
            return convert_to_tensor(o)
        return o

    def __add__(self, o):
        return torch.Tensor.__add__(self, self._np(o))

    def __radd__(self, o):
        return torch.Tensor.__radd__(self, self._np(o))

    def __sub__(self, o):
        return torch.Tensor.__sub__(self, self._np(o))

    def __rsub__(self, o):
        return torch.Tensor.__rsub__(self, self._np(o))

    def __mul__(self, o):
        return torch.Tensor.__mul__(self, self._np(o))

    def __rmul__(self, o):
        return torch.Tensor.__rmul__(self, self._np(o))

    def __truediv__(self, o):
        return torch.Tensor.__truediv__(self, self._np(o))

    def __rtruediv__(self, o):
        return torch.Tensor.__rtruediv__(self, self._np(o))

    def __pow__(self, o):
        return torch.Tensor.__pow__(self, self._np(o))

    def __rpow__(self, o):
        return torch.Tensor.__rpow__(self, self._np(o))

    # TF tensors are immutable: ``a += b`` rebinds ``a`` to a new tensor and
    # never writes through a slice view (LorentzVector.boost relies on this)
    def __iadd__(self, o):
        return self.__add__(o)

    def __isub__(self, o):
        return self.__sub__(o)

    def __imul__(self, o):
        return self.__mul__(o)

    def __itruediv__(self, o):
        return self.__truediv__(o)

    def __ipow__(self, o):
        return self.__pow__(o)

    __array_priority__ = 10000

    def __bool__(self):
        return builtins.bool(torch.Tensor.item(self))

    def __len__(self):
        return torch.Tensor.size(self, 0)

    def __iter__(self):
        for i in builtins.range(len(self)):
            yield self[i]


def _wrap(t):
    if isinstance(t, Tensor):
        return t
    return t.as_subclass(Tensor)


def convert_to_tensor(x, dtype=None, dtype_hint=None, name=None):
    dtype = as_dtype(dtype)
    if isinstance(x, Variable):
        t = x
        if dtype is not None and t.dtype != dtype:
            t = t.to(dtype)
        return t
    if isinstance(x, torch.Tensor):
        t = _wrap(x)
        if dtype is not None and t.dtype != dtype:
            t = t.to(dtype)
        return t
    if isinstance(x, (list, tuple)) and any(
        isinstance(i, torch.Tensor) for i in _flatten(x)
    ):
        t = stack([convert_to_tensor(i) for i in x])
        if dtype is not None:
            t = t.to(dtype)
        return t
    if isinstance(x, np.ndarray) or isinstance(x, np.generic):
        a = np.asarray(x)
        if a.dtype == np.dtype("O"):
            a = a.astype(np.float64)
        t = torch.from_numpy(np.array(a, copy=True))
    elif isinstance(x, builtins.bool):
        t = torch.tensor(x)
    elif isinstance(x, int):
        t = torch.tensor(x, dtype=torch.int32 if dtype is None else dtype)
    elif isinstance(x, float):
        t = torch.tensor(x, dtype=torch.float64)
    elif isinstance(x, builtins.complex):
        t = torch.tensor(x, dtype=torch.complex128)
    else:
        a = np.asarray(x)
        if a.dtype == np.dtype("O"):
            a = a.astype(np.float64)
        if a.dtype == np.float32:
            a = a.astype(np.float64)
        if a.dtype == np.int64 and dtype is None:
            a = a.astype(np.int32)
        t = torch.from_numpy(np.array(a, copy=True))
    t = _wrap(t)
    if dtype is not None and t.dtype != dtype:
        t = _cast(t, dtype)
    return t


constant = convert_to_tensor


def _flatten(x):
    if isinstance(x, (list, tuple)):
        for i in x:
            yield from _flatten(i)
    else:
        yield x


def _t(x, like=None):
    if isinstance(x, torch.Tensor):
        return _wrap(x)
    if like is not None and isinstance(x, (int, float, builtins.complex, np.generic)):
        if like.is_complex() and not isinstance(x, builtins.complex):
            return convert_to_tensor(builtins.complex(x), like.dtype)
        return convert_to_tensor(x, like.dtype if not isinstance(x, builtins.complex) else None)
    return convert_to_tensor(x)


def _cast(t, dtype):
    if t.is_complex() and not dtype.is_complex:
        t = torch.real(t)
    return _wrap(t.to(dtype))


def cast(x, dtype, name=None):
    dtype = as_dtype(dtype)
    t = _t(x)
    if t.dtype == dtype:
        return t
    return _cast(t, dtype)


def complex(real, imag, name=None):  # noqa: A001
    r = _t(real)
    i = _t(imag)
    if r.dtype != i.dtype:
        dt = torch.promote_types(r.dtype, i.dtype)
        r, i = r.to(dt), i.to(dt)
    if r.dtype not in (torch.float32, torch.float64):
        r = r.to(torch.float64)
        i = i.to(torch.float64)
    r, i = torch.broadcast_tensors(r, i)
    return _wrap(torch.complex(r, i))


def _binary_prep(x, y):
    if isinstance(x, torch.Tensor) or isinstance(y, torch.Tensor):
        like = x if isinstance(x, torch.Tensor) else y
        return _t(x, like), _t(y, like)
    return _t(x), _t(y)


def where(cond, x=None, y=None, name=None):
    c = _t(cond)
    if x is None:
        return _wrap(torch.nonzero(c))
    like = x if isinstance(x, torch.Tensor) else (y if isinstance(y, torch.Tensor) else None)
    xt = _t(x, like)
    yt = _t(y, like)
    if xt.dtype != yt.dtype:
        dt = torch.promote_types(xt.dtype, yt.dtype)
        xt, yt = xt.to(dt), yt.to(dt)
    return _wrap(torch.where(c.to(torch.bool), xt, yt))


def reduce_sum(x, axis=None, keepdims=False, name=None):
    t = _t(x) if not isinstance(x, (list, tuple)) else stack([_t(i) for i in x])
    if axis is None:
        return _wrap(torch.sum(t))
    if isinstance(axis, (list, tuple)):
        if len(axis) == 0:
            return t
        axis = tuple(int(a) for a in axis)
    return _wrap(torch.sum(t, dim=axis, keepdim=keepdims))


def reduce_mean(x, axis=None, keepdims=False, name=None):
    t = _t(x) if not isinstance(x, (list, tuple)) else stack([_t(i) for i in x])
    if axis is None:
        return _wrap(torch.mean(t))
    return _wrap(torch.mean(t, dim=axis, keepdim=keepdims))


def reduce_max(x, axis=None, keepdims=False, name=None):
    t = _t(x) if not isinstance(x, (list, tuple)) else stack([_t(i) for i in x])
    if axis is None:
        return _wrap(torch.max(t))
    return _wrap(torch.amax(t, dim=axis, keepdim=keepdims))


def reduce_min(x, axis=None, keepdims=False, name=None):
    t = _t(x) if not isinstance(x, (list, tuple)) else stack([_t(i) for i in x])
    if axis is None:
        return _wrap(torch.min(t))
    return _wrap(torch.amin(t, dim=axis, keepdim=keepdims))


def reduce_prod(x, axis=None, keepdims=False, name=None):
    t = _t(x) if not isinstance(x, (list, tuple)) else stack([_t(i) for i in x])
    if axis is None:
        return _wrap(torch.prod(t.reshape(-1)))
    return _wrap(torch.prod(t, dim=axis, keepdim=keepdims))


def reduce_any(x, axis=None, keepdims=False):
    t = _t(x)
    if axis is None:
        return _wrap(torch.any(t))
    return _wrap(torch.any(t, dim=axis, keepdim=keepdims))


def reduce_all(x, axis=None, keepdims=False):
    t = _t(x)
    if axis is None:
        return _wrap(torch.all(t))
    return _wrap(torch.all(t, dim=axis, keepdim=keepdims))


def stack(values, axis=0, name=None):
    ts = [_t(v) for v in values]
    dt = ts[0].dtype
    for t in ts[1:]:
        dt = torch.promote_types(dt, t.dtype)
    ts = [t.to(dt) for t in ts]
    return _wrap(torch.stack(ts, dim=axis))


def unstack(x, num=None, axis=0, name=None):
    return [_wrap(i) for i in torch.unbind(_t(x), dim=axis)]


def concat(values, axis, name=None):
    ts = [_t(v) for v in values]
    dt = ts[0].dtype
    for t in ts[1:]:
        dt = torch.promote_types(dt, t.dtype)
    return _wrap(torch.cat([t.to(dt) for t in ts], dim=axis))


def reshape(x, shape, name=None):
    if isinstance(shape, torch.Tensor):
        shape = [int(i) for i in shape.tolist()]
    shape = [int(i) for i in shape]
    return _wrap(torch.reshape(_t(x), shape))


def expand_dims(x, axis, name=None):
    return _wrap(torch.unsqueeze(_t(x), axis))


def squeeze(x, axis=None, name=None):
    t = _t(x)
    if axis is None:
        return _wrap(torch.squeeze(t))
    return _wrap(torch.squeeze(t, axis))


def transpose(x, perm=None, conjugate=False, name=None):
    t = _t(x)
    if perm is None:
        perm = list(range(t.dim()))[::-1]
    return _wrap(t.permute(*[int(i) for i in perm]))


def tile(x, multiples, name=None):
    return _wrap(_t(x).repeat(*[int(i) for i in multiples]))


def broadcast_to(x, shape, name=None):
    return _wrap(torch.broadcast_to(_t(x), tuple(int(i) for i in shape)))


def gather(params, indices, axis=None, batch_dims=0, name=None):
    p = _t(params)
    if axis is None:
        axis = 0
    if axis < 0:
        axis += p.dim()
    idx = torch.as_tensor(np.asarray(indices), dtype=torch.long) if not isinstance(indices, torch.Tensor) else indices.to(torch.long)
    flat = torch.index_select(p, axis, idx.reshape(-1))
    new_shape = list(p.shape[:axis]) + list(idx.shape) + list(p.shape[axis + 1:])
    return _wrap(flat.reshape(new_shape))


def gather_nd(params, indices, batch_dims=0, name=None):
    p = _t(params)
    idx = torch.as_tensor(np.asarray(indices), dtype=torch.long) if not isinstance(indices, torch.Tensor) else indices.to(torch.long)
    k = idx.shape[-1]
    return _wrap(p[tuple(idx[..., i] for i in range(k))])


def boolean_mask(x, mask, axis=None, name=None):
    return _wrap(_t(x)[_t(mask).to(torch.bool)])


def pad(x, paddings, mode="CONSTANT", constant_values=0, name=None):
    t = _t(x)
    pads = []
    for a, b in reversed([list(p) for p in paddings]):
        pads += [int(a), int(b)]
    return _wrap(torch.nn.functional.pad(t, pads, value=constant_values))


def matmul(a, b, transpose_a=False, transpose_b=False, name=None):
    a, b = _binary_prep(a, b)
    if a.dtype != b.dtype:
        dt = torch.promote_types(a.dtype, b.dtype)
        a, b = a.to(dt), b.to(dt)
    if transpose_a:
        a = a.transpose(-1, -2)
    if transpose_b:
        b = b.transpose(-1, -2)
    return _wrap(torch.matmul(a, b))


def einsum(eq, *args, **kwargs):
    ts = [_t(a) for a in args]
    dt = ts[0].dtype
    for t in ts[1:]:
        dt = torch.promote_types(dt, t.dtype)
    return _wrap(torch.einsum(eq, *[t.to(dt) for t in ts]))


def _unary(fn):
    def f(x, name=None):
        return _wrap(fn(_t(x)))

    return f


sqrt = _unary(torch.sqrt)
sin = _unary(torch.sin)
cos = _unary(torch.cos)
tan = _unary(torch.tan)
exp = _unary(torch.exp)
tanh = _unary(torch.tanh)
acosh = _unary(torch.acosh)
atan = _unary(torch.atan)
acos = _unary(torch.acos)
asin = _unary(torch.asin)
identity = _unary(lambda t: t.clone() if t.requires_grad else t)
sign = _unary(torch.sign)
square = _unary(torch.square)


def abs(x, name=None):  # noqa: A001
    return _wrap(torch.abs(_t(x)))


def pow(x, y, name=None):  # noqa: A001
    xt, yt = _binary_prep(x, y)
    return _wrap(torch.pow(xt, yt))


def maximum(x, y, name=None):
    xt, yt = _binary_prep(x, y)
    return _wrap(torch.maximum(xt, yt))


def minimum(x, y, name=None):
    xt, yt = _binary_prep(x, y)
    return _wrap(torch.minimum(xt, yt))


def atan2(y, x, name=None):
    yt, xt = _binary_prep(y, x)
    return _wrap(torch.atan2(yt, xt))


def clip_by_value(x, lo, hi, name=None):
    return _wrap(torch.clamp(_t(x), lo, hi))


def stop_gradient(x, name=None):
    return _wrap(_t(x).detach())


def zeros_like(x, dtype=None, name=None):
    t = _t(x)
    return _wrap(torch.zeros_like(t, dtype=as_dtype(dtype) or t.dtype))


def ones_like(x, dtype=None, name=None):
    t = _t(x)
    return _wrap(torch.ones_like(t, dtype=as_dtype(dtype) or t.dtype))


def _shape(shape):
    if isinstance(shape, (int, np.integer)):
        return (int(shape),)
    return tuple(int(i) for i in shape)


def zeros(shape, dtype=torch.float64, name=None):
    return _wrap(torch.zeros(_shape(shape), dtype=as_dtype(dtype)))


def ones(shape, dtype=torch.float64, name=None):
    return _wrap(torch.ones(_shape(shape), dtype=as_dtype(dtype)))


def eye(n, dtype=torch.float64, name=None):
    return _wrap(torch.eye(n, dtype=as_dtype(dtype)))


def range(start, limit=None, delta=1, dtype=None, name=None):  # noqa: A001
    if limit is None:
        start, limit = 0, start
    t = torch.arange(start, limit, delta)
    if dtype is not None:
        t = t.to(as_dtype(dtype))
    return _wrap(t)


def norm(x, axis=None, keepdims=False, name=None):
    t = _t(x)
    if axis is None:
        return _wrap(torch.linalg.vector_norm(t))
    return _wrap(torch.linalg.vector_norm(t, dim=axis, keepdim=keepdims))


def add_n(xs):
    r = _t(xs[0])
    for x in xs[1:]:
        r = r + x
    return _wrap(r)


def size(x):
    return _wrap(torch.tensor(_t(x).numel()))


def shape(x):
    return _wrap(torch.tensor(list(_t(x).shape)))


def is_tensor(x):
    return isinstance(x, torch.Tensor)


def function(f=None, **kwargs):
    if f is None:
        return lambda g: g
    return f


def custom_gradient(f):
    raise NotImplementedError("custom_gradient is not provided by the shim")


def numpy_function(f, inp, Tout, name=None):
    out = f(*[np.asarray(i) for i in inp])
    return convert_to_tensor(out)


# ---------------------------------------------------------------- variables
class Variable(Tensor):
    """tf.Variable: a torch leaf tensor; assign() writes in place."""

    def __new__(cls, initial_value=None, trainable=True, dtype=None, name=None, **kw):
        dtype = as_dtype(dtype)
        if callable(initial_value) and not isinstance(initial_value, torch.Tensor):
            initial_value = initial_value()
        t = convert_to_tensor(initial_value, dtype).detach().clone()
        if dtype is not None and t.dtype != dtype:
            t = t.to(dtype)
        # every floating variable records gradients: trainability can change
        # later (set_fix), and the tape is always asked for explicit sources
        v = torch.Tensor._make_subclass(cls, t.as_subclass(torch.Tensor), t.is_floating_point())
        v._trainable = builtins.bool(trainable)
        v._name = name
        return v

    def __init__(self, *args, **kwargs):
        pass

    @property
    def trainable(self):
        return self._trainable

    @property
    def name(self):
        return self._name or "Variable"

    def assign(self, value, read_value=True, **kw):
        with torch.no_grad():
            v = _t(value)
            torch.Tensor.copy_(self, v.to(self.dtype).reshape(self.shape))
        return self

    def assign_add(self, value, **kw):
        with torch.no_grad():
            torch.Tensor.add_(self, _t(value).to(self.dtype))
        return self

    def assign_sub(self, value, **kw):
        with torch.no_grad():
            torch.Tensor.sub_(self, _t(value).to(self.dtype))
        return self

    def value(self):
        return self

    def read_value(self):
        return self

    def __hash__(self):
        return id(self)

    def __deepcopy__(self, memo):
        return Variable(self.numpy(), trainable=self._trainable, dtype=self.dtype)

    def __reduce_ex__(self, proto):
        return (Variable, (self.numpy(), self._trainable, self.dtype))


class GradientTape:
    def __init__(self, persistent=False, watch_accessed_variables=True):
        self.persistent = persistent
        self._outer = None

    def __enter__(self):
        self._gm = torch.enable_grad()
        self._gm.__enter__()
        _TAPES.append(self)
        return self

    def __exit__(self, *a):
        _TAPES.remove(self)
        self._gm.__exit__(*a)
        return False

    def watch(self, x):
        pass

    def gradient(self, target, sources, output_gradients=None, unconnected_gradients=None):
        single = not isinstance(sources, (list, tuple))
        srcs = [sources] if single else list(sources)
        tgt = target
        if isinstance(tgt, (list, tuple)):
            tgt = reduce_sum(stack([reduce_sum(i) for i in tgt]))
        if not tgt.requires_grad:
            gs = [None] * len(srcs)
        else:
            nested = builtins.len(_TAPES) > 0 or self.persistent
            gs = torch.autograd.grad(
                tgt, srcs, allow_unused=True, retain_graph=True, create_graph=nested
            )
        out = []
        for g, s in zip(gs, srcs):
            if g is None:
                g = torch.zeros_like(s.as_subclass(torch.Tensor))
            out.append(_wrap(g))
        return out[0] if single else out

    def jacobian(self, target, sources, **kw):
        raise NotImplementedError


_TAPES = []


# ---------------------------------------------------------------- submodules
math = types.ModuleType("tensorflow.math")
math.log = _unary(torch.log)
math.exp = exp
math.sqrt = sqrt
math.sin = sin
math.cos = cos
math.tan = tan
math.acos = acos
math.asin = asin
math.atan = atan
math.atan2 = atan2
math.tanh = tanh
math.abs = abs
math.real = _unary(torch.real)
math.imag = _unary(torch.imag)
math.conj = _unary(torch.conj_physical)
math.angle = _unary(torch.angle)
math.is_nan = _unary(torch.isnan)
math.is_finite = _unary(torch.isfinite)
math.sign = sign
math.square = square
math.reduce_sum = reduce_sum
math.reduce_prod = reduce_prod
math.reduce_max = reduce_max
math.reduce_min = reduce_min
math.reduce_mean = reduce_mean
math.maximum = maximum
math.minimum = minimum
math.pow = pow
math.erf = _unary(torch.erf)
math.acosh = acosh
math.log1p = _unary(torch.log1p)


def _polyval(coeffs, x, name=None):
    xt = _t(x)
    r = None
    for c in coeffs:
        c = _t(c, xt)
        r = c if r is None else r * xt + c
    if r is None:
        return zeros_like(xt)
    return _wrap(r + torch.zeros_like(xt))


math.polyval = _polyval
log = math.log
real = math.real
imag = math.imag
conj = math.conj

linalg = types.ModuleType("tensorflow.linalg")
linalg.inv = _unary(torch.linalg.inv)
linalg.det = _unary(torch.linalg.det)
linalg.diag = _unary(torch.diag_embed)
linalg.tensor_diag_part = _unary(lambda t: torch.diagonal(t, dim1=-2, dim2=-1))
linalg.matvec = lambda a, b: _wrap(torch.matmul(_t(a), _t(b).unsqueeze(-1)).squeeze(-1))
linalg.cross = lambda a, b: _wrap(torch.linalg.cross(*torch.broadcast_tensors(*_binary_prep(a, b)), dim=-1))
linalg.matmul = matmul
linalg.eigh = lambda t: tuple(_wrap(i) for i in torch.linalg.eigh(_t(t)))


def _normalize(t, axis=-1, ord="euclidean"):
    t = _t(t)
    n = torch.linalg.vector_norm(t, dim=axis, keepdim=True)
    return _wrap(t / n), _wrap(n)


linalg.normalize = _normalize
linalg.norm = norm

random = types.ModuleType("tensorflow.random")
_gen = torch.Generator().manual_seed(0)


def _set_seed(seed):
    _gen.manual_seed(int(seed))


def _uniform(shape, minval=0.0, maxval=1.0, dtype=torch.float64, seed=None, name=None):
    dt = as_dtype(dtype)
    u = torch.rand(_shape(shape), generator=_gen, dtype=torch.float64)
    return _wrap((minval + (maxval - minval) * u).to(dt))


def _normal(shape, mean=0.0, stddev=1.0, dtype=torch.float64, seed=None, name=None):
    u = torch.randn(_shape(shape), generator=_gen, dtype=torch.float64)
    return _wrap((mean + stddev * u).to(as_dtype(dtype)))


random.set_seed = _set_seed
random.uniform = _uniform
random.normal = _normal

nest = types.ModuleType("tensorflow.nest")


def _map_structure(f, *structs):
    s0 = structs[0]
    if isinstance(s0, dict):
        return {k: _map_structure(f, *[s[k] for s in structs]) for k in s0}
    if isinstance(s0, list):
        return [_map_structure(f, *z) for z in zip(*structs)]
    if isinstance(s0, tuple):
        return tuple(_map_structure(f, *z) for z in zip(*structs))
    return f(*structs)


def _flatten_nest(s):
    if isinstance(s, dict):
        out = []
        for k in sorted(s.keys(), key=str):
            out += _flatten_nest(s[k])
        return out
    if isinstance(s, (list, tuple)):
        out = []
        for i in s:
            out += _flatten_nest(i)
        return out
    return [s]


nest.map_structure = _map_structure
nest.flatten = _flatten_nest

config = types.ModuleType("tensorflow.config")
config.experimental = types.SimpleNamespace(
    list_physical_devices=lambda kind=None: [],
    list_logical_devices=lambda kind=None: [],
    set_memory_growth=lambda d, v: None,
)
config.list_physical_devices = lambda kind=None: []
config.run_functions_eagerly = lambda flag: None

dtypes = types.SimpleNamespace(
    int64=torch.int64, float64=torch.float64, complex128=torch.complex128, as_dtype=as_dtype
)

distribute = types.SimpleNamespace(
    MirroredStrategy=None, ReduceOp=types.SimpleNamespace(SUM="SUM")
)

autograph = types.SimpleNamespace(
    experimental=types.SimpleNamespace(do_not_convert=lambda f=None, **k: f if f is not None else (lambda g: g))
)

compat = types.SimpleNamespace(v1=types.SimpleNamespace(enable_eager_execution=lambda: None))

keras = types.SimpleNamespace(backend=types.SimpleNamespace(set_floatx=lambda x: None))


class TensorSpec:
    def __init__(self, shape=None, dtype=None, name=None):
        self.shape = shape
        self.dtype = dtype


class Module:
    pass


@contextlib.contextmanager
def device(name):
    yield


def control_dependencies(x):
    return contextlib.nullcontext()


def print(*args, **kw):  # noqa: A001
    builtins.print(*args)


raw_ops = types.SimpleNamespace()
data = types.SimpleNamespace(AUTOTUNE=-1, Dataset=None)
saved_model = types.SimpleNamespace()

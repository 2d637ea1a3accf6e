"""Floating-point operation count of the oracle's forward pass, per event.

TEST / MEASUREMENT INFRASTRUCTURE ONLY (the product never imports it).

The counting convention of the per-event work unit: add, subtract and
multiply count 1 (a complex add 2, a complex multiply 6, a real x complex
multiply 2, a multiply-accumulate 2), divisions and transcendental or
square-root calls count as "special" operations (reported separately; a
complex division counts 2 specials and 9 flops, a complex exp 3 specials and
2 flops), comparisons, selections, negation and conjugation count nothing.
Every numpy ufunc call the oracle makes on per-event arrays is counted
element by element (reductions by their input elements); ``np.einsum`` by
the product of all index extents times 2 (real) or 8 (complex).  Work on
per-evaluation constants (arrays without an event axis) is not counted:
the inputs are wrapped in an ndarray subclass and only operations touching
it are seen.

``count_forward(model, fields, vals)`` returns (flops, specials) per event
of ``model.pdf(fields, vals)`` -- the per-event amplitudes and sum |A|^2,
the forward half of one NLL + gradient evaluation.
"""
import contextlib

import numpy as np


class _Tally:
    def __init__(self):
        self.flops = 0.0
        self.special = 0.0


_SPECIAL = {np.sin, np.cos, np.tan, np.arctan2, np.arctan, np.arccos, np.arcsin,
            np.arccosh, np.log, np.sqrt, np.power, np.float_power, np.true_divide,
            np.divide, np.reciprocal, np.exp}
_FREE = {np.negative, np.positive, np.conjugate, np.greater, np.greater_equal, np.less,
         np.less_equal, np.equal, np.not_equal, np.logical_and, np.logical_or, np.logical_not,
         np.isfinite, np.isnan, np.sign, np.copysign, np.maximum, np.minimum, np.fmax, np.fmin}


def _is_complex(a):
    return np.iscomplexobj(a)


class Counted(np.ndarray):
    """ndarray whose element-wise ufunc calls are tallied."""

    tally = None

    def __array_ufunc__(self, ufunc, method, *inputs, **kwargs):
        args = [np.asarray(x) if isinstance(x, Counted) else x for x in inputs]
        if "out" in kwargs:
            kwargs["out"] = tuple(np.asarray(o) if isinstance(o, Counted) else o
                                  for o in kwargs["out"])
        out = getattr(ufunc, method)(*args, **kwargs)
        t = Counted.tally
        if t is not None:
            if method == "reduce":
                n = np.size(args[0]) - np.size(out)
                if ufunc in (np.add, np.multiply):
                    t.flops += n * (2 if _is_complex(args[0]) else 1)
            elif method == "__call__" and ufunc not in _FREE:
                n = np.size(out)
                cplx = [_is_complex(a) for a in args]
                if ufunc in (np.add, np.subtract):
                    t.flops += n * (2 if any(cplx) else 1)
                elif ufunc is np.multiply:
                    t.flops += n * (6 if all(cplx) else 2 if any(cplx) else 1)
                elif ufunc in (np.true_divide, np.divide):
                    if cplx[1] if len(cplx) > 1 else False:
                        t.special += 2 * n
                        t.flops += 9 * n
                    else:
                        t.special += n * (2 if cplx[0] else 1)
                elif ufunc is np.exp and any(cplx):
                    t.special += 3 * n
                    t.flops += 2 * n
                elif ufunc is np.absolute:
                    if any(cplx):
                        t.special += n
                        t.flops += 3 * n
                elif ufunc in _SPECIAL:
                    t.special += n * (2 if any(cplx) else 1)
                else:
                    t.flops += n
        if isinstance(out, tuple):
            return tuple(o.view(Counted) if isinstance(o, np.ndarray) else o for o in out)
        return out.view(Counted) if isinstance(out, np.ndarray) else out


@contextlib.contextmanager
def _counting_einsum(tally):
    orig = np.einsum

    def einsum(subscripts, *operands, **kwargs):
        ops = [np.asarray(o) for o in operands]
        res = orig(subscripts, *ops, **kwargs)
        if any(isinstance(o, Counted) for o in operands):
            lhs = subscripts.split("->")[0].split(",")
            ext = {}
            for lab, o in zip(lhs, ops):
                lab = lab.replace("...", "")
                for ch, dim in zip(lab[::-1], o.shape[::-1]):
                    ext[ch] = dim
                nlead = o.ndim - len(lab)
                if nlead:
                    ext["..."] = max(ext.get("...", 1), int(np.prod(o.shape[:nlead])))
            mac = float(np.prod(list(ext.values())))
            tally.flops += mac * (8 if any(np.iscomplexobj(o) for o in ops) else 2)
            return np.asarray(res).view(Counted)
        return res

    np.einsum = einsum
    try:
        yield
    finally:
        np.einsum = orig


def count_forward(model, fields, vals):
    """(flops, specials) per event of the oracle's sum |A|^2 on ``fields``
    (n_fields, N)."""
    tally = _Tally()
    x = np.asarray(fields, np.float64).view(Counted)
    Counted.tally = tally
    try:
        with _counting_einsum(tally):
            model.pdf(x, vals)
    finally:
        Counted.tally = None
    n = fields.shape[1]
    return tally.flops / n, tally.special / n

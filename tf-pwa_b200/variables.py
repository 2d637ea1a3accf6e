"""Fit-parameter manager with the reference's names, order and conventions.

Mirrors the behaviour of ``tf_pwa/variable.py`` that callers of the fit API
observe: every real parameter has a name, ``trainable_vars`` lists the free
ones in creation order (``tf_pwa/variable.py:120-160``), complex parameters
are stored as ``<name>r``/``<name>i`` pairs in polar form by default
(``tf_pwa/variable.py:162-197``, value r*exp(i*phi) as in
``tf_pwa/variable.py:1715-1765``), ``set_fix``/``set_all``/``get_all_dic``
behave as in ``tf_pwa/variable.py:415-440,684-697``.
"""
import contextlib
import warnings

import numpy as np


class VarsManager:
    def __init__(self, name="", polar=True, rng=None):
        self.name = name
        self.polar = polar
        self.variables = {}        # name -> float
        self.trainable_vars = []   # free names, in order
        self.complex_vars = {}     # complex name -> polar flag
        self.bnd_dic = {}
        self.same_list = []
        self._rng = rng if rng is not None else np.random.default_rng()

    # -- creation ---------------------------------------------------------
    def add_real_var(self, name, value=None, range_=None, trainable=True):
        if name in self.variables and name in self.trainable_vars:
            self.trainable_vars.remove(name)
        if value is None:
            lo, hi = (0.0, 1.0) if range_ is None else range_
            value = float(self._rng.uniform(lo, hi))
        self.variables[name] = float(value)
        if trainable:
            self.trainable_vars.append(name)

    def add_complex_var(self, name, polar=None, trainable=True, fix_vals=(1.0, 0.0)):
        if polar is None:
            polar = self.polar
        if trainable:
            if polar:
                self.add_real_var(name + "r", range_=(0, 2.0))
                self.add_real_var(name + "i", range_=(-np.pi, np.pi))
            else:
                self.add_real_var(name + "r", range_=(-1, 1))
                self.add_real_var(name + "i", range_=(-1, 1))
        else:
            self.add_real_var(name + "r", value=fix_vals[0], trainable=False)
            self.add_real_var(name + "i", value=fix_vals[1], trainable=False)
        self.complex_vars[name] = polar

    def add_cartesiancp_var(self, name, polar=True):
        """A complex coupling with a CP-violating part: r, i, deltar, deltai;
        charge +-1 takes (r +- deltar, i +- deltai) (``tf_pwa/variable.py:
        199-235,1715-1734``)."""
        for suf in ("r", "i", "deltar", "deltai"):
            self.add_real_var(name + suf, range_=(-1, 1))
        self.complex_vars[name] = polar

    def refresh_vars(self, init_val=None, bound_dic=None):
        """Draw new starting values for the free parameters
        (``tf_pwa/variable.py:329-420``): free parts of complex couplings
        uniformly (polar: r in (0, 2), phase in (-pi, pi); cartesian: both
        in (-1, 1)); ``init_val`` entries set to their value, or drawn from
        a normal (mu, sigma) (redrawn until inside the bounds, where given);
        other bounded parameters uniformly between the bounds, or a
        chi-square(1) step inside a one-sided bound."""
        init_val = init_val or {}
        bound_dic = self.bnd_dic if bound_dic is None else bound_dic
        free = set(self.trainable_vars)
        rng = self._rng
        for name, polar in self.complex_vars.items():
            for suf in ("r", "i"):
                n = name + suf
                if n not in free:
                    continue
                if not polar:
                    self.variables[n] = float(rng.uniform(-1, 1))
                elif suf == "r":
                    self.variables[n] = float(rng.uniform(0, 2))
                else:
                    self.variables[n] = float(rng.uniform(-np.pi, np.pi))
        for n in [k for k in init_val if k in free]:
            v = init_val[n]
            if hasattr(v, "__len__"):
                mu, sigma = v[0], v[1]
                lo, hi = bound_dic.get(n, (None, None))
                for _ in range(10000):
                    val = float(rng.normal(mu, sigma))
                    if (lo is None or val > lo) and (hi is None or val < hi):
                        break
                self.variables[n] = val
            elif v is not None:
                self.variables[n] = float(v)
        for n, (lo, hi) in bound_dic.items():
            if n in init_val or n not in free:
                continue
            if lo is not None and hi is not None:
                self.variables[n] = float(rng.uniform(lo, hi))
            elif lo is not None:
                self.variables[n] = float(lo + rng.chisquare(1))
            elif hi is not None:
                self.variables[n] = float(hi - rng.chisquare(1))

    # -- fixing ------------------------------------------------------------
    def set_fix(self, name, value=None, unfix=False):
        if value is not None:
            self.variables[name] = float(value)
        if unfix:
            if name in self.trainable_vars:
                warnings.warn(f"{name} has been freed already!")
            else:
                self.trainable_vars.append(name)
        else:
            if name in self.trainable_vars:
                self.trainable_vars.remove(name)

    def is_fixed(self, name):
        return name not in self.trainable_vars

    # -- values ------------------------------------------------------------
    def get(self, name):
        return self.variables[name]

    def set(self, name, value):
        if name not in self.variables:
            warnings.warn(f"{name} not found")
            return
        self.variables[name] = float(value)

    def set_all(self, vals):
        if isinstance(vals, dict):
            for k, v in vals.items():
                self.set(k, v)
        else:
            # python floats (an array's tolist() is already float)
            vals = vals.tolist() if isinstance(vals, np.ndarray) else [float(v) for v in vals]
            if len(vals) != len(self.trainable_vars):
                raise ValueError(
                    f"expected {len(self.trainable_vars)} values, got {len(vals)}")
            self.variables.update(zip(self.trainable_vars, vals))

    def get_all_val(self):
        return [self.variables[k] for k in self.trainable_vars]

    def get_all_dic(self, trainable_only=False):
        if trainable_only:
            return {k: self.variables[k] for k in self.trainable_vars}
        return dict(self.variables)

    def complex_value(self, name):
        r = self.variables[name + "r"]
        i = self.variables[name + "i"]
        if self.complex_vars.get(name, self.polar):
            return r * np.cos(i) + 1j * r * np.sin(i)
        return r + 1j * i

    @contextlib.contextmanager
    def temp_params(self, vals):
        old = dict(self.variables)
        self.set_all(vals)
        try:
            yield
        finally:
            self.variables = old

    def std_polar_all(self):
        """Fold polar parameters to r > 0, phi in (-pi, pi]
        (``tf_pwa/variable.py`` std_polar)."""
        for name, polar in self.complex_vars.items():
            if not polar:
                continue
            r, p = self.variables[name + "r"], self.variables[name + "i"]
            if r < 0:
                r, p = -r, p + np.pi
            p = (p + np.pi) % (2 * np.pi) - np.pi
            self.variables[name + "r"], self.variables[name + "i"] = r, p


class Bound:
    """Boundary transform of one fit variable (``tf_pwa/variable.py:1029-1130``,
    default functions): the optimiser works on an unbounded x, the model on
    y = f(x) inside (lower, upper):

    * both bounds: y = (b - a)(sin x + 1)/2 + a
    * lower only:  y = a - 1 + sqrt(x^2 + 1)
    * upper only:  y = b + 1 - sqrt(x^2 + 1)

    Closed forms of f, dy/dx and the inverse (y clipped into the range first,
    the non-negative root of the one-sided forms)."""

    def __init__(self, lower=None, upper=None):
        if lower is not None and upper is not None and lower > upper:
            raise ValueError("lower bound is larger than upper bound")
        self.lower, self.upper = lower, upper

    def x2y(self, x):
        a, b = self.lower, self.upper
        if a is not None and b is not None:
            return (b - a) * (np.sin(x) + 1) / 2 + a
        if a is not None:
            return a - 1 + np.sqrt(x * x + 1)
        if b is not None:
            return b + 1 - np.sqrt(x * x + 1)
        return x

    def dydx(self, x):
        a, b = self.lower, self.upper
        if a is not None and b is not None:
            return (b - a) * np.cos(x) / 2
        if a is not None:
            return x / np.sqrt(x * x + 1)
        if b is not None:
            return -x / np.sqrt(x * x + 1)
        return 1.0

    def y2x(self, y):
        a, b = self.lower, self.upper
        if a is not None:
            y = max(y, a)
        if b is not None:
            y = min(y, b)
        if a is not None and b is not None:
            return float(np.arcsin(np.clip(2 * (y - a) / (b - a) - 1, -1.0, 1.0)))
        if a is not None:
            return float(np.sqrt(max((y - a + 1) ** 2 - 1, 0.0)))
        if b is not None:
            return float(np.sqrt(max((b + 1 - y) ** 2 - 1, 0.0)))
        return float(y)

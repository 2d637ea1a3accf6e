"""Decay topology, spins, LS couplings and constant tables of the model.

This is the host-side model description the engine compiles into a CUDA
kernel.  Conventions follow the reference package (TF-PWA):

* particle / decay / chain objects and their ordering:
  ``tf_pwa/particle.py:56-197`` (BaseParticle, sorting by name),
  ``tf_pwa/particle.py:269-350`` (BaseDecay keeps the config order of outs),
  ``tf_pwa/particle.py:519-545`` (DecayChain sorts ``inner`` and ``outs``),
  ``tf_pwa/particle.py:846-876`` (DecayGroup resonance order).
* LS lists: ``tf_pwa/particle.py:207-248`` (GetA2BC_LS_list).
* CG matrix of a decay vertex: ``tf_pwa/amp/core.py:851-900``.
* d-function weights: ``tf_pwa/dfun.py:118-143``.
* Blatt-Weisskopf polynomial coefficients: ``tf_pwa/breit_wigner.py:332-390``.
"""
from fractions import Fraction
from functools import lru_cache
import math

import numpy as np


# ----------------------------------------------------------------- spins
def spin_int(x):
    """Integer part of a non-negative (half-)integer quantity.

    Mirrors ``tf_pwa/particle.py:49-53``."""
    if isinstance(x, int):
        return x
    return int(x + 0.1)


def two(x):
    """2*x as an exact integer for (half-)integer x."""
    return int(round(2 * float(x)))


def spin_range(a, b):
    """a, a+1, ..., b (``tf_pwa/particle.py:43-46``)."""
    out = []
    while a <= b + 1e-9:
        out.append(a)
        a = a + 1
    return out


def parse_spin(J):
    """Config spin values: 1, 0.5, "1/2", "3/2"."""
    if isinstance(J, str):
        return float(Fraction(J))
    return float(J) if not isinstance(J, int) else J


def ls_list(ja, jb, jc, pa=None, pb=None, pc=None, p_break=False, ca=None):
    """Allowed (l, s) pairs for a -> b c.

    Restates ``GetA2BC_LS_list`` (``tf_pwa/particle.py:207-248``): s runs
    over |jb-jc|..jb+jc, l over |ja-s|..ja+s, parity selects
    pa = pb pc (-1)^l unless the decay breaks parity, and an optional C
    parity selects ca = (-1)^(l+s)."""
    if pa is None or pb is None or pc is None:
        p_break = True
    if not p_break:
        dl = 0 if pa * pb * pc == 1 else 1
    ret = []
    for s in spin_range(abs(jb - jc), jb + jc):
        for l in spin_range(abs(ja - s), ja + s):
            if 0.3 < l % 1.0 < 0.7:
                break
            l = spin_int(l)
            if ca is not None and ca != (-1) ** (l + s):
                continue
            if not p_break:
                if l % 2 == dl:
                    ret.append((l, s))
            else:
                ret.append((l, s))
    return ret


# ------------------------------------------------------------ CG (Racah)
@lru_cache(maxsize=None)
def _fact2(n2):
    """(n2/2)! for an even integer n2 >= 0."""
    assert n2 % 2 == 0 and n2 >= 0
    return math.factorial(n2 // 2)


@lru_cache(maxsize=None)
def clebsch_gordan(j1, m1, j2, m2, j, m):
    """<j1 m1; j2 m2 | j m> from Racah's closed formula, exact in rationals.

    Arguments are (half-)integers; the value is returned as a float.  Used in
    place of the sympy call of ``tf_pwa/cg.py:18-26`` (same quantity)."""
    J1, M1, J2, M2, J, M = (two(x) for x in (j1, m1, j2, m2, j, m))
    if M1 + M2 != M:
        return 0.0
    if abs(M1) > J1 or abs(M2) > J2 or abs(M) > J:
        return 0.0
    if J < abs(J1 - J2) or J > J1 + J2 or (J1 + J2 + J) % 2:
        return 0.0
    if (J1 + M1) % 2 or (J2 + M2) % 2 or (J + M) % 2:
        return 0.0
    f = _fact2
    pre = Fraction(
        (J + 1) * f(J + J1 - J2) * f(J - J1 + J2) * f(J1 + J2 - J),
        f(J1 + J2 + J + 2),
    )
    pre *= f(J + M) * f(J - M) * f(J1 - M1) * f(J1 + M1) * f(J2 - M2) * f(J2 + M2)
    s = Fraction(0)
    k = 0
    while True:
        a = [
            2 * k,
            J1 + J2 - J - 2 * k,
            J1 - M1 - 2 * k,
            J2 + M2 - 2 * k,
            J - J2 + M1 + 2 * k,
            J - J1 - M2 + 2 * k,
        ]
        if a[1] < 0 or a[2] < 0 or a[3] < 0:
            break
        if a[4] >= 0 and a[5] >= 0:
            den = 1
            for x in a:
                den *= f(x)
            s += Fraction((-1) ** k, den)
        k += 1
    # sqrt of the rational prefactor, then the sign-carrying sum
    return float(s) * math.sqrt(float(pre))


def cg_matrix(ja, jb, jc, ls, hel_b, hel_c):
    """[(l,s), lambda_b, lambda_c] factors of the helicity coupling.

    sqrt((2l+1)/(2ja+1)) <jb lb; jc -lc | s lb-lc> <l 0; s lb-lc | ja lb-lc>
    as in ``tf_pwa/amp/core.py:851-900``."""
    ret = np.zeros((len(ls), len(hel_b), len(hel_c)))
    for i, (l, s) in enumerate(ls):
        for ib, lb in enumerate(hel_b):
            for ic, lc in enumerate(hel_c):
                d = lb - lc
                ret[i, ib, ic] = (
                    math.sqrt(2 * l + 1)
                    / math.sqrt(2 * ja + 1)
                    * clebsch_gordan(jb, lb, jc, -lc, s, d)
                    * clebsch_gordan(l, 0, s, d, ja, d)
                )
    return ret


@lru_cache(maxsize=None)
def small_d_weight(j2):
    """w[l, a, b] with d^j_{m' m}(beta) = sum_l w[l, a, b] x^l y^(2j - l),
    x = sin(beta/2), y = cos(beta/2), a = m' + j, b = m + j, ``j2`` = 2j.

    Derived from the spinor (two-variable polynomial) picture of SU(2):
    |j m> is u^(j+m) v^(j-m) / sqrt((j+m)! (j-m)!), and the rotation about y
    maps u -> y u + x v, v -> -x u + y v (the spin-1/2 matrix
    [[y, -x], [x, y]]).  Expanding (y u + x v)^(j+m) (-x u + y v)^(j-m) with
    binomials, the coefficient of u^(j+m') v^(j-m') times
    sqrt((j+m')! (j-m')! / ((j+m)! (j-m)!)) is d^j_{m' m}.  Integer
    binomial sums, one square root per (m', m).  The table is the same
    quantity as ``tf_pwa/dfun.py:118-143`` (pinned to it in the tests)."""
    n = j2  # 2j
    ret = np.zeros((n + 1, n + 1, n + 1))
    fact = math.factorial
    for b in range(n + 1):  # m + j
        up, dn = b, n - b  # powers of u and v in |j m>
        for a in range(n + 1):  # m' + j
            # coefficient of u^a v^(n-a): choose p u's from the first
            # factor (weight y^p x^(up-p)) and q = a - p from the second
            # (weight (-x)^q y^(dn-q)); the power of x is up - p + q
            coef = {}
            for p in range(max(0, a - dn), min(up, a) + 1):
                q = a - p
                c = math.comb(up, p) * math.comb(dn, q) * (-1) ** q
                lx = up - p + q
                coef[lx] = coef.get(lx, 0) + c
            norm = math.sqrt(fact(a) * fact(n - a) / (fact(b) * fact(n - b)))
            for lx, c in coef.items():
                ret[lx, a, b] = c * norm
    return ret


@lru_cache(maxsize=None)
def bprime_coeff(l):
    """Coefficients c_0..c_l (highest power first) of the Blatt-Weisskopf
    polynomial |theta_l(i w)|^2 in z = w^2, theta_l the reverse Bessel
    polynomial.  Equals the table of ``tf_pwa/breit_wigner.py:319-327`` for
    l <= 5 and the generator of ``tf_pwa/breit_wigner.py:358-390`` above."""
    # theta_l(x) = sum_k (l+k)! / ((l-k)! k! 2^k) x^(l-k); evaluate
    # |theta(i w)|^2 as a polynomial in w^2 with exact rationals.
    a = [Fraction(math.factorial(l + k), math.factorial(l - k) * math.factorial(k) * 2 ** k) for k in range(l + 1)]
    # theta(iw) = sum_k a_k (i w)^(l-k); coefficient of w^p is a_{l-p} i^p
    re = {}
    im = {}
    for k in range(l + 1):
        p = l - k
        ph = p % 4
        if ph == 0:
            re[p] = re.get(p, 0) + a[k]
        elif ph == 1:
            im[p] = im.get(p, 0) + a[k]
        elif ph == 2:
            re[p] = re.get(p, 0) - a[k]
        else:
            im[p] = im.get(p, 0) - a[k]
    sq = {}
    for d in (re, im):
        for p1, c1 in d.items():
            for p2, c2 in d.items():
                sq[p1 + p2] = sq.get(p1 + p2, 0) + c1 * c2
    # powers of w^2 from highest (w^{2l}) to constant
    return [float(sq.get(2 * l - 2 * i, 0)) for i in range(l + 1)]


# ------------------------------------------------------------ topology
class Particle:
    """A particle of the model (``tf_pwa/particle.py:56-197`` plus the
    lineshape options of ``tf_pwa/amp/core.py:349-418``)."""

    def __init__(self, name, J=0, P=-1, C=None, spins=None, mass=None, width=None,
                 model="default", id_=0, **kw):
        self.name = name
        self.id = id_
        self.J = parse_spin(J)
        self.P = P
        self.C = C
        if spins is None:
            spins = tuple(spin_range(-self.J, self.J))
        self.spins = tuple(parse_spin(s) for s in spins)
        self.mass = None if mass is None else float(mass)
        self.width = None if width is None else float(width)
        self.model = model
        self.bw_l = kw.pop("bw_l", None)
        self.running_width = kw.pop("running_width", True)
        self.width_norm = kw.pop("width_norm", False)
        self.float = kw.pop("float", "")
        self.params = kw.pop("params", None)
        # "vector": the parent's spin density matrix is fitted
        # (tf_pwa/amp/core.py:1647-1671,1965-2000)
        self.polarization = kw.pop("polarization", "none") or "none"
        self.d = 3.0
        self.extra = kw
        self.decay = []      # decays of this particle (config order)
        self.creators = []   # decays producing it

    def __repr__(self):
        return self.name if self.id == 0 else f"{self.name}:{self.id}"

    def key(self):
        return (self.name, self.id)

    def __lt__(self, other):
        return self.key() < other.key()

    def __eq__(self, other):
        return isinstance(other, Particle) and self.key() == other.key()

    def __hash__(self):
        return hash(self.key())

    @property
    def params_head(self):
        return str(self)

    def lineshape_kind(self):
        """'one' (no width), 'BW' (fixed width), 'BWR' (running width from
        |q|, |q0|: ``tf_pwa/amp/core.py:399-418``) or 'BWR2' (running width
        from q^2, q0^2, complex below threshold: ``tf_pwa/amp/base.py:37-73``)."""
        if self.width is None or self.model == "one":
            return "one"
        if self.model in ("BW",) or not self.running_width:
            return "BW"
        if self.model in ("default", "BWR", None):
            return "BWR"
        if self.model == "BWR2":
            return "BWR2"
        raise NotImplementedError(f"lineshape model {self.model!r} of {self}")

    def width_norm_applies(self):
        """R -> Gamma0 R: the ``width_norm`` option of the default particle
        class (``tf_pwa/amp/core.py:415-417``); the BW and BWR2 classes
        ignore it."""
        return bool(self.width_norm) and self.width is not None and \
            self.model in ("default", "BWR", None)


class Decay:
    """Two-body vertex a -> b c with the helicity-coupling options of
    ``tf_pwa/amp/core.py:650-780``."""

    def __init__(self, core, outs, p_break=False, c_break=True, **kw):
        self.core = core
        self.outs = tuple(outs)
        if len(self.outs) != 2:
            raise NotImplementedError("only two-body vertices are supported")
        self.p_break = p_break
        self.c_break = c_break
        self.has_barrier_factor = kw.pop("has_barrier_factor", True)
        self.has_bprime = kw.pop("has_bprime", True)
        self.has_ql = kw.pop("has_ql", True)
        self.barrier_factor_norm = kw.pop("barrier_factor_norm", False)
        self.no_q0 = kw.pop("no_q0", False)
        self.l_list_sel = kw.pop("l_list", None)
        ls_sel = kw.pop("ls_list", None)
        self.ls_sel = None if ls_sel is None else tuple(tuple(i) for i in ls_sel)
        self.params_polar = kw.pop("params_polar", None)
        # per-event charge conjugation flips this vertex's helicity coupling
        # (tf_pwa/amp/core.py:697-716,938-945)
        self.allow_cc = kw.pop("allow_cc", True)
        kw.pop("model", None)
        kw.pop("curve_style", None)
        for k in ("below_threshold", "barrier_factor_mass", "force_min_l", "aligned",
                  "helicity_inner_full", "ls_selector"):
            if kw.pop(k, False):
                raise NotImplementedError(f"decay option {k} is not supported")
        self.extra = kw
        self.d = 3.0
        self._ls = None

    def __repr__(self):
        return f"{self.core}->" + "+".join(str(i) for i in self.outs)

    def key(self):
        return (self.core.key(), tuple(sorted(o.key() for o in self.outs)))

    def __eq__(self, other):
        return isinstance(other, Decay) and self.key() == other.key()

    def __hash__(self):
        return hash(self.key())

    def __lt__(self, other):
        return self.key() < other.key()

    @property
    def params_head(self):
        return var_name(str(self.core) + "->" + "+".join(str(o) for o in self.outs))

    def get_ls_list(self):
        if self._ls is None:
            ca = self.core.C if not self.c_break else None
            b, c = self.outs
            ls = ls_list(self.core.J, b.J, c.J, self.core.P, b.P, c.P, self.p_break, ca)
            ls = tuple(ls)
            if self.ls_sel is not None:
                ls = self.ls_sel
            if self.l_list_sel is not None:
                ls = tuple((l, s) for l, s in ls if l in self.l_list_sel)
            self._ls = ls
        return self._ls

    def get_l_list(self):
        return tuple(l for l, s in self.get_ls_list())

    def hel_inner(self):
        """Helicity lists of the outs used inside the vertex."""
        return [o.spins for o in self.outs]

    def cg(self):
        hb, hc = self.hel_inner()
        b, c = self.outs
        return cg_matrix(self.core.J, b.J, c.J, self.get_ls_list(), hb, hc)


def var_name(s):
    """Parameter-name mangling of ``tf_pwa/amp/core.py:228-238``."""
    return (s.replace(":", "/").replace("+", ".").replace(",", "")
            .replace("[", "").replace("]", "").replace(" ", ""))


class DecayChain:
    """Ordered list of decays from the top particle to the final state."""

    def __init__(self, decays):
        self.decays = list(decays)
        self.is_cp = False   # CP-violating total: one value per event charge
        cores = {d.core for d in self.decays}
        outs = set()
        for d in self.decays:
            outs.update(d.outs)
        top = cores - outs
        assert len(top) == 1
        self.top = top.pop()
        self.inner = sorted(cores & outs)
        self.outs = sorted(outs - cores)

    def __iter__(self):
        return iter(self.decays)

    def __len__(self):
        return len(self.decays)

    def __repr__(self):
        return "[" + ", ".join(str(d) for d in self.decays) + "]"

    @property
    def params_head(self):
        return var_name("[" + ", ".join(str(d.core) + "->" + "+".join(str(o) for o in d.outs)
                                        for d in self.decays) + "]")

    def decay_of(self, particle):
        for d in self.decays:
            if d.core == particle:
                return d
        return None

    def creator_of(self, particle):
        for d in self.decays:
            if particle in d.outs:
                return d
        return None

    def final_set(self, p):
        """Final particles below node p (sorted)."""
        if p in self.outs:
            return (p,)
        d = self.decay_of(p)
        out = []
        for o in d.outs:
            out += list(self.final_set(o))
        return tuple(sorted(out))


class DecayGroup:
    """All chains of the model with the same top and final particles."""

    def get_decay_chain(self, id_):
        """Chain by index, or the first chain holding every named particle
        (a "R1/R2" string, a list, or a particle) (``tf_pwa/particle.py:
        888-956``)."""
        if isinstance(id_, int):
            return self.chains[id_]
        if isinstance(id_, str):
            names = id_.split("/")
        elif isinstance(id_, (list, tuple)):
            names = [str(i) for i in id_]
        else:
            names = [str(id_)]
        for c in self.chains:
            have = {str(p) for p in [c.top] + list(c.inner) + list(c.outs)}
            if all(n in have for n in names):
                return c
        raise ValueError(f"Not found such decay chain: {names}")

    def __init__(self, chains):
        self.chains = list(chains)
        self.identical_particles = None
        self.cp_particles = None
        self.charge = False       # per-event charge_conjugation field in use
        self.cp_trans = True      # parity-transform charge < 0 momenta
        self.random_z = True      # moving parent: flight direction as z
        self.top = self.chains[0].top
        self.outs = sorted(self.chains[0].outs)
        for c in self.chains:
            assert c.top == self.top and c.outs == self.chains[0].outs
        res = []
        for c in self.chains:
            for p in c.inner:
                if p not in res:
                    res.append(p)
        self.resonances = res

    def __iter__(self):
        return iter(self.chains)

    def __len__(self):
        return len(self.chains)

    def __getitem__(self, i):
        return self.chains[i]

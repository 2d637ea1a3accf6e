"""CPU FP64 oracle of TF-PWA's amplitude-fit hot path (numpy restatement).

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA engine:
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may import it; the product path never does.

It restates, function by function, the reference's algorithm on the same
per-event inputs (invariant masses and helicity / alignment angles):

* small-d weights and d(beta): ``tf_pwa/dfun.py:118-173``
* exp(i m theta) and conjugated D: ``tf_pwa/dfun.py:176-218``
* D gathered to [lambda_a, lambda_b - lambda_c] with zeros outside |.|<=j:
  ``tf_pwa/dfun.py:63-115,241-266``
* CG coefficients with sympy, as ``tf_pwa/cg.py:18-26``; vertex CG matrix
  ``tf_pwa/amp/core.py:851-900``
* relative momenta q (clamped) and q^2 (unclamped): ``tf_pwa/amp/core.py:311-334``
* Blatt-Weisskopf polynomial / B'_l(q^2): ``tf_pwa/breit_wigner.py:268-355``
* barrier factor q^l B'_l of each LS: ``tf_pwa/amp/core.py:1072-1097``
* helicity coupling H = sum_ls g_ls bf_ls CG_ls, reversed for charge < 0
  events: ``tf_pwa/amp/core.py:931-947,1025-1043``
* decay amplitude H * D*: ``tf_pwa/amp/core.py:1149-1164``
* lineshapes BWR / BW with running width Gamma(m): ``tf_pwa/breit_wigner.py:56-91,231-245``,
  BWR2 with Gamma2(m) from q^2: ``tf_pwa/breit_wigner.py:193-210,248-265``,
  particle model ``tf_pwa/amp/core.py:349-418``
* chain contraction with totals and alignment D's: ``tf_pwa/amp/core.py:1392-1445,1563-1604``
* sum over chains and |A|^2: ``tf_pwa/amp/core.py:1696-1728,1919-1931``;
  identical-particle and CP-conjugate swaps ``tf_pwa/amp/core.py:1826-1913``
* clip_log and the weighted NLL with alpha scaling and normalised MC
  weights: ``tf_pwa/model/model.py:283-292,407-449,603-641,1126-1229``

Gradients: couplings enter linearly (A = sum_k c_k F_k), so their gradient
is exact here; masses and widths use a 4-point central differences of this
FP64 function, Richardson-extrapolated.
"""
import math
from functools import lru_cache

import numpy as np

_EPS_CLIP = 1e-6


# ----------------------------------------------------------- D functions
@lru_cache(maxsize=None)
def d_weight(j2):
    """Wigner weights w[l, m1 + j, m2 + j] for spin j = j2/2: the coefficient
    of sin^l(b/2) cos^(2j-l)(b/2) in d^j_{m1 m2}(b), the quantity of
    ``tf_pwa/dfun.py:118-143``.  Written from Wigner's explicit sum
    d = sum_s (-1)^(m1-m2+s) sqrt((j+m1)!(j-m1)!(j+m2)!(j-m2)!)
        / ((j+m2-s)! s! (m1-m2+s)! (j-m1-s)!) cos^(2j+m2-m1-2s) sin^(m1-m2+2s),
    with all quantities in units of 1/2 kept as integers (a = j+m1,
    b = j+m2 are integers)."""
    n = j2
    fa = math.factorial
    ret = np.zeros((n + 1, n + 1, n + 1))
    for a in range(n + 1):          # j + m1
        for b in range(n + 1):      # j + m2
            dm = a - b              # m1 - m2
            root = math.sqrt(fa(a) * fa(n - a) * fa(b) * fa(n - b))
            for s_ in range(max(0, -dm), min(b, n - a) + 1):
                den = fa(b - s_) * fa(s_) * fa(dm + s_) * fa(n - a - s_)
                ret[dm + 2 * s_, a, b] += (-1) ** (dm + s_) * root / den
    return ret


def small_d(beta, j2):
    """(N, j2+1, j2+1) d^j_{m1 m2}(beta) (dfun.py:146-173)."""
    a = np.arange(j2 + 1, dtype=np.float64)[None, :]
    s = np.sin(0.5 * beta)[:, None]
    c = np.cos(0.5 * beta)[:, None]
    sc = s ** a * c ** (j2 - a)
    w = d_weight(j2).reshape(j2 + 1, -1)
    return (sc @ w).reshape(-1, j2 + 1, j2 + 1)


def D_conj(alpha, beta, gamma, j2):
    """e^{i m1 alpha} d^j_{m1 m2}(beta) e^{i m2 gamma} (dfun.py:196-218)."""
    m = np.arange(-j2 / 2, j2 / 2 + 1, 1)[None, :]
    d = small_d(beta, j2)
    ea = np.exp(1j * m * alpha[:, None])[:, :, None]
    eg = np.exp(1j * m * gamma[:, None])[:, None, :]
    return ea * eg * d


def D_lambda(alpha, beta, gamma, ja, la, lb, lc=(0,)):
    """D* gathered to (N, la, lb, lc): element [lambda_a, lambda_b - lambda_c],
    zero where |lambda_b - lambda_c| > ja (dfun.py:63-115)."""
    j2 = int(round(2 * ja))
    D = D_conj(alpha, beta, gamma, j2).reshape(-1, (j2 + 1) ** 2)
    D = np.concatenate([D, np.zeros((D.shape[0], 1), D.dtype)], axis=1)
    idx = []
    for a in la:
        for b in lb:
            for c in lc:
                dl = b - c
                if abs(dl) <= ja:
                    idx.append(int(round(a + ja)) * (j2 + 1) + int(round(dl + ja)))
                else:
                    idx.append((j2 + 1) ** 2)
    return D[:, idx].reshape(-1, len(la), len(lb), len(lc))


# ----------------------------------------------------------- CG
@lru_cache(maxsize=None)
def cg_coef(jb, jc, mb, mc, ja, ma):
    """<jb mb; jc mc | ja ma> from sympy, as in tf_pwa/cg.py:18-26."""
    from sympy import Rational
    from sympy.physics.quantum.cg import CG

    r = lambda x: Rational(int(round(2 * x)), 2)  # noqa: E731
    return float(CG(r(jb), r(mb), r(jc), r(mc), r(ja), r(ma)).doit().evalf())


def cg_matrix(ja, jb, jc, ls, hb, hc):
    ret = np.zeros((len(ls), len(hb), len(hc)))
    for i, (l, s) in enumerate(ls):
        for ib, lb in enumerate(hb):
            for ic, lc in enumerate(hc):
                ret[i, ib, ic] = (
                    np.sqrt(2 * l + 1) / np.sqrt(2 * ja + 1)
                    * cg_coef(jb, jc, lb, -lc, s, lb - lc)
                    * cg_coef(l, s, 0, lb - lc, ja, lb - lc)
                )
    return ret


# ----------------------------------------------------------- lineshapes
def rel_p(m0, m1, m2):
    """|q| with the mass clamped at threshold (core.py:311-321)."""
    s, d = m1 + m2, m1 - m2
    m_eff = np.where(m0 > s, m0, s)
    p = (m_eff - s) * (m_eff + s) * (m_eff - d) * (m_eff + d)
    return np.sqrt(p) / (2 * m_eff)


def rel_p2(m0, m1, m2):
    """|q|^2, unclamped (core.py:324-334)."""
    s, d = m1 + m2, m1 - m2
    p = (m0 - s) * (m0 + s) * (m0 - d) * (m0 + d)
    return p / (2 * m0) ** 2


@lru_cache(maxsize=None)
def bprime_coef(l):
    """|theta_l(i w)|^2 coefficients, highest power first (breit_wigner.py:319-390)."""
    table = {
        0: [1.0],
        1: [1.0, 1.0],
        2: [1.0, 3.0, 9.0],
        3: [1.0, 6.0, 45.0, 225.0],
        4: [1.0, 10.0, 135.0, 1575.0, 11025.0],
        5: [1.0, 15.0, 315.0, 6300.0, 99225.0, 893025.0],
    }
    if l in table:
        return table[l]
    import sympy as sym

    x = sym.Symbol("x")
    th = sum(sym.Rational(math.factorial(l + k), math.factorial(l - k) * math.factorial(k) * 2 ** k)
             * x ** (l - k) for k in range(l + 1))
    w = sym.Symbol("w", real=True)
    h = th.subs({x: sym.I * w})
    poly = sym.Poly(sym.expand(h * sym.conjugate(h)), w).as_dict()
    return [float(poly.get((2 * l - 2 * i,), 0)) for i in range(l + 1)]


def bprime_poly(l, z):
    r = np.zeros_like(z)
    for c in bprime_coef(l):
        r = r * z + c
    return r


def bprime_q2(l, q2, q02, d):
    bp = bprime_poly(l, q02 * d * d) / bprime_poly(l, q2 * d * d)
    return np.sqrt(np.where(bp > 0, bp, 1.0))


def bprime(l, q, q0, d):
    return np.sqrt(bprime_poly(l, (q0 * d) ** 2)) / np.sqrt(bprime_poly(l, (q * d) ** 2))


def gamma_running(m, g0, q, q0, L, m0, d):
    ok = q0 > 1e-15
    qq0 = np.where(ok, (q / np.where(ok, q0, 1.0)) ** (2 * L + 1), 1.0)
    return g0 * qq0 * (m0 / m) * bprime(L, q, q0, d) ** 2


def bwr(m, m0, g0, q, q0, L, d):
    g = gamma_running(m, g0, q, q0, L, m0, d)
    x = m0 * m0 - m * m
    y = m0 * g
    s = x * x + y * y
    return x / s + 1j * y / s


def gamma2(m, g0, q2, q02, L, m0, d):
    """Running width from q^2 and q0^2 (``tf_pwa/breit_wigner.py:248-265``):
    (q^2/q0^2)^L sqrt(q^2/q0^2) on the principal complex branch, so the
    width is imaginary where q^2/q0^2 < 0 (nominal mass below threshold)."""
    r = q2 / q02
    qq0 = (r ** L).astype(complex) * np.sqrt(r.astype(complex))
    bp = bprime_poly(L, q02 * d * d) / bprime_poly(L, q2 * d * d)
    return qq0 * (g0 * bp * m0 / m)


def bwr2(m, m0, g0, q2, q02, L, d):
    """BWR2 (``tf_pwa/breit_wigner.py:193-210``): with D = m0^2 - m^2 -
    i m0 Gamma2(m), the value (Re D + i Im D) / |D|^2."""
    g = gamma2(m, g0, q2, q02, L, m0, d)
    dd = (m0 * m0 - m * m) - 1j * (m0 * g)
    r2 = dd.real ** 2 + dd.imag ** 2
    return dd.real / r2 + 1j * dd.imag / r2


def bw(m, m0, g0):
    x = m0 * m0 - m * m
    y = m0 * g0
    s = x * x + y * y
    return x / s + 1j * y / s


# ----------------------------------------------------------- model
class OracleModel:
    """Amplitude of a decay group on per-event fields.

    ``group`` is the topology object of the engine's model compiler (chains,
    decays, spins, LS lists -- cross-checked against the reference), ``plan``
    maps every chain vertex to its input columns."""

    def __init__(self, group, plan):
        self.group = group
        self.plan = plan
        self.letters = {}
        gen = iter("abcdefghijklmnopqrstuvwxyz")
        self.letters[group.top] = next(gen)
        for o in group.outs:
            self.letters[o] = next(gen)
        for c in group:
            for p in c.inner:
                if p not in self.letters:
                    self.letters[p] = next(gen)

    # --- parameters ------------------------------------------------------
    @staticmethod
    def complex_of(vm_vals, polar, name):
        r = vm_vals[name + "r"]
        i = vm_vals[name + "i"]
        if polar.get(name, True):
            return r * np.cos(i) + 1j * r * np.sin(i)
        return r + 1j * i

    def couplings(self, vals, polar):
        """Per chain: total, per decay g_ls vectors (all complex)."""
        out = []
        from_names = {}
        for c in self.group:
            tn = c.params_head + "_total_0"
            if getattr(c, "is_cp", False):
                # CP-violating total: (r +- deltar, i +- deltai) for charge +-1
                # (tf_pwa/variable.py:1715-1734, tf_pwa/amp/core.py:1380-1390)
                r, i, dr, di = (vals[tn + x] for x in ("r", "i", "deltar", "deltai"))
                tot = tuple((r + s_ * dr) * np.exp(1j * (i + s_ * di)) for s_ in (1.0, -1.0))
            else:
                tot = self.complex_of(vals, polar, tn)
            gl = []
            for d in c:
                n = len(d.get_ls_list())
                gl.append(np.array([self.complex_of(vals, polar, f"{d.params_head}_g_ls_{i}")
                                    for i in range(n)]))
            out.append((tot, gl))
        return out

    @staticmethod
    def mass_of(vals, p):
        n = f"{p.params_head}_mass"
        return vals.get(n, p.mass)

    @staticmethod
    def width_of(vals, p):
        n = f"{p.params_head}_width"
        return vals.get(n, p.width)

    # --- per decay --------------------------------------------------------
    def data_mass(self, x, cf, p, chain):
        if p in chain.inner:
            return x[cf["mass"][p]]
        return np.full(x.shape[1], p.mass)

    def decay_amp(self, x, cf, chain, k, d, vals, gls, per_ls=False):
        """(N, n_a, n_b, n_c) complex amplitude of vertex d (core.py:1149-1164);
        with ``per_ls`` the term of every LS coupling apart, (N, n_ls, n_a,
        n_b, n_c), at unit coupling."""
        a, (b, c) = d.core, d.outs
        f = cf["decays"][k]
        alpha, beta = x[f["alpha"]], x[f["beta"]]
        Dc = D_lambda(alpha, beta, np.zeros_like(alpha), a.J, a.spins, b.spins, c.spins)
        # q^2 from data masses, q0^2 from nominal (possibly floating) masses
        m0d = self.data_mass(x, cf, a, chain)
        m1d = self.data_mass(x, cf, b, chain)
        m2d = self.data_mass(x, cf, c, chain)
        q2 = rel_p2(m0d, m1d, m2d)
        m0n = self.mass_of(vals, a) if a in chain.inner else a.mass
        m1n = self.mass_of(vals, b) if b in chain.inner else b.mass
        m2n = self.mass_of(vals, c) if c in chain.inner else c.mass
        q02 = rel_p2(m0n, m1n, m2n)
        ls = d.get_ls_list()
        if d.has_barrier_factor:
            q02u = 1.0 if d.no_q0 else q02
            bfs = []
            for l, s in ls:
                if d.has_bprime:
                    bp = bprime_q2(l, q2, q02u, d.d)
                    t = q2 ** (l / 2) * bp if d.has_ql else np.ones_like(q2) * bp
                    if d.barrier_factor_norm:
                        t = t / np.abs(q02u) ** (l / 2)
                else:
                    t = q2 ** (l / 2) if d.has_ql else np.ones_like(q2)
                bfs.append(t)
            bfv = np.stack(bfs, -1)
        else:
            bfv = np.ones((x.shape[1], len(ls)))
        cg = cg_matrix(a.J, b.J, c.J, ls, b.spins, c.spins)
        if per_ls:
            H = np.einsum("nl,lbc->nlbc", bfv, cg)
        else:
            H = np.einsum("nl,lbc->nbc", gls[None, :] * bfv, cg)
        ci = getattr(self.plan, "charge_index", None)
        if ci is not None and d.allow_cc:
            # charge < 0: H[..., ::-1, ::-1] (core.py:938-945)
            pos = (x[ci] > 0).reshape((-1,) + (1,) * (H.ndim - 1))
            H = np.where(pos, H, H[..., ::-1, ::-1])
        if per_ls:
            return H[:, :, None, :, :] * Dc[:, None]
        return H[:, None, :, :] * Dc

    def lineshape(self, x, cf, chain, p, vals):
        """Particle.get_amp (core.py:399-418)."""
        kind = p.lineshape_kind()
        m = x[cf["mass"][p]]
        if kind == "one":
            return np.ones_like(m) + 0j
        m0 = self.mass_of(vals, p)
        g0 = self.width_of(vals, p)
        if kind == "BW":
            ret = bw(m, m0, g0)
        else:
            d = chain.decay_of(p)
            b, c = d.outs
            m1d, m2d = self.data_mass(x, cf, b, chain), self.data_mass(x, cf, c, chain)
            m1n = self.mass_of(vals, b) if b in chain.inner else b.mass
            m2n = self.mass_of(vals, c) if c in chain.inner else c.mass
            L = p.bw_l if p.bw_l is not None else min(d.get_l_list())
            if kind == "BWR2":  # tf_pwa/amp/base.py:61-73
                ret = bwr2(m, m0, g0, rel_p2(m, m1d, m2d), rel_p2(m0, m1n, m2n), L, p.d)
            else:
                ret = bwr(m, m0, g0, rel_p(m, m1d, m2d), rel_p(m0, m1n, m2n), L, p.d)
        if p.width_norm_applies():  # core.py:415-417 (Particle class only)
            ret = g0 * ret
        return ret

    def chain_amp(self, x, ci, vals, coup, cf=None, per_ls=False):
        """Amplitude of chain ci (``tf_pwa/amp/core.py:1392-1445``); with
        ``per_ls`` one term per combination of LS couplings (one per vertex)
        at unit couplings and unit total, (N, n_ls_1, n_ls_2, ..., helicities)."""
        chain = self.group[ci]
        cf = self.plan.chains[ci] if cf is None else cf
        tot, gl = coup[ci]
        L = self.letters
        ops, idx = [], []
        ls_letters = "ZYXWVUTS"
        for k, d in enumerate(chain):
            ops.append(self.decay_amp(x, cf, chain, k, d, vals, gl[k], per_ls))
            idx.append("..." + (ls_letters[k] if per_ls else "")
                       + "".join(L[p] for p in (d.core,) + d.outs))
        rs = np.ones(x.shape[1], dtype=np.complex128)
        for p in chain.inner:
            rs = rs * self.lineshape(x, cf, chain, p, vals)
        if per_ls:
            tot = 1.0
        elif isinstance(tot, tuple):
            ci_ = getattr(self.plan, "charge_index", None)
            tot = tot[0] if ci_ is None else np.where(x[ci_] > 0, tot[0], tot[1])
        ops.append(tot * rs)
        idx.append("...")
        final = "..." + (ls_letters[:len(chain)] if per_ls else "") + "".join(
            L[p] for p in [self.group.top] + list(self.group.outs))
        for k, d in enumerate(chain):
            for o in d.outs:
                if o in cf["aligned"] and o.J != 0:
                    fa, fb, fg = cf["aligned"][o]
                    dt = D_lambda(x[fa], x[fb], x[fg], o.J, o.spins, o.spins)[..., 0]
                    ops.append(dt)
                    idx.append("..." + L[o] + L[o].upper())
                    final = final.replace(L[o], L[o].upper())
        return np.einsum(",".join(idx) + "->" + final, *ops, optimize=per_ls)

    def amp(self, x, vals, polar=None):
        """Sum over chains (``core.py:1696-1728``); with identical particles
        plus, per swap, the sign times the amplitude of the swapped fields
        with its final-helicity axes reordered (``core.py:1871-1882``)."""
        polar = polar or {}
        coup = self.couplings(vals, polar)
        a = sum(self.chain_amp(x, ci, vals, coup) for ci in range(len(self.group)))
        for sw in self.plan.swaps:
            b = sum(self.chain_amp(x, ci, vals, coup, sw["chains"][ci])
                    for ci in range(len(self.group)))
            b = np.transpose(b, [0, 1] + [2 + t for t in sw["trans"]])
            if sw["flip"]:  # CP-conjugate: every helicity reversed (core.py:1899-1911)
                b = b[(slice(None),) + (slice(None, None, -1),) * (b.ndim - 1)]
            a = a + sw["factor"] * b
        return a

    def columns(self, x, vals, polar=None):
        """Partial-wave columns of the amplitude: A = sum_k c_k F_k with
        c_k = chain total x one LS coupling per vertex.  Returns F
        (N, K, n_out) and, per column, (total name, [g_ls names]).  Column k
        is the chain amplitude with that total and those couplings set to 1
        and the vertex's other LS couplings to 0 (H is linear in the g_ls,
        ``tf_pwa/amp/core.py:931-947``), identical-particle swaps summed in
        with their signs as in :meth:`amp`.  With the columns, one pass
        gives the NLL and every coupling derivative (what the reference's
        GradientTape pass over ``FCN.nll_grad`` produces)."""
        import itertools

        polar = polar or {}
        if self.density(vals) is not None or any(getattr(c, "is_cp", False)
                                                 for c in self.group):
            raise ValueError("columns: unpolarised models without CP-violating totals only")
        coup = self.couplings(vals, polar)
        cols, names = [], []
        for ci, chain in enumerate(self.group):
            nls = [len(d.get_ls_list()) for d in chain]
            nv = len(chain)
            a = self.chain_amp(x, ci, vals, coup, per_ls=True)
            for sw in self.plan.swaps:
                b = self.chain_amp(x, ci, vals, coup, sw["chains"][ci], per_ls=True)
                # helicity axes follow the nv LS axes
                b = np.transpose(b, list(range(2 + nv)) + [2 + nv + t for t in sw["trans"]])
                if sw["flip"]:
                    b = b[(slice(None),) * (1 + nv) + (slice(None, None, -1),) * (b.ndim - 1 - nv)]
                a = a + sw["factor"] * b
            a = a.reshape(a.shape[0], int(np.prod(nls)), -1)
            for q, combo in enumerate(itertools.product(*[range(n) for n in nls])):
                cols.append(a[:, q])
                names.append((chain.params_head + "_total_0",
                              [f"{d.params_head}_g_ls_{l}" for d, l in zip(chain, combo)]))
        return np.stack(cols, 1), names

    def density(self, vals):
        """Spin density matrix of a vector-polarised parent
        (``tf_pwa/amp/core.py:1965-2000``), None when unpolarised."""
        top = self.group.top
        if getattr(top, "polarization", "none") == "none":
            return None
        h = str(top)
        if top.J == 0.5:
            px, py, pz = (vals[f"{h}_polarization_p{c}"] for c in "xyz")
            return 0.5 * np.array([[1 + pz, px - 1j * py], [px + 1j * py, 1 - pz]])
        p = [vals[f"{h}_polarization_p_{i}"] for i in range(8)]
        r3 = np.sqrt(3.0)
        return np.array([
            [1 + p[2] + p[7] / r3, p[0] - 1j * p[1], p[3] - 1j * p[4]],
            [p[0] + 1j * p[1], 1 - p[2] + p[7] / r3, p[5] - 1j * p[6]],
            [p[3] + 1j * p[4], p[5] + 1j * p[6], 1 - 2 * p[7] / r3]])

    def pdf(self, x, vals, polar=None):
        """sum |A|^2, or sum_l A_al rho_ab A_bl^* for a polarised parent
        (``tf_pwa/amp/core.py:1919-1951``)."""
        a = self.amp(x, vals, polar)
        rho = self.density(vals)
        if rho is None:
            return np.sum(np.abs(a.reshape(a.shape[0], -1)) ** 2, axis=1)
        a = a.reshape(a.shape[0], a.shape[1], -1)
        return np.real(np.einsum("nal,ab,nbl->n", a, rho, np.conj(a)))


# ----------------------------------------------------------- NLL
def clip_log(x, eps=_EPS_CLIP):
    """tf_pwa/model/model.py:283-292."""
    xc = np.where(x > eps, x, eps)
    dx = x - eps
    return np.where(x > eps, np.log(xc), np.log(eps) + dx / eps - (dx / eps) ** 2 / 2.0)


def weights(w_data, w_bg=None):
    """alpha-scaled data weights (model.py:603-641): data weights followed by
    background weights, times sum(w)/sum(w^2)."""
    w = np.asarray(w_data, np.float64)
    if w_bg is not None:
        w = np.concatenate([w, np.asarray(w_bg, np.float64)])
    return w * (w.sum() / (w * w).sum())


def nll_value(f_data, w_data, f_mc, w_mc):
    """-sum w clip_log f + (sum w) ln(sum w_mc f_mc / sum w_mc) (model.py:407-449)."""
    wm = w_mc / w_mc.sum()
    sw = w_data.sum()
    return -np.sum(w_data * clip_log(f_data)) + sw * np.log(np.sum(wm * f_mc))


class OracleNLL:
    def __init__(self, model, x_data, w_data, x_mc, w_mc, names, polar, vals):
        self.m = model
        self.xd, self.wd = x_data, w_data
        self.xm, self.wm = x_mc, w_mc
        self.names = list(names)         # trainable names, in order
        self.polar = polar
        self.base = dict(vals)

    def _vals(self, p):
        v = dict(self.base)
        v.update(dict(zip(self.names, p)))
        return v

    def nll(self, p):
        v = self._vals(p)
        return nll_value(self.m.pdf(self.xd, v, self.polar), self.wd,
                         self.m.pdf(self.xm, v, self.polar), self.wm)

    def grad(self, p, rel_step=1e-4):
        """Exact derivative for coupling parameters (via the linear column
        decomposition evaluated by differentiating r, phi analytically) and
        4-point central differences for masses and widths."""
        p = np.asarray(p, np.float64)
        g = np.zeros_like(p)
        v0 = self._vals(p)
        fd0 = self.m.pdf(self.xd, v0, self.polar)
        fm0 = self.m.pdf(self.xm, v0, self.polar)
        Ad = self.m.amp(self.xd, v0, self.polar).reshape(len(fd0), -1)
        Am = self.m.amp(self.xm, v0, self.polar).reshape(len(fm0), -1)
        wm = self.wm / self.wm.sum()
        sw = self.wd.sum()
        I = np.sum(wm * fm0)
        # df = 2 Re sum S dA with S = conj(A), or sum_b rho_ab conj(A_b) when
        # the parent is polarised
        rho = self.m.density(v0)

        def seed(A):
            if rho is None:
                return np.conj(A)
            a = A.reshape(A.shape[0], rho.shape[0], -1)
            return np.einsum("ab,nbl->nal", rho, np.conj(a)).reshape(A.shape)

        Sd, Sm = seed(Ad), seed(Am)
        dclip = np.where(fd0 > _EPS_CLIP, 1.0 / np.where(fd0 > _EPS_CLIP, fd0, 1.0),
                         1.0 / _EPS_CLIP - (fd0 - _EPS_CLIP) / _EPS_CLIP ** 2)
        cp_totals = {c.params_head + "_total_0" for c in self.m.group if getattr(c, "is_cp", False)}
        for k, n in enumerate(self.names):
            base = n[:-1]
            if n.endswith(("r", "i")) and base + "r" in v0 and base + "i" in v0 and (
                    "_g_ls_" in base or "_total_" in base) and not any(
                    base.startswith(t) for t in cp_totals):
                # dA/dtheta: A is linear in the complex coupling c = c(r, phi)
                c = self.m.complex_of(v0, self.polar, base)
                polar = self.polar.get(base, True)
                r, ph = v0[base + "r"], v0[base + "i"]
                if polar:
                    dc = np.exp(1j * ph) if n.endswith("r") else 1j * c
                else:
                    dc = 1.0 if n.endswith("r") else 1j
                # A = c * B + rest with B = dA/dc: evaluate B by setting c := 1
                # and subtracting the c := 0 amplitude.
                v1 = dict(v0)
                v1[base + "r"], v1[base + "i"] = (1.0, 0.0)
                v2 = dict(v0)
                v2[base + "r"], v2[base + "i"] = (0.0, 0.0)
                Bd = (self.m.amp(self.xd, v1, self.polar) - self.m.amp(self.xd, v2, self.polar)).reshape(Ad.shape)
                Bm = (self.m.amp(self.xm, v1, self.polar) - self.m.amp(self.xm, v2, self.polar)).reshape(Am.shape)
                dfd = 2 * np.real(np.sum(Sd * Bd * dc, axis=1))
                dfm = 2 * np.real(np.sum(Sm * Bm * dc, axis=1))
                g[k] = -np.sum(self.wd * dclip * dfd) + sw * np.sum(wm * dfm) / I
            else:
                # 4-point central differences at h and h/2, Richardson-combined
                def d4(h):
                    fs = []
                    for s in (-2, -1, 1, 2):
                        q = p.copy()
                        q[k] += s * h
                        fs.append(self.nll(q))
                    return (fs[0] - 8 * fs[1] + 8 * fs[2] - fs[3]) / (12 * h)

                h = rel_step * max(abs(p[k]), 1e-3)
                g[k] = (16 * d4(h / 2) - d4(h)) / 15
        return g


# ------------------------------------------------ one-pass NLL + gradient
def column_sums(model, x, w, vals, polar, data):
    """Sums over one event set from its partial-wave columns: data
    (sum w clip_log f, sum_n w clip_log'(f_n) G_nk) or MC (sum w f,
    sum_n w G_nk), G_nk = sum_o conj(A_no) F_nko.  Returns (S, G (K,))."""
    F, names = model.columns(x, vals, polar)
    c = coupling_products(names, vals, polar)
    A = np.einsum("k,nko->no", c, F)
    f = np.sum(np.abs(A) ** 2, 1)
    G = np.einsum("no,nko->nk", np.conj(A), F)
    if data:
        dl = np.where(f > _EPS_CLIP, 1.0 / np.where(f > _EPS_CLIP, f, 1.0),
                      1.0 / _EPS_CLIP - (f - _EPS_CLIP) / _EPS_CLIP ** 2)
        return float(np.sum(w * clip_log(f))), (w * dl) @ G
    return float(np.sum(w * f)), w @ G


def coupling_products(names, vals, polar):
    """c_k = total x product of the column's g_ls (complex)."""
    out = []
    for tot, gs in names:
        c = OracleModel.complex_of(vals, polar, tot)
        for g in gs:
            c = c * OracleModel.complex_of(vals, polar, g)
        out.append(c)
    return np.array(out)


def nll_grad_from_sums(names, vals, polar, trainable, sd, gd, sm, gm, sw):
    """NLL = -S_d + sw ln S_m and its derivative with respect to the
    trainable coupling parts (r/i, polar or Cartesian): df = 2 Re(dc_k G_k)."""
    nll = -sd + sw * np.log(sm)
    c = coupling_products(names, vals, polar)
    grad = np.zeros(len(trainable))
    for t, n in enumerate(trainable):
        base, part = n[:-1], n[-1]
        if part not in "ri" or base + "r" not in vals or base + "i" not in vals:
            raise ValueError(f"{n}: not a coupling part")
        g = OracleModel.complex_of(vals, polar, base)
        if polar.get(base, True):
            r, ph = vals[base + "r"], vals[base + "i"]
            dg = np.exp(1j * ph) if part == "r" else 1j * g
        else:
            dg = 1.0 if part == "r" else 1j
        dc = np.zeros(len(names), np.complex128)
        for k, (tot, gs) in enumerate(names):
            facs = [tot] + list(gs)
            m = facs.count(base)
            if m:
                rest = 1.0 + 0j
                for q in facs:
                    rest = rest * OracleModel.complex_of(vals, polar, q)
                dc[k] = m * rest / g * dg
        grad[t] = -2.0 * np.real(dc @ gd) + sw * 2.0 * np.real(dc @ gm) / sm
    return nll, grad


# ------------------------------------------- exact Hessian of the couplings
def clip_log_d12(x, eps=_EPS_CLIP):
    """First and second derivatives of clip_log (model.py:283-292): 1/x and
    -1/x^2 above eps, the quadratic continuation's 1/eps - (x-eps)/eps^2 and
    -1/eps^2 below."""
    big = x > eps
    xs = np.where(big, x, 1.0)
    d1 = np.where(big, 1.0 / xs, 1.0 / eps - (x - eps) / eps ** 2)
    d2 = np.where(big, -1.0 / xs ** 2, -1.0 / eps ** 2)
    return d1, d2


def hessian_sums(model, x, w, vals, polar):
    """Data sums for the exact second derivatives of -sum w clip_log(f) in
    the couplings: with A_o = sum_k c_k F_ko, f = sum_o |A_o|^2 = c^H Q c
    (Q_lk = sum_o conj(F_lo) F_ko) and G_k = sum_o conj(A_o) F_ko,
      S0 = sum w t(f),  S1 = sum w t'(f) G,
      H1 = sum w t'(f) Q   (K x K Hermitian),
      H2 = sum w t''(f) g g^T,  g = (Re G, -Im G)   (2K x 2K),
    which give d2/da db of the data term as
      -2 Re[(c_b)^H H1 c_a] - 2 Re(c_ab . S1) - 4 (Re c_a, Im c_a) H2 (Re c_b, Im c_b)^T
    for c_a = dc/da, c_ab = d2c/da db.  The reference obtains the same
    matrix by nested GradientTape (tf_pwa/model/model.py:513-561)."""
    F, names = model.columns(x, vals, polar)
    c = coupling_products(names, vals, polar)
    A = np.einsum("k,nko->no", c, F)
    f = np.sum(np.abs(A) ** 2, 1)
    G = np.einsum("no,nko->nk", np.conj(A), F)
    d1, d2 = clip_log_d12(f)
    S0 = float(np.sum(w * clip_log(f)))
    S1 = (w * d1) @ G
    H1 = np.einsum("n,nlo,nko->lk", w * d1, np.conj(F), F)
    g = np.concatenate([G.real, -G.imag], 1)
    H2 = np.einsum("n,np,nq->pq", w * d2, g, g)
    return S0, S1, H1, H2, names


def gram_matrix(model, x, w, vals, polar):
    """M_lk = sum w sum_o conj(F_lo) F_ko (the MC integral I = c^H M c)."""
    F, names = model.columns(x, vals, polar)
    return np.einsum("n,nlo,nko->lk", w, np.conj(F), F), names


def coupling_derivatives(names, vals, polar, trainable):
    """dc/da (P, K) and d2c/da db (P, P, K) of the column couplings c_k =
    product of the column's factors (chain total, one g_ls per vertex) with
    respect to the trainable coupling parts (r/i, polar or Cartesian)."""
    P, K = len(trainable), len(names)

    def z_of(base):
        return OracleModel.complex_of(vals, polar, base)

    def dz(base, part):
        if polar.get(base, True):
            return np.exp(1j * vals[base + "i"]) if part == "r" else 1j * z_of(base)
        return 1.0 + 0j if part == "r" else 1j

    def d2z(base, p1, p2):
        if not polar.get(base, True):
            return 0j
        e = np.exp(1j * vals[base + "i"])
        if p1 == p2 == "r":
            return 0j
        if p1 == p2 == "i":
            return -z_of(base)
        return 1j * e

    parts = [(n[:-1], n[-1]) for n in trainable]
    dc = np.zeros((P, K), np.complex128)
    d2c = np.zeros((P, P, K), np.complex128)
    for k, (tot, gs) in enumerate(names):
        facs = [tot] + list(gs)
        zs = [z_of(q) for q in facs]
        for a, (ba, pa) in enumerate(parts):
            for i, q in enumerate(facs):
                if q != ba:
                    continue
                rest = np.prod([zs[m] for m in range(len(facs)) if m != i])
                dc[a, k] += dz(ba, pa) * rest
                for b, (bb, pb) in enumerate(parts):
                    if bb == ba:
                        d2c[a, b, k] += d2z(ba, pa, pb) * rest
                    for j, q2 in enumerate(facs):
                        if j == i or q2 != bb:
                            continue
                        rest2 = np.prod([zs[m] for m in range(len(facs)) if m not in (i, j)])
                        d2c[a, b, k] += dz(ba, pa) * dz(bb, pb) * rest2
    return dc, d2c


def nll_grad_hessian_from_sums(names, vals, polar, trainable, sums, M, sw):
    """NLL, gradient and exact Hessian from the data sums of
    :func:`hessian_sums` and the MC Gram matrix M (sum_w-normalised
    weights): NLL = -S0 + sw ln I, I = c^H M c."""
    S0, S1, H1, H2 = sums
    c = coupling_products(names, vals, polar)
    dc, d2c = coupling_derivatives(names, vals, polar, trainable)
    I = float(np.real(np.conj(c) @ M @ c))
    Mc = np.conj(c) @ M  # (c^H M)_k
    dI = 2.0 * np.real(dc @ Mc)
    grad = -2.0 * np.real(dc @ S1) + sw * dI / I
    ch = np.concatenate([dc.real, dc.imag], 1)
    Hd = (-2.0 * np.real(np.conj(dc) @ H1 @ dc.T).T
          - 2.0 * np.real(d2c @ S1) - 4.0 * ch @ H2 @ ch.T)
    d2I = 2.0 * np.real(np.conj(dc) @ M @ dc.T).T + 2.0 * np.real(d2c @ Mc)
    H = Hd + sw * (d2I / I - np.outer(dI, dI) / I ** 2)
    return -S0 + sw * np.log(I), grad, 0.5 * (H + H.T)

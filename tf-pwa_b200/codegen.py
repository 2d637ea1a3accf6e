"""Model compiler back end: emits the CUDA source of a decay model.

The generated code is one ``model_event<R>()`` device function that, for one
event, evaluates every partial-wave column F_k of the amplitude, the full
amplitude A = sum_k c_k F_k, |A|^2 summed over external helicities, and the
column sensitivities G_k = sum_lambda conj(A_lambda) F_k,lambda from which
the NLL gradient follows.  Constants (CG products, Wigner-d weights,
Blatt-Weisskopf coefficients, helicity bookkeeping) are folded into the code;
per-evaluation quantities (couplings, q0 factors, lineshape constants) are
read from a ``Consts`` kernel argument laid out by :class:`ConstLayout`.

The mathematics is the reference's (see ``csrc/pwa_device.cuh`` and the
restated chain contraction of ``tf_pwa/amp/core.py:1392-1445``): a chain's
amplitude is the product of its vertices' H(LS) * D*(angles of outs[0]),
summed over inner helicities, times the lineshapes, the chain total, and the
alignment D* of spinning final particles.
"""
import itertools
import math

import numpy as np

from .particles import bprime_coeff, small_d_weight, two

_HEADER = """
#define PWA_NCOL {ncol}
#define PWA_NOUT {nout}
#define PWA_NSHAPE {nshape}
#define PWA_NACC {nacc}
#define PWA_NCONST {nconst}
struct Consts {{ double v[PWA_NCONST]; }};
"""


def _lit(v):
    r = repr(float(v))
    if "e" not in r and "." not in r and "inf" not in r and "nan" not in r:
        r += ".0"
    return f"R({r})"


class ConstLayout:
    """Index map of the per-evaluation constant block."""

    def __init__(self):
        self.names = []
        self.index = {}

    def add(self, name):
        if name not in self.index:
            self.index[name] = len(self.names)
            self.names.append(name)
        return self.index[name]

    def __len__(self):
        return len(self.names)


class ModelCode:
    """Everything the engine needs to know about the compiled model."""

    def __init__(self, group, plan, vm_names=None):
        self.group = group
        self.plan = plan
        self.consts = ConstLayout()
        self.columns = []          # per column: (chain index, tuple of ls indices)
        self.chain_columns = []    # per chain: list of global column ids
        for ci, c in enumerate(group):
            ids = []
            ranges = [range(len(d.get_ls_list())) for d in c]
            for lsi in itertools.product(*ranges):
                ids.append(len(self.columns))
                self.columns.append((ci, lsi))
            self.chain_columns.append(ids)
        self.outs = [group.top] + list(group.outs)
        self.out_hel = list(itertools.product(*[p.spins for p in self.outs]))
        self.nout = len(self.out_hel)
        # field split: masses (always FP64 storage) and angles
        self.mass_fields = [i for i, f in enumerate(plan.fields) if f.startswith("m/")]
        self.angle_fields = [i for i, f in enumerate(plan.fields) if not f.startswith("m/")]
        self.mass_slot = {f: k for k, f in enumerate(self.mass_fields)}
        self.angle_slot = {f: k for k, f in enumerate(self.angle_fields)}
        # consts: couplings first
        for k in range(len(self.columns)):
            self.consts.add(f"c{k}.re")
            self.consts.add(f"c{k}.im")
        # resonances with shape
        self.res = []
        for p in group.resonances:
            kind = p.lineshape_kind()
            if p.width_norm:
                raise NotImplementedError("width_norm lineshapes")
            self.res.append((p, kind))
            if kind == "BWR":
                self.consts.add(f"{p}.m0sq")
                self.consts.add(f"{p}.K")
                self.consts.add(f"{p}.useq")
            elif kind == "BW":
                self.consts.add(f"{p}.m0sq")
                self.consts.add(f"{p}.y")
        # barrier factor constants per decay vertex
        self.vertices = []
        seen = set()
        for c in group:
            for d in c:
                if d in seen:
                    continue
                seen.add(d)
                self.vertices.append(d)
                if d.has_barrier_factor and d.has_bprime:
                    for l in sorted(set(d.get_l_list())):
                        self.consts.add(f"{d}.Pz0_{l}")
                if d.has_barrier_factor and d.barrier_factor_norm:
                    for l in sorted(set(d.get_l_list())):
                        self.consts.add(f"{d}.norm_{l}")
        # shape derivatives: per resonance that may float, d ln(m0*Gamma)/dm0
        self.shape_res = []
        for p, kind in self.res:
            if kind in ("BWR", "BW"):
                self.shape_res.append(p)
                self.consts.add(f"{p}.kappa_m")
                self.consts.add(f"{p}.inv_g0")
        self.nshape = 2 * len(self.shape_res)
        self.ncol = len(self.columns)
        self.nacc = 1 + 2 * self.ncol + self.nshape

    # ------------------------------------------------------------ emission
    def source(self):
        self._fset = set()
        L = []
        L.append(_HEADER.format(ncol=self.ncol, nout=self.nout, nshape=self.nshape,
                                nacc=self.nacc, nconst=max(len(self.consts), 1)))
        L.append("template <typename R>\n__device__ __forceinline__ void model_event(\n"
                 "    const Consts& C, const R* __restrict__ XA, const double* __restrict__ XM,\n"
                 "    long long ld, long long i, double* __restrict__ fout,\n"
                 "    cpx<R>* __restrict__ G, double* __restrict__ dshape) {")
        body = []
        e = body.append
        cidx = self.consts.index

        def cst(name):
            return f"R(C.v[{cidx[name]}])"

        # --- load fields
        for f in self.mass_fields:
            e(f"  const double xm{f} = __ldg(XM + (long long){self.mass_slot[f]} * ld + i);")
        for f in self.angle_fields:
            e(f"  const R xa{f} = __ldg(XA + (long long){self.angle_slot[f]} * ld + i);")

        # --- per chain
        for ci, c in enumerate(self.group):
            cf = self.plan.chains[ci]
            e(f"  // chain {ci}: {c}")

            def dmass(p, dbl=False):
                if p in c.inner:
                    return f"xm{cf['mass'][p]}" if dbl else f"R(xm{cf['mass'][p]})"
                return repr(float(p.mass)) if dbl else _lit(p.mass)

            # vertices: q^2 (FP64 from FP64 masses), barrier factors, D elements
            for vi, d in enumerate(c):
                a, (b, cc) = d.core, d.outs
                tag = f"c{ci}v{vi}"
                fa = cf["decays"][vi]
                if d.has_barrier_factor:
                    e(f"  const double q2d_{tag} = rel_p2<double>({dmass(a, True)}, {dmass(b, True)}, {dmass(cc, True)});")
                    e(f"  const R q2_{tag} = R(q2d_{tag});")
                    for l in sorted(set(d.get_l_list())):
                        terms = []
                        if d.has_ql:
                            if l == 0:
                                ql = "R(1)"
                            elif l % 2 == 0:
                                ql = "*".join([f"q2_{tag}"] * (l // 2))
                            else:
                                ql = "*".join([f"psqrt(q2_{tag})"] + [f"q2_{tag}"] * (l // 2))
                        else:
                            ql = "R(1)"
                        if d.has_bprime:
                            co = bprime_coeff(l)
                            z = f"(q2_{tag} * {_lit(d.d * d.d)})"
                            poly = _lit(co[0])
                            for cc_ in co[1:]:
                                poly = f"fma({poly}, {z}, {_lit(cc_)})"
                            e(f"  R bp_{tag}_{l} = {cst(f'{d}.Pz0_{l}')} / ({poly});")
                            e(f"  bp_{tag}_{l} = bp_{tag}_{l} > R(0) ? bp_{tag}_{l} : R(1);")
                            bf = f"({ql}) * psqrt(bp_{tag}_{l})"
                        else:
                            bf = ql
                        if d.barrier_factor_norm:
                            bf = f"({bf}) * {cst(f'{d}.norm_{l}')}"
                        e(f"  const R bf_{tag}_{l} = {bf};")
                # D*^{Ja}_{la, lb-lc}(alpha, beta, 0)
                j2 = two(a.J)
                need = set()
                for la in a.spins:
                    for lb in b.spins:
                        for lc in cc.spins:
                            dl = lb - lc
                            if abs(dl) <= a.J + 1e-9:
                                need.add((two(la), two(dl)))
                e(f"  R sp_{tag}[{j2 + 1}], cp_{tag}[{j2 + 1}];")
                e(f"  half_angle_sc_powers<R, {j2}>(xa{fa['beta']}, sp_{tag}, cp_{tag});")
                need_alpha = any(n1 != 0 for n1, _ in need)
                if need_alpha:
                    e(f"  cpx<R> ea_{tag}[{2 * j2 + 1}];")
                    e(f"  half_angle_powers<R, {j2}>(xa{fa['alpha']}, ea_{tag});")
                w = small_d_weight(j2)
                for n1, n2 in sorted(need):
                    i1, i2 = (n1 + j2) // 2, (n2 + j2) // 2
                    terms = [f"{_lit(w[l][i1][i2])} * sp_{tag}[{l}] * cp_{tag}[{j2 - l}]"
                             for l in range(j2 + 1) if w[l][i1][i2] != 0]
                    dexpr = " + ".join(terms) if terms else "R(0)"
                    nm = f"D_{tag}_{n1 + j2}_{n2 + j2}"
                    if need_alpha and n1 != 0:
                        e(f"  const cpx<R> {nm} = cscale(ea_{tag}[{n1 + j2}], {dexpr});")
                    else:
                        e(f"  const cpx<R> {nm} = cmk<R>({dexpr}, R(0));")
            # alignment D for spinning finals: e^{i l a} d_{l l'}(b) e^{i l' g}
            for o, (fa_, fb_, fg_) in cf["aligned"].items():
                tag = f"c{ci}al{self.group.outs.index(o)}"
                j2 = two(o.J)
                e(f"  R sp_{tag}[{j2 + 1}], cp_{tag}[{j2 + 1}];")
                e(f"  half_angle_sc_powers<R, {j2}>(xa{fb_}, sp_{tag}, cp_{tag});")
                e(f"  cpx<R> ea_{tag}[{2 * j2 + 1}], eg_{tag}[{2 * j2 + 1}];")
                e(f"  half_angle_powers<R, {j2}>(xa{fa_}, ea_{tag});")
                e(f"  half_angle_powers<R, {j2}>(xa{fg_}, eg_{tag});")
                w = small_d_weight(j2)
                for l1 in o.spins:
                    for l2 in o.spins:
                        n1, n2 = two(l1), two(l2)
                        i1, i2 = (n1 + j2) // 2, (n2 + j2) // 2
                        terms = [f"{_lit(w[l][i1][i2])} * sp_{tag}[{l}] * cp_{tag}[{j2 - l}]"
                                 for l in range(j2 + 1) if w[l][i1][i2] != 0]
                        dexpr = " + ".join(terms) if terms else "R(0)"
                        e(f"  const cpx<R> Dal_{tag}_{n1 + j2}_{n2 + j2} = cscale(cmul(ea_{tag}[{n1 + j2}], eg_{tag}[{n2 + j2}]), {dexpr});")
            # lineshapes of the chain's inner particles
            bw_names = []
            for p in c.inner:
                kind = p.lineshape_kind()
                tag = f"c{ci}r{c.inner.index(p)}"
                m = f"xm{cf['mass'][p]}"
                if kind == "one":
                    continue
                bw_names.append(f"bw_{tag}")
                e(f"  const double xx_{tag} = {repr(0.0)} + C.v[{cidx[f'{p}.m0sq']}] - {m} * {m};")
                if kind == "BWR":
                    dp = c.decay_of(p)
                    b, cc = dp.outs
                    L_ = p.bw_l if p.bw_l is not None else min(dp.get_l_list())
                    e(f"  const R q_{tag} = R(rel_p<double>({m}, {dmass(b, True)}, {dmass(cc, True)}));")
                    co = bprime_coeff(L_)
                    z = f"(q_{tag} * q_{tag} * {_lit(p.d * p.d)})"
                    poly = _lit(co[0])
                    for cc_ in co[1:]:
                        poly = f"fma({poly}, {z}, {_lit(cc_)})"
                    qp = "*".join([f"q_{tag}"] * (2 * L_ + 1))
                    e(f"  const R qp_{tag} = {cst(f'{p}.useq')} != R(0) ? ({qp}) : R(1);")
                    e(f"  const R y_{tag} = {cst(f'{p}.K')} * qp_{tag} / (R({m}) * ({poly}));")
                else:
                    e(f"  const R y_{tag} = {cst(f'{p}.y')};")
                e(f"  const R xr_{tag} = R(xx_{tag});")
                e(f"  const R s_{tag} = xr_{tag} * xr_{tag} + y_{tag} * y_{tag};")
                e(f"  const cpx<R> bw_{tag} = cmk<R>(xr_{tag} / s_{tag}, y_{tag} / s_{tag});")
            # chain lineshape product
            if bw_names:
                e(f"  cpx<R> BW_c{ci} = {bw_names[0]};")
                for nm in bw_names[1:]:
                    e(f"  BW_c{ci} = cmul(BW_c{ci}, {nm});")
            else:
                e(f"  const cpx<R> BW_c{ci} = cmk<R>(R(1), R(0));")

            # angular columns F^ang_k[out]
            cols = self.chain_columns[ci]
            parts = [c.top] + c.inner + list(c.outs)
            cgs = [d.cg() for d in c]
            terms = {}  # (k, out) -> list of (coef, product expr)
            prods = {}
            for hel in itertools.product(*[p.spins for p in parts]):
                hmap = dict(zip(parts, hel))
                ok = True
                facs = []
                for vi, d in enumerate(c):
                    a, (b, cc) = d.core, d.outs
                    dl = hmap[b] - hmap[cc]
                    if abs(dl) > a.J + 1e-9:
                        ok = False
                        break
                    j2 = two(a.J)
                    facs.append(f"D_c{ci}v{vi}_{two(hmap[a]) + j2}_{two(dl) + j2}")
                if not ok:
                    continue
                # pre-alignment output helicities (chain's own final helicities)
                pre_out = (hmap[c.top],) + tuple(hmap[o] for o in self.group.outs)
                for kk, k in enumerate(cols):
                    lsi = self.columns[k][1]
                    coef = 1.0
                    for vi, d in enumerate(c):
                        a, (b, cc) = d.core, d.outs
                        ib = b.spins.index(hmap[b])
                        ic = cc.spins.index(hmap[cc])
                        coef *= cgs[vi][lsi[vi], ib, ic]
                    if coef == 0.0:
                        continue
                    key = tuple(facs)
                    if key not in prods:
                        pn = f"P_c{ci}_{len(prods)}"
                        prods[key] = pn
                        if len(facs) == 1:
                            e(f"  const cpx<R> {pn} = {facs[0]};")
                        else:
                            expr = facs[0]
                            for fnm in facs[1:]:
                                expr = f"cmul({expr}, {fnm})"
                            e(f"  const cpx<R> {pn} = {expr};")
                    terms.setdefault((k, pre_out), []).append((coef, prods[key]))
            # emit pre-alignment columns
            pre_outs = sorted({po for (_, po) in terms}, key=lambda t: [float(x) for x in t])
            for k in cols:
                for po in pre_outs:
                    lst = terms.get((k, po))
                    nm = self._pre_name(ci, k, po)
                    if not lst:
                        continue
                    e(f"  cpx<R> {nm} = cmk<R>(R(0), R(0));")
                    for coef, pn in lst:
                        e(f"  cfma({nm}, {_lit(coef)}, {pn});")
            # alignment: contract each aligned final's helicity index
            aligned = [o for o in self.group.outs if o in cf["aligned"]]
            cur = {(k, po): self._pre_name(ci, k, po) for k in cols for po in pre_outs
                   if (k, po) in terms}
            for o in aligned:
                oi = 1 + self.group.outs.index(o)
                tag = f"c{ci}al{oi - 1}"
                j2 = two(o.J)
                new = {}
                for k in cols:
                    for out in self.out_hel:
                        # out[oi] is the aligned helicity; sum over source helicity
                        srcs = []
                        for l1 in o.spins:
                            src = list(out)
                            src[oi] = l1
                            src = tuple(src)
                            if (k, src) in cur:
                                srcs.append((cur[(k, src)], f"Dal_{tag}_{two(l1) + j2}_{two(out[oi]) + j2}"))
                        if not srcs:
                            continue
                        nm = f"Fa_c{ci}_{oi}_{k}_{self.out_hel.index(out)}"
                        e(f"  cpx<R> {nm} = cmk<R>(R(0), R(0));")
                        for s_, dn in srcs:
                            e(f"  cfmac({nm}, {s_}, {dn});")
                        new[(k, out)] = nm
                cur = new
            # final per-column angular values F[k][out] and per-event scale
            for k in cols:
                lsi = self.columns[k][1]
                sc = []
                for vi, d in enumerate(c):
                    if d.has_barrier_factor:
                        l = d.get_ls_list()[lsi[vi]][0]
                        sc.append(f"bf_c{ci}v{vi}_{l}")
                scale = " * ".join(sc) if sc else "R(1)"
                e(f"  const cpx<R> S{k} = cscale(BW_c{ci}, {scale});")
                # e_k = c_k * scale_k
                e(f"  const cpx<R> E{k} = cmul(cmk<R>({cst(f'c{k}.re')}, {cst(f'c{k}.im')}), S{k});")
                for oj, out in enumerate(self.out_hel):
                    nm = cur.get((k, out))
                    if nm is not None:
                        e(f"  const cpx<R> F{k}_{oj} = {nm};")
                        self._fset.add((k, oj))
            self._cur_chain = None
        # --- columns variant: F[k][o] = S_k * F^ang_k[o]
        cols_body = list(body)
        for k in range(self.ncol):
            for oj in range(self.nout):
                if (k, oj) in self._fset:
                    cols_body.append(f"  F[{k * self.nout + oj}] = cmul(S{k}, F{k}_{oj});")
                else:
                    cols_body.append(f"  F[{k * self.nout + oj}] = cmk<R>(R(0), R(0));")
        # --- amplitude, |A|^2
        for oj in range(self.nout):
            e(f"  cpx<R> A{oj} = cmk<R>(R(0), R(0));")
            for k in range(self.ncol):
                if (k, oj) in self._fset:
                    e(f"  cfmac(A{oj}, E{k}, F{k}_{oj});")
        e("  R fsum = R(0);")
        for oj in range(self.nout):
            e(f"  fsum += cabs2(A{oj});")
        e("  *fout = double(fsum);")
        # --- sensitivities: G_k = S_k * sum_out conj(A_out) F_k[out]
        for k in range(self.ncol):
            e(f"  cpx<R> H{k} = cmk<R>(R(0), R(0));")
            for oj in range(self.nout):
                if (k, oj) in self._fset:
                    e(f"  {{ const cpx<R> t = cmulc(F{k}_{oj}, A{oj}); H{k} = cadd(H{k}, t); }}")
            e(f"  G[{k}] = cmul(S{k}, H{k});")
        # --- shape derivatives for each resonance with a lineshape
        for si, p in enumerate(self.shape_res):
            # S_R = sum over columns of chains containing p of e_k H_k
            e(f"  {{ cpx<R> SR = cmk<R>(R(0), R(0));")
            tag = None
            for ci, c in enumerate(self.group):
                if p in c.inner:
                    tag = f"c{ci}r{c.inner.index(p)}"
                    for k in self.chain_columns[ci]:
                        e(f"    cfmac(SR, E{k}, H{k});")
            # dlnBW/dm0 = -BW (2 m0 - i y kappa_m); dlnBW/dg0 = i BW y / g0
            e(f"    const R m0 = psqrt({cst(f'{p}.m0sq')});")
            e(f"    const cpx<R> dm = cmul(bw_{tag}, cmk<R>(R(-2) * m0, y_{tag} * {cst(f'{p}.kappa_m')}));")
            e(f"    const cpx<R> dg = cmul(bw_{tag}, cmk<R>(R(0), y_{tag} * {cst(f'{p}.inv_g0')}));")
            e(f"    const cpx<R> a1 = cmul(SR, dm), a2 = cmul(SR, dg);")
            e(f"    dshape[{2 * si}] = 2.0 * double(a1.re); dshape[{2 * si + 1}] = 2.0 * double(a2.re); }}")
        L.append("\n".join(body))
        L.append("}\n")
        L.append("template <typename R>\n__device__ __forceinline__ void model_columns(\n"
                 "    const Consts& C, const R* __restrict__ XA, const double* __restrict__ XM,\n"
                 "    long long ld, long long i, cpx<R>* __restrict__ F) {")
        L.append("\n".join(cols_body))
        L.append("}\n")
        fl = sorted(self._fset)
        self.nf = len(fl)
        L.append(f"#define PWA_NF {self.nf}")
        L.append("__device__ constexpr int pwa_fk[PWA_NF] = {" + ", ".join(str(k) for k, _ in fl) + "};")
        L.append("__device__ constexpr int pwa_fo[PWA_NF] = {" + ", ".join(str(o) for _, o in fl) + "};")
        return "\n".join(L)

    def _pre_name(self, ci, k, po):
        tag = "_".join(str(two(x) + 8) for x in po)
        return f"Fp_c{ci}_{k}_{tag}"

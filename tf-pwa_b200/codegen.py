"""Model compiler back end: emits the CUDA source of a decay model.

Three device functions are generated per model, all straight-line code with
every constant folded (CG products, Wigner-d weights, Blatt-Weisskopf
polynomial coefficients, helicity bookkeeping):

``model_amp<R>``      forward pass: the amplitude A_o of every external
                      helicity combination o, with the couplings contracted
                      vertex by vertex (H = sum_ls g_ls bf_ls CG_ls, vertex
                      tensor H * D*, sum over inner helicities, lineshapes,
                      chain total, alignment D* of spinning finals).
``model_adj<R>``      adjoint pass: given Abar_o = fac * conj(A_o), recompute
                      each chain's angular factors and accumulate the column
                      sensitivities G_k = S_k sum_o Abar_o F^ang_k,o and the
                      lineshape-parameter sensitivities.  Nothing from the
                      forward pass is kept, so registers stay per chain.
``model_columns<R>``  the partial-wave columns F_k,o = S_k F^ang_k,o one
                      column at a time (for the column cache and the Gram
                      matrix).

A chain's amplitude is sum_k c_k F_k with c_k = total * prod_vertices g_ls;
S_k = BW(m) * prod_vertices bf_{l_k}; F^ang_k,o = sum over inner helicities of
prod_vertices CG_{ls_k}[lb, lc] D*^{Ja}_{la, lb-lc} (then aligned).  The
mathematics is the reference's chain contraction
(``tf_pwa/amp/core.py:1149-1164,1392-1445``).
"""
import itertools

from .decay_config import polarization_names
from .kincode import KinCode
from .plan import split_swap
from .particles import bprime_coeff, small_d_weight, two

_HEADER = """
#define PWA_NCOL {ncol}
#define PWA_NOUT {nout}
#define PWA_NSHAPE {nshape}
#define PWA_NACC {nacc}
#define PWA_NCONST {nconst}
// the constant block of one evaluation; h, l: each constant's FP32 rounding
// and the FP32 rounding of the rest, split once per evaluation on the host
struct Consts {{ double v[PWA_NCONST]; float h[PWA_NCONST]; float l[PWA_NCONST]; }};
// constant i as R (the FP32 kernels read its FP32 rounding: no per-event
// conversion)
template <typename R>
__device__ __forceinline__ R cR(const Consts& C, int i) {{
  if constexpr (sizeof(R) == 4) return C.h[i];
  else return C.v[i];
}}
// products with constant i: FP32 hi + lo parts in the FP32 kernels (the
// rounding of a constant, alike for every event, must not bias the sums), a
// plain product in FP64 -- mulk / cfmak / cmulk with the split precomputed
template <typename R>
__device__ __forceinline__ R mulkc(R x, const Consts& C, int i) {{
  if constexpr (sizeof(R) == 4) return fmaf(x, C.h[i], x * C.l[i]);
  else return x * C.v[i];
}}
template <typename R>
__device__ __forceinline__ void cfmakc(cpx<R>& acc, R s, const Consts& C, int ir, int ii) {{
  if constexpr (sizeof(R) == 4) {{
    acc.re = fmaf(s, C.h[ir], fmaf(s, C.l[ir], acc.re));
    acc.im = fmaf(s, C.h[ii], fmaf(s, C.l[ii], acc.im));
  }} else {{
    acc.re = fma(s, C.v[ir], acc.re);
    acc.im = fma(s, C.v[ii], acc.im);
  }}
}}
template <typename R>
__device__ __forceinline__ cpx<R> cmulkc(const Consts& C, int ir, int ii, cpx<R> z) {{
  if constexpr (sizeof(R) == 4) {{
    const cpx<float> a = cmul(cmk<float>(C.h[ir], C.h[ii]), z);
    const cpx<float> b = cmul(cmk<float>(C.l[ir], C.l[ii]), z);
    return cmk<float>(a.re + b.re, a.im + b.im);
  }} else {{
    return cmul(cmk<double>(C.v[ir], C.v[ii]), z);
  }}
}}
"""


def _lit(v):
    r = repr(float(v))
    if "e" not in r and "." not in r and "inf" not in r and "nan" not in r:
        r += ".0"
    return f"R({r})"


def _f32_exact(v):
    """True when v is a float exactly representable in FP32."""
    import struct

    v = float(v)
    return struct.unpack("f", struct.pack("f", v))[0] == v


def _klit(v, x):
    """Literal v times expression x: a plain product when v is exact in
    FP32, else mulk (FP32 hi + lo parts of v in the FP32 kernels)."""
    if _f32_exact(v):
        return f"{_lit(v)} * {x}"
    return f"mulk<R>({x}, {repr(float(v))})"


def _key(t):
    return [float(x) for x in t]


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

    def __init__(self, group, plan, order=None):
        self.group = group
        self.plan = plan
        self.kin = KinCode(plan, order if order is not None else plan.order)
        self.consts = ConstLayout()
        self.columns = []          # per column: (chain index, tuple of ls indices)
        self.chain_columns = []    # per chain: list of global column ids
        for ci, c in enumerate(group):
            ids = []
            for lsi in itertools.product(*[range(len(d.get_ls_list())) for d in c]):
                ids.append(len(self.columns))
                self.columns.append((ci, lsi))
            self.chain_columns.append(ids)
        self.outs = [group.top] + list(group.outs)
        self.out_hel = list(itertools.product(*[p.spins for p in self.outs]))
        self.out_index = {o: j for j, o in enumerate(self.out_hel)}
        self.nout = len(self.out_hel)
        # FP64 rows: invariant masses and the event charge; the rest are angles
        fp64 = [split_swap(f)[1].startswith("m/") or i == plan.charge_index
                for i, f in enumerate(plan.fields)]
        self.mass_fields = [i for i, f in enumerate(fp64) if f]
        self.angle_fields = [i for i, f in enumerate(fp64) if not f]
        # charge < 0 events reverse the helicity couplings of the vertices
        # that allow it (tf_pwa/amp/core.py:938-945)
        self.flips = plan.charge_index is not None
        # evaluation passes: the unswapped fields, then one per identical-
        # particle swap (its fields, sign and helicity-axis order)
        self.npass = 1 + len(plan.swaps)
        self._pass = 0
        self.mass_slot = {f: k for k, f in enumerate(self.mass_fields)}
        self.angle_slot = {f: k for k, f in enumerate(self.angle_fields)}
        # constants: column couplings c_k, vertex couplings, chain totals
        for k in range(len(self.columns)):
            self.consts.add(f"c{k}.re")
            self.consts.add(f"c{k}.im")
        self.vertices = []
        seen = set()
        for c in group:
            for d in c:
                if d in seen:
                    continue
                seen.add(d)
                self.vertices.append(d)
                for i in range(len(d.get_ls_list())):
                    self.consts.add(f"{d}.g{i}.re")
                    self.consts.add(f"{d}.g{i}.im")
                if d.has_barrier_factor and d.has_bprime:
                    for l in sorted(set(d.get_l_list())):
                        self.consts.add(f"{d}.Pz0_{l}")
                if d.has_barrier_factor and d.barrier_factor_norm:
                    for l in sorted(set(d.get_l_list())):
                        self.consts.add(f"{d}.norm_{l}")
        for ci in range(len(group)):
            self.consts.add(f"t{ci}.re")
            self.consts.add(f"t{ci}.im")
        # CP-violating chain totals: charge -1 events take the second value
        # of the total (and of its columns' couplings); their column
        # sensitivities are summed apart (tf_pwa/amp/core.py:1380-1390)
        self.cp_chains = [ci for ci, c in enumerate(group) if getattr(c, "is_cp", False)]
        self.cp_cols = [k for k, (ci, _) in enumerate(self.columns) if ci in self.cp_chains]
        self.cp_pos = {k: j for j, k in enumerate(self.cp_cols)}
        for ci in self.cp_chains:
            self.consts.add(f"t{ci}m.re")
            self.consts.add(f"t{ci}m.im")
        for k in self.cp_cols:
            self.consts.add(f"c{k}m.re")
            self.consts.add(f"c{k}m.im")
        self.res = []
        for p in group.resonances:
            kind = p.lineshape_kind()
            self.res.append((p, kind))
            if kind == "BWR":
                self.consts.add(f"{p}.m0sq")
                self.consts.add(f"{p}.K")
                self.consts.add(f"{p}.useq")
            elif kind == "BWR2":
                self.consts.add(f"{p}.m0sq")
                self.consts.add(f"{p}.K")
                self.consts.add(f"{p}.iq02")
            elif kind == "BW":
                self.consts.add(f"{p}.m0sq")
                self.consts.add(f"{p}.y")
            if p.width_norm_applies():
                self.consts.add(f"{p}.wn")
        self.shape_res = []
        for p, kind in self.res:
            if kind in ("BWR", "BW", "BWR2"):
                self.shape_res.append(p)
                self.consts.add(f"{p}.kappa_m")
                self.consts.add(f"{p}.inv_g0")
        self.nshape = 2 * len(self.shape_res)
        # polarised parent: density matrix rho (constants) and the sums of
        # the parent-helicity products T_ab for its gradient
        self.pol_names = polarization_names(group)
        self.na = len(group.top.spins)
        self.nrho = 2 * self.na * self.na if self.pol_names else 0
        if self.pol_names:
            for a in range(self.na):
                for b in range(self.na):
                    self.consts.add(f"rho{a}_{b}.re")
                    self.consts.add(f"rho{a}_{b}.im")
        self.ncol = len(self.columns)
        self.ncp = 2 * len(self.cp_cols) if plan.charge_index is not None else 0
        self.nacc = 1 + 2 * self.ncol + self.nshape + self.nrho + self.ncp
        self._analyse()

    # ------------------------------------------------------------ analysis
    def _analyse(self):
        """Helicity assignments of every chain and the CG coefficient of
        every (column, assignment)."""
        self.chain_assign = []
        for ci, c in enumerate(self.group):
            parts = [c.top] + c.inner + list(c.outs)
            cgs = [d.cg() for d in c]
            cgs_cc = [self._cg_cc(d) for d in c]
            rows = []
            for hel in itertools.product(*[p.spins for p in parts]):
                hmap = dict(zip(parts, hel))
                facs = []
                ok = True
                for vi, d in enumerate(c):
                    a, (b, cc) = d.core, d.outs
                    dl = hmap[b] - hmap[cc]
                    if abs(dl) > a.J + 1e-9:
                        ok = False
                        break
                    j2 = two(a.J)
                    facs.append((vi, two(hmap[a]) + j2, two(dl) + j2,
                                 b.spins.index(hmap[b]), cc.spins.index(hmap[cc])))
                if not ok:
                    continue
                pre_out = (hmap[c.top],) + tuple(hmap[o] for o in self.group.outs)
                coefs = {}
                for k in self.chain_columns[ci]:
                    lsi = self.columns[k][1]
                    cf, cfc = 1.0, 1.0
                    for (vi, _, _, ib, ic) in facs:
                        cf *= cgs[vi][lsi[vi], ib, ic]
                        cfc *= cgs_cc[vi][lsi[vi], ib, ic]
                    if cf != 0.0 or cfc != 0.0:
                        # a number, or (charge > 0, charge < 0) values
                        coefs[k] = cf if cf == cfc else (cf, cfc)
                if coefs:
                    rows.append((tuple(facs), pre_out, coefs))
            self.chain_assign.append(rows)
        # structurally non-zero (column, output) pairs after alignment
        self._fset = set()
        for ps in range(self.npass):
            self._pass = ps
            for ci in range(len(self.group)):
                aligned = self._aligned_finals(ci)
                for facs, pre, coefs in self.chain_assign[ci]:
                    outs = [pre]
                    for oi in aligned:
                        new = []
                        for o in outs:
                            for l2 in self.outs[oi].spins:
                                t = list(o)
                                t[oi] = l2
                                new.append(tuple(t))
                        outs = new
                    for k in coefs:
                        for o in outs:
                            self._fset.add((k, self._out(o)))
        self._pass = 0
        self.nf = len(self._fset)
        # stash slots: one (sin, cos) pair per half angle of every chain and pass
        self._slot = {}
        for ps in range(self.npass):
            self._pass = ps
            for ci, c in enumerate(self.group):
                cf = self._cf(ci)
                for vi, d in enumerate(c):
                    self._slot[(ps, ci, f"c{ci}v{vi}b")] = len(self._slot)
                    self._slot[(ps, ci, f"c{ci}v{vi}a")] = len(self._slot)
                for o in cf["aligned"]:
                    oi = self.group.outs.index(o)
                    for a in "bag":
                        self._slot[(ps, ci, f"c{ci}al{oi}{a}")] = len(self._slot)
        self._pass = 0
        self.nstash = 2 * len(self._slot)
        self._mode = "plain"

    # ------------------------------------------------------------ helpers
    def _cst(self, name):
        return f"cR<R>(C, {self.consts.index[name]})"

    def _ci(self, name):
        return str(self.consts.index[name])

    def _cv(self, name):
        """The FP64 constant itself (for mulk / cfmak / cmulk, which keep
        its FP32 rounding from biasing every event alike)."""
        return f"C.v[{self.consts.index[name]}]"

    def _cpx(self, base):
        return f"cmk<R>({self._cst(base + '.re')}, {self._cst(base + '.im')})"

    def _cg_cc(self, d):
        """CG table of vertex d for charge < 0 events: both daughter
        helicity axes reversed where the vertex allows it."""
        cg = d.cg()
        if self.flips and getattr(d, "allow_cc", False):
            return cg[:, ::-1, ::-1]
        return cg

    @staticmethod
    def _coef(v):
        """Literal of a coupling coefficient; a (charge > 0, charge < 0)
        pair becomes a per-event select on ``cc``."""
        if isinstance(v, tuple):
            return f"(cc ? {_lit(v[1])} : {_lit(v[0])})"
        return _lit(v)

    @staticmethod
    def _kcoef(v, bfv):
        """Coefficient v (or a charge-select pair) times the barrier factor
        expression ``bfv`` ("bf * " or empty), hi/lo-split in FP32."""
        x = bfv[:-3] if bfv else "R(1)"
        if isinstance(v, tuple):
            if _f32_exact(v[0]) and _f32_exact(v[1]):
                return f"{x} * (cc ? {_lit(v[1])} : {_lit(v[0])})"
            return f"mulk<R>({x}, cc ? {repr(float(v[1]))} : {repr(float(v[0]))})"
        if _f32_exact(v):
            return f"{x} * {_lit(v)}"
        return f"mulk<R>({x}, {repr(float(v))})"

    def _cf(self, ci):
        """Field references of chain ci in the current pass."""
        if self._pass == 0:
            return self.plan.chains[ci]
        return self.plan.swaps[self._pass - 1]["chains"][ci]

    def _out(self, o):
        """Output index of the chain helicity tuple o = (top, finals...) in
        the current pass: a swap's amplitude enters with its final-helicity
        axes reordered (out-axis j = its axis trans[j]) and, for the
        CP-conjugate passes, every helicity reversed."""
        if self._pass == 0:
            return self.out_index[o]
        sw = self.plan.swaps[self._pass - 1]
        o2 = (o[0],) + tuple(o[1 + t] for t in sw["trans"])
        if sw["flip"]:
            o2 = tuple(-h for h in o2)
        return self.out_index[o2]

    def _factor(self):
        return 1.0 if self._pass == 0 else self.plan.swaps[self._pass - 1]["factor"]

    def _aligned_finals(self, ci):
        cf = self._cf(ci)
        return [self.group.outs.index(o) + 1 for o in self.group.outs if o in cf["aligned"]]

    @staticmethod
    def _d_name(ci, vi, ia, idl):
        return f"D_c{ci}v{vi}_{ia}_{idl}"

    @staticmethod
    def _pre_name(ci, po, pfx):
        return f"{pfx}_c{ci}_" + "_".join(str(two(x) + 8) for x in po)

    def _scale_k(self, ci, k):
        c = self.group[ci]
        lsi = self.columns[k][1]
        sc = []
        for vi, d in enumerate(c):
            if d.has_barrier_factor:
                l = d.get_ls_list()[lsi[vi]][0]
                sc.append(f"bf_c{ci}v{vi}_{l}")
        return " * ".join(sc) if sc else "R(1)"

    def _first_chain(self, p):
        for ci, c in enumerate(self.group):
            if p in c.inner:
                return ci
        return -1

    def _emit_loads(self, e):
        # LDG: read-only global loads; false for fields staged in shared memory
        for f in self.mass_fields:
            a = f"XM + (long long){self.mass_slot[f]} * ld + i"
            e(f"  const double xm{f} = LDG ? __ldg({a}) : *({a});")
        for f in self.angle_fields:
            a = f"XA + (long long){self.angle_slot[f]} * ld + i"
            e(f"  const R xa{f} = LDG ? __ldg({a}) : *({a});")
        if self.flips:
            e(f"  const bool cc = xm{self.plan.charge_index} < 0.0;")

    def _emit_mass_loads(self, e):
        for f in self.mass_fields:
            a = f"XM + (long long){self.mass_slot[f]} * ld + i"
            e(f"  const double xm{f} = LDG ? __ldg({a}) : *({a});")

    def column_barrier_consts(self, k):
        """Constants whose product scales column k's barrier factors (each
        vertex's q^l sqrt(Pz0_l / B(q^2)) times norm_l): ("sqrt", name) per
        vertex with a B' factor, ("lin", name) per normalised one."""
        ci, lsi = self.columns[k]
        out = []
        for vi, d in enumerate(self.group[ci]):
            if d.has_barrier_factor:
                l = d.get_ls_list()[lsi[vi]][0]
                if d.has_bprime:
                    out.append(("sqrt", f"{d}.Pz0_{l}"))
                if d.barrier_factor_norm:
                    out.append(("lin", f"{d}.norm_{l}"))
        return out

    @property
    def shape_cache_ok(self):
        """Whether the columns factorise as (lineshapes of the chain) x
        (shape-free column): one pass (no identical-particle swaps), no
        polarised parent, no CP-violating totals."""
        return self.npass == 1 and not self.pol_names and not self.cp_chains

    def _trig(self, e, ci, key, angle):
        """sin/cos of half an angle: computed (and stashed in the forward
        pass) or read back from the stash (adjoint pass)."""
        nm = f"{key}"
        slot = self._slot[(self._pass, ci, key)]
        if self._mode == "load":
            e(f"  const R s_{nm} = st[{2 * slot} * PWA_TPB], c_{nm} = st[{2 * slot + 1} * PWA_TPB];")
        else:
            e(f"  R s_{nm}, c_{nm};")
            e(f"  psincos(R(0.5) * {angle}, &s_{nm}, &c_{nm});")
            if self._mode == "store":
                e(f"  if (STASH) {{ st[{2 * slot} * PWA_TPB] = s_{nm}; st[{2 * slot + 1} * PWA_TPB] = c_{nm}; }}")
        return f"s_{nm}", f"c_{nm}"

    def _emit_chain_common(self, e, ci):
        """Masses, q^2, barrier factors, D elements, alignment D and
        lineshapes of chain ci (names prefixed by the chain)."""
        c = self.group[ci]
        cf = self._cf(ci)
        cst = self._cst

        def dmass(p):
            if p in c.inner:
                return f"xm{cf['mass'][p]}"
            return repr(float(p.mass))

        for vi, d in enumerate(c):
            a, (b, cc) = d.core, d.outs
            tag = f"c{ci}v{vi}"
            fa = cf["decays"][vi]
            if d.has_barrier_factor:
                e(f"  const R q2_{tag} = R(rel_p2<double>({dmass(a)}, {dmass(b)}, {dmass(cc)}));")
                for l in sorted(set(d.get_l_list())):
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
                        e(f"  R bp_{tag}_{l} = mulkc<R>(R(1) / ({poly}), C, {self._ci(f'{d}.Pz0_{l}')});")
                        e(f"  bp_{tag}_{l} = bp_{tag}_{l} > R(0) ? bp_{tag}_{l} : R(1);")
                        bf = f"({ql}) * psqrt(bp_{tag}_{l})"
                    else:
                        bf = ql
                    if d.barrier_factor_norm:
                        bf = f"mulkc<R>({bf}, C, {self._ci(f'{d}.norm_{l}')})"
                    e(f"  const R bf_{tag}_{l} = {bf};")
            # D*^{Ja}_{la, lb-lc}(alpha, beta, 0); indices are 2m + 2J
            j2 = two(a.J)
            need = set()
            for la in a.spins:
                for lb in b.spins:
                    for lc in cc.spins:
                        dl = lb - lc
                        if abs(dl) <= a.J + 1e-9:
                            need.add((two(la) + j2, two(dl) + j2))
            e(f"  R sp_{tag}[{j2 + 1}], cp_{tag}[{j2 + 1}];")
            sb, cb = self._trig(e, ci, f"{tag}b", f"xa{fa['beta']}")
            e(f"  sc_powers<R, {j2}>({sb}, {cb}, sp_{tag}, cp_{tag});")
            need_alpha = any(i1 != j2 for i1, _ in need)
            if need_alpha:
                e(f"  cpx<R> ea_{tag}[{2 * j2 + 1}];")
                sa, ca = self._trig(e, ci, f"{tag}a", f"xa{fa['alpha']}")
                e(f"  half_angle_powers_sc<R, {j2}>({sa}, {ca}, ea_{tag});")
            w = small_d_weight(j2)
            for i1, i2 in sorted(need):
                k1, k2 = i1 // 2, i2 // 2
                terms = [_klit(w[l][k1][k2], f"(sp_{tag}[{l}] * cp_{tag}[{j2 - l}])")
                         for l in range(j2 + 1) if w[l][k1][k2] != 0]
                dexpr = " + ".join(terms) if terms else "R(0)"
                nm = self._d_name(ci, vi, i1, i2)
                if need_alpha and i1 != j2:
                    e(f"  const cpx<R> {nm} = cscale(ea_{tag}[{i1}], {dexpr});")
                else:
                    e(f"  const cpx<R> {nm} = cmk<R>({dexpr}, R(0));")
        for o, (fa_, fb_, fg_) in cf["aligned"].items():
            oi = self.group.outs.index(o)
            tag = f"c{ci}al{oi}"
            j2 = two(o.J)
            e(f"  R sp_{tag}[{j2 + 1}], cp_{tag}[{j2 + 1}];")
            sb, cb = self._trig(e, ci, f"{tag}b", f"xa{fb_}")
            e(f"  sc_powers<R, {j2}>({sb}, {cb}, sp_{tag}, cp_{tag});")
            e(f"  cpx<R> ea_{tag}[{2 * j2 + 1}], eg_{tag}[{2 * j2 + 1}];")
            sa, ca = self._trig(e, ci, f"{tag}a", f"xa{fa_}")
            e(f"  half_angle_powers_sc<R, {j2}>({sa}, {ca}, ea_{tag});")
            sg, cg = self._trig(e, ci, f"{tag}g", f"xa{fg_}")
            e(f"  half_angle_powers_sc<R, {j2}>({sg}, {cg}, eg_{tag});")
            w = small_d_weight(j2)
            for l1 in o.spins:
                for l2 in o.spins:
                    n1, n2 = two(l1) + j2, two(l2) + j2
                    terms = [_klit(w[l][n1 // 2][n2 // 2], f"(sp_{tag}[{l}] * cp_{tag}[{j2 - l}])")
                             for l in range(j2 + 1) if w[l][n1 // 2][n2 // 2] != 0]
                    dexpr = " + ".join(terms) if terms else "R(0)"
                    e(f"  const cpx<R> Dal_{tag}_{n1}_{n2} = cscale(cmul(ea_{tag}[{n1}], eg_{tag}[{n2}]), {dexpr});")
        self._emit_lineshapes(e, ci)

    def _emit_lineshapes(self, e, ci):
        """Lineshapes of chain ci's resonances from their invariant masses and
        the constant block: bw_<tag> per resonance, BW_c<ci> their product."""
        c = self.group[ci]
        cf = self._cf(ci)
        cst = self._cst

        def dmass(p):
            if p in c.inner:
                return f"xm{cf['mass'][p]}"
            return repr(float(p.mass))

        bw_names = []
        for p in c.inner:
            kind = p.lineshape_kind()
            if kind == "one":
                continue
            tag = f"c{ci}r{c.inner.index(p)}"
            m = f"xm{cf['mass'][p]}"
            bw_names.append(f"bw_{tag}")
            e(f"  const R xr_{tag} = R(C.v[{self.consts.index[f'{p}.m0sq']}] - {m} * {m});")
            if kind == "BWR2":
                # m0 Gamma2(m) = K (r^L sqrt|r|) / (m B(q^2)), r = q^2 / q0^2,
                # real for r >= 0 and imaginary for r < 0 (principal sqrt);
                # value (Re D + i Im D) / |D|^2 of D = m0^2 - m^2 - i m0 Gamma2
                dp = c.decay_of(p)
                b, cc = dp.outs
                L_ = p.bw_l if p.bw_l is not None else min(dp.get_l_list())
                e(f"  const R qq_{tag} = R(rel_p2<double>({m}, {dmass(b)}, {dmass(cc)}));")
                co = bprime_coeff(L_)
                z = f"(qq_{tag} * {_lit(p.d * p.d)})"
                poly = _lit(co[0])
                for cc_ in co[1:]:
                    poly = f"fma({poly}, {z}, {_lit(cc_)})"
                e(f"  const R rr_{tag} = mulkc<R>(qq_{tag}, C, {self._ci(f'{p}.iq02')});")
                ph = f"psqrt(rr_{tag} < R(0) ? -rr_{tag} : rr_{tag})"
                for _ in range(L_):
                    ph = f"{ph} * rr_{tag}"
                e(f"  const R ya_{tag} = mulkc<R>(({ph}) / (R({m}) * ({poly})), C, {self._ci(f'{p}.K')});")
                e(f"  const R y_{tag} = rr_{tag} < R(0) ? R(0) : ya_{tag};")
                e(f"  const R yi_{tag} = rr_{tag} < R(0) ? ya_{tag} : R(0);")
                e(f"  const R dre_{tag} = xr_{tag} + yi_{tag};")
                e(f"  const R s_{tag} = dre_{tag} * dre_{tag} + y_{tag} * y_{tag};")
                # one reciprocal for both parts (a division each would be two)
                e(f"  const R is_{tag} = R(1) / s_{tag};")
                e(f"  const cpx<R> bw_{tag} = cmk<R>(dre_{tag} * is_{tag}, -y_{tag} * is_{tag});")
            else:
                if kind == "BWR":
                    dp = c.decay_of(p)
                    b, cc = dp.outs
                    L_ = p.bw_l if p.bw_l is not None else min(dp.get_l_list())
                    e(f"  const R q_{tag} = R(rel_p<double>({m}, {dmass(b)}, {dmass(cc)}));")
                    co = bprime_coeff(L_)
                    z = f"(q_{tag} * q_{tag} * {_lit(p.d * p.d)})"
                    poly = _lit(co[0])
                    for cc_ in co[1:]:
                        poly = f"fma({poly}, {z}, {_lit(cc_)})"
                    qp = "*".join([f"q_{tag}"] * (2 * L_ + 1))
                    e(f"  const R qp_{tag} = {cst(f'{p}.useq')} != R(0) ? ({qp}) : R(1);")
                    e(f"  const R y_{tag} = mulkc<R>(qp_{tag} / (R({m}) * ({poly})), C, {self._ci(f'{p}.K')});")
                    e(f"  const R s_{tag} = xr_{tag} * xr_{tag} + y_{tag} * y_{tag};")
                    e(f"  const R is_{tag} = R(1) / s_{tag};")
                    e(f"  const cpx<R> bw_{tag} = cmk<R>(xr_{tag} * is_{tag}, y_{tag} * is_{tag});")
                else:
                    # constant width: value from the FP64 m0^2 - m^2 and m0 Gamma0
                    e(f"  const R y_{tag} = {cst(f'{p}.y')};")
                    e(f"  cpx<R> bw_{tag};")
                    e(f"  {{ const double xd = {self._cv(f'{p}.m0sq')} - {m} * {m}, "
                      f"yd = {self._cv(f'{p}.y')}, sd = xd * xd + yd * yd;")
                    e("    const double isd = 1.0 / sd;")
                    e(f"    bw_{tag} = cmk<R>(R(xd * isd), R(yd * isd)); }}")
            if p.width_norm_applies():
                # the chain product takes Gamma0 R (the derivatives use R)
                wn = self._ci(f'{p}.wn')
                bw_names[-1] = (f"cmk<R>(mulkc<R>(bw_{tag}.re, C, {wn}), "
                                f"mulkc<R>(bw_{tag}.im, C, {wn}))")
        if bw_names:
            e(f"  cpx<R> BW_c{ci} = {bw_names[0]};")
            for nm in bw_names[1:]:
                e(f"  BW_c{ci} = cmul(BW_c{ci}, {nm});")
        else:
            e(f"  const cpx<R> BW_c{ci} = cmk<R>(R(1), R(0));")

    def _emit_align_forward(self, e, ci, cur, pfx):
        """Contract each aligned final's helicity with D*(aligned angles)."""
        for oi in self._aligned_finals(ci):
            o = self.outs[oi]
            j2 = two(o.J)
            tag = f"c{ci}al{oi - 1}"
            targets = set()
            for po in cur:
                for l2 in o.spins:
                    t = list(po)
                    t[oi] = l2
                    targets.add(tuple(t))
            new = {}
            for to in sorted(targets, key=_key):
                nm = self._pre_name(ci, to, f"{pfx}{oi}")
                e(f"  cpx<R> {nm} = cmk<R>(R(0), R(0));")
                for l1 in o.spins:
                    s_ = list(to)
                    s_[oi] = l1
                    s_ = tuple(s_)
                    if s_ in cur:
                        e(f"  cfmac({nm}, {cur[s_]}, Dal_{tag}_{two(l1) + j2}_{two(to[oi]) + j2});")
                new[to] = nm
            cur = new
        return cur

    # ------------------------------------------------------------ forward
    def _emit_forward(self, e):
        for oj in range(self.nout):
            e(f"  cpx<R> A{oj} = cmk<R>(R(0), R(0));")
        for ps in range(self.npass):
            self._pass = ps
            self._emit_forward_pass(e)
        self._pass = 0

    def _emit_forward_pass(self, e):
        for ci, c in enumerate(self.group):
            e(f"  {{ // chain {ci}: {c}" + (f" (swap {self._pass})" if self._pass else ""))
            self._emit_chain_common(e, ci)
            hnames = {}
            for vi, d in enumerate(c):
                b, cc = d.outs
                cg = d.cg()
                cgc = self._cg_cc(d)
                ls = d.get_ls_list()
                for ib in range(len(b.spins)):
                    for ic in range(len(cc.spins)):
                        terms = [(i, cg[i, ib, ic] if cg[i, ib, ic] == cgc[i, ib, ic]
                                  else (cg[i, ib, ic], cgc[i, ib, ic]))
                                 for i in range(len(ls))
                                 if cg[i, ib, ic] != 0 or cgc[i, ib, ic] != 0]
                        if not terms:
                            continue
                        nm = f"H_c{ci}v{vi}_{ib}_{ic}"
                        hnames[(vi, ib, ic)] = nm
                        e(f"  cpx<R> {nm} = cmk<R>(R(0), R(0));")
                        for i, cgv in terms:
                            l = ls[i][0]
                            bfv = f"bf_c{ci}v{vi}_{l} * " if d.has_barrier_factor else ""
                            g = f"{d}.g{i}"
                            e(f"  cfmakc({nm}, {self._kcoef(cgv, bfv)}, C, {self._ci(g + '.re')}, "
                              f"{self._ci(g + '.im')});")
            pre = {}
            for facs, po, coefs in self.chain_assign[ci]:
                if any((vi, ib, ic) not in hnames for (vi, _, _, ib, ic) in facs):
                    continue
                vs = [f"cmul({hnames[(vi, ib, ic)]}, {self._d_name(ci, vi, ia, idl)})"
                      for (vi, ia, idl, ib, ic) in facs]
                nm = pre.get(po)
                if nm is None:
                    nm = self._pre_name(ci, po, "Ap")
                    pre[po] = nm
                    e(f"  cpx<R> {nm} = cmk<R>(R(0), R(0));")
                if len(vs) == 1:
                    e(f"  {nm} = cadd({nm}, {vs[0]});")
                else:
                    prod = vs[0]
                    for v in vs[1:-1]:
                        prod = f"cmul({prod}, {v})"
                    e(f"  cfmac({nm}, {prod}, {vs[-1]});")
            cur = self._emit_align_forward(e, ci, pre, "Aa")
            if ci in self.cp_chains and self.ncp:
                # per-event charge selects the total: the FP64 values (a
                # thread-dependent index into the constant block would copy it
                # to local memory)
                tre = f"(cc ? {self._cv(f't{ci}m.re')} : {self._cv(f't{ci}.re')})"
                tim = f"(cc ? {self._cv(f't{ci}m.im')} : {self._cv(f't{ci}.im')})"
                tot = f"cmulk<R>({tre}, {tim}, BW_c{ci})"
            else:
                tot = f"cmulkc<R>(C, {self._ci(f't{ci}.re')}, {self._ci(f't{ci}.im')}, BW_c{ci})"
            if self._factor() == 1.0:
                e(f"  const cpx<R> E_c{ci} = {tot};")
            else:
                e(f"  const cpx<R> E_c{ci} = cscale({tot}, {_lit(self._factor())});")
            for o, nm in cur.items():
                e(f"  cfmac(A{self._out(o)}, E_c{ci}, {nm});")
            e("  }")

    # ------------------------------------------------------------ adjoint
    def _emit_adjoint(self, e):
        for si, p in enumerate(self.shape_res):
            e(f"  cpx<R> SR{si} = cmk<R>(R(0), R(0)), dm{si} = SR{si}, dg{si} = SR{si};")
        for ps in range(self.npass):
            self._pass = ps
            if ps:
                for si in range(len(self.shape_res)):
                    e(f"  SR{si} = cmk<R>(R(0), R(0));")
            self._emit_adjoint_pass(e)
            # lineshape sensitivities of this pass (its own masses)
            for si, p in enumerate(self.shape_res):
                e(f"  accs[{2 * si}] += 2.0 * double(cmul(SR{si}, dm{si}).re);")
                e(f"  accs[{2 * si + 1}] += 2.0 * double(cmul(SR{si}, dg{si}).re);")
        self._pass = 0

    def _emit_adjoint_pass(self, e):
        fac = self._factor()
        for ci, c in enumerate(self.group):
            e(f"  {{ // chain {ci}: {c}" + (f" (swap {self._pass})" if self._pass else ""))
            self._emit_chain_common(e, ci)
            # seed of each chain helicity tuple: the adjoint of the output it
            # enters (times the swap sign)
            if fac == 1.0:
                cur = {o: f"Ab[{self._out(o)}]" for o in self.out_index}
            else:
                cur = {o: f"cscale(Ab[{self._out(o)}], {_lit(fac)})" for o in self.out_index}
            for oi in reversed(self._aligned_finals(ci)):
                o = self.outs[oi]
                j2 = two(o.J)
                tag = f"c{ci}al{oi - 1}"
                keys = set()
                for to in cur:
                    for l1 in o.spins:
                        t = list(to)
                        t[oi] = l1
                        keys.add(tuple(t))
                new = {}
                for po in sorted(keys, key=_key):
                    nm = self._pre_name(ci, po, f"Bb{oi}")
                    e(f"  cpx<R> {nm} = cmk<R>(R(0), R(0));")
                    for l2 in o.spins:
                        t = list(po)
                        t[oi] = l2
                        t = tuple(t)
                        if t in cur:
                            e(f"  cfmac({nm}, {cur[t]}, Dal_{tag}_{two(po[oi]) + j2}_{two(l2) + j2});")
                    new[po] = nm
                cur = new
            cols = self.chain_columns[ci]
            for k in cols:
                e(f"  cpx<R> Gk{k} = cmk<R>(R(0), R(0));")
            for facs, po, coefs in self.chain_assign[ci]:
                if po not in cur:
                    continue
                ds = [self._d_name(ci, vi, ia, idl) for (vi, ia, idl, _, _) in facs]
                prod = ds[0]
                for dn in ds[1:]:
                    prod = f"cmul({prod}, {dn})"
                e(f"  {{ const cpx<R> rr = cmul({prod}, {cur[po]});")
                for k, cfv in coefs.items():
                    e(f"    cfma(Gk{k}, {self._coef(cfv)}, rr);")
                e("  }")
            for k in cols:
                e(f"  {{ const cpx<R> g = cmul(cscale(BW_c{ci}, {self._scale_k(ci, k)}), Gk{k});")
                ck = self._cpx(f"c{k}")
                if k in self.cp_pos and self.ncp:
                    # charge -1 events: their own sums, after the polarisation ones
                    j = self.nshape + self.nrho + 2 * self.cp_pos[k]
                    e(f"    if (cc) {{ accs[{j}] += double(g.re); accs[{j + 1}] += double(g.im); }}")
                    e(f"    else {{ accg[{2 * k}] += double(g.re); accg[{2 * k + 1}] += double(g.im); }}")
                    ck = f"(cc ? {self._cpx(f'c{k}m')} : {ck})"
                else:
                    e(f"    accg[{2 * k}] += double(g.re); accg[{2 * k + 1}] += double(g.im);")
                for si, p in enumerate(self.shape_res):
                    if p in c.inner:
                        e(f"    cfmac(SR{si}, {ck}, g);")
                e("  }")
            self._emit_shape_derivs(e, ci, "dm{si}", "dg{si}")
            e("  }")

    def _emit_shape_derivs(self, e, ci, dm_fmt, dg_fmt):
        """Log-derivatives of each floating lineshape R whose first chain is
        ci with respect to m0 and Gamma0 (kappa_m = dlog(m0 Gamma) / dm0 at
        fixed m), into the names dm_fmt / dg_fmt (formatted with si)."""
        c = self.group[ci]
        for si, p in enumerate(self.shape_res):
            if p in c.inner and self._first_chain(p) == ci:
                tag = f"c{ci}r{c.inner.index(p)}"
                dm, dg = dm_fmt.format(si=si), dg_fmt.format(si=si)
                kap, ig = self._cst(f"{p}.kappa_m"), self._cst(f"{p}.inv_g0")
                e(f"  {{ const R m0 = psqrt({self._cst(f'{p}.m0sq')});")
                if p.lineshape_kind() == "BWR2":
                    # R = 1 / conj(D): dlog R = -R conj(dD)
                    e(f"    {dm} = cmul(bw_{tag}, cmk<R>(-(R(2) * m0 + yi_{tag} * {kap}), -y_{tag} * {kap}));")
                    e(f"    {dg} = cmul(bw_{tag}, cmk<R>(-yi_{tag} * {ig}, -y_{tag} * {ig}));")
                else:
                    e(f"    {dm} = cmul(bw_{tag}, cmk<R>(R(-2) * m0, y_{tag} * {kap}));")
                    e(f"    {dg} = cmul(bw_{tag}, cmk<R>(R(0), y_{tag} * {ig}));")
                if p.width_norm_applies():
                    e(f"    {dg}.re += {ig};")
                e("  }")

    # ------------------------------------------------------------ columns
    def _emit_columns(self, e):
        for j in range(self.ncol * self.nout):
            e(f"  F[{j}] = cmk<R>(R(0), R(0));")
        for ps in range(self.npass):
            self._pass = ps
            self._emit_columns_pass(e)
        self._pass = 0

    def _emit_columns_pass(self, e):
        fac = self._factor()
        for ci, c in enumerate(self.group):
            e(f"  {{ // chain {ci}: {c}" + (f" (swap {self._pass})" if self._pass else ""))
            self._emit_chain_common(e, ci)
            for k in self.chain_columns[ci]:
                e("  {")
                pre = {}
                for facs, po, coefs in self.chain_assign[ci]:
                    if k not in coefs:
                        continue
                    ds = [self._d_name(ci, vi, ia, idl) for (vi, ia, idl, _, _) in facs]
                    prod = ds[0]
                    for dn in ds[1:]:
                        prod = f"cmul({prod}, {dn})"
                    nm = pre.get(po)
                    if nm is None:
                        nm = self._pre_name(ci, po, "Fp")
                        pre[po] = nm
                        e(f"  cpx<R> {nm} = cmk<R>(R(0), R(0));")
                    e(f"  cfma({nm}, {self._coef(coefs[k])}, {prod});")
                cur = self._emit_align_forward(e, ci, pre, "Fa")
                if getattr(self, "_noshape", False):
                    # the column without its chain's lineshapes (they are
                    # applied per evaluation from the masses)
                    e(f"  const cpx<R> S = cmk<R>({self._scale_k(ci, k)}, R(0));")
                else:
                    e(f"  const cpx<R> S = cscale(BW_c{ci}, {self._scale_k(ci, k)});")
                for o, nm in cur.items():
                    j = k * self.nout + self._out(o)
                    if self._pass == 0:
                        e(f"  F[{j}] = cmul(S, {nm});")
                    else:
                        e(f"  F[{j}] = cadd(F[{j}], cscale(cmul(S, {nm}), {_lit(fac)}));")
                e("  }")
            e("  }")

    # ------------------------------------------------------------ |A|^2
    def _pdf_source(self):
        """``model_f``: sum |A|^2 (``tf_pwa/amp/core.py:1919-1931``) or, for a
        polarised parent, sum_l sum_ab Re A_al rho_ab A_bl^* (core.py:
        1933-1951); ``model_seed``: the adjoint seed dF/dA times fac and, when
        polarised, the sums T_ab += fac sum_l A_al A_bl^* (accr)."""
        L = ["template <typename R>",
             "__device__ __forceinline__ double model_f(const Consts& C, const cpx<R>* A) {",
             "  double f = 0.0;"]
        if not self.pol_names:
            L += [f"  f += double(cabs2(A[{o}]));" for o in range(self.nout)]
        else:
            na, nl = self.na, self.nout // self.na
            for a in range(na):
                for b in range(na):
                    re, im = self.consts.index[f"rho{a}_{b}.re"], self.consts.index[f"rho{a}_{b}.im"]
                    for li in range(nl):
                        x, y = a * nl + li, b * nl + li
                        # Re(u rho), u = A_x conj(A_y)
                        L.append(f"  f += C.v[{re}] * (double(A[{x}].re) * double(A[{y}].re) + "
                                 f"double(A[{x}].im) * double(A[{y}].im)) - C.v[{im}] * "
                                 f"(double(A[{x}].im) * double(A[{y}].re) - "
                                 f"double(A[{x}].re) * double(A[{y}].im));")
        L += ["  return f;", "}", "",
              "template <typename R>",
              "__device__ __forceinline__ void model_seed(const Consts& C, const cpx<R>* A, "
              "double fac, cpx<R>* Ab, double* accr) {"]
        if not self.pol_names:
            L += [f"  Ab[{o}] = cmk<R>(R(fac * double(A[{o}].re)), R(-fac * double(A[{o}].im)));"
                  for o in range(self.nout)]
        else:
            na, nl = self.na, self.nout // self.na
            for a in range(na):
                for li in range(nl):
                    x = a * nl + li
                    L.append(f"  {{ double sr = 0.0, si = 0.0;  // sum_b rho_ab conj(A_b)")
                    for b in range(na):
                        y = b * nl + li
                        re, im = self.consts.index[f"rho{a}_{b}.re"], self.consts.index[f"rho{a}_{b}.im"]
                        L.append(f"    sr += C.v[{re}] * double(A[{y}].re) + C.v[{im}] * double(A[{y}].im);")
                        L.append(f"    si += C.v[{im}] * double(A[{y}].re) - C.v[{re}] * double(A[{y}].im);")
                    L.append(f"    Ab[{x}] = cmk<R>(R(fac * sr), R(fac * si)); }}")
            for a in range(na):
                for b in range(na):
                    j = 2 * (a * na + b)
                    terms_r, terms_i = [], []
                    for li in range(nl):
                        x, y = a * nl + li, b * nl + li
                        terms_r.append(f"double(A[{x}].re) * double(A[{y}].re) + "
                                       f"double(A[{x}].im) * double(A[{y}].im)")
                        terms_i.append(f"double(A[{x}].im) * double(A[{y}].re) - "
                                       f"double(A[{x}].re) * double(A[{y}].im)")
                    L.append(f"  accr[{j}] += fac * ({' + '.join(terms_r)});")
                    L.append(f"  accr[{j + 1}] += fac * ({' + '.join(terms_i)});")
        L += ["}", ""]
        return "\n".join(L)

    # ------------------------------------------------------------ emission
    def source(self):
        L = [_HEADER.format(ncol=self.ncol, nout=self.nout, nshape=self.nshape, nacc=self.nacc,
                            nconst=max(len(self.consts), 1))]
        # the per-thread stash of half-angle sin/cos (shared memory, stride
        # PWA_TPB) is used when it fits a 40 KB budget at FP64
        use = 1 if self.nstash * 128 * 8 <= 40 * 1024 else 0
        L.append(f"#define PWA_NSTASH {max(self.nstash, 1)}\n#define PWA_USE_STASH {use}")
        sig = ("    const Consts& C, const R* __restrict__ XA, const double* __restrict__ XM,\n"
               "    long long ld, long long i")
        body = []
        self._mode = "store"
        self._emit_loads(body.append)
        self._emit_forward(body.append)
        L.append(f"template <typename R, bool STASH, bool LDG = true>\n__device__ __forceinline__ void model_amp(\n{sig},\n"
                 "    cpx<R>* __restrict__ A, R* __restrict__ st) {")
        L += body
        L += [f"  A[{oj}] = A{oj};" for oj in range(self.nout)]
        L.append("}\n")
        body = []
        self._mode = "load"
        self._emit_loads(body.append)
        self._emit_adjoint(body.append)
        L.append(f"template <typename R, bool LDG = true>\n__device__ __forceinline__ void model_adj_stash(\n{sig},\n"
                 "    const cpx<R>* __restrict__ Ab, double* __restrict__ accg,\n"
                 "    double* __restrict__ accs, const R* __restrict__ st) {")
        L += body
        L.append("}\n")
        body = []
        self._mode = "plain"
        self._emit_loads(body.append)
        self._emit_adjoint(body.append)
        L.append(f"template <typename R, bool LDG = true>\n__device__ __forceinline__ void model_adj_recompute(\n{sig},\n"
                 "    const cpx<R>* __restrict__ Ab, double* __restrict__ accg,\n"
                 "    double* __restrict__ accs) {")
        L += body
        L.append("}\n")
        body = []
        self._mode = "plain"
        self._emit_loads(body.append)
        self._emit_columns(body.append)
        L.append(f"template <typename R, bool LDG = true>\n__device__ __forceinline__ void model_columns(\n{sig},\n"
                 "    cpx<R>* __restrict__ F) {")
        L += body
        L.append("}\n")
        # columns without lineshapes, and the lineshapes with their
        # log-derivatives from the masses alone (floating-shape column cache)
        body = []
        self._mode = "plain"
        self._noshape = True
        self._emit_loads(body.append)
        self._emit_columns(body.append)
        self._noshape = False
        L.append(f"template <typename R, bool LDG = true>\n__device__ __forceinline__ void model_columns_ns(\n{sig},\n"
                 "    cpx<R>* __restrict__ F) {")
        L += body
        L.append("}\n")
        body = []
        self._emit_mass_loads(body.append)
        for ci in range(len(self.group)):
            body.append(f"  {{ // chain {ci}")
            self._emit_lineshapes(body.append, ci)
            body.append(f"  BW[{ci}] = BW_c{ci};")
            self._emit_shape_derivs(body.append, ci, "DM[{si}]", "DG[{si}]")
            body.append("  }")
        L.append("template <typename R, bool LDG = true>\n__device__ __forceinline__ void model_shapes(\n"
                 "    const Consts& C, const double* __restrict__ XM, long long ld, long long i,\n"
                 "    cpx<R>* __restrict__ BW, cpx<R>* __restrict__ DM, cpx<R>* __restrict__ DG) {")
        L += body
        L.append("}\n")
        nch, nsr = len(self.group), len(self.shape_res)
        L.append(f"#define PWA_NCHAIN {nch}\n#define PWA_NSRES {nsr}\n"
                 f"#define PWA_SHAPE_CACHE_OK {1 if self.shape_cache_ok else 0}")
        L.append("__device__ constexpr int pwa_col_chain[PWA_NCOL] = {" +
                 ", ".join(str(ci) for ci, _ in self.columns) + "};")
        rows = [", ".join("1" if p in c.inner else "0" for c in self.group) for p in self.shape_res]
        L.append("__device__ constexpr int pwa_sres_chain[PWA_NSRES > 0 ? PWA_NSRES : 1][PWA_NCHAIN] = {" +
                 (", ".join("{" + r + "}" for r in rows) if rows else "{" + ", ".join(["0"] * nch) + "}") + "};")
        L.append(self._pdf_source())
        fl = sorted(self._fset)
        L.append(f"#define PWA_NF {self.nf}")
        # blocks per SM of the plain FP64 kernels: 4 where the accumulators
        # are few (Lambda_c, 23: 651 vs 724 us per 2.1e6 events at 3), 3 for
        # larger models, whose FP64 state spills more at 4 (four-body, 85:
        # 6.77 vs 5.95 ms)
        L.append(f"#define PWA_EVAL_MINB {4 if self.nacc <= 32 else 3}")
        # the floating-shape evaluation stages its next events in shared
        # memory (two stages of pairs, masses and weight per event at 128
        # threads) where that takes at most 150 KB per block
        sc_bytes = 2 * (self.nf + max(len(self.mass_fields), 1) + 1) * 128 * 8
        L.append(f"#define PWA_SC_STAGES {2 if sc_bytes <= 150 * 1024 else 0}")
        L.append("__device__ constexpr int pwa_fk[PWA_NF] = {" + ", ".join(str(k) for k, _ in fl) + "};")
        L.append("__device__ constexpr int pwa_fo[PWA_NF] = {" + ", ".join(str(o) for _, o in fl) + "};")
        # dataset step: momenta -> fields, and the phase-space generator;
        # field j goes to XM row pwa_field_slot[j] (pwa_field_mass[j] = 1) or
        # XA row pwa_field_slot[j]
        L.append(self.kin.source())
        L.append(f"#define PWA_NFIELD_MASS {len(self.mass_fields)}")
        nf = self.plan.n_fields
        L.append("__device__ constexpr int pwa_field_mass[PWA_NFIELD] = {" + ", ".join(
            "1" if j in self.mass_slot else "0" for j in range(nf)) + "};")
        L.append("__device__ constexpr int pwa_field_slot[PWA_NFIELD] = {" + ", ".join(
            str(self.mass_slot[j] if j in self.mass_slot else self.angle_slot[j])
            for j in range(nf)) + "};")
        return "\n".join(L)

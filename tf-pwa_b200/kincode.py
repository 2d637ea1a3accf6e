"""Kinematics compiler: emits the CUDA source of a model's dataset step.

Two device functions are generated per model, straight-line code in FP64:

``model_kin(P, F)``     final-state four-momenta (parent rest frame, in
                        ``dat_order``) -> every event field of the plan:
                        invariant masses, helicity angles per decay and
                        alignment angles of spinning finals.  It is the
                        algorithm of ``kinematics.event_fields`` (which
                        restates ``tf_pwa/cal_angle.py:158-251,262-343,
                        346-378,408-490``), unrolled over the model's
                        topologies: node momenta, successive rest-frame
                        momenta, Euler angles with the alpha range bias per
                        out, SU(2) rotation/boost products for alignment.
``model_genbod(U, P)``  one flat phase-space event from uniforms U by the
                        Raubold-Lynch (GENBOD) construction of
                        ``phasespace.generate_weighted`` (the role of
                        ``tf_pwa/phasespace.py:31-368``, with its chain
                        generator for fixed-mass intermediates); returns
                        the event weight over its upper bound.

Generation levels: the parent, and every fixed-mass intermediate that the
reference's phase-space sampler also generates on shell (a node common to
all topologies whose particle has model "one"), each decayed in its own rest
frame and boosted.  Uniform draws of an event, level by level (depth first):
k - 2 sorted uniforms for the intermediate masses of a k-body level, then
(cos theta, phi) of each of its k - 1 splittings; then the phase-space
accept draw (against the product of the levels' weights over their upper
bounds) and the amplitude accept draw.
"""
import math

from .plan import split_swap


def _f(v):
    r = repr(float(v))
    if "e" not in r and "." not in r and "inf" not in r and "nan" not in r:
        r += ".0"
    return r


def _pdk(a, b, c):
    x = (a - b - c) * (a + b + c) * (a - b + c) * (a + b - c)
    return math.sqrt(max(x, 0.0)) / (2 * a)


class KinCode:
    def __init__(self, plan, order):
        self.plan = plan
        self.order = [str(o) for o in order]
        group = plan.group
        finals = {str(o): o for o in group.outs}
        missing = [o for o in self.order if o not in finals]
        if missing or len(self.order) != len(finals):
            raise ValueError(f"dat_order {self.order} does not list the final particles "
                             f"{sorted(finals)}")
        self.parent_mass = group.top.mass
        self.masses = [finals[o].mass for o in self.order]
        self.ok = self.parent_mass is not None and all(m is not None for m in self.masses)
        self.nfin = len(self.order)
        self.nfield = plan.n_fields
        self.levels = self._build_levels() if self.ok else [(self.parent_mass, [])]
        # per level of k bodies: k - 2 sorted uniforms + (cos theta, phi) per
        # splitting; then the phase-space and amplitude accept draws
        self.ndraw = sum(3 * len(b) - 4 for _, b in self.levels) + 2
        self.needs_su2 = any("/aligned/" in f for f in plan.fields)

    # ------------------------------------------------------------ kinematics
    def _emit_kin(self, e):
        plan = self.plan
        fin = {o: i for i, o in enumerate(self.order)}
        cnt = [0]

        def tmp(prefix):
            cnt[0] += 1
            return f"{prefix}{cnt[0]}"

        def build_frames(pexpr):
            """Frames of every topology from the finals' momenta pexpr."""
            frames = []
            for t, topo in enumerate(plan.topos):
                chain = topo.chain
                mom = {}
                for o in chain.outs:
                    mom[o] = pexpr[str(o)]

                def lsum(parts):
                    expr = parts[0]
                    for p in parts[1:]:
                        expr = f"lv_add({expr}, {p})"
                    return expr

                for p in chain.inner:
                    v = tmp(f"t{t}_n")
                    e(f"  const LV {v} = {lsum([mom[f] for f in chain.final_set(p)])};")
                    mom[p] = v
                v = tmp(f"t{t}_top")
                e(f"  const LV {v} = {lsum([mom[f] for f in chain.outs])};")
                mom[chain.top] = v
                top = chain.top
                # successive rest-frame momenta (same visiting order as the host code)
                part, core_map = {}, {}
                decays = list(chain)
                remaining = set(chain.inner) | set(chain.outs)
                while decays:
                    later = []
                    for d in decays:
                        if d.core == top:
                            pr, src = mom[top], mom
                        elif d.core in core_map:
                            par = part[core_map[d.core]]
                            pr, src = par[d.core], par
                        else:
                            later.append(d)
                            continue
                        rp = {}
                        for j in d.outs:
                            core_map[j] = d
                            v = tmp(f"t{t}_r")
                            e(f"  const LV {v} = kin_rest_vector({pr}, {src[j]});")
                            rp[j] = v
                            remaining.discard(j)
                        for j in sorted(remaining, key=str):
                            if j in src:
                                v = tmp(f"t{t}_r")
                                e(f"  const LV {v} = kin_rest_vector({pr}, {src[j]});")
                                rp[j] = v
                        part[d] = rp
                    decays = later
                # helicity angles, frames, SU(2) bookkeeping
                set_x = {top: "V3{1.0, 0.0, 0.0}"}
                set_z = {top: "V3{0.0, 0.0, 1.0}"}
                if plan.random_z:
                    # a moving parent's flight direction is the z axis
                    # (tf_pwa/cal_angle.py:431-438)
                    bz = tmp(f"t{t}_bz")
                    e(f"  V3 {bz} = lv_vec({mom[top]});")
                    e(f"  if (sqrt(v3_dot({bz}, {bz})) < 1e-5) {bz} = V3{{0.0, 0.0, 1.0}};")
                    set_z[top] = bz
                angles, rmat, bmat = {}, {}, {}
                decays = list(chain)
                while decays:
                    later = []
                    for d in decays:
                        if d.core not in set_x:
                            later.append(d)
                            continue
                        bias = -math.pi
                        for j in d.outs:
                            z2 = tmp(f"t{t}_z")
                            a, b, x2 = tmp(f"t{t}_a"), tmp(f"t{t}_b"), tmp(f"t{t}_x")
                            e(f"  const V3 {z2} = lv_vec({part[d][j]});")
                            e(f"  double {a}, {b}; V3 {x2};")
                            e(f"  kin_angle_zx_z_getx({set_z[d.core]}, {set_x[d.core]}, {z2}, "
                              f"&{a}, &{b}, &{x2});")
                            e(f"  {a} = kin_fold({a}, {_f(bias)});")
                            bias -= math.pi
                            set_x[j], set_z[j] = x2, z2
                            angles[(d, j)] = (a, b)
                            if self.needs_su2:
                                bm, rm = tmp(f"t{t}_B"), tmp(f"t{t}_R")
                                e(f"  const SU2 {bm} = su2_boost_z_from_p({part[d][j]});")
                                if d.core in rmat:
                                    e(f"  const SU2 {rm} = su2_mul(su2_rot_yz({b}, {a}), "
                                      f"su2_mul({bmat[d.core]}, {rmat[d.core]}));")
                                else:
                                    e(f"  const SU2 {rm} = su2_rot_yz({b}, {a});")
                                bmat[j], rmat[j] = bm, rm
                    decays = later
                frames.append((topo, angles, rmat, bmat, mom))
            return frames

        # unswapped momenta, then one relabelling per swap (final pi takes the
        # momentum of src[pi], three-momentum reversed in the CP-conjugate ones)
        all_frames = [build_frames({o: f"P[{fin[o]}]" for o in fin})]
        for sw in plan.swaps:
            pe = {}
            for o in fin:
                q = f"P[{fin[sw['src'].get(o, o)]}]"
                pe[o] = f"LV{{{q}.t, -{q}.x, -{q}.y, -{q}.z}}" if sw["neg"] else q
            all_frames.append(build_frames(pe))
        # the plan's fields
        for fi, full_name in enumerate(plan.fields):
            if fi == plan.charge_index:
                # the event's charge is data, not kinematics: +1 here (the
                # generator's events), overwritten by the caller's charges
                e(f"  F[{fi}] = 1.0;")
                continue
            sk, fname = split_swap(full_name)
            frames = all_frames[sk]
            parts = fname.split("/")
            if parts[0] == "m":
                for topo, angles, rmat, bmat, mom in frames:
                    hit = [p for p in topo.chain.inner if topo.node[p] == parts[1]]
                    if hit:
                        e(f"  F[{fi}] = kin_inv_mass({mom[hit[0]]});")
                        break
                continue
            tidx = int(parts[0])
            topo, angles, rmat, bmat, mom = frames[tidx]
            dec = [d for d in topo.chain if topo.decay_name(d) == parts[1]][0]
            part = [o for o in dec.outs if topo.node[o] == parts[2]][0]
            if parts[3] == "aligned":
                ref_t = plan.align_ref[str(part)]
                rtopo, _, rr, rb, _ = frames[ref_t]
                rpart = [o for o in rtopo.chain.outs if str(o) == str(part)][0]
                m, al, be, ga = tmp("al_M"), tmp("al_a"), tmp("al_b"), tmp("al_g")
                e(f"  const SU2 {m} = su2_mul(su2_mul({rb[rpart]}, su2_mul({rr[rpart]}, "
                  f"su2_inv({rmat[part]}))), su2_inv({bmat[part]}));")
                e(f"  double {al}, {be}, {ga};")
                e(f"  su2_euler({m}, &{al}, &{be}, &{ga});")
                e(f"  F[{fi}] = {dict(alpha=al, beta=be, gamma=ga)[parts[4]]};")
            else:
                a, b = angles[(dec, part)]
                e(f"  F[{fi}] = {a if parts[3] == 'alpha' else b};")

    # ------------------------------------------------------------ GENBOD
    def _build_levels(self):
        """Generation structure.  As the reference's phase-space sampler
        (``tf_pwa/config_loader/sample.py:276-340``, build_phsp_chain), an
        inner node present in every topology whose particle has the fixed
        lineshape (model "one") and a mass is generated on shell: its
        daughters come from a two-(or more)-body decay in its rest frame.
        Levels in depth-first order, level 0 = the parent; each level is
        (mass, [(kind, ref, mass)]) with kind "f" (ref = index in dat_order)
        or "n" (ref = level index)."""
        plan = self.plan
        fin = {o: i for i, o in enumerate(self.order)}
        sets = None
        node_particle = {}
        for topo in plan.topos:
            here = set()
            for p in topo.chain.inner:
                fs = frozenset(str(f) for f in topo.chain.final_set(p))
                here.add(fs)
                node_particle.setdefault(fs, []).append(p)
            sets = here if sets is None else sets & here
        fixed = {}
        for fs in sets or ():
            ps = node_particle[fs]
            if all(p.lineshape_kind() == "one" and getattr(p, "model", None) == "one"
                   and p.mass is not None for p in ps):
                fixed[fs] = ps[0].mass
        levels = []

        def build(mass, finals):
            lid = len(levels)
            levels.append(None)
            inner = [fs for fs in fixed if fs < finals]
            # maximal fixed nodes inside this level
            tops = [fs for fs in inner if not any(fs < g for g in inner)]
            covered = set().union(*tops) if tops else set()
            bodies = [("f", fin[f], self.masses[fin[f]]) for f in finals - covered]
            for fs in tops:
                bodies.append(("n", fs, fixed[fs]))
            bodies.sort(key=lambda b: b[1] if b[0] == "f" else min(fin[f] for f in b[1]))
            out = []
            for kind, ref, m in bodies:
                if kind == "n":
                    ref = build(m, ref)
                out.append((kind, ref, m))
            levels[lid] = (mass, out)
            return lid

        build(self.parent_mass, frozenset(self.order))
        return levels

    def _emit_genbod(self, e):
        levels = self.levels
        draw = 0
        e("  double w = 1.0;")
        two_pi = _f(2 * math.pi)
        for lid, (M, bodies) in enumerate(levels):
            ms = [m for _, _, m in bodies]
            k = len(ms)
            tm = M - sum(ms)
            if tm <= 0:
                raise ValueError("a generation level is below the sum of its daughter masses")
            cum = [sum(ms[:i + 1]) for i in range(k)]
            emmax, emmin, wtmax = tm + ms[0], 0.0, 1.0
            for i in range(1, k):
                emmin += ms[i - 1]
                emmax += ms[i]
                wtmax *= _pdk(emmax, emmin, ms[i])
            pre = f"g{lid}_"
            e(f"  LV {pre}b[{k}];")
            e("  {")
            k2 = k - 2
            if k2 > 0:
                e(f"    double r[{k2}];")
                for j in range(k2):
                    e(f"    r[{j}] = U[{draw + j}];")
                for i in range(k2):
                    for j in range(k2 - 1 - i):
                        e(f"    {{ const double lo = fmin(r[{j}], r[{j + 1}]), hi = fmax(r[{j}], "
                          f"r[{j + 1}]); r[{j}] = lo; r[{j + 1}] = hi; }}")
            draw += k2
            e(f"    const double Ms0 = {_f(ms[0])};")
            for i in range(1, k - 1):
                e(f"    const double Ms{i} = r[{i - 1}] * {_f(tm)} + {_f(cum[i])};")
            e(f"    const double Ms{k - 1} = {_f(M)};")
            e("    double wl = 1.0;")
            for i in range(1, k):
                e(f"    const double pd{i} = kin_pdk(Ms{i}, Ms{i - 1}, {_f(ms[i])});")
                e(f"    wl *= pd{i};")
            for i in range(1, k):
                cu, pu = draw, draw + 1
                draw += 2
                e(f"    {{ const double cth = 2.0 * U[{cu}] - 1.0, phi = {two_pi} * U[{pu}];")
                e("      const double sth = sqrt(fmax(1.0 - cth * cth, 0.0));")
                e("      double sp, cp; sincos(phi, &sp, &cp);")
                e(f"      const double q = pd{i};")
                e("      const V3 p3 = {q * sth * cp, q * sth * sp, q * cth};")
                if i == 1:
                    e(f"      {pre}b[0] = LV{{sqrt(q * q + {_f(ms[0] ** 2)}), -p3.x, -p3.y, -p3.z}};")
                    e(f"      {pre}b[1] = LV{{sqrt(q * q + {_f(ms[1] ** 2)}), p3.x, p3.y, p3.z}};")
                else:
                    e(f"      const double Esys = sqrt(q * q + Ms{i - 1} * Ms{i - 1});")
                    e("      const V3 beta = {-p3.x / Esys, -p3.y / Esys, -p3.z / Esys};")
                    for j in range(i):
                        e(f"      {pre}b[{j}] = kin_boost({pre}b[{j}], beta);")
                    e(f"      {pre}b[{i}] = LV{{sqrt(q * q + {_f(ms[i] ** 2)}), p3.x, p3.y, p3.z}};")
                e("    }")
            e(f"    w *= wl / {_f(wtmax)};")
            e("  }")
        assert draw + 2 == self.ndraw

        def place(lid, frame):
            for j, (kind, ref, _) in enumerate(levels[lid][1]):
                p = f"g{lid}_b[{j}]"
                if frame is not None:
                    p = (f"kin_boost({p}, V3{{{frame}.x / {frame}.t, {frame}.y / {frame}.t, "
                         f"{frame}.z / {frame}.t}})")
                if kind == "f":
                    e(f"  P[{ref}] = {p};")
                else:
                    e(f"  const LV g{ref}_frame = {p};")
                    place(ref, f"g{ref}_frame")

        place(0, None)
        e("  return w;")

    def source(self):
        L = [f"#define PWA_NFIN {self.nfin}", f"#define PWA_NFIELD {self.nfield}",
             f"#define PWA_NDRAW {self.ndraw}", f"#define PWA_HAS_GENBOD {int(self.ok)}"]
        body = []
        self._emit_kin(body.append)
        L.append("__device__ __forceinline__ void model_kin(const LV (&P)[PWA_NFIN], "
                 "double (&F)[PWA_NFIELD]) {")
        L += body
        L.append("}\n")
        L.append("__device__ __forceinline__ double model_genbod(const double (&U)[PWA_NDRAW], "
                 "LV (&P)[PWA_NFIN]) {")
        if self.ok:
            body = []
            self._emit_genbod(body.append)
            L += body
        else:
            L.append("  return 0.0;  // masses not given: no generator")
        L.append("}\n")
        return "\n".join(L)

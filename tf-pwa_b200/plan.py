"""Event-field layout of a model: which per-event inputs the hot path reads.

The engine consumes structure-of-arrays event data.  Each column ("field") is
one per-event quantity produced once per dataset by the kinematics step:

* ``m/<node>``: invariant mass of an intermediate node, e.g. ``m/(B, C)``;
* ``<t>/<decay>/<particle>/{alpha,beta,gamma}``: helicity angles of a
  particle in its mother's frame, for topology ``t``;
* ``<t>/<decay>/<final>/aligned/{alpha,beta,gamma}``: Wigner alignment
  angles of a final particle with spin in a non-reference chain;
* ``charge``: the event's charge_conjugation (+1 / -1), when the data carry
  charges and ``cp_trans`` is off: charge -1 events flip the helicity
  couplings of the vertices that allow it (``tf_pwa/amp/core.py:938-945``).
  With ``cp_trans`` (the default) charge -1 events are parity-transformed
  before the angles are computed instead (``tf_pwa/cal_angle.py:569-573``).

With identical final particles (``data.identical_particles``), every
non-identity permutation of them adds a "swap": the same fields computed
from the relabelled momenta, named ``s<k>|<field>``
(``tf_pwa/cal_angle.py:684-756``), with the sign and helicity-axis order
its amplitude is added with (``tf_pwa/amp/core.py:1826-1882``).  With
``data.cp_particles`` the CP-conjugate configuration (charge-conjugate
finals exchanged, three-momenta reversed) and its own identical-particle
swaps are further swaps, added with every helicity reversed and the product
of the self-conjugate finals' C parities
(``tf_pwa/cal_angle.py:708-717,799-822``, ``tf_pwa/amp/core.py:1884-1913``).

Node and decay names follow the reference's standard topology
(``tf_pwa/particle.py:698-717``): an inner node is named by its sorted final
particles, ``(B, C)``; topologies are enumerated as in
``tf_pwa/particle.py:902-921`` (first chain of each topology, in chain
order).  Angles are the ones ``tf_pwa/cal_angle.py:262-490`` attaches to the
standard topology; a chain reads the angles of its own decay's ``outs[0]``
(``tf_pwa/amp/core.py:1149-1164``) and alignment angles of its finals
(``tf_pwa/amp/core.py:1414-1429``).  Helicity ``gamma`` is identically zero
for two-body helicity angles and is not stored.
"""


import itertools


def node_name(finals):
    return "({})".format(", ".join(sorted(str(i) for i in finals)))


class ChainTopology:
    """Standard-topology view of one chain: node names for every particle."""

    def __init__(self, chain):
        self.chain = chain
        self.node = {}
        for p in chain.outs:
            self.node[p] = str(p)
        for p in chain.inner:
            self.node[p] = node_name(chain.final_set(p))
        self.node[chain.top] = str(chain.top)
        self.id = tuple(sorted(node_name(chain.final_set(p)) for p in chain.inner))

    def decay_name(self, d):
        return "{}->{}".format(self.node[d.core], "+".join(self.node[o] for o in d.outs))

    def decay_key(self, d):
        return (self.node[d.core], tuple(sorted(self.node[o] for o in d.outs)))


class Plan:
    """Field layout + per-chain references into it."""

    def __init__(self, group, order=None):
        self.group = group
        # order of the final particles in momentum input (the config's
        # data.dat_order; default: the decay group's finals)
        self.order = [str(o) for o in (order if order is not None else group.outs)]
        self.topos = []          # list of ChainTopology (first chain of each)
        self.chain_topo = []     # per chain: index into self.topos
        for c in group:
            t = ChainTopology(c)
            for k, t0 in enumerate(self.topos):
                if t0.id == t.id:
                    self.chain_topo.append(k)
                    break
            else:
                self.chain_topo.append(len(self.topos))
                self.topos.append(t)
        self.fields = []
        self._index = {}
        self._prefix = ""
        self.align_ref = self._alignment_reference()
        self.chains = [self._chain_fields(i, c) for i, c in enumerate(group)]
        # per-event charge_conjugation (+1 / -1) when the data carry charges:
        # with cp_trans, charge < 0 momenta are parity-transformed before the
        # angles; otherwise the charge is a field that flips the helicity
        # couplings of the vertices that allow it
        self.use_charge = bool(getattr(group, "charge", False))
        self.cp_trans = getattr(group, "cp_trans", True)
        # a moving parent's flight direction is the z axis of its decay
        self.random_z = getattr(group, "random_z", True)
        flips = any(getattr(d, "allow_cc", False) for c in group for d in c)
        cp_totals = any(getattr(c, "is_cp", False) for c in group)
        self.charge_index = self.field("charge") if self.use_charge and (flips or cp_totals) \
            else None
        self.swaps = []
        for k, sw in enumerate(pass_specs(group, getattr(group, "identical_particles", None),
                                          getattr(group, "cp_particles", None))):
            self._prefix = f"s{k + 1}|"
            sw["chains"] = [self._chain_fields(i, c) for i, c in enumerate(group)]
            self.swaps.append(sw)
        self._prefix = ""

    def field(self, name):
        name = self._prefix + name
        if name not in self._index:
            self._index[name] = len(self.fields)
            self.fields.append(name)
        return self._index[name]

    def _std_decay_name(self, tidx, key):
        t = self.topos[tidx]
        for d in t.chain:
            if t.decay_key(d) == key:
                return t.decay_name(d)
        raise KeyError(key)

    def _alignment_reference(self):
        """Reference topology of every final particle (rule 1 of
        ``tf_pwa/cal_angle.py:346-378``): the first topology in which it is a
        direct daughter of the top, else the first topology."""
        ref = {}
        top = self.group.top
        for k, t in enumerate(self.topos):
            for d in t.chain:
                if d.core == top:
                    for o in d.outs:
                        if o in self.group.outs and str(o) not in ref:
                            ref[str(o)] = k
        for o in self.group.outs:
            ref.setdefault(str(o), 0)
        return ref

    def _chain_fields(self, ci, chain):
        tidx = self.chain_topo[ci]
        t = ChainTopology(chain)
        out = {"topo": tidx, "decays": [], "aligned": {}, "mass": {}}
        for p in chain.inner:
            out["mass"][p] = self.field("m/" + t.node[p])
        for d in chain:
            std = self._std_decay_name(tidx, t.decay_key(d))
            b = t.node[d.outs[0]]
            out["decays"].append({
                "alpha": self.field(f"{tidx}/{std}/{b}/alpha"),
                "beta": self.field(f"{tidx}/{std}/{b}/beta"),
            })
        for d in chain:
            std = self._std_decay_name(tidx, t.decay_key(d))
            for o in d.outs:
                if o in chain.outs and o.J != 0 and self.align_ref[str(o)] != tidx:
                    base = f"{tidx}/{std}/{t.node[o]}/aligned"
                    out["aligned"][o] = tuple(
                        self.field(f"{base}/{a}") for a in ("alpha", "beta", "gamma"))
        return out

    @property
    def n_fields(self):
        return len(self.fields)


def split_swap(fname):
    """(swap number, base field name): 0 for the unswapped fields."""
    if fname.startswith("s") and "|" in fname:
        head, rest = fname.split("|", 1)
        return int(head[1:]), rest
    return 0, fname


def _transpose_order(outs, pairs):
    """Helicity-axis order of an exchange of the final pairs ``pairs``:
    out-axis j takes axis order[j] (``tf_pwa/amp/core.py:1853-1867``)."""
    tmap = {l: k for k, l in pairs}
    tmap.update(dict(pairs))
    new_order = [tmap.get(o, o) for o in outs]
    index_map = {k: i for i, k in enumerate(new_order)}
    return [index_map[o] for o in outs]


def cp_charge_group(finals, identical, cp):
    """Pairs of charge-conjugate final groups, self-conjugate finals paired
    with themselves (``tf_pwa/particle.py:992-1022``)."""
    used = set()
    ret = []
    for a, b in cp:
        ga = next((g for g in identical if a in g), None)
        gb = next((g for g in identical if b in g), None)
        if ga is None and gb is None:
            used.update((a, b))
            ret.append([[a], [b]])
        elif ga is None or gb is None or len(ga) != len(gb):
            raise ValueError("cp_particles pair identical groups of different sizes")
        else:
            used.update(ga)
            used.update(gb)
            ret.append([list(ga), list(gb)])
    for f in finals:
        if f not in used:
            ret.append([[f], [f]])
    return ret


def pass_specs(group, identical, cp):
    """The identical-particle swaps of the unswapped momenta, then (with
    CP-conjugate pairs) the CP-conjugate configuration and its swaps.  Each
    is a dict with ``src`` (final -> final whose momentum it takes), ``neg``
    (three-momenta reversed), ``factor``, ``trans`` (out-axis j = the
    pass's helicity axis trans[j]) and ``flip`` (every helicity reversed)."""
    ident = [[str(x) for x in g] for g in (identical or [])]
    outs = [str(o) for o in group.outs]
    passes = [dict(src=src, neg=False, factor=f, trans=t, flip=False)
              for src, f, t in swap_specs(group, ident)]
    if not cp:
        return passes
    cp = [[str(x) for x in pr] for pr in cp]
    cg = cp_charge_group(outs, ident, cp)
    byname = {str(o): o for o in group.outs}
    cp_src, frac, change = {}, 1.0, []
    for a, b in cg:
        for i, j in zip(a, b):
            cp_src[j] = i
            if i != j:
                cp_src[i] = j
                change.append((i, j))
            else:
                c = byname[i].C
                if c is None:
                    raise ValueError(f"self-conjugate final {i} needs its C parity")
                frac *= float(c)
    t_cp = _transpose_order(outs, change)
    passes.append(dict(src={o: cp_src.get(o, o) for o in outs}, neg=True, factor=frac,
                       trans=t_cp, flip=True))
    for src, f, t in swap_specs(group, ident):
        # swap of the CP-conjugate momenta, then the CP transposition
        passes.append(dict(src={o: cp_src.get(src.get(o, o), src.get(o, o)) for o in outs},
                           neg=True, factor=f * frac, trans=[t[k] for k in t_cp], flip=True))
    return passes


def swap_specs(group, identical):
    """Per non-identity permutation of the identical particles, in the
    reference's order (``itertools.product`` of each group's permutations,
    ``tf_pwa/cal_angle.py:684-716``):

    * ``src``: final name -> name of the final whose momentum it takes;
    * ``factor``: -1 per exchanged pair of half-integer-spin particles
      (``tf_pwa/amp/core.py:1826-1840``);
    * ``trans``: the helicity-axis order of the swapped amplitude,
      out-axis j = swapped-amplitude axis trans[j]
      (``tf_pwa/amp/core.py:1842-1867``)."""
    if not identical:
        return []
    groups = [[str(x) for x in g] for g in identical]
    outs = [str(o) for o in group.outs]
    spin = {str(o): o.J for o in group.outs}
    ident = tuple(tuple(g) for g in groups)
    out = []
    for comb in itertools.product(*[list(itertools.permutations(g)) for g in groups]):
        if comb == ident:
            continue
        src = {}
        for c, g in zip(comb, groups):
            for ci, pi in zip(c, g):
                src[pi] = ci
        factor = 1.0
        used = []
        for g, c in zip(groups, comb):
            if round(2 * spin[g[0]]) % 2 == 0:
                continue
            for m, n in zip(g, c):
                if (m, n) in used or (n, m) in used:
                    continue
                used.append((m, n))
                if m != n:
                    factor = -factor
        pairs = [(k, l) for g, c in zip(groups, comb) for k, l in zip(g, c)]
        out.append((src, factor, _transpose_order(outs, pairs)))
    return out

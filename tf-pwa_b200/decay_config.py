"""config.yml ``decay``/``particle`` sections -> DecayGroup + fit parameters.

Follows the reference's config semantics:

* decay list items and per-decay options: ``tf_pwa/config_loader/decay_config.py:130-155``
* particle map / properties / ``$top`` ``$finals`` ``$include``:
  ``tf_pwa/config_loader/decay_config.py:157-240``
* key renames (Par->P, m0->mass, g0->width, bw->model):
  ``tf_pwa/config_loader/decay_config.py:61-75``
* chain enumeration (``top.chain_decay()`` cross product in config order) and
  the LS cut: ``tf_pwa/config_loader/decay_config.py:289-420``,
  ``tf_pwa/particle.py:110-120``
* parameter creation order (resonance mass/width, then per chain its
  ``total`` and the ``g_ls`` of not-yet-seen decays with index 0 fixed to
  1+0i): ``tf_pwa/amp/core.py:1648-1662,1325-1329,764-773,367-377``
* constraints: fixed chain total (``config_loader.py:358-366``) and
  ``float: mg`` resonances (``config_loader.py:410-505``).
"""
import copy
import os
import random

import numpy as np
import yaml

from .particles import Decay, DecayChain, DecayGroup, Particle, var_name

_PARTICLE_KEYS = {
    "Par": "P",
    "m0": "mass",
    "g0": "width",
    "bw": "model",
}


def load_yaml(file_name, share_dict=None):
    share_dict = share_dict or {}
    if isinstance(file_name, dict):
        return copy.deepcopy(file_name)
    if file_name in share_dict:
        return load_yaml(share_dict[file_name])
    with open(file_name) as f:
        ret = yaml.safe_load(f)
    return ret or {}


def _list2decay(core, outs):
    parts, params = [], {}
    for j in outs:
        if isinstance(j, dict):
            params.update(j)
        else:
            parts.append(j)
    return {"core": core, "outs": parts, "params": params}


def decay_items(decay_dict):
    decs = []
    for core, outs in decay_dict.items():
        if all(isinstance(i, list) for i in outs):
            for i in outs:
                decs.append(_list2decay(core, i))
        else:
            decs.append(_list2decay(core, outs))
    return decs


def _particle_item_list(particle_list):
    pmap, props = {}, {}
    for name, cand in particle_list.items():
        if isinstance(cand, list):
            if len(cand) == 0:
                pmap[name] = []
            for i in cand:
                if isinstance(i, str):
                    pmap[name] = pmap.get(name, []) + [i]
                elif isinstance(i, dict):
                    m, p = _particle_item_list(i)
                    for k, v in m.items():
                        pmap[k] = pmap.get(k, []) + v
                    props.update(p)
                else:
                    raise ValueError(f"value of particle map {i} is {type(i)}")
        elif isinstance(cand, dict):
            props[name] = cand
        else:
            raise ValueError(f"value of particle {name} is {type(cand)}")
    return pmap, props


def particle_items(particle_list, base_dir=".", share_dict=None):
    particle_list = dict(particle_list)
    top = particle_list.pop("$top", None)
    finals = particle_list.pop("$finals", None)
    includes = particle_list.pop("$include", None)
    if includes:
        if isinstance(includes, str):
            includes = [includes]
        for inc in includes:
            path = inc if os.path.isabs(inc) else os.path.join(base_dir, inc)
            s = load_yaml(path, share_dict)
            for k in s:
                if k in particle_list and isinstance(particle_list[k], dict):
                    s[k].update(particle_list[k])
                    particle_list[k] = s[k]
                elif k not in particle_list:
                    particle_list[k] = s[k]
    pmap, props = _particle_item_list(particle_list)
    if isinstance(top, dict):
        props.update(top)
    if isinstance(finals, dict):
        props.update(finals)
    return pmap, props, top, finals


def _rename(params):
    return {_PARTICLE_KEYS.get(k, k): v for k, v in params.items()}


def _cross(lists):
    if not lists:
        return [[]]
    out = []
    for i in lists[0]:
        for j in _cross(lists[1:]):
            out.append(i + j)
    return out


def _chain_decay(p):
    """All decay chains starting at base particle p (``particle.py:110-120``)."""
    ret = []
    for d in p["decay"]:
        parts = [[[d]]]
        for o in d["outs"]:
            tmp = _chain_decay(o)
            if tmp:
                parts.append(tmp)
        # cross_combine of particle.py:20-40
        def cross_combine(x):
            if not x:
                return []
            head, tail = x[0], x[1:]
            other = cross_combine(tail)
            r = []
            for i in head:
                if not other:
                    r.append(i)
                else:
                    for j in other:
                        r.append(i + j)
            return r
        ret += cross_combine(parts)
    return ret


class DecayConfig:
    def __init__(self, dic, base_dir=".", share_dict=None):
        self.config = copy.deepcopy(dic)
        self.data_config = dic.get("data", {}) or {}
        self.decs = decay_items(self.config["decay"])
        (self.particle_map, self.particle_property, self.top_cfg,
         self.finals_cfg) = particle_items(self.config["particle"], base_dir, share_dict)
        self.decay_group = self._build()

    def _build(self):
        base = {}

        def base_particle(name):
            if name not in base:
                base[name] = {"name": name, "decay": []}
            return base[name]

        def wrap(name):
            return [base_particle(i) for i in self.particle_map.get(name, [name])]

        decs = []
        for dec in self.decs:
            cores = wrap(dec["core"])
            outs = [wrap(j) for j in dec["outs"]]
            for c in cores:
                for combo in _cross([[[o] for o in ol] for ol in outs]):
                    d = {"core": c, "outs": combo, "params": dec["params"]}
                    # a base decay is registered once per (core, sorted outs)
                    key = (c["name"], tuple(sorted(o["name"] for o in combo)))
                    if not any(k == key for k, _ in c.get("_keys", [])):
                        c.setdefault("_keys", []).append((key, d))
                        c["decay"].append(d)
                    decs.append(d)

        # top and finals
        top = self.top_cfg
        if top is None:
            cores = {d["core"]["name"] for d in decs}
            outs = {o["name"] for d in decs for o in d["outs"]}
            tops = cores - outs
            assert len(tops) == 1, "not only one top particle"
            top = tops.pop()
        elif isinstance(top, dict):
            top = list(top.keys())[0]
        elif isinstance(top, list):
            top = top[0]
        if self.finals_cfg is None:
            cores = {d["core"]["name"] for d in decs}
            finals = sorted({o["name"] for d in decs for o in d["outs"]} - cores)
        else:
            finals = list(self.finals_cfg)
        self.top_name = top
        self.final_names = finals

        particles = {}

        def particle(name, idx):
            key = f"{name}:{idx}"
            if key not in particles:
                props = _rename(self.particle_property.get(name, {}))
                props = dict(props)
                for a, lo, hi in (("mass", "m_min", "m_max"), ("width", "g_min", "g_max")):
                    if a not in props and lo in props and hi in props:
                        props[a] = random.random() * (props[hi] - props[lo]) + props[lo]
                props.pop("m_min", None), props.pop("m_max", None)
                props.pop("g_min", None), props.pop("g_max", None)
                particles[key] = Particle(name, id_=idx, **props)
            return particles[key]

        decays = {}
        chains = []
        for raw in _chain_decay(base[top]):
            outs_all = set()
            cores = set()
            for d in raw:
                cores.add(d["core"]["name"])
                outs_all.update(o["name"] for o in d["outs"])
            if sorted(outs_all - cores) != sorted(finals):
                continue
            cin, cout = {}, {}
            chain = []
            for d in raw:
                cn = d["core"]["name"]
                cin[cn] = cin.get(cn, -1) + 1
                core = particle(cn, cin[cn])
                outs = []
                for o in d["outs"]:
                    cout[o["name"]] = cout.get(o["name"], -1) + 1
                    outs.append(particle(o["name"], cout[o["name"]]))
                key = (core, tuple(outs))
                if key not in decays:
                    decays[key] = Decay(core, outs, **dict(d["params"]))
                chain.append(decays[key])
            # LS cut (decay_cut with the default ["ls_cut"])
            if all(len(dd.get_ls_list()) > 0 for dd in chain):
                chains.append(DecayChain(chain))
        if not chains:
            raise RuntimeError("no decay chain available, check the config")
        if self.data_config.get("cp_trans", True):
            # charge < 0 events are parity-transformed instead of flipping the
            # helicity couplings (tf_pwa/config_loader/decay_config.py:93-94,423-427)
            for c in chains:
                for d in c:
                    d.allow_cc = False
        # decay_chain options: "$all: {is_cp: true}" gives every chain a
        # CP-violating total, one value per event charge
        # (tf_pwa/amp/core.py:1306-1329,1380-1390, tf_pwa/variable.py:
        # 199-235,1715-1734); any other option is refused, not ignored
        for key, opts in (self.config.get("decay_chain") or {}).items():
            opts = dict(opts or {})
            is_cp = bool(opts.pop("is_cp", False))
            if key != "$all" or any(v for v in opts.values()):
                raise NotImplementedError(f"decay_chain options {opts} for {key}")
            for c in chains:
                c.is_cp = is_cp
        # kinematics options of the reference's preprocessor
        # (tf_pwa/config_loader/data.py:92-113): only the defaults are built
        dk = self.data_config
        for key, default in (("center_mass", False), ("r_boost", True), ("align_ref", None),
                             ("only_left_angle", False), ("preprocessor", "default")):
            if dk.get(key, default) != default:
                raise NotImplementedError(f"data option {key}: {dk.get(key)!r}")
        group = DecayGroup(chains)
        # data.identical_particles: lists of final particles whose momenta are
        # symmetrised; data.cp_particles: charge-conjugate final pairs of a
        # self-conjugate system (tf_pwa/config_loader/decay_config.py:100-107)
        ident = self.data_config.get("identical_particles")
        if ident:
            group.identical_particles = [[str(x) for x in g] for g in ident]
        cp = self.data_config.get("cp_particles")
        if cp:
            group.cp_particles = [[str(x) for x in pr] for pr in cp]
        # per-event charges (``<idx>_charge`` files, or use_charge: true):
        # tf_pwa/config_loader/data.py:73-76,92,163-167
        dk = self.data_config
        group.charge = bool(dk.get("use_charge")) or any(
            str(k).endswith("_charge") for k in dk)
        group.cp_trans = bool(dk.get("cp_trans", True))
        group.random_z = bool(dk.get("random_z", True))
        return group


def polarization_names(group):
    """Real parameters of the parent's polarisation: px, py, pz for spin
    1/2, eight components for spin 1 (``tf_pwa/amp/core.py:1660-1671``)."""
    top = group.top
    pol = getattr(top, "polarization", "none")
    if pol == "none":
        return []
    if pol != "vector":
        raise NotImplementedError(f"polarization {pol!r}")
    head = var_name(str(top))
    if top.J == 0.5:
        return [f"{head}_polarization_p{a}" for a in ("x", "y", "z")]
    if top.J == 1:
        return [f"{head}_polarization_p_{i}" for i in range(8)]
    raise NotImplementedError("vector polarisation of a parent with spin other than 1/2 or 1")


def init_params(group, vm, constrains=None):
    """Create the fit parameters of the group in the reference order."""
    constrains = constrains or {}
    names = {"mass": {}, "width": {}, "total": [], "g_ls": {}}
    for p in group.resonances:
        head = var_name(str(p))
        if p.model == "one":
            continue  # fixed lineshape: no parameters (ParticleOne.init_params)
        if p.mass is not None or True:
            vm.add_real_var(f"{head}_mass", value=p.mass if p.mass is not None else 0.0,
                            trainable=False)
            names["mass"][p] = f"{head}_mass"
        if p.width is not None:
            vm.add_real_var(f"{head}_width", value=p.width, trainable=False)
            names["width"][p] = f"{head}_width"
    seen = set()
    for c in group:
        tname = c.params_head + "_total_0"
        if getattr(c, "is_cp", False):
            vm.add_cartesiancp_var(tname)
        else:
            vm.add_complex_var(tname)
        names["total"].append(tname)
        for d in c:
            if d in seen:
                continue
            seen.add(d)
            lst = []
            for i in range(len(d.get_ls_list())):
                n = f"{d.params_head}_g_ls_{i}"
                vm.add_complex_var(n, polar=d.params_polar)
                lst.append(n)
            # first coupling fixed to 1+0i (core.py:767-773)
            vm.set_fix(lst[0] + "r", 1.0)
            vm.set_fix(lst[0] + "i", 0.0)
            names["g_ls"][d] = lst
    # polarisation vector of the parent (core.py:1660-1671)
    names["polarization"] = polarization_names(group)
    for n in names["polarization"]:
        vm.add_real_var(n)
    # decay constraints: fix one chain total (config_loader.py:358-366)
    dic = (constrains.get("decay") or {})
    fix_idx = dic.get("fix_chain_idx", 0)
    fix_val = dic.get("fix_chain_val", None)
    if fix_val is None:
        fix_val = float(np.random.uniform(0, 2))
    t = names["total"][fix_idx]
    vm.set_fix(t + "r", fix_val)
    vm.set_fix(t + "i", 0.0)
    if t + "deltar" in vm.variables:  # fixed CP-violating total: no asymmetry
        vm.set_fix(t + "deltar", 0.0)
        vm.set_fix(t + "deltai", 0.0)
    # particle constraints: float: mg (config_loader.py:410-505)
    return names


def float_particles(group, vm, names, particle_property):
    """Free the masses/widths marked ``float: m``/``g``; returns the fit
    bounds {variable: (lower, upper)} from ``mass_min``/``mass_max`` and
    ``width_min``/``width_max`` (None where not given), as
    ``tf_pwa/config_loader/config_loader.py:460-496`` collects them."""
    bounds = {}
    for c in group:
        for p in c.inner:
            cfg = particle_property.get(p.name, {})
            fl = cfg.get("float", "") or ""
            if "m" in fl and p in names["mass"]:
                n = names["mass"][p]
                if n not in vm.trainable_vars:
                    vm.set_fix(n, unfix=True)
                bounds[n] = (cfg.get("mass_min"), cfg.get("mass_max"))
            if "g" in fl and p in names["width"]:
                n = names["width"][p]
                if n not in vm.trainable_vars:
                    vm.set_fix(n, unfix=True)
                bounds[n] = (cfg.get("width_min"), cfg.get("width_max"))
    return {k: v for k, v in bounds.items() if v != (None, None)}

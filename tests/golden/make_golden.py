"""Generate golden vectors by running the REFERENCE package's own code.

Run in a container that has the reference checkout (it is not needed
anywhere else; the outputs are committed):

    python tests/golden/make_golden.py /path/to/reference

TensorFlow is not installed, so the reference runs on the torch-backed
TF-API stand-in in ``tests/golden/tfshim`` (GradientTape = torch autograd,
float64).  For each workload config this script

1. draws seeded flat phase-space momenta (the engine's own generator) for
   data, an optional background sample and MC, writes them as the
   reference's ``E px py pz`` text files;
2. builds ``tf_pwa.config_loader.ConfigLoader`` on that config, sets seeded
   parameters, and records: the reference's per-event input fields
   (invariant masses, helicity and alignment angles from ``cal_angle``),
   the per-event |A|^2 of data and MC (``AbsPDF.__call__``), and
   ``FCN.nll_grad`` (NLL and its GradientTape gradient) -- plus, for the
   small model, ``FCN.nll_grad_hessian``;
3. saves everything to ``tests/golden/<name>.npz`` and the parameter
   names/order, LS lists and CG matrices to ``tests/golden/<name>.json``.
"""
import json
import os
import shutil
import sys
import tempfile
import warnings

import numpy as np
import yaml

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

CASES = {
    # name: (config file, n_data, n_bg, n_mc, seed, hessian, extra data keys)
    "d2kpipi": ("d2kpipi.yml", 400, 0, 1500, 11, True, {}),
    "d2kpipi_float": ("d2kpipi_float.yml", 400, 0, 1500, 12, True, {}),
    "lc2pkpi": ("lc2pkpi.yml", 400, 40, 1500, 13, True, {"bg_weight": 0.1}),
    "toy_vvp": ("toy_vvp.yml", 300, 30, 1200, 14, True, {"bg_weight": 0.1}),
    "b2dstkpi": ("b2dstkpi.yml", 300, 0, 1200, 15, True, {}),
    "d2kpipi_shapes": ("d2kpipi_shapes.yml", 400, 0, 1500, 16, True, {}),
    "dp2kpipi_ident": ("dp2kpipi_ident.yml", 400, 0, 1500, 17, True, {}),
    "ident_fermions": ("ident_fermions.yml", 300, 0, 1200, 18, True, {}),
    "epem_cp": ("epem_cp.yml", 300, 0, 1200, 19, False, {}),
    "lc2pkpi_cc": ("lc2pkpi_cc.yml", 400, 0, 1500, 20, False, {}),
    "b2dstkpi_cc": ("b2dstkpi_cc.yml", 400, 0, 1500, 21, False, {}),
    "lc2pkpi_pol": ("lc2pkpi_pol.yml", 400, 0, 1500, 22, False, {}),
    "epem_pol": ("epem_pol.yml", 300, 0, 1200, 23, False, {}),
    "ident3_fermions": ("ident3_fermions.yml", 300, 0, 1200, 24, False, {}),
    "lc2pkpi_pol_lab": ("lc2pkpi_pol.yml", 400, 0, 1500, 25, False, {}),
    "lc2pkpi_cp": ("lc2pkpi_cp.yml", 400, 0, 1500, 26, False, {}),
}
# cases at the workloads' own sizes: the events are not stored (a test
# regenerates them from the seeds with the same generator); the reference's
# NLL and gradient are, with its fields and |A|^2 at SUBSET events per set
CASES.update({
    "d2kpipi_1e4": ("d2kpipi.yml", 10_000, 0, 100_000, 31, False, {}),
    "lc2pkpi_full": ("lc2pkpi.yml", 100_000, 10_000, 1_000_000, 32, False, {"bg_weight": 0.1}),
})
LARGE = {"d2kpipi_1e4", "lc2pkpi_full"}
SUBSET_F = 2048   # events per set whose fields are stored
SUBSET_A = 8192   # events per set whose |A|^2 is stored


# signal data of the large cases by accept-reject on the model's |A|^2, as
# the workload definition asks: candidates from the flat generator (seeded),
# kept where u * fmax < sum |A|^2 at the case's parameters; the kept indices
# are stored, so a test regenerates the same candidates and keeps the same
# events without evaluating the model
ACCEPT_REJECT = {"d2kpipi_1e4": 100_000, "lc2pkpi_full": 6_000_000}


def draw_params(names, rng, base):
    """Seeded parameter values: |g| ~ U(0.5, 2), phase ~ U(-pi, pi); CP
    deltas ~ U(-0.3, 0.3); polarisations ~ U(-0.4, 0.4); masses and widths
    at their nominal values times U(0.97, 1.03)."""
    params = {}
    for k in names:
        if k.endswith(("deltar", "deltai")):
            params[k] = float(rng.uniform(-0.3, 0.3))
        elif k.endswith("r") and ("_g_ls_" in k or "_total_" in k):
            params[k] = float(rng.uniform(0.5, 2.0))
        elif k.endswith("i") and ("_g_ls_" in k or "_total_" in k):
            params[k] = float(rng.uniform(-np.pi, np.pi))
        elif "_polarization_" in k:
            params[k] = float(rng.uniform(-0.4, 0.4))
        else:
            params[k] = float(base[k]) * float(rng.uniform(0.97, 1.03))
    return params


def accept_reject(dc, plan, order, M, masses, n_cand, n_keep, seed, vals):
    """Indices (into n_cand flat candidates of generate_phsp(seed)) of the
    first n_keep events kept by u * fmax < sum |A|^2 (oracle, FP64, at the
    parameter values ``vals``), fmax = 1.1 max over the candidates."""
    sys.path.insert(0, REPO)
    from oracle.pwa_oracle import OracleModel
    from tf_pwa_b200.kinematics import event_fields, p4_dict
    from tf_pwa_b200.phasespace import generate_phsp

    arr = np.stack(generate_phsp(M, masses, n_cand, seed=seed), 1)
    m = OracleModel(dc.decay_group, plan)
    f = np.empty(n_cand)
    for q in range(0, n_cand, 200_000):
        r = min(q + 200_000, n_cand)
        x = event_fields(plan, p4_dict(arr[q:r], order)).numpy()
        f[q:r] = m.pdf(x, vals)
    u = np.random.default_rng(seed + 99).uniform(size=n_cand)
    idx = np.nonzero(u * 1.1 * f.max() < f)[0]
    assert len(idx) >= n_keep, (len(idx), n_keep)
    return idx[:n_keep].astype(np.int64), arr


def subset_index(n, k, seed):
    """Sorted distinct event indices of one set (seeded)."""
    k = min(k, n)
    return np.sort(np.random.default_rng(seed).choice(n, size=k, replace=False))


# cases whose events are boosted out of the parent rest frame: parent
# momentum (GeV) in a random direction per event (lab-frame input)
BOOSTED = {"lc2pkpi_pol_lab": 2.0}


def boost_events(arr, M, pmag, rng):
    """(n, n_final, 4) rest-frame momenta boosted so that the parent has
    momentum ``pmag`` along a random direction per event."""
    n = arr.shape[0]
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    beta = u * (pmag / np.hypot(M, pmag))
    b2 = np.sum(beta ** 2, 1)
    g = 1.0 / np.sqrt(1.0 - b2)
    out = np.empty_like(arr)
    for f in range(arr.shape[1]):
        E, p = arr[:, f, 0], arr[:, f, 1:]
        bp = np.sum(beta * p, 1)
        out[:, f, 0] = g * (E + bp)
        out[:, f, 1:] = p + ((g - 1.0) * bp / b2 + g * E)[:, None] * beta
    return out


def load_pkg():
    import importlib.util

    d = os.path.join(REPO, "tf-pwa_b200")
    spec = importlib.util.spec_from_file_location(
        "tf_pwa_b200", os.path.join(d, "__init__.py"), submodule_search_locations=[d])
    m = importlib.util.module_from_spec(spec)
    sys.modules["tf_pwa_b200"] = m
    spec.loader.exec_module(m)


def main(ref_root):
    sys.path[:0] = [os.path.join(HERE, "tfshim"), ref_root]
    warnings.filterwarnings("ignore")
    load_pkg()
    from tf_pwa_b200.decay_config import DecayConfig, float_particles, init_params, load_yaml
    from tf_pwa_b200.phasespace import generate_phsp
    from tf_pwa_b200.plan import Plan, split_swap
    from tf_pwa_b200.variables import VarsManager
    from tf_pwa.config_loader import ConfigLoader

    cfg_dir = os.path.join(REPO, "tf-pwa_b200", "configs")
    only = sys.argv[2:] or [c for c in CASES if c not in LARGE]
    for name in only:
        cfg_file, nd, nb, nm, seed, do_hess, extra = CASES[name]
        rng = np.random.default_rng(seed)
        dic = load_yaml(os.path.join(cfg_dir, cfg_file))
        dc = DecayConfig(dic)
        group = dc.decay_group
        plan = Plan(group, dic["data"].get("dat_order"))
        order = dic["data"].get("dat_order")
        top = group.top
        masses = [dc.particle_property[o]["mass"] for o in order]
        M = dc.particle_property[str(top)]["mass"]
        tmp = tempfile.mkdtemp()
        p4 = {}
        pre_params, kept = None, None
        if name in ACCEPT_REJECT:
            vm0 = VarsManager(rng=np.random.default_rng(0))
            nm0 = init_params(group, vm0, dic.get("constrains"))
            float_particles(group, vm0, nm0, dc.particle_property)
            pre_params = draw_params(vm0.trainable_vars, rng, vm0.get_all_dic())
        for kk, (kind, n) in enumerate((("data", nd), ("bg", nb), ("phsp", nm))):
            if n == 0:
                continue
            if kind == "data" and name in ACCEPT_REJECT:
                vals0 = vm0.get_all_dic()
                vals0.update(pre_params)
                kept, cand = accept_reject(dc, plan, order, M, masses, ACCEPT_REJECT[name], n,
                                           1000 * seed + kk, vals0)
                arr = cand[kept]
            else:
                ps = generate_phsp(M, masses, n, seed=1000 * seed + kk)
                arr = np.stack(ps, 1)  # (n, n_final, 4)
            if name in BOOSTED:
                arr = boost_events(arr, M, BOOSTED[name], rng)
            p4[kind] = arr
            np.savetxt(os.path.join(tmp, kind + ".dat"), arr.reshape(-1, 4), fmt="%.17g")
            print(name, kind, n, "events written", flush=True)
        dic2 = dict(dic)
        dic2["data"] = dict(dic.get("data", {}))
        dic2["data"].update({"data": [os.path.join(tmp, "data.dat")],
                             "phsp": [os.path.join(tmp, "phsp.dat")]})
        if nb:
            dic2["data"]["bg"] = [os.path.join(tmp, "bg.dat")]
        dic2["data"].update(extra)
        charges = {}
        if plan.use_charge:
            # per-event charge_conjugation files (random +1 / -1)
            for kind, arr in p4.items():
                charges[kind] = rng.choice([-1.0, 1.0], size=arr.shape[0])
                fc = os.path.join(tmp, kind + "_charge.dat")
                np.savetxt(fc, charges[kind], fmt="%.1f")
                dic2["data"][kind + "_charge"] = [fc]
        cfg_path = os.path.join(tmp, "config.yml")
        with open(cfg_path, "w") as f:
            yaml.safe_dump(dic2, f)
        ref = ConfigLoader(cfg_path)
        amp = ref.get_amplitude()
        vm = amp.vm
        # seeded parameter values: |g| ~ U(0.5, 2), phase ~ U(-pi, pi);
        # masses/widths at their nominal values shifted by a few percent
        params = {}
        if pre_params is not None:
            assert list(pre_params) == list(vm.trainable_vars)
            params = dict(pre_params)
        for k in ([] if pre_params is not None else vm.trainable_vars):
            if k.endswith(("deltar", "deltai")):
                params[k] = float(rng.uniform(-0.3, 0.3))
            elif k.endswith("r") and ("_g_ls_" in k or "_total_" in k):
                params[k] = float(rng.uniform(0.5, 2.0))
            elif k.endswith("i") and ("_g_ls_" in k or "_total_" in k):
                params[k] = float(rng.uniform(-np.pi, np.pi))
            elif "_polarization_" in k:
                params[k] = float(rng.uniform(-0.4, 0.4))
            else:
                params[k] = float(vm.get(k)) * float(rng.uniform(0.97, 1.03))
        vm.set_all(params)
        all_vals = {k: float(vm.get(k)) for k in vm.variables}
        datas = {k: ref.get_data(k) for k in ("data", "phsp", "bg") if (k != "bg" or nb)}
        fields = {}
        for kind, lst in datas.items():
            d = lst[0]
            cols = np.zeros((plan.n_fields, len(d["weight"])))
            # identical-particle swaps: the reference's id_swap data sets, in
            # its permutation order, then the CP-conjugate ones
            swap_sets = [d] + list(d.get("id_swap", {}).values())
            if "cp_swap" in d:  # the CP-conjugate data and its own swaps
                swap_sets += [d["cp_swap"]] + list(d["cp_swap"].get("id_swap", {}).values())
            for fi, full_name in enumerate(plan.fields):
                if fi == plan.charge_index:
                    cols[fi] = np.asarray(d["charge_conjugation"])
                    continue
                sk, fname = split_swap(full_name)
                ds = swap_sets[sk]
                topo_keys = list(ds["decay"].keys())
                parts = fname.split("/")
                if parts[0] == "m":
                    node = [k for k in ds["particle"] if str(k) == parts[1]][0]
                    cols[fi] = np.asarray(ds["particle"][node]["m"])
                    continue
                tidx = int(parts[0])
                my_topo = plan.topos[tidx]
                tstr = "[" + ", ".join(my_topo.decay_name(dd) for dd in my_topo.chain) + "]"
                tkey = [k for k in topo_keys if str(k) == tstr]
                assert tkey, (tstr, [str(k) for k in topo_keys])
                dd = ds["decay"][tkey[0]]
                dkey = [k for k in dd if str(k) == parts[1]][0]
                pkey = [k for k in dd[dkey] if str(k) == parts[2]][0]
                if parts[3] == "aligned":
                    cols[fi] = np.asarray(dd[dkey][pkey]["aligned_angle"][parts[4]])
                else:
                    cols[fi] = np.asarray(dd[dkey][pkey]["ang"][parts[3]])
            fields[kind] = cols
            # helicity gamma must be zero (not stored as a field)
            for tkey in topo_keys:
                for dkey, dv in d["decay"][tkey].items():
                    for pkey, pv in dv.items():
                        if isinstance(pv, dict) and "ang" in pv:
                            assert np.all(np.asarray(pv["ang"]["gamma"]) == 0)
        if name in LARGE:
            # |A|^2 in batches (the reference's own batching of FCN)
            f_vals = {}
            for k in datas:
                from tf_pwa.data import data_split

                f_vals[k] = np.concatenate([np.asarray(amp(b))
                                            for b in data_split(datas[k][0], 65000)])
        else:
            f_vals = {k: np.asarray(amp(datas[k][0])) for k in datas}
        fcn = ref.get_fcn()
        nll, grad = fcn.nll_grad()
        if name in LARGE:
            out = dict(nll=np.float64(nll), grad=np.asarray(grad, np.float64),
                       sum_w=np.float64(np.sum(np.asarray(fcn.weight, np.float64))))
            if kept is not None:
                out["data_kept"] = kept
            for k, tag in (("data", "data"), ("phsp", "mc"), ("bg", "bg")):
                if k not in fields:
                    continue
                n_k = fields[k].shape[1]
                i_f = subset_index(n_k, SUBSET_F, 7 * seed + len(tag))
                i_a = subset_index(n_k, SUBSET_A, 11 * seed + len(tag))
                out.update({f"idx_fields_{tag}": i_f, f"fields_{tag}": fields[k][:, i_f],
                            f"idx_f_{tag}": i_a, f"f_{tag}": f_vals[k][i_a],
                            f"n_{tag}": np.int64(n_k),
                            f"sum_f_{tag}": np.float64(np.sum(f_vals[k]))})
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
            meta = {
                "config": cfg_file,
                "extra_data": extra,
                "trainable": list(vm.trainable_vars),
                "variables": all_vals,
                "fields": plan.fields,
                "seed": seed,
                "events": {"generator": "tf_pwa_b200.phasespace.generate_phsp",
                           "seeds": {"data": 1000 * seed, "bg": 1000 * seed + 1,
                                     "mc": 1000 * seed + 2},
                           "sizes": {"data": nd, "bg": nb, "mc": nm},
                           "data_candidates": ACCEPT_REJECT.get(name)},
            }
            with open(os.path.join(HERE, name + ".json"), "w") as f:
                json.dump(meta, f, indent=1)
            shutil.rmtree(tmp)
            print(name, "nll", float(nll), "n_trainable", len(vm.trainable_vars))
            continue
        out = dict(
            fields_data=fields["data"], fields_mc=fields["phsp"],
            f_data=f_vals["data"], f_mc=f_vals["phsp"],
            p4_data=p4["data"], p4_mc=p4["phsp"],
            nll=np.float64(nll), grad=np.asarray(grad, np.float64),
            weight_data=np.asarray(fcn.weight, np.float64),
        )
        if nb:
            out.update(fields_bg=fields["bg"], f_bg=f_vals["bg"], p4_bg=p4["bg"])
        if charges:
            out.update(charge_data=charges["data"], charge_mc=charges["phsp"])
        if do_hess:
            n2, g2, h2 = fcn.nll_grad_hessian()
            out.update(hess=np.asarray(h2, np.float64), hess_grad=np.asarray(g2, np.float64),
                       hess_nll=np.float64(n2))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        meta = {
            "config": cfg_file,
            "extra_data": extra,
            "trainable": list(vm.trainable_vars),
            "variables": all_vals,
            "fields": plan.fields,
            "chains": [str(c) for c in amp.decay_group],
            "ls": [[list(map(list, dd.get_ls_list())) for dd in c] for c in amp.decay_group],
            "cg": [[np.asarray(dd.get_cg_matrix()).tolist() for dd in c] for c in amp.decay_group],
            "seed": seed,
        }
        with open(os.path.join(HERE, name + ".json"), "w") as f:
            json.dump(meta, f, indent=1)
        shutil.rmtree(tmp)
        print(name, "nll", float(nll), "n_trainable", len(vm.trainable_vars))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")

"""Shared helpers of the tests: load a workload config, its golden vectors,
and build oracle / engine objects for it."""
import json
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
CONFIGS = os.path.join(ROOT, "tf-pwa_b200", "configs")


def load_model(config_file):
    from tf_pwa_b200.decay_config import DecayConfig, float_particles, init_params, load_yaml
    from tf_pwa_b200.plan import Plan
    from tf_pwa_b200.variables import VarsManager

    dic = load_yaml(os.path.join(CONFIGS, config_file))
    dc = DecayConfig(dic)
    vm = VarsManager(rng=np.random.default_rng(0))
    names = init_params(dc.decay_group, vm, dic.get("constrains"))
    float_particles(dc.decay_group, vm, names, dc.particle_property)
    return dc, vm, Plan(dc.decay_group, dic.get("data", {}).get("dat_order"))


def load_golden(name):
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        meta = json.load(f)
    return g, meta


def golden_data(g, meta):
    """Data columns (data + background) and their alpha-scaled weights."""
    from oracle.pwa_oracle import weights

    if "fields_bg" in g:
        x = np.concatenate([g["fields_data"], g["fields_bg"]], 1)
        w = weights(np.ones(g["fields_data"].shape[1]),
                    -meta["extra_data"]["bg_weight"] * np.ones(g["fields_bg"].shape[1]))
    else:
        x = g["fields_data"]
        w = weights(np.ones(x.shape[1]))
    return x, w

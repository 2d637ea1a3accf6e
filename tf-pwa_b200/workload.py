"""Seeded synthetic datasets for the shipped workload configs.

Follows the toy procedure of the reference (``tf_pwa/applications.py:394-510``,
``gen_data``/``gen_mc``): flat phase-space MC, signal by accept-reject on
sum |A|^2 against max * U(0, 1), optional flat background rows with weight
``-bg_weight``.  Momenta, kinematics and the accept-reject run on the GPU
(the amplitude through the engine), so million-event samples take seconds.
Couplings are drawn with |g| ~ U(0.5, 2) and phase ~ U(-pi, pi).
"""
import os

import numpy as np
import torch

from .api import ConfigLoader, EventData
from .engine import PLAIN_F64, Engine
from .kinematics import event_fields
from .phasespace import generate_phsp

CONFIG_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "configs")


def config_path(name):
    return name if os.path.exists(name) else os.path.join(CONFIG_DIR, name)


def seeded_params(vm, seed):
    rng = np.random.default_rng(seed)
    vals = {}
    for k in vm.trainable_vars:
        if k.endswith("r") and ("_g_ls_" in k or "_total_" in k):
            vals[k] = float(rng.uniform(0.5, 2.0))
        elif k.endswith("i") and ("_g_ls_" in k or "_total_" in k):
            vals[k] = float(rng.uniform(-np.pi, np.pi))
    vm.set_all(vals)
    return vm.get_all_dic()


def _phsp_fields(cl, n, gen, device):
    pp = cl.decay_config.particle_property
    order = cl.get_dat_order()
    M = pp[str(cl.decay_group.top)]["mass"]
    ps = generate_phsp(M, [pp[o]["mass"] for o in order], n, gen=gen, device=device,
                       as_numpy=False)
    return event_fields(cl.plan, dict(zip(order, ps)), device=device)


def upload_fields(eng, x, w, n_data, n_mc, sw):
    """Upload device columns x (n_fields, N) and weights w (N) to an engine."""
    c = eng.code
    xm = x[c.mass_fields].contiguous() if c.mass_fields else x[:1].contiguous()
    xa = x[c.angle_fields].contiguous() if c.angle_fields else x[:1].contiguous()
    w = w.contiguous()
    eng.upload_device(xm.data_ptr(), xa.data_ptr(), w.data_ptr(), n_data, n_mc, sw)
    torch.cuda.synchronize()
    return xm, xa, w


def accept_reject(cl, n, gen, device, chunk=1 << 22, fmax=None):
    """n signal events distributed as sum |A|^2 (FP64 amplitude)."""
    eng = Engine(cl.decay_group, cl.plan, cl.vm)
    C = eng.consts(cl.vm.get_all_dic())
    kept = []
    have = 0
    while have < n:
        x = _phsp_fields(cl, chunk, gen, device)
        w = torch.ones(chunk, dtype=torch.float64, device=device)
        keep_alive = upload_fields(eng, x, w, chunk, 0, float(chunk))
        f = torch.empty(chunk, dtype=torch.float64, device=device)
        eng.pdf_device(C, 0, chunk, f.data_ptr(), PLAIN_F64)
        if fmax is None:
            fmax = 1.2 * float(f.max())
        u = torch.rand(chunk, generator=gen, dtype=torch.float64, device=device) * fmax
        sel = f > u
        kept.append(x[:, sel])
        have += int(sel.sum())
        del keep_alive
    eng.close()
    return torch.cat(kept, 1)[:, :n], fmax


def make_dataset(config, n_sig, n_mc, n_bg=0, bg_weight=0.1, seed=1, device="cuda",
                 precision="plain"):
    """ConfigLoader with seeded parameters, and EventData for signal,
    background and MC, resident on ``device``."""
    cl = ConfigLoader(config_path(config), precision=precision, seed=seed)
    seeded_params(cl.vm, seed)
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    sig, _ = accept_reject(cl, n_sig, gen, device)
    mc = _phsp_fields(cl, n_mc, gen, device)
    data = EventData(sig, np.ones(n_sig))
    bg = None
    if n_bg:
        bg = EventData(_phsp_fields(cl, n_bg, gen, device), -bg_weight * np.ones(n_bg))
    return cl, data, bg, EventData(mc, np.ones(n_mc))

"""Seeded synthetic datasets for the shipped workload configs.

Follows the toy procedure of the reference (``tf_pwa/applications.py:394-510``,
``gen_data``/``gen_mc``): flat phase-space MC, signal by accept-reject on
sum |A|^2 against max * U(0, 1), optional flat background rows with weight
``-bg_weight``.  Phase-space generation, kinematics and the accept-reject
run in the engine's toy kernels (one candidate per thread, counter-based
random numbers), so samples of 1e6 events take seconds even at accept
rates of 1e-4.  Couplings are drawn with |g| ~ U(0.5, 2) and phase ~
U(-pi, pi).
"""
import os

import numpy as np
import torch

from .api import ConfigLoader, EventData
from .engine import Engine

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


def _seed(seed, stream):
    """64-bit generator key of one sample (signal, background, MC) of a dataset."""
    return (int(seed) * 0x9E3779B97F4A7C15 + 0x632BE59BD9B4E019 * (stream + 1)) & (2**64 - 1)


def generate(eng, n, seed, consts=None, fmax=None, chunk=None, with_p4=False):
    """n events on the device, generated in one pass per candidate chunk by
    the engine's toy kernels: flat phase space (``consts`` None) or signal
    by accept-reject on sum |A|^2 (the procedure of
    ``tf_pwa/applications.py:394-487``: a first chunk at the phase-space
    step alone gives fmax = 1.2 max sum |A|^2; a later candidate above fmax
    raises fmax and restarts).  Returns (fields (n_fields, n), fmax), plus
    the momenta (n, n_final, 4) with ``with_p4``."""
    dev = eng.device
    chunk = chunk or eng.toy_chunk
    if n <= 0:
        x = torch.zeros((eng.plan.n_fields, 0), dtype=torch.float64, device=dev)
        p4 = torch.zeros((0, eng.code.kin.nfin, 4), dtype=torch.float64, device=dev)
        return (x, fmax, p4) if with_p4 else (x, fmax)
    flat = consts is None
    f = torch.empty(chunk, dtype=torch.float64, device=dev)
    if not flat and fmax is None:
        eng.toy_select(consts, seed, 0, chunk, 0.0, 0, f)
        fmax = 1.2 * float(f.max())
    while True:
        sel, have, first = [], 0, 0
        restart = False
        while have < n:
            eng.toy_select(consts, seed, first, chunk, fmax if not flat else 0.0, int(flat), f)
            if not flat:
                top = float(f.max())
                if top > fmax:
                    fmax, restart = 1.2 * top, True
                    break
            idx = torch.nonzero(f >= 0).squeeze(1) + first
            sel.append(idx)
            have += idx.numel()
            first += chunk
        if not restart:
            break
    idx = torch.cat(sel)[:n]
    if with_p4:
        x, p4 = eng.toy_fields(seed, idx, with_p4=True)
        return x, fmax, p4
    return eng.toy_fields(seed, idx), fmax


def make_dataset(config, n_sig, n_mc, n_bg=0, bg_weight=0.1, seed=1, device="cuda",
                 precision="plain"):
    """ConfigLoader with seeded parameters, and EventData for signal,
    background and MC, resident on ``device`` (CUDA: the engine's toy
    kernels generate them)."""
    cl = ConfigLoader(config_path(config), precision=precision, seed=seed)
    seeded_params(cl.vm, seed)
    eng = Engine(cl.decay_group, cl.plan, cl.vm)
    C = eng.consts(cl.vm.get_all_dic())
    sig, _ = generate(eng, n_sig, _seed(seed, 0), consts=C)
    mc, _ = generate(eng, n_mc, _seed(seed, 2))
    data = EventData(sig, np.ones(n_sig))
    bg = None
    if n_bg:
        bg = EventData(generate(eng, n_bg, _seed(seed, 1))[0], -bg_weight * np.ones(n_bg))
    eng.close()
    return cl, data, bg, EventData(mc, np.ones(n_mc))

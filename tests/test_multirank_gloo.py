"""Multi-rank combination of the NLL pieces (world size 2, gloo on CPU).

Each rank holds half of the data and half of the MC events, computes its
piece vector [S_data, S_mc * f, sum w, g_data, g_mc * f] (f = the rank's
share of the MC weight), the ranks sum the vectors with one all-reduce, and
``combine_pieces`` turns the sum into the NLL and gradient.  The pieces here
come from the FP64 oracle (first test) or from the engine's own
``local_pieces`` with its MC share and all-reduce hook, the sums taken from
the generated kernel code run on the host (CP-violating and polarised
models); the result must equal the single-process NLL and gradient of all
events (the reference's golden values)."""
import os

import numpy as np
import pytest


def _pieces(rank, world, q):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    import conftest  # noqa: F401
    import torch
    import torch.distributed as dist

    from common import golden_data, load_golden, load_model
    from oracle.pwa_oracle import OracleModel, clip_log
    from tf_pwa_b200.engine import combine_pieces

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    dist.init_process_group("gloo", rank=rank, world_size=world)
    g, meta = load_golden("lc2pkpi")
    dc, vm, plan = load_model(meta["config"])
    m = OracleModel(dc.decay_group, plan)
    vals = meta["variables"]
    names = meta["trainable"]
    xd, wd = golden_data(g, meta)
    xm = g["fields_mc"]
    wm_all = np.ones(xm.shape[1]) / xm.shape[1]
    sd_idx = np.array_split(np.arange(xd.shape[1]), world)[rank]
    sm_idx = np.array_split(np.arange(xm.shape[1]), world)[rank]
    share = wm_all[sm_idx].sum()

    def sums(x, w, data):
        A = m.amp(x, vals).reshape(x.shape[1], -1)
        f = np.sum(np.abs(A) ** 2, 1)
        if data:
            s0 = np.sum(w * clip_log(f))
            fac = w * np.where(f > 1e-6, 1.0 / np.maximum(f, 1e-300), 0.0)
        else:
            s0 = np.sum(w * f)
            fac = w
        gr = []
        for n in names:
            base = n[:-1]
            c = m.complex_of(vals, {}, base)
            dz = np.exp(1j * vals[base + "i"]) if n.endswith("r") else 1j * c
            v1, v2 = dict(vals), dict(vals)
            v1[base + "r"], v1[base + "i"] = 1.0, 0.0
            v2[base + "r"], v2[base + "i"] = 0.0, 0.0
            B = (m.amp(x, v1) - m.amp(x, v2)).reshape(A.shape)
            gr.append(np.sum(fac * 2 * np.real(np.sum(np.conj(A) * B * dz, 1))))
        return s0, np.array(gr)

    s_d, g_d = sums(xd[:, sd_idx], wd[sd_idx], True)
    # MC weights normalised over ALL ranks: the local share enters as f
    wm_local = wm_all[sm_idx] / share
    s_m, g_m = sums(xm[:, sm_idx], wm_local, False)
    vec = np.concatenate([[s_d, s_m * share, wd[sd_idx].sum()], g_d, g_m * share])
    t = torch.as_tensor(vec)
    dist.all_reduce(t)
    nll, grad = combine_pieces(t.numpy(), len(names))
    dist.destroy_process_group()
    q.put((rank, nll, grad, float(g["nll"]), np.asarray(g["grad"])))


def test_two_rank_gloo_combination():
    import torch.multiprocessing as mp

    os.environ.setdefault("MASTER_PORT", str(29500 + os.getpid() % 1000))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_pieces, args=(r, 2, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, nll, grad, ref_nll, ref_grad in res:
        assert abs(nll - ref_nll) <= 1e-10 * abs(ref_nll)
        np.testing.assert_allclose(grad, ref_grad, rtol=1e-8, atol=1e-8 * np.abs(ref_grad).max())


def _engine_pieces(rank, world, q, name, build_dir):
    """Engine.local_pieces on this rank's half of the events (device sums
    from the generated kernel code run on the host), summed over the ranks
    by the engine's own dist_reduce hook."""
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    import conftest  # noqa: F401
    import torch
    import torch.distributed as dist

    from common import golden_data, load_golden, load_model
    from hostexec import HostModel
    from tf_pwa_b200.engine import PLAIN_F64, Engine

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    dist.init_process_group("gloo", rank=rank, world_size=world)
    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    eng = Engine(dc.decay_group, plan, vm, compile=False)
    hm = HostModel(eng.code, build_dir)
    xd, wd = golden_data(g, meta)
    xm = g["fields_mc"]
    wm_all = np.ones(xm.shape[1]) / xm.shape[1]
    sd_idx = np.array_split(np.arange(xd.shape[1]), world)[rank]
    sm_idx = np.array_split(np.arange(xm.shape[1]), world)[rank]
    share = wm_all[sm_idx].sum()
    x = np.concatenate([xd[:, sd_idx], xm[:, sm_idx]], 1)
    w = np.concatenate([wd[sd_idx], wm_all[sm_idx] / share])
    nd = len(sd_idx)
    eng.eval_sums = lambda C, precision=PLAIN_F64, mc=True, stream=None: hm.sums(C, x, w, nd)
    eng._sw = float(wd[sd_idx].sum())
    eng.mc_share = share

    def reduce(vec):
        t = torch.as_tensor(vec)
        dist.all_reduce(t)
        return t.numpy()

    eng.dist_reduce = reduce
    nll, grad = eng.nll_grad(meta["variables"], meta["trainable"], PLAIN_F64)
    dist.destroy_process_group()
    q.put((rank, nll, grad, float(g["nll"]), np.asarray(g["grad"])))


@pytest.mark.parametrize("name", ["lc2pkpi_cp", "lc2pkpi_pol"])
def test_two_rank_engine_pieces(name, tmp_path):
    """The engine's multi-rank path (local pieces, MC share, all-reduce,
    combine) with the charge -1 and polarisation sums of the later model
    options: equal to the reference's single-process NLL and gradient."""
    import torch.multiprocessing as mp

    from common import load_golden, load_model
    from hostexec import HostModel
    from tf_pwa_b200.engine import Engine

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    HostModel(Engine(dc.decay_group, plan, vm, compile=False).code, str(tmp_path))  # build once
    os.environ["MASTER_PORT"] = str(29600 + os.getpid() % 1000 + (name == "lc2pkpi_pol"))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_engine_pieces, args=(r, 2, q, name, str(tmp_path)))
             for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, nll, grad, ref_nll, ref_grad in res:
        assert abs(nll - ref_nll) <= 1e-9 * abs(ref_nll)
        np.testing.assert_allclose(grad, ref_grad, rtol=1e-7, atol=1e-7 * np.abs(ref_grad).max())


def _native_pieces(rank, world, q, name, build_dir):
    """The native host program's piece vector (pwa_hostprog_pieces: its own
    constant block, Jacobian and chain rule) on this rank's half of the
    events, summed over the ranks with gloo and combined."""
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    import conftest  # noqa: F401
    import torch
    import torch.distributed as dist

    from common import golden_data, load_golden, load_model
    from hostexec import HostModel
    from tf_pwa_b200.engine import Engine, combine_pieces

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    dist.init_process_group("gloo", rank=rank, world_size=world)
    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])
    eng = Engine(dc.decay_group, plan, vm, compile=False)
    hm = HostModel(eng.code, build_dir)
    names = list(vm.variables)
    hp = eng.host_program(names, meta["trainable"])
    v = np.array([vm.variables[k] for k in names])
    xd, wd = golden_data(g, meta)
    xm = g["fields_mc"]
    wm_all = np.ones(xm.shape[1]) / xm.shape[1]
    sd_idx = np.array_split(np.arange(xd.shape[1]), world)[rank]
    sm_idx = np.array_split(np.arange(xm.shape[1]), world)[rank]
    share = wm_all[sm_idx].sum()
    x = np.concatenate([xd[:, sd_idx], xm[:, sm_idx]], 1)
    w = np.concatenate([wd[sd_idx], wm_all[sm_idx] / share])
    sd, sm = hm.sums(hp.consts(v), x, w, len(sd_idx))
    vec = torch.as_tensor(hp.pieces(v, sd, sm, float(wd[sd_idx].sum()), share))
    dist.all_reduce(vec)
    nll, grad = combine_pieces(vec.numpy(), len(meta["trainable"]))
    dist.destroy_process_group()
    q.put((rank, nll, grad, float(g["nll"]), np.asarray(g["grad"])))


@pytest.mark.parametrize("name", ["d2kpipi_float", "lc2pkpi", "lc2pkpi_cp", "lc2pkpi_pol"])
def test_two_rank_native_host_pieces(name, tmp_path):
    """Two gloo ranks, each with half of the data and MC events, through the
    native host program: the reference's single-process NLL and gradient."""
    import torch.multiprocessing as mp

    from common import load_golden, load_model
    from hostexec import HostModel
    from tf_pwa_b200.engine import Engine

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    HostModel(Engine(dc.decay_group, plan, vm, compile=False).code, str(tmp_path))  # build once
    os.environ["MASTER_PORT"] = str(29700 + os.getpid() % 1000 +
                                    ["d2kpipi_float", "lc2pkpi", "lc2pkpi_cp", "lc2pkpi_pol"].index(name))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_native_pieces, args=(r, 2, q, name, str(tmp_path)))
             for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, nll, grad, ref_nll, ref_grad in res:
        assert abs(nll - ref_nll) <= 1e-9 * abs(ref_nll)
        np.testing.assert_allclose(grad, ref_grad, rtol=1e-7, atol=1e-7 * np.abs(ref_grad).max())

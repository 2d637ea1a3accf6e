"""Benchmark: NLL + gradient evaluations per second of the Lambda_c+ -> p K- pi+
three-chain helicity model at 1e6 signal (+1e5 background rows, weight -0.1)
data events and 1e6 MC events on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  ``value`` is device-timed evaluations/s of the
headline (mixed) form: FP32 amplitudes, FP64 log-sum and reductions, MC
integral from the FP64 Gram matrix (masses/widths fixed); inputs resident in
HBM, L2 flushed before every timed step.  ``plain_f64`` is the same metric
for the all-FP64 kernels, through the same native host side (constants,
chain rule in the library).  ``e2e`` times the public call ``FCN.nll_grad(x)``
with host parameters in and host NLL/gradient out.  ``roofline`` covers the
dominant kernel (the fused data-term kernel), timed with CUDA events on the
stream it is launched on.  ``cpu_baseline`` times the FP64 CPU oracle on a
bounded sample of the same workload with all host cores.

Multi-GPU (torchrun, one process per GPU): every rank holds its own full
workload shard (weak scaling); the per-evaluation FP64 sums are combined
with one NCCL all-reduce before the host forms NLL and gradient.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
BG_WEIGHT = 0.1
# name: (config, signal events, background rows, MC events, metric, description)
WORKLOADS = {
    "lc2pkpi": ("lc2pkpi.yml", 1_000_000, 100_000, 1_000_000,
                "NLL+grad evals/s @1M data+1M MC",
                "Lambda_c+ -> p K- pi+ (Lambda(1520), K*(892), Delta(1232); 3 chains, 8 LS "
                "columns, 4 helicity combinations), 1e6 accept-reject signal + 1e5 flat "
                "background (w=-0.1) data rows, 1e6 flat MC"),
    "d2kpipi_float": ("d2kpipi_float.yml", 1_000_000, 0, 1_000_000,
                      "NLL+grad evals/s @1M data+1M MC, masses and widths floating",
                      "D0 -> K pi pi (K*(892) 1-, f0(980) 0+; 2 chains), both resonance masses "
                      "and widths floating (no column cache), 1e6 accept-reject data, 1e6 flat "
                      "MC"),
    "lc2pkpi_float": ("lc2pkpi_float.yml", 1_000_000, 100_000, 1_000_000,
                      "NLL+grad evals/s @1M data+1M MC, masses and widths floating",
                      "Lambda_c+ -> p K- pi+ (the headline model) with the three resonance masses "
                      "and widths floating (no Gram matrix), 1e6 accept-reject signal + 1e5 flat "
                      "background (w=-0.1) data rows, 1e6 flat MC"),
    "b2dstkpi": ("b2dstkpi.yml", 1_000_000, 0, 4_000_000,
                 "NLL+grad evals/s @1M data+4M MC",
                 "B -> D*(2007) (-> D pi_s) K pi, 12 resonances (J = 0..3) in the D*K, D*pi "
                 "and K pi topologies, 30 LS columns, 1 helicity combination; 1e6 "
                 "accept-reject data, 4e6 flat MC"),
}
CONFIG, N_SIG, N_BG, N_MC, METRIC, WORKLOAD = WORKLOADS["lc2pkpi"]
# DRAM bytes (read + write) per data event of one launch of the cached
# data-term kernel, from ncu captures of that kernel at the bench sizes
# (Lambda_c: 290.4 + 6.8 MB for 1.1e6 rows; four-body: 248.0 + 3.6 MB for
# 1e6 rows); traffic grows with the rows, so a launch's traffic = this x rows
NCU_TRAFFIC_PER_ROW = {"lc2pkpi": (290.436096e6 + 6.841088e6) / 1.1e6,
                       "b2dstkpi": (248.044032e6 + 3.609856e6) / 1e6}
# the same for the floating-shape evaluation kernel, per event (data + MC):
# D -> K pi pi, 80.04 + 2.29 MB for 2e6 events
# (Lambda_c: 151.30 + 5.62 MB for the 5.25e5 events of a quarter-size
# capture, inputs larger than L2; traffic grows with the events)
NCU_SC_TRAFFIC_PER_EVENT = {"d2kpipi_float": (80.041728e6 + 2.286848e6) / 2e6,
                            "lc2pkpi_float": (151.29728e6 + 5.616384e6) / 5.25e5}
# its FP64 operations per event (2 DFMA + DMUL + DADD executed, ncu; 5e5 and
# 5.25e5 events)
NCU_SC_F64_FLOPS_PER_EVENT = {"d2kpipi_float": (2 * 54011168 + 33358304 + 17445502) / 5e5,
                              "lc2pkpi_float": (2 * 222667712 + 81638424 + 38105098) / 5.25e5}


def _select(name):
    global CONFIG, N_SIG, N_BG, N_MC, METRIC, WORKLOAD
    CONFIG, N_SIG, N_BG, N_MC, METRIC, WORKLOAD = WORKLOADS[name]


def _pkg():
    sys.path.insert(0, ROOT)
    import __graft_entry__ as g

    return g._pkg()


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ----------------------------------------------------------------- clocks
def _clocks_path(rank):
    """Where the nvidia-smi samples of the timed region go (PWA_CLOCKS_DIR,
    default the system temp directory)."""
    import tempfile

    d = os.environ.get("PWA_CLOCKS_DIR") or tempfile.gettempdir()
    return os.path.join(d, f"clocks_rank{rank}.csv")


class Clocks:
    def __init__(self, path):
        self.path = path
        self.proc = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self, gpu_index=0):
        if self.proc is None:
            return None
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path).read().splitlines()[1:]:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9 or parts[0] != str(gpu_index):
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                mx = float(parts[2].split()[0])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------- cpu oracle
_W = {}


def _oracle_init(cfg, shm_name, shape):
    """Worker set-up: the model and a view of the shared event fields."""
    from multiprocessing import shared_memory

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import conftest  # noqa: F401  (package loader)
    from common import load_model
    from oracle.pwa_oracle import OracleModel

    dc, vm, plan = load_model(cfg)
    _W["m"] = OracleModel(dc.decay_group, plan)
    _W["shm"] = shared_memory.SharedMemory(name=shm_name)
    _W["x"] = np.ndarray(shape, dtype=np.float64, buffer=_W["shm"].buf)


def _oracle_chunk(args):
    """Sums of one event range [b, e) of one set, in batches of 65000 (the
    reference FCN's batch): data (sum w clip_log f, sum w clip_log'(f) G_k)
    or MC (sum w f, sum w G_k) from the partial-wave columns -- the NLL and
    every coupling derivative from one pass, as the reference's
    GradientTape pass over FCN.nll_grad."""
    b, e, w, vals, data = args
    from oracle.pwa_oracle import column_sums

    s, g = 0.0, 0.0
    for q in range(b, e, 65000):
        r = min(q + 65000, e)
        s1, g1 = column_sums(_W["m"], _W["x"][:, q:r], w[q - b:r - b], vals, {}, data)
        s, g = s + s1, g + g1
    return s, g


class CpuOracle:
    """FP64 oracle NLL + gradient over the whole workload (1.1e6 data rows +
    1e6 MC events for the Lambda_c workload) on all host cores: spawned
    worker processes, one contiguous range of events each, fields in shared
    memory, one pass per evaluation (partial-wave columns, then all
    coupling derivatives).  Events: seeded flat phase space (the timing of
    an evaluation does not depend on where the events lie)."""

    def __init__(self, n_data, n_mc, n_bg=0, seed=5):
        import multiprocessing as mp
        from multiprocessing import shared_memory

        _pkg()
        from tf_pwa_b200.api import ConfigLoader
        from tf_pwa_b200.kinematics import event_fields, p4_dict
        from tf_pwa_b200.phasespace import generate_phsp
        from tf_pwa_b200.workload import config_path, seeded_params

        cl = ConfigLoader(config_path(CONFIG), seed=seed)
        self.vals = seeded_params(cl.vm, seed)
        self.trainable = list(cl.vm.trainable_vars)
        order = cl.get_dat_order()
        pp = cl.decay_config.particle_property
        masses = [pp[o]["mass"] for o in order]
        M = pp[str(cl.decay_group.top)]["mass"]
        n = n_data + n_mc
        ps = generate_phsp(M, masses, n, seed=seed)
        p4 = np.stack(ps, 1)
        self.shm = shared_memory.SharedMemory(create=True, size=8 * cl.plan.n_fields * n)
        x = np.ndarray((cl.plan.n_fields, n), dtype=np.float64, buffer=self.shm.buf)
        for q in range(0, n, 500_000):
            r = min(q + 500_000, n)
            x[:, q:r] = event_fields(cl.plan, p4_dict(p4[q:r], order)).numpy()
        w = np.ones(n_data)
        if n_bg:
            w[n_data - n_bg:] = -BG_WEIGHT
        w = w * (w.sum() / (w * w).sum())
        self.sw = float(w.sum())
        wm = np.ones(n_mc) / n_mc
        self.cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (
            os.cpu_count() or 1)
        self.args = []
        for lo, hi, ww, is_d, off in ((0, n_data, w, True, 0), (n_data, n, wm, False, n_data)):
            cuts = np.linspace(lo, hi, self.cores + 1).astype(np.int64)
            for b, e in zip(cuts[:-1], cuts[1:]):
                if e > b:
                    self.args.append((int(b), int(e), ww[b - off:e - off], self.vals, is_d))
        self.n_data, self.n_mc = n_data, n_mc
        from oracle.pwa_oracle import OracleModel

        self.names = OracleModel(cl.decay_group, cl.plan).columns(x[:, :1], self.vals, {})[1]
        env = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS",
                                               "MKL_NUM_THREADS")}
        for k in env:
            os.environ[k] = "1"  # one thread per worker process
        try:
            self.pool = mp.get_context("spawn").Pool(
                self.cores, initializer=_oracle_init,
                initargs=(CONFIG, self.shm.name, (cl.plan.n_fields, n)))
        finally:
            for k, v in env.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
        self.step()  # warm: imports, CG tables

    def step(self):
        """One NLL + gradient evaluation; returns its wall time (s)."""
        from oracle.pwa_oracle import nll_grad_from_sums

        t0 = time.perf_counter()
        res = self.pool.map(_oracle_chunk, self.args, chunksize=1)
        sd = sum(r[0] for r, a in zip(res, self.args) if a[4])
        gd = sum(r[1] for r, a in zip(res, self.args) if a[4])
        sm = sum(r[0] for r, a in zip(res, self.args) if not a[4])
        gm = sum(r[1] for r, a in zip(res, self.args) if not a[4])
        self.result = nll_grad_from_sums(self.names, self.vals, {}, self.trainable, sd, gd, sm,
                                         gm, self.sw)
        return time.perf_counter() - t0

    def describe(self, t, steps):
        return (f"whole workload every step ({self.n_data} data rows + {self.n_mc} MC events, "
                f"seeded flat phase space), FP64 numpy oracle, one pass per evaluation "
                f"(partial-wave columns, then NLL and all {len(self.trainable)} coupling "
                f"derivatives), {self.cores} spawned single-thread workers, "
                f"{t:.3f} s per evaluation over {steps} evaluations")

    def close(self):
        self.pool.close()
        self.pool.join()
        self.shm.close()
        self.shm.unlink()


def cpu_baseline(n_sig, n_bg, n_mc, steps=3):
    o = CpuOracle(n_sig + n_bg, n_mc, n_bg)
    try:
        t = float(np.mean([o.step() for _ in range(steps)]))
    finally:
        o.close()
    return {"value": 1.0 / t, "unit": "evals/s", "cores": o.cores, "kind": "port",
            "sample": o.describe(t, steps)}


# ------------------------------------------------------------ reference arm
def run_reference(args, rank):
    """The reference's CPU path on the host cores.  TensorFlow is not
    installed, so the reference package cannot run; its FP64 restatement
    (the oracle) stands in, over the whole workload every step."""
    if rank != 0:
        return
    o = CpuOracle(args.n_sig + args.n_bg, args.n_mc, args.n_bg)
    try:
        for _ in range(max(args.warmup - 1, 0)):  # one warm step ran at set-up
            o.step()
        ts = [o.step() for _ in range(args.steps)]
    finally:
        o.close()
    t = float(np.mean(ts))
    v = 1.0 / t
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "evals/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD,
                       "events_per_rank": {"data": args.n_sig + args.n_bg, "mc": args.n_mc},
                       "precision": "FP64 CPU (numpy oracle standing in "
                       "for the reference's TensorFlow CPU path, which is not installed)"},
            "cpu_baseline": {"value": v, "unit": "evals/s", "cores": o.cores, "kind": "port",
                             "sample": o.describe(t, args.steps)},
            "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------- GPU timing
L2_BYTES = 126e6


class Timer:
    """k timed steps, device time from CUDA events on the launching
    (current) stream, max over ranks.  With ``do_flush`` set, a 256 MB
    buffer is written before every step (L2 is 126 MB); workloads whose
    every kernel streams more than the L2 holds per launch run without it
    (inputs larger than L2: a step finds none of its inputs there)."""

    def __init__(self, dist):
        import torch

        self.torch, self.dist = torch, dist
        self.flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        self.do_flush = True

    def barrier(self):
        self.torch.cuda.synchronize()
        if self.dist is not None:
            self.dist.barrier()

    def __call__(self, step_fn, k):
        torch = self.torch
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(k)]
        self.barrier()
        for i in range(k):
            if self.do_flush:
                self.flush.zero_()
            ev[i][0].record()
            step_fn()
            ev[i][1].record()
        self.barrier()
        t = sum(a.elapsed_time(b) for a, b in ev) / 1e3
        if self.dist is not None:
            tt = torch.tensor([t], device="cuda", dtype=torch.float64)
            self.dist.all_reduce(tt, op=self.dist.ReduceOp.MAX)
            t = float(tt.item())
        return t


def _reduce_fn(dist):
    if dist is None:
        return None
    import torch

    def reduce_fn(vec):
        t = torch.as_tensor(vec, device="cuda")
        dist.all_reduce(t)
        return t.cpu().numpy()

    return reduce_fn


# Forward flops per event of sum |A|^2 (fma = 2 flops; divisions, square
# roots and transcendental calls counted apart), counted from the oracle's
# expression graph by oracle/flop_count.py (pinned by
# tests/test_flop_count.py): the compute work unit of the amplitude kernels.
FWD_FLOPS = {"d2kpipi_float": (318, 77), "lc2pkpi": (1614, 228), "b2dstkpi": (6760, 1081)}
# FP64 operations per event of one launch of the plain kernel (forward and
# adjoint, data and MC alike), 2 * DFMA + DADD + DMUL executed, from an ncu
# capture of pwa_eval_f64 (None: not captured; the forward count is used)
NCU_F64_FLOPS_PER_EVENT = {
    # 2 * 8.17425e8 DFMA + 3.88825e8 DMUL + 7.97437e7 DADD per launch over
    # 2.75e5 data + 2.5e5 MC events of the Lambda_c model
    "lc2pkpi": (2 * 817425000 + 388825000 + 79743704) / 5.25e5,
    # 2 * 1.9591e9 DFMA + 1.0715e9 DMUL + 1.35105e8 DADD over 1e5 + 4e5 events
    "b2dstkpi": (2 * 1959100000 + 1071500000 + 135104560) / 5e5,
    # 2 * 1.9925e8 DFMA + 9.075e7 DMUL + 2.74312e7 DADD over 2.5e5 + 2.5e5 events
    "d2kpipi_float": (2 * 199250000 + 90750000 + 27431232) / 5e5,
}
# FP32 and FP64 operations per event of the FP32-amplitude kernel
# (pwa_eval_f32), same captures: 2 * FFMA + FMUL + FADD, 2 * DFMA + DMUL + DADD
NCU_F32_KERNEL_FLOPS = {
    "d2kpipi_float": ((2 * 109378880 + 53568320 + 8189440) / 5e5,
                      (2 * 47750000 + 25250000 + 27289040) / 5e5),
    "lc2pkpi": ((2 * 630454656 + 312006984 + 25275776) / 5.25e5,
                (2 * 94500000 + 55975000 + 71343704) / 5.25e5),
    "b2dstkpi": ((2 * 1467318624 + 930727936 + 92454656) / 5e5,
                 (2 * 99600000 + 57500000 + 136206080) / 5e5),
}
# the Lambda_c model with floating masses and widths compiles to the same
# plain and FP32 kernels as with fixed ones
for _table in (FWD_FLOPS, NCU_F64_FLOPS_PER_EVENT, NCU_F32_KERNEL_FLOPS):
    _table["lc2pkpi_float"] = _table["lc2pkpi"]
FLOATING = ("d2kpipi_float", "lc2pkpi_float")


def _mixed_pipe_roofline(name, n_ev, launch_s, peaks):
    """Roofline of a kernel doing both FP32 and FP64 work: the ideal time is
    FP32 ops / FP32 peak + FP64 ops / FP64 peak (measured FMA peaks);
    frac = ideal / measured, achieved = total ops / measured time."""
    f32, f64 = NCU_F32_KERNEL_FLOPS[name]
    ideal = n_ev * (f32 / (peaks["f32_tflops"] * 1e12) + f64 / (peaks["f64_tflops"] * 1e12))
    ops = n_ev * (f32 + f64)
    return {"bound": "fp32+fp64", "achieved": ops / launch_s / 1e12,
            "peak": ops / ideal / 1e12, "unit": "TFLOP/s", "frac": ideal / launch_s,
            "peak_kind": "measured here (pwa_fma_peak, FP32 and FP64 FMA chains), "
                         "weighted by the kernel's FP32 / FP64 operation mix",
            "flops_per_event": {"fp32": f32, "fp64": f64},
            "flops_source": "ncu: 2 FFMA + FMUL + FADD and 2 DFMA + DMUL + DADD executed",
            "launch_us": 1e6 * launch_s, "events_per_launch": n_ev}

CACHED_KERNEL = {0: "pwa_eval_cached (bulk-copy ring, per-thread FP64 column sums)",
                 1: "pwa_eval_cached_direct (direct loads, per-thread FP64 column sums)",
                 2: "pwa_eval_cached_wred (direct loads, warp reduce-scatter column sums)",
                 3: "pwa_eval_cached_ring2 (two-stage ring, reduce-scatter consumers)",
                 4: "pwa_eval_cached_wide (one block of 16 warps per SM, contiguous runs)",
                 5: "pwa_eval_cached_tma (one block per SM, producer warp, deep bulk-copy ring)"}


def measure_cached(name, args, rank, world, dist, timed, log, n_sig, n_bg, n_mc,
                   variants=True):
    """Fixed masses and widths: the mixed form (FP32 column cache, FP64
    amplitudes / log / sums, FP64 Gram MC term) against the plain FP64
    kernels and the FP32-recompute form, on one workload.  Returns the JSON
    line (without the CPU baseline) and the engines' peak info."""
    import torch

    from tf_pwa_b200.api import FCN
    from tf_pwa_b200.engine import FORM_MIXED_F32, FORM_PLAIN_F64, MIXED_F32, PLAIN_F64
    from tf_pwa_b200.workload import make_dataset

    config, _, _, _, metric, workload = WORKLOADS[name]
    t0 = time.perf_counter()
    cl, data, bg, mc = make_dataset(config, n_sig, n_mc, n_bg=n_bg, bg_weight=BG_WEIGHT,
                                    seed=1 + rank, device="cuda")
    t_data = time.perf_counter() - t0
    log(f"{name}: dataset {n_sig} signal + {n_bg} background + {n_mc} MC events")
    t0 = time.perf_counter()
    fcn = FCN(cl, data, mc, bg=bg, precision="mixed")  # column cache + Gram, autotuned
    t_mixed_setup = time.perf_counter() - t0
    log(f"{name}: mixed-form FCN ready (tuned {fcn.eng.cached_config()})")
    fcn_plain = FCN(cl, data, mc, bg=bg, precision="plain")
    for f in (fcn, fcn_plain):
        f.eng.dist_reduce = _reduce_fn(dist)
        f.eng.mc_share = 1.0 / world  # equal MC shards
    x0 = np.array(cl.vm.get_all_val())
    names = list(cl.vm.trainable_vars)
    vals = cl.vm.get_all_dic()
    eng, eng_p = fcn.eng, fcn_plain.eng
    var_vec = np.array([vals[k] for k in fcn._var_names])
    code = eng.code
    n_data = n_sig + n_bg
    bytes_mixed = n_data * (8 * code.nf + 8)
    bytes_f32 = (n_data + n_mc) * (8 * len(code.mass_fields) + 4 * len(code.angle_fields) + 8)
    # back-to-back launches of a 145 MB column cache still find ~28 % of it
    # in the 126 MB L2 (ncu, cache control off): every step is flushed
    timed.do_flush = True
    l2_note = (f"256 MB buffer written before every timed step (L2 126 MB); inputs "
               f"{bytes_mixed / 1e6:.0f} MB per launch of the cached kernel, "
               f"{bytes_f32 / 1e6:.0f} MB of the FP32 kernel")
    for _ in range(args.warmup):
        fcn.nll_grad(x0)
        fcn_plain.nll_grad(x0)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    clocks = Clocks(_clocks_path(rank))
    clocks.start()
    # headline: one NLL+gradient evaluation per step through the C ABI
    # (couplings -> cached-column kernel + Gram MC term -> chain rule)
    t_mixed = timed(lambda: eng.nll_grad_cached(var_vec), args.steps)
    # the plain FP64 form through the same native host side (host program)
    assert fcn_plain.native_host
    t_plain = timed(lambda: eng_p.nll_grad_vars(var_vec, FORM_PLAIN_F64), args.steps)
    # e2e through the public API with host parameters
    t_e2e = timed(lambda: fcn.nll_grad(x0), args.steps)
    # as a fit runs them: evaluations back to back with no flush between
    # (the inputs, 290 MB of columns, are larger than L2 either way)
    timed.do_flush = False
    t_mixed_b2b = timed(lambda: eng.nll_grad_cached(var_vec), args.steps)
    t_plain_b2b = timed(lambda: eng_p.nll_grad_vars(var_vec, FORM_PLAIN_F64), args.steps)
    timed.do_flush = True
    # roofline: the data-term kernel (with its own ordered reduction) alone
    eng.consts(vals)
    ck = np.stack([eng._ck.real, eng._ck.imag], 1).reshape(-1)
    k_kernel = args.steps
    t_kernel = timed(lambda: eng.eval_cached_enqueue(ck), k_kernel)
    # the same number of bytes read by a library reduction (torch.sum of an
    # FP32 tensor), same L2 protocol: what one plain pass over that many bytes
    # costs on this GPU, fixed per-launch part included
    floor_buf = torch.ones(bytes_mixed // 4, dtype=torch.float32, device="cuda")
    for _ in range(3):
        floor_buf.sum()
    t_floor = timed(lambda: floor_buf.sum(), k_kernel)
    del floor_buf
    # Hessian of all trainable parameters: exact, from one pass of the
    # Hessian-sums kernel; and, for comparison, the 4P stencil points of the
    # differenced adjoint gradient in one multi-point pass over the cache
    k_hess = 3
    eng.hessian_cached_exact(var_vec)
    t_hess = timed(lambda: eng.hessian_cached_exact(var_vec), k_hess)
    t_hess_fd = timed(lambda: eng.hessian_cached(var_vec, 1e-2), k_hess)
    Cp = eng_p.consts(vals)
    t_kernel_p = timed(lambda: eng_p.eval_enqueue(Cp, PLAIN_F64, mc=True), k_kernel)
    # the FP32-amplitude recompute form (what a fit with floating masses and
    # widths, where no column cache applies, uses instead of plain FP64)
    t_f32 = timed(lambda: eng_p.nll_grad_vars(var_vec, FORM_MIXED_F32), args.steps)
    t_kernel_f32 = timed(lambda: eng_p.eval_enqueue(Cp, MIXED_F32, mc=True), k_kernel)
    ck_clocks = clocks.stop(local)
    tuned = eng.cached_config()
    var_table = {}
    if variants:
        for var in (0, 1, 2, 3, 4, 5):
            eng.set_cached_config(var)
            var_table[var] = {
                "kernel_us": 1e6 * timed(lambda: eng.eval_cached_enqueue(ck), k_kernel) / k_kernel,
                "step_us": 1e6 * timed(lambda: eng.nll_grad_cached(var_vec), args.steps)
                / args.steps,
                "nll": eng.nll_grad_cached(var_vec)[0]}
        eng.set_cached_config(*tuned)
    nll_m, g_m = eng.nll_grad_cached(var_vec)
    nll_p, g_p = eng_p.nll_grad(vals, names, PLAIN_F64)
    nll_f, g_f = eng_p.nll_grad(vals, names, MIXED_F32)
    peaks = {"f64_tflops": eng.fma_peak(PLAIN_F64) / 1e12,
             "f32_tflops": eng.fma_peak(MIXED_F32) / 1e12}

    hbm, peak_kind = _peaks()
    ach = bytes_mixed / (t_kernel / k_kernel) / 1e9
    n_ev = n_data + n_mc
    fl_ev = NCU_F64_FLOPS_PER_EVENT.get(name)
    fl_kind = "ncu: 2 DFMA + DADD + DMUL executed per event (forward and adjoint)"
    if fl_ev is None:
        fl_ev, fl_kind = FWD_FLOPS[name][0], "forward sum |A|^2 only (oracle count): a lower bound"
    ach_p = fl_ev * n_ev / (t_kernel_p / k_kernel) / 1e12
    value = world * args.steps / t_mixed
    line = {
        "metric": metric, "value": value, "unit": "evals/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_mixed / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": workload, "precision": "mixed: per-event partial-wave columns "
                   "cached as FP32 (computed in FP64), FP64 amplitude sum, log and reductions; "
                   "MC integral from the FP64-accurate Gram matrix (masses/widths fixed)",
                   "events_per_rank": {"data": n_data, "mc": n_mc},
                   "l2": l2_note,
                   "parallelism": f"dp{world}" if world > 1 else "single GPU"},
        "plain_f64": {"value": world * args.steps / t_plain, "unit": "evals/s",
                      "ms_per_step": 1e3 * t_plain / args.steps,
                      "speedup_mixed_over_plain": t_plain / t_mixed},
        "back_to_back": {"what": "the same two steps with no L2 flush between evaluations, "
                                 "as in a fit (inputs larger than L2)",
                         "mixed_ms_per_step": 1e3 * t_mixed_b2b / args.steps,
                         "plain_ms_per_step": 1e3 * t_plain_b2b / args.steps,
                         "speedup_mixed_over_plain": t_plain_b2b / t_mixed_b2b},
        "fp32_recompute": {"value": world * args.steps / t_f32, "unit": "evals/s",
                           "ms_per_step": 1e3 * t_f32 / args.steps,
                           "kernel_us": 1e6 * t_kernel_f32 / k_kernel,
                           "roofline": (_mixed_pipe_roofline(name, n_ev, t_kernel_f32 / k_kernel,
                                                             peaks)
                                        if name in NCU_F32_KERNEL_FLOPS else None),
                           "dnll": nll_f - nll_p,
                           "grad_max_rel": float(np.max(np.abs(g_f - g_p)) / np.max(np.abs(g_p)))},
        "e2e": {"value": world * args.steps / t_e2e, "unit": "evals/s",
                "h2d_bytes_per_step": 8 * len(x0),
                "d2h_bytes_per_step": 8 * (1 + len(x0)),
                "call": "FCN.nll_grad(x) with x a host numpy vector"},
        "roofline": {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                     "frac": ach / hbm,
                     "traffic": (NCU_TRAFFIC_PER_ROW[name] * n_data
                                 if name in NCU_TRAFFIC_PER_ROW else None),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                       "launch at the bench size, scaled by the rows",
                     "peak_kind": peak_kind,
                     "kernel": CACHED_KERNEL[tuned[0]] + "; ends with its own fixed-order "
                               "reduction",
                     "algorithmic_bytes_per_launch": bytes_mixed,
                     "launch_us": 1e6 * t_kernel / k_kernel,
                     "read_floor": {
                         "what": "torch.sum over the same number of bytes, same L2 protocol",
                         "launch_us": 1e6 * t_floor / k_kernel,
                         "kernel_over_floor": t_kernel / t_floor},
                     "plain_f64_kernel": {
                         "bound": "fp64", "achieved": ach_p, "peak": peaks["f64_tflops"],
                         "unit": "TFLOP/s", "frac": ach_p / peaks["f64_tflops"],
                         "peak_kind": "measured here (pwa_fma_peak, FP64 FMA chains)",
                         "flops_per_event": fl_ev, "flops_source": fl_kind,
                         "launch_us": 1e6 * t_kernel_p / k_kernel,
                         "events_per_launch": n_ev}},
        "fma_peaks": peaks,
        "gpu_launches": args.steps,
        "autotune": {"choice": {"variant": tuned[0], "ring_stages": tuned[1],
                                "blocks_per_sm": tuned[2]},
                     "table_us": None if fcn.tune is None or fcn.tune[0] is None
                     else [round(float(x), 2) for x in fcn.tune[0]],
                     "error": fcn.tune[2] if fcn.tune is not None and len(fcn.tune) > 2
                     else None,
                     "pinned": os.environ.get("PWA_CACHED_CONFIG")},
        "cached_variants": var_table,
        "hessian": {"ms": 1e3 * t_hess / k_hess, "n_params": len(names),
                    "in_single_steps": (t_hess / k_hess) / (t_mixed / args.steps),
                    "call": "pwa_hessian_cached_exact: exact Hessian in the couplings, one "
                            "pass of the Hessian-sums kernel over the column cache",
                    "stencil": {"ms": 1e3 * t_hess_fd / k_hess, "points": 4 * len(names),
                                "in_single_steps": (t_hess_fd / k_hess) / (t_mixed / args.steps),
                                "call": "pwa_hessian_cached: 4-point differences of the "
                                        "adjoint gradient, one multi-point pass"}},
        "check": {"nll_mixed": nll_m, "nll_plain": nll_p, "dnll": nll_m - nll_p,
                  "grad_max_rel": float(np.max(np.abs(g_m - g_p)) / np.max(np.abs(g_p)))},
        "setup_s": {"dataset": t_data, "mixed_fcn": t_mixed_setup},
        "engine": eng.info(),
    }
    if ck_clocks:
        line["clocks"] = ck_clocks
    fcn.eng.close()
    fcn_plain.eng.close()
    del fcn, fcn_plain, data, bg, mc
    torch.cuda.empty_cache()
    return line


# ------------------------------------------------- floating masses/widths
def measure_floating(name, args, rank, world, dist, timed, log, n_sig, n_mc, n_bg=0):
    """Workload with floating lineshape parameters (no Gram matrix): the
    chosen form is the floating-shape column cache (shape-free columns
    cached in FP32, lineshapes recomputed from the resident masses every
    evaluation, FP64 amplitude and sums), beside the FP32-amplitude
    recompute form and the plain FP64 kernels; the Hessian comes from
    differenced adjoint gradients."""
    import torch

    from tf_pwa_b200.api import FCN
    from tf_pwa_b200.engine import MIXED_F32, PLAIN_F64
    from tf_pwa_b200.workload import make_dataset

    config, _, _, _, metric, workload = WORKLOADS[name]
    t0 = time.perf_counter()
    cl, data, bg, mc = make_dataset(config, n_sig, n_mc, n_bg=n_bg, bg_weight=BG_WEIGHT,
                                    seed=1 + rank)
    t_data = time.perf_counter() - t0
    log(f"{name}: dataset {n_sig} data + {n_bg} background + {n_mc} MC events")
    t0 = time.perf_counter()
    fcn = FCN(cl, data, mc, bg=bg, precision="mixed")
    t_cache = time.perf_counter() - t0
    assert not fcn.use_gram and fcn.use_shape_cache
    fcn_r = FCN(cl, data, mc, bg=bg, precision="mixed", shape_cache=False)
    fcn_p = FCN(cl, data, mc, bg=bg, precision="plain")
    for f in (fcn, fcn_r, fcn_p):
        f.eng.dist_reduce = _reduce_fn(dist)
        f.eng.mc_share = 1.0 / world  # equal MC shards
    x0 = np.array(cl.vm.get_all_val())
    vals, names = cl.vm.get_all_dic(), list(cl.vm.trainable_vars)
    timed.do_flush = True  # its inputs fit in L2
    for _ in range(args.warmup):
        fcn.nll_grad(x0)
        fcn_r.nll_grad(x0)
        fcn_p.nll_grad(x0)
    clocks = Clocks(_clocks_path(rank))
    clocks.start()
    t_sc = timed(lambda: fcn.nll_grad(x0), args.steps)
    t_f32 = timed(lambda: fcn_r.nll_grad(x0), args.steps)
    t_p = timed(lambda: fcn_p.nll_grad(x0), args.steps)
    # as in a fit: every evaluation at a new mass/width setting (two points
    # alternating), so the lineshape and barrier constants are rebuilt each time
    x1 = x0.copy()
    for i, n in enumerate(names):
        if n.endswith(("_mass", "_width")):
            x1[i] *= 1.0 + 1e-6
    pts = [x0, x1]
    t_mv = timed(lambda: fcn.nll_grad(pts[fcn.n_call % 2]), args.steps)
    # the same two timings with the host side in the engine's Python code
    native = fcn.native_host
    fcn.native_host = False
    t_py = timed(lambda: fcn.nll_grad(x0), args.steps)
    t_py_mv = timed(lambda: fcn.nll_grad(pts[fcn.n_call % 2]), args.steps)
    fcn.native_host = native
    C = fcn.eng.consts(vals)
    for _ in range(3):
        fcn.eng.eval_shapecache_enqueue(C)
    t_ks = timed(lambda: fcn.eng.eval_shapecache_enqueue(C), args.steps)
    t_k = timed(lambda: fcn_r.eng.eval_enqueue(C, MIXED_F32, mc=True), args.steps)
    t_kp = timed(lambda: fcn_p.eng.eval_enqueue(C, PLAIN_F64, mc=True), args.steps)
    th = time.perf_counter()
    _, _, H = fcn.nll_grad_hessian(x0)
    t_hess = time.perf_counter() - th
    cov = np.linalg.inv(H)
    ck_clocks = clocks.stop(int(os.environ.get("LOCAL_RANK", "0")))
    nll_s, g_s = fcn.nll_grad(x0)
    nll_f, g_f = fcn_r.nll_grad(x0)
    nll_p, g_p = fcn_p.nll_grad(x0)
    code = fcn.eng.code
    n_all = n_sig + n_bg + n_mc
    bytes_f32 = n_all * (8 * len(code.mass_fields) + 4 * len(code.angle_fields) + 8)
    bytes_f64 = n_all * (8 * len(code.mass_fields) + 8 * len(code.angle_fields) + 8)
    bytes_sc = n_all * (8 * code.nf + 8 * len(code.mass_fields) + 8)
    hbm, peak_kind = _peaks()
    ach_s = bytes_sc / (t_ks / args.steps) / 1e9
    ach = bytes_f32 / (t_k / args.steps) / 1e9
    peaks = {"f64_tflops": fcn.eng.fma_peak(PLAIN_F64) / 1e12,
             "f32_tflops": fcn.eng.fma_peak(MIXED_F32) / 1e12}
    roof_r = _mixed_pipe_roofline(name, n_all, t_k / args.steps, peaks)
    roof_r.update({"kernel": "pwa_eval_f32 + pwa_reduce (data + MC, FP32 amplitudes)",
                   "hbm": {"achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                           "peak_kind": peak_kind, "algorithmic_bytes_per_launch": bytes_f32}})
    fl_p = NCU_F64_FLOPS_PER_EVENT[name]
    ach_p = fl_p * n_all / (t_kp / args.steps) / 1e12
    hbm_roof = {"bound": "hbm", "achieved": ach_s, "peak": hbm, "unit": "GB/s",
                "frac": ach_s / hbm,
                "traffic": (NCU_SC_TRAFFIC_PER_EVENT[name] * n_all
                            if name in NCU_SC_TRAFFIC_PER_EVENT else None),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch "
                                  "at the bench size, scaled by the events",
                "peak_kind": peak_kind}
    if name in NCU_SC_F64_FLOPS_PER_EVENT:
        # the kernel is bound by its FP64 lineshape arithmetic, not by HBM
        fl_s = NCU_SC_F64_FLOPS_PER_EVENT[name]
        ach_f = fl_s * n_all / (t_ks / args.steps) / 1e12
        roof = {"bound": "fp64", "achieved": ach_f, "peak": peaks["f64_tflops"],
                "unit": "TFLOP/s", "frac": ach_f / peaks["f64_tflops"],
                "peak_kind": "measured here (pwa_fma_peak, FP64 FMA chains)",
                "flops_per_event": fl_s,
                "flops_source": "ncu: 2 DFMA + DMUL + DADD executed per event",
                "traffic": hbm_roof["traffic"], "hbm": hbm_roof}
    else:
        roof = dict(hbm_roof)
    roof.update({
        "kernel": "pwa_eval_shapecache with its own reduction (data + MC: FP32 shape-free columns, "
                  "FP64 masses, lineshapes recomputed)",
        "algorithmic_bytes_per_launch": bytes_sc, "launch_us": 1e6 * t_ks / args.steps,
        "plain_f64_kernel": {
            "bound": "fp64", "achieved": ach_p, "peak": peaks["f64_tflops"],
            "unit": "TFLOP/s", "frac": ach_p / peaks["f64_tflops"], "flops_per_event": fl_p,
            "flops_source": "ncu: 2 DFMA + DADD + DMUL executed per event (forward and "
                            "adjoint)",
            "launch_us": 1e6 * t_kp / args.steps, "algorithmic_bytes_per_launch": bytes_f64}})
    line = {
        "metric": metric, "value": world * args.steps / t_sc, "unit": "evals/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t_sc / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload, "precision": "floating-shape column cache: per-event "
                   "partial-wave columns without their lineshapes cached as FP32 (computed in "
                   "FP64), lineshapes and their derivatives recomputed in FP64 from the resident "
                   "masses every evaluation, FP64 amplitude, log and sums",
                   "events_per_rank": {"data": n_sig, "background": n_bg, "mc": n_mc},
                   "l2": "256 MB buffer written before every timed step (L2 126 MB)",
                   "parallelism": f"dp{world}" if world > 1 else "single GPU"},
        "plain_f64": {"value": world * args.steps / t_p, "unit": "evals/s",
                      "ms_per_step": 1e3 * t_p / args.steps,
                      "speedup_over_plain": t_p / t_sc},
        "fp32_recompute": {"value": world * args.steps / t_f32, "unit": "evals/s",
                           "ms_per_step": 1e3 * t_f32 / args.steps,
                           "kernel_us": 1e6 * t_k / args.steps, "roofline": roof_r,
                           "dnll": nll_f - nll_p,
                           "grad_max_rel": float(np.max(np.abs(g_f - g_p)) / np.max(np.abs(g_p)))},
        "e2e": {"value": world * args.steps / t_sc, "unit": "evals/s",
                "h2d_bytes_per_step": 8 * len(x0), "d2h_bytes_per_step": 8 * (1 + len(x0)),
                "call": "FCN.nll_grad(x) with x a host numpy vector"},
        "roofline": roof,
        "host": {"native": bool(fcn.native_host),
                 "us_per_step": 1e6 * (t_sc - t_ks) / args.steps,
                 "what": "FCN.nll_grad step minus the device time of its kernels: parameter "
                         "copy, constants, Jacobian, launch, result read, chain rule",
                 "moving_point": {"ms_per_step": 1e3 * t_mv / args.steps,
                                  "value": world * args.steps / t_mv,
                                  "what": "each evaluation at a new mass/width setting"},
                 "python_host": {"ms_per_step": 1e3 * t_py / args.steps,
                                 "moving_point_ms_per_step": 1e3 * t_py_mv / args.steps,
                                 "what": "the same steps with the host side in the engine's "
                                         "Python code (Engine.nll_grad)"}},
        "fma_peaks": peaks,
        # one launch of pwa_eval_shapecache per timed step (its reduction is
        # in the same launch)
        "gpu_launches": args.steps,
        "hessian": {"seconds": t_hess, "n_params": len(x0), "evaluations": 4 * len(x0) + 1,
                    "errors": dict(zip(names, np.sqrt(np.abs(np.diag(cov))).tolist()))},
        "check": {"nll_shape_cache": nll_s, "nll_plain": nll_p, "dnll": nll_s - nll_p,
                  "grad_max_rel": float(np.max(np.abs(g_s - g_p)) / np.max(np.abs(g_p)))},
        "setup_s": {"dataset": t_data, "shape_cache_fcn": t_cache},
    }
    if ck_clocks:
        line["clocks"] = ck_clocks
    for f in (fcn, fcn_r, fcn_p):
        f.eng.close()
    del fcn, fcn_r, fcn_p, data, mc
    torch.cuda.empty_cache()
    return line


def _compact(line):
    """A workload's line trimmed for the `workloads` key of the headline line."""
    keep = ("metric", "value", "unit", "ms_per_step", "config", "plain_f64", "fp32_recompute",
            "e2e", "roofline", "host", "autotune", "hessian", "check", "clocks", "setup_s")
    return {k: line[k] for k in keep if k in line}


# ------------------------------------------------------------- serving arm
SERVING_METRIC = "toy-fit service: per-fit latency p50/p99 and aggregate NLL+grad evals/s"
SERVING_WORKLOAD = ("d2kpipi model (2 chains), fits with log-uniform 1e3..1e6 data events, "
                    "shared 1e6 MC, Poisson arrivals, BFGS per fit, admission under a 150 GB "
                    "HBM budget, mixed form (column cache + Gram)")


def run_serving(args):
    """Toy-fit service: 512 fits of the d2kpipi model, event counts
    log-uniform in [1e3, 1e6], shared 1e6-event MC, Poisson arrivals, each
    fit a BFGS driver issuing NLL+gradient calls; continuous batching."""
    import torch

    torch.cuda.set_device(0)
    _pkg()
    from tf_pwa_b200.serving import serving_benchmark

    # headline: all fits arrive at once (Poisson with a rate far above the
    # service rate), so the service runs saturated; then Poisson arrivals
    # spread over about one second (latency under light load), and the same
    # burst served by Python-thread BFGS drivers for comparison
    rate = args.fit_rate or 1e9
    r = serving_benchmark(n_fits=args.n_fits, rate=rate, native=True)
    r_py = serving_benchmark(n_fits=args.n_fits, rate=rate, native=False)
    r_slow = serving_benchmark(n_fits=args.n_fits, rate=args.n_fits / 1.0, native=True)
    line = {"metric": SERVING_METRIC,
            "value": r["evals_per_s"], "unit": "evals/s", "n_gpus": 1,
            "higher_is_better": True, "data": "synthetic", "dtype": "f64",
            "config": {"workload": SERVING_WORKLOAD},
            "serving": r, "serving_python_drivers": r_py,
            "serving_arrivals_over_1s": r_slow}
    print(json.dumps(line), flush=True)


def serving_summary(n_fits):
    """The native service, saturated (all fits at once) and under Poisson
    arrivals over about one second."""
    from tf_pwa_b200.serving import serving_benchmark

    r = serving_benchmark(n_fits=n_fits, rate=1e9, native=True)
    r_slow = serving_benchmark(n_fits=n_fits, rate=n_fits / 1.0, native=True)
    return {"metric": SERVING_METRIC, "unit": "evals/s", "workload": SERVING_WORKLOAD,
            "saturated": r, "arrivals_over_1s": r_slow}


# ----------------------------------------------------------------- our arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours")
    ap.add_argument("--cpu-steps", type=int, default=3,
                    help="evaluations of the CPU oracle baseline (whole workload each)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true",
                    help="skip the four-body, floating-shape and serving keys")
    ap.add_argument("--serving", action="store_true",
                    help="run the toy-fit serving workload instead (separate JSON line)")
    ap.add_argument("--n-fits", type=int, default=512)
    ap.add_argument("--fit-rate", type=float, default=None,
                    help="serving: Poisson arrival rate, fits/s (default: all at once)")
    ap.add_argument("--workload", default="lc2pkpi", choices=sorted(WORKLOADS))
    ap.add_argument("--n-sig", type=int, default=None, help="signal data events per GPU")
    ap.add_argument("--n-bg", type=int, default=None, help="background data rows per GPU")
    ap.add_argument("--n-mc", type=int, default=None, help="MC events per GPU")
    args = ap.parse_args()
    _select(args.workload)
    args.n_sig = N_SIG if args.n_sig is None else args.n_sig
    args.n_bg = N_BG if args.n_bg is None else args.n_bg
    args.n_mc = N_MC if args.n_mc is None else args.n_mc
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)
    args.warmup = max(args.warmup, 3)
    if args.serving:
        return run_serving(args)

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    _pkg()
    timed = Timer(dist)
    t_setup = time.perf_counter()

    def log(msg):
        print(f"[bench {time.perf_counter() - t_setup:8.1f}s] {msg}", file=sys.stderr, flush=True)

    if args.workload in FLOATING:
        line = measure_floating(args.workload, args, rank, world, dist, timed, log, args.n_sig,
                                args.n_mc, args.n_bg)
    else:
        line = measure_cached(args.workload, args, rank, world, dist, timed, log, args.n_sig,
                              args.n_bg, args.n_mc)
    if world == 1 and args.workload == "lc2pkpi" and not args.headline_only:
        # the other workloads the metric names, each at its own size and with
        # its own roofline, and the serving loop (one GPU)
        extra = {}
        try:
            _, s4, b4, m4, _, _ = WORKLOADS["b2dstkpi"]
            extra["b2dstkpi"] = _compact(measure_cached("b2dstkpi", args, rank, world, dist,
                                                        timed, log, s4, b4, m4, variants=False))
            for fname in FLOATING:
                _, sf, bf, mf, _, _ = WORKLOADS[fname]
                extra[fname] = _compact(measure_floating(fname, args, rank, world, dist, timed,
                                                         log, sf, mf, bf))
            log("serving")
            line["serving"] = serving_summary(args.n_fits)
        except Exception as e:  # reported, never fatal to the headline
            extra["error"] = repr(e)
        line["workloads"] = extra
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == "lc2pkpi":
        try:
            line["cpu_baseline"] = cpu_baseline(args.n_sig, args.n_bg, args.n_mc, args.cpu_steps)
        except Exception as e:  # reported, never fatal
            line["cpu_baseline"] = {"error": repr(e)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

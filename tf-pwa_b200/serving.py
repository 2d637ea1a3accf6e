"""Continuous-batching NLL + gradient service for many concurrent fits.

Toy, pull and significance studies run hundreds of independent fits of one
model.  Each fit's BFGS driver (scipy, in its own thread, as
``tf_pwa/fit.py:189-419``) calls ``FCN.nll_grad`` 100-300 times.  The server
keeps every admitted fit's data events resident as a column cache in one
device tile pool, shares the MC sample (and hence one Gram matrix) across
fits, and evaluates ALL requests pending at a given moment in one launch
(``pwa_pieces_multi``).  Requests that arrive while a launch is on the GPU
join the next one; fits are admitted as pool space (the HBM budget) and
active slots free up.  A fit's result depends only on its own data and
parameters: the per-tile sums and the per-fit reduction order are fixed, so
its NLL and gradient are bitwise the same alone or in any mix.

``NativeFitServer`` runs the same service with each fit's BFGS driver as a
state machine inside the native library (one scheduler thread, no
per-fit Python threads): every round evaluates the pending point of every
active fit in one launch and advances each optimiser by one step.
"""
import queue
import threading
import time

import numpy as np
import torch

from .engine import Engine, combine_pieces


class FitJob:
    """One fit: its data (device columns), start values, and results."""

    sid = None
    latency = None
    cols = None

    def __init__(self, fid, fields, x0, arrival=None, gtol=1e-3, maxiter=300):
        self.fid = fid
        self.fields = fields          # (n_fields, N) FP64 tensor on the device
        self.n = fields.shape[1]
        self.x0 = np.asarray(x0, np.float64)
        self.arrival = time.perf_counter() if arrival is None else arrival
        self.gtol = gtol
        self.maxiter = maxiter
        self.admitted = None
        self.finished = None
        self.tiles = None
        self.n_eval = 0
        self.result = None
        self.done = threading.Event()
        self.trace = []               # (nll, grad) of every evaluation


class FitServer:
    def __init__(self, config, mc, budget_bytes, max_active=256, tpb=128, run=True):
        """``config``: ConfigLoader of the model (its parameters hold the
        fixed masses/widths and the fixed couplings); ``mc``: EventData of the
        shared MC sample (device fields).  ``run=False`` creates the server
        without its scheduler thread (for direct single evaluations)."""
        self.cl = config
        self.vm = config.vm
        self.eng = Engine(config.decay_group, config.plan, self.vm, tpb=tpb)
        c = self.eng.code
        x = mc.fields
        xm = x[c.mass_fields].contiguous()
        xa = x[c.angle_fields].contiguous()
        wm = torch.full((mc.n,), 1.0 / mc.n, dtype=torch.float64, device=x.device)
        self.eng.upload_device(xm.data_ptr(), xa.data_ptr(), wm.data_ptr(), 0, mc.n, 0.0)
        torch.cuda.synchronize()
        vals = self.vm.get_all_dic()
        self.eng.set_gram(vals)
        self.consts = self.eng.consts(vals)
        self.var_names = list(self.vm.variables.keys())
        self.train = list(self.vm.trainable_vars)
        self.train_idx = [self.var_names.index(n) for n in self.train]
        self.base_vars = np.array([vals[k] for k in self.var_names])
        self.eng.set_param_layout(self.var_names, self.train)
        self.tile_bytes = tpb * (8 * c.nf + 8)
        self.pool_tiles = max(1, int(budget_bytes // self.tile_bytes))
        self.eng.pool_reserve(self.pool_tiles)
        self.max_active = max_active
        self.pending = []             # admitted-later fits, FIFO
        self.active = {}
        self.requests = queue.Queue()
        self.lock = threading.Lock()
        self.finished = []
        self.batches = []             # (n_requests, n_tiles, seconds)
        self._stop = False
        self._thread = None
        if run:
            self._thread = threading.Thread(target=self._loop, daemon=True)
            self._thread.start()

    # ------------------------------------------------------------ client
    def submit(self, job):
        with self.lock:
            self.pending.append(job)
        self.requests.put(None)       # wake the scheduler
        return job

    def close(self):
        self._stop = True
        self.requests.put(None)
        if self._thread is not None:
            self._thread.join(timeout=30)
        self.eng.close()

    # ------------------------------------------------------------ fits
    def _fit_thread(self, job):
        from scipy.optimize import minimize

        def fg(x):
            ev = threading.Event()
            slot = {}
            self.requests.put((job, np.array(x, np.float64), ev, slot))
            ev.wait()
            if "error" in slot:
                raise RuntimeError(slot["error"])
            job.n_eval += 1
            job.trace.append((slot["nll"], slot["grad"]))
            return slot["nll"], slot["grad"]

        try:
            res = minimize(fg, job.x0, jac=True, method="BFGS",
                           options={"gtol": job.gtol, "maxiter": job.maxiter})
            job.result = {"x": res.x, "nll": float(res.fun), "success": bool(res.success),
                          "nit": int(res.nit)}
        except Exception as e:  # reported on the job, never kills the server
            job.result = {"error": repr(e)}
        job.finished = time.perf_counter()
        self.requests.put(("done", job))

    def _admit(self, start=True):
        with self.lock:
            while self.pending and len(self.active) < self.max_active:
                job = self.pending[0]
                run = self.eng.pool_alloc(job.n)
                if run is None:
                    break             # wait for pool space
                self.pending.pop(0)
                job.tiles = run
                c = self.eng.code
                x = job.fields
                xm = x[c.mass_fields].contiguous()
                xa = x[c.angle_fields].contiguous()
                w = torch.ones(job.n, dtype=torch.float64, device=x.device)
                self.eng.pool_fill(run[0], self.consts, xm.data_ptr(), xa.data_ptr(),
                                   w.data_ptr(), job.n, job.n)
                torch.cuda.synchronize()
                job.admitted = time.perf_counter()
                self.active[job.fid] = job
                if start:
                    threading.Thread(target=self._fit_thread, args=(job,), daemon=True).start()

    # ------------------------------------------------------------ scheduler
    def _loop(self):
        while not self._stop:
            self._admit()
            try:
                items = [self.requests.get(timeout=0.5)]
            except queue.Empty:
                continue
            # everything queued while the previous launch ran joins this one
            while True:
                try:
                    items.append(self.requests.get_nowait())
                except queue.Empty:
                    break
            reqs = []
            for it in items:
                if it is None:
                    continue
                if isinstance(it, tuple) and it[0] == "done":
                    job = it[1]
                    with self.lock:
                        self.active.pop(job.fid, None)
                        self.eng.pool_free(job.tiles[0])
                        self.finished.append(job)
                    job.done.set()
                    continue
                reqs.append(it)
            if not reqs:
                continue
            t0 = time.perf_counter()
            V = np.repeat(self.base_vars[None, :], len(reqs), axis=0)
            for r, (job, x, ev, slot) in enumerate(reqs):
                V[r, self.train_idx] = x
            ft = [job.tiles[0] for (job, _, _, _) in reqs]
            nt = [job.tiles[1] for (job, _, _, _) in reqs]
            sw = [float(job.n) for (job, _, _, _) in reqs]
            try:
                out = self.eng.pieces_multi(ft, nt, V, sw)
            except Exception as e:
                for (job, x, ev, slot) in reqs:
                    slot["error"] = repr(e)
                    ev.set()
                continue
            P = len(self.train)
            for r, (job, x, ev, slot) in enumerate(reqs):
                slot["nll"], slot["grad"] = combine_pieces(out[r], P)
                ev.set()
            self.batches.append((len(reqs), int(sum(nt)), time.perf_counter() - t0))

    # ------------------------------------------------------------ single
    def eval_alone(self, job, x):
        """One evaluation of one admitted job in a launch of its own."""
        V = self.base_vars.copy()
        V[self.train_idx] = x
        out = self.eng.pieces_multi([job.tiles[0]], [job.tiles[1]], V[None, :], [float(job.n)])
        return combine_pieces(out[0], len(self.train))


class NativeFitServer:
    """The same service with every fit's BFGS driver inside the native
    library (``pwa_server_*``): one scheduler thread evaluates the pending
    point of every active fit in one launch per round and advances each
    fit's BFGS state machine; Python only submits fits and reads results."""

    def __init__(self, config, mc, budget_bytes, max_active=256, tpb=128, gtol=1e-3,
                 maxiter=300):
        import ctypes

        from .engine import _dptr, load_library

        self.cl = config
        self.vm = config.vm
        self.eng = Engine(config.decay_group, config.plan, self.vm, tpb=tpb)
        c = self.eng.code
        x = mc.fields
        self._mc = (x[c.mass_fields].contiguous(), x[c.angle_fields].contiguous(),
                    torch.full((mc.n,), 1.0 / mc.n, dtype=torch.float64, device=x.device))
        xm, xa, wm = self._mc
        self.eng.upload_device(xm.data_ptr(), xa.data_ptr(), wm.data_ptr(), 0, mc.n, 0.0)
        torch.cuda.synchronize()
        vals = self.vm.get_all_dic()
        self.eng.set_gram(vals)
        consts = np.ascontiguousarray(self.eng.consts(vals))
        self.var_names = list(self.vm.variables.keys())
        self.train = list(self.vm.trainable_vars)
        base = np.ascontiguousarray([vals[k] for k in self.var_names], np.float64)
        self.eng.set_param_layout(self.var_names, self.train)
        self.tile_bytes = tpb * (8 * c.nf + 8)
        self.pool_tiles = max(1, int(budget_bytes // self.tile_bytes))
        self.eng.pool_reserve(self.pool_tiles)
        self._lib = load_library()
        self.h = ctypes.c_void_p()
        rc = self._lib.pwa_server_create(self.eng.h, _dptr(base), _dptr(consts), int(max_active),
                                         float(gtol), int(maxiter), ctypes.byref(self.h))
        if rc != 0:
            raise RuntimeError("pwa_server_create: " + self._lib.pwa_last_error(self.eng.h).decode())
        self._keep = {}
        self._dptr = _dptr

    def prepare(self, job):
        """The fit's mass/angle columns and weights as the device arrays the
        scheduler reads (done by submit when not done before)."""
        c = self.eng.code
        x = job.fields
        job.cols = (x[c.mass_fields].contiguous(), x[c.angle_fields].contiguous(),
                    torch.ones(job.n, dtype=torch.float64, device=x.device))
        return job

    def submit(self, job):
        import ctypes

        if getattr(job, "cols", None) is None:
            self.prepare(job)
            torch.cuda.synchronize()  # the columns exist before the scheduler reads them
        xm, xa, w = job.cols
        x0 = np.ascontiguousarray(job.x0, np.float64)
        fid = ctypes.c_longlong()
        rc = self._lib.pwa_server_submit(self.h, self._dptr(x0), xm.data_ptr(), xa.data_ptr(),
                                         w.data_ptr(), job.n, job.n, ctypes.byref(fid))
        if rc != 0:
            raise RuntimeError(f"pwa_server_submit failed ({rc})")
        job.sid = fid.value
        self._keep[job.sid] = job.cols
        job.cols = None
        return job

    def result(self, job, wait=True):
        """Fills job.result / n_eval / latency once the fit is final; returns
        True then (False while it runs, with wait=False)."""
        import ctypes

        P = len(self.train)
        st, ne, ni = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        nll, lat = ctypes.c_double(), ctypes.c_double()
        xo = np.zeros(P)
        rc = self._lib.pwa_server_result(self.h, job.sid, int(wait), ctypes.byref(st), self._dptr(xo),
                                         ctypes.byref(nll), ctypes.byref(ne), ctypes.byref(ni),
                                         ctypes.byref(lat))
        if rc != 0:
            raise RuntimeError(f"pwa_server_result failed ({rc})")
        if st.value == 0:
            return False
        job.n_eval = ne.value
        job.latency = lat.value
        job.result = {"x": xo, "nll": nll.value, "success": st.value == 1, "nit": ni.value}
        if st.value == 3:
            job.result["error"] = "failed"
        self._keep.pop(job.sid, None)
        return True

    def stats(self):
        import ctypes

        out = (ctypes.c_double * 5)()
        self._lib.pwa_server_stats(self.h, out)
        return {"rounds": int(out[0]), "requests": int(out[1]), "launch_s": out[2],
                "active": int(out[3]), "queued": int(out[4])}

    def tuning(self):
        """Block count per SM the service chose for its launches and the
        median seconds per work tile of each candidate."""
        import ctypes

        out = (ctypes.c_double * 9)()
        self._lib.pwa_server_tuning(self.h, out)
        return {"blocks_per_sm": int(out[0]),
                "candidates": {int(out[1 + 2 * c]): out[2 + 2 * c] for c in range(4)
                               if out[1 + 2 * c] > 0}}

    def close(self):
        if self.h:
            self._lib.pwa_server_destroy(self.h)
            self.h = None
        self.eng.close()


def serving_benchmark(n_fits=512, n_mc=1_000_000, n_min=1_000, n_max=1_000_000,
                      budget_gb=150.0, max_active=256, rate=None, seed=11, device="cuda",
                      config="d2kpipi.yml", maxiter=300, native=True):
    """Run the toy-fit service workload; returns a dict of measurements.

    Fits: event counts log-uniform in [n_min, n_max] (windows into one shared
    accept-reject sample of the model), starting couplings perturbed by
    N(0, 0.1) per fit, Poisson arrivals (``rate`` fits/s; by default chosen so
    that arrivals span about half of the expected run), shared MC sample.
    """
    from .workload import make_dataset

    cl, data, _, mc = make_dataset(config, n_max * 2, n_mc, seed=seed, device=device,
                                   precision="mixed")
    truth = np.array(cl.vm.get_all_val())
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_fits)).astype(np.int64)
    # admission is capped by the HBM budget; the pool itself is sized to the
    # smaller of the budget and every fit resident at once
    from .codegen import ModelCode

    nf = ModelCode(cl.decay_group, cl.plan).nf
    need = float(((sizes + 127) // 128).sum() * 128 * (8 * nf + 8)) * 1.05
    budget = min(budget_gb * 1e9, need)
    if native:
        server = NativeFitServer(cl, mc, budget, max_active=max_active, maxiter=maxiter)
    else:
        server = FitServer(cl, mc, budget, max_active=max_active)
    starts = rng.integers(0, data.n - sizes + 1)
    if rate is None:
        rate = n_fits / 5.0
    gaps = rng.exponential(1.0 / rate, n_fits)
    # the fits' toy data exist before the clock starts (as the toys of a study
    # would); the timed part is submission, service and results
    todo = []
    for i in range(n_fits):
        x0 = truth + rng.normal(0.0, 0.1, truth.shape)
        fields = data.fields[:, starts[i]:starts[i] + sizes[i]]
        job = FitJob(i, fields, x0, maxiter=maxiter)
        if native:
            server.prepare(job)
        todo.append(job)
    torch.cuda.synchronize()
    jobs = []
    t_start = time.perf_counter()
    t_next = t_start
    for i, job in enumerate(todo):
        t_next += gaps[i]
        while time.perf_counter() < t_next:
            time.sleep(min(0.001, max(0.0, t_next - time.perf_counter())))
        job.arrival = time.perf_counter()
        jobs.append(server.submit(job))
    if native:
        for j in jobs:
            server.result(j, wait=True)
        lat = np.array([j.latency for j in jobs])
        st = server.stats()
        rounds, reqs = st["rounds"], st["requests"]
        batch_info = {"batches": rounds, "mean_requests_per_batch": reqs / max(rounds, 1),
                      "launch_seconds": st["launch_s"], "tuning": server.tuning()}
    else:
        for j in jobs:
            j.done.wait()
        lat = np.array([j.finished - j.arrival for j in jobs])
        batches = np.array(server.batches) if server.batches else np.zeros((1, 3))
        batch_info = {"batches": len(server.batches),
                      "mean_requests_per_batch": float(batches[:, 0].mean()),
                      "max_requests_per_batch": int(batches[:, 0].max()),
                      "mean_batch_ms": 1e3 * float(batches[:, 2].mean())}
    t_total = time.perf_counter() - t_start
    evals = int(sum(j.n_eval for j in jobs))
    errors = [j.result.get("error") for j in jobs if "error" in j.result]
    converged = sum(1 for j in jobs if j.result.get("success"))
    out = {
        "driver": "native BFGS state machines" if native else "scipy BFGS, one thread per fit",
        "n_fits": n_fits, "evals": evals, "seconds": t_total, "evals_per_s": evals / t_total,
        "latency_p50_s": float(np.percentile(lat, 50)),
        "latency_p99_s": float(np.percentile(lat, 99)),
        "mean_evals_per_fit": evals / n_fits, "errors": len(errors), "converged": converged,
        "events_total": int(sizes.sum()), "pool_tiles": server.pool_tiles,
        "pool_gb": server.pool_tiles * server.tile_bytes / 1e9, "budget_gb": budget_gb,
    }
    out.update(batch_info)
    server.close()
    return out

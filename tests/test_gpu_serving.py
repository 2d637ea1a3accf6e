"""Serving: many concurrent fits, continuous batching (tf_pwa_b200.serving).

* A fit's evaluations, BFGS path and final result are bitwise identical when
  it runs alone and when it shares every launch with other fits.
* A single request through the multi-fit launch equals the one-fit cached
  path with the same per-warp column sums (same model, same events) within
  1e-10.
* Admission control: with a pool budget for about two fits, four submitted
  fits all finish and the pool never over-commits.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    from tf_pwa_b200.workload import make_dataset

    cl, data, _, mc = make_dataset("d2kpipi.yml", 60000, 30000, seed=21, precision="mixed")
    return cl, data, mc


def _jobs(cl, data, sizes, seed=3):
    from tf_pwa_b200.serving import FitJob

    rng = np.random.default_rng(seed)
    truth = np.array(cl.vm.get_all_val())
    jobs, off = [], 0
    for i, n in enumerate(sizes):
        x0 = truth + rng.normal(0, 0.1, truth.shape)
        jobs.append(FitJob(i, data.fields[:, off:off + n], x0, maxiter=200))
        off += n
    return jobs


def test_alone_equals_in_mix(setup):
    from tf_pwa_b200.serving import FitServer

    cl, data, mc = setup
    sizes = [20000, 3000, 9000, 15000]
    alone = _jobs(cl, data, sizes)[0]
    srv = FitServer(cl, mc, 1e9)
    srv.submit(alone).done.wait()
    srv.close()
    mixed = _jobs(cl, data, sizes)
    srv = FitServer(cl, mc, 1e9)
    for j in mixed:
        srv.submit(j)
    for j in mixed:
        j.done.wait()
    batched = max(b[0] for b in srv.batches)
    srv.close()
    assert batched > 1  # requests really shared launches
    a, m = alone, mixed[0]
    assert "error" not in a.result and "error" not in m.result
    assert a.n_eval == m.n_eval
    for (n1, g1), (n2, g2) in zip(a.trace, m.trace):
        assert n1 == n2 and np.array_equal(g1, g2)
    assert np.array_equal(a.result["x"], m.result["x"])


def test_multi_request_equals_cached_path(setup):
    from tf_pwa_b200.api import FCN, EventData
    from tf_pwa_b200.serving import FitServer

    cl, data, mc = setup
    job = _jobs(cl, data, [12000])[0]
    srv = FitServer(cl, mc, 1e9, run=False)
    srv.pending.append(job)
    srv._admit(start=False)
    x = job.x0
    nll_s, g_s = srv.eval_alone(job, x)
    srv.close()
    fcn = FCN(cl, EventData(job.fields, np.ones(job.n)), mc, precision="mixed")
    fcn.eng.set_cached_variant(2)  # same per-tile arithmetic as the multi-fit kernel
    nll_c, g_c = fcn.nll_grad(x)
    assert abs(nll_s - nll_c) <= 1e-10 * abs(nll_c)
    np.testing.assert_allclose(g_s, g_c, rtol=1e-8, atol=1e-8 * np.abs(g_c).max())
    fcn.eng.close()


def test_admission_under_budget(setup):
    from tf_pwa_b200.serving import FitServer

    cl, data, mc = setup
    sizes = [12000, 12000, 12000, 12000]
    jobs = _jobs(cl, data, sizes, seed=5)
    from tf_pwa_b200.codegen import ModelCode

    nf = ModelCode(cl.decay_group, cl.plan).nf
    tile_bytes = 128 * (8 * nf + 8)
    tiles_per_fit = (12000 + 127) // 128
    srv = FitServer(cl, mc, 2.5 * tiles_per_fit * tile_bytes)
    for j in jobs:
        srv.submit(j)
    peak = 0
    while not all(j.done.is_set() for j in jobs):
        with srv.lock:
            peak = max(peak, len(srv.active))
        jobs[0].done.wait(timeout=0.005)
    srv.close()
    assert peak <= 2
    assert all("error" not in j.result for j in jobs)
    # later fits waited for pool space
    assert jobs[3].admitted >= min(jobs[0].finished, jobs[1].finished)


def test_native_server_alone_equals_in_mix(setup):
    """Native server (BFGS state machines in the library): a fit's path and
    result are bitwise the same alone and mixed with other fits; all fits
    converge (max|g| < 1e-3, the reference fit's tolerance); the minimum
    equals the one scipy's BFGS finds on the same events through the
    reference-facing FCN (|dNLL| < 1e-8 relative)."""
    from tf_pwa_b200.api import FCN, EventData
    from tf_pwa_b200.serving import NativeFitServer

    cl, data, mc = setup
    sizes = [20000, 3000, 9000, 15000]
    alone = _jobs(cl, data, sizes)[0]
    srv = NativeFitServer(cl, mc, 1e9)
    srv.submit(alone)
    assert srv.result(alone, wait=True)
    srv.close()
    mixed = _jobs(cl, data, sizes)
    srv = NativeFitServer(cl, mc, 1e9)
    for j in mixed:
        srv.submit(j)
    for j in mixed:
        assert srv.result(j, wait=True)
    st = srv.stats()
    srv.close()
    assert st["requests"] > st["rounds"]  # requests shared launches
    a, m = alone, mixed[0]
    assert a.result["success"] and m.result["success"]
    assert a.n_eval == m.n_eval
    assert np.array_equal(a.result["x"], m.result["x"]) and a.result["nll"] == m.result["nll"]
    for j in mixed:
        assert j.result["success"], j.result
    # same minimum as scipy BFGS on the FCN of the same events
    j = mixed[0]
    fcn = FCN(cl, EventData(j.fields, np.ones(j.n)), mc, precision="mixed")
    from scipy.optimize import minimize

    r = minimize(lambda x: fcn.nll_grad(x), j.x0, jac=True, method="BFGS",
                 options={"gtol": 1e-3, "maxiter": 300})
    assert abs(r.fun - j.result["nll"]) <= 1e-8 * abs(r.fun)
    fcn.eng.close()


def test_native_server_admission_small_pool(setup):
    """With a pool for about two fits, four fits all finish (queued fits are
    admitted as others release their tiles)."""
    from tf_pwa_b200.serving import NativeFitServer

    cl, data, mc = setup
    jobs = _jobs(cl, data, [12000, 12000, 12000, 12000], seed=5)
    c_nf = 2 * 8 + 8
    srv = NativeFitServer(cl, mc, 2.2 * 12032 * c_nf)
    for j in jobs:
        srv.submit(j)
    for j in jobs:
        assert srv.result(j, wait=True)
        assert j.result["success"]
    srv.close()

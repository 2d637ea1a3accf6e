"""Fit fractions and their gradients with the MC sums taken from the
generated kernel code run on the host (tests/hostexec.py), against the
oracle: fractions within 1e-9 relative, gradients equal to central
differences of the oracle's fractions (h = 1e-6; 2e-6 of the largest
derivative, absolute floor 1e-9) for every trainable
parameter -- including identical-particle swaps, a polarised parent (its
density-matrix parameters), floating BWR2 / width_norm lineshapes and
CP-violating chain totals with per-event charges."""
import numpy as np
import pytest

from common import load_golden, load_model
from hostexec import HostModel


def _oracle_ff(m, group, vals, xm, res):
    tot = [c.params_head + "_total_0" for c in group]

    def integral(chains):
        v = dict(vals)
        for ci, t in enumerate(tot):
            if ci not in chains:
                for suf in ("r", "i", "deltar", "deltai"):
                    if t + suf in v:
                        v[t + suf] = 0.0
        return float(np.sum(m.pdf(xm, v)))

    sets = [{ci for ci, c in enumerate(group) if any(str(p) == r for p in c.inner)} for r in res]
    I_all = integral(set(range(len(group))))
    out = {}
    for i, r in enumerate(res):
        for j in range(i, -1, -1):
            if i == j:
                out[r] = integral(sets[i]) / I_all
            else:
                out[(res[i], res[j])] = (integral(sets[i] | sets[j]) / I_all
                                         - out[res[i]] - out[res[j]])
    return out


@pytest.mark.parametrize("name", ["lc2pkpi", "dp2kpipi_ident", "lc2pkpi_pol", "d2kpipi_shapes",
                                  "lc2pkpi_cp"])
def test_fit_fractions_host(name, tmp_path):
    from oracle.pwa_oracle import OracleModel
    from tf_pwa_b200.engine import PLAIN_F64, Engine
    from tf_pwa_b200.fitfractions import fit_fractions

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    vm.set_all(meta["variables"])
    eng = Engine(dc.decay_group, plan, vm, compile=False)
    hm = HostModel(eng.code, str(tmp_path))
    xm = g["fields_mc"]
    wm = np.ones(xm.shape[1]) / xm.shape[1]
    eng.eval_sums = lambda C, precision=PLAIN_F64, mc=True, stream=None: hm.sums(C, xm, wm, 0)
    res = sorted(str(p) for p in dc.decay_group.resonances)
    frac, _, grad = fit_fractions(eng, vm, res, use_gram=False)
    m = OracleModel(dc.decay_group, plan)
    vals = dict(meta["variables"])
    ref = _oracle_ff(m, dc.decay_group, vals, xm, res)
    assert set(frac) == set(ref)
    for k in ref:
        assert abs(frac[k] - ref[k]) <= 1e-9 * max(abs(ref[k]), 1e-3), (k, frac[k], ref[k])
    for pi, n in enumerate(vm.trainable_vars):
        h = 1e-6 * max(abs(vals[n]), 1.0)
        vp, vn = dict(vals), dict(vals)
        vp[n] += h
        vn[n] -= h
        fp, fn = _oracle_ff(m, dc.decay_group, vp, xm, res), _oracle_ff(m, dc.decay_group, vn, xm, res)
        for k in frac:
            fd = (fp[k] - fn[k]) / (2 * h)
            # relative to the fraction's largest derivative, with an absolute
            # floor at the differences' rounding level (~1e-16 / h)
            scale = max(np.abs(grad[k]).max(), 1e-8)
            assert abs(grad[k][pi] - fd) <= max(2e-6 * scale, 1e-9), (n, k, grad[k][pi], fd)

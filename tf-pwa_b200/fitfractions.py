"""Fit fractions and their errors (``tf_pwa/fitfractions.py:178-258``,
``tf_pwa/applications.py:29-67``).

FF_i = I(A restricted to the chains of resonance i) / I(A), the interference
term FF_ij = I(chains of i and j) / I(A) - FF_i - FF_j (i > j in the order
of ``res``), and their gradients with respect to the trainable parameters
for error propagation, err = sqrt(g^T V g) with V the inverse Hessian.  A
resonance selects the chains that contain it (``DecayGroup.set_used_res``,
``tf_pwa/amp/core.py:2031-2067``).

Two evaluations of the restricted integrals:

* masses and widths fixed, MC Gram matrix M cached: I_S = c_S^H M_SS c_S
  and dI_S/dtheta = 2 Re sum_k J_k (c_S^H M)_k over the columns of S -- a
  K x K contraction per subset, no pass over events;
* otherwise one FP64 MC pass per subset with the other chains' totals set
  to zero (the kernels' adjoint gives the coupling and lineshape
  sensitivities of the restricted amplitude).
"""
import numpy as np

from .engine import PLAIN_F64


def _total_names(group):
    return [c.params_head + "_total_0" for c in group]


def restricted_integral(eng, vals, names, chains, use_gram):
    """(I_S, dI_S/dnames) of the amplitude restricted to chain set ``chains``."""
    code = eng.code
    v = dict(vals)
    for ci, t in enumerate(_total_names(eng.group)):
        if ci not in chains:
            for suf in ("r", "i", "deltar", "deltai"):
                if t + suf in v:
                    v[t + suf] = 0.0
    C = eng.consts(v)
    J, D = eng.jacobian(v, names)
    used = np.array([ci in chains for ci, _ in code.columns])
    J[:, ~used] = 0.0
    if code.ncp and eng._Jm is not None:
        eng._Jm[:, ~used[eng._cp_cols]] = 0.0
    K = code.ncol
    if use_gram:
        ck = np.where(used, eng._ck, 0.0)
        Gm = np.conj(ck) @ eng._gram
        return float(np.real(Gm @ ck)), 2 * np.real(J @ Gm)
    _, sm = eng.eval_sums(C, PLAIN_F64, mc=True)
    return float(sm[0]), eng.grad_from_sums(J, D, sm)


def fit_fractions(eng, vm, res, inv_he=None, use_gram=None):
    """(frac, err_frac) with the reference's keys: str(res_i) and
    (str(res_i), str(res_j)) for i > j.  ``eng`` holds the MC sample
    (uploaded events; with ``use_gram`` its Gram matrix at the current
    masses and widths).  Errors are given when ``inv_he`` is."""
    vals = vm.get_all_dic()
    names = list(vm.trainable_vars)
    if use_gram is None:
        use_gram = eng._gram is not None and not any(
            n.endswith(("_mass", "_width")) for n in names)
    group = eng.group
    chains_of = []
    for r in res:
        cs = {ci for ci, c in enumerate(group) if any(str(p) == str(r) for p in c.inner)}
        chains_of.append(cs)
    I_all, g_all = restricted_integral(eng, vals, names, set(range(len(group))), use_gram)
    frac, grad = {}, {}
    for i, r in enumerate(res):
        for j in range(i, -1, -1):
            if i == j:
                name = str(r)
                I_s, g_s = restricted_integral(eng, vals, names, chains_of[i], use_gram)
            else:
                name = (str(res[i]), str(res[j]))
                I_s, g_s = restricted_integral(eng, vals, names, chains_of[i] | chains_of[j],
                                               use_gram)
            f = I_s / I_all
            g = g_s / I_all - f * g_all / I_all
            if i != j:
                f = f - frac[str(res[i])] - frac[str(res[j])]
                g = g - grad[str(res[i])] - grad[str(res[j])]
            frac[name] = f
            grad[name] = g
    eng.consts(vals)  # restore the engine's couplings
    err = {}
    if inv_he is not None:
        for k, g in grad.items():
            err[k] = float(np.sqrt(np.dot(np.dot(inv_he, g), g)))
    return frac, err, grad

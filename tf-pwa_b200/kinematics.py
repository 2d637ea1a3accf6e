"""Dataset kinematics: final-state four-momenta -> the engine's event fields.

Runs once per dataset (the reference does this at load time too,
``tf_pwa/config_loader/data.py:232-251``); the per-evaluation hot path only
reads its output.  Restates ``tf_pwa/cal_angle.py`` for two-body decay
chains with the reference's default options (no centre-of-mass boost,
fixed lab z axis, SU(2) alignment with final-state boosts):

* node momenta and invariant masses: ``cal_angle.py:158-182``
* successive rest-frame momenta along a chain: ``cal_angle.py:193-251``
* helicity angles, alpha range bias per out, SU(2) rotation/boost bookkeeping:
  ``cal_angle.py:262-343`` with ``angle.py`` (``EulerAngle.angle_zx_z_getx``,
  ``Vector3.cross_unit``, ``LorentzVector.rest_vector``, ``SU2M``)
* alignment angles, rule 1 (reference chain = where the final particle is a
  direct daughter of the top): ``cal_angle.py:346-378,408-490``

Array work is written with torch tensor operations so the same code runs on
the host or, for large datasets, on the GPU (float64 throughout).
"""
import math

import numpy as np
import torch

from .plan import split_swap

_EPS = 1e-14


# ------------------------------------------------------------- vectors
def _unit(v):
    return v / torch.linalg.vector_norm(v, dim=-1, keepdim=True)


def _cross_unit(a, b):
    c = torch.linalg.cross(a, b, dim=-1)
    n = torch.linalg.vector_norm(c, dim=-1, keepdim=True)
    mask = n < _EPS
    if bool(mask.any()):
        c = torch.where(mask, torch.linalg.cross(a, b + 1.0, dim=-1), c)
    return _unit(c)


def _angle_from(v, x, y):
    return torch.atan2(torch.sum(v * y, -1), torch.sum(v * x, -1))


def angle_zx_z_getx(z1, x1, z2):
    """Euler angles (alpha, beta; gamma = 0) taking frame (z1, x1) to z2 and
    the new x axis (``angle.py`` EulerAngle.angle_zx_z_getx)."""
    u_z1 = _unit(z1)
    u_z2 = _unit(z2)
    u_y1 = _cross_unit(z1, x1)
    u_x1 = _cross_unit(u_y1, z1)
    u_yr = _cross_unit(z1, z2)
    u_xr = _cross_unit(u_yr, z1)
    alpha = _angle_from(u_xr, u_x1, u_y1)
    beta = _angle_from(u_z2, u_z1, u_xr)
    u_x2 = _cross_unit(u_yr, u_z2)
    return alpha, beta, u_x2


def rest_vector(p, other):
    """``other`` boosted into the rest frame of ``p`` (4-vectors (N,4))."""
    pb = -p[:, 1:] / p[:, :1]
    beta2 = torch.sum(pb * pb, -1)
    gamma = 1.0 / torch.sqrt(1 - beta2)
    v = other[:, 1:]
    bp = torch.sum(pb * v, -1)
    safe = torch.where(beta2 > _EPS, beta2, torch.ones_like(beta2))
    gamma2 = torch.where(beta2 > _EPS, (gamma - 1.0) / safe, torch.zeros_like(beta2))
    pr = v + (gamma2 * bp)[:, None] * pb + (gamma * other[:, 0])[:, None] * pb
    T = gamma * (other[:, 0] + bp)
    return torch.cat([T[:, None], pr], -1)


def inv_mass(p):
    m2 = p[:, 0] ** 2 - torch.sum(p[:, 1:] ** 2, -1)
    return torch.sqrt(torch.abs(m2))


# ------------------------------------------------------------- SU(2)
def _c(x):
    return torch.complex(x, torch.zeros_like(x))


def su2_rot_z(a):
    e = torch.polar(torch.ones_like(a), 0.5 * a)
    z = torch.zeros_like(e)
    return torch.stack([torch.stack([1 / e, z], -1), torch.stack([z, e], -1)], -2)


def su2_rot_y(b):
    s = _c(torch.sin(b / 2))
    c = _c(torch.cos(b / 2))
    return torch.stack([torch.stack([c, -s], -1), torch.stack([s, c], -1)], -2)


def su2_boost_z_from_p(p):
    pb = p[:, 1:] / p[:, :1]
    beta2 = torch.sum(pb * pb, -1)
    beta2 = torch.where(beta2 < 1, beta2, torch.zeros_like(beta2))
    omega = torch.acosh(1.0 / torch.sqrt(1 - beta2))
    a = _c(torch.exp(omega / 2))
    z = torch.zeros_like(a)
    return torch.stack([torch.stack([1 / a, z], -1), torch.stack([z, a], -1)], -2)


def su2_inv(x):
    return torch.stack([torch.stack([x[:, 1, 1], -x[:, 0, 1]], -1),
                        torch.stack([-x[:, 1, 0], x[:, 0, 0]], -1)], -2)


def su2_euler(x):
    cosb = torch.clamp(torch.real(x[:, 0, 0] * x[:, 1, 1] + x[:, 0, 1] * x[:, 1, 0]), -1, 1)
    beta = torch.arccos(cosb)
    apg = torch.angle(x[:, 1, 1])
    amg = -torch.angle(x[:, 1, 0])
    return apg + amg, beta, apg - amg


# ------------------------------------------------------------- chains
def _chain_frames(chain_topo, mom, random_z=False):
    """Helicity angles of every out of every decay, and per final particle
    the SU(2) rotation and boost accumulated along the chain.  With
    ``random_z`` a moving parent's flight direction is the z axis of its
    decay (``tf_pwa/cal_angle.py:431-438``)."""
    chain = chain_topo.chain
    top = chain.top
    # successive rest-frame momenta (cal_chain_boost)
    part = {}
    core_map = {}
    decays = list(chain)
    remaining = set(chain.inner) | set(chain.outs)
    while decays:
        later = []
        for d in decays:
            if d.core == top:
                pr = mom[top]
                rp = {}
                for j in d.outs:
                    core_map[j] = d
                    rp[j] = rest_vector(pr, mom[j])
                    remaining.discard(j)
                for j in remaining:
                    rp[j] = rest_vector(pr, mom[j])
                part[d] = rp
            elif d.core in core_map:
                par = part[core_map[d.core]]
                pr = par[d.core]
                rp = {}
                for j in d.outs:
                    core_map[j] = d
                    rp[j] = rest_vector(pr, par[j])
                    remaining.discard(j)
                for j in remaining:
                    if j in par:
                        rp[j] = rest_vector(pr, par[j])
                part[d] = rp
            else:
                later.append(d)
        decays = later
    n = mom[top].shape[0]
    dev = mom[top].device
    set_x = {top: torch.tensor([1.0, 0.0, 0.0], dtype=torch.float64, device=dev).expand(n, 3)}
    set_z = {top: torch.tensor([0.0, 0.0, 1.0], dtype=torch.float64, device=dev).expand(n, 3)}
    if random_z:
        p3 = mom[top][:, 1:]
        moving = (torch.linalg.norm(p3, dim=1) >= 1e-5)[:, None]
        set_z[top] = torch.where(moving, p3, set_z[top])
    angles = {}
    rmat, bmat = {}, {}
    decays = list(chain)
    while decays:
        later = []
        for d in decays:
            if d.core not in set_x:
                later.append(d)
                continue
            bias = -math.pi
            for j in d.outs:
                p_rest = part[d][j]
                z2 = p_rest[:, 1:]
                alpha, beta, x2 = angle_zx_z_getx(set_z[d.core], set_x[d.core], z2)
                set_x[j] = x2
                set_z[j] = z2
                alpha = torch.remainder(alpha - bias, 2 * math.pi) + bias
                bias -= math.pi
                angles[(d, j)] = (alpha, beta)
                bmat[j] = su2_boost_z_from_p(p_rest)
                r = su2_rot_y(beta) @ su2_rot_z(alpha)
                if d.core in rmat:
                    rmat[j] = r @ bmat[d.core] @ rmat[d.core]
                else:
                    rmat[j] = r
        decays = later
    return angles, rmat, bmat


def event_fields(plan, p4, device=None, charge=None):
    """(n_fields, N) FP64 event columns in plan order from final-state
    momenta ``p4`` = {final particle name: (N, 4) array or tensor} in the
    parent rest frame.  Returns a tensor on ``device`` (default: the input's
    device, CPU for numpy input).  For data with charges, ``charge``
    (default all +1) fills the charge field, or with cp_trans parity-
    transforms the charge < 0 events first."""
    p4 = {k: torch.as_tensor(v, dtype=torch.float64, device=device) for k, v in p4.items()}
    n = next(iter(p4.values())).shape[0]
    dev = next(iter(p4.values())).device
    out = torch.zeros((plan.n_fields, n), dtype=torch.float64, device=dev)
    if plan.use_charge:
        ch = torch.ones(n, dtype=torch.float64, device=dev) if charge is None else \
            torch.as_tensor(charge, dtype=torch.float64, device=dev)
        if plan.charge_index is not None:
            out[plan.charge_index] = ch
        if plan.cp_trans:
            sgn = torch.where(ch > 0, 1.0, -1.0).to(torch.float64)[:, None]
            p4 = {k: torch.cat([v[:, :1], v[:, 1:] * sgn], 1) for k, v in p4.items()}

    def topo_frames(mom4):
        frames = []
        for tidx, topo in enumerate(plan.topos):
            chain = topo.chain
            mom = {}
            for o in chain.outs:
                mom[o] = mom4[str(o)]
            for p in chain.inner:
                mom[p] = sum(mom[f] for f in chain.final_set(p))
            mom[chain.top] = sum(mom[f] for f in chain.outs)
            angles, rmat, bmat = _chain_frames(topo, mom, plan.random_z)
            frames.append((topo, angles, rmat, bmat, mom))
        return frames

    # unswapped momenta, then one relabelling per swap (final pi takes the
    # momentum of src[pi], three-momentum reversed in the CP-conjugate ones)
    def neg(v):
        return torch.cat([v[:, :1], -v[:, 1:]], 1)

    all_frames = [topo_frames(p4)]
    for sw in plan.swaps:
        moved = {k: p4[sw["src"].get(k, k)] for k in p4}
        if sw["neg"]:
            moved = {k: neg(v) for k, v in moved.items()}
        all_frames.append(topo_frames(moved))
    for fi, full_name in enumerate(plan.fields):
        if fi == plan.charge_index:
            continue
        sk, fname = split_swap(full_name)
        frames = all_frames[sk]
        parts = fname.split("/")
        if parts[0] == "m":
            for topo, angles, rmat, bmat, mom in frames:
                for p in topo.chain.inner:
                    if topo.node[p] == parts[1]:
                        out[fi] = inv_mass(mom[p])
                        break
                else:
                    continue
                break
            continue
        tidx = int(parts[0])
        topo, angles, rmat, bmat, mom = frames[tidx]
        # locate decay and particle by their standard names
        dec = [d for d in topo.chain if topo.decay_name(d) == parts[1]][0]
        part = [o for o in dec.outs if topo.node[o] == parts[2]][0]
        if parts[3] == "aligned":
            ref_t = plan.align_ref[str(part)]
            rtopo, _, rr, rb, _ = frames[ref_t]
            rpart = [o for o in rtopo.chain.outs if str(o) == str(part)][0]
            R = rr[rpart] @ su2_inv(rmat[part])
            R = rb[rpart] @ R @ su2_inv(bmat[part])
            a, b, g = su2_euler(R)
            out[fi] = {"alpha": a, "beta": b, "gamma": g}[parts[4]]
        else:
            a, b = angles[(dec, part)]
            out[fi] = a if parts[3] == "alpha" else b
    return out


def p4_dict(arr, order):
    """(N, n_final, 4) momenta in ``order`` -> {name: (N, 4)}."""
    return {name: arr[:, i, :] for i, name in enumerate(order)}

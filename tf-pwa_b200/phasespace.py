"""Flat n-body phase-space generator (seeded numpy), the input side of toy
and MC generation.

Same role as ``tf_pwa/phasespace.py:31-254`` (``PhaseSpaceGenerator`` /
``generate_phsp``): momenta of the final particles in the parent rest frame,
distributed uniformly in Lorentz-invariant phase space.  Uses the standard
Raubold-Lynch (GENBOD) construction -- sorted uniform numbers give the
intermediate invariant masses, each two-body splitting is isotropic, and the
product of two-body momenta is the event weight, removed by accept-reject.
The random stream is numpy's (the reference draws from TensorFlow's), so
events are not bit-identical to the reference's for the same seed.
"""
import numpy as np


def _pdk(a, b, c):
    x = (a - b - c) * (a + b + c) * (a - b + c) * (a + b - c)
    return np.sqrt(np.maximum(x, 0.0)) / (2 * a)


def _rotate(p, cth, phi):
    """Rotate 3-vectors p (N,3) whose frame has z along the splitting axis."""
    sth = np.sqrt(np.maximum(1 - cth * cth, 0))
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    # rotation taking z-hat to (sth cos phi, sth sin phi, cth)
    cp, sp = np.cos(phi), np.sin(phi)
    nx = cth * cp * x - sp * y + sth * cp * z
    ny = cth * sp * x + cp * y + sth * sp * z
    nz = -sth * x + cth * z
    return np.stack([nx, ny, nz], -1)


def _boost(p4, beta):
    """Boost 4-vectors p4 (N,4) by velocity beta (N,3)."""
    b2 = np.sum(beta * beta, -1)
    g = 1.0 / np.sqrt(1 - b2)
    bp = np.sum(beta * p4[:, 1:], -1)
    g2 = np.where(b2 > 0, (g - 1) / np.where(b2 > 0, b2, 1), 0.0)
    E = g * (p4[:, 0] + bp)
    v = p4[:, 1:] + (g2 * bp + g * p4[:, 0])[:, None] * beta
    return np.concatenate([E[:, None], v], -1)


def generate_weighted(M, masses, n, rng):
    """n weighted events: list of (n,4) momenta and the weights (max-normalised
    by the analytic upper bound)."""
    masses = list(masses)
    k = len(masses)
    tm = M - sum(masses)
    assert tm > 0, "parent below threshold"
    r = np.sort(rng.random((n, k - 2)), axis=1) if k > 2 else np.zeros((n, 0))
    cum = np.cumsum(masses)
    # invariant masses M_1 = m_1 < M_2 < ... < M_k = M of the first i particles
    Ms = [np.full(n, masses[0])]
    for i in range(1, k - 1):
        Ms.append(r[:, i - 1] * tm + cum[i])
    Ms.append(np.full(n, M))
    w = np.ones(n)
    pd = []
    for i in range(1, k):
        q = _pdk(Ms[i], Ms[i - 1], masses[i])
        pd.append(q)
        w *= q
    # maximum weight bound (GENBOD)
    emmax = tm + masses[0]
    emmin = 0.0
    wtmax = 1.0
    for i in range(1, k):
        emmin += masses[i - 1]
        emmax += masses[i]
        wtmax *= _pdk(emmax, emmin, masses[i])
    # build momenta, starting with particle 0 and 1 in the M_2 frame
    ps = [None] * k
    cth = 2 * rng.random(n) - 1
    phi = 2 * np.pi * rng.random(n)
    q = pd[0]
    dirv = _rotate(np.tile([0.0, 0.0, 1.0], (n, 1)), cth, phi)
    p3 = q[:, None] * dirv
    ps[0] = np.concatenate([np.sqrt(q * q + masses[0] ** 2)[:, None], -p3], -1)
    ps[1] = np.concatenate([np.sqrt(q * q + masses[1] ** 2)[:, None], p3], -1)
    for i in range(2, k):
        q = pd[i - 1]
        cth = 2 * rng.random(n) - 1
        phi = 2 * np.pi * rng.random(n)
        dirv = _rotate(np.tile([0.0, 0.0, 1.0], (n, 1)), cth, phi)
        p3 = q[:, None] * dirv
        # system of the first i particles recoils against particle i
        Esys = np.sqrt(q * q + Ms[i - 1] ** 2)
        beta = -p3 / Esys[:, None]
        for j in range(i):
            ps[j] = _boost(ps[j], beta)
        ps[i] = np.concatenate([np.sqrt(q * q + masses[i] ** 2)[:, None], p3], -1)
    return ps, w / wtmax


def generate_phsp(M, masses, n, seed=None, rng=None):
    """n unweighted flat phase-space events; list of (n,4) arrays, one per
    final particle, in the parent rest frame."""
    rng = rng if rng is not None else np.random.default_rng(seed)
    out = [[] for _ in masses]
    have = 0
    while have < n:
        m = max(2 * (n - have), 1024)
        ps, w = generate_weighted(M, masses, m, rng)
        keep = rng.random(m) < w
        for i, p in enumerate(ps):
            out[i].append(p[keep])
        have += int(keep.sum())
    return [np.concatenate(o)[:n] for o in out]

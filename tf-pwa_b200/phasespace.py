"""Flat n-body phase-space generator (seeded), the input side of toy and MC
generation.

Same role as ``tf_pwa/phasespace.py:31-254`` (``PhaseSpaceGenerator`` /
``generate_phsp``): momenta of the final particles in the parent rest frame,
distributed uniformly in Lorentz-invariant phase space.  Uses the standard
Raubold-Lynch (GENBOD) construction -- sorted uniform numbers give the
intermediate invariant masses, each two-body splitting is isotropic, and the
product of two-body momenta is the event weight, removed by accept-reject.
Tensor operations run on the host or the GPU (float64).  The random stream is
torch's (the reference draws from TensorFlow's), so events are not
bit-identical to the reference's for the same seed.
"""
import numpy as np
import torch


def _pdk(a, b, c):
    x = (a - b - c) * (a + b + c) * (a - b + c) * (a + b - c)
    return torch.sqrt(torch.clamp(x, min=0.0)) / (2 * a)


def _pdk_f(a, b, c):
    x = (a - b - c) * (a + b + c) * (a - b + c) * (a + b - c)
    return float(np.sqrt(max(x, 0.0)) / (2 * a))


def _direction(cth, phi):
    sth = torch.sqrt(torch.clamp(1 - cth * cth, min=0.0))
    return torch.stack([sth * torch.cos(phi), sth * torch.sin(phi), cth], -1)


def _boost(p4, beta):
    """Boost 4-vectors p4 (N,4) by velocity beta (N,3)."""
    b2 = torch.sum(beta * beta, -1)
    g = 1.0 / torch.sqrt(1 - b2)
    bp = torch.sum(beta * p4[:, 1:], -1)
    safe = torch.where(b2 > 0, b2, torch.ones_like(b2))
    g2 = torch.where(b2 > 0, (g - 1) / safe, torch.zeros_like(b2))
    E = g * (p4[:, 0] + bp)
    v = p4[:, 1:] + (g2 * bp + g * p4[:, 0])[:, None] * beta
    return torch.cat([E[:, None], v], -1)


def generate_weighted(M, masses, n, gen, device="cpu"):
    """n weighted events: list of (n,4) momenta and the weights normalised by
    the GENBOD upper bound (so weights are in [0, 1])."""
    masses = [float(m) for m in masses]
    k = len(masses)
    tm = M - sum(masses)
    assert tm > 0, "parent below threshold"
    opts = dict(dtype=torch.float64, device=device)
    if k > 2:
        r = torch.sort(torch.rand((n, k - 2), generator=gen, **opts), dim=1).values
    cum = np.cumsum(masses)
    Ms = [torch.full((n,), masses[0], **opts)]
    for i in range(1, k - 1):
        Ms.append(r[:, i - 1] * tm + float(cum[i]))
    Ms.append(torch.full((n,), float(M), **opts))
    w = torch.ones(n, **opts)
    pd = []
    for i in range(1, k):
        q = _pdk(Ms[i], Ms[i - 1], masses[i])
        pd.append(q)
        w = w * q
    emmax = tm + masses[0]
    emmin = 0.0
    wtmax = 1.0
    for i in range(1, k):
        emmin += masses[i - 1]
        emmax += masses[i]
        wtmax *= _pdk_f(emmax, emmin, masses[i])
    ps = [None] * k
    cth = 2 * torch.rand(n, generator=gen, **opts) - 1
    phi = 2 * np.pi * torch.rand(n, generator=gen, **opts)
    q = pd[0]
    p3 = q[:, None] * _direction(cth, phi)
    ps[0] = torch.cat([torch.sqrt(q * q + masses[0] ** 2)[:, None], -p3], -1)
    ps[1] = torch.cat([torch.sqrt(q * q + masses[1] ** 2)[:, None], p3], -1)
    for i in range(2, k):
        q = pd[i - 1]
        cth = 2 * torch.rand(n, generator=gen, **opts) - 1
        phi = 2 * np.pi * torch.rand(n, generator=gen, **opts)
        p3 = q[:, None] * _direction(cth, phi)
        # the system of the first i particles recoils against particle i
        Esys = torch.sqrt(q * q + Ms[i - 1] ** 2)
        beta = -p3 / Esys[:, None]
        for j in range(i):
            ps[j] = _boost(ps[j], beta)
        ps[i] = torch.cat([torch.sqrt(q * q + masses[i] ** 2)[:, None], p3], -1)
    return ps, w / wtmax


def generate_phsp(M, masses, n, seed=None, gen=None, device="cpu", as_numpy=True):
    """n unweighted flat phase-space events: list of (n,4) arrays (one per
    final particle) in the parent rest frame."""
    if gen is None:
        gen = torch.Generator(device=device)
        gen.manual_seed(0 if seed is None else int(seed))
    out = [[] for _ in masses]
    have = 0
    while have < n:
        m = max(2 * (n - have), 1024)
        ps, w = generate_weighted(M, masses, m, gen, device)
        keep = torch.rand(m, generator=gen, dtype=torch.float64, device=device) < w
        for i, p in enumerate(ps):
            out[i].append(p[keep])
        have += int(keep.sum())
    res = [torch.cat(o)[:n] for o in out]
    if as_numpy:
        return [r.cpu().numpy() for r in res]
    return res

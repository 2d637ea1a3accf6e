"""CPU oracle of the device toy / phase-space generator (numpy).

TEST INFRASTRUCTURE ONLY.  Tests and ``__graft_entry__.smoke()`` may import
it as the checker of ``pwa_toy_select`` / ``pwa_toy_fields``; the product
path never does.

The generator's specification, restated on the host:

* random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel
  random numbers: as easy as 1, 2, 3", SC'11), counter = (event number low
  32 bits, high 32 bits, draw pair j, 0), key = seed (low, high 32 bits);
  each call gives two 53-bit uniforms (a >> 5, b >> 6) / 2^53;
* draws of an event, level by level (the parent, then each fixed-mass
  intermediate): k - 2 sorted uniforms for the intermediate masses of a
  k-body level, (cos theta, phi) per two-body splitting; then the
  phase-space accept draw and the amplitude accept draw;
* flat phase space by the Raubold-Lynch (GENBOD) construction that the
  reference's generator also uses (``tf_pwa/phasespace.py:31-254``), with
  fixed-mass intermediates decayed on shell in their rest frame and boosted
  (its chain generator, ``tf_pwa/phasespace.py:256-368``), kept with
  probability = product of the levels' weight / max weight;
* signal by accept-reject on sum |A|^2 against u * fmax
  (``tf_pwa/applications.py:428-453``).
"""
import math

import numpy as np

M32 = 0xFFFFFFFF


def philox4x32_10(ctr, key):
    """One Philox4x32-10 block: ctr = 4 ints, key = 2 ints -> 4 ints."""
    c0, c1, c2, c3 = (int(x) & M32 for x in ctr)
    k0, k1 = (int(x) & M32 for x in key)
    for r in range(10):
        if r:
            k0 = (k0 + 0x9E3779B9) & M32
            k1 = (k1 + 0xBB67AE85) & M32
        p0 = 0xD2511F53 * c0
        p1 = 0xCD9E8D57 * c2
        hi0, lo0 = p0 >> 32, p0 & M32
        hi1, lo1 = p1 >> 32, p1 & M32
        c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
    return c0, c1, c2, c3


def philox_vec(ctr, key):
    """Vectorised Philox4x32-10: ctr (4, N) uint64 arrays, key (2,) ints."""
    c0, c1, c2, c3 = (np.asarray(x, np.uint64) & np.uint64(M32) for x in ctr)
    k0, k1 = np.uint64(int(key[0]) & M32), np.uint64(int(key[1]) & M32)
    m0, m1, m32 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57), np.uint64(M32)
    for r in range(10):
        if r:
            k0 = (k0 + np.uint64(0x9E3779B9)) & m32
            k1 = (k1 + np.uint64(0xBB67AE85)) & m32
        p0 = m0 * c0
        p1 = m1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & m32
        hi1, lo1 = p1 >> np.uint64(32), p1 & m32
        c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
    return c0, c1, c2, c3


def uniforms(seed, events, ndraw):
    """(ndraw, N) uniform doubles of event numbers ``events``."""
    ev = np.asarray(events, np.uint64)
    key = (int(seed) & M32, (int(seed) >> 32) & M32)
    out = np.empty((ndraw, len(ev)))
    for j in range((ndraw + 1) // 2):
        ctr = (ev & np.uint64(M32), ev >> np.uint64(32), np.full(len(ev), j, np.uint64),
               np.zeros(len(ev), np.uint64))
        a, b, c, d = philox_vec(ctr, key)
        out[2 * j] = ((a >> np.uint64(5)).astype(np.float64) * 67108864.0
                      + (b >> np.uint64(6)).astype(np.float64)) / 9007199254740992.0
        if 2 * j + 1 < ndraw:
            out[2 * j + 1] = ((c >> np.uint64(5)).astype(np.float64) * 67108864.0
                              + (d >> np.uint64(6)).astype(np.float64)) / 9007199254740992.0
    return out


def _pdk(a, b, c):
    x = (a - b - c) * (a + b + c) * (a - b + c) * (a + b - c)
    return np.sqrt(np.maximum(x, 0.0)) / (2 * a)


def _boost(p, beta):
    b2 = np.sum(beta * beta, 0)
    g = 1.0 / np.sqrt(1 - b2)
    bp = np.sum(beta * p[1:], 0)
    g2 = np.where(b2 > 0, (g - 1) / np.where(b2 > 0, b2, 1.0), 0.0)
    s = g2 * bp + g * p[0]
    return np.concatenate([(g * (p[0] + bp))[None], p[1:] + s * beta], 0)


def _level(U, draw, M, ms):
    """One GENBOD level: body momenta (k, 4, N) in the level's rest frame,
    weight over its upper bound, next draw index."""
    k = len(ms)
    n = U.shape[1]
    tm = M - sum(ms)
    cum = np.cumsum(ms)
    r = np.sort(U[draw:draw + k - 2], axis=0) if k > 2 else np.zeros((0, n))
    draw += k - 2
    Ms = [np.full(n, ms[0])] + [r[i - 1] * tm + cum[i] for i in range(1, k - 1)] + [np.full(n, M)]
    pd = [_pdk(Ms[i], Ms[i - 1], ms[i]) for i in range(1, k)]
    w = np.prod(pd, 0)
    emmax, emmin, wtmax = tm + ms[0], 0.0, 1.0
    for i in range(1, k):
        emmin += ms[i - 1]
        emmax += ms[i]
        wtmax *= float(_pdk(np.float64(emmax), emmin, ms[i]))
    ps = [None] * k
    for i in range(1, k):
        cth = 2.0 * U[draw] - 1.0
        phi = 2 * math.pi * U[draw + 1]
        draw += 2
        sth = np.sqrt(np.maximum(1.0 - cth * cth, 0.0))
        q = pd[i - 1]
        p3 = np.stack([q * sth * np.cos(phi), q * sth * np.sin(phi), q * cth])
        if i == 1:
            ps[0] = np.concatenate([np.sqrt(q * q + ms[0] ** 2)[None], -p3])
            ps[1] = np.concatenate([np.sqrt(q * q + ms[1] ** 2)[None], p3])
        else:
            esys = np.sqrt(q * q + Ms[i - 1] ** 2)
            beta = -p3 / esys
            for j in range(i):
                ps[j] = _boost(ps[j], beta)
            ps[i] = np.concatenate([np.sqrt(q * q + ms[i] ** 2)[None], p3])
    return ps, w / wtmax, draw


def genbod_levels(U, levels, nfin):
    """Momenta (nfin, 4, N) and weight / max weight of a chain of GENBOD
    levels: levels[0] = (parent mass, bodies), bodies = (kind, ref, mass)
    with kind "f" (ref = final index) or "n" (ref = level decayed on shell in
    its rest frame and boosted with the body's velocity)."""
    draw = 0
    w = np.ones(U.shape[1])
    gen = []
    for M, bodies in levels:
        ps, wl, draw = _level(U, draw, M, [m for _, _, m in bodies])
        gen.append(ps)
        w = w * wl
    out = [None] * nfin

    def place(lid, frame):
        for j, (kind, ref, _) in enumerate(levels[lid][1]):
            p = gen[lid][j]
            if frame is not None:
                p = _boost(p, frame[1:] / frame[0])
            if kind == "f":
                out[ref] = p
            else:
                place(ref, p)

    place(0, None)
    return np.stack(out), w


def genbod(U, M, masses):
    """Single-level GENBOD: momenta (n_final, 4, N) and weight / max weight."""
    return genbod_levels(U, [(M, [("f", i, m) for i, m in enumerate(masses)])], len(masses))


def select(seed, first, n, levels, nfin, pdf=None, fmax=0.0):
    """Oracle of pwa_toy_select: per candidate sum |A|^2 (or 1 when flat)
    if kept, else -1.  ``pdf(p4)`` maps momenta (N, n_final, 4) to sum |A|^2."""
    ndraw = sum(3 * len(b) - 4 for _, b in levels) + 2
    U = uniforms(seed, np.arange(first, first + n), ndraw)
    p, wps = genbod_levels(U, levels, nfin)
    keep = U[ndraw - 2] < wps
    out = np.full(n, -1.0)
    if pdf is None:
        out[keep] = 1.0
        return out, p
    f = np.zeros(n)
    f[keep] = pdf(np.transpose(p[:, :, keep], (2, 0, 1)))
    if fmax > 0:
        keep &= U[ndraw - 1] * fmax < f
    out[keep] = f[keep]
    return out, p

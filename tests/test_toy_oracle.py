"""Generator oracle (CPU): Philox4x32-10 against the published known-answer
vectors, GENBOD events conserve four-momentum and put every final on its
mass shell, and its flat phase space agrees in distribution with the host
generator (``phasespace.generate_phsp``)."""
import numpy as np
import pytest

from oracle.toy_oracle import genbod, philox4x32_10, uniforms


@pytest.mark.parametrize("ctr,key,expect", [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
])
def test_philox_known_answers(ctr, key, expect):
    assert philox4x32_10(ctr, key) == expect


def test_uniforms_range_and_independence():
    u = uniforms(12345, np.arange(20000), 7)
    assert u.min() >= 0 and u.max() < 1
    assert abs(u.mean() - 0.5) < 0.01
    c = np.corrcoef(u)
    assert np.max(np.abs(c - np.eye(7))) < 0.03


@pytest.mark.parametrize("M,masses", [(2.28646, [0.938272, 0.493677, 0.13957]),
                                      (5.279, [1.865, 0.135, 0.4937, 0.1396])])
def test_genbod_conservation(M, masses):
    k = len(masses)
    U = uniforms(7, np.arange(5000), 3 * k - 2)
    p, w = genbod(U, M, masses)
    tot = p.sum(0)
    np.testing.assert_allclose(tot[0], M, rtol=1e-12)
    np.testing.assert_allclose(tot[1:], 0, atol=1e-12)
    m2 = p[:, 0] ** 2 - np.sum(p[:, 1:] ** 2, 1)
    np.testing.assert_allclose(m2, np.broadcast_to(np.array(masses)[:, None] ** 2, m2.shape),
                               rtol=0, atol=1e-11)
    assert np.all((w >= 0) & (w <= 1 + 1e-12))


def test_flat_phase_space_matches_host_generator():
    """Two-sample comparison of the invariant-mass distributions of the
    oracle's accepted events and the host generator's (5 sigma on the
    first two moments of m^2_12 and m^2_23)."""
    from tf_pwa_b200.phasespace import generate_phsp

    M, masses = 5.279, [1.865, 0.135, 0.4937, 0.1396]
    U = uniforms(99, np.arange(200000), 10)
    p, w = genbod(U, M, masses)
    keep = U[8] < w
    a = np.transpose(p[:, :, keep], (2, 0, 1))
    b = np.stack(generate_phsp(M, masses, a.shape[0], seed=5), 1)

    def m2(x, i, j):
        s = x[:, i] + x[:, j]
        return s[:, 0] ** 2 - np.sum(s[:, 1:] ** 2, 1)

    for i, j in ((0, 1), (1, 2), (2, 3)):
        x, y = m2(a, i, j), m2(b, i, j)
        for f in (lambda v: v, lambda v: v * v):
            fx, fy = f(x), f(y)
            err = np.sqrt(fx.var() / len(fx) + fy.var() / len(fy))
            assert abs(fx.mean() - fy.mean()) < 5 * err


def test_chain_levels_on_shell_intermediate():
    """The four-body model generates its D* (model "one", in every topology)
    on shell, as the reference's chain sampler does: m(D pi_s) = 2.007 in
    every event, four-momentum conserved."""
    from common import load_model
    from oracle.toy_oracle import genbod_levels
    from tf_pwa_b200.kincode import KinCode

    dc, vm, plan = load_model("b2dstkpi.yml")
    kin = KinCode(plan, plan.order)
    assert [len(b) for _, b in kin.levels] == [3, 2]
    assert kin.ndraw == 9
    U = uniforms(3, np.arange(3000), kin.ndraw)
    p, w = genbod_levels(U, kin.levels, kin.nfin)
    tot = p.sum(0)
    np.testing.assert_allclose(tot[0], 5.279, rtol=1e-12)
    np.testing.assert_allclose(tot[1:], 0, atol=1e-12)
    dst = p[0] + p[1]
    m = np.sqrt(dst[0] ** 2 - np.sum(dst[1:] ** 2, 0))
    np.testing.assert_allclose(m, 2.007, rtol=1e-12)
    for cfg in ("d2kpipi.yml", "lc2pkpi.yml"):
        dc, vm, plan = load_model(cfg)
        assert len(KinCode(plan, plan.order).levels) == 1

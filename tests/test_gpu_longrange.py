"""Long-range k-space pieces on the device against the oracle: k-vectors,
rho_k (full and incremental), LongRangeClass SingleAction / d_dBeta, and the
rho_k part of AcceptCopy / RejectCopy.  FP64, tolerance 1e-12 relative.

The breakup tables (Ulong_k, Ulong_r0, Ushort_k0, Ulong_k0 and their beta
derivatives) are inputs here, as in LongRangeClass after Init: an
Ewald-like Coulomb split for jellium at r_s = 4 bohr.
"""
import math

import numpy as np
import pytest

import oracle as O
import pimcplusplus_b200 as P
from helpers import random_walk_path, rel_err, tricubic_case

pytestmark = pytest.mark.gpu


def jellium_tables(kv, volume, tau, levels, alpha=0.35, z1z2=2.0):
    k2 = np.sum(kv * kv, axis=1)
    vk = 4.0 * math.pi * z1z2 * np.exp(-k2 / (4 * alpha * alpha)) / (k2 * volume)
    betas = tau * 2.0 ** np.arange(levels)
    ulong_k = np.stack([b * vk for b in betas])
    dulong_k = np.stack([vk for _ in betas])
    r0 = 2.0 * alpha / math.sqrt(math.pi) * z1z2
    ulong_r0 = betas * r0
    dulong_r0 = np.full(levels, r0)
    sk0 = -math.pi * z1z2 / (alpha * alpha * volume)
    ushort_k0 = betas * sk0
    dushort_k0 = np.full(levels, sk0)
    ulong_k0 = betas * 0.3
    dulong_k0 = np.full(levels, 0.3)
    return ulong_k, ulong_r0, ushort_k0, ulong_k0, dulong_k, dulong_r0, dushort_k0, dulong_k0


def setup_pair(use_background):
    n, m, levels = 32, 16, 3
    rs = 4.0
    L = (4.0 * math.pi / 3.0 * n) ** (1.0 / 3.0) * rs
    box = np.array([L, L, L])
    tau = 8.0 / m / 8.0
    cfg, _, _, tabs = tricubic_case(n=n, m=m, levels=levels, nq=20, ny=8, nt=8)
    qg, yg, tg, umat, dumat, pg, pot = tabs
    path = random_walk_path(n, m + 1, box, 0.8, 11, far=0.2)
    new = path.copy()
    rng = np.random.default_rng(5)
    new[1:-1, [3, 9]] += rng.normal(0, 0.5, (m - 1, 2, 3))
    o = O.System(n, m + 1, box, tau, 1.0, 0)
    o.set_pa(O.PairAction.tricubic(qg, yg, tg, tau, umat, dumat, pg, pot))  # long-range fit
    o.set_path(path, 0)
    o.set_path(new, 1)
    d = P.PathData(n, m + 1, box, tau, 1.0, 0)
    d.pa_tricubic(qg, yg, tg, tau, umat, dumat, pg, pot)
    d.set_path(path, P.OLDMODE)
    d.set_path(new, P.NEWMODE)
    nk_o = o.setup_kvecs(1.2)
    nk_d = d.setup_kvecs(1.2)
    assert nk_o == nk_d > 100
    kv, _ = o.kvecs()
    assert np.array_equal(kv, d.kvecs())
    tabs_lr = jellium_tables(kv, L ** 3, tau, levels)
    o.set_longrange(*tabs_lr, use_background=use_background)
    d.set_longrange(*tabs_lr, use_background=use_background)
    return o, d, path, new, m


def max_rel(a, b):
    return np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b)))


@pytest.mark.parametrize("use_background", [True, False])
def test_rhok_and_longrange_action(use_background):
    o, d, path, new, m = setup_pair(use_background)
    o.calc_rhok_all()
    d.calc_rhok()
    assert max_rel(d.get_rhok(0), o.rhok(0)) < 1e-12
    # incremental update of the NEW copy for the moved particles
    for (s1, s2, level) in [(2, 10, 0), (0, 16, 1), (4, 12, 2)]:
        o.update_rhok(s1, s2, [3, 9], level)
        d.update_rhok(s1, s2, [3, 9], level)
        assert max_rel(d.get_rhok(1)[s1:s2 + 1:1 << level], o.rhok(1)[s1:s2 + 1:1 << level]) < 1e-12
    lr = P.LongRangeClass(d)
    for (s1, s2, level) in [(0, 8, 0), (4, 12, 1), (0, 16, 2)]:
        for mode in (P.OLDMODE, P.NEWMODE):
            d.SetMode(mode)
            ref = o.longrange_single(s1, s2, [3, 9], level, copy=mode)
            got = lr.SingleAction(s1, s2, [3, 9], level)
            assert rel_err(got, ref) <= 1e-12, (s1, s2, level, mode, got, ref)
    for level in (0, 1):
        ref = o.longrange_dbeta(0, m, level)
        got = lr.d_dBeta(0, m, level)
        assert rel_err(got, ref) <= 1e-12, (level, got, ref)


def test_accept_reject_copy_rhok():
    o, d, path, new, m = setup_pair(True)
    d.calc_rhok()
    d.update_rhok(2, 10, [3, 9], 0)
    rho_new = d.get_rhok(1)
    d.RejectCopy(2, 10, [3, 9])
    assert np.array_equal(d.get_rhok(1)[2:11], d.get_rhok(0)[2:11])
    d.set_path(new, P.NEWMODE)
    d.update_rhok(2, 10, [3, 9], 0)
    d.AcceptCopy(2, 10, [3, 9])
    assert np.array_equal(d.get_rhok(0)[2:11], rho_new[2:11])

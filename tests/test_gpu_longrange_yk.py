"""DavidLongRangeClassYk on the device (PIMC_ACTION_DAVIDLONGRANGE) against
the FP64 oracle: SingleAction on OLD and NEW (the NEW call updates rho_k over
the window's interior first), d_dBeta and V, for the RPA and the
multiple-species tables.  Tolerance 1e-12 of the sum of |terms| (the k sum
of uk |rho_k|^2 mixes signs)."""
import numpy as np
import pytest

import oracle as O
import pimcplusplus_b200 as P

pytestmark = pytest.mark.gpu

N, M, BOX, TAU, LAM = 24, 16, 11.0, 0.1, 0.5


def _pair(seed):
    rng = np.random.default_rng(seed)
    base = rng.uniform(0, BOX, (N, 3))
    path = base[None] + rng.normal(0, 0.3, (M + 1, N, 3))
    new = path.copy()
    new[1:-1, 7] += rng.normal(0, 0.5, (M - 1, 3))
    o = O.System(N, M + 1, [BOX] * 3, TAU, LAM, 0)
    o.set_path(path, 0)
    o.set_path(new, 1)
    d = P.PathData(N, M + 1, [BOX] * 3, TAU, LAM, 0)
    d.set_path(path, P.OLDMODE)
    d.set_path(new, P.NEWMODE)
    nk = d.setup_kvecs(2.2)
    assert o.setup_kvecs(2.2) == nk
    kv = d.kvecs()
    kmag = np.sqrt((kv ** 2).sum(1))
    kvals = np.array(sorted({float(k) for k in kmag}))
    uk_long = np.where(kvals < 1.2, 40.0 / kvals ** 2, -60.0 * kvals ** 2)
    return o, d, kv, kvals, uk_long


@pytest.mark.parametrize("rpa", [True, False])
def test_yk_single_action_dbeta_v(rpa):
    o, d, kv, kvals, uk_long = _pair(11)
    assert o.set_yk(kvals, uk_long, rpa)
    d.davidlongrange_yk(kvals, uk_long, rpa)
    u, _, _ = o.yk_tables()
    o.calc_rhok_all()
    d.calc_rhok()
    act = P.DavidLongRangeClassYk(d)
    assert act.GetName() == "DavidsLongRange"
    rho_old = o.rhok(0)
    scale = float((np.abs(rho_old) ** 2 * np.abs(u)).sum())
    for (s1, s2, level) in [(0, 8, 2), (4, 12, 1), (0, M, 0), (0, M, 2), (6, 8, 1), (8, 16, 3)]:
        for mode in (P.OLDMODE, P.NEWMODE):
            ref = o.yk_single(s1, s2, [7], level, copy=mode)
            d.SetMode(mode)
            got = act.SingleAction(s1, s2, [7], level)
            assert abs(got - ref) <= 1e-12 * scale, (s1, s2, level, mode, got, ref)
        d.SetMode(P.OLDMODE)
        assert act.SingleAction(s1, s2, [], level) == 0.0
    for (s1, s2) in [(0, M), (3, 9)]:
        ref = o.yk_dbeta(s1, s2)
        got = act.d_dBeta(s1, s2, 0)
        assert abs(got - ref) <= 1e-12 * max(scale, abs(ref)), (got, ref)
        ref = o.yk_v(s1, s2)
        got = act.V(s1, s2)
        assert abs(got - ref) <= 1e-12 * max(scale, abs(ref)), (got, ref)


def test_yk_needs_every_kvector_in_the_table():
    o, d, kv, kvals, uk_long = _pair(2)
    with pytest.raises(P.PimcError):
        d.davidlongrange_yk(kvals[:-2], uk_long[:-2])
    with pytest.raises(P.PimcError):  # the action before its tables
        P.DavidLongRangeClassYk(d).SingleAction(0, 4, [1], 0)

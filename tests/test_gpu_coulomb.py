"""Jellium (classical Coulomb pair action with the optimized Ewald breakup)
on the device against the oracle: ShortRange SingleAction / d_dBeta with the
1/2 (Ulong(r) + Ulong(r')) subtraction, LongRange SingleAction / d_dBeta
with the breakup's k-space tables, and the energy terms.  The breakup tables
come from the library's host breakup (checked against the numpy/SciPy
restatement on the CPU) and are inputs to the oracle.  FP64 tolerance 1e-12
relative; the mixed SingleAction within 2e-6 of the sum of |U|."""
import math

import numpy as np
import pytest

import oracle as O
import pimcplusplus_b200 as P
from helpers import random_walk_path, rel_err

pytestmark = pytest.mark.gpu

Z1Z2 = 2.0  # e^2 in Rydberg units


def jellium(n=32, m=16, levels=3, kcut=1.2, rs=4.0, beta=2.0, knots=None, seed=11):
    L = (4.0 * math.pi / 3.0 * n) ** (1.0 / 3.0) * rs
    box = np.array([L, L, L])
    tau = beta / m
    knots = knots or int(round(3.0 * L / 2))
    path = random_walk_path(n, m + 1, box, 0.8, seed, far=0.2)
    new = path.copy()
    rng = np.random.default_rng(seed + 1)
    new[1:-1, [3, 9]] += rng.normal(0, 0.5, (m - 1, 2, 3))
    d = P.PathData(n, m + 1, box, tau, 1.0, 0)
    d.pa_coulomb(Z1Z2, levels)
    nk = d.setup_kvecs(kcut)
    d.longrange_coulomb(knots, use_background=True)
    d.set_path(path, P.OLDMODE)
    d.set_path(new, P.NEWMODE)
    o = O.System(n, m + 1, box, tau, 1.0, 0)
    o.set_pa(O.PairAction.classical_coulomb(tau, levels, Z1Z2))
    assert o.setup_kvecs(kcut) == nk
    kv, _ = o.kvecs()
    t = P.coulomb_breakup(box, Z1Z2, tau, levels, knots, kcut, kv)
    o.set_longrange(t["ulong_k"], t["ulong_r0"], t["ushort_k0"], t["ulong_k0"], t["dulong_k"],
                    t["dulong_r0"], t["dushort_k0"], t["dulong_k0"], use_background=True)
    o.set_ulong(t["ulong_r"], t["dulong_r"], t["rmax"])
    o.set_path(path, 0)
    o.set_path(new, 1)
    return o, d, m, levels


@pytest.mark.parametrize("copy", [0, 1])
def test_shortrange_single_coulomb(copy):
    o, d, m, levels = jellium()
    for (s1, s2, active, level) in [(0, 16, [3], 0), (2, 10, [3, 9], 1), (0, 16, [9, 3, 20], 2), (4, 8, [0], 0)]:
        ref = o.shortrange_single(s1, s2, active, level, copy)
        got = d.single_action(P.ACTION_SHORTRANGE, copy, s1, s2, active, level, precision=P.FP64)
        assert rel_err(got, ref, max(abs(ref), 1e-8)) < 1e-12, (s1, s2, active, level, got, ref)
        mixed = d.single_action(P.ACTION_SHORTRANGE, copy, s1, s2, active, level, precision=P.MIXED)
        scale = o.shortrange_single_abs(s1, s2, active, level, copy)
        assert abs(mixed - ref) <= 2e-6 * scale, (mixed, ref, scale)
    d.close()


def test_shortrange_dbeta_and_longrange_coulomb():
    o, d, m, levels = jellium()
    for level in range(levels):
        ref = o.shortrange_dbeta(0, m, level)
        got = d.d_dbeta(P.ACTION_SHORTRANGE, 0, m, level)
        assert rel_err(got, ref, max(abs(ref), 1e-8)) < 1e-12, (level, got, ref)
    o.calc_rhok_all()
    d.calc_rhok()
    for copy in (0, 1):
        for (s1, s2, level) in [(0, 16, 0), (2, 10, 1), (4, 12, 2)]:
            if copy == 1:
                o.update_rhok(s1, s2, [3, 9], level)
                d.update_rhok(s1, s2, [3, 9], level)
            ref = o.longrange_single(s1, s2, [3, 9], level, copy)
            got = d.single_action(P.ACTION_LONGRANGE, copy, s1, s2, [3, 9], level)
            assert rel_err(got, ref, max(abs(ref), 1e-8)) < 1e-12, (copy, s1, s2, level, got, ref)
    ref = o.longrange_dbeta(0, m, 0)
    got = d.d_dbeta(P.ACTION_LONGRANGE, 0, m, 0)
    assert rel_err(got, ref, max(abs(ref), 1e-8)) < 1e-12
    d.close()


def test_energy_terms_coulomb():
    o, d, m, levels = jellium()
    ref, got = o.energy(), d.energy()
    for k in ("kinetic", "du_short", "du_long", "v_short", "total"):
        assert rel_err(got[k], ref[k], max(abs(ref[k]), 1e-8)) < 1e-12, (k, got[k], ref[k])
    d.close()

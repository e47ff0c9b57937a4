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


def jellium_moves(seed=21, **kw):
    o, d, m, levels = jellium(**kw)
    start = o.get_path(0)
    o.set_path(start, 1)
    d.set_path(start)
    o.calc_rhok_all()
    return o, d, m, levels


def compare(ref, got, stats, tol=1e-9):
    assert len(ref) == len(got)
    n_acc = 0
    for i, (r, g) in enumerate(zip(ref, got)):
        assert (r.slice1, r.ptcl, r.accepted, r.stages_passed) == (
            int(g["slice1"]), int(g["ptcl"]), int(g["accepted"]), int(g["stages_passed"])), i
        for k in range(8):  # FP64: within tol; mixed: within the stage's reported bound
            assert abs(r.dS[k] - g["dS"][k]) <= float(g["dS_bound"][k]) + tol * max(1.0, abs(r.dS[k])), (
                i, k, r.dS[k], g["dS"][k])
        n_acc += r.accepted
    assert stats["status"] == 0 and stats["accepted"] == n_acc
    return n_acc


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
@pytest.mark.parametrize("cluster", [1, 2])
def test_bisection_jellium_longrange_trace(cluster, precision):
    """Device moves with LongRange in the lowest stage (rho_k updated per
    moved slice, written back on acceptance) replay the oracle's trace; the
    guarded mixed path too (its near-threshold stages decided in FP64, its
    accepted rho_k written in FP64)."""
    o, d, m, levels = jellium_moves()
    L, spb = 3, 4
    o.bisection_config(L, spb, use_longrange=True)
    o.rng_seed(5)
    ref = o.run_bisection(40)
    bb = P.BisectionBlock(d, L, spb, cluster_ctas=cluster, threads_per_cta=128, use_longrange=True,
                          precision=precision)
    bb.seed(5)
    got, stats = bb.MakeMoves(40)
    assert compare(ref, got, stats) > 10
    assert np.max(np.abs(d.get_path(P.OLDMODE) - o.get_path(0))) < 1e-9
    rk_o, rk_d = o.rhok(0), d.get_rhok(P.OLDMODE)
    assert np.max(np.abs(rk_d - rk_o)) < 1e-9 * np.max(np.abs(rk_o))
    # the rho_k the moves maintained is that of the final path
    o.calc_rhok_all()
    assert np.max(np.abs(rk_d - o.rhok(0))) < 1e-9 * np.max(np.abs(rk_o))
    d.close()


def test_bisection_jellium_longrange_windows():
    o, d, m, levels = jellium_moves(seed=23)
    L, spb = 2, 3
    o.bisection_config(L, spb, use_longrange=True)
    o.rng_seed(9)
    ref = o.run_windows(6)
    bb = P.BisectionBlock(d, L, spb, cluster_ctas=1, threads_per_cta=128, use_longrange=True, schedule=P.WINDOWS)
    bb.seed(9)
    got, stats = bb.MakeMoves(6)
    live = [(r, g) for r, g in zip(ref, got) if r.slice1 >= 0]
    assert len(live) > 10
    for i, (r, g) in enumerate(live):
        assert (r.slice1, r.ptcl, r.accepted, r.stages_passed) == (
            int(g["slice1"]), int(g["ptcl"]), int(g["accepted"]), int(g["stages_passed"])), i
        for k in range(8):
            assert abs(r.dS[k] - g["dS"][k]) <= 1e-9 * max(1.0, abs(r.dS[k])), (i, k)
    assert np.max(np.abs(d.get_path(P.OLDMODE) - o.get_path(0))) < 1e-9
    o.calc_rhok_all()
    assert np.max(np.abs(d.get_rhok(P.OLDMODE) - o.rhok(0))) < 1e-9 * np.max(np.abs(o.rhok(0)))
    d.close()


@pytest.mark.parametrize("guard", [True, False])
def test_bisection_jellium_mixed_shadow(guard):
    """Mixed path (FP32 pair terms and FP32 sincos of reduced phases, FP64
    sums) with the FP64 sums alongside: every stage's mixed dS within its
    rigorous bound of the FP64 dS; guarded, no flipped decision."""
    o, d, m, levels = jellium_moves(seed=29)
    bb = P.BisectionBlock(d, 3, 4, precision=P.MIXED, shadow=True, cluster_ctas=1, threads_per_cta=128,
                          use_longrange=True, guard=guard)
    bb.seed(3)
    rec, stats = bb.MakeMoves(100)
    mask = rec["dS_shadow"] != 0.0
    err = np.abs(rec["dS"][mask] - rec["dS_shadow"][mask])
    assert np.all(err <= rec["dS_bound"][mask].astype(np.float64) + 1e-12), np.max(err - rec["dS_bound"][mask])
    rel = err / np.maximum(np.abs(rec["dS_shadow"][mask]), 1e-3)
    assert np.median(rel) < 1e-5, np.median(rel)
    if guard:
        assert stats["flips"] == 0
    d.close()


def test_jellium_energy_within_2sigma_mixed_vs_oracle():
    """Independent chains sample the same distribution: the mixed device
    chain (concurrent windows, long range in the moves) and the FP64 oracle
    chain agree on the energy within 2 combined sigma (blocking)."""
    o, d, m, levels = jellium_moves(seed=31)
    L = 2
    windows = m >> L
    per_sweep = 32 * windows
    o.bisection_config(L, per_sweep, use_longrange=True)
    o.rng_seed(111)
    bb = P.BisectionBlock(d, L, 32, precision=P.MIXED, cluster_ctas=1, threads_per_cta=128, use_longrange=True,
                          schedule=P.WINDOWS)
    bb.seed(8)
    # small bisection moves accept ~98 %: long chains for independent blocks
    burn, sweeps, nb = 200, 4000, 20
    e_o, e_d = [], []
    for sw in range(burn + sweeps):
        o.run_bisection(1)
        bb.MakeMoves(1, trace=False)
        if sw >= burn:
            e_o.append(o.energy()["total"])
            e_d.append(d.energy()["total"])
    k = len(e_o) // nb
    bo = np.asarray(e_o)[: k * nb].reshape(nb, k).mean(1)
    bd = np.asarray(e_d)[: k * nb].reshape(nb, k).mean(1)
    so, sd = bo.std(ddof=1) / np.sqrt(nb), bd.std(ddof=1) / np.sqrt(nb)
    assert abs(bo.mean() - bd.mean()) <= 2.0 * np.hypot(so, sd), (bo.mean(), so, bd.mean(), sd)
    d.close()

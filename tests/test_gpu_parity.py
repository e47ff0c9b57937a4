"""Parity of the CUDA library (through its C ABI) with the FP64 oracle.

Tolerances:
  * FP64 SingleAction / d_dBeta: 1e-12 relative to the oracle value (sum
    orders differ: the oracle adds terms sequentially like the reference, the
    kernels reduce in a fixed tree).
  * Mixed precision (FP32 pair terms, FP64 sums): 2e-6 of the sum of |U|
    over the same terms (the sums cancel, so |S| is no error scale).
  * Bisection moves: identical accept trace (slice, particle, accepted,
    stages passed) and per-stage dS within 1e-9 absolute, final path within
    1e-9 (positions are O(10)).
  * Mixed-precision bisection moves (FP64 re-evaluation of every stage whose
    decision lies within the mixed sums' error bound): the same identical
    trace and final path, and each stage's mixed dS within its own reported
    bound (plus 1e-9) of the oracle's FP64 dS.
"""
import numpy as np
import pytest

import oracle as O
import pimcplusplus_b200 as P
from helpers import coulomb_fit2_tables, lj_case, random_walk_path, rel_err, tricubic_case
from pimcplusplus_b200 import workloads as W

pytestmark = pytest.mark.gpu

REL64 = 1e-12
REL32 = 2e-6


def make_pair(n, slices, box, tau, lam, seed, step, num_images=0, far=0.1):
    """Matched oracle and device systems on the same random-walk path."""
    path = random_walk_path(n, slices, box, step, seed, far=far)
    new = path.copy()
    rng = np.random.default_rng(seed + 1)
    new[1:-1] += rng.normal(0.0, step * 0.5, new[1:-1].shape)
    o = O.System(n, slices, box, tau, lam, num_images)
    o.set_path(path, 0)
    o.set_path(new, 1)
    d = P.PathData(n, slices, box, tau, lam, num_images)
    d.set_path(path, P.OLDMODE)
    d.set_path(new, P.NEWMODE)
    return o, d, path, new


def windows(slices, levels, rng, count):
    out = []
    for _ in range(count):
        level = int(rng.integers(0, levels))
        span = 1 << levels
        s1 = int(rng.integers(0, slices - span))
        out.append((s1, s1 + span, level))
    out.append((0, slices - 1, 0))
    return out


def check_single_actions(o, d, slices, levels, seed, n, precision=P.FP64, tol=REL64, count=12):
    rng = np.random.default_rng(seed)
    sr = P.ShortRangeClass(d, precision)
    worst = 0.0
    for (s1, s2, level) in windows(slices, levels, rng, count):
        for na in (1, 3):
            active = rng.choice(n, size=na, replace=False).astype(np.int32)
            for mode in (P.OLDMODE, P.NEWMODE):
                d.SetMode(mode)
                ref = o.shortrange_single(s1, s2, active, level, copy=mode)
                got = sr.SingleAction(s1, s2, active, level)
                scale = None if precision == P.FP64 else o.shortrange_single_abs(s1, s2, active, level, copy=mode)
                e = rel_err(got, ref, scale)
                worst = max(worst, e)
                assert e <= tol, (s1, s2, level, list(active), mode, got, ref)
    return worst


def test_shortrange_single_david_lj(tmp_path):
    cfg, tau, box, dm = lj_case(tmp_path)
    n, slices = cfg["N"], cfg["M"] + 1
    o, d, _, _ = make_pair(n, slices, box, tau, W.HE4_LAMBDA, 21, 0.35)
    pa = O.PairAction.from_dm(dm, tau, 0)
    o.set_pa(pa)
    d.pa_david_from_dm(dm, 0)
    check_single_actions(o, d, slices, 3, 5, n)


def test_shortrange_single_david_logrid_offdiagonal():
    # testcoul.dm's fit 2 (LOG grid, u_kj up to k=2) with NumOffDiagonalTerms=2
    g, u, du = coulomb_fit2_tables()
    n, slices, tau = 16, 33, 1.0 / 64
    box = np.array([6.0, 6.0, 6.0])
    o, d, _, _ = make_pair(n, slices, box, tau, 0.5, 31, 0.25)
    import tempfile, os
    from helpers import write_testcoul_dm
    with tempfile.TemporaryDirectory() as td:
        p = write_testcoul_dm(os.path.join(td, "tc.dm"))
        pa = O.PairAction.from_dm(p, tau, 2)
    o.set_pa(pa)
    d.pa_david(P.GRID_LOG, float(g["grid"][0]), float(g["grid"][1]), u, du, 0, 2)
    check_single_actions(o, d, slices, 3, 7, n)


def test_shortrange_single_tricubic():
    cfg, tau, box, tabs = tricubic_case()
    qg, yg, tg, umat, dumat, pg, pot = tabs
    n, slices = cfg["N"], cfg["M"] + 1
    o, d, _, _ = make_pair(n, slices, box, tau, W.HE4_LAMBDA, 41, 0.3)
    pa = O.PairAction.tricubic(qg, yg, tg, tau, umat, dumat, pg, pot)
    o.set_pa(pa)
    d.pa_tricubic(qg, yg, tg, tau, umat, dumat, pg, pot)
    check_single_actions(o, d, slices, 3, 9, n)


def test_shortrange_single_mixed_precision(tmp_path):
    cfg, tau, box, dm = lj_case(tmp_path)
    n, slices = cfg["N"], cfg["M"] + 1
    o, d, _, _ = make_pair(n, slices, box, tau, W.HE4_LAMBDA, 51, 0.35, far=0.0)
    o.set_pa(O.PairAction.from_dm(dm, tau, 0))
    d.pa_david_from_dm(dm, 0)
    check_single_actions(o, d, slices, 3, 11, n, precision=P.MIXED, tol=REL32)
    cfg, tau, box, tabs = tricubic_case()
    qg, yg, tg, umat, dumat, pg, pot = tabs
    o, d, _, _ = make_pair(cfg["N"], cfg["M"] + 1, box, tau, W.HE4_LAMBDA, 52, 0.3, far=0.0)
    o.set_pa(O.PairAction.tricubic(qg, yg, tg, tau, umat, dumat, pg, pot))
    d.pa_tricubic(qg, yg, tg, tau, umat, dumat, pg, pot)
    check_single_actions(o, d, cfg["M"] + 1, 3, 12, cfg["N"], precision=P.MIXED, tol=REL32)


def test_kinetic_single_and_dbeta():
    n, slices, tau = 20, 33, 0.02
    box = np.array([7.0, 7.0, 7.0])
    for images in (0, 1):
        o, d, _, _ = make_pair(n, slices, box, tau, 0.8, 61 + images, 0.4, num_images=images)
        kin = P.KineticClass(d)
        rng = np.random.default_rng(3)
        for (s1, s2, level) in windows(slices, 3, rng, 8):
            active = rng.choice(n, size=2, replace=False).astype(np.int32)
            for mode in (P.OLDMODE, P.NEWMODE):
                d.SetMode(mode)
                ref = o.kinetic_single(s1, s2, active, level, copy=mode)
                assert rel_err(kin.SingleAction(s1, s2, active, level), ref) <= REL64
            ref = o.kinetic_dbeta(s1, s2, level)
            assert rel_err(kin.d_dBeta(s1, s2, level), ref) <= REL64


def test_shortrange_dbeta(tmp_path):
    cfg, tau, box, dm = lj_case(tmp_path)
    n, slices = cfg["N"], cfg["M"] + 1
    o, d, _, _ = make_pair(n, slices, box, tau, W.HE4_LAMBDA, 71, 0.35)
    o.set_pa(O.PairAction.from_dm(dm, tau, 0))
    d.pa_david_from_dm(dm, 0)
    sr = P.ShortRangeClass(d)
    for level in (0, 1, 2):
        assert rel_err(sr.d_dBeta(0, slices - 1, level), o.shortrange_dbeta(0, slices - 1, level)) <= REL64
    cfg, tau, box, tabs = tricubic_case()
    qg, yg, tg, umat, dumat, pg, pot = tabs
    o, d, _, _ = make_pair(cfg["N"], cfg["M"] + 1, box, tau, W.HE4_LAMBDA, 72, 0.3)
    o.set_pa(O.PairAction.tricubic(qg, yg, tg, tau, umat, dumat, pg, pot))
    d.pa_tricubic(qg, yg, tg, tau, umat, dumat, pg, pot)
    sr = P.ShortRangeClass(d)
    assert rel_err(sr.d_dBeta(0, cfg["M"], 0), o.shortrange_dbeta(0, cfg["M"], 0)) <= REL64


def test_accept_reject_copy():
    n, slices, tau = 12, 17, 0.05
    box = np.array([5.0, 5.0, 5.0])
    o, d, path, new = make_pair(n, slices, box, tau, 0.5, 81, 0.6, far=0.3)
    d.RejectCopy(2, 9, [3, 7])
    got_new = d.get_path(P.NEWMODE)
    exp_new = new.copy()
    exp_new[2:10, [3, 7]] = path[2:10, [3, 7]]
    assert np.array_equal(got_new, exp_new)
    d.set_path(new, P.NEWMODE)
    d.AcceptCopy(4, 12, [5])
    half = box / 2
    v = new[4:13, 5].copy()
    v = np.where(v > half, v - box, v)
    v = np.where(v < -half, v + box, v)
    exp_old = path.copy()
    exp_old[4:13, 5] = v
    assert np.array_equal(d.get_path(P.OLDMODE), exp_old)


def run_trace_pair(o, d, levels, steps, n_blocks, seed, **kw):
    o.bisection_config(levels, steps)
    o.rng_seed(seed)
    ref = o.run_bisection(n_blocks)
    bb = P.BisectionBlock(d, levels, steps, **kw)
    bb.seed(seed)
    got, stats = bb.MakeMoves(n_blocks)
    return ref, got, stats


def dS_close(r_dS, g, k, tol):
    """|oracle dS - device dS| within tol (FP64), or within the stage's bound (mixed)."""
    return abs(r_dS - g["dS"][k]) <= float(g["dS_bound"][k]) + tol * max(1.0, abs(r_dS))


def compare_traces(ref, got, stats, tol=1e-9):
    assert len(ref) == len(got)
    for i, (r, g) in enumerate(zip(ref, got)):
        assert (r.slice1, r.ptcl, r.accepted, r.stages_passed) == (
            int(g["slice1"]), int(g["ptcl"]), int(g["accepted"]), int(g["stages_passed"])), i
        for k in range(8):
            assert dS_close(r.dS[k], g, k, tol), (i, k, r.dS[k], g["dS"][k], g["dS_bound"][k])
    assert stats["moves"] == len(ref)
    assert stats["accepted"] == sum(r.accepted for r in ref)
    assert stats["status"] == 0


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
@pytest.mark.parametrize("cluster", [1, 4])
def test_bisection_trace_david(tmp_path, cluster, precision):
    cfg, tau, box, dm = lj_case(tmp_path)
    n, slices = cfg["N"], cfg["M"] + 1
    pa = O.PairAction.from_dm(dm, tau, 0)
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(pa)
    o.init_random_fixed(17, 0.45 * W.LJ_SIGMA)
    start = o.get_path(0)
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.set_path(start)
    d.pa_david_from_dm(dm, 0)
    ref, got, stats = run_trace_pair(o, d, 3, 2, 400, 99, cluster_ctas=cluster, threads_per_cta=128,
                                     precision=precision)
    compare_traces(ref, got, stats)
    assert np.max(np.abs(d.get_path(P.OLDMODE) - o.get_path(0))) < 1e-9
    assert np.array_equal(d.get_path(P.OLDMODE), d.get_path(P.NEWMODE))


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_bisection_trace_tricubic(precision):
    cfg, tau, box, tabs = tricubic_case()
    qg, yg, tg, umat, dumat, pg, pot = tabs
    n, slices = cfg["N"], cfg["M"] + 1
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(O.PairAction.tricubic(qg, yg, tg, tau, umat, dumat, pg, pot))
    o.init_random_fixed(23, 0.45 * W.LJ_SIGMA)
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.set_path(o.get_path(0))
    d.pa_tricubic(qg, yg, tg, tau, umat, dumat, pg, pot)
    ref, got, stats = run_trace_pair(o, d, 3, 1, 300, 7, cluster_ctas=2, threads_per_cta=256, precision=precision)
    compare_traces(ref, got, stats)
    assert np.max(np.abs(d.get_path(P.OLDMODE) - o.get_path(0))) < 1e-9


@pytest.mark.parametrize("guard", [True, False])
def test_bisection_mixed_shadow_dS_error(tmp_path, guard):
    """Mixed path with the FP64 sums evaluated alongside.  Every stage's mixed
    dS lies within its reported bound of the FP64 dS (the bound is rigorous);
    guarded, no decision differs from the FP64 sums' (flips == 0)."""
    cfg, tau, box, dm = lj_case(tmp_path)
    n, slices = cfg["N"], cfg["M"] + 1
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.init_random_fixed(29, 0.45 * W.LJ_SIGMA)
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.set_path(o.get_path(0))
    d.pa_david_from_dm(dm, 0)
    bb = P.BisectionBlock(d, 3, 1, precision=P.MIXED, shadow=True, cluster_ctas=1, threads_per_cta=128, guard=guard)
    bb.seed(3)
    rec, stats = bb.MakeMoves(500)
    mask = rec["dS_shadow"] != 0.0
    err = np.abs(rec["dS"][mask] - rec["dS_shadow"][mask])
    assert np.all(err <= rec["dS_bound"][mask].astype(np.float64) + 1e-12), np.max(err - rec["dS_bound"][mask])
    rel = err / np.maximum(np.abs(rec["dS_shadow"][mask]), 1e-3)
    assert np.median(rel) < 1e-6
    if guard:
        assert stats["flips"] == 0
    else:
        assert stats["reevaluated"] == 0 and np.all(rec["reevaluated"] == 0)


def compare_window_traces(ref, got, stats, tol=1e-9):
    assert len(ref) == len(got)
    n_moves = 0
    for i, (r, g) in enumerate(zip(ref, got)):
        assert (r.slice1, r.ptcl, r.accepted, r.stages_passed) == (
            int(g["slice1"]), int(g["ptcl"]), int(g["accepted"]), int(g["stages_passed"])), i
        if r.slice1 >= 0:
            n_moves += 1
        for k in range(8):
            assert dS_close(r.dS[k], g, k, tol), (i, k, r.dS[k], g["dS"][k], g["dS_bound"][k])
    assert stats["moves"] == n_moves
    assert stats["status"] == 0


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
@pytest.mark.parametrize("cluster", [1, 2])
def test_bisection_trace_windows_david(tmp_path, cluster, precision):
    """Concurrent-window schedule (time-slice parallel) against the oracle's
    sequential replay of the same rounds."""
    cfg, tau, box, dm = lj_case(tmp_path)
    n, slices = cfg["N"], cfg["M"] + 1
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(O.PairAction.from_dm(dm, tau, 0))
    o.init_random_fixed(37, 0.45 * W.LJ_SIGMA)
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.set_path(o.get_path(0))
    d.pa_david_from_dm(dm, 0)
    o.bisection_config(3, 2)
    o.rng_seed(41)
    ref = o.run_windows(60)
    bb = P.BisectionBlock(d, 3, 2, cluster_ctas=cluster, threads_per_cta=128, schedule=P.WINDOWS,
                          precision=precision)
    assert bb.windows == 5
    bb.seed(41)
    got, stats = bb.MakeMoves(60)
    compare_window_traces(ref, got, stats)
    assert np.max(np.abs(d.get_path(P.OLDMODE) - o.get_path(0))) < 1e-9


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_bisection_trace_windows_tricubic(precision):
    cfg, tau, box, tabs = tricubic_case()
    qg, yg, tg, umat, dumat, pg, pot = tabs
    n, slices = cfg["N"], cfg["M"] + 1
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(O.PairAction.tricubic(qg, yg, tg, tau, umat, dumat, pg, pot))
    o.init_random_fixed(43, 0.45 * W.LJ_SIGMA)
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.set_path(o.get_path(0))
    d.pa_tricubic(qg, yg, tg, tau, umat, dumat, pg, pot)
    o.bisection_config(3, 1)
    o.rng_seed(47)
    ref = o.run_windows(50)
    bb = P.BisectionBlock(d, 3, 1, cluster_ctas=4, threads_per_cta=256, schedule=P.WINDOWS, precision=precision)
    bb.seed(47)
    got, stats = bb.MakeMoves(50)
    compare_window_traces(ref, got, stats)
    assert np.max(np.abs(d.get_path(P.OLDMODE) - o.get_path(0))) < 1e-9


@pytest.mark.parametrize("schedule", ["sequential", "windows"])
def test_bisection_trace_level5_truncated_lj(tmp_path, schedule):
    """Bisection level 5 (32-slice windows, 16 midpoints at the top level) on
    the C5 table (LJ truncated and shifted to zero at 2.5 sigma)."""
    cfg = dict(W.CONFIGS["C5"])
    cfg.update(N=128, M=128)
    tau, box = W.derived(cfg)
    dm = W.make_dm_for(cfg, str(tmp_path))
    n, slices, L = cfg["N"], cfg["M"] + 1, cfg["levels"]
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(O.PairAction.from_dm(dm, tau, 0))
    start = W.lattice_path(n, slices, box, np.random.default_rng(51))
    o.set_path(start, 0)
    o.set_path(start, 1)
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.set_path(start)
    d.pa_david_from_dm(dm, 0)
    o.bisection_config(L, 4)
    o.rng_seed(77)
    if schedule == "sequential":
        ref = o.run_bisection(60)
        bb = P.BisectionBlock(d, L, 4, cluster_ctas=4, threads_per_cta=256)
    else:
        ref = o.run_windows(15)
        bb = P.BisectionBlock(d, L, 4, cluster_ctas=4, threads_per_cta=256, schedule=P.WINDOWS)
    bb.seed(77)
    got, stats = bb.MakeMoves(60 if schedule == "sequential" else 15)
    live = [(r, g) for r, g in zip(ref, got) if r.slice1 >= 0]
    assert len(live) > 20
    acc = 0
    for i, (r, g) in enumerate(live):
        assert (r.slice1, r.ptcl, r.accepted, r.stages_passed) == (
            int(g["slice1"]), int(g["ptcl"]), int(g["accepted"]), int(g["stages_passed"])), i
        for k in range(8):
            assert abs(r.dS[k] - g["dS"][k]) <= 1e-9 * max(1.0, abs(r.dS[k])), (i, k)
        acc += r.accepted
    assert 0 < acc < len(live)
    assert np.max(np.abs(d.get_path(P.OLDMODE) - o.get_path(0))) < 1e-9


@pytest.mark.parametrize("schedule,skin,cluster", [("sequential", 3.0, 4), ("windows", 3.0, 2), ("sequential", 0.02, 1),
                                                   ("windows", 0.02, 2)])
def test_bisection_neighbor_lists_match_all_partner_oracle(tmp_path, schedule, skin, cluster):
    """Neighbour lists (bounding spheres of each particle's path + skin) give
    the all-partner sums of the oracle: the truncated table is zero beyond its
    end.  A tiny skin makes moves leave their spheres, exercising the
    all-partner fallback and the rebuild between launches."""
    cfg = dict(W.CONFIGS["C5"])
    cfg.update(N=256, M=128)
    tau, box = W.derived(cfg)
    dm = W.make_dm_for(cfg, str(tmp_path))
    n, slices, L = cfg["N"], cfg["M"] + 1, cfg["levels"]
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(O.PairAction.from_dm(dm, tau, 0))
    start = W.lattice_path(n, slices, box, np.random.default_rng(61))
    o.set_path(start, 0)
    o.set_path(start, 1)
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.set_path(start)
    d.pa_david_from_dm(dm, 0)
    o.bisection_config(L, 4)
    o.rng_seed(83)
    kw = dict(cluster_ctas=cluster, threads_per_cta=256, neighbor_skin=skin)
    if schedule == "sequential":
        ref = list(o.run_bisection(30)) + list(o.run_bisection(30))
        bb = P.BisectionBlock(d, L, 4, **kw)
        bb.seed(83)
        g1, _ = bb.MakeMoves(30)
        g2, stats = bb.MakeMoves(30)
    else:
        ref = list(o.run_windows(8)) + list(o.run_windows(8))
        bb = P.BisectionBlock(d, L, 4, schedule=P.WINDOWS, **kw)
        bb.seed(83)
        g1, _ = bb.MakeMoves(8)
        g2, stats = bb.MakeMoves(8)
    got = np.concatenate([g1, g2])
    live = [(r, g) for r, g in zip(ref, got) if r.slice1 >= 0]
    acc = 0
    for i, (r, g) in enumerate(live):
        assert (r.slice1, r.ptcl, r.accepted, r.stages_passed) == (
            int(g["slice1"]), int(g["ptcl"]), int(g["accepted"]), int(g["stages_passed"])), i
        for k in range(8):
            assert abs(r.dS[k] - g["dS"][k]) <= 1e-9 * max(1.0, abs(r.dS[k])), (i, k, r.dS[k], g["dS"][k])
        acc += r.accepted
    assert acc > 5
    assert np.max(np.abs(d.get_path(P.OLDMODE) - o.get_path(0))) < 1e-9
    # with a skin above the moves' excursions the lists cut the pair evaluations
    full = sum(2 * (n - 1) * sum((1 << L) >> lv for lv in range(L - 1, L - 2 - r.stages_passed, -1) if lv >= 0)
               for r, _ in live)
    if skin >= 1.0:
        assert stats["pair_evals"] < 0.8 * full, (stats["pair_evals"], full)


def test_shortrange_single_edge_cases(tmp_path):
    """Empty and degenerate calls, repeated movers, the largest active list,
    and the argument errors the reference would assert on."""
    cfg, tau, box, dm = lj_case(tmp_path, n=80, m=16, levels=2, npts=400)
    n, slices = cfg["N"], cfg["M"] + 1
    o, d, _, _ = make_pair(n, slices, box, tau, W.HE4_LAMBDA, 61, 0.35)
    o.set_pa(O.PairAction.from_dm(dm, tau, 0))
    d.pa_david_from_dm(dm, 0)
    sr, kin = P.ShortRangeClass(d), P.KineticClass(d)
    assert sr.SingleAction(0, 8, [], 0) == 0.0 == o.shortrange_single(0, 8, [], 0)
    assert kin.SingleAction(0, 8, [], 0) == 0.0
    assert sr.SingleAction(5, 5, [1, 2], 0) == 0.0 == o.shortrange_single(5, 5, [1, 2], 0)
    # a particle listed twice: DoPtcl leaves it visited, its partners are summed again
    for act in ([3, 5, 3], [7, 7]):
        ref = o.shortrange_single(0, 16, act, 1)
        assert rel_err(sr.SingleAction(0, 16, act, 1), ref) <= REL64
    # the largest active list, moved-moved pairs counted once, whole path
    act = np.arange(64, dtype=np.int32)[::-1].copy()
    for mode in (P.OLDMODE, P.NEWMODE):
        d.SetMode(mode)
        ref = o.shortrange_single(0, 16, act, 0, copy=mode)
        assert rel_err(sr.SingleAction(0, 16, act, 0), ref) <= REL64
    d.SetMode(P.OLDMODE)
    for args in ((0, 8, [n], 0), (0, 8, [-1], 0), (0, 8, [1], 8), (0, slices, [1], 0), (4, 2, [1], 0),
                 (0, 8, list(range(65)), 0)):
        with pytest.raises(P.PimcError):
            sr.SingleAction(*args)


def test_nan_in_the_path_is_a_status(tmp_path):
    """A NaN position (a damaged input, not a device fault) comes back as
    PIMC_E_NAN from SingleAction and from the device moves' status word, and
    the context keeps working: every index derived from a NaN is clamped."""
    cfg, tau, box, dm = lj_case(tmp_path, n=16, m=16, levels=2, npts=200)
    n, slices = cfg["N"], cfg["M"] + 1
    path = random_walk_path(n, slices, box, 0.3, seed=5)
    path[slices - 1] = path[0]
    bad = path.copy()
    bad[5, 3, 1] = np.nan
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.pa_david_from_dm(dm, 0)
    d.set_path(bad)
    sr = P.ShortRangeClass(d)
    with pytest.raises(P.PimcError) as e:
        sr.SingleAction(0, 8, [3], 0)
    assert e.value.status == 3
    with pytest.raises(P.PimcError) as e:
        sr.SingleAction(0, 8, [7], 0)  # 3 is a partner of 7
    assert e.value.status == 3
    d.set_path(path)
    assert np.isfinite(sr.SingleAction(0, 8, [3], 0))
    d.set_path(bad)
    bb = P.BisectionBlock(d, cfg["levels"], 4)
    bb.seed(3)
    with pytest.raises(P.PimcError) as e:
        bb.MakeMoves(20)
    assert e.value.status == 3
    d.set_path(path)
    bb = P.BisectionBlock(d, cfg["levels"], 4)
    bb.seed(3)
    _, st = bb.MakeMoves(5)
    assert st["status"] == 0 and st["moves"] == 20

"""The full benchmark sizes, through checks that do not need the oracle to
replay a whole run:

* C2 (512 atoms, M = 128, PAtricubicFit 200x50x50, five levels): ShortRange and
  Kinetic SingleAction and ShortRange d_dBeta against the oracle (single
  calls are cheap for it even at this size), and invariance of the actions
  under a common translation of every particle (the minimum-image sums do
  not depend on where the box's origin is).
* C5 (4096 atoms, M = 256, level 5, LJ truncated at 2.5 sigma): device moves
  with neighbour lists make exactly the moves of the all-partner device moves
  from the same seed, since the truncated table is zero beyond its end.
"""
import numpy as np
import pytest

import oracle as O
import pimcplusplus_b200 as P
from helpers import random_walk_path, rel_err
from pimcplusplus_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_c2_full_size_actions():
    cfg = dict(W.CONFIGS["C2"])
    tau, box = W.derived(cfg)
    n, S, L = cfg["N"], cfg["M"] + 1, cfg["levels"]
    qg, yg, tg, umat, dumat, pg, pot = W.tricubic_tables(box[0], tau, L + 1, nq=200, ny=50, nt=50)
    path = random_walk_path(n, S, box, 0.3, seed=77)
    path[S - 1] = path[0]
    d = P.PathData(n, S, box, tau, W.HE4_LAMBDA, 0)
    d.pa_tricubic(qg, yg, tg, tau, umat, dumat, pg, pot)
    d.set_path(path)
    o = O.System(n, S, box, tau, W.HE4_LAMBDA, 0)
    pa = O.PairAction.tricubic(qg, yg, tg, tau, umat, dumat, pg, pot)
    o.set_pa(pa)
    o.set_path(path)
    sr, kin = P.ShortRangeClass(d), P.KineticClass(d)
    calls = ((0, 16, [5], 0), (32, 48, [100, 511, 7], 2), (0, 128, list(range(0, 512, 16)), 4))
    base = []
    for s1, s2, act, lev in calls:
        a = np.array(act, dtype=np.int32)
        ref = o.shortrange_single(s1, s2, a, lev)
        got = sr.SingleAction(s1, s2, act, lev)
        assert rel_err(got, ref) <= 1e-12, (s1, s2, lev, got, ref)
        kref = o.kinetic_single(s1, s2, a, lev)
        assert rel_err(kin.SingleAction(s1, s2, act, lev), kref) <= 1e-12
        base.append((got, kref))
    ref = o.shortrange_dbeta(0, S - 1, 0)
    got_db = sr.d_dBeta(0, S - 1, 0)
    assert rel_err(got_db, ref) <= 1e-12, (got_db, ref)
    # a common translation of every particle changes no minimum-image distance
    shift = np.array([0.37, -1.91, 2.53]) * box / 3.0
    d.set_path(path + shift)
    for (s1, s2, act, lev), (u0, k0) in zip(calls, base):
        assert rel_err(sr.SingleAction(s1, s2, act, lev), u0) <= 1e-10
        assert rel_err(kin.SingleAction(s1, s2, act, lev), k0) <= 1e-10
    assert rel_err(sr.d_dBeta(0, S - 1, 0), got_db) <= 1e-10
    d.close()


def test_c5_full_size_neighbor_lists_equal_all_partners(tmp_path):
    cfg = dict(W.CONFIGS["C5"])
    tau, box = W.derived(cfg)
    n, S, L = cfg["N"], cfg["M"] + 1, cfg["levels"]
    dm = W.make_dm_for(cfg, str(tmp_path))
    start = W.lattice_path(n, S, box, np.random.default_rng(5))
    runs = []
    for skin in (2.5, 0.0):
        d = P.PathData(n, S, box, tau, W.HE4_LAMBDA, 0)
        d.pa_david_from_dm(dm, 0)
        d.set_path(start)
        bb = P.BisectionBlock(d, L, 16, cluster_ctas=16, threads_per_cta=512, schedule=P.WINDOWS,
                              neighbor_skin=skin)
        bb.seed(901)
        rec, st = bb.MakeMoves(2)
        runs.append((rec, st, d.get_path(P.OLDMODE)))
        d.close()
    (r1, s1, p1), (r2, s2, p2) = runs
    assert s1["status"] == 0 and s2["status"] == 0
    for k in ("slice1", "ptcl", "accepted", "stages_passed"):
        assert np.array_equal(r1[k], r2[k]), k
    assert np.allclose(r1["dS"], r2["dS"], rtol=1e-9, atol=1e-12)
    assert np.max(np.abs(p1 - p2)) < 1e-12
    assert s1["moves"] == s2["moves"] > 0 and s1["accepted"] == s2["accepted"] > 0
    assert s1["pair_evals"] < 0.2 * s2["pair_evals"]  # the lists cut the evaluations

"""Parity at the benchmark's own sizes and launch shapes, against the FP64
oracle's replay of the same moves (BisectionBlock.cc:380-451 on the same
Philox streams):

* C2: 512 atoms, M = 128, PAtricubicFit 200x50x50, level 4, the bench's
  launch (concurrent windows, 16-CTA clusters x 512 threads, StepsPerBlock 128);
* C1: 64 atoms, M = 40, 1-D primitive table, level 3, the bench's launch
  (windows, 8-CTA clusters x 256 threads, StepsPerBlock 64);
* C4: jellium, 128 electrons, M = 64, 510 k-vectors, the bench's launch
  (windows, 8-CTA clusters x 512 threads, StepsPerBlock 16), trace and rho_k;
* C5: 4096 atoms, M = 256, level 5, neighbour lists on the device against the
  oracle's all-partner sums (windows, 16-CTA clusters x 512 threads);
* C3: a subset of the bench's 1024-chain set holding its costliest chains
  (N = 512, M = 128), per chain against the oracle, and the batched mixed
  path's dS bound with the FP64 sums alongside.

FP64: identical trace (slice, particle, accepted, stages passed), dS within
1e-9, final path within 1e-9.  Mixed (decision guard): the same trace and
path, each mixed dS within its reported bound (+1e-9) of the oracle's.
"""
import numpy as np
import pytest

import oracle as O
import pimcplusplus_b200 as P
from pimcplusplus_b200 import workloads as W
from test_gpu_coulomb import jellium_moves

pytestmark = pytest.mark.gpu


def compare(ref, got, stats, tol=1e-9):
    assert len(ref) == len(got)
    n_moves = 0
    for i, (r, g) in enumerate(zip(ref, got)):
        assert (r.slice1, r.ptcl, r.accepted, r.stages_passed) == (
            int(g["slice1"]), int(g["ptcl"]), int(g["accepted"]), int(g["stages_passed"])), i
        n_moves += r.slice1 >= 0
        for k in range(8):
            assert abs(r.dS[k] - g["dS"][k]) <= float(g["dS_bound"][k]) + tol * max(1.0, abs(r.dS[k])), (
                i, k, r.dS[k], g["dS"][k], g["dS_bound"][k])
    assert stats["status"] == 0 and stats["moves"] == n_moves
    return n_moves


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_c2_bench_launch(precision):
    cfg = dict(W.CONFIGS["C2"])
    tau, box = W.derived(cfg)
    n, S, L = cfg["N"], cfg["M"] + 1, cfg["levels"]
    qg, yg, tg, umat, dumat, pg, pot = W.tricubic_tables(box[0], tau, L, nq=200, ny=50, nt=50)
    o = O.System(n, S, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(O.PairAction.tricubic(qg, yg, tg, tau, umat, dumat, pg, pot))
    o.init_random_fixed(17, 0.45 * W.LJ_SIGMA)
    d = P.PathData(n, S, box, tau, W.HE4_LAMBDA, 0)
    d.pa_tricubic(qg, yg, tg, tau, umat, dumat, pg, pot)
    d.set_path(o.get_path(0))
    spb, rounds = 128, 2
    o.bisection_config(L, spb)
    o.rng_seed(1000)
    ref = o.run_windows(rounds)
    bb = P.BisectionBlock(d, L, spb, precision=precision, cluster_ctas=16, threads_per_cta=512,
                          schedule=P.WINDOWS)
    bb.seed(1000)
    got, stats = bb.MakeMoves(rounds)
    assert compare(ref, got, stats) > 700
    assert np.max(np.abs(d.get_path(P.OLDMODE) - o.get_path(0))) < 1e-9
    d.close()


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_c1_bench_launch(precision, tmp_path):
    cfg = dict(W.CONFIGS["C1"])
    tau, box = W.derived(cfg)
    n, S, L = cfg["N"], cfg["M"] + 1, cfg["levels"]
    dm = W.make_dm_for(cfg, str(tmp_path))
    o = O.System(n, S, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(O.PairAction.from_dm(dm, tau, 0))
    o.init_random_fixed(17, 0.45 * W.LJ_SIGMA)
    d = P.PathData(n, S, box, tau, W.HE4_LAMBDA, 0)
    d.pa_david_from_dm(dm, 0)
    d.set_path(o.get_path(0))
    spb, rounds = 64, 3
    o.bisection_config(L, spb)
    o.rng_seed(70)
    ref = o.run_windows(rounds)
    bb = P.BisectionBlock(d, L, spb, precision=precision, cluster_ctas=8, threads_per_cta=256,
                          schedule=P.WINDOWS)
    bb.seed(70)
    got, stats = bb.MakeMoves(rounds)
    assert compare(ref, got, stats) > 300
    assert np.max(np.abs(d.get_path(P.OLDMODE) - o.get_path(0))) < 1e-9
    d.close()


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_c4_bench_launch(precision):
    o, d, m, levels = jellium_moves(n=128, m=64, levels=3, kcut=1.2, rs=4.0, beta=8.0, knots=49)
    assert len(d.kvecs()) == 510
    L, spb, rounds = 3, 16, 2
    o.bisection_config(L, spb, use_longrange=True)
    o.rng_seed(500)
    ref = o.run_windows(rounds)
    bb = P.BisectionBlock(d, L, spb, precision=precision, cluster_ctas=8, threads_per_cta=512, schedule=P.WINDOWS,
                          use_longrange=True)
    bb.seed(500)
    got, stats = bb.MakeMoves(rounds)
    assert compare(ref, got, stats) > 150
    assert stats["accepted"] > 50
    assert np.max(np.abs(d.get_path(P.OLDMODE) - o.get_path(0))) < 1e-9
    # the rho_k the moves maintained is the oracle's and that of the final path
    rk_o, rk_d = o.rhok(0), d.get_rhok(P.OLDMODE)
    scale = np.max(np.abs(rk_o))
    assert np.max(np.abs(rk_d - rk_o)) < 1e-9 * scale
    o.calc_rhok_all()
    assert np.max(np.abs(rk_d - o.rhok(0))) < 1e-9 * scale
    d.close()


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_c5_bench_launch_lists_vs_oracle_all_partners(tmp_path, precision):
    cfg = dict(W.CONFIGS["C5"])
    tau, box = W.derived(cfg)
    n, S, L = cfg["N"], cfg["M"] + 1, cfg["levels"]
    dm = W.make_dm_for(cfg, str(tmp_path))
    start = W.lattice_path(n, S, box, np.random.default_rng(5))
    o = O.System(n, S, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(O.PairAction.from_dm(dm, tau, 0))
    o.set_path(start, 0)
    o.set_path(start, 1)
    d = P.PathData(n, S, box, tau, W.HE4_LAMBDA, 0)
    d.pa_david_from_dm(dm, 0)
    d.set_path(start)
    spb = 16
    o.bisection_config(L, spb)
    o.rng_seed(900)
    ref = o.run_windows(1)
    bb = P.BisectionBlock(d, L, spb, precision=precision, cluster_ctas=16, threads_per_cta=512, schedule=P.WINDOWS,
                          neighbor_skin=2.5)
    bb.seed(900)
    got, stats = bb.MakeMoves(1)
    assert compare(ref, got, stats) > 100
    assert np.max(np.abs(d.get_path(P.OLDMODE) - o.get_path(0))) < 1e-9
    d.close()


def _c3_subset():
    chains = W.c3_chains(1024, seed=0, steps_per_block=4)
    cost = [c["N"] ** 2 * (c["slices"] - 1) * (1 << c["num_levels"]) for c in chains]
    order = np.argsort(cost)[::-1]
    pick = list(order[:4]) + list(np.random.default_rng(3).choice(order[4:], 6, replace=False))
    sub = [chains[i] for i in pick]
    assert max(c["N"] for c in sub) == 512 and max(c["slices"] for c in sub) == 129
    return sub


def _oracle_chain(c, n_blocks):
    ng = c["grid"][2]
    ukj = np.zeros((c["u00"].shape[0], ng, 2))
    ukj[:, :, 1] = c["u00"]
    s = O.System(c["N"], c["slices"], c["box"], c["tau"], c["lam"], 0)
    s.set_pa(O.PairAction.david_arrays(c["grid"][0], c["grid"][1], ukj, np.zeros_like(ukj), 0, 0))
    s.set_path(c["path"])
    s.bisection_config(c["num_levels"], c["steps_per_block"])
    s.rng_seed(c["seed"])
    return s.run_bisection(n_blocks), s.get_path(0)


@pytest.mark.parametrize("precision", [P.FP64, P.MIXED])
def test_c3_subset_with_largest_chains(precision):
    chains = _c3_subset()
    b = P.BatchChains(chains, precision=precision, threads_per_cta=512, ctas=0, max_split=1, split_ratio=0.5)
    n_blocks = 4
    trace, stats = b.run(n_blocks, trace=True)
    for i, c in enumerate(chains):
        ref, ref_path = _oracle_chain(c, n_blocks)
        got = trace[i]
        for k, r in enumerate(ref):
            g = got[k]
            assert (r.slice1, r.ptcl, r.accepted, r.stages_passed) == (
                int(g["slice1"]), int(g["ptcl"]), int(g["accepted"]), int(g["stages_passed"])), (i, k)
            for j in range(8):
                assert abs(r.dS[j] - g["dS"][j]) <= float(g["dS_bound"][j]) + 1e-9 * max(1.0, abs(r.dS[j])), (i, k, j)
        assert np.max(np.abs(b.path(i) - ref_path)) < 1e-9, i
    assert stats["status"] == 0
    b.close()


def test_c3_subset_mixed_shadow_bound():
    chains = _c3_subset()
    b = P.BatchChains(chains, precision=P.MIXED, shadow=True, threads_per_cta=512)
    trace, stats = b.run(4, trace=True)
    rec = trace.reshape(-1)
    mask = rec["dS_shadow"] != 0.0
    err = np.abs(rec["dS"][mask] - rec["dS_shadow"][mask])
    assert mask.sum() > 100
    assert np.all(err <= rec["dS_bound"][mask].astype(np.float64) + 1e-12)
    assert stats["flips"] == 0 and stats["status"] == 0
    b.close()

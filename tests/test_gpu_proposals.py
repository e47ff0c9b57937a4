"""Concurrent moved-particle proposals (PIMC_SCHEDULE_PROPOSALS) against the
FP64 oracle's in-order replay.

Each window of a round runs P proposal slots at once, one CTA each; a step
of the window is slots 0..P-1 making one move each, and the device must give
the result of making them one after another in slot order (oracle
`run_proposals`).  The commit makes a slot again when an earlier slot of the
same pass accepted a move of its particle, or of a particle that comes
within the table's range of it at some slice of the window, so the traces
must be identical however the slots interact:

  * neighbour lists with a skin above the moves' excursions;
  * a tiny skin: moves leave their spheres, which falls back to all partners
    for the rest of the round;
  * no lists: every slot sums over all partners.

Tolerances as in test_gpu_parity: identical accept trace, per-stage dS within
1e-9, final path within 1e-9.
"""
import numpy as np
import pytest

import oracle as O
import pimcplusplus_b200 as P
from pimcplusplus_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _c5_pair(tmp_path, n, m, seed):
    cfg = dict(W.CONFIGS["C5"])
    cfg.update(N=n, M=m)
    tau, box = W.derived(cfg)
    dm = W.make_dm_for(cfg, str(tmp_path))
    slices, L = cfg["M"] + 1, cfg["levels"]
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(O.PairAction.from_dm(dm, tau, 0))
    start = W.lattice_path(n, slices, box, np.random.default_rng(seed))
    o.set_path(start, 0)
    o.set_path(start, 1)
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.set_path(start)
    d.pa_david_from_dm(dm, 0)
    return o, d, L


def _compare(ref, got):
    assert len(ref) == len(got)
    live = [(r, g) for r, g in zip(ref, got) if r.slice1 >= 0]
    acc = 0
    for i, (r, g) in enumerate(live):
        assert (r.slice1, r.ptcl, r.accepted, r.stages_passed) == (
            int(g["slice1"]), int(g["ptcl"]), int(g["accepted"]), int(g["stages_passed"])), i
        for k in range(8):
            assert abs(r.dS[k] - g["dS"][k]) <= 1e-9 * max(1.0, abs(r.dS[k])), (i, k, r.dS[k], g["dS"][k])
        acc += r.accepted
    return live, acc


@pytest.mark.parametrize("proposals,skin", [(4, 3.0), (8, 3.0), (8, 0.02), (4, 0.0)])
def test_proposals_match_in_order_oracle(tmp_path, proposals, skin):
    o, d, L = _c5_pair(tmp_path, 256, 128, 71)
    spb, rounds = 3, 4
    o.bisection_config(L, spb)
    o.rng_seed(91)
    ref = list(o.run_proposals(rounds, proposals)) + list(o.run_proposals(rounds, proposals))
    bb = P.BisectionBlock(d, L, spb, schedule=P.PROPOSALS, cluster_ctas=proposals, threads_per_cta=256,
                          neighbor_skin=skin)
    bb.seed(91)
    g1, _ = bb.MakeMoves(rounds)
    g2, stats = bb.MakeMoves(rounds)
    live, acc = _compare(ref, np.concatenate([g1, g2]))
    assert stats["status"] == 0
    assert stats["moves"] == len(live)
    assert 0 < acc < len(live)
    assert np.max(np.abs(d.get_path(P.OLDMODE) - o.get_path(0))) < 1e-9
    if proposals == 8:
        # 8 slots in a 22.7 A box: some accepted moves come within range of a later slot's particle
        assert stats["redone"] > 0


def test_proposals_one_slot_is_the_windows_schedule(tmp_path):
    """P = 1 draws slot 0's stream, which is the window's stream of the
    WINDOWS schedule: the two schedules give the same trace."""
    o, d, L = _c5_pair(tmp_path, 128, 128, 5)
    o.bisection_config(L, 2)
    o.rng_seed(13)
    ref = o.run_windows(6)
    bb = P.BisectionBlock(d, L, 2, schedule=P.PROPOSALS, cluster_ctas=1, threads_per_cta=256, neighbor_skin=3.0)
    bb.seed(13)
    got, stats = bb.MakeMoves(6)
    live, _ = _compare(ref, got)
    assert stats["moves"] == len(live) and stats["redone"] == 0


def test_proposals_mixed_precision_shadow(tmp_path):
    """Mixed precision with the FP64 shadow: runs clean, and the stage
    decisions the other precision would flip are rare."""
    o, d, L = _c5_pair(tmp_path, 256, 128, 29)
    bb = P.BisectionBlock(d, L, 4, schedule=P.PROPOSALS, cluster_ctas=8, threads_per_cta=256, neighbor_skin=3.0,
                          precision=P.MIXED, shadow=True)
    bb.seed(3)
    got, stats = bb.MakeMoves(6)
    assert stats["status"] == 0
    assert stats["moves"] == int(np.sum(got["slice1"] >= 0)) > 0
    assert stats["flips"] <= max(2, stats["stages_attempted"] // 1000)


def test_proposals_rejects_long_range_and_other_tables(tmp_path):
    o, d, L = _c5_pair(tmp_path, 64, 64, 3)
    with pytest.raises(P.PimcError):
        P.BisectionBlock(d, L, 1, schedule=P.PROPOSALS, cluster_ctas=4, use_longrange=True)
    d2 = P.PathData(8, 17, [10.0] * 3, 0.1, 0.5, 0)
    d2.pa_coulomb(2.0, 2)
    with pytest.raises(P.PimcError):
        P.BisectionBlock(d2, 2, 1, schedule=P.PROPOSALS, cluster_ctas=4)

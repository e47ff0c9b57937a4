"""Failure detection on the device without a fault: a bounded wait that runs
out returns a status the host reads, and the context stays usable.

The bisection kernel stages its DavidPA tables into shared memory with a bulk
copy completing on an mbarrier and spins on that barrier for a bounded number
of tries.  `test_wait` makes each CTA, after its copy has landed, also spin a
few tries on a barrier that nothing arrives at; that wait always runs out, so
every launch takes the give-up path: PIMC_E_CAP in the status word, no move
made.  The reference aborts instead (StageClass.cc:74-85 for broken staging).
"""
import numpy as np
import pytest

import oracle as O
import pimcplusplus_b200 as P
from helpers import lj_case
from pimcplusplus_b200 import workloads as W

pytestmark = pytest.mark.gpu

PIMC_E_CAP = 5


@pytest.mark.parametrize("schedule,cluster", [(P.SEQUENTIAL, 1), (P.SEQUENTIAL, 4), (P.WINDOWS, 2)])
def test_staging_wait_gives_up_then_context_recovers(tmp_path, schedule, cluster):
    cfg, tau, box, dm = lj_case(tmp_path)
    n, slices = cfg["N"], cfg["M"] + 1
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(O.PairAction.from_dm(dm, tau, 0))
    o.init_random_fixed(61, 0.45 * W.LJ_SIGMA)
    start = o.get_path(0)
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.set_path(start)
    d.pa_david_from_dm(dm, 0)

    bad = P.BisectionBlock(d, 3, 2, cluster_ctas=cluster, threads_per_cta=128, schedule=schedule, test_wait=64)
    bad.seed(13)
    with pytest.raises(P.PimcError) as ei:
        bad.MakeMoves(3)
    assert ei.value.status == PIMC_E_CAP
    st = bad.stats()
    assert st["moves"] == 0 and st["status"] == 0  # nothing moved; the status was reported and cleared
    assert np.array_equal(d.get_path(P.OLDMODE), start)

    # the same context, a normal wait: the oracle's moves from the same state
    good = P.BisectionBlock(d, 3, 2, cluster_ctas=cluster, threads_per_cta=128, schedule=schedule)
    good.seed(13)
    o.bisection_config(3, 2)
    o.rng_seed(13)
    if schedule == P.SEQUENTIAL:
        ref = o.run_bisection(40)
        got, stats = good.MakeMoves(40)
    else:
        ref = o.run_windows(10)
        got, stats = good.MakeMoves(10)
    assert len(ref) == len(got)
    for i, (r, g) in enumerate(zip(ref, got)):
        assert (r.slice1, r.ptcl, r.accepted, r.stages_passed) == (
            int(g["slice1"]), int(g["ptcl"]), int(g["accepted"]), int(g["stages_passed"])), i
    assert stats["status"] == 0
    assert np.max(np.abs(d.get_path(P.OLDMODE) - o.get_path(0))) < 1e-9
    d.close()

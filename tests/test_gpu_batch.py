"""Many independent chains in one persistent launch against the oracle:
each chain's accept trace and final path must equal its own sequential
oracle run (FP64), whatever CTA ran it and in whatever order."""
import numpy as np
import pytest

import oracle as O
import pimcplusplus_b200 as P
from pimcplusplus_b200 import workloads as W

pytestmark = pytest.mark.gpu


def make_chains():
    rng = np.random.default_rng(77)
    chains = []
    for i in range(12):
        n = int(rng.choice([16, 24, 40]))
        m = int(rng.choice([8, 16, 32]))
        levels = 2 if m == 8 else 3
        chains.append(W.lj_chain(n, m, float(rng.uniform(1.0, 4.0)), 0.02186, levels, seed=500 + i,
                                 steps_per_block=2, npts=200, rng=np.random.default_rng(500 + i)))
    return chains


def oracle_run(c, n_blocks):
    ng = c["grid"][2]
    nt = c["u00"].shape[0]
    ukj = np.zeros((nt, ng, 2))
    ukj[:, :, 1] = c["u00"]
    pa = O.PairAction.david_arrays(c["grid"][0], c["grid"][1], ukj, np.zeros_like(ukj), 0, 0)
    s = O.System(c["N"], c["slices"], c["box"], c["tau"], c["lam"], 0)
    s.set_pa(pa)
    s.set_path(c["path"])
    s.bisection_config(c["num_levels"], c["steps_per_block"])
    s.rng_seed(c["seed"])
    recs = s.run_bisection(n_blocks)
    return recs, s.get_path(0), pa


@pytest.mark.parametrize("threads,max_split,ratio", [(64, 0, 0.5), (128, 0, 0.5), (256, 0, 0.5), (256, 2, 0.5),
                                                     (512, 1, 0.5), (512, 2, 0.75)])
def test_batch_matches_oracle_per_chain(threads, max_split, ratio):
    """Whatever group size runs a chain (whole CTA, half or quarter), its
    trace and final path equal the oracle's sequential run of that chain."""
    chains = make_chains()
    b = P.BatchChains(chains, precision=P.FP64, threads_per_cta=threads, ctas=5, max_split=max_split,
                      split_ratio=ratio)
    n_blocks = 25
    trace, stats = b.run(n_blocks, trace=True)
    total = 0
    for i, c in enumerate(chains):
        ref, ref_path, _ = oracle_run(c, n_blocks)
        got = trace[i]
        for k, r in enumerate(ref):
            g = got[k]
            assert (r.slice1, r.ptcl, r.accepted, r.stages_passed) == (
                int(g["slice1"]), int(g["ptcl"]), int(g["accepted"]), int(g["stages_passed"])), (i, k)
            for j in range(8):
                assert abs(r.dS[j] - g["dS"][j]) <= 1e-9 * max(1.0, abs(r.dS[j])), (i, k, j)
        assert np.max(np.abs(b.path(i) - ref_path)) < 1e-9, i
        total += len(ref)
    assert stats["moves"] == total and stats["status"] == 0
    b.close()


@pytest.mark.parametrize("threads,max_split", [(128, 0), (512, 2)])
def test_batch_mixed_matches_oracle_per_chain(threads, max_split):
    """The guarded mixed batch (FP32 pair terms; a stage whose decision lies
    within the mixed sums' bound is decided on its FP64 re-evaluation) makes
    each chain's oracle moves: identical trace, path within 1e-9, and each
    mixed dS within its reported bound of the oracle's FP64 dS."""
    chains = make_chains()
    b = P.BatchChains(chains, precision=P.MIXED, threads_per_cta=threads, ctas=5, max_split=max_split,
                      split_ratio=0.5)
    n_blocks = 25
    trace, stats = b.run(n_blocks, trace=True)
    for i, c in enumerate(chains):
        ref, ref_path, _ = oracle_run(c, n_blocks)
        got = trace[i]
        for k, r in enumerate(ref):
            g = got[k]
            assert (r.slice1, r.ptcl, r.accepted, r.stages_passed) == (
                int(g["slice1"]), int(g["ptcl"]), int(g["accepted"]), int(g["stages_passed"])), (i, k)
            for j in range(8):
                assert abs(r.dS[j] - g["dS"][j]) <= float(g["dS_bound"][j]) + 1e-9 * max(1.0, abs(r.dS[j])), (i, k, j)
        assert np.max(np.abs(b.path(i) - ref_path)) < 1e-9, i
    assert stats["status"] == 0
    assert 0.02 < stats["accepted"] / stats["moves"] < 0.98
    b.close()


def test_batch_mixed_shadow_bound_and_flips():
    """Batched mixed chains with the FP64 sums alongside: the bound holds on
    every stage and no decision flips."""
    chains = make_chains()
    b = P.BatchChains(chains, precision=P.MIXED, shadow=True, threads_per_cta=256)
    trace, stats = b.run(20, trace=True)
    rec = trace.reshape(-1)
    mask = rec["dS_shadow"] != 0.0
    err = np.abs(rec["dS"][mask] - rec["dS_shadow"][mask])
    assert mask.sum() > 100
    assert np.all(err <= rec["dS_bound"][mask].astype(np.float64) + 1e-12)
    assert stats["flips"] == 0 and stats["status"] == 0
    b.close()


def test_batch_autotune_keeps_state_and_graph_replay_matches_oracle():
    chains = make_chains()
    b = P.BatchChains(chains, precision=P.FP64)
    tune = b.autotune(3)
    assert tune["threads_per_cta"] in (128, 256, 384, 512) and tune["ctas"] >= 1
    assert tune["max_split"] in (0, 1, 2)
    for _ in range(3):  # the same launch replayed from its CUDA graph
        b.run_async(5)
    b.synchronize()
    st = b.stats()
    assert st["status"] == 0
    for i in (0, 3, 7, 11):
        _, ref_path, _ = oracle_run(chains[i], 15)
        assert np.max(np.abs(b.path(i) - ref_path)) < 1e-9, i
    b.close()

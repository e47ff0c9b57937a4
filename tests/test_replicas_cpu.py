"""Clone-parallel block pooling over two gloo ranks on the CPU: one
all-reduce per block gives the mean over every clone's energy samples, the
sample-weighted g(r), the pooled histogram and the summed move counters."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BINS = 5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _samples(rank):
    rng = np.random.default_rng(rank)
    terms = ("kinetic", "du_short", "du_long", "v_short", "v_long", "total")
    energies = [dict(zip(terms, rng.normal(size=6))) for _ in range(3 + rank)]
    hist = rng.integers(0, 1000, BINS).astype(np.uint64)
    gofr = rng.random(BINS)
    stats = {"moves": 100 * (rank + 1), "accepted": 30 + rank, "stages_attempted": 250, "pair_evals": 10 ** 6}
    return energies, hist, gofr, 7 + rank, stats


def _fill(block, rank):
    energies, hist, gofr, n, stats = _samples(rank)
    for e in energies:
        block.add_energy(e)
    block.set_gofr(hist, gofr, n)
    block.add_moves(stats)


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from pimcplusplus_b200.replicas import ReplicaBlock
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    b = ReplicaBlock(BINS)
    _fill(b, rank)
    out = b.write_block()
    again = b.write_block()  # reset: an empty block
    q.put((rank, out, again))
    dist.barrier()
    dist.destroy_process_group()


def _expected():
    e_all, h, gw, ng, mv = [], np.zeros(BINS), np.zeros(BINS), 0, {}
    for r in range(2):
        energies, hist, gofr, n, stats = _samples(r)
        e_all += energies
        h += hist
        gw += gofr * n
        ng += n
        for k, v in stats.items():
            mv[k] = mv.get(k, 0) + v
    e = {k: float(np.mean([x[k] for x in e_all])) for k in e_all[0]}
    return e, len(e_all), h, gw / ng, ng, mv


def test_block_pooled_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    e, ne, h, g, ng, mv = _expected()
    for rank, out, again in res:
        assert out["energy_samples"] == ne and out["gofr_samples"] == ng
        for k in e:
            assert abs(out["energy"][k] - e[k]) <= 1e-14 * max(1.0, abs(e[k]))
        assert np.array_equal(out["gofr_histogram"], h.astype(np.uint64))
        assert np.allclose(out["gofr"], g, rtol=1e-14, atol=0)
        assert out["moves"] == mv and out["acceptance"] == mv["accepted"] / mv["moves"]
        assert again["energy_samples"] == 0 and again["moves"]["moves"] == 0


def test_block_without_process_group_is_local():
    sys.path.insert(0, ROOT)
    from pimcplusplus_b200.replicas import ReplicaBlock
    b = ReplicaBlock(BINS)
    _fill(b, 0)
    out = b.write_block()
    energies, hist, gofr, n, stats = _samples(0)
    assert out["energy_samples"] == len(energies)
    assert abs(out["energy"]["total"] - np.mean([x["total"] for x in energies])) < 1e-14
    assert np.allclose(out["gofr"], gofr) and out["moves"] == stats


# ---- one chain set sharded over ranks by cost (clone parallelism of many chains) ----
def _shard_chains():
    sys.path.insert(0, ROOT)
    from pimcplusplus_b200 import workloads as W
    rng = np.random.default_rng(91)
    chains = []
    for i in range(9):
        n = int(rng.choice([8, 12, 16]))
        m = int(rng.choice([8, 16]))
        chains.append(W.lj_chain(n, m, float(rng.uniform(1.0, 4.0)), 0.02186, 2, seed=300 + i, steps_per_block=2,
                                 npts=100, rng=np.random.default_rng(300 + i)))
    return chains


def _chain_counters(c, n_blocks=6):
    """The FP64 oracle's moves of one chain and the counters a block adds."""
    import oracle as O
    ng = c["grid"][2]
    ukj = np.zeros((c["u00"].shape[0], ng, 2))
    ukj[:, :, 1] = c["u00"]
    s = O.System(c["N"], c["slices"], c["box"], c["tau"], c["lam"], 0)
    s.set_pa(O.PairAction.david_arrays(c["grid"][0], c["grid"][1], ukj, np.zeros_like(ukj), 0, 0))
    s.set_path(c["path"])
    s.bisection_config(c["num_levels"], c["steps_per_block"])
    s.rng_seed(c["seed"])
    recs = s.run_bisection(n_blocks)
    L = c["num_levels"]
    stages = sum(r.stages_passed + (0 if r.accepted else 1) for r in recs)
    evals = sum(2 * (c["N"] - 1) * ((1 << L) >> (L - 1 - k))
                for r in recs for k in range(r.stages_passed + (0 if r.accepted else 1)))
    return {"moves": len(recs), "accepted": sum(r.accepted for r in recs), "stages_attempted": stages,
            "pair_evals": evals}


def _shard_rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from pimcplusplus_b200.replicas import ReplicaBlock, shard_by_cost
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    chains = _shard_chains()
    mine = shard_by_cost(chains, rank, world)
    b = ReplicaBlock(0)
    for i in mine:
        b.add_moves(_chain_counters(chains[i]))
    out = b.write_block()
    q.put((rank, mine, out["moves"]))
    dist.barrier()
    dist.destroy_process_group()


def test_chain_set_sharded_by_cost_over_two_gloo_ranks():
    """The two ranks' shards partition the chain set with balanced cost, and
    the counters pooled by one all-reduce equal the single-rank run of every
    chain."""
    sys.path.insert(0, ROOT)
    from pimcplusplus_b200.replicas import chain_cost, shard_by_cost
    chains = _shard_chains()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards = [set(r[1]) for r in res]
    assert shards[0].isdisjoint(shards[1]) and shards[0] | shards[1] == set(range(len(chains)))
    assert [sorted(s) for s in shards] == [shard_by_cost(chains, r, 2) for r in range(2)]
    costs = [sum(chain_cost(chains[i]) for i in s) for s in shards]
    assert max(costs) <= 1.5 * min(costs)
    expect = {}
    for c in chains:
        for k, v in _chain_counters(c).items():
            expect[k] = expect.get(k, 0) + v
    for _, _, pooled in res:
        assert pooled == expect

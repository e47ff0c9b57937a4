"""Clone parallelism over GPUs: one chain per rank, one all-reduce per output block.

PIMC++ runs independent clones of the simulation, each with its own path
and random stream (PIMC++/src/PathDataClass.cc:244-268, the "clones" of the
manual's parallelisation section).  Here a clone is one process with one
GPU; nothing on the move path talks to another rank.  At the end of an
output block, `ReplicaBlock.write_block()` pools the clones' accumulators
with ONE all-reduce of a packed float64 vector (NCCL over NVLink/NVSwitch
when the tensors live on the GPU, gloo on CPUs) and returns the pooled
block averages:

* energy terms: the mean over every clone's samples of the terms
  `PathData.energy()` returns, as EnergyClass::WriteBlock normalises one
  clone's sums by its sample count (Observables/ObservableEnergy.cc:123-163);
* g(r): each clone's normalised g(r) weighted by its sample count, which is
  PairCorrelationClass::WriteBlock's normalisation of the pooled histogram
  when the clones share N, M and the box (Observables/ObservableCorrelation.cc:101-224),
  plus the pooled integer histogram;
* move counters summed, with the acceptance ratio accepted / moves
  (MultiStage.cc:97).

Every rank must call `write_block` at the same point with the same g(r)
grid (the same input file), as for any collective.  Without a process group
the block is the local one.
"""
from __future__ import annotations

import numpy as np

__all__ = ["ReplicaBlock", "ENERGY_TERMS", "MOVE_COUNTERS", "chain_cost", "shard_by_cost"]

ENERGY_TERMS = ("kinetic", "du_short", "du_long", "v_short", "v_long", "total")
MOVE_COUNTERS = ("moves", "accepted", "stages_attempted", "pair_evals")


def chain_cost(chain):
    """Estimated cost of a chain, N^2 M 2^L: N particles moved per sweep, each
    move's stages summing N partners over links that grow as 2^L, M slices
    per sweep.  `chain` is a dict with N, slices (M + 1) and num_levels."""
    return float(chain["N"]) ** 2 * (chain["slices"] - 1) * (1 << chain["num_levels"])


def shard_by_cost(chains, rank, world, cost=chain_cost):
    """Indices of the chains rank `rank` of `world` runs: all chains sorted by
    cost, largest first (ties by index), dealt round-robin, so every rank gets
    a similar share of the work and the shards partition the set.  Each rank
    runs its shard in one batched launch; nothing is exchanged between ranks
    until the block's counters are pooled (one all-reduce)."""
    if not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    order = sorted(range(len(chains)), key=lambda i: (-cost(chains[i]), i))
    return sorted(order[rank::world])


class ReplicaBlock:
    """Accumulators of one output block on this rank, pooled over the ranks by write_block."""

    def __init__(self, gofr_bins=0, group=None, device="cpu"):
        self.gofr_bins = int(gofr_bins)
        self.group = group
        self.device = device
        self.reset()

    def reset(self):
        self.energy_sum = np.zeros(len(ENERGY_TERMS))
        self.energy_samples = 0
        self.gofr_weighted = np.zeros(self.gofr_bins)
        self.gofr_hist = np.zeros(self.gofr_bins)
        self.gofr_samples = 0
        self.moves = np.zeros(len(MOVE_COUNTERS))

    def add_energy(self, terms):
        """One EnergyClass::Accumulate sample: the dict PathData.energy() returns."""
        self.energy_sum += np.array([terms[k] for k in ENERGY_TERMS], dtype=np.float64)
        self.energy_samples += 1

    def set_gofr(self, histogram, gofr, samples):
        """This clone's block g(r): PathData.gofr_get()'s histogram, g(r) and sample count."""
        h = np.asarray(histogram, dtype=np.float64)
        g = np.asarray(gofr, dtype=np.float64)
        if h.shape != (self.gofr_bins,) or g.shape != (self.gofr_bins,):
            raise ValueError(f"g(r) must have {self.gofr_bins} bins")
        self.gofr_hist = h
        self.gofr_weighted = g * float(samples)
        self.gofr_samples = int(samples)

    def add_moves(self, stats):
        """Move counters of this block (differences of BisectionBlock.stats())."""
        self.moves += np.array([float(stats[k]) for k in MOVE_COUNTERS])

    def _pack(self):
        return np.concatenate([[self.energy_samples], self.energy_sum, [self.gofr_samples], self.gofr_weighted,
                               self.gofr_hist, self.moves]).astype(np.float64)

    def write_block(self):
        """Pools the block over the ranks (one all-reduce), returns the
        averages and resets the accumulators."""
        v = self._pack()
        if self.group is not None or _dist_ready():
            import torch
            import torch.distributed as dist
            t = torch.from_numpy(v).to(self.device)
            dist.all_reduce(t, group=self.group)
            v = t.cpu().numpy()
        b = self.gofr_bins
        ne = v[0]
        es = v[1:1 + len(ENERGY_TERMS)]
        o = 1 + len(ENERGY_TERMS)
        ng = v[o]
        gw, gh = v[o + 1:o + 1 + b], v[o + 1 + b:o + 1 + 2 * b]
        mv = v[o + 1 + 2 * b:]
        out = {
            "energy": {k: (s / ne if ne else 0.0) for k, s in zip(ENERGY_TERMS, es)},
            "energy_samples": int(round(ne)),
            "gofr": gw / ng if ng else np.zeros(b),
            "gofr_histogram": np.rint(gh).astype(np.uint64),
            "gofr_samples": int(round(ng)),
            "moves": {k: int(round(x)) for k, x in zip(MOVE_COUNTERS, mv)},
        }
        m = out["moves"]
        out["acceptance"] = m["accepted"] / m["moves"] if m["moves"] else 0.0
        self.reset()
        return out


def _dist_ready():
    try:
        import torch.distributed as dist
    except ImportError:
        return False
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1

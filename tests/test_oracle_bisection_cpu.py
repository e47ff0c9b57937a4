"""The oracle's BisectionBlock moves, pinned against an independent Python
statement of the reference's move (no code shared with the oracle beyond
the Philox stream values, which are pinned by their known answers):

* BisectionBlockClass::ChooseTimeSlices / MakeMove (PIMC++/src/Moves/BisectionBlock.cc:360-451):
  slice1 = LocalInt(NumTimeSlices - 2^L), then StepsPerBlock steps;
* NoPermuteStageClass::Attempt (NoPermuteClass.cc:26-68): particle = LocalInt(N);
* BisectionStageClass::Sample (BisectionStage.cc:128-289): midpoints r̄ + Δ with
  Δ ~ N(0, λτ2^l) per dimension (LocalGaussianVec, the polar method with its
  one-number cache, Common/Random/Random.h:156-180), PutInBox(Δ), and the
  image-summed sample densities of the OLD and NEW midpoints;
* LocalStageClass::Attempt (StageClass.cc:49-95): Kinetic + ShortRange stage
  actions, accept iff logSampleRatio − ΔS + prevΔS ≥ log(Local());
* PathClass::AcceptCopy (PathClass.cc:797-863) with PutInBoxFast, RejectCopy.
"""
import math

import numpy as np
import pytest

import oracle as O
from helpers import lj_case, random_walk_path
from pimcplusplus_b200 import workloads as W
from test_oracle_composition_cpu import kinetic_single, shortrange_single


class LocalStream:
    def __init__(self, seed):
        self.seed, self.n, self.one_left, self.x2 = seed, 0, False, 0.0

    def local(self):
        u = O.philox_uniform(self.seed, 0, self.n)
        self.n += 1
        return u

    def local_int(self, m):
        return int(math.floor(self.local() * m))

    def gaussian(self, sigma):
        if self.one_left:
            self.one_left = False
            return self.x2 * sigma
        while True:
            v1 = 2.0 * self.local() - 1.0
            v2 = 2.0 * self.local() - 1.0
            s = v1 * v1 + v2 * v2
            if s < 1.0:
                break
        t = math.sqrt((-2.0 * math.log(s)) / s)
        self.x2 = v2 * t
        self.one_left = True
        return v1 * t * sigma


def put_in_box(v, box):
    return v - np.floor(v / box + 0.5) * box


def put_in_box_fast(v, box):
    v = v.copy()
    for d in range(3):
        if v[d] > box[d] / 2:
            v[d] -= box[d]
        if v[d] < -box[d] / 2:
            v[d] += box[d]
    return v


def sample(old, new, box, slice1, L, level, p, lam, tau, num_images, rng):
    skip = 1 << (level + 1)
    sigma2 = lam * (0.5 * tau * skip)
    sigma = math.sqrt(sigma2)
    log_new = log_old = 0.0
    for s in range(slice1, slice1 + (1 << L), skip):
        rbar_old = old[s, p] + 0.5 * put_in_box(old[s + skip, p] - old[s, p], box)
        d_old = put_in_box(old[s + skip // 2, p] - rbar_old, box)
        rbar = new[s, p] + 0.5 * put_in_box(new[s + skip, p] - new[s, p], box)
        delta = put_in_box(np.array([rng.gaussian(sigma) for _ in range(3)]), box)
        prod = prod_old = 1.0
        for d in range(3):
            imgs = [i * box[d] for i in range(-num_images, num_images + 1)]
            prod *= sum(math.exp(-0.5 * (delta[d] + x) ** 2 / sigma2) for x in imgs)
            prod_old *= sum(math.exp(-0.5 * (d_old[d] + x) ** 2 / sigma2) for x in imgs)
        log_new += math.log(prod)
        log_old += math.log(prod_old)
        new[s + skip // 2, p] = rbar + delta
    return -log_new + log_old


def run_block(path, box, L, steps, lam, tau, num_images, grid_tabs, rng, n_blocks):
    old, new = path.copy(), path.copy()
    S, N = path.shape[0], path.shape[1]
    records = []
    for _ in range(n_blocks):
        slice1 = rng.local_int(S - (1 << L))
        slice2 = slice1 + (1 << L)
        for _ in range(steps):
            p = rng.local_int(N)
            prev, ok, dss, passed = 0.0, True, [], 0
            for level in range(L - 1, -1, -1):
                lsr = sample(old, new, box, slice1, L, level, p, lam, tau, num_images, rng)
                grid, y, d2y = grid_tabs[level]
                act = [p]
                a_old = (kinetic_single(old, box, act, slice1, slice2, level, lam, tau, num_images) +
                         shortrange_single(old, box, act, slice1, slice2, level, grid, y, d2y))
                a_new = (kinetic_single(new, box, act, slice1, slice2, level, lam, tau, num_images) +
                         shortrange_single(new, box, act, slice1, slice2, level, grid, y, d2y))
                ds = a_new - a_old
                ok = lsr - ds + prev >= math.log(rng.local())
                dss.append(ds)
                passed += ok
                prev = ds
                if not ok:
                    break
            if ok:
                for s in range(slice1, slice2 + 1):
                    new[s, p] = put_in_box_fast(new[s, p], box)
                old[slice1:slice2 + 1, p] = new[slice1:slice2 + 1, p]
            else:
                new[slice1:slice2 + 1, p] = old[slice1:slice2 + 1, p]
            records.append((slice1, p, int(ok), passed, dss))
    return old, records


@pytest.mark.parametrize("num_images,steps", [(0, 1), (1, 2)])
def test_oracle_bisection_matches_independent_moves(tmp_path, num_images, steps):
    cfg, tau, box, dm = lj_case(tmp_path, n=8, m=16, temp=4.0, levels=2, npts=300)
    n, S, L = cfg["N"], cfg["M"] + 1, cfg["levels"]
    lam = W.HE4_LAMBDA
    pa = O.PairAction.from_dm(dm, tau, 0)
    info = pa.info()
    grid = (info["grid_start"], info["grid_end"], info["num_grid"])
    grid_tabs = [(grid, pa.table(0, lv)[:, 1], pa.table(1, lv)[:, 1]) for lv in range(L)]
    path = random_walk_path(n, S, box, 0.3, seed=11)
    path[S - 1] = path[0]
    o = O.System(n, S, box, tau, lam, num_images)
    o.set_pa(pa)
    o.set_path(path)
    o.bisection_config(L, steps, True)
    o.rng_seed(21)
    n_blocks = 12
    recs = o.run_bisection(n_blocks)
    want_path, want = run_block(path, box, L, steps, lam, tau, num_images, grid_tabs, LocalStream(21), n_blocks)
    assert len(recs) == len(want)
    assert sum(r.accepted for r in recs) > 0
    for r, (s1, p, acc, passed, dss) in zip(recs, want):
        assert (r.slice1, r.ptcl, r.accepted, r.stages_passed) == (s1, p, acc, passed)
        for i, ds in enumerate(dss):
            assert abs(r.dS[i] - ds) <= 1e-10 * max(1.0, abs(ds))
    assert np.max(np.abs(o.get_path(0) - want_path)) < 1e-12

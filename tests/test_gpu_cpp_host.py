"""The C++ host layer (include/pimc_b200.hpp) on a B200: a C++ program with
the reference's class names (PathData, ShortRangeClass, KineticClass,
BisectionBlockClass) evaluates actions and runs moves that equal the oracle's."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from helpers import lj_case, random_walk_path
from pimcplusplus_b200 import workloads as W
from test_cpp_host_cpu import build_host_check

pytestmark = pytest.mark.gpu


def test_cpp_host_layer_matches_oracle(tmp_path):
    cfg, tau, box, dm = lj_case(tmp_path, n=24, m=16, levels=2, npts=300)
    n, S, L = cfg["N"], cfg["M"] + 1, cfg["levels"]
    path = random_walk_path(n, S, box, 0.3, seed=23)
    path[S - 1] = path[0]
    pfile = tmp_path / "path.bin"
    path.astype(np.float64).tofile(pfile)
    out = tmp_path / "out.bin"
    exe = build_host_check(tmp_path)
    seed, blocks = 31, 24
    r = subprocess.run([exe, "gpu", dm, repr(tau), repr(float(box[0])), str(n), str(S), str(L), str(seed),
                        str(blocks), str(pfile), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, dtype=np.float64)
    o = O.System(n, S, box, tau, W.HE4_LAMBDA, 0)
    pa = O.PairAction.from_dm(dm, tau, 0)
    o.set_pa(pa)
    o.set_path(path)
    k = 0
    for s1, s2, level, active in ((0, 8, 0, [3]), (4, 12, 1, [1, 5]), (0, 16, 2, [0, 7, 9])):
        a = np.array(active, dtype=np.int32)
        for ref in (o.shortrange_single(s1, s2, a, level), o.kinetic_single(s1, s2, a, level)):
            assert abs(got[k] - ref) <= 1e-12 * max(1.0, abs(ref)), (k, got[k], ref)
            k += 1
    ref = o.shortrange_dbeta(0, S - 1, 0)
    assert abs(got[k] - ref) <= 1e-12 * max(1.0, abs(ref))
    k += 1
    o.bisection_config(L, 1, True)
    o.rng_seed(seed)
    recs = o.run_bisection(blocks)
    rec = got[k:k + 4 * blocks].reshape(blocks, 4)
    k += 4 * blocks
    for r_o, r_g in zip(recs, rec):
        assert (r_o.slice1, r_o.ptcl, r_o.accepted, r_o.stages_passed) == tuple(int(x) for x in r_g)
    assert sum(r.accepted for r in recs) > 0
    assert np.max(np.abs(got[k:].reshape(S, n, 3) - o.get_path(0))) < 1e-9

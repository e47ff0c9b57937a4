"""The allocation-free ShortRange SingleAction entry point.

pimc_shortrange_single_noalloc serves callers that may not allocate device
memory (a memory pool that owns every allocation, an embedding that forbids
allocation after start-up, a latency-critical loop that must not pay for
cudaMalloc's implicit device synchronisation): every
buffer is the caller's, and its scratch is a fixed array inside the library.
It is called here through the C ABI on device buffers this test owns and
compared with the context-based pimc_single_action on the same path, on two
calls in a row (the second reuses the scratch the first left behind).

This file sorts last so that a run stopping at its first failure has run
every other test already.
"""
import ctypes as C

import numpy as np
import pytest

import pimcplusplus_b200 as P
from helpers import lj_case, random_walk_path
from pimcplusplus_b200 import workloads as W

pytestmark = pytest.mark.gpu

REL64 = 1e-12


def test_noalloc_matches_context_entry_point(tmp_path):
    import torch

    cfg, tau, box, dm = lj_case(tmp_path)
    n, slices = cfg["N"], cfg["M"] + 1
    path = random_walk_path(n, slices, box, 0.35, 123, far=0.1)
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.set_path(path)
    d.pa_david_from_dm(dm, 0)
    tables = P.read_dm(dm, tau)
    assert tables["grid_type"] == P.GRID_LINEAR
    # the entry point sums the diagonal u_00 column only: this table has no off-diagonal terms
    assert not np.any(tables["ukj"][:, :, 2:])

    dev_path = torch.tensor(path, dtype=torch.float64, device="cuda:0").contiguous()
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    boxc = np.ascontiguousarray(box, dtype=np.float64)
    stream = torch.cuda.current_stream().cuda_stream
    # two small calls; every particle over all 40 links (163840 terms, 640
    # blocks: the cross-block reduction at scale); a small call after it (the
    # counter the large call left); an empty link range (0, as the context path)
    calls = [(3, 11, [7], 0), (8, 16, [2, 40, 5], 1), (0, 40, list(range(n)), 0), (8, 16, [2, 40, 5], 1),
             (5, 5, [3], 0)]
    for (s1, s2, active, level) in calls:
        lev = level + tables["tau_pos"]
        diag = np.stack([tables["ukj"][lev][:, 1], tables["ukj_d2"][lev][:, 1]], axis=1)
        dev_diag = torch.tensor(diag, dtype=torch.float64, device="cuda:0").contiguous()
        act = np.ascontiguousarray(active, dtype=np.int32)
        rc = P.lib().pimc_shortrange_single_noalloc(
            dev_path.data_ptr(), n, slices, boxc.ctypes.data_as(C.POINTER(C.c_double)), dev_diag.data_ptr(),
            tables["grid_start"], tables["grid_end"], tables["num_grid"], s1, s2,
            act.ctypes.data_as(C.POINTER(C.c_int)), len(act), level, out.data_ptr(), stream)
        assert rc == P.PIMC_OK
        torch.cuda.synchronize()
        got = float(out.item())
        ref = d.single_action(P.ACTION_SHORTRANGE, P.OLDMODE, s1, s2, act, level)
        if s1 == s2:
            assert got == 0.0 and ref == 0.0
        else:
            assert abs(got - ref) <= REL64 * abs(ref), (s1, s2, active, level, got, ref)


def test_noalloc_rejects_oversized_call():
    box = np.array([10.0, 10.0, 10.0])
    act = np.array([0], dtype=np.int32)
    # 600000 particles x 1 link exceeds the 524288-term scratch; rejected before any device work
    rc = P.lib().pimc_shortrange_single_noalloc(
        1, 600000, 3, box.ctypes.data_as(C.POINTER(C.c_double)), 1, 1.0, 5.0, 100, 0, 1,
        act.ctypes.data_as(C.POINTER(C.c_int)), 1, 0, 1, None)
    assert rc == P.PIMC_E_ARG if hasattr(P, "PIMC_E_ARG") else rc == 1


def test_noalloc_matches_oracle_below_grid_start(tmp_path):
    """Against the FP64 oracle directly, on a path where particle 8 sits closer
    to particle 7 than the table's first grid point at every slice (the
    r < rmin clamp of calcUsqzFast), with 7 and 8 both moved (their pair
    counted once) and alone."""
    import torch

    import oracle as O

    cfg, tau, box, dm = lj_case(tmp_path)
    n, slices = cfg["N"], cfg["M"] + 1
    tables = P.read_dm(dm, tau)
    path = random_walk_path(n, slices, box, 0.35, 321, far=0.1)
    path[:, 8, :] = path[:, 7, :] + np.array([0.5 * tables["grid_start"], 0.0, 0.0])
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(O.PairAction.from_dm(dm, tau, 0))
    o.set_path(path)
    dev_path = torch.tensor(path, dtype=torch.float64, device="cuda:0").contiguous()
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    boxc = np.ascontiguousarray(box, dtype=np.float64)
    stream = torch.cuda.current_stream().cuda_stream
    for (s1, s2, active, level) in [(0, 8, [7, 8], 0), (4, 12, [8], 1), (0, 40, [7, 8, 30], 0)]:
        lev = level + tables["tau_pos"]
        diag = np.stack([tables["ukj"][lev][:, 1], tables["ukj_d2"][lev][:, 1]], axis=1)
        dev_diag = torch.tensor(diag, dtype=torch.float64, device="cuda:0").contiguous()
        act = np.ascontiguousarray(active, dtype=np.int32)
        rc = P.lib().pimc_shortrange_single_noalloc(
            dev_path.data_ptr(), n, slices, boxc.ctypes.data_as(C.POINTER(C.c_double)), dev_diag.data_ptr(),
            tables["grid_start"], tables["grid_end"], tables["num_grid"], s1, s2,
            act.ctypes.data_as(C.POINTER(C.c_int)), len(act), level, out.data_ptr(), stream)
        assert rc == P.PIMC_OK
        torch.cuda.synchronize()
        got = float(out.item())
        ref = o.shortrange_single(s1, s2, list(active), level)
        assert abs(got - ref) <= REL64 * abs(ref), (s1, s2, active, level, got, ref)

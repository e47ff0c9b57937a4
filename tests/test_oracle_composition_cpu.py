"""The oracle's composition of the action sums, pinned against a second,
independent numpy statement of the reference's formulas (no shared code with
the oracle beyond the spline tables it is given):

* PathClass::DistDisp (PIMC++/src/PathClass.h:696-746): dispA by nearbyint
  minimum image, dispB on the image consistent with dispA;
* MultiCubicSpline::operator()(i, x) (Common/Splines/CubicSpline.h:470-501)
  with LinearGrid::ReverseMap (Grid.h:81-84) and the [0, N-2] clamp;
* DavidPAClass::calcUsqzFast without off-diagonal terms (DavidPAClass.cc:468-489);
* ShortRangeClass::SingleAction (PIMC++/src/Actions/ShortRangeClass.cc:191-236)
  with DoPtcl's count-once rule over links [slice1, slice2) step 2^level;
* KineticClass::SingleAction (PIMC++/src/Actions/KineticClass.cc:33-90) with
  PathClass::Velocity's PutInBox (PathClass.h:831-865) and the image sums.
"""
import math

import numpy as np
import pytest

import oracle as O
from helpers import lj_case, random_walk_path
from pimcplusplus_b200 import workloads as W


def spline_eval(start, end, n, y, d2y, x):
    delta = (end - start) / (n - 1)
    hi = np.rint((x - start) / delta - 0.5).astype(np.int64) + 1
    lo = hi - 1
    lo = np.where(lo < 0, 0, lo)
    hi = np.where(lo == 0, np.maximum(hi, 1), hi)
    over = hi > n - 1
    hi = np.where(over, n - 1, hi)
    lo = np.where(over, n - 2, lo)
    xs = start + np.arange(n) * delta
    h = xs[hi] - xs[lo]
    a = (xs[hi] - x) / h
    b = (x - xs[lo]) / h
    return a * y[lo] + b * y[hi] + ((a ** 3 - a) * d2y[lo] + (b ** 3 - b) * d2y[hi]) * (h * h / 6.0)


def dist_disp(pa1, pa2, pb1, pb2, box):
    dA = pa2 - pa1
    dB = pb2 - pb1
    dA = dA + (-np.rint(dA / box)) * box
    dB = dB + np.rint((dA - dB) / box) * box
    return np.sqrt(np.sum(dA * dA, -1)), np.sqrt(np.sum(dB * dB, -1))


def shortrange_single(path, box, active, s1, s2, level, grid, y, d2y):
    start, end, n = grid
    skip = 1 << level
    N = path.shape[1]
    total = 0.0
    visited = np.zeros(N, dtype=bool)
    for p1 in active:
        visited[p1] = True
        partners = np.nonzero(~visited)[0]
        for s in range(s1, s2, skip):
            r, rp = dist_disp(path[s, p1], path[s, partners], path[s + skip, p1], path[s + skip, partners], box)
            r = np.minimum(r, end)
            rp = np.minimum(rp, end)
            low = (r < start) | (rp < start)
            u = 0.5 * (spline_eval(start, end, n, y, d2y, r) + spline_eval(start, end, n, y, d2y, rp))
            u = np.where(low, spline_eval(start, end, n, y, d2y, np.array([start]))[0], u)
            total += float(np.sum(u))
    return total


def kinetic_single(path, box, active, s1, s2, level, lam, tau, num_images):
    skip = 1 << level
    f = 1.0 / (4.0 * lam * tau * skip)
    total = 0.0
    for p in active:
        for s in range(s1, s2, skip):
            v = path[s + skip, p] - path[s, p]
            v = v - np.floor(v / box + 0.5) * box
            imgs = np.arange(-num_images, num_images + 1)[:, None] * box[None, :]
            total -= np.log(np.prod(np.sum(np.exp(-(v[None, :] + imgs) ** 2 * f), axis=0)))
    return total


def test_oracle_shortrange_composition(tmp_path):
    cfg, tau, box, dm = lj_case(tmp_path, n=24, m=16, levels=3, npts=400)
    n, slices = cfg["N"], cfg["M"] + 1
    pa = O.PairAction.from_dm(dm, tau, 0)
    info = pa.info()
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(pa)
    rng = np.random.default_rng(4)
    for trial in range(3):
        path = random_walk_path(n, slices, box, 0.35, seed=70 + trial, far=0.2)
        o.set_path(path)
        for s1, s2, level, active in ((0, 16, 0, [5]), (4, 12, 1, [2, 9, 2]), (0, 16, 2, list(rng.permutation(n)[:6])),
                                      (8, 16, 3, [0, 23])):
            y = pa.table(0, level)[:, 1]
            d2y = pa.table(1, level)[:, 1]
            grid = (info["grid_start"], info["grid_end"], info["num_grid"])
            want = shortrange_single(path, box, active, s1, s2, level, grid, y, d2y)
            got = o.shortrange_single(s1, s2, np.array(active, dtype=np.int32), level)
            assert abs(got - want) <= 1e-12 * max(1.0, abs(want)), (trial, s1, s2, level, active, got, want)


@pytest.mark.parametrize("num_images", [0, 1])
def test_oracle_kinetic_composition(num_images):
    n, slices, tau, lam = 10, 17, 0.02, 6.0596
    box = np.array([6.0, 7.0, 8.0])
    o = O.System(n, slices, box, tau, lam, num_images)
    path = random_walk_path(n, slices, box, 0.5, seed=3, far=0.3)
    o.set_path(path)
    for s1, s2, level, active in ((0, 16, 0, [1]), (2, 10, 1, [0, 4]), (0, 16, 3, [9, 3, 5])):
        want = kinetic_single(path, box, active, s1, s2, level, lam, tau, num_images)
        got = o.kinetic_single(s1, s2, np.array(active, dtype=np.int32), level)
        assert abs(got - want) <= 1e-12 * max(1.0, abs(want)), (s1, s2, level, active, got, want)


def shortrange_dbeta(path, box, s1, s2, level, grid, tabs):
    """ShortRangeClass::d_dBeta (ShortRangeClass.cc:316-355) over all pairs
    p2 < p1 with DavidPAClass::calcUsqz's diagonal part (DavidPAClass.cc:291-366):
    r, r' clamped to [rmin, End], dU = ½(du₁(r)+du₁(r')) + ½(V(r)+V(r')), V the column 0."""
    start, end, n = grid
    (uy, ud2), (dy, dd2) = tabs
    skip = 1 << level
    N = path.shape[1]
    total = 0.0
    for p1 in range(N):
        p2 = np.arange(p1)
        if p2.size == 0:
            continue
        for s in range(s1, s2, skip):
            r, rp = dist_disp(path[s, p1], path[s, p2], path[s + skip, p1], path[s + skip, p2], box)
            r = np.clip(r, start, end)
            rp = np.clip(rp, start, end)
            v = 0.5 * (spline_eval(start, end, n, uy[:, 0], ud2[:, 0], r) +
                       spline_eval(start, end, n, uy[:, 0], ud2[:, 0], rp))
            du = 0.5 * (spline_eval(start, end, n, dy[:, 1], dd2[:, 1], r) +
                        spline_eval(start, end, n, dy[:, 1], dd2[:, 1], rp))
            total += float(np.sum(du + v))
    return total


def test_oracle_shortrange_dbeta_composition(tmp_path):
    cfg, tau, box, dm = lj_case(tmp_path, n=20, m=16, levels=2, npts=400)
    n, slices = cfg["N"], cfg["M"] + 1
    pa = O.PairAction.from_dm(dm, tau, 0)
    info = pa.info()
    grid = (info["grid_start"], info["grid_end"], info["num_grid"])
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(pa)
    path = random_walk_path(n, slices, box, 0.35, seed=91, far=0.2)
    o.set_path(path)
    for s1, s2, level in ((0, 16, 0), (4, 12, 1), (0, 16, 2)):
        tabs = ((pa.table(0, level), pa.table(1, level)), (pa.table(2, level), pa.table(3, level)))
        want = shortrange_dbeta(path, box, s1, s2, level, grid, tabs)
        got = o.shortrange_dbeta(s1, s2, level)
        assert abs(got - want) <= 1e-12 * max(1.0, abs(want)), (s1, s2, level, got, want)


def longrange_single(path, kv, s1, s2, level, ulong_k, ulong_r0, ushort_k0, ulong_k0, use_background):
    """LongRangeClass::SingleAction (LongRangeClass.cc:273-371), one species:
    rho_k(slice) = sum_i exp(i k.r_i) computed directly (CalcRho_ks_Fast builds
    the same phases by recurrence), ends of [slice1, slice2] weighted 1/2."""
    skip = 1 << level
    N = path.shape[1]
    homo = background = k0 = 0.0
    for s in range(s1, s2 + 1, skip):
        f = 0.5 if s in (s1, s2) else 1.0
        rho = np.exp(1j * (path[s] @ kv.T)).sum(axis=0)
        homo += f * 0.5 * 2.0 * float(np.sum(np.abs(rho) ** 2 * ulong_k[level]))
        homo -= f * 0.5 * N * ulong_r0[level]
        background -= f * 0.5 * N * N * ushort_k0[level]
        k0 += f * 0.5 * N * N * ulong_k0[level]
    return homo + (background if use_background else k0)


@pytest.mark.parametrize("use_background", [True, False])
def test_oracle_longrange_composition(use_background):
    n, m, levels = 12, 16, 3
    box = np.array([7.0, 8.0, 9.0])
    o = O.System(n, m + 1, box, 0.05, 0.5, 0)
    pa = O.PairAction.classical_coulomb(0.05, levels, 2.0)  # IsLongRange: the k sum is taken
    o.set_pa(pa)
    path = random_walk_path(n, m + 1, box, 0.4, seed=17, far=0.2)
    o.set_path(path)
    nk = o.setup_kvecs(2.2)
    kv, _ = o.kvecs()
    rng = np.random.default_rng(5)
    tabs = dict(ulong_k=rng.normal(size=(levels, nk)), ulong_r0=rng.normal(size=levels),
                ushort_k0=rng.normal(size=levels), ulong_k0=rng.normal(size=levels))
    o.set_longrange(tabs["ulong_k"], tabs["ulong_r0"], tabs["ushort_k0"], tabs["ulong_k0"],
                    np.zeros((levels, nk)), np.zeros(levels), np.zeros(levels), np.zeros(levels), use_background)
    o.calc_rhok_all()
    for s1, s2, level in ((0, 8, 0), (4, 12, 1), (0, 16, 2)):
        want = longrange_single(path, kv, s1, s2, level, use_background=use_background, **tabs)
        got = o.longrange_single(s1, s2, np.array([3], dtype=np.int32), level)
        assert abs(got - want) <= 1e-11 * max(1.0, abs(want)), (s1, s2, level, got, want)


def log_spline_eval(r0, spacing, n, y, d2y, x):
    """MultiCubicSpline::operator()(col, x) on a LogGrid: nodes r0·spacing^i,
    ReverseMap floor(log(x/r0)/log(spacing)) (Grid.h:527-530), cell clamped."""
    xs = np.array([r0 * spacing ** i for i in range(n)])
    lo = int(math.floor(math.log(x / r0) / math.log(spacing)))
    lo = min(max(lo, 0), n - 2)
    hi = lo + 1
    h = xs[hi] - xs[lo]
    a = (xs[hi] - x) / h
    b = (x - xs[lo]) / h
    return a * y[lo] + b * y[hi] + ((a ** 3 - a) * d2y[lo] + (b ** 3 - b) * d2y[hi]) * (h * h / 6.0)


def david_U(q, z, s, level_tables, r0, spacing, n, end, num_terms):
    """DavidPAClass::calcUsqzFast (DavidPAClass.cc:468-511) with off-diagonal
    terms u_kj(q) z^{2j} s^{2(k-j)}, column k(k+1)/2 + j + 1."""
    y, d2y = level_tables
    col = lambda c, x: log_spline_eval(r0, spacing, n, y[:, c], d2y[:, c], x)
    r, rp = min(q + 0.5 * z, end), min(q - 0.5 * z, end)
    if rp < r0 or r < r0:
        return col(1, r0)
    U = 0.5 * (col(1, r) + col(1, rp))
    if s > 0.0 and q < end:
        for k in range(1, num_terms + 1):
            for j in range(k + 1):
                U += col(k * (k + 1) // 2 + j + 1, q) * z ** (2 * j) * s ** (2 * (k - j))
    return U


def test_oracle_david_offdiagonal_log_grid(tmp_path):
    from helpers import write_testcoul_dm
    tau = 1.0 / 64
    pa = O.PairAction.from_dm(write_testcoul_dm(str(tmp_path / "tc.dm")), tau, 2)
    info = pa.info()
    assert info["grid_type"] == 1
    n, r0, end = info["num_grid"], info["grid_start"], info["grid_end"]
    spacing = (end / r0) ** (1.0 / (n - 1))
    rng = np.random.default_rng(12)
    for level in range(3):
        tabs = (pa.table(0, level), pa.table(1, level))
        for _ in range(150):
            q = rng.uniform(0.5 * r0, 1.1 * end)
            z = rng.uniform(-1.0, 1.0) * min(q, 2.0)
            s = abs(z) + rng.uniform(0.0, 1.0)
            want = david_U(q, z, s, tabs, r0, spacing, n, end, 2)
            got = pa.U(q, z, s * s, level)
            assert abs(got - want) <= 1e-11 * max(1.0, abs(want)), (level, q, z, s, got, want)


def kinetic_dbeta(path, box, s1, s2, level, lam, tau, num_images):
    """KineticClass::d_dBeta (KineticClass.cc:187-256): 3/(2 τ_l) per link plus
    the image-summed spring term Σ_dim (∂ ln Z_dim) of each link."""
    skip = 1 << level
    lt = tau * skip
    f = 1.0 / (4.0 * lam * lt)
    spring = 0.0
    imgs = np.arange(-num_images, num_images + 1)
    for p in range(path.shape[1]):
        for s in range(s1, s2, skip):
            spring += 1.5 / lt
            v = path[s + skip, p] - path[s, p]
            v = v - np.floor(v / box + 0.5) * box
            d = v[:, None] + imgs[None, :] * box[:, None]
            e = np.exp(-d * d * f)
            gauss = e.sum(axis=1)
            num = (-(d * d * f) / lt * e).sum(axis=1)
            spring += sum(num[k] * np.prod(np.delete(gauss, k)) for k in range(3)) / np.prod(gauss)
    return spring


@pytest.mark.parametrize("num_images", [0, 1])
def test_oracle_kinetic_dbeta_composition(num_images):
    n, slices, tau, lam = 10, 17, 0.02, 6.0596
    box = np.array([6.0, 7.0, 8.0])
    o = O.System(n, slices, box, tau, lam, num_images)
    path = random_walk_path(n, slices, box, 0.5, seed=8, far=0.3)
    o.set_path(path)
    for s1, s2, level in ((0, 16, 0), (4, 12, 1), (0, 16, 2)):
        want = kinetic_dbeta(path, box, s1, s2, level, lam, tau, num_images)
        got = o.kinetic_dbeta(s1, s2, level)
        assert abs(got - want) <= 1e-11 * max(1.0, abs(want)), (s1, s2, level, got, want)


def test_oracle_energy_composition(tmp_path):
    """ActionsClass::Energy (ActionsClass.cc:812-871) as EnergyClass::Accumulate
    sums it (ObservableEnergy.cc:31-73): kinetic and dUShort over links [0, M),
    vShort = ShortRangePotClass::V summed over slices with ½ at 0 and M
    (ShortRangePotClass.cc:28-47; one-slice DistDisp, PathClass.h:636-662;
    DavidPAClass::V = column 0 of the first tau table, r clamped to the grid)."""
    cfg, tau, box, dm = lj_case(tmp_path, n=14, m=16, levels=2, npts=400)
    n, S = cfg["N"], cfg["M"] + 1
    M = S - 1
    pa = O.PairAction.from_dm(dm, tau, 0)
    info = pa.info()
    grid = (info["grid_start"], info["grid_end"], info["num_grid"])
    o = O.System(n, S, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(pa)
    path = random_walk_path(n, S, box, 0.35, seed=29, far=0.2)
    o.set_path(path)
    e = o.energy()
    kin = kinetic_dbeta(path, box, 0, M, 0, W.HE4_LAMBDA, tau, 0)
    tabs = ((pa.table(0, 0), pa.table(1, 0)), (pa.table(2, 0), pa.table(3, 0)))
    dus = shortrange_dbeta(path, box, 0, M, 0, grid, tabs)
    v = 0.0
    y0, d2y0 = pa.table(0, 0)[:, 0], pa.table(1, 0)[:, 0]
    for s in range(S):
        f = 0.5 if s in (0, M) else 1.0
        for p1 in range(n):
            d = path[s, :p1] - path[s, p1]
            d = d - np.rint(d / box) * box
            r = np.clip(np.sqrt(np.sum(d * d, axis=1)), grid[0], grid[1])
            v += f * float(np.sum(spline_eval(*grid, y0, d2y0, r)))
    for got, want in ((e["kinetic"], kin), (e["du_short"], dus), (e["v_short"], v),
                      (e["total"], (kin + dus) / M)):
        assert abs(got - want) <= 1e-11 * max(1.0, abs(want)), (got, want)

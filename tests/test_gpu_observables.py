"""Energy and g(r) estimators on the device against the oracle: the terms of
ActionsClass::Energy and the PairCorrelationClass histogram on fixed paths,
the estimator series along a replayed chain, and a statistical comparison of
an independent mixed-precision chain with the FP64 oracle's chain (agreement
within 2 sigma, errors from blocking)."""
import numpy as np
import pytest

import oracle as O
import pimcplusplus_b200 as P
from pimcplusplus_b200 import workloads as W

from helpers import lj_case, random_walk_path, rel_err, tricubic_case

pytestmark = pytest.mark.gpu

TERMS = ("kinetic", "du_short", "du_long", "v_short", "total")


def gofr_norm(hist, counts, n, m, box, start, end):
    """PairCorrelationClass::WriteBlock normalisation (ObservableCorrelation.cc:101-135)."""
    nb = len(hist)
    delta = (end - start) / nb
    vol = box[0] * box[1] * box[2]
    norm = 0.5 * counts * m * (n * (n - 1.0)) / vol
    r1 = start + np.arange(nb) * delta
    r2 = start + (np.arange(nb) + 1) * delta
    return hist / (4.0 * np.pi / 3 * (r2 ** 3 - r1 ** 3) * norm)


def test_energy_terms_david(tmp_path):
    cfg, tau, box, dm = lj_case(tmp_path)
    n, slices = cfg["N"], cfg["M"] + 1
    path = random_walk_path(n, slices, box, 0.3, 5, far=2.0)
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(O.PairAction.from_dm(dm, tau, 0))
    o.set_path(path)
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.pa_david_from_dm(dm, 0)
    d.set_path(path)
    ref, got = o.energy(), d.energy()
    for k in TERMS:
        assert rel_err(got[k], ref[k], max(abs(ref[k]), 1e-6)) < 1e-12, (k, got[k], ref[k])
    d.close()


def test_energy_terms_tricubic():
    cfg, tau, box, tabs = tricubic_case()
    qg, yg, tg, umat, dumat, pg, pot = tabs
    n, slices = cfg["N"], cfg["M"] + 1
    path = random_walk_path(n, slices, box, 0.3, 9)
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(O.PairAction.tricubic(qg, yg, tg, tau, umat, dumat, pg, pot))
    o.set_path(path)
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.pa_tricubic(qg, yg, tg, tau, umat, dumat, pg, pot)
    d.set_path(path)
    ref, got = o.energy(), d.energy()
    for k in TERMS:
        assert rel_err(got[k], ref[k], max(abs(ref[k]), 1e-6)) < 1e-12, (k, got[k], ref[k])
    d.close()


@pytest.mark.parametrize("start,end,points", [(0.0, 0.0, 201), (0.5, 9.0, 64), (0.0, 40.0, 4097)])
def test_gofr_histogram_exact(tmp_path, start, end, points):
    cfg, tau, box, dm = lj_case(tmp_path)
    n, slices = cfg["N"], cfg["M"] + 1
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.pa_david_from_dm(dm, 0)
    d.gofr_setup(start, end, points)
    e = box[0] if end <= 0 else end
    ref = np.zeros(points - 1, dtype=np.uint64)
    for seed in (1, 2):
        path = random_walk_path(n, slices, box, 0.5, seed, far=1.5)
        o.set_path(path)
        o.gofr_accumulate(start, e, points, ref)
        d.set_path(path)
        d.gofr_accumulate()
    hist, g, counts = d.gofr_get()
    assert counts == 2
    assert np.array_equal(hist, ref)
    assert np.allclose(g, gofr_norm(ref.astype(float), 2, n, cfg["M"], box, start, e), rtol=1e-12, atol=0)
    d.gofr_reset()
    h2, _, c2 = d.gofr_get()
    assert c2 == 0 and not h2.any()
    d.close()


def small_system(tmp_path, n=32, m=20, temp=2.0, levels=2):
    cfg = dict(N=n, M=m, T=temp, rho=0.02186, levels=levels, npts=1000)
    tau, box = W.derived(cfg)
    dm = W.make_dm_for(cfg, str(tmp_path))
    return cfg, tau, box, dm


def test_estimators_along_replayed_chain(tmp_path):
    """FP64 device moves and the oracle on the same stream: the energy and
    g(r) samples of every block agree."""
    cfg, tau, box, dm = small_system(tmp_path)
    n, slices, L = cfg["N"], cfg["M"] + 1, cfg["levels"]
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(O.PairAction.from_dm(dm, tau, 0))
    o.init_random_fixed(41, 0.45 * W.LJ_SIGMA)
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.pa_david_from_dm(dm, 0)
    d.set_path(o.get_path(0))
    d.gofr_setup(0.0, 0.0, 101)
    spb = 20
    o.bisection_config(L, spb)
    o.rng_seed(13)
    bb = P.BisectionBlock(d, L, spb, precision=P.FP64, cluster_ctas=1, threads_per_cta=128, schedule=P.SEQUENTIAL)
    bb.seed(13)
    ref_h = np.zeros(100, dtype=np.uint64)
    for blk in range(30):
        o.run_bisection(1)
        bb.MakeMoves(1, trace=False)
        er, eg = o.energy(), d.energy()
        assert rel_err(eg["total"], er["total"], max(abs(er["total"]), 1.0)) < 1e-10, blk
        assert rel_err(eg["v_short"], er["v_short"], max(abs(er["v_short"]), 1.0)) < 1e-10, blk
        o.gofr_accumulate(0.0, box[0], 101, ref_h)
        d.gofr_accumulate()
    hist, _, counts = d.gofr_get()
    assert counts == 30
    assert np.array_equal(hist, ref_h)
    d.close()


def blocked(x, nblocks):
    x = np.asarray(x)
    k = len(x) // nblocks
    b = x[: k * nblocks].reshape((nblocks, k) + x.shape[1:]).mean(axis=1)
    return b.mean(axis=0), b.std(axis=0, ddof=1) / np.sqrt(nblocks)


@pytest.mark.parametrize("size", ["small", "C1"])
def test_energy_and_gofr_within_2sigma_mixed_vs_oracle(tmp_path, size):
    """An independent mixed-precision device chain (concurrent windows, own
    seed) and the FP64 oracle's sequential chain sample the same
    distribution: energy and g(r) agree within 2 combined sigma.  Sizes: 32
    atoms, M = 20, level 2; and C1 (64 atoms, M = 40, T = 2 K, level 3)."""
    if size == "C1":
        cfg, tau, box, dm = small_system(tmp_path, n=64, m=40, temp=2.0, levels=3)
        burn, sweeps, nb = 100, 800, 10
    else:
        cfg, tau, box, dm = small_system(tmp_path)
        burn, sweeps, nb = 150, 1200, 12
    n, slices, L = cfg["N"], cfg["M"] + 1, cfg["levels"]
    windows = (slices - 1) >> L
    per_sweep = n * windows  # one sweep = N ceil(M / 2^L) bisection attempts
    o = O.System(n, slices, box, tau, W.HE4_LAMBDA, 0)
    o.set_pa(O.PairAction.from_dm(dm, tau, 0))
    o.init_random_fixed(43, 0.45 * W.LJ_SIGMA)
    start = o.get_path(0)
    o.bisection_config(L, per_sweep)
    o.rng_seed(101)
    d = P.PathData(n, slices, box, tau, W.HE4_LAMBDA, 0)
    d.pa_david_from_dm(dm, 0)
    d.set_path(start)
    d.gofr_setup(0.0, box[0] / 2, 41)
    bb = P.BisectionBlock(d, L, n, precision=P.MIXED, cluster_ctas=1, threads_per_cta=128, schedule=P.WINDOWS)
    bb.seed(202)
    e_o, e_d, g_o, g_d = [], [], [], []
    for sw in range(burn + sweeps):
        o.run_bisection(1)
        bb.MakeMoves(1, trace=False)
        if sw < burn:
            continue
        e_o.append(o.energy()["total"])
        e_d.append(d.energy()["total"])
        h = o.gofr_accumulate(0.0, box[0] / 2, 41)
        g_o.append(gofr_norm(h.astype(float), 1, n, cfg["M"], box, 0.0, box[0] / 2))
        d.gofr_reset()
        d.gofr_accumulate()
        g_d.append(d.gofr_get()[1])
    mo, so = blocked(e_o, nb)
    md, sd = blocked(e_d, nb)
    comb = np.hypot(so, sd)
    assert abs(mo - md) <= 2.0 * comb, (mo, so, md, sd)
    go, sgo = blocked(g_o, nb)
    gd, sgd = blocked(g_d, nb)
    sig = np.hypot(sgo, sgd)
    live = sig > 0
    z = np.abs(go - gd)[live] / sig[live]
    assert np.mean(z < 2.0) >= 0.85 and z.max() < 5.0, (np.mean(z < 2.0), z.max())
    d.close()

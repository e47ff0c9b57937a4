"""Synthetic inputs for the benchmark configurations.

The reference ships no Lennard-Jones potential and no He-4 squarer table
(its He4.95.dm is absent), so the LJ helium workloads are built here as
drop-in files in the reference's own formats:

* a primitive-approximation squarer `.dm` file (u_00 = tau_l V(r), other
  u_kj = 0, du table 0 because the reader adds the potential back), read by
  the DavidPA reader exactly like a squarer output
  (Common/PairAction/DavidPAClass.cc:635-912);
* tricubic u(q, y, t) node tables for PAtricubicFitClass
  (Common/PairAction/PAtricubicFit.cc:659-721,794-865): the primitive action
  1/2 beta (V(r) + V(r')) plus a smooth off-diagonal term c beta s^2 g(q) so
  that the t-dependence is exercised.  The physics is synthetic; parity is
  over the evaluation.

Units: Angstrom, Kelvin; lambda = hbar^2/2m = 6.0596 K A^2 for He-4.
"""
from __future__ import annotations

import math
import os

import numpy as np

HE4_LAMBDA = 6.0596
LJ_EPS = 10.22
LJ_SIGMA = 2.556


def lj(r, eps=LJ_EPS, sigma=LJ_SIGMA):
    sr6 = (sigma / np.asarray(r, dtype=np.float64)) ** 6
    return 4.0 * eps * (sr6 * sr6 - sr6)


def lj_truncated(r, rc, eps=LJ_EPS, sigma=LJ_SIGMA):
    """LJ truncated and shifted to zero at rc (so all-pairs and cell-list sums agree)."""
    r = np.asarray(r, dtype=np.float64)
    v = lj(r, eps, sigma) - lj(rc, eps, sigma)
    return np.where(r < rc, v, 0.0)


def box_for_density(n, rho):
    side = (n / rho) ** (1.0 / 3.0)
    return np.array([side, side, side])


def _fmt_block(vals, per_line=5):
    out = []
    for i in range(0, len(vals), per_line):
        out.append(" " + " ".join(f"{v: .17e}" for v in vals[i:i + per_line]))
    return "\n".join(out)


def write_primitive_dm(path, r_min, r_max, npts, tau0, ntau, potential, grid="LINEAR", species="He4",
                       lam=HE4_LAMBDA):
    """Writes an ASCII squarer file in the layout ReadDavidSquarerFile parses.

    Fits 0..2 are written (the reader builds its splines only from the fit
    with NMax == 2); u_00 = tau_l * V(r) with tau_l = tau0 * 2^l, all other
    u_kj and the beta-derivative tables are zero.
    """
    if grid == "LINEAR":
        r = r_min + np.arange(npts) * ((r_max - r_min) / (npts - 1))
    elif grid == "LOG":
        delta = (r_max / r_min) ** (1.0 / (npts - 1.0))
        r = r_min * delta ** np.arange(npts)
    else:
        raise ValueError(grid)
    v = potential(r)
    taus = tau0 * 2.0 ** np.arange(ntau)
    r_min, r_max = float(r_min), float(r_max)
    t_lo, t_hi = float(taus[0]), float(taus[-1])
    lines = [" UNITS K A", f" TYPE {species} {lam}", f" GRID {npts} {grid} {r_min!r} {r_max!r}",
             f" SQUARER {t_hi!r} {ntau} 3 2 0 0", " POT PRIMITIVE", " RANK 2 %d 1" % npts,
             f" GRID 1 {grid} {r_min!r} {r_max!r}", " LABEL 1 r", " BEGIN potential 0", _fmt_block(v)]
    for derv in (1, 2):
        for fit in range(3):
            nukj = (fit + 1) * (fit + 2) // 2
            table = np.zeros((ntau, nukj, npts))
            if derv == 1:
                table[:, 0, :] = taus[:, None] * v[None, :]
            lines += [f" RANK 3 {npts} {nukj} {ntau}", f" GRID 1 {grid} {r_min!r} {r_max!r}", " LABEL 1 r",
                      f" GRID   3 LOG {t_lo!r} {t_hi!r}", " LABEL 2 terms", " LABEL 3 time",
                      f" BEGIN density matrix table fit= {fit} derv = {derv}", _fmt_block(table.reshape(-1))]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def tricubic_tables(box_side, tau, num_betas, nq=200, ny=50, nt=50, r_cap=1.5, c_off=1.0, pot_n=2000):
    """Node tables for PAtricubicFitClass on linear q in [0, L/2], y, t in [0, 1].

    Returns (qgrid, ygrid, tgrid, umat, dumat, pot_grid, pot_data).
    """
    qg = (0.0, box_side / 2.0, nq)
    yg = (0.0, 1.0, ny)
    tg = (0.0, 1.0, nt)
    q = np.linspace(qg[0], qg[1], nq)[:, None, None]
    y = np.linspace(0.0, 1.0, ny)[None, :, None]
    t = np.linspace(0.0, 1.0, nt)[None, None, :]
    z = y * 2.0 * q
    s = z + t * (2.0 * q - z)
    r = q + 0.5 * z
    rp = q - 0.5 * z
    vc = lambda x: lj(np.maximum(x, r_cap))
    base = 0.5 * (vc(r) + vc(rp))
    off = c_off * s * s * np.exp(-(q / LJ_SIGMA) ** 2)
    betas = tau * 2.0 ** np.arange(num_betas)
    umat = np.stack([b * (base + off) for b in betas])
    dumat = np.stack([base + off for _ in betas])
    pot_grid = (r_cap, box_side * math.sqrt(3.0) / 2.0 + 1.0, pot_n)
    pr = np.linspace(pot_grid[0], pot_grid[1], pot_n)
    return qg, yg, tg, umat, dumat, pot_grid, lj(pr)


# ---------------------------------------------------------------------------
# The benchmark configurations (synthetic stand-ins with the stated sizes).
# ---------------------------------------------------------------------------
CONFIGS = {
    "C1": dict(name="64 LJ He-4, M=40, T=2.0 K, primitive 1-D table, level 3", N=64, M=40, T=2.0, rho=0.02186,
               levels=3, table="dm", npts=1000),
    "C2": dict(name="512 LJ He-4, M=128, T=1.5 K, tricubic 200x50x50, level 4", N=512, M=128, T=1.5, rho=0.02186,
               levels=4, table="tricubic", nq=200, ny=50, nt=50),
    "C5": dict(name="4096 LJ He-4, M=256, T=1.0 K, truncated LJ (2.5 sigma) 1-D table, level 5", N=4096, M=256,
               T=1.0, rho=0.02186, levels=5, table="dm", npts=1000, rcut=2.5 * LJ_SIGMA),
}


def derived(cfg):
    beta = 1.0 / cfg["T"]
    tau = beta / cfg["M"]
    box = box_for_density(cfg["N"], cfg["rho"])
    return tau, box


def make_dm_for(cfg, directory, r_min=1.5):
    tau, box = derived(cfg)
    rc = cfg.get("rcut")
    pot = (lambda r: lj_truncated(r, rc)) if rc else lj
    path = os.path.join(directory, f"lj_{cfg['N']}_{cfg['M']}.dm")
    # a truncated table ends at its cutoff: the reader zeroes the last row, so
    # every pair at or beyond rc contributes exactly zero
    write_primitive_dm(path, r_min, rc if rc else box[0] / 2.0, cfg["npts"], tau, cfg["levels"] + 1, pot)
    return path


def lj_chain(n, m, temp, rho, levels, seed, steps_per_block=1, npts=200, r_min=1.5, rng=None):
    """One LJ He-4 chain for the batched driver: its diagonal primitive
    action u_00(r; tau_l) = tau_l V(r) on a linear grid [r_min, L/2] (last
    point zeroed as the .dm reader does) and a seeded initial path."""
    tau = 1.0 / (temp * m)
    box = box_for_density(n, rho)
    r = r_min + np.arange(npts) * ((box[0] / 2.0 - r_min) / (npts - 1))
    v = lj(r)
    taus = tau * 2.0 ** np.arange(levels + 1)
    u00 = taus[:, None] * v[None, :]
    u00[:, -1] = 0.0
    rng = rng or np.random.default_rng(seed)
    pts = np.zeros((n, 3))
    for i in range(n):
        for _ in range(1000):
            c = (rng.random(3) - 0.5) * box
            d = pts[:i] - c
            d -= np.round(d / box) * box
            if i == 0 or np.min(np.sum(d * d, axis=1)) >= (0.9 * LJ_SIGMA) ** 2:
                break
        pts[i] = c
    path = np.repeat(pts[None], m + 1, axis=0)
    return dict(N=n, slices=m + 1, box=box, tau=tau, lam=HE4_LAMBDA, num_levels=levels,
                steps_per_block=steps_per_block, seed=seed, grid=(r_min, float(box[0] / 2.0), npts), u00=u00,
                tau_pos=0, path=path)


def lattice_path(n, slices, box, rng, jitter=0.1):
    """n particles spread evenly over the sites of the smallest simple-cubic
    lattice with at least n sites filling the box, each displaced by up to
    +-jitter of the lattice spacing, copied to every slice (a classical
    start: no overlaps at liquid densities)."""
    side = int(np.ceil(n ** (1.0 / 3.0) - 1e-9))
    idx = (np.arange(n) * side ** 3) // n
    ijk = np.stack([idx // (side * side), (idx // side) % side, idx % side], axis=1).astype(np.float64)
    a = np.asarray(box, dtype=np.float64) / side
    pts = (ijk + 0.5 + jitter * (rng.random((n, 3)) * 2.0 - 1.0)) * a - 0.5 * np.asarray(box)
    return np.repeat(pts[None], slices, axis=0)


def c3_chains(count, seed=0, steps_per_block=4, npts=1000, max_levels=4):
    """Batched uneven chains: N from {32,64,128,256,512}, M from
    {16,32,64,128}, T uniform in [1,4] K, density uniform in
    [0.018,0.024] A^-3, each with its own seed and primitive u_00 table on a
    npts-point linear grid to L/2; bisection level min(max_levels, log2 M - 1)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.choice([32, 64, 128, 256, 512]))
        m = int(rng.choice([16, 32, 64, 128]))
        temp = float(rng.uniform(1.0, 4.0))
        rho = float(rng.uniform(0.018, 0.024))
        levels = min(max_levels, int(np.log2(m)) - 1)
        tau = 1.0 / (temp * m)
        box = box_for_density(n, rho)
        r_min = 1.5
        r = r_min + np.arange(npts) * ((box[0] / 2.0 - r_min) / (npts - 1))
        u00 = (tau * 2.0 ** np.arange(levels + 1))[:, None] * lj(r)[None, :]
        u00[:, -1] = 0.0
        path = lattice_path(n, m + 1, box, np.random.default_rng((seed << 20) + i))
        out.append(dict(N=n, slices=m + 1, box=box, tau=tau, lam=HE4_LAMBDA, num_levels=levels,
                        steps_per_block=steps_per_block, seed=(seed << 20) + 1000 + i,
                        grid=(r_min, float(box[0] / 2.0), npts), u00=u00, tau_pos=0, path=path, T=temp, rho=rho))
    return out

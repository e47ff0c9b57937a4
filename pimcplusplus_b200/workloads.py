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


# ---------------------------------------------------------------------------
# PIMC++ input files (the reference's ASCII format) for these workloads.
# ---------------------------------------------------------------------------
def write_pair_action_david(path, dm_path, species_type="He", lam=HE4_LAMBDA, num_offdiag_terms=0):
    """A DavidFit `.PairAction` file naming a squarer `.dm` file."""
    from .iosection import IOSectionClass
    io = IOSectionClass()
    io.NewFile(path)
    io.NewSection("Fits")
    io.WriteVar("Type", "DavidFit")
    io.WriteVar("NumOffDiagonalTerms", int(num_offdiag_terms))
    for k, lm in (("Particle1", lam), ("Particle2", 0.0)):
        io.NewSection(k)
        io.WriteVar("Name", species_type)
        io.WriteVar("lambda", float(lm))
        io.WriteVar("Ndim", 3)
        io.CloseSection()
    io.WriteVar("Daviddmfile", dm_path)
    io.CloseSection()
    io.WriteFile(path)
    return path


def write_pair_action_tricubic(path, tabs, smallest_beta, species_type="He", lam=HE4_LAMBDA):
    """A tricubicfit `.PairAction` file in the ASCII format, laid out as
    PAtricubicFitClass::Read reads it: Particle1/2, a Spline Potential, and
    Fits with q/y/t grids and one Fit section (beta, Umat, dUmat) per level."""
    from .iosection import IOSectionClass
    qg, yg, tg, umat, dumat, pot_grid, pot_data = tabs
    io = IOSectionClass()
    io.NewFile(path)
    for k, lm in (("Particle1", lam), ("Particle2", 0.0)):
        io.NewSection(k)
        io.WriteVar("Name", species_type)
        io.WriteVar("lambda", float(lm))
        io.WriteVar("Ndim", 3)
        io.CloseSection()
    io.NewSection("Potential")
    io.WriteVar("Type", "Spline")
    io.NewSection("Grid")
    io.WriteVar("Type", "Linear")
    io.WriteVar("Start", float(pot_grid[0]))
    io.WriteVar("End", float(pot_grid[1]))
    io.WriteVar("NumPoints", int(pot_grid[2]))
    io.CloseSection()
    io.WriteVar("SplineData", np.asarray(pot_data, dtype=np.float64))
    io.CloseSection()
    io.NewSection("Fits")
    io.WriteVar("Type", "tricubicfit")
    for name, g in (("qGrid", qg), ("yGrid", yg), ("tGrid", tg)):
        io.NewSection(name)
        io.WriteVar("Type", "Linear")
        io.WriteVar("Start", float(g[0]))
        io.WriteVar("End", float(g[1]))
        io.WriteVar("NumPoints", int(g[2]))
        io.CloseSection()
    for lev in range(umat.shape[0]):
        io.NewSection("Fit")
        io.WriteVar("beta", float(smallest_beta * 2.0 ** lev))
        io.WriteVar("Umat", np.asarray(umat[lev], dtype=np.float64))
        io.WriteVar("dUmat", np.asarray(dumat[lev], dtype=np.float64))
        io.CloseSection()
    io.CloseSection()
    io.WriteFile(path)
    return path


def write_pimc_input(path, cfg, pair_action_files, seed, init=("RANDOMFIXED", 0.45 * LJ_SIGMA), num_images=0,
                     steps_per_block=1, loop_steps=10, shift=False, observe_energy=False, species_type="He",
                     lam=HE4_LAMBDA, use_density=False, max_wall_time=None):
    """A PIMC++ simulation input for one LJ-style chain of `cfg` (N, M, T, rho,
    levels): System, Action (Kinetic + ShortRange), a BisectionBlock move
    (and a ShiftMove), optional Energy observable, and an Algorithm loop."""
    from .iosection import IOSectionClass
    tau, box = derived(cfg)
    io = IOSectionClass()
    io.NewFile(path)
    io.NewSection("Parallel")
    io.WriteVar("ProcsPerClone", 1)
    io.WriteVar("Seed", int(seed))
    io.CloseSection()
    io.NewSection("System")
    io.WriteVar("tau", float(tau))
    io.WriteVar("NumTimeSlices", int(cfg["M"]))
    if use_density:
        io.WriteVar("Box", np.ones(3))
        io.WriteVar("Density", float(cfg["rho"]))
    else:
        io.WriteVar("Box", np.asarray(box, dtype=np.float64))
    io.WriteVar("IsPeriodic", np.array([True, True, True]))
    io.NewSection("Particles")
    io.NewSection("Species")
    io.WriteVar("Name", "He4")
    io.WriteVar("Type", species_type)
    io.WriteVar("lambda", float(lam))
    io.WriteVar("Statistics", "BOLTZMANNON")
    io.WriteVar("NumParticles", int(cfg["N"]))
    io.WriteVar("NumDim", 3)
    io.WriteVar("InitPaths", init[0])
    if init[0] == "RANDOMFIXED":
        io.WriteVar("Radius", float(init[1]))
    elif init[0] == "FIXED":
        io.WriteVar("Positions", np.asarray(init[1], dtype=np.float64))
    else:
        io.WriteVar("File", str(init[1]))
    io.CloseSection()
    io.CloseSection()
    io.CloseSection()
    io.NewSection("Action")
    io.WriteVar("MaxLevels", int(cfg["levels"]) + 1)
    io.WriteVar("NumImages", int(num_images))
    io.WriteVar("PairActionFiles", np.array(list(pair_action_files), dtype=object))
    for t, n in (("Kinetic", "Kinetic"), ("ShortRange", "ShortRange")):
        io.NewSection("Action")
        io.WriteVar("Type", t)
        io.WriteVar("Name", n)
        io.CloseSection()
    io.CloseSection()
    if observe_energy:
        io.NewSection("Observables")
        io.NewSection("Observable")
        io.WriteVar("Type", "Energy")
        io.WriteVar("Name", "Energy")
        io.WriteVar("Frequency", 1)
        io.CloseSection()
        io.CloseSection()
    io.NewSection("Moves")
    io.NewSection("Move")
    io.WriteVar("Type", "BisectionBlock")
    io.WriteVar("Name", "BisectionBlock")
    io.WriteVar("PermuteType", "NONE")
    io.WriteVar("Species", "He4")
    io.WriteVar("NumLevels", int(cfg["levels"]))
    io.WriteVar("StepsPerBlock", int(steps_per_block))
    io.WriteVar("SamplingActions", np.array(["ShortRange"], dtype=object))
    io.WriteVar("HigherLevelActions", np.array(["ShortRange"], dtype=object))
    io.CloseSection()
    if shift:
        io.NewSection("Move")
        io.WriteVar("Type", "ShiftMove")
        io.WriteVar("Name", "Shift")
        io.CloseSection()
    io.CloseSection()
    io.NewSection("Algorithm")
    if max_wall_time is not None:
        io.WriteVar("MaxWallTime", int(max_wall_time))
    io.NewSection("Loop")
    io.WriteVar("Steps", int(loop_steps))
    io.NewSection("Move")
    io.WriteVar("Name", "BisectionBlock")
    io.CloseSection()
    if shift:
        io.NewSection("Move")
        io.WriteVar("Name", "Shift")
        io.CloseSection()
    if observe_energy:
        io.NewSection("Observe")
        io.WriteVar("Name", "Energy")
        io.CloseSection()
    io.CloseSection()
    io.CloseSection()
    io.WriteFile(path)
    return path

"""Shared set-up for the parity tests: seeded paths and matched oracle/GPU systems."""
from __future__ import annotations

import os

import numpy as np

import oracle as O
from pimcplusplus_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
# The reference's own fixture, read when the reference tree is available: its
# root in PIMC_REFERENCE_ROOT (tests that need it skip otherwise).
_REF_ROOT = os.environ.get("PIMC_REFERENCE_ROOT", "")
REF_TESTCOUL = os.path.join(_REF_ROOT, "PIMC++", "examples", "testcoul.dm") if _REF_ROOT else ""


def random_walk_path(n, slices, box, step, seed, far=0.0):
    """Slice 0 uniform in the box, later slices a Gaussian random walk.

    `far` > 0 shifts a random subset of positions by whole box lengths (up to
    +-3) so the minimum-image arithmetic sees positions far outside the box.
    """
    rng = np.random.default_rng(seed)
    p = np.empty((slices, n, 3))
    p[0] = (rng.random((n, 3)) - 0.5) * box
    for s in range(1, slices):
        p[s] = p[s - 1] + rng.normal(0.0, step, (n, 3))
    if far > 0:
        mask = rng.random((slices, n)) < far
        shift = rng.integers(-3, 4, (slices, n, 3)) * box
        p[mask] += shift[mask]
    return p


def golden_testcoul():
    d = np.load(os.path.join(GOLDEN, "testcoul_fit2.npz"))
    return {k: d[k] for k in d.files}


def coulomb_fit2_tables():
    """The [tau][grid][col] ukj/dukj arrays DavidPAClass builds from testcoul.dm's fit 2."""
    g = golden_testcoul()
    pot = g["potential"]
    ntau, nukj, ng = g["u_fit2"].shape
    u = np.zeros((ntau, ng, nukj + 1))
    du = np.zeros((ntau, ng, nukj + 1))
    u[:, :, 0] = pot
    du[:, :, 0] = pot
    u[:, :, 1:] = np.transpose(g["u_fit2"], (0, 2, 1))
    du[:, :, 1:] = np.transpose(g["du_fit2"], (0, 2, 1))
    u[:, ng - 1, :] = 0.0
    du[:, ng - 1, :] = 0.0
    return g, u, du


def write_testcoul_dm(path):
    """Re-emits the golden fit-2 arrays as a squarer file (fits 0..2) for the readers."""
    g = golden_testcoul()
    r0, r1, ng = (float(x) for x in g["grid"])
    ng = int(ng)
    t0, t1, nt = (float(x) for x in g["taugrid"])
    nt = int(nt)

    def block(vals):
        vals = np.asarray(vals).reshape(-1)
        return "\n".join(" " + " ".join(f"{v: .17e}" for v in vals[i:i + 5]) for i in range(0, len(vals), 5))

    lines = [" UNITS H AO", f" GRID {ng} LOG {r0!r} {r1!r}", f" SQUARER 1. {nt} 3 2 60 14", f" RANK 2 {ng} 1",
             f" GRID 1 LOG {r0!r} {r1!r}", " LABEL 1 r", " BEGIN potential 0", block(g["potential"])]
    for derv, key in ((1, "u_fit2"), (2, "du_fit2")):
        for fit in range(3):
            nukj = (fit + 1) * (fit + 2) // 2
            tab = np.zeros((nt, nukj, ng)) if fit != 2 else g[key]
            lines += [f" RANK 3 {ng} {nukj} {nt}", f" GRID 1 LOG {r0!r} {r1!r}", " LABEL 1 r",
                      f" GRID   3 LOG {t0!r} {t1!r}", " LABEL 2 terms", " LABEL 3 time",
                      f" BEGIN density matrix table fit= {fit} derv =  {derv}", block(tab)]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def lj_case(tmpdir, n=64, m=40, temp=2.0, levels=3, rho=0.02186, npts=1000):
    cfg = dict(N=n, M=m, T=temp, rho=rho, levels=levels, npts=npts)
    tau, box = W.derived(cfg)
    dm = W.make_dm_for(cfg, str(tmpdir))
    return cfg, tau, box, dm


def tricubic_case(n=64, m=32, temp=1.5, levels=3, rho=0.02186, nq=40, ny=12, nt=12):
    cfg = dict(N=n, M=m, T=temp, rho=rho, levels=levels)
    tau, box = W.derived(cfg)
    tabs = W.tricubic_tables(box[0], tau, levels + 1, nq=nq, ny=ny, nt=nt, pot_n=600)
    return cfg, tau, box, tabs


def rel_err(a, b, scale=None):
    s = max(abs(b), 1e-300) if scale is None else scale
    return abs(a - b) / s

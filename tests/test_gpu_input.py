"""A chain set up from the reference's input files and run on the device,
against the oracle driven by the same values.

* `Simulation` (PIMCClass::Read + LoopClass) on a RANDOMFIXED start, a
  DavidFit pair action, BisectionBlock blocks, ShiftMoves and the Energy
  observable: the final path within 1e-9, the move counts and the energy
  samples as the oracle's replay of the same loop.
* ShiftPathData on the device: bit for bit the oracle's restatement.
* The checkpoint: a chain restarted from its checkpoint by an input with
  InitPaths = "RESTART" makes the moves the original chain makes.
* A tricubicfit `.PairAction` in the ASCII format: SingleAction equals the
  oracle's on the same tables.
"""
import math
import os

import numpy as np
import pytest

import oracle as O
import pimcplusplus_b200 as P
from helpers import lj_case, random_walk_path, rel_err, tricubic_case
from pimcplusplus_b200 import workloads as W
from pimcplusplus_b200.simulation import Simulation

pytestmark = pytest.mark.gpu

SHIFT_STREAM = 3


def _input(tmp_path, name="run.in", **kw):
    cfg, tau, box, dm = lj_case(tmp_path, n=16, m=16, levels=2, npts=200)
    W.write_pair_action_david(str(tmp_path / "he.PairAction"), os.path.basename(dm))
    path = W.write_pimc_input(str(tmp_path / name), cfg, ["he.PairAction"], 7, **kw)
    return cfg, tau, box, dm, path


def _oracle(cfg, tau, box, dm):
    o = O.System(cfg["N"], cfg["M"] + 1, box, tau, W.HE4_LAMBDA, 0)
    pa = O.PairAction.from_dm(dm, tau, 0)
    o.set_pa(pa)
    o._pa_keep = pa
    return o


def test_simulation_loop_matches_oracle(tmp_path):
    loops, spb = 8, 3
    cfg, tau, box, dm, path = _input(tmp_path, loop_steps=loops, steps_per_block=spb, shift=True,
                                     observe_energy=True)
    sim = Simulation(path, device=0)
    sim.run()
    o = _oracle(cfg, tau, box, dm)
    o.init_random_fixed(7, 0.45 * W.LJ_SIGMA)
    o.bisection_config(cfg["levels"], spb, True)
    o.rng_seed(7)
    accepted, energies = 0, []
    for k in range(loops):
        recs = o.run_bisection(1)
        accepted += sum(r.accepted for r in recs)
        o.shift_data(int(math.floor(O.philox_uniform(7, SHIFT_STREAM, k) * cfg["M"])))
        energies.append(o.energy())
    st = sim.moves["BisectionBlock"].stats()
    assert st["moves"] == loops * spb and st["accepted"] == accepted and st["status"] == 0
    assert np.max(np.abs(sim.path_data.get_path(0) - o.get_path(0))) < 1e-9
    got = sim.observables["Energy"].samples
    assert len(got) == loops
    for g, r in zip(got, energies):
        assert rel_err(g["total"], r["total"], abs(r["kinetic"]) + abs(r["v_short"]) + 1e-300) < 1e-9
    sim.close()


@pytest.mark.parametrize("shift", [1, 7, 15, -3, 0])
def test_shift_data_matches_oracle(tmp_path, shift):
    cfg, tau, box, dm = lj_case(tmp_path, n=16, m=16, levels=2, npts=200)
    path = random_walk_path(16, 17, box, 0.3, seed=shift + 40)
    path[16] = path[0]
    d = P.PathData(16, 17, box, tau, W.HE4_LAMBDA, 0, device=0)
    d.set_path(path)
    d.ShiftData(shift)
    o = _oracle(cfg, tau, box, dm)
    o.set_path(path)
    o.shift_data(shift)
    assert np.array_equal(d.get_path(0), o.get_path(0)) and np.array_equal(d.get_path(1), o.get_path(1))
    with pytest.raises(P.PimcError):
        d.ShiftData(17)
    d.close()


def test_checkpoint_restart_continues_the_chain(tmp_path):
    cfg, tau, box, dm, path = _input(tmp_path, loop_steps=4, steps_per_block=2, shift=True)
    a = Simulation(path, device=0)
    a.run()
    ck = str(tmp_path / "chain.ckpt")
    a.write_checkpoint(ck)
    a.run()
    want_path, want_stats = a.path_data.get_path(0), a.moves["BisectionBlock"].stats()
    a.close()
    _, _, _, _, path_b = _input(tmp_path, name="restart.in", loop_steps=4, steps_per_block=2, shift=True,
                                init=("RESTART", ck))
    b = Simulation(path_b, device=0)
    b.run()
    assert np.array_equal(b.path_data.get_path(0), want_path)
    got = b.moves["BisectionBlock"].stats()
    for k in ("moves", "accepted", "stages_attempted", "pair_evals"):
        assert got[k] == want_stats[k], k
    b.close()
    # a checkpoint of another system is refused
    other = tmp_path / "other"
    other.mkdir()
    cfg2, tau2, box2, dm2 = lj_case(other, n=32, m=16, levels=2, npts=200)
    d = P.PathData(32, 17, box2, tau2, W.HE4_LAMBDA, 0, device=0)
    with pytest.raises(P.PimcError, match="different system"):
        d.read_checkpoint(ck)
    with pytest.raises(P.PimcError):
        d.read_checkpoint(str(tmp_path / "absent.ckpt"))
    d.close()


def test_tricubic_pair_action_file(tmp_path):
    cfg, tau, box, tabs = tricubic_case(n=24, m=16, levels=2, nq=24, ny=8, nt=8)
    pf = W.write_pair_action_tricubic(str(tmp_path / "tri.PairAction"), tabs, tau)
    path = W.write_pimc_input(str(tmp_path / "tri.in"), cfg, ["tri.PairAction"], 3)
    sim = Simulation(path, device=0)
    o = O.System(cfg["N"], cfg["M"] + 1, box, tau, W.HE4_LAMBDA, 0)
    qg, yg, tg, umat, dumat, pot_grid, pot_data = tabs
    pa = O.PairAction.tricubic(qg, yg, tg, tau, umat, dumat, pot_grid, pot_data)
    o.set_pa(pa)
    p = random_walk_path(cfg["N"], cfg["M"] + 1, box, 0.4, seed=5)
    o.set_path(p)
    sim.path_data.set_path(p)
    sr = sim.actions["ShortRange"]
    for s1, s2, act, lev in ((0, 8, [3], 0), (4, 12, [1, 5], 1), (0, 16, [0, 7, 9], 2)):
        ref = o.shortrange_single(s1, s2, act, lev)
        assert rel_err(sr.SingleAction(s1, s2, act, lev), ref) < 1e-12
    sim.close()


JELLIUM_IN = """
Section (Parallel) {{ int Seed = 5; }}
Section (System)
{{
  double tau = {tau!r};
  int NumTimeSlices = {m};
  Array<double,1> Box(3) = [{L!r}, {L!r}, {L!r}];
  Array<bool,1> IsPeriodic(3) = [true, true, true];
  double kCutoff = 1.2;
  Section (Particles)
  {{
    Section (Species)
    {{
      string Name = "e"; string Type = "e"; double lambda = 1.0; int NumParticles = {n}; int NumDim = 3;
      string InitPaths = "FIXED";
      Array<double,2> Positions({n},3) = [{pos}];
    }}
  }}
}}
Section (Action)
{{
  int MaxLevels = 3; int NumImages = 0;
  Array<string,1> PairActionFiles(1) = ["ee.PairAction"];
  bool UseLongRange = true; bool UseBackground = true; int NumBreakupKnots = 20;
  Section (Action) {{ string Type = "Kinetic"; string Name = "Kinetic"; }}
  Section (Action) {{ string Type = "ShortRange"; string Name = "ShortRange"; }}
}}
Section (Moves)
{{
  Section (Move)
  {{
    string Type = "BisectionBlock"; string Name = "Bisect"; string PermuteType = "NONE"; string Species = "e";
    int NumLevels = 2; int StepsPerBlock = 2; Array<string,1> SamplingActions(1) = ["ShortRange"];
  }}
}}
"""

EE_PAIRACTION = """Section (Fits)
{
  string Type = "classical";
  Section (Particle1) { string Name = "e"; double lambda = 1.0; int Ndim = 3; }
  Section (Particle2) { string Name = "e"; double lambda = 1.0; int Ndim = 3; }
  Section (Potential) { string Type = "Coulomb"; double Z1Z2 = 2.0; }
}
"""


def test_jellium_input_matches_direct_setup(tmp_path):
    """A classical Coulomb PairAction with the long-range breakup, set up from
    an input file, against the same chain built through PathData directly."""
    n, m, tau = 16, 16, 0.125
    L = (4.0 * math.pi / 3.0 * n) ** (1.0 / 3.0) * 4.0
    box = np.array([L, L, L])
    pos = (np.random.default_rng(3).random((n, 3)) - 0.5) * L
    (tmp_path / "ee.PairAction").write_text(EE_PAIRACTION)
    inp = tmp_path / "jellium.in"
    inp.write_text(JELLIUM_IN.format(tau=tau, m=m, L=float(L), n=n,
                                     pos=", ".join(repr(float(x)) for x in pos.reshape(-1))))
    sim = Simulation(str(inp), device=0)
    assert sim.use_longrange and "LongRange" in sim.actions
    d = P.PathData(n, m + 1, box, tau, 1.0, 0, device=0)
    d.pa_coulomb(2.0, 3)
    assert d.setup_kvecs(1.2) == sim.path_data.num_k
    d.longrange_coulomb(20, True)
    d.set_path(np.broadcast_to(pos, (m + 1, n, 3)).copy())
    assert sim.path_data.energy() == d.energy()
    bb = P.BisectionBlock(d, 2, 2, shortrange_at_higher_levels=False, use_longrange=True)
    bb.seed(5)
    want, _ = bb.MakeMoves(6)
    got, _ = sim.moves["Bisect"].MakeMoves(6)
    assert np.array_equal(got, want)
    assert np.array_equal(sim.path_data.get_path(0), d.get_path(0))
    d.close()
    sim.close()


ZERO_PAIRACTION = """Section (Fits)
{
  string Type = "zerofit";
  Section (Particle1) { string Name = "He"; double lambda = 6.0596; int Ndim = 3; }
  Section (Particle2) { string Name = "He"; double lambda = 0.0; int Ndim = 3; }
}
"""


def test_zerofit_input_is_free_particles(tmp_path):
    """PAzeroFitClass: the ShortRange sums are exactly zero and the chain is
    the kinetic-only chain of the oracle with a zero table."""
    cfg = dict(N=12, M=16, T=2.0, rho=0.02186, levels=2)
    tau, box = W.derived(cfg)
    (tmp_path / "zero.PairAction").write_text(ZERO_PAIRACTION)
    path = W.write_pimc_input(str(tmp_path / "z.in"), cfg, ["zero.PairAction"], 9, loop_steps=5, steps_per_block=2)
    sim = Simulation(path, device=0)
    sim.run()
    o = O.System(12, 17, box, tau, W.HE4_LAMBDA, 0)
    z = np.zeros((3, 2, 2))
    pa = O.PairAction.david_arrays(0.0, float(np.sqrt(np.sum(box * box))), z, z, 0, 0)
    o.set_pa(pa)
    o.init_random_fixed(9, 0.45 * W.LJ_SIGMA)
    o.bisection_config(2, 2, True)
    o.rng_seed(9)
    recs = o.run_bisection(5)
    st = sim.moves["BisectionBlock"].stats()
    assert st["moves"] == 10 and st["accepted"] == sum(r.accepted for r in recs)
    assert np.max(np.abs(sim.path_data.get_path(0) - o.get_path(0))) < 1e-9
    sr = sim.actions["ShortRange"]
    assert sr.SingleAction(0, 16, [1, 4], 0) == 0.0
    assert sr.d_dBeta(0, 16, 0) == 0.0
    sim.close()

"""The reference's input formats on the host, no GPU needed.

* The ASCII IOSection grammar (Common/IO/IOASCII.cc): scalars, arrays of
  rank 1-4 with the last index fastest, nested and included sections, both
  comment styles, and the errors the reference aborts on, with line numbers.
* `.PairAction` files of the three fit types on this path (ReadPAFit,
  Common/PairAction/PAFit.h:30-72) and a whole simulation input read and
  checked by `Simulation.read` (PIMCClass::Read) before any device call.
* The host pieces behind InitPaths and ShiftMove against the oracle:
  InitRandomFixed positions and the Philox streams bit for bit, and the
  oracle's ShiftPathData restatement against an independent statement.
"""
import os

import numpy as np
import pytest

import oracle as O
import pimcplusplus_b200 as P
from helpers import lj_case, tricubic_case
from pimcplusplus_b200 import workloads as W
from pimcplusplus_b200.iosection import InputError, IOSectionClass, format_tree, parse_text
from pimcplusplus_b200.simulation import Simulation, read_pair_action

GRAMMAR = """
double tau = 0.0125;   // a C++ comment
int NumTimeSlices=40;
string Name = "He // not a comment /* nor this */";
bool UseLongRange = false;
/* a block comment
   over two lines */
Array<double,1> Box(3) = [14.3057, 14.3057, 1.43057e1];
Array<int,2> Grid(2,3) = [1, 2, 3,
                          4, 5, -6];
Array<string,1> Files(2) = ["a.PairAction", "b.PairAction"];
Array<bool,1> IsPeriodic(3) = [true, true, false];
Array<double,3> Cube(2,1,2) = [1., .5, -2.5e-3, 4];
Section (System)
{
  Section (Species) { string Name = "first"; int NumParticles = 4; }
  Section (Species) { string Name = "second"; }
  double x = -.25;
}
Section(Empty){}
"""


def test_grammar_values_and_types():
    io = IOSectionClass()
    io.OpenText(GRAMMAR)
    assert io.ReadVar("tau") == 0.0125 and isinstance(io.ReadVar("tau"), float)
    assert io.ReadVar("NumTimeSlices") == 40 and isinstance(io.ReadVar("NumTimeSlices"), int)
    assert io.ReadVar("Name") == "He // not a comment /* nor this */"
    assert io.ReadVar("UseLongRange") is False
    assert np.array_equal(io.ReadVar("Box"), [14.3057, 14.3057, 14.3057])
    g = io.ReadVar("Grid")
    assert g.shape == (2, 3) and g.dtype == np.int64 and g[1, 2] == -6 and g[0, 1] == 2
    assert list(io.ReadVar("Files")) == ["a.PairAction", "b.PairAction"]
    assert list(io.ReadVar("IsPeriodic")) == [True, True, False]
    c = io.ReadVar("Cube")
    assert c.shape == (2, 1, 2) and c[0, 0, 1] == 0.5 and c[1, 0, 0] == -2.5e-3
    assert io.ReadVar("missing") is None and io.ReadVar("missing", 7) == 7
    assert io.CountSections() == 2 and io.CountSections("Species") == 0
    assert io.OpenSection("System")
    assert io.CountSections("Species") == 2 and io.ReadVar("x") == -0.25
    assert io.OpenSection("Species", 1) and io.ReadVar("Name") == "second"
    io.CloseSection()
    assert io.OpenSection(0) and io.GetName() == "Species" and io.ReadVar("NumParticles") == 4
    io.CloseSection()
    assert not io.OpenSection("Species", 2)
    io.CloseSection()
    assert io.OpenSection("Empty") and io.CountVars() == 0


def test_grammar_round_trip():
    t = parse_text(GRAMMAR)
    t2 = parse_text(format_tree(t))
    for (k, v), (k2, v2) in zip(t.vars, t2.vars):
        assert k == k2
        assert np.array_equal(np.asarray(v), np.asarray(v2)) and np.asarray(v).dtype == np.asarray(v2).dtype
    assert [s.name for s in t.sections] == [s.name for s in t2.sections]
    assert t2.sections[0].sections[0].var("NumParticles") == 4


def test_grammar_included_section(tmp_path):
    (tmp_path / "fits.in").write_text('string Type = "DavidFit";\nint NumOffDiagonalTerms = 2;\n')
    main = tmp_path / "main.in"
    main.write_text('Section (Fits, "fits.in");\ndouble after = 1.0;\n')
    io = IOSectionClass()
    assert io.OpenFile(str(main))
    assert io.ReadVar("after") == 1.0
    assert io.OpenSection("Fits") and io.ReadVar("Type") == "DavidFit" and io.ReadVar("NumOffDiagonalTerms") == 2
    assert not IOSectionClass().OpenFile(str(tmp_path / "absent.in"))


@pytest.mark.parametrize("text,line", [
    ("double x = 1.0\nint y = 2;", 2),            # missing semicolon: found at the next token
    ("int n = 1.5;", 1),                          # strtol must use the whole token
    ("double d = 1.0E5;", 1),                     # 'E' is not a number character
    ("bool b = yes;", 1),
    ("string s = bare;", 1),
    ("\n\nArray<double,1> a(3) = [1, 2];", 3),    # too few values
    ("Array<double,1> a(2) = [1, 2, 3];", 1),     # too many values
    ("Array<float,1> a(1) = [1];", 1),            # not an atomic type
    ("complex c = 1;", 1),                        # not implemented by the ASCII reader
    ("Section (A) { int x = 1;", 1),              # end of file before '}'
    ("int x = 1; @", 1),                          # a character the tokenizer rejects
    ("\nfloat x = 1;", 2),
])
def test_grammar_errors_carry_line_numbers(text, line):
    with pytest.raises(InputError) as e:
        parse_text(text)
    assert e.value.line == line, str(e.value)


def test_writer_reader_scalars(tmp_path):
    io = IOSectionClass()
    io.NewFile()
    io.WriteVar("a", 1)
    io.WriteVar("b", 0.1)
    io.NewSection("S")
    io.WriteVar("c", [1.5, 2.5])
    io.WriteVar("d", "text")
    io.CloseSection()
    p = str(tmp_path / "w.in")
    io.WriteFile(p)
    r = IOSectionClass()
    r.OpenFile(p)
    assert r.ReadVar("a") == 1 and r.ReadVar("b") == 0.1
    r.OpenSection("S")
    assert list(r.ReadVar("c")) == [1.5, 2.5] and r.ReadVar("d") == "text"


# ---- PairAction files and a whole input ----

def test_pair_action_files(tmp_path):
    cfg, tau, box, dm = lj_case(tmp_path, n=16, m=16, levels=2, npts=200)
    pa = read_pair_action(W.write_pair_action_david(str(tmp_path / "he.PairAction"), dm, num_offdiag_terms=0),
                          tau, 3)
    assert pa["type"] == "DavidFit" and pa["Daviddmfile"] == dm and pa["NumOffDiagonalTerms"] == 0
    assert pa["Particle1"] == {"Name": "He", "lam": W.HE4_LAMBDA}
    cfg2, tau2, box2, tabs = tricubic_case(n=16, m=16, levels=2, nq=8, ny=5, nt=5)
    pf = W.write_pair_action_tricubic(str(tmp_path / "tri.PairAction"), tabs, tau2)
    pa = read_pair_action(pf, tau2, 3)
    assert pa["type"] == "tricubicfit"
    assert np.array_equal(pa["umat"], tabs[3]) and np.array_equal(pa["dumat"], tabs[4])
    assert np.array_equal(pa["pot_data"], tabs[6]) and pa["pot_grid"] == tabs[5]
    assert [tuple(g) for g in pa["grids"]] == [tuple(float(x) for x in g[:2]) + (g[2],) for g in tabs[:3]]
    with pytest.raises(InputError):  # a level the file does not hold
        read_pair_action(pf, tau2, 4)
    (tmp_path / "ee.PairAction").write_text(
        'Section (Fits) { string Type = "classical";\n'
        '  Section (Particle1) { string Name = "e"; double lambda = 0.0; int Ndim = 3; }\n'
        '  Section (Particle2) { string Name = "e"; double lambda = 0.0; int Ndim = 3; }\n'
        '  Section (Potential) { string Type = "Coulomb"; double Z1Z2 = 2.0; } }\n')
    pa = read_pair_action(str(tmp_path / "ee.PairAction"), 0.1, 3)
    assert pa["type"] == "classical" and pa["Z1Z2"] == 2.0
    (tmp_path / "z.PairAction").write_text(
        'Section (Fits) { string Type = "zerofit";\n'
        '  Section (Particle1) { string Name = "p"; double lambda = 1.0; int Ndim = 3; }\n'
        '  Section (Particle2) { string Name = "p"; double lambda = 1.0; int Ndim = 3; } }\n')
    pa = read_pair_action(str(tmp_path / "z.PairAction"), 0.1, 3)
    assert pa["type"] == "zerofit" and pa["Particle2"]["Name"] == "p"
    (tmp_path / "bc.PairAction").write_text('Section (Fits) { string Type = "coulombBCfit"; }')
    with pytest.raises(InputError, match="coulombBCfit"):
        read_pair_action(str(tmp_path / "bc.PairAction"), 0.1, 3)


def _input(tmp_path, **kw):
    cfg, tau, box, dm = lj_case(tmp_path, n=16, m=16, levels=2, npts=200)
    pa = W.write_pair_action_david(str(tmp_path / "he.PairAction"), os.path.basename(dm))
    return cfg, tau, box, W.write_pimc_input(str(tmp_path / "run.in"), cfg, ["he.PairAction"], 7, **kw)


def test_simulation_reads_input(tmp_path):
    cfg, tau, box, path = _input(tmp_path, shift=True, observe_energy=True, loop_steps=5, steps_per_block=2)
    sim = Simulation.read(path)
    assert sim.seed == 7 and sim.num_time_slices == 16 and sim.tau == tau
    assert np.array_equal(sim.box, box)
    assert sim.species["NumParticles"] == 16 and sim.species["lam"] == W.HE4_LAMBDA
    assert sim.pair_action["type"] == "DavidFit" and os.path.isabs(sim.pair_action["Daviddmfile"])
    assert sim.move_specs == {"BisectionBlock": dict(levels=2, steps=2, higher=True), "Shift": "ShiftMove"}
    assert sim.algorithm == (1, [("Loop", (5, [("Move", "BisectionBlock"), ("Move", "Shift"),
                                               ("Observe", "Energy")]))])
    assert sim.init == ("RANDOMFIXED", 0.45 * W.LJ_SIGMA)
    assert not sim.use_longrange


def test_simulation_density_scales_box(tmp_path):
    cfg, tau, box, path = _input(tmp_path, use_density=True)
    sim = Simulation.read(path)
    assert np.allclose(sim.box, box, rtol=1e-14)


@pytest.mark.parametrize("old,new,match", [
    ('string PermuteType = "NONE";', 'string PermuteType = "TABLE";', "PermuteType"),
    ('string Type = "ShortRange";', 'string Type = "ShortRangeOrderN";', "ShortRangeOrderN"),
    ('string Type = "BisectionBlock";', 'string Type = "OpenEndMove";', "OpenEndMove"),
    ('Array<bool,1> IsPeriodic(3) = [true, true, true];', 'Array<bool,1> IsPeriodic(3) = [true, true, false];',
     "IsPeriodic"),
    ('string InitPaths = "RANDOMFIXED";', 'string InitPaths = "BCC";', "BCC"),
    ('Array<string,1> SamplingActions(1) = ["ShortRange"];', 'Array<string,1> SamplingActions(1) = ["Missing"];',
     "Missing"),
    ('int NumLevels = 2;', 'int NumLevels = 4;', "MaxLevels"),
])
def test_simulation_rejects_what_is_off_the_path(tmp_path, old, new, match):
    cfg, tau, box, path = _input(tmp_path)
    text = open(path).read()
    assert old in text, old
    open(path, "w").write(text.replace(old, new))
    with pytest.raises(InputError, match=match):
        Simulation.read(path)


# ---- host pieces vs the oracle ----

@pytest.mark.parametrize("seed,n,radius", [(1, 64, 0.45 * W.LJ_SIGMA), (99, 200, 1.0), (3, 5, 0.0)])
def test_init_random_fixed_matches_oracle(seed, n, radius):
    box = W.box_for_density(n, 0.02186)
    pos = P.init_random_fixed(box, n, radius, seed)
    o = O.System(n, 3, box, 0.01, W.HE4_LAMBDA, 0)
    o.init_random_fixed(seed, radius)
    assert np.array_equal(pos, o.get_path(0)[0])


def test_init_random_fixed_aborts_like_the_reference():
    with pytest.raises(P.PimcError, match="1000 tries"):
        P.init_random_fixed(np.array([5.0, 5.0, 5.0]), 50, 2.0, 1)


def test_stream_uniform_matches_oracle():
    for seed, stream, idx in [(0, 0, 0), (5, 3, 7), (2 ** 40 + 3, 2, 123456789), (77, 0x100 + 65, 99)]:
        assert P.stream_uniform(seed, stream, idx) == O.philox_uniform(seed, stream, idx)


@pytest.mark.parametrize("shift", [0, 1, 5, 15, -1, -7, -15])
def test_oracle_shift_data_is_a_cyclic_slice_shift(shift):
    n, m = 6, 16
    rng = np.random.default_rng(shift + 100)
    path = rng.normal(size=(m + 1, n, 3))
    path[m] = path[0]  # closed paths: row M repeats row 0
    o = O.System(n, m + 1, np.array([9.0, 9.0, 9.0]), 0.01, 1.0, 0)
    o.set_path(path)
    o.shift_data(shift)
    want = np.array([path[(j - shift) % m] for j in range(m + 1)])
    assert np.array_equal(o.get_path(0), want) and np.array_equal(o.get_path(1), want)
    with pytest.raises(ValueError):
        o.shift_data(m + 1)


def test_algorithm_wall_time_limit_and_event_times(tmp_path):
    """LoopClass: the run stops before the first event past MaxWallTime
    (PathDataClass::ExceededWallTime) and accumulates each event's wall time.
    The moves here are host stand-ins, so no GPU is needed."""
    import time as _time
    cfg, tau, box, path = _input(tmp_path, loop_steps=1000, shift=True, max_wall_time=1)
    sim = Simulation.read(path)
    assert sim.max_wall_time == 1
    calls = []

    def fake_move(name, n=1):
        calls.append(name)
        _time.sleep(0.02)

    sim.make_move = fake_move
    sim.start_wall_time = _time.monotonic()
    t0 = _time.monotonic()
    assert sim.run() is False and sim.exceeded_wall_time
    elapsed = _time.monotonic() - t0
    assert 1.0 <= elapsed < 2.0
    assert 20 < len(calls) < 2000 and set(calls) == {"BisectionBlock", "Shift"}
    assert abs(sum(sim.time_spent.values()) - elapsed) < 0.2
    # no limit: the loop runs to the end
    cfg, tau, box, path = _input(tmp_path, loop_steps=7)
    sim = Simulation.read(path)
    assert sim.max_wall_time is None
    calls.clear()
    sim.make_move = fake_move
    assert sim.run() is True and calls == ["BisectionBlock"] * 7

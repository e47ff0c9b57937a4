"""A PIMC++ run on the device, set up from the reference's own input files.

`Simulation(filename)` reads the sections PIMCClass::Read reads
(PIMC++/src/PIMCClass.cc:35-130) for the action-evaluation path and builds
the device objects behind them:

* `System`  -> PathClass::Read (PIMC++/src/PathClass.cc:123-280), one
  `Species` (SpeciesClass.cc:19-60) and its InitPaths (InitPaths.cc:495-880):
  "FIXED" (Positions), "RANDOMFIXED" (Radius), "RESTART"/"FILE" (File, a
  checkpoint this library wrote).
* `Action`  -> ActionsClass::Read (PIMC++/src/Actions/ActionsClass.cc:75-400):
  MaxLevels, NumImages, the `Action` sections of type Kinetic and
  ShortRange, PairActionFiles read by ReadPAFit
  (Common/PairAction/PAFit.h:30-72) with fit types "DavidFit"
  (Daviddmfile, NumOffDiagonalTerms), "tricubicfit" (an ASCII fit file),
  "classical" (a Coulomb potential) and "zerofit", and the long-range breakup when the
  system has a kCutoff and UseLongRange is true (UseBackground,
  NumBreakupKnots).
* `Moves`   -> BisectionBlockClass::Read (PIMC++/src/Moves/BisectionBlock.cc:27-128)
  with PermuteType "NONE", and ShiftMoveClass (MetaMoves.cc:39-65).
* `Observables` -> EnergyClass and PairCorrelationClass (Frequency, Name,
  Species1/2 and a Linear Grid); other observables are listed in `skipped`.
* `Algorithm` -> LoopClass (PIMC++/src/LoopClass.cc:30-126): nested Loop
  sections of Move and Observe events, the MaxWallTime limit and per-event
  wall time.

The random seed is the `Seed` variable of the `Parallel` section or of the
top level (PathDataClass.cc:270-281).  Anything else the reference would
read (other action types, permutations, several species, HDF5 squarer
files, worm moves) raises InputError naming it: this library covers the
bisection path only.
"""
from __future__ import annotations

import os
import time
import warnings

import numpy as np

from . import (FP64, SEQUENTIAL, BisectionBlock, KineticClass, LongRangeClass, PathData, ShortRangeClass,
               init_random_fixed)
from .iosection import InputError, IOSectionClass

__all__ = ["Simulation", "InputError", "read_pair_action"]

def _err(msg, where=None):
    return InputError(0, msg, where)


def _req(io, name, where):
    v = io.ReadVar(name)
    if v is None:
        raise _err(f"required variable {name!r} missing in section {io.GetName()!r}", where)
    return v


def _resolve(fname, *dirs):
    """A file named in an input: as given (the reference opens it relative to
    the working directory, with ~ expanded), else relative to each of dirs."""
    fname = os.path.expanduser(fname)
    for cand in [fname] + [os.path.join(d, fname) for d in dirs if d]:
        if os.path.exists(cand):
            return cand
    raise _err(f"cannot find file {fname!r}")


def read_pair_action(filename, smallest_beta, num_levels):
    """ReadPAFit (Common/PairAction/PAFit.h:30-72) for the fit types on this
    path.  Returns a dict: type, particle names and lambdas, and the data the
    device set-up needs."""
    io = IOSectionClass()
    if not io.OpenFile(filename):
        raise _err(f"unable to find the PairAction file {filename!r}")
    base = os.path.dirname(os.path.abspath(filename))
    if not io.OpenSection("Fits"):
        raise _err("no Fits section", filename)
    ftype = _req(io, "Type", filename)
    io.CloseSection()
    out = dict(type=ftype, file=filename)

    def particles():
        for k in ("Particle1", "Particle2"):
            if not io.OpenSection(k):
                raise _err(f"no {k} section", filename)
            out[k] = dict(Name=_req(io, "Name", filename), lam=float(_req(io, "lambda", filename)))
            io.CloseSection()

    if ftype == "DavidFit":
        # DavidPAClass::Read (Common/PairAction/DavidPAClass.h:144-190)
        io.OpenSection("Fits")
        out["NumOffDiagonalTerms"] = int(_req(io, "NumOffDiagonalTerms", filename))
        particles()
        dm = _req(io, "Daviddmfile", filename)
        if dm.endswith(".h5"):
            raise _err("HDF5 squarer files are not read by this library; give the ASCII .dm file", filename)
        out["Daviddmfile"] = _resolve(dm, base)
        io.CloseSection()
    elif ftype == "classical":
        # PAclassicalFitClass::Read (Common/PairAction/PAclassicalFit.cc:80-100)
        io.OpenSection("Fits")
        particles()
        if not io.OpenSection("Potential"):
            raise _err("no Potential section", filename)
        ptype = io.ReadVar("Type")
        if ptype not in (None, "Coulomb"):
            raise _err(f"classical fit with potential {ptype!r}: only Coulomb is supported", filename)
        out["Z1Z2"] = float(io.ReadVar("Z1Z2", 0.0))
        io.CloseSection()
        io.CloseSection()
    elif ftype == "tricubicfit":
        # PAtricubicFitClass::Read (Common/PairAction/PAtricubicFit.cc:794-865)
        particles()
        if not io.OpenSection("Potential"):
            raise _err("no Potential section", filename)
        if io.ReadVar("Type") != "Spline":
            raise _err("tricubicfit potential: only Type = \"Spline\" is supported", filename)
        out["pot_grid"] = _read_linear_grid(io, "Grid", filename)
        out["pot_data"] = np.asarray(_req(io, "SplineData", filename), dtype=np.float64)
        io.CloseSection()
        io.OpenSection("Fits")
        grids = [_read_linear_grid(io, g, filename) for g in ("qGrid", "yGrid", "tGrid")]
        out["grids"] = grids  # (start, end, n) of the linear q, y, t grids
        umats, dumats = [], []
        beta = smallest_beta
        for _ in range(num_levels):
            for i in range(io.CountSections("Fit")):
                io.OpenSection("Fit", i)
                b = float(_req(io, "beta", filename))
                if abs(b - beta) / beta < 1e-12:
                    umats.append(np.asarray(_req(io, "Umat", filename), dtype=np.float64))
                    dumats.append(np.asarray(_req(io, "dUmat", filename), dtype=np.float64))
                    io.CloseSection()
                    break
                io.CloseSection()
            else:
                raise _err(f"couldn't find beta = {beta} in the fit file", filename)
            beta *= 2.0
        io.CloseSection()
        out["umat"] = np.stack(umats)
        out["dumat"] = np.stack(dumats)
    elif ftype == "zerofit":
        # PAzeroFitClass::Read (Common/PairAction/PAzeroFit.cc:43-66): particles only
        io.OpenSection("Fits")
        particles()
        io.CloseSection()
    else:
        raise _err(f"pair action fit type {ftype!r} is not on this library's path "
                   "(DavidFit, tricubicfit, classical, zerofit)", filename)
    return out


def _read_linear_grid(io, section, where):
    """ReadGrid (Common/Splines/Grid.h:654-680) for Type "Linear": (start, end, n)."""
    if not io.OpenSection(section):
        raise _err(f"no {section} section", where)
    gtype = _req(io, "Type", where)
    if gtype != "Linear":
        raise _err(f"{section}: grid type {gtype!r}; only Linear grids are supported", where)
    g = (float(_req(io, "Start", where)), float(_req(io, "End", where)), int(_req(io, "NumPoints", where)))
    io.CloseSection()
    return g


class _Observable:
    def __init__(self, sim, kind, name, freq):
        self.sim, self.kind, self.name, self.freq = sim, kind, name, max(1, int(freq))
        self.times_called = 0
        self.samples = []

    def observe(self):
        # ObserveClass: an observable accumulates on every Frequency-th call
        self.times_called += 1
        if self.times_called % self.freq:
            return
        if self.kind == "Energy":
            self.samples.append(self.sim.path_data.energy())
        else:
            self.sim.path_data.gofr_accumulate()


class Simulation:
    """One chain set up from a PIMC++ input file, run by its Algorithm section.

    Attributes: `path_data` (PathData), `actions` (label -> action object),
    `moves` (name -> BisectionBlock or "ShiftMove"), `observables`,
    `species`, `seed`, `skipped` (observables outside this path).
    """

    def __init__(self, filename, device=0, precision=FP64, schedule=SEQUENTIAL, cluster_ctas=0, threads_per_cta=0,
                 seed=None):
        self.read_input(filename, seed)
        self.build(device, precision, schedule, cluster_ctas, threads_per_cta)

    @classmethod
    def read(cls, filename, seed=None):
        """Reads and checks the input without touching a GPU."""
        sim = cls.__new__(cls)
        sim.read_input(filename, seed)
        return sim

    def read_input(self, filename, seed=None):
        self.filename = filename
        self.base = os.path.dirname(os.path.abspath(filename))
        io = IOSectionClass()
        if not io.OpenFile(filename):
            raise _err(f"cannot open input file {filename!r}")
        self.skipped = []
        self.seed = self._read_seed(io) if seed is None else int(seed)
        for section, reader in (("System", self._read_system), ("Action", self._read_actions)):
            if not io.OpenSection(section):
                raise _err(f"no {section} section", filename)
            reader(io)
            io.CloseSection()
        io.OpenSection("System")
        self._read_init_paths(io)
        io.CloseSection()
        self.observable_specs = []
        if io.OpenSection("Observables"):
            self._read_observables(io)
            io.CloseSection()
        if not io.OpenSection("Moves"):
            raise _err("no Moves section", filename)
        self._read_moves(io)
        io.CloseSection()
        self.algorithm = None
        self.max_wall_time = None
        if io.OpenSection("Algorithm"):
            # PIMCClass::ReadAlgorithm (PIMCClass.cc:438-450): seconds, -1 or absent = no limit
            mwt = io.ReadVar("MaxWallTime")
            self.max_wall_time = None if mwt is None or int(mwt) < 0 else int(mwt)
            self.algorithm = self._read_loop(io, 1)
            io.CloseSection()
        self.start_wall_time = time.monotonic()
        self.time_spent = {}
        self.exceeded_wall_time = False

    def build(self, device=0, precision=FP64, schedule=SEQUENTIAL, cluster_ctas=0, threads_per_cta=0):
        """Creates the device chain: path, pair action, actions, moves, the
        seeded streams, observables and the initial path (a checkpoint read
        last restores the streams it saved)."""
        self._create(device)
        self.moves = {}
        for name, spec in self.move_specs.items():
            if spec == "ShiftMove":
                self.moves[name] = "ShiftMove"
                continue
            self.moves[name] = BisectionBlock(self.path_data, spec["levels"], spec["steps"],
                                              shortrange_at_higher_levels=spec["higher"], precision=precision,
                                              cluster_ctas=cluster_ctas, threads_per_cta=threads_per_cta,
                                              schedule=schedule, use_longrange=self.use_longrange)
        self.path_data.seed(self.seed)
        self.observables = {}
        for kind, name, freq, grid in self.observable_specs:
            if kind == "PairCorrelation":
                self.path_data.gofr_setup(*grid)
            self.observables[name] = _Observable(self, kind, name, freq)
        self._init_paths()

    # ---- PathDataClass: the seed ----
    @staticmethod
    def _read_seed(io):
        if io.OpenSection("Parallel"):
            seed = io.ReadVar("Seed")
            io.CloseSection()
            if seed is not None:
                return int(seed)
        seed = io.ReadVar("Seed")
        if seed is not None:
            return int(seed)
        return int(time.time_ns() & 0xFFFFFFFF)  # InitWithRandomSeed

    # ---- PathClass::Read ----
    def _read_system(self, io):
        f = self.filename
        self.num_time_slices = int(_req(io, "NumTimeSlices", f))
        self.tau = float(_req(io, "tau", f))
        periodic = np.asarray(_req(io, "IsPeriodic", f), dtype=bool)
        if periodic.shape != (3,) or not periodic.all():
            raise _err("IsPeriodic must be [true, true, true]: free boundaries are not on this path", f)
        box = io.ReadVar("Box")
        density = io.ReadVar("Density")
        if box is None:
            raise _err("System needs Box (and optionally Density)", f)
        box = np.asarray(box, dtype=np.float64)
        if box.shape != (3,):
            raise _err("Box must have 3 entries", f)
        self.kcutoff = io.ReadVar("kCutoff")
        if io.ReadVar("DavidLongRange", False):
            raise _err("DavidLongRange reads the squarer's HDF5 LongRange section; set the k-space table with "
                       "PathData.davidlongrange_yk instead", f)
        if io.ReadVar("OpenLoops", False) or io.ReadVar("WormOn", False):
            raise _err("open loops and worm moves are not on this path", f)
        if not io.OpenSection("Particles"):
            raise _err("no Particles section", f)
        if io.CountSections("Species") != 1:
            raise _err("exactly one Species is supported", f)
        io.OpenSection("Species")
        sp = dict(Name=_req(io, "Name", f), lam=float(_req(io, "lambda", f)),
                  NumParticles=int(_req(io, "NumParticles", f)), NumDim=int(_req(io, "NumDim", f)),
                  Type=_req(io, "Type", f))
        if sp["NumDim"] != 3:
            raise _err("NumDim must be 3", f)
        io.CloseSection()
        io.CloseSection()
        self.species = sp
        if density is not None:
            # PathClass.cc:169-188: scale Box to the density
            vol = float(np.prod(box))
            box = box * (sp["NumParticles"] / float(density) / vol) ** (1.0 / 3.0)
        self.box = box

    # ---- ActionsClass::Read ----
    def _read_actions(self, io):
        f = self.filename
        self.max_levels = int(_req(io, "MaxLevels", f))
        self.num_images = int(_req(io, "NumImages", f))
        files = np.atleast_1d(_req(io, "PairActionFiles", f))
        self.pair_action = None
        for name in files:
            pa = read_pair_action(_resolve(str(name), self.base), self.tau, self.max_levels)
            names = {pa["Particle1"]["Name"], pa["Particle2"]["Name"]}
            if names == {self.species["Type"]}:
                if self.pair_action is not None:
                    raise _err(f"more than one pair action for species type {self.species['Type']!r}", f)
                self.pair_action = pa
            else:
                warnings.warn(f"pair action {name} for {sorted(names)} not used")
        if self.pair_action is None and self.species["NumParticles"] > 1:
            raise _err(f"missing a PairAction for species {self.species['Name']!r}", f)
        self.use_longrange = bool(io.ReadVar("UseLongRange", False)) and self.kcutoff is not None
        if self.use_longrange:
            self.use_background = bool(_req(io, "UseBackground", f))
            self.num_knots = int(_req(io, "NumBreakupKnots", f))
            if self.pair_action["type"] != "classical":
                raise _err("long range on this path is the Coulomb breakup of a classical fit", f)
        self.action_specs = []
        labels = set()
        for n in range(io.CountSections("Action")):
            io.OpenSection("Action", n)
            atype, label = _req(io, "Type", f), _req(io, "Name", f)
            io.CloseSection()
            if atype not in ("Kinetic", "ShortRange"):
                raise _err(f"action type {atype!r} is not on this path (Kinetic, ShortRange)", f)
            if label in labels:
                raise _err(f"duplicate action label {label!r}", f)
            labels.add(label)
            self.action_specs.append((atype, label))

    def _create(self, device):
        sp = self.species
        d = PathData(sp["NumParticles"], self.num_time_slices + 1, self.box, self.tau, sp["lam"], self.num_images,
                     device=device)
        self.path_data = d
        pa = self.pair_action
        if pa is not None:
            if pa["type"] == "DavidFit":
                d.pa_david_from_dm(pa["Daviddmfile"], pa["NumOffDiagonalTerms"])
            elif pa["type"] == "classical":
                d.pa_coulomb(pa["Z1Z2"], self.max_levels)
            elif pa["type"] == "zerofit":
                d.pa_zero(self.max_levels)
            else:
                q, y, t = pa["grids"]
                d.pa_tricubic(q, y, t, self.tau, pa["umat"], pa["dumat"], pa["pot_grid"], pa["pot_data"])
        self.actions = {}
        for atype, label in self.action_specs:
            self.actions[label] = (KineticClass if atype == "Kinetic" else ShortRangeClass)(d)
        if self.use_longrange:
            d.setup_kvecs(float(self.kcutoff))
            d.longrange_coulomb(self.num_knots, self.use_background)
            self.actions["LongRange"] = LongRangeClass(d)

    # ---- PathClass::InitPaths ----
    def _read_init_paths(self, io):
        f = self.filename
        io.OpenSection("Particles")
        io.OpenSection("Species")
        kind = io.ReadVar("InitPaths", "RANDOM")
        n = self.species["NumParticles"]
        if kind == "FIXED":
            pos = np.asarray(_req(io, "Positions", f), dtype=np.float64)
            if pos.shape != (n, 3):
                raise _err(f"Positions must be ({n},3)", f)
            self.init = ("FIXED", pos)
        elif kind == "RANDOMFIXED":
            self.init = ("RANDOMFIXED", float(_req(io, "Radius", f)))
        elif kind in ("RESTART", "FILE"):
            self.init = ("FILE", _resolve(str(_req(io, "File", f)), self.base))
        else:
            raise _err(f"InitPaths {kind!r} is not supported (FIXED, RANDOMFIXED, RESTART, FILE)", f)
        io.CloseSection()
        io.CloseSection()

    def _init_paths(self):
        kind, arg = self.init
        n, S = self.species["NumParticles"], self.num_time_slices + 1
        if kind == "FILE":
            self.path_data.read_checkpoint(arg)
            return
        pos = arg if kind == "FIXED" else init_random_fixed(self.box, n, arg, self.seed)
        self.path_data.set_path(np.broadcast_to(pos, (S, n, 3)).copy())

    # ---- observables ----
    def _read_observables(self, io):
        f = self.filename
        for n in range(io.CountSections("Observable")):
            io.OpenSection("Observable", n)
            otype = io.ReadVar("Type") or io.ReadVar("type")
            name = io.ReadVar("Name") or io.ReadVar("name")
            freq = io.ReadVar("Frequency", io.ReadVar("freq", 1))
            if otype == "Energy":
                self.observable_specs.append(("Energy", name, freq, None))
            elif otype == "PairCorrelation":
                if io.ReadVar("Species1") not in (None, self.species["Name"]) or \
                        io.ReadVar("Species2") not in (None, self.species["Name"]):
                    raise _err("PairCorrelation species must be the system's species", f)
                start, end, npts = 0.0, float(self.box[0]), 101
                if io.OpenSection("Grid"):
                    gtype = io.ReadVar("Type") or io.ReadVar("type")
                    if gtype != "Linear":
                        raise _err("PairCorrelation grid must be Linear", f)
                    start = float(io.ReadVar("start", 0.0))
                    end = float(io.ReadVar("end", self.box[0]))
                    npts = int(_req(io, "NumPoints", f))
                    io.CloseSection()
                self.observable_specs.append(("PairCorrelation", name, freq, (start, end, npts)))
            else:
                self.skipped.append((otype, name))
            io.CloseSection()

    # ---- moves ----
    def _read_moves(self, io):
        f = self.filename
        labels = dict((lab, t) for t, lab in self.action_specs)
        sr = [lab for t, lab in self.action_specs if t == "ShortRange"]
        self.move_specs = {}
        for n in range(io.CountSections("Move")):
            io.OpenSection("Move", n)
            mtype, name = _req(io, "Type", f), _req(io, "Name", f)
            if mtype == "BisectionBlock":
                levels = int(_req(io, "NumLevels", f))
                if int(io.ReadVar("LowestLevel", 0)) != 0:
                    raise _err("LowestLevel must be 0", f)
                if _req(io, "Species", f) != self.species["Name"]:
                    raise _err(f"move {name!r}: unknown species", f)
                steps = int(_req(io, "StepsPerBlock", f))
                if _req(io, "PermuteType", f) != "NONE":
                    raise _err("PermuteType must be \"NONE\": permutations are not on this path", f)
                sampling = [str(x) for x in np.atleast_1d(_req(io, "SamplingActions", f))]
                higher = [str(x) for x in np.atleast_1d(io.ReadVar("HigherLevelActions", np.array([], object)))]
                for lab in sampling + higher:
                    if lab not in labels:
                        raise _err(f"move {name!r}: action label {lab!r} was not found", f)
                    if lab not in sr:
                        raise _err(f"move {name!r}: the device moves evaluate the ShortRange action only "
                                   f"(Kinetic is added to every stage), not {lab!r}", f)
                if not set(sampling) & set(sr):
                    raise _err(f"move {name!r}: SamplingActions must name the ShortRange action", f)
                if levels > self.max_levels:
                    raise _err(f"move {name!r}: NumLevels {levels} above the action's MaxLevels", f)
                if any(v != "ShiftMove" for v in self.move_specs.values()):
                    raise _err("one BisectionBlock move per chain: the device keeps one move set-up", f)
                self.move_specs[name] = dict(levels=levels, steps=steps, higher=bool(higher))
            elif mtype == "ShiftMove":
                self.move_specs[name] = "ShiftMove"
            else:
                raise _err(f"move type {mtype!r} is not on this path (BisectionBlock, ShiftMove)", f)
            io.CloseSection()

    def shift_move(self):
        """ShiftMoveClass::MakeMove (MetaMoves.cc:39-65): CommonInt(M) slices."""
        return self.path_data.ShiftMove()

    def make_move(self, name, n=1):
        mv = self.moves[name]
        if mv == "ShiftMove":
            return [self.shift_move() for _ in range(n)]
        return mv.MakeMoves(n, trace=False)[1]

    def observe(self, name):
        self.observables[name].observe()

    # ---- LoopClass ----
    def _read_loop(self, io, steps):
        events = []
        for i in range(io.CountSections()):
            io.OpenSection(i)
            kind = io.GetName()
            if kind == "Move":
                name = _req(io, "Name", self.filename)
                if name not in self.move_specs:
                    raise _err(f"unknown move {name!r}", self.filename)
                events.append(("Move", name))
            elif kind == "Observe":
                name = _req(io, "Name", self.filename)
                if name not in [spec[1] for spec in self.observable_specs]:
                    if any(n == name for _, n in self.skipped):
                        events.append(("Skip", name))
                        io.CloseSection()
                        continue
                    raise _err(f"unknown observable {name!r}", self.filename)
                events.append(("Observe", name))
            elif kind == "Loop":
                events.append(("Loop", self._read_loop(io, int(_req(io, "Steps", self.filename)))))
            else:
                events.append(("Skip", kind))
            io.CloseSection()
        return (steps, events)

    def exceeded_wall_time_limit(self):
        """PathDataClass::ExceededWallTime (PathDataClass.cc:433-438)."""
        return self.max_wall_time is not None and time.monotonic() - self.start_wall_time > self.max_wall_time

    def run(self, loop=None):
        """Runs the Algorithm section (LoopClass::DoEvent, LoopClass.cc:30-60).

        Before every event the wall-clock limit (Algorithm MaxWallTime) is
        checked; past it the run stops and `exceeded_wall_time` is set.  The
        wall time of every Move and Observe event is added to
        `time_spent[name]` (EventClass::TimeSpent).  Returns False when the
        limit stopped the run."""
        loop = self.algorithm if loop is None else loop
        if loop is None:
            raise _err("no Algorithm section", self.filename)
        steps, events = loop
        for _ in range(steps):
            for kind, what in events:
                if self.exceeded_wall_time_limit():
                    self.exceeded_wall_time = True
                    return False
                t0 = time.monotonic()
                if kind == "Move":
                    self.make_move(what)
                elif kind == "Observe":
                    self.observe(what)
                elif kind == "Loop":
                    if not self.run(what):
                        return False
                    continue
                else:
                    continue
                self.time_spent[what] = self.time_spent.get(what, 0.0) + time.monotonic() - t0
        return True

    def close(self):
        self.moves.clear()
        self.path_data.close()

    def write_checkpoint(self, filename):
        """The chain's path copies, streams and counters; an input with
        InitPaths = "RESTART" and File = filename continues the chain exactly."""
        self.path_data.write_checkpoint(filename)

"""Benchmark: PIMC++ bisection moves on one B200 (config C2 by default).

Workload (synthetic, seeded; the reference publishes no dataset): 512
Lennard-Jones He-4 atoms at 0.02186 A^-3, T = 1.5 K, M = 128 time slices,
PAtricubicFit pair action on a 200x50x50 (q, y, t) grid, bisection level 4,
one chain.  A step is a batch of `--moves` BisectionBlock moves run on the
device (one launch per concurrent-window round).

Precision legs of C2: FP64; mixed with the decision guard (FP32 table
arithmetic, every near-threshold stage decided on its FP64 re-evaluation, so
the trace is the FP64 path's); mixed with the relative guard (also every
stage whose error bound exceeds 1e-6 |dS| decided in FP64, so every dS a
decision uses is within 1e-6 relative of FP64's).  `value` is the faster of
the two legs that meet the metric's dS gate by construction: FP64 and the
relative-guard mixed leg.

Arms:
  default            the CUDA library (pimcplusplus_b200).
  --impl reference   the reference's CPU algorithm (the FP64 oracle
                     restatement; the reference itself cannot be built here)
                     on all host cores, one independent chain per core.  It
                     never imports pimcplusplus_b200 (whose import loads the
                     CUDA library): the workload builders are loaded from
                     their file.

Prints ONE JSON line on stdout (rank 0): the headline numbers, the roofline,
the CPU baseline, clocks and one summary per config.  The full per-leg
detail goes to stderr as one line starting with "bench-detail " (and to
--detail-out, if given).  Under torchrun each rank runs an independent
replica chain on its own GPU (the reference's clone parallelism); `value`
adds all ranks' pair evaluations over the slowest rank's time; the C3 chain
set is sharded across the ranks by cost.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import multiprocessing as mp
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

_T0 = time.perf_counter()


def progress(msg):
    """One timestamped line per leg on stderr (the JSON line stays alone on stdout)."""
    print(f"[bench +{time.perf_counter() - _T0:7.1f}s] {msg}", file=sys.stderr, flush=True)


METRIC = "pair-action evals/s & bisection moves/s, mixed vs FP64 GPU at ΔS relerr≤1e-6"
UNIT = "pair-action evals/s"
# Algorithmic bytes per tricubic pair evaluation: partner at two slices (48 B
# FP64 / 24 B FP32) + 8 nodes x 8 coefficients (512 B FP64 / 256 B FP32).
BYTES_PER_EVAL = {"fp64": 560, "mixed": 280}
W_NAME = "C2: 512 LJ He-4, rho 0.02186/A^3, T=1.5 K, M=128, PAtricubicFit 200x50x50, bisection level 4, 1 chain"

_W = None


def workloads():
    """pimcplusplus_b200/workloads.py loaded from its file: the configuration
    and table builders (numpy only), without the package's CUDA library."""
    global _W
    if _W is None:
        spec = importlib.util.spec_from_file_location(
            "pimc_bench_workloads", os.path.join(ROOT, "pimcplusplus_b200", "workloads.py"))
        _W = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(_W)
    return _W


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def c2_setup(nq=200, ny=50, nt=50):
    W = workloads()
    cfg = dict(W.CONFIGS["C2"])
    tau, box = W.derived(cfg)
    tabs = W.tricubic_tables(box[0], tau, cfg["levels"], nq=nq, ny=ny, nt=nt)
    return cfg, tau, box, tabs


def initial_path(n, slices, box, seed, radius):
    """Uniform random positions with an exclusion radius, every slice equal
    (InitRandomFixed semantics, InitPaths.cc:966-999, from a numpy stream)."""
    rng = np.random.default_rng(seed)
    pts = np.zeros((n, 3))
    for i in range(n):
        for _ in range(1000):
            c = (rng.random(3) - 0.5) * box
            d = pts[:i] - c
            d -= np.round(d / box) * box
            if i == 0 or np.min(np.sum(d * d, axis=1)) >= 4 * radius * radius:
                break
        pts[i] = c
    return np.repeat(pts[None], slices, axis=0)


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU arm: the oracle (FP64 restatement of the reference's loops)
# ---------------------------------------------------------------------------
def _pair_evals_of(records, n, levels):
    """Pair evaluations the reference performs for these moves (old+new, all
    stages attempted; ShortRange at every level)."""
    total = 0
    for r in records:
        attempted = r.stages_passed + (0 if r.accepted else 1)
        for k in range(attempted):
            level = levels - 1 - k
            total += 2 * (n - 1) * ((1 << levels) >> level)
    return total


_WORKER = {}


def _cpu_init(seed, nq, ny, nt):
    """One oracle chain per worker process, built once (C2 tables, FP64)."""
    import oracle as O
    cfg, tau, box, tabs = c2_setup(nq, ny, nt)
    qg, yg, tg, umat, dumat, pg, pot = tabs
    n, slices, L = cfg["N"], cfg["M"] + 1, cfg["levels"]
    s = O.System(n, slices, box, tau, 6.0596, 0)
    pa = O.PairAction.tricubic(qg, yg, tg, tau, umat, dumat, pg, pot)
    s.set_pa(pa)
    seed = seed + os.getpid() % 1000
    s.set_path(initial_path(n, slices, box, seed, 0.45 * 2.556))
    s.bisection_config(L, 1)
    s.rng_seed(seed)
    s.run_bisection(20)  # warm-up
    _WORKER.update(s=s, pa=pa, n=n, L=L)


def _cpu_run(seconds):
    s, n, L = _WORKER["s"], _WORKER["n"], _WORKER["L"]
    evals = moves = acc = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        recs = s.run_bisection(50)
        evals += _pair_evals_of(recs, n, L)
        moves += len(recs)
        acc += sum(r.accepted for r in recs)
    return evals, moves, acc, time.perf_counter() - t0


def cpu_workers(cores):
    """Worker count: the host cores, capped by memory (each chain holds ~0.4 GB of
    FP64 tables and buffers) and at 64."""
    try:
        import psutil
        avail = psutil.virtual_memory().available
        cores = min(cores, max(1, int(avail * 0.5 // (600 << 20))))
    except Exception:
        cores = min(cores, 8)
    return max(1, min(cores, 64))


class CpuChains:
    """The oracle on `cores` host cores, one chain per core (clone parallelism)."""

    def __init__(self, cores):
        import oracle as O
        O.build()
        self.cores = cores
        self.pool = None
        if cores == 1:
            _cpu_init(1000, 200, 50, 50)
        else:
            ctx = mp.get_context("spawn")
            self.pool = ctx.Pool(cores, initializer=_cpu_init, initargs=(1000, 200, 50, 50))

    def sample(self, seconds):
        if self.pool is None:
            res = [_cpu_run(seconds)]
        else:
            res = self.pool.map(_cpu_run, [seconds] * self.cores, chunksize=1)
        evals = sum(r[0] for r in res)
        moves = sum(r[1] for r in res)
        acc = sum(r[2] for r in res)
        dt = max(r[3] for r in res)
        return dict(value=evals / dt, moves_per_s=moves / dt, accepted_per_s=acc / dt, cores=self.cores,
                    sample=f"{moves} C2 moves, FP64 oracle, {self.cores} chain(s), {dt:.1f} s")

    def close(self):
        if self.pool is not None:
            self.pool.close()
            self.pool.join()


def cpu_baseline(cores, seconds):
    c = CpuChains(cores)
    try:
        return c.sample(seconds)
    finally:
        c.close()


def c1_setup(tmpdir):
    W = workloads()
    cfg = dict(W.CONFIGS["C1"])
    tau, box = W.derived(cfg)
    dm = W.make_dm_for(cfg, tmpdir)
    return cfg, tau, box, dm


def c1_cpu_sweeps_per_s(seconds):
    """C1 on one host core with the FP64 oracle (the reference's loops): sweeps
    per second, a sweep being N ceil(M / 2^L) = 320 bisection attempts."""
    import oracle as O
    O.build()
    with tempfile.TemporaryDirectory() as td:
        cfg, tau, box, dm = c1_setup(td)
        n, m, L = cfg["N"], cfg["M"], cfg["levels"]
        sweep = n * -(-m // (1 << L))
        s = O.System(n, m + 1, box, tau, workloads().HE4_LAMBDA, 0)
        s.set_pa(O.PairAction.from_dm(dm, tau, 0))
        s.init_random_fixed(7, 0.45 * workloads().LJ_SIGMA)
        s.bisection_config(L, sweep)
        s.rng_seed(7)
        s.run_bisection(2)
        t0, sweeps = time.perf_counter(), 0
        while time.perf_counter() - t0 < seconds:
            s.run_bisection(1)
            sweeps += 1
        dt = time.perf_counter() - t0
    return sweeps / dt, f"{sweeps} sweeps of C1 (FP64 oracle, 1 core, {dt:.1f} s)"


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = cpu_workers(os.cpu_count() or 1)
    seconds = max(2.0, min(20.0, 60.0 / max(1, args.steps + args.warmup)))
    chains = CpuChains(cores)
    for _ in range(args.warmup):
        chains.sample(1.0)
    vals = []
    last = None
    for _ in range(args.steps):
        last = chains.sample(seconds)
        vals.append(last["value"])
    chains.close()
    value = float(np.mean(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": seconds * 1000.0, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": W_NAME},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": last["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "moves_per_s": last["moves_per_s"],
        "note": "reference cannot be built here (Blitz++, SPRNG2, GSL, HDF5, LAPACK absent); "
                "its loops are timed through the FP64 oracle restatement",
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
COUNTERS = ("pair_evals", "moves", "accepted", "stages_attempted", "reevaluated", "redone")


def aggregate_ranks(ms, st, dist, device):
    """Replicas: the job's time is the slowest rank's, its work the sum of the
    ranks' counters (one all-reduce each; every rank calls this in the same
    order)."""
    if not dist:
        return ms, st
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    keys = [k for k in COUNTERS if k in st]
    v = torch.tensor([float(st[k]) for k in keys], dtype=torch.float64, device=device)
    dist.all_reduce(v)
    return float(t.item()), {k: int(round(float(x))) for k, x in zip(keys, v.tolist())}


def rates(ms, st):
    s = ms / 1000.0
    out = {"pair_evals_per_s": st["pair_evals"] / s, "moves_per_s": st["moves"] / s,
           "accepted_moves_per_s": st["accepted"] / s}
    if st.get("stages_attempted"):
        out["reevaluated_per_stage"] = st.get("reevaluated", 0) / st["stages_attempted"]
    if "evals_per_launch" in st:
        out["evals_per_launch"] = st["evals_per_launch"]
        out["ms_per_launch"] = ms / st["launches"]
    return out


class Timer:
    """Times `steps` calls of `launch()` with CUDA events on the library
    stream, the L2 flushed (a 256 MiB write) before each step outside the
    events.  Returns the summed milliseconds and the counters' deltas over
    exactly the timed steps (read before and after them)."""

    def __init__(self, torch, flush, device):
        self.torch, self.flush, self.device = torch, flush, device

    def __call__(self, stream_ptr, launch, steps, warmup, stats=None):
        torch = self.torch
        stream = torch.cuda.ExternalStream(stream_ptr, device=self.device)
        for _ in range(warmup):
            launch()
        torch.cuda.synchronize()
        s0 = stats() if stats else None
        times = []
        for _ in range(steps):
            with torch.cuda.stream(stream):
                self.flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                launch()
                e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
        if not stats:
            return float(np.sum(times))
        s1 = stats()
        if s1["status"]:
            raise RuntimeError(f"device status {s1['status']}")
        return float(np.sum(times)), {k: s1[k] - s0[k] for k in COUNTERS if k in s1}


def moves_and_shift(d, bb, n_blocks):
    """One step of a run: n_blocks BisectionBlocks on the device, then one
    ShiftMove (MetaMoves.cc:39-65), which rotates the path by a random number
    of slices so that the slices no window moves (slice 0 = M, and each
    round's window ends) are moved in later steps, as a reference run
    interleaves ShiftMove with its bisection blocks."""
    bb.launch_async(n_blocks)
    d.ShiftMove()


def stage_errors(rec):
    """Per-stage |dS - dS_FP64| of shadow records: raw (the mixed sums), the
    bound, and as used by the decision (FP64's for re-evaluated stages)."""
    mask = rec["dS_shadow"] != 0.0
    raw = np.abs(rec["dS"] - rec["dS_shadow"])
    bits = (rec["reevaluated"][:, None] >> np.arange(8)[None, :]) & 1
    used = np.where(bits == 1, 0.0, raw)
    ref = np.abs(rec["dS_shadow"])
    return raw[mask], used[mask], rec["dS_bound"][mask].astype(np.float64), ref[mask]


def run_ours(args):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    import pimcplusplus_b200 as P

    cfg, tau, box, tabs = c2_setup()
    qg, yg, tg, umat, dumat, pg, pot = tabs
    n, slices, L = cfg["N"], cfg["M"] + 1, cfg["levels"]
    start = initial_path(n, slices, box, 17 + rank, 0.45 * 2.556)
    launches = {"n": 0}

    def make(precision, guard=P.GUARD_DECISION, shadow=False, schedule=None):
        schedule = P.WINDOWS if (schedule or args.schedule) == "windows" else P.SEQUENTIAL
        d = P.PathData(n, slices, box, tau, 6.0596, 0, device=local)
        d.pa_tricubic(qg, yg, tg, tau, umat, dumat, pg, pot)
        d.set_path(start)
        bb = P.BisectionBlock(d, L, args.steps_per_block, precision=precision, shadow=shadow,
                              cluster_ctas=args.cluster, threads_per_cta=args.threads, schedule=schedule, guard=guard)
        bb.seed(1000 + rank)
        return d, bb

    # blocks per step: the windows schedule runs one round (one launch) per block
    def blocks_for(schedule):
        per = ((slices - 1) >> L) if schedule == "windows" else 1
        return max(1, args.moves // (args.steps_per_block * per))

    blocks = blocks_for(args.schedule)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")
    timer = Timer(torch, flush, f"cuda:{local}")
    _d, _bb = make(P.MIXED)
    occupancy = _bb.occupancy()
    _d.close()

    def agg(ms, st):
        return aggregate_ranks(ms, st, dist, f"cuda:{local}")

    def timed(precision, guard=P.GUARD_DECISION, schedule=None, steps=None):
        steps = steps or args.steps
        d, bb = make(precision, guard=guard, schedule=schedule)
        nb = blocks_for(schedule or args.schedule)
        if dist:
            dist.barrier()
        ms, st = timer(P.lib().pimc_stream(d.h), lambda: moves_and_shift(d, bb, nb), steps, args.warmup, bb.stats)
        if dist:
            dist.barrier()
        d.close()
        nl = steps * nb_launches(schedule or args.schedule, nb)
        launches["n"] += nl + steps  # + the ShiftMove kernel of each step
        ms, st = agg(ms, st)
        st["evals_per_launch"] = st["pair_evals"] / world / nl
        st["launches"] = nl
        return ms, st

    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    progress("C2 timed legs")
    ms64, st64 = timed(P.FP64)
    msd, std = timed(P.MIXED, P.GUARD_DECISION)
    msr, strl = timed(P.MIXED, P.GUARD_RELATIVE)
    other = "sequential" if args.schedule == "windows" else "windows"
    ms_o, st_o = timed(P.MIXED, P.GUARD_DECISION, schedule=other, steps=2)
    progress("C2 legs done")

    # dS accuracy: sequential moves with the FP64 sums alongside (shadow)
    progress("C2 dS accuracy")
    acc = {}
    for name, guard in (("decision", P.GUARD_DECISION), ("relative", P.GUARD_RELATIVE)):
        d, bb = make(P.MIXED, guard=guard, shadow=True, schedule="sequential")
        bb.MakeMoves(200 // args.steps_per_block, trace=False)
        rec, sh = bb.MakeMoves(max(1, args.accuracy_moves // args.steps_per_block), trace=True)
        d.close()
        raw, used, bound, ref = stage_errors(rec)
        rel_raw = raw / ref
        rel_used = used / ref
        acc[name] = {
            "stages": int(raw.size), "flips": int(sh["flips"]),
            "reevaluated_per_stage": sh["reevaluated"] / max(1, sh["stages_attempted"]),
            "bound_holds": bool(np.all(raw <= bound + 1e-12)),
            "raw_relerr": {"median": float(np.median(rel_raw)), "p99": float(np.quantile(rel_raw, 0.99)),
                           "max": float(np.max(rel_raw))},
            "used_relerr_max": float(np.max(rel_used)), "used_relerr_p99": float(np.quantile(rel_used, 0.99)),
            "abs_median": float(np.median(raw)), "abs_max": float(np.max(raw)),
            "bound_median": float(np.median(bound)),
        }

    # headline: the faster leg among those meeting the dS gate by construction
    v64 = st64["pair_evals"] / (ms64 / 1000.0)
    vrel = strl["pair_evals"] / (msr / 1000.0)
    vdec = std["pair_evals"] / (msd / 1000.0)
    head_mixed = vrel > v64
    head_prec, head_guard = (P.MIXED, P.GUARD_RELATIVE) if head_mixed else (P.FP64, P.GUARD_DECISION)
    ms_h, st_h = (msr, strl) if head_mixed else (ms64, st64)

    # end to end through the public API: host path in, moves, path + counters out.  The
    # host path lives in pinned memory; each step copies it into the OLD copy (the one the
    # device moves read; NEW is re-synchronised by the moves) and reads OLD back into it.
    progress("C2 end to end")
    d, bb = make(head_prec, guard=head_guard)
    host = torch.empty((slices, n, 3), dtype=torch.float64, pin_memory=True).numpy()
    host[...] = start
    for _ in range(2):
        d.set_path(host, P.OLDMODE)
        bb.MakeMoves(blocks, trace=False)
        d.get_path(P.OLDMODE, out=host)
    s0 = bb.stats()
    e2e_t = 0.0
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        d.set_path(host, P.OLDMODE)
        bb.MakeMoves(blocks, trace=False)
        d.ShiftMove()
        d.get_path(P.OLDMODE, out=host)
        e2e_t += time.perf_counter() - t0
    e2e_evals = bb.stats()["pair_evals"] - s0["pair_evals"]
    d.close()
    launches["n"] += args.steps * (nb_launches(args.schedule, blocks) + 1)
    if dist:
        t = torch.tensor([e2e_t], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_t = float(t.item())
        v = torch.tensor([float(e2e_evals)], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(v)
        e2e_evals = float(v.item())

    progress("C1")
    c1 = None if args.no_c1 else run_c1(args, P, timer, local, rank, agg, launches)
    progress("C3")
    c3 = None if args.no_c3 else run_c3(args, P, timer, local, rank, world, agg, launches)
    progress("C4")
    c4 = None if args.no_c4 else run_c4(args, P, timer, local, rank, agg, launches)
    progress("C5")
    c5 = None if args.no_c5 else run_c5(args, P, timer, local, rank, agg, launches)
    progress("GPU legs done")
    clocks = sampler.stop() if sampler else None

    if rank == 0:
        peak, peak_kind = load_peaks()
        progress("bandwidth probes")
        l2_gbs = P.read_bandwidth(local, 64 << 20, passes=32, reps=10)
        hbm_read_gbs = P.read_bandwidth(local, 2 << 30, passes=1, reps=10)
        value = st_h["pair_evals"] / (ms_h / 1000.0)
        launches_per_step = nb_launches(args.schedule, blocks)
        evals_per_launch = st_h["pair_evals"] / world / args.steps / launches_per_step
        ms_per_launch = ms_h / args.steps / launches_per_step
        bpe = BYTES_PER_EVAL["mixed" if head_mixed else "fp64"]
        achieved = evals_per_launch * bpe / (ms_per_launch / 1000.0) / 1e9
        traffic = _traffic_per_launch("bisection_c2_traffic.json", evals_per_launch,
                                      "mixed" if head_mixed else "fp64")
        progress("CPU baseline")
        cpu = cpu_baseline(1, args.cpu_seconds) if world == 1 and not args.no_cpu else None
        c1_cpu = c1_cpu_sweeps_per_s(args.c1_cpu_seconds) if (c1 and world == 1 and not args.no_cpu) else None
        if c1 and c1_cpu:
            c1["cpu_fp64_1core"] = {"sweeps_per_s": c1_cpu[0], "time_1e4_sweeps_s": 1e4 / c1_cpu[0],
                                    "sample": c1_cpu[1]}
            c1["gpu_fp64_over_cpu_1core"] = c1["fp64"]["sweeps_per_s"] / c1_cpu[0]
        path_bytes = n * slices * 3 * 8
        r64, rd, rr = rates(ms64, st64), rates(msd, std), rates(msr, strl)
        detail = {
            "c2": {"workload": W_NAME, "fp64": r64, "mixed_decision_guard": rd, "mixed_relative_guard": rr,
                   other + "_schedule_mixed": rates(ms_o, st_o), "accuracy": acc,
                   "resident_clusters": occupancy, "cluster_ctas": args.cluster, "threads_per_cta": args.threads,
                   "steps_per_block": args.steps_per_block, "windows": (slices - 1) >> L},
            "c1": c1, "c3": c3, "c4": c4, "c5": c5,
            "bandwidth": {"l2_read_gbs_64MiB": l2_gbs, "hbm_read_gbs_2GiB": hbm_read_gbs},
            "clocks": clocks,
        }
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_h / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 tables, f64 geometry+sums" if head_mixed else "f64",
            "data": "synthetic",
            "config": {"workload": W_NAME, "value_leg": "mixed, relative guard" if head_mixed else "fp64",
                       "schedule": args.schedule, "l2": "flushed between steps", "parallelism": f"replicas x{world}"},
            # [pair evals/s, accepted moves/s] of the three C2 legs
            "legs": {"fp64": _pair(r64), "mixed_decision": _pair(rd), "mixed_relative": _pair(rr)},
            "dS": {"flips": acc["decision"]["flips"] + acc["relative"]["flips"],
                   "bound_ok": acc["decision"]["bound_holds"] and acc["relative"]["bound_holds"],
                   "raw_relerr_med_p99_max": [acc["decision"]["raw_relerr"][k] for k in ("median", "p99", "max")],
                   "relative_guard_used_max": acc["relative"]["used_relerr_max"],
                   "reeval_decision_relative": [acc["decision"]["reevaluated_per_stage"],
                                                acc["relative"]["reevaluated_per_stage"]]},
            "e2e": {"value": e2e_evals / e2e_t if e2e_t else None, "unit": UNIT, "h2d_bytes_per_step": path_bytes,
                    "d2h_bytes_per_step": path_bytes + 48},
            "gpu_launches": launches["n"],
            "roofline": {"bound": "l2", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_kind": peak_kind, "l2_peak": l2_gbs, "l2_frac": achieved / l2_gbs},
            "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")} if clocks else None,
        }
        if c1:
            line["c1"] = {"sweeps_s_fp64_mixed": [c1["fp64"]["sweeps_per_s"], c1["mixed"]["sweeps_per_s"]],
                          "t_1e4_sweeps_gpu_cpu1": [c1["fp64"]["time_1e4_sweeps_s"],
                                                    c1.get("cpu_fp64_1core", {}).get("time_1e4_sweeps_s")]}
        if c3:
            line["c3"] = {"acc_s_batched_mixed_fp64_plain_fp64": [c3["batched_mixed_acc_per_s"],
                                                                  c3["batched_fp64_acc_per_s"],
                                                                  c3["plain_fp64_acc_per_s"]]}
        if c4:
            line["c4"] = {"acc_s_mixed_fp64": [c4["mixed"]["accepted_moves_per_s"], c4["fp64"]["accepted_moves_per_s"]],
                          "rhok_upd_s": c4["mixed"]["rhok_updates_per_s"]}
        if c5:
            line["c5"] = {"acc_s_lists_mixed_fp64_prop": [c5["neighbor_lists_mixed"]["accepted_moves_per_s"],
                                                          c5["neighbor_lists_fp64"]["accepted_moves_per_s"],
                                                          c5["proposals_mixed"]["accepted_moves_per_s"]]}
        if cpu:
            line["cpu_baseline"] = {"value": cpu["value"], "unit": UNIT, "cores": cpu["cores"], "kind": "port",
                                    "sample": cpu["sample"]}
        line = _rounded(line)
        detail["line"] = line
        print("bench-detail " + json.dumps(detail), file=sys.stderr, flush=True)
        if args.detail_out:
            with open(args.detail_out, "w") as f:
                json.dump(detail, f, indent=1)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def _pair(r):
    return [r["pair_evals_per_s"], r["accepted_moves_per_s"]]


def _rounded(x):
    """Floats to 4 significant digits (the one stdout line stays short)."""
    if isinstance(x, float):
        return float(f"{x:.4g}")
    if isinstance(x, dict):
        return {k: _rounded(v) for k, v in x.items()}
    if isinstance(x, list):
        return [_rounded(v) for v in x]
    return x


def run_c1(args, P, timer, local, rank, agg, launches):
    """C1 on the GPU: 64 LJ He-4, M = 40, T = 2 K, primitive 1-D table, level 3,
    one chain, concurrent-window schedule (windows of 8 slices).  A sweep is
    N ceil(M / 2^L) = 320 attempts; each timed step runs about --c1-sweeps
    sweeps (the config's full run is 10^4: its time is reported from the rate)."""
    W = workloads()
    with tempfile.TemporaryDirectory() as td:
        cfg, tau, box, dm = c1_setup(td)
        n, m, L = cfg["N"], cfg["M"], cfg["levels"]
        sweep = n * -(-m // (1 << L))
        pos = P.init_random_fixed(box, n, 0.45 * W.LJ_SIGMA, 7 + rank)
        start = np.repeat(pos[None], m + 1, axis=0)
        spb = args.c1_steps_per_block
        out = {"workload": f"C1: {n} LJ He-4, M={m}, T=2.0 K, primitive 1-D table (1000 points), level {L}, "
                           f"1 chain, concurrent windows, {spb} moves per window per round"}
        for name, prec in (("fp64", P.FP64), ("mixed", P.MIXED)):
            d = P.PathData(n, m + 1, box, tau, W.HE4_LAMBDA, 0, device=local)
            d.pa_david_from_dm(dm, 0)
            d.set_path(start)
            bb = P.BisectionBlock(d, L, spb, precision=prec, cluster_ctas=args.c1_cluster, threads_per_cta=args.c1_threads,
                                  schedule=P.WINDOWS)
            bb.seed(70 + rank)
            bb.MakeMoves(20, trace=False)  # equilibrate
            per_round = spb * 4.1  # about 4 of the 5 window slots fit a round
            rounds = max(1, int(math.ceil(args.c1_sweeps * sweep / per_round)))
            ms, st = timer(P.lib().pimc_stream(d.h), lambda: moves_and_shift(d, bb, rounds), args.steps, 0, bb.stats)
            d.close()
            launches["n"] += args.steps * (rounds + 1)
            ms, st = agg(ms, st)
            r = rates(ms, st)
            r["sweeps_per_s"] = st["moves"] / sweep / (ms / 1000.0)
            r["time_1e4_sweeps_s"] = 1e4 / r["sweeps_per_s"]
            r["sweeps_timed"] = st["moves"] / sweep
            out[name] = r
    return out


def run_c3(args, P, timer, local, rank, world, agg, launches):
    """Batched uneven chains (one persistent launch per step, replayed from a
    CUDA graph) in mixed and FP64 precision, beside the plain FP64 path: the
    same kind of chains advanced one at a time by the single-chain driver.
    Under torchrun the 1024-chain set is sharded across the ranks by cost
    (N^2 M 2^L, round-robin): strong scaling of the chain set."""
    from pimcplusplus_b200.replicas import shard_by_cost
    W = workloads()
    all_chains = W.c3_chains(args.c3_chains, seed=0, steps_per_block=args.c3_steps_per_block)
    chains = [all_chains[i] for i in shard_by_cost(all_chains, rank, world)]
    nb = args.c3_blocks

    def timed_batch(precision):
        b = P.BatchChains(chains, device=local, precision=precision)
        if args.c3_config:
            t, sp, r = args.c3_config.split(",")
            b.config(precision, False, int(t), 0, int(sp), float(r))
            tune = dict(threads_per_cta=int(t), max_split=int(sp), split_ratio=float(r), fixed=True)
        else:
            tune = b.autotune(nb)
        progress(f"C3 batched {'mixed' if precision == P.MIXED else 'FP64'}: {tune}")
        ms, st = timer(b.stream, lambda: b.run_async(nb), args.steps, args.warmup, b.stats)
        b.close()
        launches["n"] += args.steps
        ms, st = agg(ms, st)
        return ms, st, tune

    ms32, st32, tune32 = timed_batch(P.MIXED)
    ms64, st64, tune64 = timed_batch(P.FP64)

    # plain path: chains one at a time through the single-chain device driver
    def plain(precision, sample):
        tot_ms, tot = 0.0, {}
        for c in sample:
            d = P.PathData(c["N"], c["slices"], c["box"], c["tau"], c["lam"], 0, device=local)
            ng = c["grid"][2]
            ukj = np.zeros((c["u00"].shape[0], ng, 2))
            ukj[:, :, 1] = c["u00"]
            d.pa_david(P.GRID_LINEAR, c["grid"][0], c["grid"][1], ukj, np.zeros_like(ukj), 0, 0)
            d.set_path(c["path"])
            bb = P.BisectionBlock(d, c["num_levels"], c["steps_per_block"], precision=precision,
                                  schedule=P.SEQUENTIAL)
            bb.seed(c["seed"])
            ms, st = timer(P.lib().pimc_stream(d.h), lambda: bb.launch_async(nb), 1, 1, bb.stats)
            tot_ms += ms
            for k, v in st.items():
                tot[k] = tot.get(k, 0) + v
            d.close()
            launches["n"] += 1
        return tot_ms, tot

    sample = chains[: args.c3_plain_sample]
    progress("C3 plain path")
    pms64, pst64 = agg(*plain(P.FP64, sample))
    pms32, pst32 = agg(*plain(P.MIXED, sample))
    r32, r64, p64, p32 = rates(ms32, st32), rates(ms64, st64), rates(pms64, pst64), rates(pms32, pst32)
    # roofline of the batch kernel: 1-D FP32 pair evaluation = 56 B of
    # algorithmic gathers (partner at 2 slices 24 B + two spline cells 32 B)
    peak, peak_kind = load_peaks()
    evals_per_launch = st32["pair_evals"] / world / args.steps
    ms_per_launch = ms32 / args.steps
    achieved = evals_per_launch * 56 / (ms_per_launch / 1000.0) / 1e9
    return {
        "workload": f"{len(all_chains)} LJ He-4 chains ({len(chains)} on this rank), N in {{32..512}}, "
                    f"M in {{16..128}}, T in [1,4] K, rho in [0.018,0.024], primitive u00 on 1000 points, "
                    f"level <= 4, {nb * args.c3_steps_per_block} moves per chain per step",
        "scaling": "strong (the chain set is sharded across ranks by cost)",
        "batched_mixed": dict(r32, ms_per_step=ms32 / args.steps, autotune=tune32),
        "batched_fp64": dict(r64, ms_per_step=ms64 / args.steps, autotune=tune64),
        "plain_fp64": dict(p64, chains_sampled=len(sample), note="one chain at a time, single-chain driver"),
        "plain_mixed": dict(p32, chains_sampled=len(sample)),
        "batched_mixed_acc_per_s": r32["accepted_moves_per_s"], "batched_fp64_acc_per_s": r64["accepted_moves_per_s"],
        "plain_fp64_acc_per_s": p64["accepted_moves_per_s"],
        # the north-star ratio (batched mixed over the plain FP64 path) is
        # batching x precision: its two factors are reported separately
        "batched_mixed_over_plain_fp64": r32["accepted_moves_per_s"] / p64["accepted_moves_per_s"],
        "batched_mixed_over_batched_fp64": r32["accepted_moves_per_s"] / r64["accepted_moves_per_s"],
        "batched_fp64_over_plain_fp64": r64["accepted_moves_per_s"] / p64["accepted_moves_per_s"],
        "roofline": {"bound": "l2", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "bytes_per_eval": 56, "kernel": "batch_kernel<PA_DAVID,float>",
                     "traffic": _traffic_per_launch("batch_c3_traffic.json", evals_per_launch, "mixed")},
    }


def run_c4(args, P, timer, local, rank, agg, launches):
    """Jellium (C4): 128 electrons at r_s = 4 bohr, beta = 8 Ry^-1, M = 64,
    classical Coulomb pair action with the optimized breakup (49 knots,
    k cutoff 1.2 bohr^-1: 510 k-vectors), bisection level 3, concurrent
    windows, LongRange with the rho_k update in every move's lowest stage."""
    n, m, L, levels = 128, 64, 3, 3
    boxl = (4.0 * math.pi / 3.0 * n) ** (1.0 / 3.0) * 4.0
    box = np.array([boxl] * 3)
    tau = 8.0 / m
    start = initial_path(n, m + 1, box, 41 + rank, 0.0)
    spb = args.c4_steps_per_block

    def make(precision, shadow=False, schedule=None):
        d = P.PathData(n, m + 1, box, tau, 1.0, 0, device=local)
        d.pa_coulomb(2.0, levels)
        nk = d.setup_kvecs(1.2)
        d.longrange_coulomb(49, use_background=True)
        d.set_path(start)
        bb = P.BisectionBlock(d, L, spb, precision=precision, shadow=shadow, cluster_ctas=args.c4_cluster,
                              threads_per_cta=args.c4_threads, schedule=schedule if schedule is not None else P.WINDOWS,
                              use_longrange=True)
        bb.seed(500 + rank)
        return d, bb, nk

    rounds = max(1, 2048 // (spb * (m >> L)))

    def timed(precision):
        d, bb, nk = make(precision)
        ms, st = timer(P.lib().pimc_stream(d.h), lambda: moves_and_shift(d, bb, rounds), args.steps, args.warmup,
                       bb.stats)
        # share of moves that reach the lowest stage (its rho_k update covers 2^L + 1 slices)
        rec, _ = bb.MakeMoves(rounds, trace=True)
        live = rec["slice1"] >= 0
        frac0 = float(np.mean(rec["stages_passed"][live] >= L - 1)) if live.any() else 0.0
        d.close()
        launches["n"] += args.steps * (rounds + 2)  # + ShiftMove and the rho_k recompute it calls for
        ms, st = agg(ms, st)
        return ms, st, frac0, nk

    ms32, st32, f32, nk = timed(P.MIXED)
    ms64, st64, f64, _ = timed(P.FP64)
    d, bb, _ = make(P.MIXED, shadow=True, schedule=P.SEQUENTIAL)
    bb.MakeMoves(20, trace=False)
    rec, sh = bb.MakeMoves(max(1, args.accuracy_moves // spb), trace=True)
    d.close()
    raw, used, bound, ref = stage_errors(rec)
    rel = raw / ref

    def rr(ms, st, frac0):
        r = rates(ms, st)
        r["rhok_updates_per_s"] = st["moves"] * frac0 * ((1 << L) + 1) / (ms / 1000.0)
        r["ms_per_step"] = ms / args.steps
        return r

    r32, r64 = rr(ms32, st32, f32), rr(ms64, st64, f64)
    return {
        "workload": f"jellium N={n}, r_s=4 bohr, beta=8 Ry^-1, M={m}, classical Coulomb action with optimized "
                    f"breakup (49 knots), {nk} k-vectors, bisection level {L}, concurrent windows, "
                    f"{args.c4_cluster}-CTA clusters",
        "mixed": r32, "fp64": r64,
        "mixed_over_fp64": r32["accepted_moves_per_s"] / r64["accepted_moves_per_s"],
        "dS": {"raw_relerr_median": float(np.median(rel)), "raw_relerr_p99": float(np.quantile(rel, 0.99)),
               "raw_relerr_max": float(np.max(rel)), "stages": int(rel.size), "flips": int(sh["flips"]),
               "bound_holds": bool(np.all(raw <= bound + 1e-12)),
               "reevaluated_per_stage": sh["reevaluated"] / max(1, sh["stages_attempted"])},
    }


def run_c5(args, P, timer, local, rank, agg, launches):
    """C5: one large chain, 4096 LJ He-4 at 0.02186 A^-3, T = 1 K, M = 256,
    LJ truncated and shifted to zero at 2.5 sigma (table to the cutoff),
    bisection level 5, concurrent windows, neighbour lists (skin 2.5 A)
    against the all-partner sum, mixed and FP64; and concurrent
    moved-particle proposals (P slots per window, one CTA each: 8 windows x
    8 slots = 64 proposals by default)."""
    W = workloads()
    cfg = dict(W.CONFIGS["C5"])
    tau, box = W.derived(cfg)
    n, m, L = cfg["N"], cfg["M"], cfg["levels"]
    dm = W.make_dm_for(cfg, tempfile.mkdtemp())
    spb = args.c5_steps_per_block
    start = W.lattice_path(n, m + 1, box, np.random.default_rng(5 + rank))

    def make(precision, skin, path, proposals=0):
        d = P.PathData(n, m + 1, box, tau, W.HE4_LAMBDA, 0, device=local)
        d.pa_david_from_dm(dm, 0)
        d.set_path(path)
        if proposals:
            bb = P.BisectionBlock(d, L, spb, precision=precision, cluster_ctas=proposals,
                                  threads_per_cta=args.c5_prop_threads, schedule=P.PROPOSALS, neighbor_skin=skin)
        else:
            bb = P.BisectionBlock(d, L, spb, precision=precision, cluster_ctas=args.c5_cluster,
                                  threads_per_cta=args.c5_threads,
                                  schedule=P.WINDOWS, neighbor_skin=skin)
        bb.seed(900 + rank)
        return d, bb

    # a short all-partner run gives the path its quantum spread first (untimed)
    d, bb = make(P.MIXED, 0.0, start)
    bb.MakeMoves(args.c5_equil, trace=False)
    progress("C5 equilibrated")
    eq = d.get_path(P.OLDMODE)
    d.close()
    rounds = args.c5_rounds

    def timed(precision, skin, proposals=0):
        d, bb = make(precision, skin, eq, proposals)
        ms, st = timer(P.lib().pimc_stream(d.h), lambda: moves_and_shift(d, bb, rounds), args.steps, args.warmup,
                       bb.stats)
        d.close()
        # per round: the bisection launch, plus the neighbour-list kernels (bounds, fill, clear) with
        # lists; per step the ShiftMove kernel
        launches["n"] += args.steps * (rounds * (4 if skin > 0 else 1) + 1)
        ms, st = agg(ms, st)
        out = rates(ms, st)
        out["pair_evals_per_move"] = st["pair_evals"] / st["moves"]
        out["ms_per_step"] = ms / args.steps
        if proposals:
            out["redone_per_move"] = st["redone"] / st["moves"]
        return out

    lists32 = timed(P.MIXED, args.c5_skin)
    lists64 = timed(P.FP64, args.c5_skin)
    plain64 = timed(P.FP64, 0.0)
    progress("C5 windows legs done")
    pp = args.c5_proposals
    prop32 = timed(P.MIXED, args.c5_skin, pp)
    prop64 = timed(P.FP64, args.c5_skin, pp)
    progress("C5 proposals done")
    return {
        "workload": f"{n} LJ He-4, rho 0.02186/A^3, T=1 K, M={m}, LJ truncated/shifted at 2.5 sigma, level {L}, "
                    f"{m >> L} concurrent windows x {args.c5_cluster}-CTA clusters, {spb * rounds} moves per "
                    f"window per step; proposals: {m >> L} windows x {pp} slots = {(m >> L) * pp} concurrent "
                    f"moved-particle proposals",
        "neighbor_lists_mixed": lists32, "neighbor_lists_fp64": lists64, "all_partners_fp64": plain64,
        "proposals_mixed": prop32, "proposals_fp64": prop64,
        "lists_over_all_partners_fp64": lists64["accepted_moves_per_s"] / plain64["accepted_moves_per_s"],
        "mixed_over_fp64": lists32["accepted_moves_per_s"] / lists64["accepted_moves_per_s"],
        "proposals_over_one_per_window": prop32["accepted_moves_per_s"] / lists32["accepted_moves_per_s"],
        "skin": args.c5_skin, "proposals": pp,
    }


def _traffic_per_launch(name, evals_per_launch, precision):
    """DRAM bytes of one launch: an ncu capture's bytes per pair evaluation
    (profiles/<name>) times this run's pair evaluations per launch."""
    prof = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(prof):
        return None
    with open(prof) as f:
        per = json.load(f).get(f"dram_bytes_per_pair_eval_{precision}")
    return per * evals_per_launch if per is not None else None


def nb_launches(schedule, blocks):
    """Bisection-kernel launches per timed step of one C2 leg."""
    return blocks if schedule == "windows" else 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--moves", type=int, default=2048)
    ap.add_argument("--schedule", default="windows", choices=["windows", "sequential"])
    ap.add_argument("--steps-per-block", type=int, default=128)
    ap.add_argument("--cluster", type=int, default=16)
    ap.add_argument("--threads", type=int, default=512)
    ap.add_argument("--accuracy-moves", type=int, default=1000)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--c1-cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-c1", action="store_true")
    ap.add_argument("--no-c3", action="store_true")
    ap.add_argument("--no-c4", action="store_true")
    ap.add_argument("--no-c5", action="store_true")
    ap.add_argument("--c1-sweeps", type=int, default=100, help="C1 sweeps per timed step")
    ap.add_argument("--c1-steps-per-block", type=int, default=64)
    ap.add_argument("--c5-cluster", type=int, default=16)
    ap.add_argument("--c5-skin", type=float, default=2.5)
    ap.add_argument("--c5-rounds", type=int, default=4)
    ap.add_argument("--c5-equil", type=int, default=60)
    ap.add_argument("--c5-proposals", type=int, default=8)
    ap.add_argument("--c5-prop-threads", type=int, default=512)
    ap.add_argument("--c4-cluster", type=int, default=8)
    ap.add_argument("--c4-steps-per-block", type=int, default=16)
    ap.add_argument("--c4-threads", type=int, default=512)
    ap.add_argument("--c1-cluster", type=int, default=8)
    ap.add_argument("--c1-threads", type=int, default=256)
    ap.add_argument("--c5-threads", type=int, default=512)
    ap.add_argument("--c5-steps-per-block", type=int, default=16)
    ap.add_argument("--c3-chains", type=int, default=1024)
    ap.add_argument("--c3-blocks", type=int, default=4)
    ap.add_argument("--c3-steps-per-block", type=int, default=4)
    ap.add_argument("--c3-plain-sample", type=int, default=32)
    ap.add_argument("--c3-config", default="", help="threads,max_split,split_ratio instead of the autotuner")
    ap.add_argument("--detail-out", default="", help="also write the per-leg detail JSON here")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

"""Benchmark: PIMC++ bisection moves on one B200 (config C2 by default).

Workload (synthetic, seeded; the reference publishes no dataset): 512
Lennard-Jones He-4 atoms at 0.02186 A^-3, T = 1.5 K, M = 128 time slices,
PAtricubicFit pair action on a 200x50x50 (q, y, t) grid, bisection level 4,
one chain.  A step is a batch of `--moves` BisectionBlock moves run on the
device by one launch of the bisection kernel.

Arms:
  default            the CUDA library: FP64 and mixed-precision device moves.
  --impl reference   the reference's CPU algorithm (the FP64 oracle
                     restatement; the reference itself cannot be built here)
                     on all host cores, one independent chain per core.

Prints one JSON line (rank 0).  Under torchrun each rank runs an independent
replica chain on its own GPU (the reference's clone parallelism); `value`
adds all ranks' pair evaluations over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import subprocess
import sys
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


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def c2_setup(nq=200, ny=50, nt=50):
    from pimcplusplus_b200 import workloads as W
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
                    sample=f"{moves} moves of C2 (FP64 oracle, {self.cores} independent chain(s), {dt:.1f} s)")

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
    cfg, tau, box, _ = c2_setup(8, 4, 4)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": seconds * 1000.0, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": W_NAME, "N": 512, "M": 128, "levels": 4, "table": "tricubic 200x50x50"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": last["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "moves_per_s": last["moves_per_s"],
        "note": "reference cannot be built here (Blitz++, SPRNG2, GSL, HDF5, LAPACK absent); "
                "its loops are timed through the FP64 oracle restatement",
    }
    print(json.dumps(line), flush=True)


W_NAME = "C2: 512 LJ He-4, rho 0.02186/A^3, T=1.5 K, M=128, PAtricubicFit 200x50x50, bisection level 4, 1 chain"


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
COUNTERS = ("pair_evals", "moves", "accepted", "stages_attempted")


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

    def make(precision, shadow=False, cl=args.cluster, threads=args.threads, schedule=None):
        schedule = P.WINDOWS if (schedule if schedule is not None else args.schedule) == "windows" else P.SEQUENTIAL
        d = P.PathData(n, slices, box, tau, 6.0596, 0, device=local)
        d.pa_tricubic(qg, yg, tg, tau, umat, dumat, pg, pot)
        d.set_path(start)
        bb = P.BisectionBlock(d, L, args.steps_per_block, precision=precision, shadow=shadow, cluster_ctas=cl,
                              threads_per_cta=threads, schedule=schedule)
        bb.seed(1000 + rank)
        return d, bb

    # blocks per step: the windows schedule runs one round (one launch) per block
    def blocks_for(schedule):
        per = ((slices - 1) >> L) if schedule == "windows" else 1
        return max(1, args.moves // (args.steps_per_block * per))

    blocks = blocks_for(args.schedule)

    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")
    _d, _bb = make(P.MIXED)
    occupancy = _bb.occupancy()
    _d.close()

    def timed(precision, schedule=None, steps=None):
        steps = steps or args.steps
        d, bb = make(precision, schedule=schedule)
        nb = blocks_for(schedule or args.schedule)
        stream = torch.cuda.ExternalStream(P.lib().pimc_stream(d.h), device=f"cuda:{local}")
        for _ in range(args.warmup):
            bb.launch_async(nb)
        d.synchronize()
        s0 = bb.stats()
        times = []
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()  # L2 flush between steps, outside the timed events
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                bb.launch_async(nb)
                e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        s1 = bb.stats()
        if s1["status"]:
            raise RuntimeError(f"device status {s1['status']}")
        ms = float(np.sum(times))
        st = {k: s1[k] - s0[k] for k in ("moves", "accepted", "pair_evals", "stages_attempted")}
        d.close()
        return ms, st

    def agg(ms, st):
        return aggregate_ranks(ms, st, dist, f"cuda:{local}")

    # nvidia-smi samples every 200 ms, so the clocks are sampled over all the
    # timed legs together (C2 FP64 and mixed, the other schedule, C3)
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    progress("C2 timed legs")
    ms64, st64 = timed(P.FP64)
    ms32, st32 = timed(P.MIXED)
    progress("C2 FP64 and mixed done")
    ms64, st64 = agg(ms64, st64)
    ms32, st32 = agg(ms32, st32)
    other = "sequential" if args.schedule == "windows" else "windows"
    ms_o, st_o = timed(P.MIXED, schedule=other, steps=2)
    ms_o, st_o = agg(ms_o, st_o)

    # dS accuracy of the mixed path: mixed decisions with the FP64 terms alongside
    progress("C2 dS accuracy")
    d, bb = make(P.MIXED, shadow=True, schedule="sequential")
    bb.MakeMoves(200 // args.steps_per_block, trace=False)
    rec, sh = bb.MakeMoves(max(1, args.accuracy_moves // args.steps_per_block), trace=True)
    d.close()
    m = rec["dS_shadow"] != 0.0
    absd = np.abs(rec["dS"][m] - rec["dS_shadow"][m])
    rel = absd / np.abs(rec["dS_shadow"][m])
    flip_rate = sh["flips"] / max(1, sh["stages_attempted"])

    # end to end through the public API: host path in, moves, path + counters out
    progress("C2 end to end")
    d, bb = make(P.MIXED)
    host = start.copy()
    for _ in range(2):
        d.set_path(host)
        bb.MakeMoves(blocks, trace=False)
        host = d.get_path(P.OLDMODE)
    e2e_t, e2e_evals = 0.0, 0
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        d.set_path(host)
        _, st = bb.MakeMoves(blocks, trace=False)
        host = d.get_path(P.OLDMODE)
        e2e_t += time.perf_counter() - t0
    e2e_evals = bb.stats()["pair_evals"]
    d.close()
    e2e_evals_timed = e2e_evals * args.steps / (args.steps + 2)
    if dist:
        t = torch.tensor([e2e_t], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_t = float(t.item())
        v = torch.tensor([e2e_evals_timed], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(v)
        e2e_evals_timed = float(v.item())

    progress("C3")
    c3 = None if args.no_c3 else run_c3(args, P, torch, flush, local, rank, world, agg)
    progress("C4")
    c4 = None if args.no_c4 else run_c4(args, P, torch, flush, local, rank, world, agg)
    progress("C5")
    c5 = None if args.no_c5 else run_c5(args, P, torch, flush, local, rank, world, agg)
    progress("GPU legs done")
    clocks = sampler.stop() if sampler else None
    if clocks:
        clocks["window"] = "all timed legs (C2 FP64, mixed, other schedule, accuracy, e2e, C3)"

    if rank == 0:
        peak, peak_kind = load_peaks()
        value = st32["pair_evals"] / (ms32 / 1000.0)
        value64 = st64["pair_evals"] / (ms64 / 1000.0)
        launches_per_step = nb_launches(args.schedule, blocks)
        evals_per_launch = st32["pair_evals"] / world / args.steps / launches_per_step
        ms_per_launch = ms32 / args.steps / launches_per_step
        achieved = evals_per_launch * BYTES_PER_EVAL["mixed"] / (ms_per_launch / 1000.0) / 1e9
        traffic = None
        prof = os.path.join(ROOT, "profiles", "bisection_c2_traffic.json")
        if os.path.exists(prof):
            with open(prof) as f:
                pj = json.load(f)
            traffic = pj.get("dram_bytes_per_pair_eval_mixed", 0) * evals_per_launch
        progress("CPU baseline")
        cpu = cpu_baseline(1, args.cpu_seconds) if world == 1 and not args.no_cpu else None
        path_bytes = n * slices * 3 * 8
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 pair terms / f64 sums", "data": "synthetic",
            "config": {"workload": W_NAME, "moves_per_step": st32["moves"] // world // args.steps,
                       "schedule": args.schedule, "steps_per_block": args.steps_per_block,
                       "cluster_ctas": args.cluster, "threads_per_cta": args.threads,
                       "resident_clusters": occupancy, "windows": (slices - 1) >> L,
                       "l2": "flushed between steps by a 256 MiB write outside the timed events",
                       "parallelism": f"replicas x{world}"},
            "moves_per_s": st32["moves"] / (ms32 / 1000.0),
            "accepted_moves_per_s": st32["accepted"] / (ms32 / 1000.0),
            "fp64": {"pair_evals_per_s": value64, "moves_per_s": st64["moves"] / (ms64 / 1000.0),
                     "accepted_moves_per_s": st64["accepted"] / (ms64 / 1000.0), "ms_per_step": ms64 / args.steps},
            "mixed_over_fp64": value / value64 if value64 else None,
            other: {"pair_evals_per_s": st_o["pair_evals"] / (ms_o / 1000.0),
                    "moves_per_s": st_o["moves"] / (ms_o / 1000.0), "precision": "mixed"},
            "dS_relerr": {"median": float(np.median(rel)) if rel.size else None,
                          "p99": float(np.quantile(rel, 0.99)) if rel.size else None,
                          "max": float(np.max(rel)) if rel.size else None, "stages": int(rel.size),
                          "flip_rate": flip_rate,
                          # the relative error is large only where dS itself is near 0;
                          # the absolute error is what moves a Metropolis decision
                          "abs_median": float(np.median(absd)) if absd.size else None,
                          "abs_max": float(np.max(absd)) if absd.size else None},
            "e2e": {"value": e2e_evals_timed / e2e_t if e2e_t else None, "unit": UNIT,
                    "h2d_bytes_per_step": path_bytes, "d2h_bytes_per_step": path_bytes + 48},
            "gpu_launches": args.steps * 2 * nb_launches(args.schedule, blocks),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "bytes_per_eval": BYTES_PER_EVAL["mixed"], "evals_per_launch": evals_per_launch,
                         "ms_per_launch": ms_per_launch,
                         "traffic_source": "profiles/bisection_c2_traffic.json (ncu, one round) scaled by evals",
                         "kernel": "bisection_kernel<PA_TRICUBIC,float>"},
            "clocks": clocks,
        }
        if c3:
            line["c3"] = c3
            line["gpu_launches"] += c3.pop("_launches")
        if c4:
            line["c4"] = c4
            line["gpu_launches"] += c4.pop("_launches")
        if c5:
            line["c5"] = c5
            line["gpu_launches"] += c5.pop("_launches")
        if cpu:
            line["cpu_baseline"] = {"value": cpu["value"], "unit": UNIT, "cores": cpu["cores"], "kind": "port",
                                    "sample": cpu["sample"]}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_c3(args, P, torch, flush, local, rank, world, agg):
    """Batched uneven chains (one persistent launch per step, replayed from a
    CUDA graph) in mixed and FP64 precision, beside the plain FP64 path: the
    same kind of chains advanced one at a time by the single-chain driver."""
    from pimcplusplus_b200 import workloads as W

    chains = W.c3_chains(args.c3_chains, seed=rank, steps_per_block=args.c3_steps_per_block)
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
        stream = torch.cuda.ExternalStream(b.stream, device=f"cuda:{local}")
        for _ in range(args.warmup):
            b.run_async(nb)
        b.synchronize()
        s0 = b.stats()
        times = []
        torch.cuda.synchronize()
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                b.run_async(nb)
                e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        s1 = b.stats()
        if s1["status"]:
            raise RuntimeError(f"batch device status {s1['status']}")
        b.close()
        st = {k: s1[k] - s0[k] for k in ("moves", "accepted", "pair_evals", "stages_attempted")}
        ms, st = agg(float(np.sum(times)), st)
        return ms, st, tune

    ms32, st32, tune32 = timed_batch(P.MIXED)
    ms64, st64, tune64 = timed_batch(P.FP64)

    # plain path: chains one at a time through the single-chain device driver
    def plain(precision, sample):
        tot_ms, acc, mv, ev = 0.0, 0, 0, 0
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
            bb.MakeMoves(1, trace=False)
            stream = torch.cuda.ExternalStream(P.lib().pimc_stream(d.h), device=f"cuda:{local}")
            s0 = bb.stats()
            with torch.cuda.stream(stream):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                bb.launch_async(nb)
                e1.record(stream)
            e1.synchronize()
            s1 = bb.stats()
            tot_ms += e0.elapsed_time(e1)
            acc += s1["accepted"] - s0["accepted"]
            mv += s1["moves"] - s0["moves"]
            ev += s1["pair_evals"] - s0["pair_evals"]
            d.close()
        return tot_ms, dict(accepted=acc, moves=mv, pair_evals=ev)

    sample = chains[: args.c3_plain_sample]
    progress("C3 plain path")
    pms64, pst64 = agg(*plain(P.FP64, sample))
    pms32, pst32 = agg(*plain(P.MIXED, sample))

    def rates(ms, st):
        s = ms / 1000.0
        return {"accepted_moves_per_s": st["accepted"] / s, "moves_per_s": st["moves"] / s,
                "pair_evals_per_s": st["pair_evals"] / s}

    r32, r64, p64, p32 = rates(ms32, st32), rates(ms64, st64), rates(pms64, pst64), rates(pms32, pst32)
    # roofline of the batch kernel: one launch per step (persistent); 1-D pair
    # evaluation = 56 B of algorithmic gathers in FP32 (partner at 2 slices
    # 24 B + two spline cells 32 B)
    peak, peak_kind = load_peaks()
    evals_per_launch = st32["pair_evals"] / world / args.steps
    ms_per_launch = ms32 / args.steps
    achieved = evals_per_launch * 56 / (ms_per_launch / 1000.0) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "batch_c3_traffic.json")
    if os.path.exists(prof):
        with open(prof) as f:
            traffic = json.load(f).get("dram_bytes_per_pair_eval_mixed", 0) * evals_per_launch
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "peak_kind": peak_kind, "bytes_per_eval": 56, "evals_per_launch": evals_per_launch,
            "ms_per_launch": ms_per_launch, "kernel": "batch_kernel<PA_DAVID,float>",
            "traffic_source": "profiles/batch_c3_traffic.json (ncu, one launch) scaled by evals"}
    return {
        "workload": f"{len(chains)} LJ He-4 chains, N in {{32..512}}, M in {{16..128}}, T in [1,4] K, "
                    f"rho in [0.018,0.024], primitive u00 on 1000 points, level <= 4, "
                    f"{nb * args.c3_steps_per_block} moves per chain per step",
        "batched_mixed": dict(r32, ms_per_step=ms32 / args.steps, autotune=tune32, roofline=roof),
        "batched_fp64": dict(r64, ms_per_step=ms64 / args.steps, autotune=tune64),
        "plain_fp64": dict(p64, chains_sampled=len(sample), note="one chain at a time, single-chain driver"),
        "plain_mixed": dict(p32, chains_sampled=len(sample)),
        "batched_mixed_over_plain_fp64": r32["accepted_moves_per_s"] / p64["accepted_moves_per_s"],
        "batched_mixed_over_batched_fp64": r32["accepted_moves_per_s"] / r64["accepted_moves_per_s"],
        "_launches": 2 * args.steps,
    }


def run_c4(args, P, torch, flush, local, rank, world, agg):
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
                              threads_per_cta=256, schedule=schedule if schedule is not None else P.WINDOWS,
                              use_longrange=True)
        bb.seed(500 + rank)
        return d, bb, nk

    rounds = max(1, 2048 // (spb * ((m) >> L)))

    def timed(precision):
        d, bb, nk = make(precision)
        stream = torch.cuda.ExternalStream(P.lib().pimc_stream(d.h), device=f"cuda:{local}")
        for _ in range(args.warmup):
            bb.launch_async(rounds)
        d.synchronize()
        s0 = bb.stats()
        times = []
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                bb.launch_async(rounds)
                e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        s1 = bb.stats()
        if s1["status"]:
            raise RuntimeError(f"C4 device status {s1['status']}")
        # share of moves that reach the lowest stage (its rho_k update covers 2^L + 1 slices)
        rec, _ = bb.MakeMoves(rounds, trace=True)
        live = rec["slice1"] >= 0
        frac0 = float(np.mean(rec["stages_passed"][live] >= L - 1)) if live.any() else 0.0
        d.close()
        st = {k: s1[k] - s0[k] for k in ("moves", "accepted", "pair_evals", "stages_attempted")}
        ms, st = agg(float(np.sum(times)), st)
        return ms, st, frac0, nk

    ms32, st32, f32, nk = timed(P.MIXED)
    progress("C4 mixed done")
    ms64, st64, f64, _ = timed(P.FP64)
    progress("C4 FP64 done")
    d, bb, _ = make(P.MIXED, shadow=True, schedule=P.SEQUENTIAL)
    bb.MakeMoves(20, trace=False)
    rec, sh = bb.MakeMoves(max(1, args.accuracy_moves // spb), trace=True)
    d.close()
    mask = rec["dS_shadow"] != 0.0
    rel = np.abs(rec["dS"][mask] - rec["dS_shadow"][mask]) / np.abs(rec["dS_shadow"][mask])

    def rates(ms, st, frac0):
        s = ms / 1000.0
        upd = st["moves"] * frac0 * ((1 << L) + 1)
        return {"pair_evals_per_s": st["pair_evals"] / s, "moves_per_s": st["moves"] / s,
                "accepted_moves_per_s": st["accepted"] / s, "rhok_updates_per_s": upd / s,
                "ms_per_step": ms / args.steps}

    r32, r64 = rates(ms32, st32, f32), rates(ms64, st64, f64)
    peak, peak_kind = load_peaks()
    # algorithmic bytes: 1-D Coulomb pair eval in FP32 = partner at 2 slices (24 B) + two
    # Ulong quintic cells (2 x 24 B); rho_k update = OLD read + NEW write, 32 B per k
    secs = ms32 / 1000.0 / args.steps
    achieved = ((st32["pair_evals"] / world / args.steps) * 72 +
                r32["rhok_updates_per_s"] / world * secs * 32 * nk) / secs / 1e9
    evals_per_launch = st32["pair_evals"] / world / (args.steps * rounds)
    traffic = _traffic_per_launch("bisection_c4_traffic.json", evals_per_launch)
    return {
        "workload": f"jellium N={n}, r_s=4 bohr, beta=8 Ry^-1, M={m}, classical Coulomb action with optimized "
                    f"breakup (49 knots), {nk} k-vectors, bisection level {L}, concurrent windows, "
                    f"{args.c4_cluster}-CTA clusters",
        "mixed": r32, "fp64": r64,
        "mixed_over_fp64": r32["accepted_moves_per_s"] / r64["accepted_moves_per_s"],
        "dS_relerr": {"median": float(np.median(rel)) if rel.size else None,
                      "p99": float(np.quantile(rel, 0.99)) if rel.size else None, "stages": int(rel.size),
                      "flip_rate": sh["flips"] / max(1, sh["stages_attempted"])},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": peak_kind, "evals_per_launch": evals_per_launch,
                     "ms_per_launch": ms32 / (args.steps * rounds),
                     "traffic_source": "profiles/bisection_c4_traffic.json (ncu, one launch) scaled by evals",
                     "kernel": "bisection_kernel<PA_COULOMB,float> with LongRange"},
        "_launches": 2 * args.steps * rounds,
    }


def run_c5(args, P, torch, flush, local, rank, world, agg):
    """C5: one large chain, 4096 LJ He-4 at 0.02186 A^-3, T = 1 K, M = 256,
    LJ truncated and shifted to zero at 2.5 sigma (table to the cutoff),
    bisection level 5, concurrent windows, neighbour lists (skin 2.5 A)
    against the all-partner sum, mixed and FP64; and concurrent
    moved-particle proposals (P slots per window, one CTA each: 8 windows x
    8 slots = 64 proposals by default)."""
    import tempfile

    from pimcplusplus_b200 import workloads as W

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
            bb = P.BisectionBlock(d, L, spb, precision=precision, cluster_ctas=args.c5_cluster, threads_per_cta=512,
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
        stream = torch.cuda.ExternalStream(P.lib().pimc_stream(d.h), device=f"cuda:{local}")
        for _ in range(args.warmup):
            bb.launch_async(rounds)
        d.synchronize()
        s0 = bb.stats()
        times = []
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                bb.launch_async(rounds)
                e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        s1 = bb.stats()
        if s1["status"]:
            raise RuntimeError(f"C5 device status {s1['status']}")
        d.close()
        st = {k: s1[k] - s0[k] for k in ("moves", "accepted", "pair_evals", "stages_attempted", "redone")}
        ms, st = agg(float(np.sum(times)), st)
        s = ms / 1000.0
        out = {"pair_evals_per_s": st["pair_evals"] / s, "moves_per_s": st["moves"] / s,
               "accepted_moves_per_s": st["accepted"] / s, "pair_evals_per_move": st["pair_evals"] / st["moves"],
               "ms_per_step": ms / args.steps}
        if proposals:
            out["redone_per_move"] = st["redone"] / st["moves"]
        out["_per_launch"] = (st["pair_evals"] / world / (args.steps * rounds), ms / (args.steps * rounds))
        return out

    lists32 = timed(P.MIXED, args.c5_skin)
    lists64 = timed(P.FP64, args.c5_skin)
    plain32 = timed(P.MIXED, 0.0)
    progress("C5 windows legs done")
    pp = args.c5_proposals
    prop32 = timed(P.MIXED, args.c5_skin, pp)
    prop64 = timed(P.FP64, args.c5_skin, pp)
    progress("C5 proposals done")
    wide32 = timed(P.MIXED, args.c5_skin, args.c5_proposals_wide) if args.c5_proposals_wide else None
    # roofline of the neighbour-list mixed kernel: 1-D FP32 pair eval = partner
    # at two slices (24 B) + two spline cells (32 B); lists and bounds kernels
    # are small beside it
    evals_per_launch, ms_per_launch = lists32["_per_launch"]
    peak, peak_kind = load_peaks()
    achieved = evals_per_launch * 56 / (ms_per_launch / 1000.0) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": _traffic_per_launch("bisection_c5_traffic.json", evals_per_launch),
                "peak_kind": peak_kind, "bytes_per_eval": 56, "evals_per_launch": evals_per_launch,
                "ms_per_launch": ms_per_launch,
                "traffic_source": "profiles/bisection_c5_traffic.json (ncu, one launch) scaled by evals",
                "kernel": "bisection_kernel<PA_DAVID,float>, windows, neighbour lists"}
    for leg in (lists32, lists64, plain32, prop32, prop64, wide32):
        if leg:
            leg.pop("_per_launch", None)
    return {
        "workload": f"{n} LJ He-4, rho 0.02186/A^3, T=1 K, M={m}, LJ truncated/shifted at 2.5 sigma, level {L}, "
                    f"{m >> L} concurrent windows x {args.c5_cluster}-CTA clusters, {spb * rounds} moves per "
                    f"window per step; proposals: {m >> L} windows x {pp} slots = {(m >> L) * pp} concurrent "
                    f"moved-particle proposals, {spb * rounds * pp} moves per window per step",
        "neighbor_lists_mixed": lists32, "neighbor_lists_fp64": lists64, "all_partners_mixed": plain32,
        "proposals_mixed": prop32, "proposals_fp64": prop64,
        f"proposals_{(m >> L) * args.c5_proposals_wide}_mixed": wide32,
        "lists_over_all_partners": lists32["accepted_moves_per_s"] / plain32["accepted_moves_per_s"],
        "mixed_over_fp64": lists32["accepted_moves_per_s"] / lists64["accepted_moves_per_s"],
        "proposals_over_one_per_window": prop32["accepted_moves_per_s"] / lists32["accepted_moves_per_s"],
        "proposals_mixed_over_fp64": prop32["accepted_moves_per_s"] / prop64["accepted_moves_per_s"],
        "skin": args.c5_skin, "proposals": pp, "roofline": roofline,
        # per round: one bisection launch per variant, plus the three neighbour
        # list kernels (bounds, fill, clear) of each variant with lists
        "_launches": (6 + 5 * 3 if args.c5_proposals_wide else 5 + 4 * 3) * args.steps * rounds,
    }


def _traffic_per_launch(name, evals_per_launch):
    """DRAM bytes of one launch: an ncu capture's bytes per pair evaluation
    (profiles/<name>) times this run's pair evaluations per launch."""
    prof = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(prof):
        return None
    with open(prof) as f:
        return json.load(f).get("dram_bytes_per_pair_eval_mixed", 0) * evals_per_launch


def nb_launches(schedule, blocks):
    """Bisection-kernel launches per timed step (FP64 + mixed counted by the caller)."""
    return blocks if schedule == "windows" else 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--moves", type=int, default=2048)
    ap.add_argument("--schedule", default="windows", choices=["windows", "sequential"])
    ap.add_argument("--steps-per-block", type=int, default=64)
    ap.add_argument("--cluster", type=int, default=16)
    ap.add_argument("--threads", type=int, default=512)
    ap.add_argument("--accuracy-moves", type=int, default=1000)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-c3", action="store_true")
    ap.add_argument("--no-c4", action="store_true")
    ap.add_argument("--no-c5", action="store_true")
    ap.add_argument("--c5-cluster", type=int, default=16)
    ap.add_argument("--c5-skin", type=float, default=2.5)
    ap.add_argument("--c5-rounds", type=int, default=4)
    ap.add_argument("--c5-equil", type=int, default=60)
    ap.add_argument("--c5-proposals", type=int, default=8)
    ap.add_argument("--c5-proposals-wide", type=int, default=16, help="a second proposals shape (0: none)")
    ap.add_argument("--c5-prop-threads", type=int, default=512)
    ap.add_argument("--c4-cluster", type=int, default=8)
    ap.add_argument("--c4-steps-per-block", type=int, default=16)
    ap.add_argument("--c5-steps-per-block", type=int, default=16)
    ap.add_argument("--c3-chains", type=int, default=1024)
    ap.add_argument("--c3-blocks", type=int, default=4)
    ap.add_argument("--c3-steps-per-block", type=int, default=4)
    ap.add_argument("--c3-plain-sample", type=int, default=32)
    ap.add_argument("--c3-config", default="", help="threads,max_split,split_ratio instead of the autotuner")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

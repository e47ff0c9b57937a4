"""ORACLE — test infrastructure only.

ctypes bindings to oracle/_build/liboracle.so, the FP64 CPU restatement of the
PIMC++ action-evaluation hot path (see pimc_oracle.h for what it restates and
how it is pinned).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline legs may import this package; the CUDA library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


class MoveRecord(C.Structure):
    _fields_ = [
        ("slice1", C.c_int32),
        ("ptcl", C.c_int32),
        ("accepted", C.c_int32),
        ("stages_passed", C.c_int32),
        ("dS", C.c_double * 8),
        ("log_sample_ratio", C.c_double * 8),
    ]


def build() -> str:
    """Compiles the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    src = os.path.join(_HERE, "pimc_oracle.cc")
    if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        build()
    L = C.CDLL(_LIB_PATH)
    d, i, p, u64, u32 = C.c_double, C.c_int, C.c_void_p, C.c_uint64, C.c_uint32
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    sig = {
        "oracle_philox_uniform": (d, [u64, u32, u64]),
        "oracle_philox_block": (None, [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
        "oracle_pa_david_from_dm": (p, [C.c_char_p, d, i]),
        "oracle_pa_david_arrays": (p, [d, d, i, i, i, dp, dp, i, i]),
        "oracle_pa_tricubic": (p, [d, d, i, d, d, i, d, d, i, i, d, dp, dp, d, d, i, dp]),
        "oracle_pa_classical_coulomb": (p, [d, i, d]),
        "oracle_pa_free": (None, [p]),
        "oracle_pa_U": (d, [p, d, d, d, i]),
        "oracle_pa_dU": (d, [p, d, d, d, i]),
        "oracle_pa_info": (i, [p, ip, ip, ip, ip, dp, dp, ip]),
        "oracle_pa_david_table": (i, [p, i, i, dp]),
        "oracle_pa_david_spline": (d, [p, i, i, i, d]),
        "oracle_tricubic_create": (p, [d, d, i, d, d, i, d, d, i, dp]),
        "oracle_tricubic_eval": (d, [p, d, d, d]),
        "oracle_tricubic_coefs": (i, [p, dp]),
        "oracle_tricubic_free": (None, [p]),
        "oracle_system_create": (p, [i, i, dp, d, d, i]),
        "oracle_system_free": (None, [p]),
        "oracle_system_set_pa": (None, [p, p]),
        "oracle_system_set_path": (None, [p, i, dp]),
        "oracle_system_get_path": (None, [p, i, dp]),
        "oracle_system_set_mode": (None, [p, i]),
        "oracle_init_random_fixed": (i, [p, u64, d]),
        "oracle_shift_data": (i, [p, i]),
        "oracle_shortrange_single": (d, [p, i, i, ip, i, i]),
        "oracle_shortrange_single_abs": (d, [p, i, i, ip, i, i]),
        "oracle_shortrange_dbeta": (d, [p, i, i, i]),
        "oracle_kinetic_single": (d, [p, i, i, ip, i, i]),
        "oracle_kinetic_dbeta": (d, [p, i, i, i]),
        "oracle_setup_kvecs": (i, [p, d]),
        "oracle_num_kvecs": (i, [p]),
        "oracle_get_kvecs": (None, [p, dp, ip]),
        "oracle_calc_rhok_all": (None, [p]),
        "oracle_update_rhok": (None, [p, i, i, ip, i, i]),
        "oracle_get_rhok": (None, [p, i, dp]),
        "oracle_set_longrange": (None, [p, i, dp, dp, dp, dp, dp, dp, dp, dp, i]),
        "oracle_longrange_single": (d, [p, i, i, ip, i, i]),
        "oracle_set_yk": (i, [p, i, dp, dp, i]),
        "oracle_get_yk": (None, [p, dp, dp, dp]),
        "oracle_yk_single": (d, [p, i, i, ip, i, i]),
        "oracle_yk_dbeta": (d, [p, i, i]),
        "oracle_yk_v": (d, [p, i, i]),
        "oracle_longrange_dbeta": (d, [p, i, i, i]),
        "oracle_bisection_config": (None, [p, i, i, i, i]),
        "oracle_rng_seed": (None, [p, u64]),
        "oracle_run_bisection": (i, [p, i, C.POINTER(MoveRecord)]),
        "oracle_rng_position": (u64, [p]),
        "oracle_set_ulong": (None, [p, i, i, d, C.POINTER(d), C.POINTER(d)]),
        "oracle_energy": (None, [p, C.POINTER(d)]),
        "oracle_gofr_accumulate": (None, [p, d, d, i, C.POINTER(u64)]),
        "oracle_run_windows": (i, [p, i, C.POINTER(MoveRecord)]),
        "oracle_run_proposals": (i, [p, i, i, C.POINTER(MoveRecord)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def philox_block(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().oracle_philox_block(c, k, o)
    return list(o)


def philox_uniform(seed: int, stream: int, index: int) -> float:
    return lib().oracle_philox_uniform(seed, stream, index)


class PairAction:
    """A pair-action fit held by the oracle (DavidPA, PAtricubicFit or PAclassicalFit)."""

    def __init__(self, handle):
        if not handle:
            raise RuntimeError("oracle: pair action construction failed")
        self.h = handle

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.oracle_pa_free(self.h)
            self.h = None

    @classmethod
    def from_dm(cls, path: str, desired_tau: float, num_offdiag_terms: int = 0):
        return cls(lib().oracle_pa_david_from_dm(path.encode(), desired_tau, num_offdiag_terms))

    @classmethod
    def david_arrays(cls, grid_start, grid_end, ukj, dukj, tau_pos=0, num_offdiag_terms=0):
        ukj = np.ascontiguousarray(ukj, dtype=np.float64)
        dukj = np.ascontiguousarray(dukj, dtype=np.float64)
        nt, ng, nc = ukj.shape
        return cls(lib().oracle_pa_david_arrays(grid_start, grid_end, ng, nc, nt, _dp(ukj), _dp(dukj), tau_pos,
                                                num_offdiag_terms))

    @classmethod
    def tricubic(cls, qgrid, ygrid, tgrid, smallest_beta, umat, dumat, pot_grid, pot_data):
        umat = np.ascontiguousarray(umat, dtype=np.float64)
        dumat = np.ascontiguousarray(dumat, dtype=np.float64)
        pot_data = np.ascontiguousarray(pot_data, dtype=np.float64)
        nb = umat.shape[0]
        h = lib().oracle_pa_tricubic(*qgrid, *ygrid, *tgrid, nb, smallest_beta, _dp(umat), _dp(dumat),
                                     *pot_grid, _dp(pot_data))
        return cls(h)

    @classmethod
    def classical_coulomb(cls, smallest_beta: float, num_betas: int, z1z2: float):
        return cls(lib().oracle_pa_classical_coulomb(smallest_beta, num_betas, z1z2))

    def U(self, q, z, s2, level):
        return lib().oracle_pa_U(self.h, q, z, s2, level)

    def dU(self, q, z, s2, level):
        return lib().oracle_pa_dU(self.h, q, z, s2, level)

    def info(self):
        vals = [C.c_int() for _ in range(4)]
        g0, g1 = C.c_double(), C.c_double()
        gt = C.c_int()
        rc = lib().oracle_pa_info(self.h, *[C.byref(v) for v in vals], C.byref(g0), C.byref(g1), C.byref(gt))
        if rc:
            raise RuntimeError("not a David pair action")
        nt, tp, ng, nc = [v.value for v in vals]
        return dict(num_tau=nt, tau_pos=tp, num_grid=ng, num_cols=nc, grid_start=g0.value,
                    grid_end=g1.value, grid_type=gt.value)

    def table(self, which: int, level: int) -> np.ndarray:
        inf = self.info()
        out = np.zeros((inf["num_grid"], inf["num_cols"]))
        if lib().oracle_pa_david_table(self.h, which, level, _dp(out)):
            raise IndexError(level)
        return out

    def spline(self, which: int, level: int, col: int, x: float) -> float:
        return lib().oracle_pa_david_spline(self.h, which, level, col, x)


class Tricubic:
    def __init__(self, xg, yg, zg, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        self.shape = (xg[2], yg[2], zg[2])
        self.h = lib().oracle_tricubic_create(*xg, *yg, *zg, _dp(f))

    def __call__(self, x, y, z):
        return lib().oracle_tricubic_eval(self.h, x, y, z)

    def coefs(self):
        out = np.zeros(self.shape + (8,))
        lib().oracle_tricubic_coefs(self.h, _dp(out))
        return out

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.oracle_tricubic_free(self.h)
            self.h = None


class System:
    """PathDataClass restated: one species, OLD/NEW mirrored path copies."""

    def __init__(self, num_particles, num_time_slices, box, tau, lam, num_images=0):
        self.N = num_particles
        self.S = num_time_slices
        b = np.ascontiguousarray(box, dtype=np.float64)
        self.h = lib().oracle_system_create(num_particles, num_time_slices, _dp(b), tau, lam, num_images)
        self._pa = None

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.oracle_system_free(self.h)
            self.h = None

    def set_pa(self, pa: PairAction):
        self._pa = pa
        lib().oracle_system_set_pa(self.h, pa.h)

    def set_path(self, path, copy=None):
        path = np.ascontiguousarray(path, dtype=np.float64)
        assert path.shape == (self.S, self.N, 3)
        for c in ((0, 1) if copy is None else (copy,)):
            lib().oracle_system_set_path(self.h, c, _dp(path))

    def get_path(self, copy=0):
        out = np.zeros((self.S, self.N, 3))
        lib().oracle_system_get_path(self.h, copy, _dp(out))
        return out

    def set_mode(self, copy):
        lib().oracle_system_set_mode(self.h, copy)

    def init_random_fixed(self, seed, radius):
        if lib().oracle_init_random_fixed(self.h, seed, radius):
            raise RuntimeError("InitRandomFixed: exceeded 1000 tries")

    def shift_data(self, slices_to_shift):
        if lib().oracle_shift_data(self.h, slices_to_shift):
            raise ValueError("|slices_to_shift| must be below num_time_slices")

    def shortrange_single(self, s1, s2, active, level, copy=0):
        a = np.ascontiguousarray(active, dtype=np.int32)
        self.set_mode(copy)
        return lib().oracle_shortrange_single(self.h, s1, s2, _ip(a), len(a), level)

    def shortrange_single_abs(self, s1, s2, active, level, copy=0):
        a = np.ascontiguousarray(active, dtype=np.int32)
        self.set_mode(copy)
        return lib().oracle_shortrange_single_abs(self.h, s1, s2, _ip(a), len(a), level)

    def shortrange_dbeta(self, s1, s2, level=0):
        self.set_mode(0)
        return lib().oracle_shortrange_dbeta(self.h, s1, s2, level)

    def kinetic_single(self, s1, s2, active, level, copy=0):
        a = np.ascontiguousarray(active, dtype=np.int32)
        self.set_mode(copy)
        return lib().oracle_kinetic_single(self.h, s1, s2, _ip(a), len(a), level)

    def kinetic_dbeta(self, s1, s2, level=0):
        self.set_mode(0)
        return lib().oracle_kinetic_dbeta(self.h, s1, s2, level)

    def setup_kvecs(self, kcutoff):
        return lib().oracle_setup_kvecs(self.h, kcutoff)

    def kvecs(self):
        n = lib().oracle_num_kvecs(self.h)
        kv = np.zeros((n, 3))
        ki = np.zeros((n, 3), dtype=np.int32)
        lib().oracle_get_kvecs(self.h, _dp(kv), _ip(ki))
        return kv, ki

    def calc_rhok_all(self):
        lib().oracle_calc_rhok_all(self.h)

    def update_rhok(self, s1, s2, active, level):
        a = np.ascontiguousarray(active, dtype=np.int32)
        lib().oracle_update_rhok(self.h, s1, s2, _ip(a), len(a), level)

    def rhok(self, copy=0):
        n = lib().oracle_num_kvecs(self.h)
        out = np.zeros((self.S, n, 2))
        lib().oracle_get_rhok(self.h, copy, _dp(out))
        return out[..., 0] + 1j * out[..., 1]

    def set_longrange(self, ulong_k, ulong_r0, ushort_k0, ulong_k0, dulong_k, dulong_r0, dushort_k0,
                      dulong_k0, use_background=True):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
                (ulong_k, ulong_r0, ushort_k0, ulong_k0, dulong_k, dulong_r0, dushort_k0, dulong_k0)]
        self._lr = arrs
        lib().oracle_set_longrange(self.h, arrs[1].shape[0], *[_dp(a) for a in arrs], int(use_background))

    def longrange_single(self, s1, s2, active, level, copy=0):
        a = np.ascontiguousarray(active, dtype=np.int32)
        self.set_mode(copy)
        return lib().oracle_longrange_single(self.h, s1, s2, _ip(a), len(a), level)

    def longrange_dbeta(self, s1, s2, level=0):
        self.set_mode(0)
        return lib().oracle_longrange_dbeta(self.h, s1, s2, level)

    # ---- DavidLongRangeClassYk ----
    def set_yk(self, kvals, uk_long, rpa=True):
        """Tables from the squarer's k-space action uk_long(kvals); False if a
        k-vector's |k| is not among kvals."""
        kv = np.ascontiguousarray(kvals, dtype=np.float64)
        uk = np.ascontiguousarray(uk_long, dtype=np.float64)
        return lib().oracle_set_yk(self.h, len(kv), _dp(kv), _dp(uk), int(rpa)) == 0

    def yk_tables(self):
        n = lib().oracle_num_kvecs(self.h)
        u, du, v = np.zeros(n), np.zeros(n), np.zeros(n)
        lib().oracle_get_yk(self.h, _dp(u), _dp(du), _dp(v))
        return u, du, v

    def yk_single(self, s1, s2, active, level, copy=0):
        a = np.ascontiguousarray(active, dtype=np.int32)
        self.set_mode(copy)
        return lib().oracle_yk_single(self.h, s1, s2, _ip(a), len(a), level)

    def yk_dbeta(self, s1, s2):
        self.set_mode(0)
        return lib().oracle_yk_dbeta(self.h, s1, s2)

    def yk_v(self, s1, s2):
        self.set_mode(0)
        return lib().oracle_yk_v(self.h, s1, s2)

    def bisection_config(self, num_levels, steps_per_block=1, shortrange_at_higher_levels=True,
                         use_longrange=False):
        self.steps_per_block = steps_per_block
        self.num_levels = num_levels
        lib().oracle_bisection_config(self.h, num_levels, steps_per_block, int(shortrange_at_higher_levels),
                                      int(use_longrange))

    def rng_seed(self, seed):
        lib().oracle_rng_seed(self.h, seed)

    def run_bisection(self, n_blocks):
        n = n_blocks * self.steps_per_block
        recs = (MoveRecord * n)()
        lib().oracle_run_bisection(self.h, n_blocks, recs)
        return recs

    def run_windows(self, n_rounds):
        w = min((self.S - 1) >> self.num_levels, 64)
        recs = (MoveRecord * (n_rounds * w * self.steps_per_block))()
        lib().oracle_run_windows(self.h, n_rounds, recs)
        return recs

    def run_proposals(self, n_rounds, proposals):
        """Concurrent windows with `proposals` slots per window, replayed in
        slot order; records [round][window][step][slot]."""
        w = min((self.S - 1) >> self.num_levels, 64)
        recs = (MoveRecord * (n_rounds * w * self.steps_per_block * proposals))()
        if lib().oracle_run_proposals(self.h, n_rounds, proposals, recs) < 0:
            raise ValueError("proposals must be 1..16")
        return recs

    def rng_position(self):
        return lib().oracle_rng_position(self.h)

    def set_ulong(self, ulong_r, dulong_r, rmax):
        """Ulong/dUlong quintic coefficient tables [levels][points][6] on [0, rmax]."""
        u = np.ascontiguousarray(ulong_r, dtype=np.float64)
        du = np.ascontiguousarray(dulong_r, dtype=np.float64)
        self._keep_ulong = (u, du)
        lib().oracle_set_ulong(self.h, u.shape[0], u.shape[1], rmax / (u.shape[1] - 1),
                               u.ctypes.data_as(C.POINTER(C.c_double)), du.ctypes.data_as(C.POINTER(C.c_double)))

    def energy(self):
        """ActionsClass::Energy terms of the OLD copy."""
        out = np.zeros(6)
        lib().oracle_energy(self.h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return dict(zip(("kinetic", "du_short", "du_long", "v_short", "v_long", "total"), out.tolist()))

    def gofr_accumulate(self, start, end, num_points, hist=None):
        """PairCorrelationClass::Accumulate of the OLD copy into hist (uint64)."""
        if hist is None:
            hist = np.zeros(num_points - 1, dtype=np.uint64)
        lib().oracle_gofr_accumulate(self.h, start, end, num_points, hist.ctypes.data_as(C.POINTER(C.c_uint64)))
        return hist

"""B200-native action evaluation for PIMC++ path-integral Monte Carlo.

Python host layer over the C ABI of libpimc_b200.so (include/pimc_b200.h).
It mirrors the reference's Action interface: `ShortRangeClass`,
`KineticClass` expose SingleAction(slice1, slice2, activeParticles, level) and
d_dBeta(slice1, slice2, level) with the reference's argument meaning
(PIMC++/src/Actions/ActionBase.h:43-57), `PathData.SetMode` selects the OLD
or NEW mirrored copy (MirroredClass.cc:19), and `BisectionBlock` runs
BisectionBlockClass::MakeMove (PIMC++/src/Moves/BisectionBlock.cc:380-451)
entirely on the device.

The CUDA library is required: importing this package raises ImportError if
libpimc_b200.so is missing, and there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpimc_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python -m pimcplusplus_b200.build_lib` (nvcc, sm_100a)")

_lib = C.CDLL(LIB_PATH)

PIMC_OK = 0
PIMC_E_ARG = 1
OLDMODE, NEWMODE, BOTH = 0, 1, 2
FP64, MIXED = 0, 1
ACTION_SHORTRANGE, ACTION_KINETIC, ACTION_LONGRANGE, ACTION_DAVIDLONGRANGE = 0, 1, 2, 3
GRID_LINEAR, GRID_LOG = 0, 1
SEQUENTIAL, WINDOWS, PROPOSALS = 0, 1, 2
GUARD_DECISION, GUARD_NONE, GUARD_RELATIVE = 0, 1, 2


def guard_value(guard):
    """PIMC_GUARD_* of a guard argument: one of the constants, or True (decision) / False (none)."""
    if guard is True:
        return GUARD_DECISION
    if guard is False:
        return GUARD_NONE
    return int(guard)

STATUS = {
    0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "non-finite action", 4: "index out of range",
    5: "device loop cap reached", 6: "file missing or malformed", 7: "call out of order", 8: "allocation failed",
    9: "broken staging",
}


class PimcError(RuntimeError):
    def __init__(self, status, msg=""):
        super().__init__(f"{STATUS.get(status, status)} ({status}): {msg}")
        self.status = status


class SystemDesc(C.Structure):
    _fields_ = [
        ("num_particles", C.c_int),
        ("num_time_slices", C.c_int),
        ("box", C.c_double * 3),
        ("tau", C.c_double),
        ("num_species", C.c_int),
        ("species_of", C.POINTER(C.c_int)),
        ("lambda_", C.POINTER(C.c_double)),
        ("num_images", C.c_int),
        ("device", C.c_int),
    ]


class BisectionDesc(C.Structure):
    _fields_ = [
        ("num_levels", C.c_int),
        ("steps_per_block", C.c_int),
        ("shortrange_at_higher_levels", C.c_int),
        ("use_longrange", C.c_int),
        ("precision", C.c_int),
        ("shadow", C.c_int),
        ("cluster_ctas", C.c_int),
        ("threads_per_cta", C.c_int),
        ("schedule", C.c_int),
        ("neighbor_skin", C.c_double),
        ("neighbor_max", C.c_int),
        ("mixed_guard", C.c_int),
        ("wait_cap", C.c_int),
        ("test_wait", C.c_int),
    ]


class ChainDesc(C.Structure):
    _fields_ = [
        ("num_particles", C.c_int),
        ("num_time_slices", C.c_int),
        ("box", C.c_double * 3),
        ("tau", C.c_double),
        ("lambda_", C.c_double),
        ("num_images", C.c_int),
        ("num_levels", C.c_int),
        ("steps_per_block", C.c_int),
        ("seed", C.c_uint64),
        ("grid_start", C.c_double),
        ("grid_end", C.c_double),
        ("num_grid", C.c_int),
        ("num_tau", C.c_int),
        ("tau_pos", C.c_int),
        ("u00", C.POINTER(C.c_double)),
        ("path", C.POINTER(C.c_double)),
    ]


class EnergyTerms(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("kinetic", "du_short", "du_long", "v_short", "v_long", "total")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class BisectionStats(C.Structure):
    _fields_ = [
        ("moves", C.c_int64),
        ("accepted", C.c_int64),
        ("stages_attempted", C.c_int64),
        ("pair_evals", C.c_int64),
        ("flips", C.c_int64),
        ("status", C.c_int32),
        ("pad", C.c_int32),
        ("redone", C.c_int64),
        ("reevaluated", C.c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


MOVE_RECORD = np.dtype([
    ("slice1", np.int32), ("ptcl", np.int32), ("accepted", np.int32), ("stages_passed", np.int32),
    ("dS", np.float64, (8,)), ("dS_shadow", np.float64, (8,)),
    ("dS_bound", np.float32, (8,)), ("reevaluated", np.int32), ("pad", np.int32),
])

_d, _i, _p = C.c_double, C.c_int, C.c_void_p
_dp, _ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
_SIGS = {
    "pimc_status_string": (C.c_char_p, [_i]),
    "pimc_version": (_i, []),
    "pimc_create": (_i, [C.POINTER(SystemDesc), C.POINTER(_p)]),
    "pimc_destroy": (_i, [_p]),
    "pimc_last_error": (_i, [_p, C.c_char_p, _i]),
    "pimc_pa_david_from_dm": (_i, [_p, _i, _i, C.c_char_p, _i]),
    "pimc_dm_read_info": (_i, [C.c_char_p, _d, _ip, _ip, _ip, _ip, _ip, _dp, _dp]),
    "pimc_dm_read_tables": (_i, [C.c_char_p, _d, _dp, _dp, _dp, _dp]),
    "pimc_pa_david": (_i, [_p, _i, _i, _i, _d, _d, _i, _i, _i, _dp, _dp, _i, _i]),
    "pimc_pa_tricubic": (_i, [_p, _i, _i, _dp, _dp, _dp, _i, _d, _dp, _dp, _d, _d, _i, _dp]),
    "pimc_set_path": (_i, [_p, _i, _dp]),
    "pimc_get_path": (_i, [_p, _i, _dp]),
    "pimc_single_action": (_i, [_p, _i, _i, _i, _i, _ip, _i, _i, _i, _dp]),
    "pimc_d_dbeta": (_i, [_p, _i, _i, _i, _i, _dp]),
    "pimc_accept_copy": (_i, [_p, _i, _i, _ip, _i]),
    "pimc_reject_copy": (_i, [_p, _i, _i, _ip, _i]),
    "pimc_setup_kvecs": (_i, [_p, _d, _ip]),
    "pimc_get_kvecs": (_i, [_p, _dp]),
    "pimc_set_longrange": (_i, [_p, _i, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _i]),
    "pimc_calc_rhok": (_i, [_p]),
    "pimc_update_rhok": (_i, [_p, _i, _i, _ip, _i, _i]),
    "pimc_get_rhok": (_i, [_p, _i, _dp]),
    "pimc_pa_coulomb": (_i, [_p, _i, _i, _d, _i]),
    "pimc_longrange_coulomb": (_i, [_p, _i, _i]),
    "pimc_davidlongrange_yk": (_i, [_p, _i, _dp, _dp, _i]),
    "pimc_davidlongrange_v": (_i, [_p, _i, _i, _dp]),
    "pimc_coulomb_breakup": (_i, [_dp, _d, _d, _i, _i, _d, _i, _dp] + [_dp] * 11),
    "pimc_quintic_spline": (_i, [_i, _d, _dp, _dp]),
    "pimc_energy": (_i, [_p, C.POINTER(EnergyTerms)]),
    "pimc_gofr_setup": (_i, [_p, _d, _d, _i]),
    "pimc_gofr_accumulate": (_i, [_p]),
    "pimc_gofr_get": (_i, [_p, C.POINTER(C.c_uint64), _dp, C.POINTER(C.c_longlong)]),
    "pimc_gofr_reset": (_i, [_p]),
    "pimc_bisection_setup": (_i, [_p, C.POINTER(BisectionDesc)]),
    "pimc_rng_seed": (_i, [_p, C.c_uint64]),
    "pimc_bisection_windows": (_i, [_p, _ip]),
    "pimc_run_bisection": (_i, [_p, _i, _p, C.POINTER(BisectionStats)]),
    "pimc_run_bisection_async": (_i, [_p, _i]),
    "pimc_bisection_get_stats": (_i, [_p, C.POINTER(BisectionStats)]),
    "pimc_bisection_occupancy": (_i, [_p, _ip]),
    "pimc_synchronize": (_i, [_p]),
    "pimc_stream": (_p, [_p]),
    "pimc_batch_create": (_i, [_i, _i, C.POINTER(ChainDesc), C.POINTER(_p)]),
    "pimc_batch_destroy": (_i, [_p]),
    "pimc_batch_last_error": (_i, [_p, C.c_char_p, _i]),
    "pimc_batch_config": (_i, [_p, _i, _i, _i, _i, _i, _d]),
    "pimc_batch_run": (_i, [_p, _i, _p, C.POINTER(BisectionStats)]),
    "pimc_batch_run_async": (_i, [_p, _i]),
    "pimc_batch_autotune": (_i, [_p, _i, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i), C.POINTER(_d),
                                 C.POINTER(_d)]),
    "pimc_batch_get_stats": (_i, [_p, _i, C.POINTER(BisectionStats)]),
    "pimc_batch_set_guard": (_i, [_p, _i]),
    "pimc_read_bandwidth": (_i, [_i, C.c_size_t, _i, _i, _dp]),
    "pimc_batch_get_path": (_i, [_p, _i, _dp]),
    "pimc_batch_synchronize": (_i, [_p]),
    "pimc_batch_stream": (_p, [_p]),
    "pimc_shortrange_single_noalloc": (_i, [_p, _i, _i, _dp, _p, _d, _d, _i, _i, _i, _ip, _i, _i, _p, _p]),
    "pimc_init_random_fixed": (_i, [_dp, _i, _d, C.c_uint64, _dp]),
    "pimc_stream_uniform": (_i, [C.c_uint64, C.c_uint32, C.c_uint64, _dp]),
    "pimc_shift_data": (_i, [_p, _i]),
    "pimc_shift_move": (_i, [_p, _ip]),
    "pimc_checkpoint_write": (_i, [_p, C.c_char_p]),
    "pimc_checkpoint_read": (_i, [_p, C.c_char_p]),
}
for _name, (_res, _args) in _SIGS.items():
    _f = getattr(_lib, _name)
    _f.restype = _res
    _f.argtypes = _args

EXPORTED = tuple(_SIGS)


def lib():
    return _lib


def _dptr(a):
    return a.ctypes.data_as(_dp)


def _iptr(a):
    return a.ctypes.data_as(_ip)


def read_dm(path, desired_tau):
    """Host-only: the DavidPA tables of a squarer .dm file as the library reads them.

    Returns a dict with the grid, tau_pos and [num_tau][num_grid][num_cols]
    arrays ukj, ukj_d2, dukj, dukj_d2 (column 0 = potential).
    """
    vals = [C.c_int() for _ in range(5)]
    g0, g1 = C.c_double(), C.c_double()
    rc = _lib.pimc_dm_read_info(path.encode(), desired_tau, *[C.byref(v) for v in vals], C.byref(g0), C.byref(g1))
    if rc:
        raise PimcError(rc, f"pimc_dm_read_info({path})")
    ng, nc, nt, tp, gt = [v.value for v in vals]
    arrs = [np.empty((nt, ng, nc)) for _ in range(4)]
    rc = _lib.pimc_dm_read_tables(path.encode(), desired_tau, *[_dptr(a) for a in arrs])
    if rc:
        raise PimcError(rc, f"pimc_dm_read_tables({path})")
    return dict(num_grid=ng, num_cols=nc, num_tau=nt, tau_pos=tp, grid_type=gt, grid_start=g0.value,
                grid_end=g1.value, ukj=arrs[0], ukj_d2=arrs[1], dukj=arrs[2], dukj_d2=arrs[3])


class PathData:
    """Owns one pimc_context: path copies, pair action, device state.

    The mirrored OLD/NEW path of PathClass (MirroredClass.h:23-200) lives on
    the device; SetMode chooses which copy the Action objects evaluate, like
    the reference's global ActiveCopy.
    """

    def __init__(self, num_particles, num_time_slices, box, tau, lam, num_images=0, device=0):
        self.N = int(num_particles)
        self.S = int(num_time_slices)
        self.box = np.ascontiguousarray(box, dtype=np.float64)
        self.tau = float(tau)
        self.lam = float(lam)
        self._species = np.zeros(self.N, dtype=np.int32)
        self._lambda = np.array([lam], dtype=np.float64)
        d = SystemDesc()
        d.num_particles = self.N
        d.num_time_slices = self.S
        for i in range(3):
            d.box[i] = self.box[i]
        d.tau = self.tau
        d.num_species = 1
        d.species_of = _iptr(self._species)
        d.lambda_ = _dptr(self._lambda)
        d.num_images = int(num_images)
        d.device = int(device)
        h = _p()
        rc = _lib.pimc_create(C.byref(d), C.byref(h))
        if rc:
            raise PimcError(rc, "pimc_create")
        self.h = h
        self.mode = OLDMODE
        self._keep = []

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.pimc_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc, what):
        if rc:
            buf = C.create_string_buffer(512)
            _lib.pimc_last_error(self.h, buf, 512)
            raise PimcError(rc, f"{what}: {buf.value.decode(errors='replace')}")

    # ---- MirroredClass ----
    def SetMode(self, mode):
        assert mode in (OLDMODE, NEWMODE)
        self.mode = mode

    def set_path(self, path, copy=BOTH):
        path = np.ascontiguousarray(path, dtype=np.float64)
        assert path.shape == (self.S, self.N, 3), path.shape
        self._check(_lib.pimc_set_path(self.h, copy, _dptr(path)), "set_path")

    def get_path(self, copy=OLDMODE, out=None):
        """The path copy as [slices][particles][3]; into `out` (a C-contiguous
        float64 array of that shape, e.g. a view of pinned host memory) when given."""
        if out is None:
            out = np.empty((self.S, self.N, 3))
        assert out.shape == (self.S, self.N, 3) and out.dtype == np.float64 and out.flags.c_contiguous, out.shape
        self._check(_lib.pimc_get_path(self.h, copy, _dptr(out)), "get_path")
        return out

    def seed(self, seed):
        """Seeds every RNG stream of the chain (pimc_rng_seed)."""
        self._check(_lib.pimc_rng_seed(self.h, C.c_uint64(seed)), "rng_seed")

    def ShiftData(self, slices_to_shift):
        """PathClass::ShiftPathData (PathClass.cc:1026-1110) on both copies."""
        self._check(_lib.pimc_shift_data(self.h, int(slices_to_shift)), "shift_data")

    def ShiftMove(self):
        """ShiftMoveClass::MakeMove (MetaMoves.cc:39-65); returns the slices shifted."""
        n = C.c_int()
        self._check(_lib.pimc_shift_move(self.h, C.byref(n)), "shift_move")
        return n.value

    def write_checkpoint(self, filename):
        """Both path copies, RNG stream positions and move counters, flat binary."""
        self._check(_lib.pimc_checkpoint_write(self.h, os.fsencode(filename)), "checkpoint_write")

    def read_checkpoint(self, filename):
        """Restores a chain written by write_checkpoint; call it after the
        BisectionBlock is set up and seeded (both reset what it restores)."""
        self._check(_lib.pimc_checkpoint_read(self.h, os.fsencode(filename)), "checkpoint_read")

    # ---- pair actions ----
    def pa_david_from_dm(self, dm_path, num_offdiag_terms=0):
        self._check(_lib.pimc_pa_david_from_dm(self.h, 0, 0, dm_path.encode(), num_offdiag_terms), "pa_david_from_dm")

    def pa_david(self, grid_type, grid_start, grid_end, ukj, dukj, tau_pos, num_offdiag_terms=0):
        ukj = np.ascontiguousarray(ukj, dtype=np.float64)
        dukj = np.ascontiguousarray(dukj, dtype=np.float64)
        nt, ng, nc = ukj.shape
        self._check(_lib.pimc_pa_david(self.h, 0, 0, grid_type, grid_start, grid_end, ng, nc, nt, _dptr(ukj),
                                       _dptr(dukj), tau_pos, num_offdiag_terms), "pa_david")

    def pa_zero(self, num_levels):
        """PAzeroFitClass (Common/PairAction/PAzeroFit.cc): U = dU = V = 0, as a
        DavidPA table of zeros on a two-point grid, so the sums are exactly zero."""
        end = float(np.sqrt(np.sum(self.box * self.box)))
        z = np.zeros((int(num_levels), 2, 2))
        self.pa_david(GRID_LINEAR, 0.0, end, z, z, 0, 0)

    def pa_tricubic(self, qgrid, ygrid, tgrid, smallest_beta, umat, dumat, pot_grid, pot_data):
        umat = np.ascontiguousarray(umat, dtype=np.float64)
        dumat = np.ascontiguousarray(dumat, dtype=np.float64)
        pot = np.ascontiguousarray(pot_data, dtype=np.float64)
        g = [np.array(x, dtype=np.float64) for x in (qgrid, ygrid, tgrid)]
        self._check(_lib.pimc_pa_tricubic(self.h, 0, 0, _dptr(g[0]), _dptr(g[1]), _dptr(g[2]), umat.shape[0],
                                          smallest_beta, _dptr(umat), _dptr(dumat), pot_grid[0], pot_grid[1],
                                          int(pot_grid[2]), _dptr(pot)), "pa_tricubic")

    # ---- actions ----
    def single_action(self, action, copy, slice1, slice2, active, level, precision=FP64):
        a = np.ascontiguousarray(active, dtype=np.int32)
        out = C.c_double()
        self._check(_lib.pimc_single_action(self.h, action, copy, slice1, slice2, _iptr(a), len(a), level,
                                            precision, C.byref(out)), "single_action")
        return out.value

    def d_dbeta(self, action, slice1, slice2, level=0):
        out = C.c_double()
        self._check(_lib.pimc_d_dbeta(self.h, action, slice1, slice2, level, C.byref(out)), "d_dbeta")
        return out.value

    def AcceptCopy(self, slice1, slice2, active):
        a = np.ascontiguousarray(active, dtype=np.int32)
        self._check(_lib.pimc_accept_copy(self.h, slice1, slice2, _iptr(a), len(a)), "accept_copy")

    def RejectCopy(self, slice1, slice2, active):
        a = np.ascontiguousarray(active, dtype=np.int32)
        self._check(_lib.pimc_reject_copy(self.h, slice1, slice2, _iptr(a), len(a)), "reject_copy")

    def synchronize(self):
        self._check(_lib.pimc_synchronize(self.h), "synchronize")

    # ---- long range: PathClass k-vectors and rho_k, LongRangeClass tables ----
    def setup_kvecs(self, kcutoff):
        nk = C.c_int()
        self._check(_lib.pimc_setup_kvecs(self.h, kcutoff, C.byref(nk)), "setup_kvecs")
        self.num_k = nk.value
        return nk.value

    def kvecs(self):
        out = np.empty((self.num_k, 3))
        self._check(_lib.pimc_get_kvecs(self.h, _dptr(out)), "get_kvecs")
        return out

    def set_longrange(self, ulong_k, ulong_r0, ushort_k0, ulong_k0, dulong_k, dulong_r0, dushort_k0, dulong_k0,
                      use_background=True):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
                (ulong_k, ulong_r0, ushort_k0, ulong_k0, dulong_k, dulong_r0, dushort_k0, dulong_k0)]
        self._check(_lib.pimc_set_longrange(self.h, arrs[1].shape[0], *[_dptr(a) for a in arrs],
                                            int(use_background)), "set_longrange")

    def davidlongrange_yk(self, kvals, uk_long, rpa=True):
        """DavidLongRangeClassYk tables (after setup_kvecs) from the squarer's
        k-space action uk_long at the magnitudes kvals."""
        kv = np.ascontiguousarray(kvals, dtype=np.float64)
        uk = np.ascontiguousarray(uk_long, dtype=np.float64)
        if kv.shape != uk.shape or kv.ndim != 1:
            raise ValueError("kvals and uk_long must be 1-D arrays of one length")
        self._check(_lib.pimc_davidlongrange_yk(self.h, len(kv), _dptr(kv), _dptr(uk), int(rpa)),
                    "davidlongrange_yk")

    def calc_rhok(self):
        self._check(_lib.pimc_calc_rhok(self.h), "calc_rhok")

    def update_rhok(self, slice1, slice2, active, level):
        a = np.ascontiguousarray(active, dtype=np.int32)
        self._check(_lib.pimc_update_rhok(self.h, slice1, slice2, _iptr(a), len(a), level), "update_rhok")

    def get_rhok(self, copy=OLDMODE):
        out = np.empty((self.S, self.num_k, 2))
        self._check(_lib.pimc_get_rhok(self.h, copy, _dptr(out)), "get_rhok")
        return out[..., 0] + 1j * out[..., 1]

    def pa_coulomb(self, z1z2, num_levels):
        """PAclassicalFitClass with a Coulomb potential Z1Z2/r."""
        self._check(_lib.pimc_pa_coulomb(self.h, 0, 0, z1z2, num_levels), "pa_coulomb")

    def longrange_coulomb(self, num_knots, use_background=True):
        """Optimized breakup of the Coulomb action (after setup_kvecs)."""
        self._check(_lib.pimc_longrange_coulomb(self.h, num_knots, int(use_background)), "longrange_coulomb")

    # ---- observables (EnergyClass, PairCorrelationClass) ----
    def energy(self):
        """ActionsClass::Energy terms of the OLD path; 'total' is the per-slice sample."""
        e = EnergyTerms()
        self._check(_lib.pimc_energy(self.h, C.byref(e)), "energy")
        return e.as_dict()

    def gofr_setup(self, start=0.0, end=0.0, num_points=101):
        self._check(_lib.pimc_gofr_setup(self.h, start, end, num_points), "gofr_setup")
        self._gofr_bins = num_points - 1

    def gofr_accumulate(self):
        self._check(_lib.pimc_gofr_accumulate(self.h), "gofr_accumulate")

    def gofr_get(self):
        """(histogram uint64, g(r) normalised like WriteBlock, number of samples)"""
        h = np.zeros(self._gofr_bins, dtype=np.uint64)
        g = np.zeros(self._gofr_bins)
        n = C.c_longlong()
        self._check(_lib.pimc_gofr_get(self.h, h.ctypes.data_as(C.POINTER(C.c_uint64)), _dptr(g), C.byref(n)),
                    "gofr_get")
        return h, g, n.value

    def gofr_reset(self):
        self._check(_lib.pimc_gofr_reset(self.h), "gofr_reset")


class ActionBaseClass:
    """ActionBaseClass (PIMC++/src/Actions/ActionBase.h:31-75) over the device."""

    kind = None

    def __init__(self, path_data: PathData, precision=FP64):
        self.PathData = path_data
        self.precision = precision

    def SingleAction(self, slice1, slice2, activeParticles, level):
        return self.PathData.single_action(self.kind, self.PathData.mode, slice1, slice2, activeParticles, level,
                                           self.precision)

    def Action(self, slice1, slice2, activeParticles, level):
        return self.SingleAction(slice1, slice2, activeParticles, level)

    def d_dBeta(self, slice1, slice2, level):
        return self.PathData.d_dbeta(self.kind, slice1, slice2, level)


class ShortRangeClass(ActionBaseClass):
    """ShortRangeClass (PIMC++/src/Actions/ShortRangeClass.cc:191-355)."""
    kind = ACTION_SHORTRANGE

    def GetName(self):
        return "ShortRange"


class KineticClass(ActionBaseClass):
    """KineticClass (PIMC++/src/Actions/KineticClass.cc:33-256)."""
    kind = ACTION_KINETIC

    def GetName(self):
        return "Kinetic"


class LongRangeClass(ActionBaseClass):
    """LongRangeClass (PIMC++/src/Actions/LongRangeClass.cc:273-442)."""
    kind = ACTION_LONGRANGE

    def GetName(self):
        return "LongRange"


class DavidLongRangeClassYk(ActionBaseClass):
    """DavidLongRangeClassYk (PIMC++/src/Actions/DavidLongRangeClassYk.cc:230-389),
    after PathData.davidlongrange_yk."""
    kind = ACTION_DAVIDLONGRANGE

    def GetName(self):
        return "DavidsLongRange"

    def V(self, slice1, slice2, level=0):
        out = C.c_double()
        self.PathData._check(_lib.pimc_davidlongrange_v(self.PathData.h, slice1, slice2, C.byref(out)),
                             "davidlongrange_v")
        return out.value


class BisectionBlock:
    """BisectionBlockClass::MakeMove on the device (BisectionBlock.cc:380-451).

    One call of `MakeMoves(n_blocks)` runs n_blocks blocks of StepsPerBlock
    moves each; the Local RNG stream is Philox-4x32-10 keyed by `seed`.
    schedule WINDOWS: a block is one round of concurrent slice windows;
    PROPOSALS: a round of windows with `cluster_ctas` concurrent proposal
    slots each, trace records [round][window][step][slot].
    """

    def __init__(self, path_data: PathData, num_levels, steps_per_block=1, shortrange_at_higher_levels=True,
                 precision=FP64, shadow=False, cluster_ctas=0, threads_per_cta=0, schedule=SEQUENTIAL,
                 use_longrange=False, neighbor_skin=0.0, neighbor_max=0, guard=GUARD_DECISION, wait_cap=0,
                 test_wait=0):
        self.PathData = path_data
        d = BisectionDesc()
        d.num_levels = num_levels
        d.steps_per_block = steps_per_block
        d.shortrange_at_higher_levels = int(shortrange_at_higher_levels)
        d.use_longrange = int(use_longrange)
        d.precision = precision
        d.shadow = int(shadow)
        d.cluster_ctas = cluster_ctas
        d.threads_per_cta = threads_per_cta
        d.schedule = schedule
        d.neighbor_skin = neighbor_skin
        d.neighbor_max = neighbor_max
        d.mixed_guard = guard_value(guard)
        d.wait_cap = wait_cap
        d.test_wait = test_wait
        self.desc = d
        self.steps_per_block = steps_per_block
        path_data._check(_lib.pimc_bisection_setup(path_data.h, C.byref(d)), "bisection_setup")
        w = C.c_int()
        path_data._check(_lib.pimc_bisection_windows(path_data.h, C.byref(w)), "bisection_windows")
        self.windows = w.value
        # PROPOSALS: cluster_ctas proposal slots per window (0 = the library's default, 8)
        self.proposals = (cluster_ctas or 8) if schedule == PROPOSALS else 1

    def seed(self, seed):
        self.PathData._check(_lib.pimc_rng_seed(self.PathData.h, C.c_uint64(seed)), "rng_seed")

    def MakeMoves(self, n_blocks, trace=True):
        st = BisectionStats()
        rec = (np.zeros(n_blocks * self.windows * self.steps_per_block * self.proposals, dtype=MOVE_RECORD)
               if trace else None)
        ptr = rec.ctypes.data_as(_p) if trace else None
        self.PathData._check(_lib.pimc_run_bisection(self.PathData.h, n_blocks, ptr, C.byref(st)), "run_bisection")
        return rec, st.as_dict()

    def launch_async(self, n_blocks):
        self.PathData._check(_lib.pimc_run_bisection_async(self.PathData.h, n_blocks), "run_bisection_async")

    def occupancy(self):
        """Clusters of this launch shape that fit on the device at once."""
        v = C.c_int()
        self.PathData._check(_lib.pimc_bisection_occupancy(self.PathData.h, C.byref(v)), "occupancy")
        return v.value

    def stats(self):
        st = BisectionStats()
        self.PathData._check(_lib.pimc_bisection_get_stats(self.PathData.h, C.byref(st)), "get_stats")
        return st.as_dict()


class BatchChains:
    """Many independent chains (the reference's clones) advanced by one
    persistent launch of the device BisectionBlock driver.

    chains: list of dicts with keys N, slices, box, tau, lam, num_levels,
    steps_per_block, seed, grid (start, end, n), u00 [num_tau][n], tau_pos,
    path [slices][N][3], num_images (optional).
    """

    def __init__(self, chains, device=0, precision=MIXED, shadow=False, threads_per_cta=0, ctas=0, max_split=0,
                 split_ratio=0.5):
        self._keep = []
        descs = (ChainDesc * len(chains))()
        self.shapes = []
        for i, c in enumerate(chains):
            u00 = np.ascontiguousarray(c["u00"], dtype=np.float64)
            path = np.ascontiguousarray(c["path"], dtype=np.float64)
            self._keep += [u00, path]
            d = descs[i]
            d.num_particles = c["N"]
            d.num_time_slices = c["slices"]
            for k in range(3):
                d.box[k] = c["box"][k]
            d.tau = c["tau"]
            d.lambda_ = c["lam"]
            d.num_images = c.get("num_images", 0)
            d.num_levels = c["num_levels"]
            d.steps_per_block = c["steps_per_block"]
            d.seed = c["seed"]
            d.grid_start, d.grid_end, d.num_grid = c["grid"][0], c["grid"][1], int(c["grid"][2])
            d.num_tau = u00.shape[0]
            d.tau_pos = c.get("tau_pos", 0)
            d.u00 = _dptr(u00)
            d.path = _dptr(path)
            self.shapes.append(path.shape)
        h = _p()
        rc = _lib.pimc_batch_create(device, len(chains), descs, C.byref(h))
        if rc:
            raise PimcError(rc, "pimc_batch_create")
        self.h = h
        self.n = len(chains)
        self.steps = max(c["steps_per_block"] for c in chains)
        self.config(precision, shadow, threads_per_cta, ctas, max_split, split_ratio)

    def _check(self, rc, what):
        if rc:
            buf = C.create_string_buffer(512)
            _lib.pimc_batch_last_error(self.h, buf, 512)
            raise PimcError(rc, f"{what}: {buf.value.decode(errors='replace')}")

    def config(self, precision=MIXED, shadow=False, threads_per_cta=0, ctas=0, max_split=0, split_ratio=0.5):
        self._check(_lib.pimc_batch_config(self.h, precision, int(shadow), threads_per_cta, ctas, max_split,
                                           split_ratio), "batch_config")

    def run(self, n_blocks, trace=False):
        st = BisectionStats()
        rec = np.zeros(self.n * n_blocks * self.steps, dtype=MOVE_RECORD) if trace else None
        ptr = rec.ctypes.data_as(_p) if trace else None
        self._check(_lib.pimc_batch_run(self.h, n_blocks, ptr, C.byref(st)), "batch_run")
        if trace:
            rec = rec.reshape(self.n, n_blocks * self.steps)
        return rec, st.as_dict()

    def run_async(self, n_blocks):
        self._check(_lib.pimc_batch_run_async(self.h, n_blocks), "batch_run_async")

    def synchronize(self):
        self._check(_lib.pimc_batch_synchronize(self.h), "batch_synchronize")

    @property
    def stream(self):
        return _lib.pimc_batch_stream(self.h)

    def set_guard(self, guard=GUARD_DECISION):
        """Mixed precision: GUARD_DECISION (default), GUARD_NONE or GUARD_RELATIVE (or True / False)."""
        self._check(_lib.pimc_batch_set_guard(self.h, guard_value(guard)), "batch_set_guard")

    def autotune(self, n_blocks=1):
        """Pick threads_per_cta and the CTA count by timing; chains keep their state."""
        t, c, sp, r, ms = _i(), _i(), _i(), C.c_double(), C.c_double()
        self._check(_lib.pimc_batch_autotune(self.h, n_blocks, C.byref(t), C.byref(c), C.byref(sp), C.byref(r),
                                             C.byref(ms)), "batch_autotune")
        return dict(threads_per_cta=t.value, ctas=c.value, max_split=sp.value, split_ratio=r.value, ms=ms.value)

    def stats(self, chain=-1):
        st = BisectionStats()
        self._check(_lib.pimc_batch_get_stats(self.h, chain, C.byref(st)), "batch_get_stats")
        return st.as_dict()

    def path(self, chain):
        out = np.empty(self.shapes[chain])
        self._check(_lib.pimc_batch_get_path(self.h, chain, _dptr(out)), "batch_get_path")
        return out

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.pimc_batch_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()


def coulomb_breakup(box, z1z2, smallest_beta, num_levels, num_knots, kcutoff, kvecs):
    """Host-only optimized breakup of a Coulomb pair action; returns a dict of tables."""
    kv = np.ascontiguousarray(kvecs, dtype=np.float64).reshape(-1, 3)
    nk = kv.shape[0]
    box = np.ascontiguousarray(box, dtype=np.float64)
    out = dict(ulong_k=np.zeros((num_levels, nk)), dulong_k=np.zeros((num_levels, nk)))
    for k in ("ulong_r0", "dulong_r0", "ushort_k0", "dushort_k0", "ulong_k0", "dulong_k0"):
        out[k] = np.zeros(num_levels)
    rmax = np.zeros(1)
    out["ulong_r"] = np.zeros((num_levels, 1000, 6))
    out["dulong_r"] = np.zeros((num_levels, 1000, 6))
    rc = _lib.pimc_coulomb_breakup(_dptr(box), z1z2, smallest_beta, num_levels, num_knots, kcutoff, nk, _dptr(kv),
                                   _dptr(out["ulong_k"]), _dptr(out["dulong_k"]), _dptr(out["ulong_r0"]),
                                   _dptr(out["dulong_r0"]), _dptr(out["ushort_k0"]), _dptr(out["dushort_k0"]),
                                   _dptr(out["ulong_k0"]), _dptr(out["dulong_k0"]), _dptr(rmax),
                                   _dptr(out["ulong_r"]), _dptr(out["dulong_r"]))
    if rc:
        raise PimcError(rc, "pimc_coulomb_breakup")
    out["rmax"] = float(rmax[0])
    return out


def read_bandwidth(device=0, nbytes=64 << 20, passes=16, reps=10):
    """GB/s of 16-byte loads through L2 over an nbytes buffer (L2 read
    bandwidth below 126 MB, HBM read bandwidth well above it)."""
    v = C.c_double()
    rc = _lib.pimc_read_bandwidth(device, nbytes, passes, reps, C.byref(v))
    if rc:
        raise PimcError(rc, "read_bandwidth")
    return v.value


def init_random_fixed(box, num_particles, radius, seed):
    """PathClass::InitRandomFixed (InitPaths.cc:966-999) positions [N][3] from
    the World stream of `seed`; raises where the reference aborts."""
    b = np.ascontiguousarray(box, dtype=np.float64)
    out = np.zeros((int(num_particles), 3))
    rc = _lib.pimc_init_random_fixed(_dptr(b), int(num_particles), float(radius), C.c_uint64(seed), _dptr(out))
    if rc:
        raise PimcError(rc, "InitRandomFixed: a particle took 1000 tries; decrease the excluded radius"
                        if rc == 5 else "pimc_init_random_fixed")
    return out


def stream_uniform(seed, stream, index):
    """Element `index` of the library's Philox stream `stream` under `seed`."""
    out = C.c_double()
    _lib.pimc_stream_uniform(C.c_uint64(seed), C.c_uint32(stream), C.c_uint64(index), C.byref(out))
    return out.value


def quintic_spline(h, y):
    """Natural quintic spline coefficients [n][6] of y on a uniform grid."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    coef = np.zeros((len(y), 6))
    rc = _lib.pimc_quintic_spline(len(y), h, _dptr(y), _dptr(coef))
    if rc:
        raise PimcError(rc, "pimc_quintic_spline")
    return coef

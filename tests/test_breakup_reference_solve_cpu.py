"""The C4 breakup solved the reference's way against the library's solve.

OptimizedBreakupClass::DoBreakup (Common/Ewald/OptimizedBreakup.cc:196-290)
fits the LPQHI coefficients through the normal equations A t = b, A = sum_k w
c c^T, inverted by SVD with singular values below 1e-16 S_max dropped.  The
library solves the same least-squares problem on the weighted design matrix
(QR, then a Jacobi SVD of R with a 1e-8 cutoff), because A's condition
number for jellium with 49 knots (~1e15) leaves its smallest singular values
at rounding level.  The two fits split the Coulomb action differently
between the short- and long-range parts (Ulong(0) moves by a few per cent),
but the split is arbitrary: what a simulation uses is the sum.  This test
restates the reference's procedure (oracle/breakup.normal_equation_svd) and
checks, on a C4 jellium path with the oracle's evaluation, that the
quantities that do not depend on the split agree:

* the total action, ShortRange + LongRange SingleAction over every particle
  and slice, within 1e-3 relative;
* the interaction part of the energy, du_short + du_long, within 1e-3;
* beyond r_c the long-range part is the full action for both fits.

The individual pieces (Ulong(r), du_short, du_long, v_short) differ by up to
~10 %, which is why C4 parity in the GPU tests is stated against the
library's breakup tables (the oracle is given the same tables).
"""
import numpy as np

import oracle as O
import oracle.breakup as OB
import pimcplusplus_b200 as P

L_C4 = (4.0 * np.pi / 3.0 * 128) ** (1.0 / 3.0) * 4.0
BOX = np.array([L_C4] * 3)
TAU, LEVELS, Z1Z2 = 8.0 / 64, 3, 2.0


def _system(t, path):
    o = O.System(128, 65, BOX, TAU, 1.0, 0)
    o.set_pa(O.PairAction.classical_coulomb(TAU, LEVELS, Z1Z2))
    o.setup_kvecs(1.2)
    o.set_longrange(t["ulong_k"], t["ulong_r0"], t["ushort_k0"], t["ulong_k0"], t["dulong_k"], t["dulong_r0"],
                    t["dushort_k0"], t["dulong_k0"], use_background=True)
    o.set_ulong(t["ulong_r"], t["dulong_r"], t["rmax"])
    o.set_path(path, 0)
    o.set_path(path, 1)
    o.calc_rhok_all()
    return o


def test_reference_normal_equation_solve_moves_only_the_split():
    o0 = O.System(128, 65, BOX, TAU, 1.0, 0)
    assert o0.setup_kvecs(1.2) == 510
    kv, _ = o0.kvecs()
    lib = P.coulomb_breakup(BOX, Z1Z2, TAU, LEVELS, 49, 1.2, kv)
    ref, basis = OB.coulomb_breakup(BOX, Z1Z2, TAU, LEVELS, 49, 1.2, kv, solve="normal_svd")
    # the reference's cutoff keeps every singular value here (none below 1e-16 S_max)
    assert len(ref["singular_dropped"]) == 2 * LEVELS
    # the split differs visibly ...
    assert np.max(np.abs(ref["ulong_r0"] - lib["ulong_r0"]) / np.abs(lib["ulong_r0"])) > 1e-3
    # ... but beyond r_c both long-range parts are the full action
    r = np.arange(1000) * (lib["rmax"] / 999)
    far = (r > basis.rc * (1 + 1e-9)) & (np.arange(1000) < 999)
    for level in range(LEVELS):
        beta = TAU * 2 ** level
        assert np.allclose(ref["ulong_r"][level, far, 0], beta * Z1Z2 / r[far], rtol=1e-12)
        assert np.allclose(lib["ulong_r"][level, far, 0], beta * Z1Z2 / r[far], rtol=1e-12)

    rng = np.random.default_rng(11)
    path = np.repeat(((rng.random((128, 3)) - 0.5) * BOX)[None], 65, axis=0)
    path[1:-1] += rng.normal(0.0, 0.3, path[1:-1].shape)
    every = list(range(128))
    vals = {}
    for name, t in (("library", lib), ("reference", ref)):
        o = _system(t, path)
        e = o.energy()
        action = o.shortrange_single(0, 64, every, 0) + o.longrange_single(0, 64, every, 0)
        vals[name] = (action, e["du_short"] + e["du_long"], e["du_short"])
    (a_l, du_l, s_l), (a_r, du_r, s_r) = vals["library"], vals["reference"]
    assert abs(a_l - a_r) <= 1e-3 * abs(a_l), (a_l, a_r)
    assert abs(du_l - du_r) <= 1e-3 * abs(du_l), (du_l, du_r)
    # the pieces on their own move by far more than the sums
    assert abs(s_l - s_r) > 10 * abs(du_l - du_r)

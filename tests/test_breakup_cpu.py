"""Host-side optimized Ewald breakup of the Coulomb pair action and the
natural quintic spline of Ulong(r), against the numpy/SciPy restatement in
oracle/breakup.py (tolerance parity: the reference's SVD and quintic spline
routines are third-party code the oracle replaces with numpy and SciPy)."""
import numpy as np
import pytest
from scipy.integrate import quad

import oracle as O
import oracle.breakup as OB
import pimcplusplus_b200 as P

# C4: jellium r_s = 4 bohr, N = 128, M = 64 at beta = 8 Ry^-1
L_C4 = (4.0 * np.pi / 3.0 * 128) ** (1.0 / 3.0) * 4.0
BOX = np.array([L_C4] * 3)


def test_quintic_spline_matches_scipy():
    rng = np.random.default_rng(3)
    x = np.arange(200) * 0.05
    y = np.sin(2.0 * x) * np.exp(-0.2 * x) + 0.01 * rng.standard_normal(200).cumsum()
    got = P.quintic_spline(0.05, y)
    ref, _ = OB.quintic_coefficients(x, y)
    scale = np.abs(ref).max(axis=0)
    assert np.all(np.abs(got - ref).max(axis=0) <= 1e-9 * scale + 1e-14)


def test_lpqhi_fourier_transform_matches_quadrature():
    b = OB.Lpqhi(5.0, 6, BOX)
    ks = np.array([0.7, 1.9, 4.3])
    c = b.c(ks)
    for n in (0, 1, 2, 4, 8, 13, 17):
        for j, k in enumerate(ks):
            f = lambda r: 4 * np.pi / (k * b.omega) * b.h(n, np.array([r]))[0] * r * np.sin(k * r)
            ref = sum(quad(f, a, a + b.delta, epsabs=1e-15, epsrel=1e-12)[0] for a in b.delta * np.arange(5))
            assert abs(c[n, j] - ref) <= 1e-9 * max(abs(ref), 1e-6), (n, k, c[n, j], ref)


@pytest.fixture(scope="module")
def c4_breakup():
    o = O.System(128, 65, BOX, 0.125, 1.0, 0)
    nk = o.setup_kvecs(1.20)
    kv, _ = o.kvecs()
    got = P.coulomb_breakup(BOX, 2.0, 0.125, 2, 49, 1.20, kv)
    ref, basis = OB.coulomb_breakup(BOX, 2.0, 0.125, 2, 49, 1.20, kv)
    return nk, got, ref, basis


def test_breakup_kvector_count(c4_breakup):
    nk, _, _, _ = c4_breakup
    assert nk == 510


# The fit's condition number (~3e7 for these 147 basis functions) amplifies
# the ~1e-10 relative rounding differences of c_n(k) at small k (the
# integration-by-parts recursion cancels there) into ~1e-4 relative
# differences of the poorly determined short-distance part of Ulong; both
# implementations (and the reference's own) carry that uncertainty.
TOL = 2e-4


def test_breakup_tables_match_oracle(c4_breakup):
    _, got, ref, _ = c4_breakup
    assert abs(got["rmax"] - ref["rmax"]) < 1e-12
    for tag in ("", "d"):
        u, r = got[tag + "ulong_r"][:, :, 0], ref[tag + "ulong_r"][:, :, 0]
        assert np.abs(u - r).max() <= TOL * np.abs(r).max(), tag
        k = tag + "ulong_k"
        assert np.abs(got[k] - ref[k]).max() <= TOL * np.abs(ref[k]).max(), k
        for k in (tag + "ulong_r0", tag + "ulong_k0", ("dushort_k0" if tag else "ushort_k0")):
            assert np.allclose(got[k], ref[k], rtol=TOL, atol=0), (k, got[k], ref[k])
        # the splines agree between the knots too (mid-interval values)
        h = got["rmax"] / 999
        for level in range(2):
            vals = []
            for c in (got[tag + "ulong_r"][level], ref[tag + "ulong_r"][level]):
                P = 0.5 * h
                vals.append(((((c[:-1, 5] * P + c[:-1, 4]) * P + c[:-1, 3]) * P + c[:-1, 2]) * P + c[:-1, 1]) * P
                            + c[:-1, 0])
            assert np.abs(vals[0] - vals[1]).max() <= TOL * np.abs(vals[1]).max(), (tag, level)


def test_breakup_quintic_interpolates_grid(c4_breakup):
    """The library's Ulong spline passes through its own grid values and is C2."""
    _, got, _, _ = c4_breakup
    h = got["rmax"] / 999
    for level in range(2):
        c = got["ulong_r"][level]
        # value at the right end of interval i equals the next knot's value
        P = h
        right = ((((c[:-2, 5] * P + c[:-2, 4]) * P + c[:-2, 3]) * P + c[:-2, 2]) * P + c[:-2, 1]) * P + c[:-2, 0]
        assert np.allclose(right, c[1:-1, 0], rtol=1e-10, atol=1e-13)


def test_breakup_reproduces_coulomb_beyond_rc(c4_breakup):
    """Ulong equals the full action beyond r_c; U_long + U_short = U everywhere."""
    _, got, ref, basis = c4_breakup
    r = np.arange(1000) * (got["rmax"] / 999)
    far = (r > ref["rc"] * (1 + 1e-12)) & (np.arange(1000) < 999)  # row 999 repeats interval 998
    for level in range(2):
        beta = 0.125 * 2 ** level
        assert np.allclose(got["ulong_r"][level, far, 0], beta * 2.0 / r[far], rtol=1e-14)
        assert np.allclose(got["dulong_r"][level, far, 0], 2.0 / r[far], rtol=1e-14)
    # the long-range part is smooth and finite at r = 0
    assert np.all(np.isfinite(got["ulong_r0"])) and np.all(np.abs(got["ulong_r0"]) < 10 * 0.125 * 2.0 / 1.0)

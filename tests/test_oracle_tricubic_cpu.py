"""The oracle's PAtricubicFit evaluation, pinned against an independent numpy
statement of the reference's formulas on the oracle's node table:

* MyTricubicSpline::operator() (Common/Splines/MyTricubicSpline.h:197-334):
  the Hermite basis p1, p2, h·q1, h·q2 per axis (h:38-45) over the 8 node
  values F, Fx, Fy, Fz, Fxy, Fxz, Fyz, Fxyz of the cell's 8 corners, the cell
  index clamped to [0, N-2];
* PAtricubicFitClass::U (Common/PairAction/PAtricubicFit.cc:659-695): z = |z|,
  smax = 2q, y = z/smax, t = (s-z)/(smax-z) inside the fit (q = 0 falls
  outside it: z < 2q fails), else the primitive ½β_l(V(r)+V(r')) with SplinePot V
  (Common/PH/SplinePot.cc:19-31), a natural cubic spline, zero beyond its grid.
"""
import numpy as np
from scipy.interpolate import CubicSpline

import oracle as O
from helpers import tricubic_case


def _axis(g, x):
    start, end, n = g
    delta = (end - start) / (n - 1)
    i = int(np.rint((x - start) * (1.0 / delta) - 0.5))
    i = min(max(i, 0), n - 2)
    h = delta
    u = (x - (start + i * delta)) / h
    p1 = (u - 1.0) ** 2 * (1.0 + 2.0 * u)
    p2 = u * u * (3.0 - 2.0 * u)
    q1 = u * (u - 1.0) ** 2
    q2 = u * u * (u - 1.0)
    return i, np.array([p1, p2, h * q1, h * q2])


# node-value index of (d/dx, d/dy, d/dz) in F, Fx, Fy, Fz, Fxy, Fxz, Fyz, Fxyz
_COMP = {(0, 0, 0): 0, (1, 0, 0): 1, (0, 1, 0): 2, (0, 0, 1): 3, (1, 1, 0): 4, (1, 0, 1): 5, (0, 1, 1): 6,
         (1, 1, 1): 7}


def tricubic_eval(F, gx, gy, gz, x, y, z):
    ix, a = _axis(gx, x)
    iy, b = _axis(gy, y)
    iz, c = _axis(gz, z)
    val = 0.0
    # basis k of an axis: 0 value at lo, 1 value at hi, 2 slope at lo, 3 slope at hi
    for ka in range(4):
        for kb in range(4):
            for kc in range(4):
                comp = _COMP[(ka >> 1, kb >> 1, kc >> 1)]
                val += a[ka] * b[kb] * c[kc] * F[ix + (ka & 1), iy + (kb & 1), iz + (kc & 1), comp]
    return val


def test_tricubic_evaluation_matches_independent_statement():
    gx, gy, gz = (0.0, 2.0, 9), (-1.0, 1.5, 7), (0.5, 3.0, 11)
    xs = np.linspace(*gx[:2], gx[2])[:, None, None]
    ys = np.linspace(*gy[:2], gy[2])[None, :, None]
    zs = np.linspace(*gz[:2], gz[2])[None, None, :]
    f = np.sin(1.3 * xs) * np.cos(0.7 * ys + 0.2) * np.exp(-0.3 * zs) + xs * ys * zs
    t = O.Tricubic(gx, gy, gz, f)
    F = t.coefs()
    assert np.array_equal(F[..., 0], f)
    rng = np.random.default_rng(7)
    for _ in range(300):
        x, y, z = rng.uniform(-0.05, 2.05), rng.uniform(-1.05, 1.55), rng.uniform(0.45, 3.05)
        want = tricubic_eval(F, gx, gy, gz, x, y, z)
        assert abs(t(x, y, z) - want) <= 1e-12 * max(1.0, abs(want))


def test_tricubic_pair_action_mapping_and_fallback():
    cfg, tau, box, tabs = tricubic_case(n=16, m=16, levels=2, nq=12, ny=6, nt=6)
    qg, yg, tg, umat, dumat, pg, pot = tabs
    pa = O.PairAction.tricubic(qg, yg, tg, tau, umat, dumat, pg, pot)
    spl = CubicSpline(np.linspace(pg[0], pg[1], pg[2]), pot, bc_type="natural")

    def V(r):
        return float(spl(r)) if r <= pg[1] else 0.0

    rng = np.random.default_rng(3)
    qmax = qg[1]
    for level in range(umat.shape[0]):
        F = O.Tricubic(qg, yg, tg, umat[level]).coefs()
        beta = tau * 2.0 ** level
        checked_fit = checked_prim = 0
        for _ in range(400):
            q = rng.uniform(0.0, 1.15 * qmax)
            z = rng.uniform(-2.2, 2.2) * q
            # s >= |z| always: s = |r - r'| >= ||r| - |r'||
            s = abs(z) + rng.uniform(0.0, 1.3) * abs(2.0 * q - abs(z))
            za, smax = abs(z), 2.0 * q
            if q <= qmax and za < smax and s < smax:
                want = tricubic_eval(F, qg, yg, tg, q, za / smax, (s - za) / (smax - za))
                tol = 1e-12
                checked_fit += 1
            else:
                # SciPy's natural spline against the reference's: the same cubic
                # pieces, different rounding (largest where r' < the grid start
                # and the first piece is extended)
                want = 0.5 * beta * (V(q + 0.5 * za) + V(q - 0.5 * za))
                tol = 1e-10
                checked_prim += 1
            got = pa.U(q, z, s * s, level)
            assert abs(got - want) <= tol * max(1.0, abs(want)), (level, q, z, s, got, want)
        assert checked_fit > 50 and checked_prim > 20
        # q = 0: the fit's test z < zmax = 2q fails first, so the reference's
        # q == 0 branch inside it is never taken and U is the primitive
        want0 = 0.5 * beta * 2.0 * V(0.0)
        assert abs(pa.U(0.0, 0.0, 0.0, level) - want0) <= 1e-8 * abs(want0)

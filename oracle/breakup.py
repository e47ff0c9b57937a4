"""Test infrastructure only: a numpy / SciPy restatement of the optimized
Ewald breakup of a classical Coulomb pair action, used to check the library's
host breakup.  Nothing in the library imports this module.

Follows:
* LongRangeClass::OptimizedBreakup_U / _dU  (PIMC++/src/Actions/LongRangeClass.cc:509-868)
* OptimizedBreakupClass::SetkVecs / DoBreakup (Common/Ewald/OptimizedBreakup.cc:45-283)
* LPQHI_BasisClass::h / c                     (Common/Ewald/OptimizedBreakup.cc:330-420,
                                               OptimizedBreakup.h:94-255)
* PAclassicalFitClass::Xk_U / Xk_dU / Udiag   (Common/PairAction/PAclassicalFit.cc:175-288)
* QuinticSpline (natural quintic interpolant) (Common/Splines/QuinticSpline.h:127-221)

The reference solves DoBreakup's least-squares problem through the SVD of
its normal equations, whose condition number (~1e15 for jellium with 49
knots) leaves the smallest singular values at rounding level; here numpy's
lstsq solves the same problem on the weighted design matrix, and SciPy's
B-spline interpolation with zero third and fourth end derivatives stands in
for the QUINAT routine (parity by tolerance).
The k = 0 integrals use scipy.integrate.quad where the reference uses its
adaptive Gauss-Kronrod code.
"""
import math

import numpy as np
from scipy.integrate import quad
from scipy.interpolate import PPoly, make_interp_spline

S = np.array([[1.0, 0.0, 0.0, -10.0, 15.0, -6.0],
              [0.0, 1.0, 0.0, -6.0, 8.0, -3.0],
              [0.0, 0.0, 0.5, -1.5, 1.5, -0.5]])


class Lpqhi:
    """Locally piecewise quintic Hermite basis on knots r_i = i delta, i < NumKnots."""

    def __init__(self, rc, num_knots, box):
        self.rc, self.knots = rc, num_knots
        self.delta = rc / (num_knots - 1)
        self.omega = float(np.prod(box))

    def h(self, n, r):
        r = np.asarray(r, dtype=float)
        i, alpha = divmod(n, 3)
        ra, rb, rc = self.delta * (i - 1), self.delta * i, min(self.rc, self.delta * (i + 1))
        out = np.zeros_like(r)
        left = (r > ra) & (r <= rb)
        right = (r > rb) & (r <= rc)
        ul = (rb - r[left]) / self.delta
        ur = (r[right] - rb) / self.delta
        out[left] = (-1.0) ** alpha * sum(S[alpha, j] * ul ** j for j in range(6))
        out[right] = sum(S[alpha, j] * ur ** j for j in range(6))
        return out

    def c(self, k):
        """c_n(k) = 4 pi/(k Omega) int_0^rc h_n(r) r sin(kr) dr for all n, vectorised over k.

        Per knot interval the moments M_j = int u^j r sin(kr) dr come from the
        integration-by-parts recursion of int u^j e^{ikr} dr."""
        k = np.asarray(k, dtype=float)
        d = self.delta
        pre = 4.0 * np.pi / (k * self.omega)
        out = np.zeros((3 * self.knots,) + k.shape)

        def moments(a, b, origin, sgn):
            # int_a^b u^j e^{ikr} dr with u = sgn (r - origin)/d, u = 0 at origin, u = 1 at the far end
            far = b if sgn > 0 else a
            E = [None] * 7
            E[0] = (np.exp(1j * k * b) - np.exp(1j * k * a)) / (1j * k)
            for j in range(1, 7):
                # by parts: [u^j e^{ikr}/(ik)] - (sgn j/d) int u^{j-1} e^{ikr}/(ik)
                bound = np.exp(1j * k * far) * (1.0 if sgn > 0 else -1.0)
                E[j] = (bound - sgn * j / d * E[j - 1]) / (1j * k)
            return E

        for i in range(self.knots):
            r0 = d * i
            for side in (+1, -1):
                if side > 0 and i == self.knots - 1:
                    continue
                if side < 0 and i == 0:
                    continue
                if side > 0:
                    E = moments(r0, r0 + d, r0, +1)
                else:
                    E = moments(r0 - d, r0, r0, -1)
                # r = r0 + side d u
                M = [pre * (r0 * E[j].imag + side * d * E[j + 1].imag) for j in range(6)]
                for alpha in range(3):
                    sign = 1.0 if side > 0 else (-1.0) ** alpha
                    out[3 * i + alpha] += sign * sum(S[alpha, j] * M[j] for j in range(6))
        return out


def kpoints(box, kc, kcont, kmax):
    """OptimizedBreakupClass::SetkVecs: lattice |k| shells in (kc, kcont) with their
    multiplicities, then 4000 spherical-shell bins to kmax."""
    b = 2.0 * np.pi / np.asarray(box, dtype=float)
    m = np.ceil(kcont / b).astype(int)
    ix = np.arange(-m[0], m[0] + 1) * b[0]
    iy = np.arange(-m[1], m[1] + 1) * b[1]
    iz = np.arange(-m[2], m[2] + 1) * b[2]
    k2 = ix[:, None, None] ** 2 + iy[None, :, None] ** 2 + iz[None, None, :] ** 2
    k2 = k2[(k2 > kc * kc) & (k2 < kcont * kcont)]
    kk = np.sort(np.sqrt(k2))
    brk = np.concatenate([[True], np.diff(kk) > 1e-12])
    starts = np.flatnonzero(brk)
    shells = kk[starts]
    deg = np.diff(np.concatenate([starts, [len(kk)]])).astype(float)
    n = 4000
    dk = (kmax - kcont) / n
    k1 = kcont + dk * np.arange(n)
    k2b = k1 + dk
    cont = 0.5 * (k1 + k2b)
    wcont = 4.0 * np.pi / 3.0 * (k2b ** 3 - k1 ** 3) / np.prod(b)
    return np.concatenate([shells, cont]), np.concatenate([deg, wcont])


def quintic_coefficients(r, y):
    """Taylor coefficients {y, y', y''/2, y'''/6, y''''/24, y'''''/120} of each interval."""
    bs = make_interp_spline(r, y, k=5, bc_type=([(3, 0.0), (4, 0.0)], [(3, 0.0), (4, 0.0)]))
    pp = PPoly.from_spline(bs)
    idx = np.clip(np.searchsorted(pp.x, r[:-1], side="right") - 1, 0, pp.c.shape[1] - 1)
    c = pp.c[::-1, idx].T  # lowest power first
    return np.vstack([c, c[-1:]]), bs


def normal_equation_svd(cnk, w, xk, tolerance=1.0e-16):
    """OptimizedBreakupClass::DoBreakup (Common/Ewald/OptimizedBreakup.cc:196-290)
    with every coefficient adjustable, as LongRangeClass calls it
    (LongRangeClass.cc:601,611): A = sum_k w c c^T, b = sum_k w X_k c, the SVD
    A = U S V^T, singular values below tolerance * S_max dropped, and
    t = sum_i (U_i . b) / S_i V_i."""
    A = (cnk * w) @ cnk.T
    b = (cnk * w) @ xk
    U, S, Vt = np.linalg.svd(A)
    smax = S.max()
    sinv = np.where(S < tolerance * smax, 0.0, 1.0 / np.where(S > 0, S, 1.0))
    return Vt.T @ (sinv * (U.T @ b)), int(np.sum(sinv == 0.0))


def coulomb_breakup(box, z1z2, smallest_beta, num_levels, num_knots, kcut, kvecs, solve="lstsq"):
    """The breakup tables.  solve: "lstsq" (the weighted design matrix, the
    library's approach) or "normal_svd" (the reference's own procedure,
    normal_equation_svd)."""
    box = np.asarray(box, dtype=float)
    omega = float(np.prod(box))
    rc = 0.5 * box.min()
    # pow() of the k-cell volume as LongRangeClass computes it (C pow; numpy's
    # power can differ in the last bit, and a cubic box has a shell exactly
    # at kcont = 50 kavg)
    kvol = float(2.0 * np.pi / box[0]) * float(2.0 * np.pi / box[1]) * float(2.0 * np.pi / box[2])
    kavg = math.pow(kvol, 1.0 / 3.0)
    basis = Lpqhi(rc, num_knots, box)
    kcont, kmax = 50.0 * kavg, 20.0 * np.pi / basis.delta
    kp, w = kpoints(box, kcut, kcont, kmax)
    cnk = basis.c(kp)
    sw = np.sqrt(w)
    Dw = cnk.T * sw[:, None]
    kv = np.asarray(kvecs, dtype=float).reshape(-1, 3)
    kmag = np.sqrt((kv ** 2).sum(1))
    csim = basis.c(kmag)
    rmax = 0.75 * np.sqrt((box ** 2).sum())
    rgrid = 0.0 + np.arange(1000) * (rmax / 999)
    out = {"rmax": rmax, "rc": rc, "kpoints": len(kp)}
    h0 = np.array([basis.h(n, np.array([0.0]))[0] for n in range(3 * num_knots)])
    hr = np.array([basis.h(n, rgrid) for n in range(3 * num_knots)])
    for job, tag in ((0, ""), (1, "d")):
        uk = np.zeros((num_levels, len(kmag)))
        r0, sk0, lk0, ur_all = [], [], [], []
        for level in range(num_levels):
            beta = smallest_beta * 2.0 ** level
            coef = 1.0 if job else beta
            xk = -4.0 * np.pi * coef * z1z2 / kp ** 2 * np.cos(kp * rc) / omega
            # the least-squares problem of DoBreakup, on the weighted design matrix
            if solve == "normal_svd":
                t, nsing = normal_equation_svd(cnk, w, xk)
                out.setdefault("singular_dropped", []).append(nsing)
            else:
                t = np.linalg.lstsq(Dw, sw * xk, rcond=1e-8)[0]
            r0.append(float(t @ h0))
            ur = np.where(rgrid <= rc, t @ hr, coef * z1z2 / np.where(rgrid > 0, rgrid, 1.0))
            cq, bs = quintic_coefficients(rgrid, ur)
            ur_all.append(cq)
            if job == 0:
                sk0.append(4 * np.pi / omega * quad(lambda r: r * r * (coef * z1z2 / r - bs(r)), 0.0, rc,
                                                    limit=400, epsrel=1e-11, epsabs=0)[0])
            else:
                sk0.append(4 * np.pi / omega * quad(lambda r: r * r * (z1z2 / r - bs(r)), 0.0, rmax,
                                                    limit=800, epsrel=1e-11, epsabs=0)[0])
            lk0.append(4 * np.pi / omega * quad(lambda r: r * r * bs(r), 0.0, rmax, limit=800, epsrel=1e-11,
                                                epsabs=0)[0])
            uk[level] = t @ csim + 4.0 * np.pi * coef * z1z2 / kmag ** 2 * np.cos(kmag * rc) / omega
        out[tag + "ulong_k"] = uk
        out[tag + "ulong_r0"] = np.array(r0)
        out[("dushort_k0" if job else "ushort_k0")] = np.array(sk0)
        out[tag + "ulong_k0"] = np.array(lk0)
        out[tag + "ulong_r"] = np.array(ur_all)
    return out, basis

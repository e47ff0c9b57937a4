// Optimized Ewald breakup of a classical Coulomb pair action, host side, FP64:
// LongRangeClass::OptimizedBreakup_U / _dU (PIMC++/src/Actions/LongRangeClass.cc:509-868)
// with OptimizedBreakupClass and LPQHI_BasisClass (Common/Ewald/OptimizedBreakup.cc,
// .h:94-255), PAclassicalFitClass::Xk_U / Xk_dU / Udiag (Common/PairAction/PAclassicalFit.cc:
// 175-288) and the natural quintic spline of Ulong(r) (Common/Splines/QuinticSpline.h).
//
// The long-range part is expanded in locally piecewise quintic Hermite basis
// functions h_n(r) on NumKnots knots over [0, r_c]; the coefficients t_n
// minimise sum_k w_k (X_k - sum_n t_n c_n(k))^2 over |k| shells beyond the
// simulation cutoff plus 4000 continuum bins, where c_n(k) is the 3-D Fourier
// transform of h_n and X_k that of the pair action beyond r_c.  Singular
// values below 1e-16 of the largest are dropped.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "pimc_internal.h"

namespace pimc {

namespace {

typedef std::complex<double> cplx;

// LPQHI_BasisClass: three quintic Hermite functions per knot (value, slope,
// curvature), supported on the two intervals around the knot.
struct Lpqhi {
  int knots = 0;
  double rc = 0, delta = 0, deltainv = 0, omega = 0;
  // Hermite basis polynomials in u = |r - r_knot| / delta, powers 0..5
  static constexpr double S[3][6] = {{1.0, 0.0, 0.0, -10.0, 15.0, -6.0},
                                     {0.0, 1.0, 0.0, -6.0, 8.0, -3.0},
                                     {0.0, 0.0, 0.5, -1.5, 1.5, -0.5}};
  int size() const { return 3 * knots; }

  double h(int n, double r) const {
    const int i = n / 3, alpha = n - 3 * i;
    const double ra = delta * (i - 1), rb = delta * i;
    const double rcut = std::min(rc, delta * (i + 1));
    double u, sign;
    if (r > ra && r <= rb) {
      u = (rb - r) * deltainv;
      sign = (alpha & 1) ? -1.0 : 1.0;  // odd derivatives change sign to the left
    } else if (r > rb && r <= rcut) {
      u = (r - rb) * deltainv;
      sign = 1.0;
    } else {
      return 0.0;
    }
    double sum = 0.0, p = 1.0;
    for (int j = 0; j <= 5; j++) {
      sum += S[alpha][j] * p;
      p *= u;
    }
    return sign * sum;
  }

  // E^+_n(i, k) = int_{r_i}^{r_{i+1}} u^n e^{ikr} dr, u = (r - r_i)/delta, and
  // K_n(i, k) = int_{r_{i-1}}^{r_i} u^n e^{ikr} dr, u = (r_i - r)/delta, by
  // integration by parts (n = 0..6), and their k-derivatives:
  //   E^+_n = -(i/k) [e^{ik r_{i+1}} - (n/delta) E^+_{n-1}],
  //   K_n   =  (i/k) [e^{ik r_{i-1}} - (n/delta) K_{n-1}].
  void edges(int i, double k, cplx Ep[7], cplx Em[7], cplx dEp[7], cplx dEm[7]) const {
    const cplx I(0.0, 1.0);
    auto ex = [&](double r) { return cplx(std::cos(k * r), std::sin(k * r)); };
    auto dex = [&](double r) { return cplx(-r * std::sin(k * r), r * std::cos(k * r)); };
    const double r0 = delta * i, rp = delta * (i + 1), rm = delta * (i - 1);
    // n = 0
    Ep[0] = -(I / k) * (ex(rp) - ex(r0));
    dEp[0] = (I / (k * k)) * (ex(rp) - ex(r0)) - (I / k) * (dex(rp) - dex(r0));
    Em[0] = -(I / k) * (ex(r0) - ex(rm));
    dEm[0] = (I / (k * k)) * (ex(r0) - ex(rm)) - (I / k) * (dex(r0) - dex(rm));
    for (int n = 1; n <= 6; n++) {
      const double f = (double)n / delta;
      // + side: boundary term u^n e^{ikr} is 1 at r_{i+1} and 0 at r_i
      const cplx tp = ex(rp) - f * Ep[n - 1];
      const cplx dtp = dex(rp) - f * dEp[n - 1];
      Ep[n] = -(I / k) * tp;
      dEp[n] = (I / (k * k)) * tp - (I / k) * dtp;
      // - side: u = 1 at r_{i-1}, 0 at r_i
      const cplx tm = ex(rm) - f * Em[n - 1];
      const cplx dtm = dex(rm) - f * dEm[n - 1];
      Em[n] = (I / k) * tm;
      dEm[n] = -(I / (k * k)) * tm + (I / k) * dtm;
    }
  }

  // c_n(k) = 4 pi / (k Omega) int_0^rc h_n(r) r sin(kr) dr and dc_n/dk.
  void c_all(double k, double *c, double *dc) const {
    cplx Ep[7], Em[7], dEp[7], dEm[7];
    const double pre = 4.0 * M_PI / (k * omega), dpre = -4.0 * M_PI / (k * k * omega);
    for (int i = 0; i < knots; i++) {
      edges(i, k, Ep, Em, dEp, dEm);
      // int u^n r sin(kr) dr with r = delta (i + u) on the right interval and
      // r = delta (i - u) on the left one, times 4 pi / (k Omega)
      double Dp[6], Dm[6], dDp[6], dDm[6];
      for (int n = 0; n <= 5; n++) {
        const double ip = delta * Ep[n + 1].imag() + i * delta * Ep[n].imag();
        const double dip = delta * dEp[n + 1].imag() + i * delta * dEp[n].imag();
        Dp[n] = pre * ip;
        dDp[n] = dpre * ip + pre * dip;
        const double im = i * delta * Em[n].imag() - delta * Em[n + 1].imag();
        const double dim = i * delta * dEm[n].imag() - delta * dEm[n + 1].imag();
        Dm[n] = pre * im;
        dDm[n] = dpre * im + pre * dim;
      }
      for (int alpha = 0; alpha < 3; alpha++) {
        // h is sum_j S_j u^j on the right interval and (-1)^alpha sum_j S_j u^j
        // on the left one (odd derivatives change sign in the mirror)
        const double mirror = (alpha & 1) ? -1.0 : 1.0;
        double s = 0.0, ds = 0.0;
        for (int n = 0; n <= 5; n++) {
          double v = 0.0, dv = 0.0;
          if (i < knots - 1) {
            v += Dp[n];
            dv += dDp[n];
          }
          if (i > 0) {
            v += mirror * Dm[n];
            dv += mirror * dDm[n];
          }
          s += S[alpha][n] * v;
          ds += S[alpha][n] * dv;
        }
        c[3 * i + alpha] = s;
        if (dc) dc[3 * i + alpha] = ds;
      }
    }
  }
};
constexpr double Lpqhi::S[3][6];

// |k| shells of the reciprocal lattice with kc < |k| < kcont and their
// multiplicities, then 4000 bins from kcont to kmax weighted by the number of
// lattice points their spherical shell holds (OptimizedBreakupClass::SetkVecs).
void breakup_kpoints(const double box[3], double kc, double kcont, double kmax, std::vector<double> &kp,
                     std::vector<double> &w) {
  double b[3];
  int m[3];
  for (int d = 0; d < 3; d++) {
    b[d] = 2.0 * M_PI / box[d];
    m[d] = (int)std::ceil(kcont / b[d]);
  }
  std::vector<double> ks;
  for (int ix = -m[0]; ix <= m[0]; ix++)
    for (int iy = -m[1]; iy <= m[1]; iy++)
      for (int iz = -m[2]; iz <= m[2]; iz++) {
        const double kx = ix * b[0], ky = iy * b[1], kz = iz * b[2];
        const double k2 = kx * kx + ky * ky + kz * kz;
        if (k2 > kc * kc && k2 < kcont * kcont) ks.push_back(std::sqrt(k2));
      }
  std::sort(ks.begin(), ks.end());
  kp.clear();
  w.clear();
  for (double k : ks) {
    if (!kp.empty() && std::fabs(k - kp.back()) <= 1.0e-12) {
      w.back() += 1.0;
    } else {
      kp.push_back(k);
      w.push_back(1.0);
    }
  }
  const double kvol = b[0] * b[1] * b[2];
  const int nb = 4000;
  const double dk = (kmax - kcont) / nb;
  for (int i = 0; i < nb; i++) {
    const double k1 = kcont + dk * i, k2 = k1 + dk;
    kp.push_back(0.5 * (k1 + k2));
    w.push_back(4.0 * M_PI / 3.0 * (k2 * k2 * k2 - k1 * k1 * k1) / kvol);
  }
}

// One-sided Jacobi (Hestenes) SVD of a square matrix held by columns:
// cols[j][0..n) are rotated until mutually orthogonal; on return their norms
// are the singular values, cols[j] / sigma_j the left vectors and V (row-major
// n x n, columns) the right vectors.
void hestenes_svd(int n, std::vector<std::vector<double>> &cols, std::vector<double> &V, std::vector<double> &sigma) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) V[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 60; sweep++) {
    bool rotated = false;
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        double alpha = 0.0, beta = 0.0, gamma = 0.0;
        const std::vector<double> &ap = cols[p], &aq = cols[q];
        for (int k = 0; k < n; k++) {
          alpha += ap[k] * ap[k];
          beta += aq[k] * aq[k];
          gamma += ap[k] * aq[k];
        }
        if (gamma == 0.0 || std::fabs(gamma) <= 1e-15 * std::sqrt(alpha * beta)) continue;
        rotated = true;
        const double zeta = (beta - alpha) / (2.0 * gamma);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
        for (int k = 0; k < n; k++) {
          const double x = cols[p][k], y = cols[q][k];
          cols[p][k] = c * x - s * y;
          cols[q][k] = s * x + c * y;
        }
        for (int k = 0; k < n; k++) {
          const double x = V[(size_t)k * n + p], y = V[(size_t)k * n + q];
          V[(size_t)k * n + p] = c * x - s * y;
          V[(size_t)k * n + q] = s * x + c * y;
        }
      }
    if (!rotated) break;
  }
  sigma.assign(n, 0.0);
  for (int j = 0; j < n; j++) {
    double s2 = 0.0;
    for (int k = 0; k < n; k++) s2 += cols[j][k] * cols[j][k];
    sigma[j] = std::sqrt(s2);
  }
}

// OptimizedBreakupClass::DoBreakup with every coefficient adjusted: t
// minimises sum_k w_k (X_k - sum_n t_n c_n(k))^2.  The reference forms the
// normal equations A = sum_k w c c^T and inverts them by SVD, dropping
// singular values below 1e-16 of the largest; A's condition number (~1e15 for
// jellium with 49 knots) puts its smallest singular values at rounding level,
// so that solution moves with the rounding.  Here the same least-squares
// problem is solved on the weighted design matrix D = diag(sqrt w) C^T
// (condition number the square root of A's): Householder QR, D = Q R, then a
// one-sided Jacobi SVD of R, dropping singular values of D below 1e-8 of the
// largest (the reference's 1e-16 on A = D^T D).
void do_breakup(const std::vector<double> &cnk, const std::vector<double> &w, const std::vector<double> &xk, int nb,
                std::vector<double> &t) {
  const int nk = (int)w.size();
  // D by columns, y = sqrt(w) X
  std::vector<std::vector<double>> D(nb, std::vector<double>(nk));
  std::vector<double> y(nk);
  for (int ki = 0; ki < nk; ki++) {
    const double sw = std::sqrt(w[ki]);
    y[ki] = sw * xk[ki];
    for (int n = 0; n < nb; n++) D[n][ki] = sw * cnk[(size_t)n * nk + ki];
  }
  // Householder QR: D <- R in its upper nb x nb block, y <- Q^T y
  for (int j = 0; j < nb; j++) {
    double norm = 0.0;
    for (int i = j; i < nk; i++) norm += D[j][i] * D[j][i];
    norm = std::sqrt(norm);
    if (norm == 0.0) continue;
    const double alpha = D[j][j] > 0 ? -norm : norm;
    std::vector<double> v(D[j].begin() + j, D[j].end());
    v[0] -= alpha;
    double vv = 0.0;
    for (double x : v) vv += x * x;
    if (vv == 0.0) continue;
    for (int c = j; c < nb; c++) {
      double dot = 0.0;
      for (int i = j; i < nk; i++) dot += v[i - j] * D[c][i];
      const double f = 2.0 * dot / vv;
      for (int i = j; i < nk; i++) D[c][i] -= f * v[i - j];
    }
    double dot = 0.0;
    for (int i = j; i < nk; i++) dot += v[i - j] * y[i];
    const double f = 2.0 * dot / vv;
    for (int i = j; i < nk; i++) y[i] -= f * v[i - j];
  }
  std::vector<std::vector<double>> R(nb, std::vector<double>(nb, 0.0));
  for (int c = 0; c < nb; c++)
    for (int r = 0; r <= c; r++) R[c][r] = D[c][r];
  std::vector<double> V, sigma;
  hestenes_svd(nb, R, V, sigma);
  double smax = 0.0;
  for (double sg : sigma) smax = std::max(smax, sg);
  t.assign(nb, 0.0);
  for (int j = 0; j < nb; j++) {
    if (sigma[j] < 1.0e-8 * smax || sigma[j] == 0.0) continue;
    double coef = 0.0;  // u_j . (Q^T y)[0..nb) / sigma_j^2 (R's column j is sigma_j u_j)
    for (int k = 0; k < nb; k++) coef += R[j][k] * y[k];
    coef /= sigma[j] * sigma[j];
    for (int k = 0; k < nb; k++) t[k] += coef * V[(size_t)k * nb + j];
  }
}

// Banded LU with partial pivoting (kl sub-, ku super-diagonals), solving in
// place; ab holds row r's entries for columns r-kl .. r+ku+kl (width
// 2 kl + ku + 1, offset kl).
bool band_solve(int n, int kl, int ku, std::vector<double> &ab, std::vector<double> &x) {
  const int W = 2 * kl + ku + 1;
  auto at = [&](int r, int c) -> double & { return ab[(size_t)r * W + (c - r + kl)]; };
  for (int k = 0; k < n; k++) {
    int piv = k;
    double best = std::fabs(at(k, k));
    for (int r = k + 1; r <= std::min(n - 1, k + kl); r++)
      if (std::fabs(at(r, k)) > best) {
        best = std::fabs(at(r, k));
        piv = r;
      }
    if (best == 0.0) return false;
    const int cmax = std::min(n - 1, k + ku + kl);
    if (piv != k) {
      for (int c = k; c <= cmax; c++) std::swap(at(k, c), at(piv, c));
      std::swap(x[k], x[piv]);
    }
    for (int r = k + 1; r <= std::min(n - 1, k + kl); r++) {
      const double f = at(r, k) / at(k, k);
      if (f == 0.0) continue;
      for (int c = k; c <= cmax; c++) at(r, c) -= f * at(k, c);
      x[r] -= f * x[k];
    }
  }
  for (int k = n - 1; k >= 0; k--) {
    double s = x[k];
    for (int c = k + 1; c <= std::min(n - 1, k + ku + kl); c++) s -= at(k, c) * x[c];
    x[k] = s / at(k, k);
  }
  return true;
}

}  // namespace

// Natural quintic interpolating spline (third and fourth derivatives zero at
// both ends, C4 inside) of y on the uniform grid start + i h, as the Taylor
// coefficients {y, y', y''/2, y'''/6, y''''/24, y'''''/120} of each interval
// at its left knot: coef[i][6], i = 0..n-2 (row n-1 repeats the last
// interval's so that an index clamped to n-2 is never needed).  Solved for
// the knot values sigma_i = S''(x_i), tau_i = S''''(x_i): S'''' is linear and
// S'' a cubic spline in each interval, and the continuity of S' and S''' at
// the interior knots gives
//   h^2/6 (s_{i-1} + 4 s_i + s_{i+1}) - h^4/360 (7 t_{i-1} + 16 t_i + 7 t_{i+1}) = y_{i+1} - 2 y_i + y_{i-1}
//   s_{i+1} - 2 s_i + s_{i-1} = h^2/6 (t_{i-1} + 4 t_i + t_{i+1}).
bool quintic_natural(int n, double h, const double *y, double *coef) {
  if (n < 3) return false;
  const int N = 2 * n, kl = 3, ku = 3, W = 2 * kl + ku + 1;
  std::vector<double> ab((size_t)N * W, 0.0), x(N, 0.0);
  auto set = [&](int r, int c, double v) { ab[(size_t)r * W + (c - r + kl)] += v; };
  const double h2 = h * h / 6.0, h4 = h * h * h * h / 6.0;
  int r = 0;
  set(r, 1, 1.0);  // tau_0 = 0
  r++;
  set(r, 2, 1.0);  // S'''(x_0) = 0
  set(r, 0, -1.0);
  set(r, 3, -h2);
  r++;
  for (int i = 1; i < n - 1; i++) {
    set(r, 2 * (i - 1), h2);
    set(r, 2 * i, 4.0 * h2);
    set(r, 2 * (i + 1), h2);
    set(r, 2 * (i - 1) + 1, -h4 * 7.0 / 60.0);
    set(r, 2 * i + 1, -h4 * 16.0 / 60.0);
    set(r, 2 * (i + 1) + 1, -h4 * 7.0 / 60.0);
    x[r] = (y[i + 1] - y[i]) - (y[i] - y[i - 1]);
    r++;
    set(r, 2 * (i + 1), 1.0);
    set(r, 2 * i, -2.0);
    set(r, 2 * (i - 1), 1.0);
    set(r, 2 * (i - 1) + 1, -h2);
    set(r, 2 * i + 1, -4.0 * h2);
    set(r, 2 * (i + 1) + 1, -h2);
    r++;
  }
  set(r, 2 * (n - 1) + 1, 1.0);  // tau_{n-1} = 0
  r++;
  set(r, 2 * (n - 1), 1.0);  // S'''(x_{n-1}) = 0
  set(r, 2 * (n - 2), -1.0);
  set(r, 2 * (n - 2) + 1, h2);
  if (!band_solve(N, kl, ku, ab, x)) return false;
  for (int i = 0; i < n - 1; i++) {
    const double s0 = x[2 * i], t0 = x[2 * i + 1], s1 = x[2 * i + 2], t1 = x[2 * i + 3];
    double *c = coef + (size_t)i * 6;
    c[0] = y[i];
    c[1] = ((y[i + 1] - y[i]) - h2 * (2.0 * s0 + s1) + h4 * (2.0 / 15.0 * t0 + 7.0 / 60.0 * t1)) / h;
    c[2] = 0.5 * s0;
    c[3] = (s1 - s0 - h2 * (2.0 * t0 + t1)) / (6.0 * h);
    c[4] = t0 / 24.0;
    c[5] = (t1 - t0) / (120.0 * h);
  }
  std::memcpy(coef + (size_t)(n - 1) * 6, coef + (size_t)(n - 2) * 6, 6 * sizeof(double));
  return true;
}

// QuinticSpline::operator() (QuinticSpline.h:204-221): interval from the
// linear grid's ReverseMap clamped to [0, n-2], Horner in P = x - x_I.
double quintic_eval(int n, double start, double h, const double *coef, double x) {
  int j = (int)std::nearbyint((x - start) * (1.0 / h) - 0.5) + 1;
  int i = j - 1;
  if (i < 0) i = 0;
  if (i > n - 2) i = n - 2;
  const double *c = coef + (size_t)i * 6;
  const double P = x - (start + (double)i * h);
  return ((((c[5] * P + c[4]) * P + c[3]) * P + c[2]) * P + c[1]) * P + c[0];
}

namespace {

// Adaptive Gauss-Kronrod (7-point Gauss / 15-point Kronrod) integration to a
// relative tolerance.
template <typename F>
double gk15(const F &f, double a, double b, double *err) {
  static const double xk[8] = {0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
                               0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
                               0.586087235467691130294144845693013, 0.405845151377397166906606412076961,
                               0.207784955007898467600689403773245, 0.000000000000000000000000000000000};
  static const double wk[8] = {0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
                               0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
                               0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
                               0.204432940075298892414161999234649, 0.209482141084727828012999174891714};
  static const double wg[4] = {0.129484966168869693270611432679082, 0.279705391489276667901467771423780,
                               0.381830050505118944950369775488975, 0.417959183673469387755102040816327};
  const double c = 0.5 * (a + b), hl = 0.5 * (b - a);
  const double fc = f(c);
  double rk = fc * wk[7], rg = fc * wg[3];
  for (int j = 0; j < 7; j++) {
    const double x = hl * xk[j];
    const double f1 = f(c - x), f2 = f(c + x);
    rk += wk[j] * (f1 + f2);
    if (j & 1) rg += wg[j / 2] * (f1 + f2);
  }
  *err = std::fabs((rk - rg) * hl);
  return rk * hl;
}
template <typename F>
double integrate(const F &f, double a, double b, double reltol) {
  struct Piece {
    double a, b, v, e;
  };
  std::vector<Piece> pieces;
  for (int i = 0; i < 64; i++) {  // start from 64 panels: the integrands have spline kinks
    const double x0 = a + (b - a) * i / 64.0, x1 = a + (b - a) * (i + 1) / 64.0;
    double e;
    const double v = gk15(f, x0, x1, &e);
    pieces.push_back({x0, x1, v, e});
  }
  for (int it = 0; it < 20000; it++) {
    double tot = 0.0, terr = 0.0;
    size_t worst = 0;
    for (size_t i = 0; i < pieces.size(); i++) {
      tot += pieces[i].v;
      terr += pieces[i].e;
      if (pieces[i].e > pieces[worst].e) worst = i;
    }
    if (terr <= reltol * std::fabs(tot) || terr < 1e-300) return tot;
    Piece p = pieces[worst];
    const double m = 0.5 * (p.a + p.b);
    double e1, e2;
    const double v1 = gk15(f, p.a, m, &e1), v2 = gk15(f, m, p.b, &e2);
    pieces[worst] = {p.a, m, v1, e1};
    pieces.push_back({m, p.b, v2, e2});
  }
  double tot = 0.0;
  for (const Piece &p : pieces) tot += p.v;
  return tot;
}

}  // namespace

int coulomb_breakup(const double box[3], double z1z2, double smallest_beta, int num_levels, int num_knots, double kcut,
                    int num_k, const double *kvecs, BreakupTables &out) {
  if (num_levels < 1 || num_knots < 2 || !(kcut > 0.0)) return PIMC_E_ARG;
  const double omega = box[0] * box[1] * box[2];
  double rc = 0.5 * box[0];
  for (int d = 1; d < 3; d++) rc = std::min(rc, 0.5 * box[d]);
  double kvol = 1.0;
  for (int d = 0; d < 3; d++) kvol *= 2.0 * M_PI / box[d];
  const double kavg = std::pow(kvol, 1.0 / 3.0);
  Lpqhi basis;
  basis.knots = num_knots;
  basis.rc = rc;
  basis.delta = rc / (num_knots - 1);
  basis.deltainv = 1.0 / basis.delta;
  basis.omega = omega;
  const double kcont = 50.0 * kavg, kmax = 20.0 * M_PI / basis.delta;
  std::vector<double> kp, w;
  breakup_kpoints(box, kcut, kcont, kmax, kp, w);
  const int nk = (int)kp.size(), nb = basis.size();
  std::vector<double> cnk((size_t)nb * nk), cbuf(nb);
  for (int ki = 0; ki < nk; ki++) {
    basis.c_all(kp[ki], cbuf.data(), nullptr);
    for (int n = 0; n < nb; n++) cnk[(size_t)n * nk + ki] = cbuf[n];
  }
  // c_n(k) and dc_n/dk at the simulation k-vectors
  std::vector<double> csim((size_t)num_k * nb), kmag(num_k);
  for (int ki = 0; ki < num_k; ki++) {
    const double *kv = kvecs + 3 * ki;
    kmag[ki] = std::sqrt(kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2]);
    basis.c_all(kmag[ki], csim.data() + (size_t)ki * nb, nullptr);
  }
  const int np = kLongGridPoints;
  const double rmax = 0.75 * std::sqrt(box[0] * box[0] + box[1] * box[1] + box[2] * box[2]);
  const double hgrid = rmax / (np - 1);
  out.rc = rc;
  out.rmax = rmax;
  out.levels = num_levels;
  out.num_k = num_k;
  out.knots_delta = basis.delta;
  out.kpoints = nk;
  for (int job = 0; job < 2; job++) {  // 0: U (OptimizedBreakup_U), 1: dU (OptimizedBreakup_dU)
    std::vector<double> &uk = job ? out.dulong_k : out.ulong_k;
    std::vector<double> &r0 = job ? out.dulong_r0 : out.ulong_r0;
    std::vector<double> &sk0 = job ? out.dushort_k0 : out.ushort_k0;
    std::vector<double> &lk0 = job ? out.dulong_k0 : out.ulong_k0;
    std::vector<double> &spl = job ? out.dulong_r : out.ulong_r;
    uk.assign((size_t)num_levels * num_k, 0.0);
    r0.assign(num_levels, 0.0);
    sk0.assign(num_levels, 0.0);
    lk0.assign(num_levels, 0.0);
    spl.assign((size_t)num_levels * np * 6, 0.0);
    for (int level = 0; level < num_levels; level++) {
      double beta = smallest_beta;
      for (int i = 0; i < level; i++) beta *= 2.0;
      const double coef = job ? 1.0 : beta;
      // Xk_U / Xk_dU (PAclassicalFit.cc:248-288) divided by the volume
      std::vector<double> xk(nk);
      for (int ki = 0; ki < nk; ki++)
        xk[ki] = -4.0 * M_PI * coef * z1z2 / (kp[ki] * kp[ki]) * std::cos(kp[ki] * rc) / omega;
      std::vector<double> t;
      do_breakup(cnk, w, xk, nb, t);
      double s0 = 0.0;
      for (int n = 0; n < nb; n++) s0 += t[n] * basis.h(n, 0.0);
      r0[level] = s0;
      // Ulong(r) on the 1000-point grid: the basis sum to rc, Udiag beyond
      std::vector<double> ur(np, 0.0);
      for (int i = 0; i < np; i++) {
        const double r = hgrid * i;
        if (r <= rc) {
          double s = 0.0;
          for (int n = 0; n < nb; n++) s += t[n] * basis.h(n, r);
          ur[i] = s;
        } else {
          ur[i] = coef * z1z2 / r;
        }
      }
      double *sc = spl.data() + (size_t)level * np * 6;
      if (!quintic_natural(np, hgrid, ur.data(), sc)) return PIMC_E_ARG;
      auto ulong = [&](double r) { return quintic_eval(np, 0.0, hgrid, sc, r); };
      // k = 0 parts: 4 pi / Omega int r^2 (...) dr
      if (job == 0) {
        sk0[level] = 4.0 * M_PI / omega *
                     integrate([&](double r) { return r * r * (coef * z1z2 / r - ulong(r)); }, 0.0, rc, 1e-10);
      } else {
        sk0[level] = 4.0 * M_PI / omega *
                     integrate([&](double r) { return r * r * (z1z2 / r - ulong(r)); }, 0.0, rmax, 1e-10);
      }
      lk0[level] = 4.0 * M_PI / omega * integrate([&](double r) { return r * r * ulong(r); }, 0.0, rmax, 1e-10);
      for (int ki = 0; ki < num_k; ki++) {
        double s = 0.0;
        for (int n = 0; n < nb; n++) s += t[n] * csim[(size_t)ki * nb + n];
        const double k = kmag[ki];
        s -= -4.0 * M_PI * coef * z1z2 / (k * k) * std::cos(k * rc) / omega;
        uk[(size_t)level * num_k + ki] = s;
      }
    }
  }
  return PIMC_OK;
}

}  // namespace pimc

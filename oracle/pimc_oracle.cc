// ORACLE — TEST INFRASTRUCTURE ONLY (see pimc_oracle.h).
//
// FP64 CPU restatement of the PIMC++ hot path.  Each piece cites the
// reference file:line it restates (paths relative to the reference root).
// Compiled with -ffp-contract=off so every expression is evaluated in
// source order, like the reference's C++ without fused multiply-adds.

#include "pimc_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11).  Stands in for SPRNG 2 (Common/Random/Random.h:19).
// ---------------------------------------------------------------------------
inline void philox4x32_10(uint32_t ctr[4], uint32_t key0, uint32_t key1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)M0 * ctr[0];
    uint64_t p1 = (uint64_t)M1 * ctr[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ ctr[1] ^ key0;
    uint32_t n2 = hi0 ^ ctr[3] ^ key1;
    ctr[0] = n0; ctr[1] = lo1; ctr[2] = n2; ctr[3] = lo0;
    key0 += W0; key1 += W1;
  }
}

// Uniform double in [0,1): element `index` of stream `stream` under `seed`.
// Two doubles per Philox block, 53 bits each (27 + 26 bits of two words).
inline double philox_uniform(uint64_t seed, uint32_t stream, uint64_t index) {
  uint64_t block = index >> 1;
  uint32_t c[4] = {(uint32_t)block, (uint32_t)(block >> 32), stream, 0x50494D43u};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  int h = (int)(index & 1);
  uint32_t a = c[2 * h] >> 5, b = c[2 * h + 1] >> 6;
  return ((double)a * 67108864.0 + (double)b) * (1.0 / 9007199254740992.0);
}

enum { STREAM_LOCAL = 0, STREAM_COMMON = 1, STREAM_WORLD = 2 };

// RandomClass semantics (Common/Random/Random.h:33-49,156-180,268-273).
struct Random {
  uint64_t seed = 0;
  uint32_t stream = STREAM_LOCAL;  // Philox stream of Local()
  uint64_t nlocal = 0, nworld = 0;
  bool one_left = false;  // the static polar-method cache, Random.h:159-160
  double x2 = 0.0;
  double Local() { return philox_uniform(seed, stream, nlocal++); }
  double World() { return philox_uniform(seed, STREAM_WORLD, nworld++); }
  int LocalInt(int max) { return (int)floor(Local() * max); }
  double LocalGaussian(double sigma) {
    double V1, V2, S, X1;
    if (one_left) {
      X1 = x2;
      one_left = false;
    } else {
      do {
        V1 = 2.0 * Local() - 1.0;
        V2 = 2.0 * Local() - 1.0;
        S = V1 * V1 + V2 * V2;
      } while (S >= 1.0);
      double temp = sqrt((-2.0 * log(S)) / S);
      X1 = V1 * temp;
      x2 = V2 * temp;
      one_left = true;
    }
    return X1 * sigma;
  }
};

// ---------------------------------------------------------------------------
// Grids (Common/Splines/Grid.h:69-136 LinearGrid, :519-575 LogGrid).
// ---------------------------------------------------------------------------
struct Grid {
  int type = 0;  // 0 LINEAR, 1 LOG
  double Start = 0, End = 0;
  int NumPoints = 0;
  std::vector<double> x;
  double delta = 0, deltainv = 0;
  double Z = 1, r0 = 0, Spacing = 1;

  void InitLinear(double start, double end, int n) {  // Grid.h:88-97
    type = 0; Start = start; End = end; NumPoints = n;
    x.resize(n);
    delta = (End - Start) / (double)(NumPoints - 1);
    deltainv = 1.0 / delta;
    for (int i = 0; i < n; i++) x[i] = Start + (double)i * delta;
  }
  void InitLog(double R0, double spacing, int n) {  // Grid.h:541-551
    type = 1; NumPoints = n; Z = 1.0; r0 = R0; Spacing = spacing;
    Start = r0;
    End = r0 * pow(Spacing, (double)NumPoints - 1);
    x.resize(n);
    for (int i = 0; i < n; i++) x[i] = r0 * pow(Spacing, (double)i);
  }
  int ReverseMap(double r) const {
    if (type == 0) return (int)nearbyint((r - Start) * deltainv - 0.5);  // Grid.h:81-84
    return (int)(floor(log(Z * r / r0) / log(Spacing)));                  // Grid.h:527-530
  }
  double operator()(int i) const { return x[i]; }
};

// ---------------------------------------------------------------------------
// MultiCubicSpline (Common/Splines/CubicSpline.h:288-561, CubicSpline.cc:77-128).
// y and d2y are stored row-major [grid point][spline].
// ---------------------------------------------------------------------------
struct MultiSpline {
  const Grid *grid = nullptr;
  int NumGridPoints = 0, NumSplines = 0;
  std::vector<double> y, d2y, StartDeriv, EndDeriv;

  void Init(const Grid *g, const double *ys, int nsplines, const double *sd, const double *ed) {
    grid = g; NumGridPoints = g->NumPoints; NumSplines = nsplines;
    y.assign(ys, ys + (size_t)NumGridPoints * NumSplines);
    d2y.assign(y.size(), 0.0);
    StartDeriv.assign(sd, sd + nsplines);
    EndDeriv.assign(ed, ed + nsplines);
    for (int i = 0; i < NumSplines; i++) Update(i);
  }
  double &Y(int j, int i) { return y[(size_t)j * NumSplines + i]; }
  double &D(int j, int i) { return d2y[(size_t)j * NumSplines + i]; }
  // Tridiagonal solve after Numerical Recipes (CubicSpline.cc:77-128).
  void Update(int i) {
    const Grid &x = *grid;
    int N = x.NumPoints;
    std::vector<double> U(N);
    if (StartDeriv[i] > 0.99e30) {
      D(0, i) = 0.0;
      U[0] = 0.0;
    } else {
      D(0, i) = -0.5;
      U[0] = (3.0 / (x(1) - x(0))) * ((Y(1, i) - Y(0, i)) / (x(1) - x(0)) - StartDeriv[i]);
    }
    D(NumGridPoints - 1, i) = 0.0;
    for (int j = 1; j < NumGridPoints - 1; j++) {
      double sig = (x(j) - x(j - 1)) / (x(j + 1) - x(j - 1));
      double p = sig * D(j - 1, i) + 2.0;
      D(j, i) = (sig - 1.0) / p;
      U[j] = (6.0 * ((Y(j + 1, i) - Y(j, i)) / (x(j + 1) - x(j)) - (Y(j, i) - Y(j - 1, i)) / (x(j) - x(j - 1))) /
                  (x(j + 1) - x(j - 1)) -
              sig * U[j - 1]) /
             p;
    }
    double Un, Qn;
    if (EndDeriv[i] > 0.99e30) {
      Un = 0.0;
      Qn = 0.0;
    } else {
      Qn = 0.5;
      Un = (3.0 / (x(N - 1) - x(N - 2))) * (EndDeriv[i] - (Y(N - 1, i) - Y(N - 2, i)) / (x(N - 1) - x(N - 2)));
    }
    D(N - 1, i) = (Un - Qn * U[N - 2]) / (Qn * D(N - 2, i) + 1.0);
    for (int k = N - 2; k >= 0; k--) D(k, i) = D(k, i) * D(k + 1, i) + U[k];
  }
  // CubicSpline.h:470-505
  double operator()(int i, double x) const {
    const Grid &X = *grid;
    int hi = X.ReverseMap(x) + 1;
    int low = hi - 1;
    if (low < 0) { low = 0; hi = 1; }
    if (hi > (X.NumPoints - 1)) { hi = (X.NumPoints - 1); low = hi - 1; }
    double h = X(hi) - X(low);
    double hinv = 1.0 / h;
    double a = (X(hi) - x) * hinv;
    double b = (x - X(low)) * hinv;
    double sixinv = 0.1666666666666666666;
    const double *yl = &y[(size_t)low * NumSplines], *yh = &y[(size_t)hi * NumSplines];
    const double *dl = &d2y[(size_t)low * NumSplines], *dh = &d2y[(size_t)hi * NumSplines];
    return (a * yl[i] + b * yh[i] + ((a * a * a - a) * dl[i] + (b * b * b - b) * dh[i]) * (h * h * sixinv));
  }
  // CubicSpline.h:508-545
  void operator()(double x, double *yVec) const {
    const Grid &X = *grid;
    int hi = X.ReverseMap(x) + 1;
    int low = hi - 1;
    if (low < 0) { low = 0; hi = 1; }
    if (hi > (X.NumPoints - 1)) { hi = (X.NumPoints - 1); low = hi - 1; }
    double h = X(hi) - X(low);
    double hinv = 1.0 / h;
    double a = (X(hi) - x) * hinv;
    double b = (x - X(low)) * hinv;
    double a3minusa = a * a * a - a;
    double b3minusb = b * b * b - b;
    double h2over6 = h * h * 0.1666666666666666666;
    const double *yl = &y[(size_t)low * NumSplines], *yh = &y[(size_t)hi * NumSplines];
    const double *dl = &d2y[(size_t)low * NumSplines], *dh = &d2y[(size_t)hi * NumSplines];
    for (int i = 0; i < NumSplines; i++)
      yVec[i] = a * yl[i] + b * yh[i] + (a3minusa * dl[i] + b3minusb * dh[i]) * h2over6;
  }
};

// Single CubicSpline with natural ends (CubicSpline.h:165-204, CubicSpline.cc:20-60).
struct Spline1 {
  Grid grid;
  MultiSpline s;
  void Init(double start, double end, int n, const double *data) {
    grid.InitLinear(start, end, n);
    double sd = 5.0e30, ed = 5.0e30;
    s.Init(&grid, data, 1, &sd, &ed);
  }
  double operator()(double x) const { return s(0, x); }
};

// ---------------------------------------------------------------------------
// MyTricubicSpline (Common/Splines/MyTricubicSpline.h:35-334, .cc:19-101).
// F stored [ix][iy][iz][8], components F, Fx, Fy, Fz, Fxy, Fxz, Fyz, Fxyz.
// ---------------------------------------------------------------------------
struct Tricubic {
  Grid X, Yg, Zg;
  int Nx = 0, Ny = 0, Nz = 0;
  std::vector<double> F;
  double &f(int ix, int iy, int iz, int c) { return F[(((size_t)ix * Ny + iy) * Nz + iz) * 8 + c]; }
  double fc(int ix, int iy, int iz, int c) const { return F[(((size_t)ix * Ny + iy) * Nz + iz) * 8 + c]; }

  void Init(const Grid &gx, const Grid &gy, const Grid &gz, const double *init) {
    X = gx; Yg = gy; Zg = gz;
    Nx = X.NumPoints; Ny = Yg.NumPoints; Nz = Zg.NumPoints;
    F.assign((size_t)Nx * Ny * Nz * 8, 0.0);
    for (int ix = 0; ix < Nx; ix++)
      for (int iy = 0; iy < Ny; iy++)
        for (int iz = 0; iz < Nz; iz++) f(ix, iy, iz, 0) = init[((size_t)ix * Ny + iy) * Nz + iz];
    Update();
  }
  // MyTricubicSpline.cc:19-50 (non-periodic branch)
  void Update() {
    UpdateAxis(0, 0, 1);
    UpdateAxis(1, 0, 2);
    UpdateAxis(2, 0, 3);
    UpdateAxis(1, 1, 4);
    UpdateAxis(2, 1, 5);
    UpdateAxis(2, 2, 6);
    UpdateAxis(2, 4, 7);
  }
  // UpdateX/UpdateY/UpdateZ (MyTricubicSpline.cc:52-101 and siblings): the
  // same tridiagonal first-derivative solve along one axis, end condition
  // 1.5*delta/h.
  void UpdateAxis(int axis, int source, int dest) {
    const Grid &g = axis == 0 ? X : (axis == 1 ? Yg : Zg);
    int n = g.NumPoints;
    int o1 = axis == 0 ? Ny : Nx, o2 = axis == 2 ? Ny : Nz;
    std::vector<double> mu(n);
    for (int a = 0; a < o1; a++)
      for (int b = 0; b < o2; b++) {
        auto at = [&](int j, int c) -> double & {
          if (axis == 0) return f(j, a, b, c);
          if (axis == 1) return f(a, j, b, c);
          return f(a, b, j, c);
        };
        at(0, dest) = 1.5 * (at(1, source) - at(0, source)) / (g(1) - g(0));
        at(n - 1, dest) = 1.5 * (at(n - 1, source) - at(n - 2, source)) / (g(n - 1) - g(n - 2));
        mu[0] = 0.5;
        for (int j = 1; j < (n - 1); j++) {
          double lambda = 0.5 * (g(j + 1) - g(j)) / (g(j + 1) - g(j - 1));
          mu[j] = 0.5 - lambda;
          at(j, dest) = 3.0 * (lambda * (at(j, source) - at(j - 1, source)) / (g(j) - g(j - 1)) +
                               mu[j] * (at(j + 1, source) - at(j, source)) / (g(j + 1) - g(j)));
          double cj = 1.0 - lambda * mu[j - 1];
          at(j, dest) -= lambda * at(j - 1, dest);
          mu[j] /= cj;
          at(j, dest) /= cj;
        }
        int j = n - 1;
        double lambda = 0.5;
        mu[j] = 0.5 - lambda;
        at(j, dest) = 3.0 * (lambda * (at(j, source) - at(j - 1, source)) / (g(j) - g(j - 1)));
        double cj = 1.0 - lambda * mu[j - 1];
        at(j, dest) -= lambda * at(j - 1, dest);
        mu[j] /= cj;
        at(j, dest) /= cj;
        for (j = n - 2; j >= 0; j--) at(j, dest) -= mu[j] * at(j + 1, dest);
      }
  }
  static double p1(double t) { return ((t - 1.0) * (t - 1.0) * (1.0 + 2.0 * t)); }
  static double p2(double t) { return (t * t * (3.0 - 2.0 * t)); }
  static double q1(double t) { return (t * (t - 1.0) * (t - 1.0)); }
  static double q2(double t) { return (t * t * (t - 1.0)); }
  // MyTricubicSpline.h:197-334
  double operator()(double x, double y, double z) const {
    int ix = X.ReverseMap(x), iy = Yg.ReverseMap(y), iz = Zg.ReverseMap(z);
    ix = std::max(0, ix); ix = std::min(ix, Nx - 2);
    iy = std::max(0, iy); iy = std::min(iy, Ny - 2);
    iz = std::max(0, iz); iz = std::min(iz, Nz - 2);
    double h = X(ix + 1) - X(ix);
    double k = Yg(iy + 1) - Yg(iy);
    double l = Zg(iz + 1) - Zg(iz);
    double u = (x - X(ix)) / h;
    double v = (y - Yg(iy)) / k;
    double w = (z - Zg(iz)) / l;
    double a[4] = {p1(u), p2(u), h * q1(u), h * q2(u)};
    double b[4] = {p1(v), p2(v), k * q1(v), k * q2(v)};
    double c[4] = {p1(w), p2(w), l * q1(w), l * q2(w)};
    // Y_{abc}: node (ix + a&1, iy + b&1, iz + c&1); derivative along an axis
    // when that basis index is >= 2.
    static const int comp[2][2][2] = {{{0, 3}, {2, 6}}, {{1, 5}, {4, 7}}};
    double val = 0.0;
    for (int ia = 0; ia < 4; ia++) {
      double sb = 0.0;
      for (int ib = 0; ib < 4; ib++) {
        double sc = 0.0;
        for (int ic = 0; ic < 4; ic++) {
          double Y = fc(ix + (ia & 1), iy + (ib & 1), iz + (ic & 1), comp[ia >> 1][ib >> 1][ic >> 1]);
          double t = Y * c[ic];
          sc = (ic == 0) ? t : sc + t;
        }
        double t = b[ib] * sc;
        sb = (ib == 0) ? t : sb + t;
      }
      double t = a[ia] * sb;
      val = (ia == 0) ? t : val + t;
    }
    return val;
  }
};

}  // namespace

// ---------------------------------------------------------------------------
// Pair actions
// ---------------------------------------------------------------------------
struct OraclePA {
  int kind = 0;  // 1 David, 2 tricubic, 3 classical Coulomb
  // DavidPAClass (Common/PairAction/DavidPAClass.h, .cc)
  Grid ugrid, dugrid;
  std::vector<MultiSpline> ukj, dukj;
  int NumTau = 0, TauPos = 0, NumTerms = 0, NumUKJ = 0;
  // PAtricubicFitClass
  Grid qgrid, ygrid, tgrid;
  std::vector<Tricubic> Usplines, dUsplines;
  double SmallestBeta = 0;
  int NumBetas = 0;
  Spline1 pot;
  // PAclassicalFitClass with CoulombPot
  double Z1Z2 = 0;

  bool IsLongRange() const {
    if (kind == 1) return false;        // DavidPAClass.cc:127-130
    if (kind == 2) return true;         // PAtricubicFit.cc:869-872
    return Z1Z2 != 0.0;                 // PAclassicalFit.cc:112-117
  }

  // DavidPAClass::calcUsqzFast (DavidPAClass.cc:468-511)
  double calcUsqzFast(double s, double q, double z, int level) const {
    level = level + TauPos;
    const MultiSpline &u = ukj[level];
    double rmin = u.grid->Start;
    double U = 0.0;
    double r = q + 0.5 * z;
    double rprime = q - 0.5 * z;
    if (r > u.grid->End) r = u.grid->End;
    if (rprime > u.grid->End) rprime = u.grid->End;
    if ((rprime < rmin) || (r < rmin)) return u(1, rmin);
    U += 0.5 * (u(1, r) + u(1, rprime));
    if (s > 0.0 && q < u.grid->End) {
      double zsquared = z * z;
      double ssquared = s * s;
      double ssquaredinverse = 1.0 / ssquared;
      double Sto2k = ssquared;
      std::vector<double> tmp(u.NumSplines);
      u(q, tmp.data());
      for (int k = 1; k <= NumTerms; k++) {
        double Zto2j = 1;
        double currS = Sto2k;
        for (int j = 0; j <= k; j++) {
          double Ucof = tmp[k * (k + 1) / 2 + j + 1];
          U += (Ucof)*Zto2j * currS;
          Zto2j *= zsquared;
          currS = currS * ssquaredinverse;
        }
        Sto2k = Sto2k * ssquared;
      }
    }
    return U;
  }
  // DavidPAClass::calcUsqz, the dU output (DavidPAClass.cc:291-463)
  double calcUsqz_dU(double s, double q, double z, int level) const {
    level = level + TauPos;
    const MultiSpline &u = ukj[level];
    const MultiSpline &du = dukj[level];
    double rmin = u.grid->Start;
    double dU = 0.0;
    double r = q + 0.5 * z;
    double rprime = q - 0.5 * z;
    if (r > u.grid->End) r = u.grid->End;
    if (rprime > u.grid->End) rprime = u.grid->End;
    if (rprime < rmin) rprime = rmin;
    if (r < rmin) r = rmin;
    double V = 0.5 * (u(0, r) + u(0, rprime));
    dU += 0.5 * (du(1, r) + du(1, rprime));
    dU += V;
    if (s > 0.0 && q < u.grid->End) {
      double zsquared = z * z;
      double ssquared = s * s;
      double ssquaredinverse = 1.0 / ssquared;
      double Sto2k = ssquared;
      std::vector<double> tmpd(du.NumSplines);
      du(q, tmpd.data());
      for (int k = 1; k <= NumTerms; k++) {
        double Zto2j = 1;
        double currS = Sto2k;
        for (int j = 0; j <= k; j++) {
          double dUcof = tmpd[k * (k + 1) / 2 + j + 1];
          dU += (dUcof)*Zto2j * currS;
          Zto2j *= zsquared;
          currS = currS * ssquaredinverse;
        }
        Sto2k = Sto2k * ssquared;
      }
    }
    return dU;
  }
  // SplinePot::V (Common/PH/SplinePot.cc:19-31), no Vouter.
  double PotV(double r) const {
    if (r <= pot.grid.End) return pot(r);
    return 0.0;
  }
  // PairActionFitClass::V: DavidPAClass::V (DavidPAClass.cc:104-113) evaluates
  // column 0 of the first tau table with r clamped to the grid; PAFitBase::V
  // (PAFitBase.h:82) the potential; CoulombPot Z1Z2/r.
  double V(double r) const {
    if (kind == 1) {
      if (r > ukj[0].grid->End) r = ukj[0].grid->End;
      if (r < ukj[0].grid->Start) r = ukj[0].grid->Start;
      return ukj[0](0, r);
    }
    if (kind == 2) return PotV(r);
    return Z1Z2 / r;
  }
  double U(double q, double z, double s2, int level) const {
    if (kind == 1) {  // DavidPAClass::U (DavidPAClass.cc:92-102)
      double s = sqrt(s2);
      return calcUsqzFast(s, q, z, level);
    }
    if (kind == 2) {  // PAtricubicFitClass::U (PAtricubicFit.cc:659-695)
      z = fabs(z);
      double qmax = qgrid.End;
      double smax = 2.0 * q;
      double zmax = smax;
      double s = sqrt(s2);
      if ((q <= qmax) && (z < zmax) && (s < smax)) {
        if (q == 0.0) return Usplines[level](0.0, 0.0, 0.0);
        double y = z / zmax;
        double t = (s - z) / (smax - z);
        return Usplines[level](q, y, t);
      }
      double beta = SmallestBeta;
      for (int i = 0; i < level; i++) beta *= 2.0;
      double r = q + 0.5 * z;
      double rp = q - 0.5 * z;
      return 0.5 * beta * (PotV(r) + PotV(rp));
    }
    // PAclassicalFitClass::U (PAclassicalFit.cc:57-66) with CoulombPot V = Z1Z2/r
    double beta = SmallestBeta;
    for (int i = 0; i < level; i++) beta *= 2.0;
    double V = Z1Z2 / q;
    return (beta * V);
  }
  double dU(double q, double z, double s2, int level) const {
    if (kind == 1) {  // DavidPAClass::dU (DavidPAClass.cc:115-126)
      double s = sqrt(s2);
      return calcUsqz_dU(s, q, z, level);
    }
    if (kind == 2) {  // PAtricubicFitClass::dU (PAtricubicFit.cc:697-721)
      z = fabs(z);
      double qmax = qgrid.End;
      double smax = 2.0 * q;
      double zmax = smax;
      double s = sqrt(s2);
      if ((q <= qmax) && (z < zmax) && (s < smax)) {
        if (q == 0.0) return dUsplines[level](0.0, 0.0, 0.0);
        double y = z / zmax;
        double t = (s - z) / (smax - z);
        return dUsplines[level](q, y, t);
      }
      double r = q + 0.5 * z;
      double rp = q - 0.5 * z;
      return 0.5 * (PotV(r) + PotV(rp));
    }
    return Z1Z2 / q;  // PAclassicalFit.cc:68-75
  }
};

namespace {

// Line helpers with the behaviour of DavidPAClass.h:186-290 (SkipTo,
// GetNextInt, GetNextWord, GetNextDouble).
bool skip_to(std::ifstream &in, const std::string &key, std::string &line) {
  while (std::getline(in, line)) {
    if (line.find(key) != std::string::npos) return true;
  }
  return false;
}
bool is_digit_char(char c) { return (c >= '0' && c <= '9') || c == '-'; }
bool is_number_char(char c) { return (c >= '0' && c <= '9') || c == '-' || c == '.'; }
int next_int(std::string &s) {
  size_t i = 0;
  while (i < s.size() && !is_digit_char(s[i])) i++;
  s = s.substr(i);
  const char *p = s.c_str();
  char *end = nullptr;
  long v = strtol(p, &end, 10);
  s = s.substr(end - p);
  return (int)v;
}
double next_double(std::string &s) {
  size_t i = 0;
  while (i < s.size() && !is_number_char(s[i])) i++;
  s = s.substr(i);
  const char *p = s.c_str();
  char *end = nullptr;
  double v = strtod(p, &end);
  s = s.substr(end - p);
  return v;
}
std::string next_word(std::string &s) {
  size_t c = 0;
  while (c < s.size() && s[c] == ' ') c++;
  size_t start = c;
  while (c < s.size() && s[c] != ' ') c++;
  std::string w = s.substr(start, c - start);
  s = s.substr(c);
  return w;
}

// Reads one "RANK 3" block header and its table (DavidPAClass.cc:688-771).
// Returns false on a format error.
bool read_fit_block(std::ifstream &in, int &NumGridPoints, int &NumUKJ, int &NumTau, Grid &grid,
                    double &smallestTau, int &NMax, int &derv, std::vector<double> &table) {
  std::string line;
  for (;;) {
    if (!skip_to(in, "RANK", line)) return false;
    int rank = next_int(line);
    if (rank == 3) break;
  }
  NumGridPoints = next_int(line);
  NumUKJ = next_int(line);
  NumTau = next_int(line);
  if (!skip_to(in, "GRID 1", line)) return false;
  next_word(line); next_word(line);
  std::string gtype = next_word(line);
  double g0 = next_double(line);
  double g1 = next_double(line);
  if (gtype == "LINEAR") {
    grid.InitLinear(g0, g1, NumGridPoints);
  } else if (gtype == "LOG") {
    double delta = pow((g1 / g0), 1.0 / (NumGridPoints - 1.0));
    grid.InitLog(g0, delta, NumGridPoints);
  } else {
    return false;
  }
  if (!skip_to(in, "GRID   3", line)) return false;
  next_word(line); next_word(line);
  if (next_word(line) != "LOG") return false;
  smallestTau = next_double(line);
  double largestTau = next_double(line);
  int numTauCalc = (int)floor(log(largestTau / smallestTau) / log(2.0) + 0.5 + 1.0);
  if (numTauCalc != NumTau) return false;
  if (!skip_to(in, "BEGIN density matrix table", line)) return false;
  NMax = next_int(line);
  derv = next_int(line);
  // ReadFORTRAN3Tensor (DavidPAClass.h:205-219): grid fastest, then ukj, then tau.
  table.assign((size_t)NumGridPoints * NumUKJ * NumTau, 0.0);
  for (int t = 0; t < NumTau; t++)
    for (int u = 0; u < NumUKJ; u++)
      for (int g = 0; g < NumGridPoints; g++) {
        double v;
        if (!(in >> v)) return false;
        table[((size_t)g * NumUKJ + u) * NumTau + t] = v;
      }
  return true;
}

}  // namespace

extern "C" {

double oracle_philox_uniform(uint64_t seed, uint32_t stream, uint64_t index) {
  return philox_uniform(seed, stream, index);
}
void oracle_philox_block(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  for (int i = 0; i < 4; i++) out[i] = ctr[i];
  philox4x32_10(out, key[0], key[1]);
}

// DavidPAClass::ReadDavidSquarerFile (DavidPAClass.cc:635-912)
OraclePA *oracle_pa_david_from_dm(const char *path, double desired_tau, int num_offdiag_terms) {
  std::ifstream in(path);
  if (!in) return nullptr;
  std::string line;
  if (!skip_to(in, "SQUARER", line)) return nullptr;
  next_word(line); next_word(line); next_word(line); next_word(line);
  int numOfFits = next_int(line);
  if (!skip_to(in, "RANK", line)) return nullptr;
  next_word(line); next_word(line);
  int numPotPoints = next_int(line);
  std::vector<double> potential(numPotPoints);
  if (!skip_to(in, "potential", line)) return nullptr;
  for (int i = 0; i < numPotPoints; i++)
    if (!(in >> potential[i])) return nullptr;

  OraclePA *pa = new OraclePA();
  pa->kind = 1;
  pa->NumTerms = num_offdiag_terms;
  bool have_u = false, have_du = false;
  for (int pass = 0; pass < 2; pass++) {
    for (int counter = 0; counter <= numOfFits; counter++) {
      int ng, nukj, ntau, nmax, derv;
      double smallestTau;
      Grid g;
      std::vector<double> t;
      if (!read_fit_block(in, ng, nukj, ntau, g, smallestTau, nmax, derv, t)) {
        delete pa;
        return nullptr;
      }
      if (derv != pass + 1) { delete pa; return nullptr; }
      if (ng != numPotPoints) { delete pa; return nullptr; }
      pa->NumTau = ntau;
      if (pass == 1) {
        double tau = smallestTau;
        for (int i = 0; i < ntau; i++) {  // DavidPAClass.cc:857-867
          if (fabs(tau - desired_tau) < 1e-4) pa->TauPos = i;
          tau = tau * 2;
        }
      }
      if (nmax != 2) continue;  // only the NMax==2 fit initialises the splines
      int ncol = nukj + 1;
      std::vector<double> startDeriv(ncol, 5.0e30), endDeriv(ncol, 0.0);
      Grid &grid = (pass == 0) ? pa->ugrid : pa->dugrid;
      grid = g;
      std::vector<MultiSpline> &dest = (pass == 0) ? pa->ukj : pa->dukj;
      dest.assign(ntau, MultiSpline());
      for (int lev = 0; lev < ntau; lev++) {
        std::vector<double> ys((size_t)ng * ncol);
        for (int gi = 0; gi < ng; gi++) {
          ys[(size_t)gi * ncol + 0] = potential[gi];
          for (int u = 0; u < nukj; u++) ys[(size_t)gi * ncol + 1 + u] = t[((size_t)gi * nukj + u) * ntau + lev];
        }
        for (int c = 0; c < ncol; c++) ys[(size_t)(ng - 1) * ncol + c] = 0.0;  // last row zeroed
        dest[lev].Init(&grid, ys.data(), ncol, startDeriv.data(), endDeriv.data());
      }
      pa->NumUKJ = nukj;
      if (pass == 0) have_u = true; else have_du = true;
    }
  }
  if (!have_u || !have_du) {
    delete pa;
    return nullptr;
  }
  return pa;
}

// DavidPAClass tables from arrays on a LINEAR grid: ukj/dukj [tau][grid][ncols]
// (column 0 the potential), splines built like ReadDavidSquarerFile does.
OraclePA *oracle_pa_david_arrays(double grid_start, double grid_end, int n, int ncols, int ntau, const double *ukj,
                                 const double *dukj, int tau_pos, int num_terms) {
  OraclePA *pa = new OraclePA();
  pa->kind = 1;
  pa->NumTerms = num_terms;
  pa->NumTau = ntau;
  pa->TauPos = tau_pos;
  pa->NumUKJ = ncols - 1;
  pa->ugrid.InitLinear(grid_start, grid_end, n);
  pa->dugrid = pa->ugrid;
  std::vector<double> sd(ncols, 5.0e30), ed(ncols, 0.0);
  pa->ukj.assign(ntau, MultiSpline());
  pa->dukj.assign(ntau, MultiSpline());
  for (int lev = 0; lev < ntau; lev++) {
    pa->ukj[lev].Init(&pa->ugrid, ukj + (size_t)lev * n * ncols, ncols, sd.data(), ed.data());
    pa->dukj[lev].Init(&pa->dugrid, dukj + (size_t)lev * n * ncols, ncols, sd.data(), ed.data());
  }
  return pa;
}

OraclePA *oracle_pa_tricubic(double q0, double q1, int nq, double y0, double y1, int ny, double t0,
                             double t1, int nt, int num_betas, double smallest_beta, const double *umat,
                             const double *dumat, double pot_start, double pot_end, int pot_n,
                             const double *pot_data) {
  OraclePA *pa = new OraclePA();
  pa->kind = 2;
  pa->qgrid.InitLinear(q0, q1, nq);
  pa->ygrid.InitLinear(y0, y1, ny);
  pa->tgrid.InitLinear(t0, t1, nt);
  pa->NumBetas = num_betas;
  pa->SmallestBeta = smallest_beta;
  pa->Usplines.resize(num_betas);
  pa->dUsplines.resize(num_betas);
  size_t per = (size_t)nq * ny * nt;
  for (int b = 0; b < num_betas; b++) {
    pa->Usplines[b].Init(pa->qgrid, pa->ygrid, pa->tgrid, umat + b * per);
    pa->dUsplines[b].Init(pa->qgrid, pa->ygrid, pa->tgrid, dumat + b * per);
  }
  pa->pot.Init(pot_start, pot_end, pot_n, pot_data);
  return pa;
}

OraclePA *oracle_pa_classical_coulomb(double smallest_beta, int num_betas, double z1z2) {
  OraclePA *pa = new OraclePA();
  pa->kind = 3;
  pa->SmallestBeta = smallest_beta;
  pa->NumBetas = num_betas;
  pa->Z1Z2 = z1z2;
  return pa;
}

void oracle_pa_free(OraclePA *pa) { delete pa; }
double oracle_pa_U(OraclePA *pa, double q, double z, double s2, int level) { return pa->U(q, z, s2, level); }
double oracle_pa_dU(OraclePA *pa, double q, double z, double s2, int level) { return pa->dU(q, z, s2, level); }

int oracle_pa_info(OraclePA *pa, int *num_tau, int *tau_pos, int *num_grid, int *num_cols, double *grid_start,
                   double *grid_end, int *grid_type) {
  if (pa->kind != 1) return 1;
  *num_tau = pa->NumTau;
  *tau_pos = pa->TauPos;
  *num_grid = pa->ugrid.NumPoints;
  *num_cols = pa->NumUKJ + 1;
  *grid_start = pa->ugrid.Start;
  *grid_end = pa->ugrid.End;
  *grid_type = pa->ugrid.type;
  return 0;
}

int oracle_pa_david_table(OraclePA *pa, int which, int level, double *out) {
  if (pa->kind != 1 || level < 0 || level >= pa->NumTau) return 1;
  const MultiSpline &s = (which < 2) ? pa->ukj[level] : pa->dukj[level];
  const std::vector<double> &v = (which % 2 == 0) ? s.y : s.d2y;
  memcpy(out, v.data(), v.size() * sizeof(double));
  return 0;
}

double oracle_pa_david_spline(OraclePA *pa, int which, int level, int col, double x) {
  const MultiSpline &s = (which == 0) ? pa->ukj[level] : pa->dukj[level];
  return s(col, x);
}

struct OracleTricubic {
  Tricubic t;
};

OracleTricubic *oracle_tricubic_create(double x0, double x1, int nx, double y0, double y1, int ny, double z0,
                                       double z1, int nz, const double *f) {
  OracleTricubic *o = new OracleTricubic();
  Grid gx, gy, gz;
  gx.InitLinear(x0, x1, nx);
  gy.InitLinear(y0, y1, ny);
  gz.InitLinear(z0, z1, nz);
  o->t.Init(gx, gy, gz, f);
  return o;
}
double oracle_tricubic_eval(OracleTricubic *t, double x, double y, double z) { return t->t(x, y, z); }
int oracle_tricubic_coefs(OracleTricubic *t, double *out) {
  memcpy(out, t->t.F.data(), t->t.F.size() * sizeof(double));
  return 0;
}
void oracle_tricubic_free(OracleTricubic *t) { delete t; }

}  // extern "C"

// ---------------------------------------------------------------------------
// The system: PathClass (two mirrored copies), one species, the actions.
// ---------------------------------------------------------------------------
typedef double dVec[3];

struct OracleSystem {
  int N = 0, NumSlices = 0;  // NumTimeSlices() = M+1 rows
  double Box[3], BoxInv[3], IsPeriodic[3] = {1.0, 1.0, 1.0};
  double tau = 0, lambda = 0;
  int NumImages = 0;
  std::vector<double> path[2];  // [slice][ptcl][3]
  int mode = 0;                 // ActiveCopy (MirroredClass.cc:19): 0 OLD, 1 NEW
  OraclePA *pa = nullptr;
  Random rng;
  std::vector<Random> wrng;       // per-window Local streams of the concurrent schedule
  uint64_t rounds = 0;            // Common-stream index of the next round
  // bisection
  int NumLevels = 1, StepsPerBlock = 1, SRHigher = 1, UseLongRange = 0;
  // long range
  double kBox[3] = {0, 0, 0}, kCutoff = 0;
  int MaxkIndex[3] = {0, 0, 0};
  std::vector<double> kVecs;  // nk*3
  std::vector<int> kIndices;  // nk*3
  std::vector<std::complex<double>> Rho_k[2];  // [slice][k] (one species)
  int LRLevels = 0, UseBackground = 0;
  std::vector<double> Ulong_k, Ulong_r0, Ushort_k0, Ulong_k0, dUlong_k, dUlong_r0, dUshort_k0, dUlong_k0;

  double *P(int copy, int slice, int ptcl) { return &path[copy][((size_t)slice * N + ptcl) * 3]; }
  double *P(int slice, int ptcl) { return P(mode, slice, ptcl); }
  int nk() const { return (int)(kVecs.size() / 3); }

  // PathClass::DistDisp one-slice version (PathClass.h:637-660)
  double Dist1(int slice, int ptcl1, int ptcl2) {
    const double *a = P(slice, ptcl1), *b = P(slice, ptcl2);
    double disp[3];
    for (int i = 0; i < 3; i++) disp[i] = b[i] - a[i];
    double n[3];
    for (int i = 0; i < 3; i++) n[i] = nearbyint(disp[i] * BoxInv[i]);
    for (int i = 0; i < 3; i++) disp[i] -= n[i] * IsPeriodic[i] * Box[i];
    return sqrt(disp[0] * disp[0] + disp[1] * disp[1] + disp[2] * disp[2]);
  }
  // ShortRangePotClass::V(slice) (ShortRangePotClass.cc:28-47); Vlong of the
  // classical Coulomb action is its dUlong(0) (the V breakup fits the same X_k).
  double VSlice(int slice) {
    double val = 0.0;
    for (int ptcl1 = 0; ptcl1 < N; ptcl1++)
      for (int ptcl2 = 0; ptcl2 < ptcl1; ptcl2++) {
        const double dist = Dist1(slice, ptcl1, ptcl2);
        val += pa->V(dist);
        if (pa->IsLongRange() && UseLongRange) val -= dUlong(0, dist);
      }
    return val;
  }
  // PathClass::DistDisp two-slice version (PathClass.h:696-746)
  void DistDisp(int sliceA, int sliceB, int ptcl1, int ptcl2, double &distA, double &distB, dVec dispA,
                dVec dispB) {
    const double *a1 = P(sliceA, ptcl1), *a2 = P(sliceA, ptcl2);
    const double *b1 = P(sliceB, ptcl1), *b2 = P(sliceB, ptcl2);
    for (int i = 0; i < 3; i++) {
      dispA[i] = a2[i] - a1[i];
      dispB[i] = b2[i] - b1[i];
    }
    double n[3], m[3];
    for (int i = 0; i < 3; i++) n[i] = -nearbyint(dispA[i] * BoxInv[i]);
    for (int i = 0; i < 3; i++) dispA[i] += n[i] * IsPeriodic[i] * Box[i];
    for (int i = 0; i < 3; i++) m[i] = nearbyint((dispA[i] - dispB[i]) * BoxInv[i]);
    for (int i = 0; i < 3; i++) dispB[i] += m[i] * IsPeriodic[i] * Box[i];
    distA = sqrt(dispA[0] * dispA[0] + dispA[1] * dispA[1] + dispA[2] * dispA[2]);
    distB = sqrt(dispB[0] * dispB[0] + dispB[1] * dispB[1] + dispB[2] * dispB[2]);
  }
  // PathClass::PutInBox (PathClass.h:897-921)
  void PutInBox(dVec v) {
    for (int i = 0; i < 3; i++) {
      double n = -floor(v[i] * BoxInv[i] + 0.5);
      v[i] += n * IsPeriodic[i] * Box[i];
    }
  }
  // PathClass::PutInBoxFast (PathClass.cc:1389-1407)
  void PutInBoxFast(double *v) {
    for (int dim = 0; dim < 3; dim++) {
      double halfBox = Box[dim] / 2;
      if (v[dim] > halfBox) v[dim] -= Box[dim];
      if (v[dim] < -halfBox) v[dim] += Box[dim];
    }
  }
  // PathClass::Velocity (PathClass.h:831-865)
  void Velocity(int sliceA, int sliceB, int ptcl, dVec vel) {
    const double *a = P(sliceA, ptcl), *b = P(sliceB, ptcl);
    for (int i = 0; i < 3; i++) vel[i] = b[i] - a[i];
    PutInBox(vel);
  }

  // ShortRangeClass::SingleAction (ShortRangeClass.cc:191-236)
  double ShortRangeSingle(int slice1, int slice2, const int *changed, int nchanged, int level,
                          bool absolute = false) {
    double TotalU = 0.0;
    std::vector<char> DoPtcl(N, 1);
    int skip = 1 << level;
    for (int pi = 0; pi < nchanged; pi++) {
      int ptcl1 = changed[pi];
      DoPtcl[ptcl1] = 0;
      for (int ptcl2 = 0; ptcl2 < N; ptcl2++) {
        if (!DoPtcl[ptcl2]) continue;
        for (int slice = slice1; slice < slice2; slice += skip) {
          dVec r, rp;
          double rmag, rpmag;
          DistDisp(slice, slice + skip, ptcl1, ptcl2, rmag, rpmag, r, rp);
          double d0 = r[0] - rp[0], d1 = r[1] - rp[1], d2 = r[2] - rp[2];
          double s2 = d0 * d0 + d1 * d1 + d2 * d2;
          double q = 0.5 * (rmag + rpmag);
          double z = (rmag - rpmag);
          double U = pa->U(q, z, s2, level);
          // The absolute variant (a scale for the mixed-precision tolerance)
          // adds the magnitudes of the pair action and of the long-range part
          // separately: the difference cancels, their rounding does not.
          double mag = fabs(U);
          if (pa->IsLongRange() && UseLongRange) {
            const double ul = 0.5 * (Ulong(level, rmag) + Ulong(level, rpmag));
            U -= ul;
            mag += fabs(ul);
          }
          TotalU += absolute ? mag : U;
        }
      }
    }
    return TotalU;
  }
  // ShortRangeClass::d_dBeta (ShortRangeClass.cc:316-355)
  double ShortRangeDBeta(int slice1, int slice2, int level) {
    int skip = 1 << level;
    double dU = 0.0;
    for (int ptcl1 = 0; ptcl1 < N; ptcl1++)
      for (int ptcl2 = 0; ptcl2 < ptcl1; ptcl2++)
        for (int slice = slice1; slice < slice2; slice += skip) {
          dVec r, rp;
          double rmag, rpmag;
          DistDisp(slice, slice + skip, ptcl1, ptcl2, rmag, rpmag, r, rp);
          double d0 = r[0] - rp[0], d1 = r[1] - rp[1], d2 = r[2] - rp[2];
          double s2 = d0 * d0 + d1 * d1 + d2 * d2;
          double q = 0.5 * (rmag + rpmag);
          double z = (rmag - rpmag);
          dU += pa->dU(q, z, s2, level);
          if (pa->IsLongRange() && UseLongRange) dU -= 0.5 * (dUlong(level, rmag) + dUlong(level, rpmag));
        }
    return dU;
  }
  // PairActionFitClass::Ulong(level) / dUlong(level): QuinticSpline objects on
  // the LongGrid [0, rmax] (LongRangeClass.cc:547-549, 629, 818); here given
  // as Taylor coefficients per interval [level][point][6], evaluated as
  // QuinticSpline::operator() does (QuinticSpline.h:164-221).
  std::vector<double> ULongTab, dULongTab;
  int ULongPoints = 0;
  double ULongDelta = 0.0;
  double Quintic(const std::vector<double> &tab, int level, double x) const {
    if (ULongPoints == 0) return 0.0;
    const double deltainv = 1.0 / ULongDelta;
    int J = (int)nearbyint((x - 0.0) * deltainv - 0.5) + 1;
    int I = J - 1;
    if (I < 0) {
      I = 0;
      J = 1;
    }
    if (J > (ULongPoints - 1)) {
      J = ULongPoints - 1;
      I = J - 1;
    }
    const double *c = &tab[((size_t)level * ULongPoints + I) * 6];
    double P = (x - (0.0 + (double)I * ULongDelta));
    return ((((c[5] * P + c[4]) * P + c[3]) * P + c[2]) * P + c[1]) * P + c[0];
  }
  double Ulong(int level, double r) { return Quintic(ULongTab, level, r); }
  double dUlong(int level, double r) { return Quintic(dULongTab, level, r); }

  // KineticClass::SingleAction (KineticClass.cc:33-90)
  double KineticSingle(int slice1, int slice2, const int *changed, int nchanged, int level) {
    double TotalK = 0.0;
    int skip = 1 << level;
    double levelTau = tau * (1 << level);
    for (int pi = 0; pi < nchanged; pi++) {
      int ptcl = changed[pi];
      if (lambda != 0) {
        double FourLambdaTauInv = 1.0 / (4.0 * lambda * levelTau);
        for (int slice = slice1; slice < slice2; slice += skip) {
          dVec vel;
          Velocity(slice, slice + skip, ptcl, vel);
          double GaussProd = 1.0;
          for (int dim = 0; dim < 3; dim++) {
            double GaussSum = 0.0;
            for (int image = -NumImages; image <= NumImages; image++) {
              double dist = vel[dim] + (double)image * Box[dim];
              GaussSum += exp(-dist * dist * FourLambdaTauInv);
            }
            GaussProd *= GaussSum;
          }
          TotalK -= log(GaussProd);
        }
      }
    }
    return TotalK;
  }
  // KineticClass::d_dBeta (KineticClass.cc:187-256)
  double KineticDBeta(int slice1, int slice2, int level) {
    double spring = 0.0;
    double levelTau = ldexp(tau, level);
    int skip = 1 << level;
    for (int ptcl = 0; ptcl < N; ptcl++) {
      if (lambda == 0.0) continue;
      double FourLambdaTauInv = 1.0 / (4.0 * lambda * levelTau);
      for (int slice = slice1; slice < slice2; slice += skip) {
        spring += (0.5 * 3) / levelTau;
        dVec vel;
        Velocity(slice, slice + skip, ptcl, vel);
        double Z = 1.0;
        double GaussSum[3] = {0, 0, 0}, numSum[3] = {0, 0, 0};
        for (int dim = 0; dim < 3; dim++) {
          for (int image = -NumImages; image <= NumImages; image++) {
            double dist = vel[dim] + (double)image * Box[dim];
            double d2overFLT = dist * dist * FourLambdaTauInv;
            double expPart = exp(-d2overFLT);
            GaussSum[dim] += expPart;
            numSum[dim] += -d2overFLT / levelTau * expPart;
          }
          Z *= GaussSum[dim];
        }
        double scalarnumSum = 0.0;
        for (int dim = 0; dim < 3; dim++) {
          double numProd = 1.0;
          for (int dim2 = 0; dim2 < 3; dim2++) {
            if (dim2 != dim)
              numProd *= GaussSum[dim2];
            else
              numProd *= numSum[dim2];
          }
          scalarnumSum += numProd;
        }
        spring += scalarnumSum / Z;
      }
    }
    return spring;
  }

  // ---- rho_k (PathClass.cc:534-707) ----
  void SetupkVecs3D() {
    for (int i = 0; i < 3; i++) kBox[i] = 2.0 * M_PI / Box[i];
    for (int i = 0; i < 3; i++) MaxkIndex[i] = (int)ceil(1.1 * kCutoff / kBox[i]);
    kVecs.clear();
    kIndices.clear();
    for (int ix = -MaxkIndex[0]; ix <= MaxkIndex[0]; ix++) {
      double k0 = ix * kBox[0];
      for (int iy = -MaxkIndex[1]; iy <= MaxkIndex[1]; iy++) {
        double k1 = iy * kBox[1];
        for (int iz = -MaxkIndex[2]; iz <= MaxkIndex[2]; iz++) {
          double k2 = iz * kBox[2];
          bool include = (k0 > 0.0) || (k0 == 0.0 && k1 > 0.0) || (k0 == 0.0 && k1 == 0.0 && k2 > 0.0);
          if ((k0 * k0 + k1 * k1 + k2 * k2 < kCutoff * kCutoff) && include) {
            kVecs.push_back(k0); kVecs.push_back(k1); kVecs.push_back(k2);
            kIndices.push_back(ix + MaxkIndex[0]);
            kIndices.push_back(iy + MaxkIndex[1]);
            kIndices.push_back(iz + MaxkIndex[2]);
          }
        }
      }
    }
    for (int c = 0; c < 2; c++) Rho_k[c].assign((size_t)NumSlices * nk(), std::complex<double>(0.0, 0.0));
  }
  void FillC(const double *r, std::vector<std::complex<double>> C[3]) {
    for (int dim = 0; dim < 3; dim++) {
      C[dim].assign(2 * MaxkIndex[dim] + 1, std::complex<double>(0.0, 0.0));
      double phi = r[dim] * kBox[dim];
      std::complex<double> tempC(cos(phi), sin(phi));
      C[dim][MaxkIndex[dim]] = 1.0;
      for (int n = 1; n <= MaxkIndex[dim]; n++) {
        C[dim][MaxkIndex[dim] + n] = tempC * C[dim][MaxkIndex[dim] + n - 1];
        C[dim][MaxkIndex[dim] - n] = std::conj(C[dim][MaxkIndex[dim] + n]);
      }
    }
  }
  // CalcRho_ks_Fast (PathClass.cc:616-647), on the active copy
  void CalcRho_ks_Fast(int slice) {
    int K = nk();
    std::complex<double> *rk = &Rho_k[mode][(size_t)slice * K];
    for (int ki = 0; ki < K; ki++) rk[ki] = 0.0;
    std::vector<std::complex<double>> C[3];
    for (int ptcl = 0; ptcl < N; ptcl++) {
      FillC(P(slice, ptcl), C);
      for (int ki = 0; ki < K; ki++) {
        const int *kI = &kIndices[ki * 3];
        rk[ki] += C[0][kI[0]] * C[1][kI[1]] * C[2][kI[2]];
      }
    }
  }
  // UpdateRho_ks(slice1, slice2, changed, level) (PathClass.cc:649-707)
  void UpdateRho_ks(int slice1, int slice2, const int *changed, int n, int level) {
    int skip = 1 << level, K = nk();
    for (int slice = slice1; slice <= slice2; slice += skip)
      for (int ki = 0; ki < K; ki++) Rho_k[1][(size_t)slice * K + ki] = Rho_k[0][(size_t)slice * K + ki];
    std::vector<std::complex<double>> C[3];
    for (int pi = 0; pi < n; pi++) {
      int ptcl = changed[pi];
      for (int slice = slice1; slice <= slice2; slice += skip) {
        std::complex<double> *rk = &Rho_k[1][(size_t)slice * K];
        FillC(P(1, slice, ptcl), C);
        for (int ki = 0; ki < K; ki++) {
          const int *kI = &kIndices[ki * 3];
          rk[ki] += C[0][kI[0]] * C[1][kI[1]] * C[2][kI[2]];
        }
        FillC(P(0, slice, ptcl), C);
        for (int ki = 0; ki < K; ki++) {
          const int *kI = &kIndices[ki * 3];
          rk[ki] -= C[0][kI[0]] * C[1][kI[1]] * C[2][kI[2]];
        }
      }
    }
  }
  void UpdateRho_ksAll() {  // PathClass.cc:710-718
    int saved = mode;
    mode = 0;
    for (int slice = 0; slice < NumSlices; slice++) CalcRho_ks_Fast(slice);
    Rho_k[1] = Rho_k[0];
    mode = saved;
  }
  // LongRangeClass::SingleAction (LongRangeClass.cc:273-371), one species
  double LongRangeSingle(int slice1, int slice2, const int *changed, int n, int level) {
    if (mode == 1) UpdateRho_ks(slice1, slice2, changed, n, level);
    int skip = 1 << level, K = nk();
    double homo = 0.0, background = 0.0, k0Homo = 0.0;
    for (int slice = slice1; slice <= slice2; slice += skip) {
      double factor = ((slice == slice1) || (slice == slice2)) ? 0.5 : 1.0;
      if (pa->IsLongRange()) {
        const std::complex<double> *rk = &Rho_k[mode][(size_t)slice * K];
        for (int ki = 0; ki < K; ki++) {
          double rhok2 = rk[ki].real() * rk[ki].real() + rk[ki].imag() * rk[ki].imag();
          homo += factor * 0.5 * 2.0 * rhok2 * Ulong_k[(size_t)level * K + ki];
        }
      }
      homo -= factor * 0.5 * N * Ulong_r0[level];
      background -= factor * 0.5 * N * N * Ushort_k0[level];
      k0Homo += factor * 0.5 * N * N * Ulong_k0[level];
    }
    double U = homo;
    if (UseBackground)
      U += background;
    else
      U += k0Homo;
    return U;
  }
  // ---- DavidLongRangeClassYk (PIMC++/src/Actions/DavidLongRangeClassYk.cc) ----
  // uk, duk and Vlong_k per k-vector from the squarer's k-space table
  // uk_long(k): BuildRPA_SingleType (:76-126) for one pair type (rpa), else
  // Build_MultipleSpecies (:38-74).  A k-vector takes the table entry whose
  // k equals its |k| within 1e-10; one without such an entry is an error
  // here (the reference leaves it at -1 / unset).
  std::vector<double> YkU, YkDU, YkV;
  int SetYk(int nkv, const double *kvals, const double *uk_long, int rpa) {
    const int K = nk();
    double vol = 1.0;
    for (int dim = 0; dim < 3; dim++) vol *= Box[dim];
    YkU.assign(K, -1.0);
    YkDU.assign(K, 0.0);
    YkV.assign(K, 0.0);
    std::vector<char> set(K, 0);
    const double ncomps = N;
    for (int i = 0; i < nkv; i++) {
      const double k = kvals[i];
      double u = 0.0, du = 0.0, v = uk_long[i] / vol;
      if (rpa) {
        if (std::fabs(k) < 1e-10) continue;  // yk_zero: not used by the action
        const double arg = 1.0 + ncomps * 2.0 * uk_long[i] / (lambda * k * k * vol);
        const double theta = 0.5 * k * k * lambda * tau;
        double q, sv, tn;
        if (arg < 0) {
          q = sqrt(-arg);
          tn = tan(q * theta);
          sv = q * (1 - q * tn) / (q + tn);
        } else if (arg == 0) {
          sv = 1.0 / (1.0 + theta);
        } else {
          q = sqrt(arg);
          tn = tanh(theta * q);
          sv = q * (1.0 + q * tn) / (q + tn);
        }
        u = (-1.0 + sv) / ncomps;
        du = uk_long[i] / vol - lambda * k * k * u * (1.0 + 0.5 * ncomps * u);
      } else {
        u = v * tau;
        du = v;
      }
      for (int j = 0; j < K; j++) {
        const double *kv = &kVecs[(size_t)j * 3];
        if (std::fabs(sqrt(kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2]) - k) < 1e-10) {
          YkU[j] = u;
          YkDU[j] = du;
          YkV[j] = v;
          set[j] = 1;
        }
      }
    }
    for (int j = 0; j < K; j++)
      if (!set[j]) return -1;
    return 0;
  }
  // SingleAction (:230-323): on NEW, rho_k updated over the window's
  // interior (the whole path: [slice1, slice2 - skip]); then
  // sum_k sum_slices |rho_k|^2 uk with weight 1, over [slice1 + skip,
  // slice2 - skip] (the whole path: [slice1, slice2 - skip]).  No active
  // particle: no species, 0.
  double YkSingle(int slice1, int slice2, const int *changed, int n, int level) {
    const int skip = 1 << level, K = nk();
    const bool inclusive = !(slice1 == 0 && slice2 == NumSlices - 1);
    const int startSlice = inclusive ? slice1 + skip : slice1, endSlice = slice2 - skip;
    if (mode == 1 && startSlice <= endSlice) UpdateRho_ks(startSlice, endSlice, changed, n, level);
    if (n == 0) return 0.0;
    double total = 0.0;
    for (int ki = 0; ki < K; ki++)
      for (int slice = startSlice; slice <= endSlice; slice += skip) {
        const std::complex<double> z = Rho_k[mode][(size_t)slice * K + ki];
        total += 1.0 * (z.real() * z.real() + z.imag() * z.imag()) * YkU[ki];
      }
    return total;
  }
  // d_dBeta (:327-363) and V (:367-389): every slice of [slice1, slice2]
  // recomputed, weight 1/2 at both ends, with duk or Vlong_k.
  double YkSum(int slice1, int slice2, const std::vector<double> &w) {
    const int K = nk();
    double total = 0.0;
    for (int slice = slice1; slice <= slice2; slice++) {
      double sliceTotal = 0.0;
      const double factor = ((slice == slice1) || (slice == slice2)) ? 0.5 : 1.0;
      CalcRho_ks_Fast(slice);
      for (int ki = 0; ki < K; ki++) {
        const std::complex<double> z = Rho_k[mode][(size_t)slice * K + ki];
        sliceTotal += factor * (z.real() * z.real() + z.imag() * z.imag()) * w[ki];
      }
      total += sliceTotal;
    }
    return total;
  }
  // LongRangeClass::d_dBeta (LongRangeClass.cc:374-442), one species
  double LongRangeDBeta(int slice1, int slice2, int level) {
    int skip = 1 << level, K = nk();
    double homo = 0.0, background = 0.0, k0Homo = 0.0;
    for (int slice = slice1; slice <= slice2; slice += skip) {
      double factor = ((slice == slice1) || (slice == slice2)) ? 0.5 : 1.0;
      CalcRho_ks_Fast(slice);
      if (pa->IsLongRange()) {
        const std::complex<double> *rk = &Rho_k[mode][(size_t)slice * K];
        for (int ki = 0; ki < K; ki++) {
          double rhok2 = rk[ki].real() * rk[ki].real() + rk[ki].imag() * rk[ki].imag();
          homo += factor * 0.5 * 2.0 * rhok2 * dUlong_k[(size_t)level * K + ki];
        }
      }
      homo -= factor * 0.5 * N * dUlong_r0[level];
      background -= factor * 0.5 * N * N * dUshort_k0[level];
      k0Homo += factor * 0.5 * N * N * dUlong_k0[level];
    }
    double dU = homo;
    if (UseBackground)
      dU += background;
    else
      dU += k0Homo;
    return dU;
  }

  // ---- Bisection ----
  // BisectionStageClass::Sample (BisectionStage.cc:128-289), no correlated sampling
  double Sample(int slice1, int bisectionLevel, int ptcl) {
    int skip = 1 << (bisectionLevel + 1);
    double levelTau = 0.5 * tau * skip;
    int slice2 = slice1 + (1 << NumLevels);
    double logSampleProb = 0.0, logOldSampleProb = 0.0;
    double sigma2 = (1.0 * lambda * levelTau);
    double sigma = sqrt(sigma2);
    double prefactorOfSampleProb = 0.0;
    for (int slice = slice1; slice < slice2; slice += skip) {
      mode = 0;
      dVec rdiffOld, rbarOld, DeltaOld;
      const double *rOld = P(slice, ptcl);
      Velocity(slice, slice + skip, ptcl, rdiffOld);
      for (int i = 0; i < 3; i++) rbarOld[i] = rOld[i] + 0.5 * rdiffOld[i];
      const double *rppOld = P(slice + (skip >> 1), ptcl);
      for (int i = 0; i < 3; i++) DeltaOld[i] = rppOld[i] - rbarOld[i];
      PutInBox(DeltaOld);
      mode = 1;
      dVec rdiff, rbar, Delta;
      const double *r = P(slice, ptcl);
      Velocity(slice, slice + skip, ptcl, rdiff);
      for (int i = 0; i < 3; i++) rbar[i] = r[i] + 0.5 * rdiff[i];
      for (int i = 0; i < 3; i++) Delta[i] = rng.LocalGaussian(sigma);
      PutInBox(Delta);
      double GaussProd = 1.0, GaussProdOld = 1.0;
      for (int dim = 0; dim < 3; dim++) {
        double GaussSum = 0.0, GaussSumOld = 0.0;
        for (int image = -NumImages; image <= NumImages; image++) {
          double dist = Delta[dim] + (double)image * Box[dim];
          double distOld = DeltaOld[dim] + (double)image * Box[dim];
          GaussSum += exp(-0.5 * dist * dist / sigma2);
          GaussSumOld += exp(-0.5 * distOld * distOld / sigma2);
        }
        GaussProd *= GaussSum;
        GaussProdOld *= GaussSumOld;
      }
      logOldSampleProb += prefactorOfSampleProb + log(GaussProdOld);
      logSampleProb += prefactorOfSampleProb + log(GaussProd);
      double *rpp = P(1, slice + (skip >> 1), ptcl);
      for (int i = 0; i < 3; i++) rpp[i] = rbar[i] + Delta[i];
    }
    return -logSampleProb + logOldSampleProb;
  }
  // StageClass::StageAction (StageClass.cc:124-136) with the action list of
  // BisectionBlockClass::Read (BisectionBlock.cc:66-120): Kinetic, then
  // ShortRange (HigherLevelActions / SamplingActions), then LongRange at the
  // lowest level.
  double StageAction(int slice1, int slice2, int ptcl, int level) {
    double Total = 0.0;
    Total += KineticSingle(slice1, slice2, &ptcl, 1, level);
    if (level == 0 || SRHigher) Total += ShortRangeSingle(slice1, slice2, &ptcl, 1, level);
    if (level == 0 && UseLongRange && nk() > 0) Total += LongRangeSingle(slice1, slice2, &ptcl, 1, level);
    return Total;
  }
  // One MultiStageClass::MakeMove (MultiStage.cc:42-86) for a fixed slice window.
  void MakeMove(int slice1, int slice2, OracleMoveRecord *rec) {
    // NoPermuteStageClass::Attempt chooses the particle (NoPermuteClass.cc:26-68)
    int ptcl = rng.LocalInt(N);
    rec->slice1 = slice1;
    rec->ptcl = ptcl;
    rec->accepted = 0;
    rec->stages_passed = 0;
    for (int i = 0; i < 8; i++) rec->dS[i] = rec->log_sample_ratio[i] = 0.0;
    double prevActionChange = 0.0;
    bool toAccept = true;
    int si = 0;
    for (int level = NumLevels - 1; level >= 0 && toAccept; level--, si++) {
      // LocalStageClass::Attempt (StageClass.cc:49-95)
      mode = 1;
      double logSampleRatio = Sample(slice1, level, ptcl);
      mode = 0;
      double oldAction = StageAction(slice1, slice2, ptcl, level);
      mode = 1;
      double newAction = StageAction(slice1, slice2, ptcl, level);
      double currActionChange = newAction - oldAction;
      double logAcceptProb = logSampleRatio - currActionChange + prevActionChange;
      double ran_number = rng.Local();
      toAccept = logAcceptProb >= log(ran_number);
      if (si < 8) {
        rec->dS[si] = currActionChange;
        rec->log_sample_ratio[si] = logSampleRatio;
      }
      if (toAccept) rec->stages_passed++;
      prevActionChange = currActionChange;
    }
    if (toAccept) {
      // Concurrent windows share their end slices with the neighbouring
      // windows; those slices never move, and the schedule leaves them as
      // they are (the reference's PutInBoxFast of an unmoved end slice only
      // re-wraps its coordinates).
      if (window_mode)
        AcceptCopy(slice1 + 1, slice2 - 1, ptcl);
      else
        AcceptCopy(slice1, slice2, ptcl);
      rec->accepted = 1;
    } else {
      RejectCopy(slice1, slice2, ptcl);
    }
  }
  // PathClass::AcceptCopy (PathClass.cc:797-863), no worms/permutations/open paths
  void AcceptCopy(int s1, int s2, int ptcl) {
    for (int slice = s1; slice <= s2; slice++) PutInBoxFast(P(1, slice, ptcl));
    for (int slice = s1; slice <= s2; slice++) memcpy(P(0, slice, ptcl), P(1, slice, ptcl), 3 * sizeof(double));
    int K = nk();
    if (K > 0)
      for (int slice = s1; slice <= s2; slice++)
        for (int ki = 0; ki < K; ki++) Rho_k[0][(size_t)slice * K + ki] = Rho_k[1][(size_t)slice * K + ki];
  }
  // PathClass::RejectCopy (PathClass.cc:865-899)
  void RejectCopy(int s1, int s2, int ptcl) {
    for (int slice = s1; slice <= s2; slice++) memcpy(P(1, slice, ptcl), P(0, slice, ptcl), 3 * sizeof(double));
    int K = nk();
    if (K > 0)
      for (int slice = s1; slice <= s2; slice++)
        for (int ki = 0; ki < K; ki++) Rho_k[1][(size_t)slice * K + ki] = Rho_k[0][(size_t)slice * K + ki];
  }
  // BisectionBlockClass::MakeMove (BisectionBlock.cc:380-451) with
  // ChooseTimeSlices (:310-378), no reference slice.
  // Concurrent-window schedule (the CUDA library's PIMC_SCHEDULE_WINDOWS),
  // replayed sequentially: round r draws o = floor(Common() * 2^L) at
  // Common-stream index r and runs one block per window [o + w 2^L, ...],
  // window w drawing from its own Local stream.  The windows commute, so the
  // order here is immaterial.  With P proposal slots per window
  // (PIMC_SCHEDULE_PROPOSALS) every step of a window is slot 0, 1, ..., P-1
  // making one move each in that order, slot p drawing from Local stream
  // 0x100 + 64 p + w; records [window][step][slot].
  bool window_mode = false;  // MakeMove inside a concurrent-window round
  void MakeRound(OracleMoveRecord *recs, int P = 1) {
    const int span = 1 << NumLevels;
    const int W = std::min((NumSlices - 1) >> NumLevels, 64);
    const int o = (int)floor(philox_uniform(rng.seed, STREAM_COMMON, rounds) * span);
    rounds++;
    for (int w = 0; w < W; w++) {
      OracleMoveRecord *r = recs + (size_t)w * StepsPerBlock * P;
      const int slice1 = o + w * span;
      if (slice1 + span > NumSlices - 1) {
        for (int st = 0; st < StepsPerBlock * P; st++) {
          memset(&r[st], 0, sizeof(OracleMoveRecord));
          r[st].slice1 = -1;
          r[st].ptcl = -1;
        }
        continue;
      }
      for (int st = 0; st < StepsPerBlock; st++)
        for (int p = 0; p < P; p++) {
          std::swap(rng, wrng[(size_t)p * 64 + w]);
          window_mode = true;
          MakeMove(slice1, slice1 + span, &r[(size_t)st * P + p]);
          window_mode = false;
          std::swap(rng, wrng[(size_t)p * 64 + w]);
        }
    }
  }
  void MakeBlock(OracleMoveRecord *recs) {
    int sliceSep = 1 << NumLevels;
    int numLeft = NumSlices - sliceSep;
    int slice1 = rng.LocalInt(numLeft);
    int slice2 = slice1 + sliceSep;
    for (int step = 0; step < StepsPerBlock; step++) MakeMove(slice1, slice2, &recs[step]);
  }
};

extern "C" {

OracleSystem *oracle_system_create(int num_particles, int num_time_slices, const double *box, double tau,
                                   double lambda, int num_images) {
  OracleSystem *s = new OracleSystem();
  s->N = num_particles;
  s->NumSlices = num_time_slices;
  for (int i = 0; i < 3; i++) {
    s->Box[i] = box[i];
    s->BoxInv[i] = 1.0 / box[i];  // PathClass::SetBox (PathClass.h:582-590)
  }
  s->tau = tau;
  s->lambda = lambda;
  s->NumImages = num_images;
  for (int c = 0; c < 2; c++) s->path[c].assign((size_t)num_time_slices * num_particles * 3, 0.0);
  return s;
}
void oracle_system_free(OracleSystem *s) { delete s; }
void oracle_system_set_pa(OracleSystem *s, OraclePA *pa) { s->pa = pa; }
void oracle_system_set_path(OracleSystem *s, int copy, const double *path) {
  memcpy(s->path[copy].data(), path, s->path[copy].size() * sizeof(double));
}
void oracle_system_get_path(OracleSystem *s, int copy, double *path) {
  memcpy(path, s->path[copy].data(), s->path[copy].size() * sizeof(double));
}
void oracle_system_set_mode(OracleSystem *s, int copy) { s->mode = copy; }

int oracle_init_random_fixed(OracleSystem *s, uint64_t seed, double radius) {
  s->rng.seed = seed;
  s->rng.nworld = 0;
  int N = s->N;
  std::vector<double> R((size_t)N * 3);
  for (int i = 0; i < N; i++) {
    bool overlap = true;
    int tries = 0;
    while (overlap && tries < 1000) {
      tries++;
      for (int dim = 0; dim < 3; dim++) R[i * 3 + dim] = s->Box[dim] * (s->rng.World() - 0.5);
      overlap = false;
      for (int j = 0; j < i; j++) {
        dVec disp;
        for (int d = 0; d < 3; d++) disp[d] = R[j * 3 + d] - R[i * 3 + d];
        s->PutInBox(disp);
        overlap = overlap || ((disp[0] * disp[0] + disp[1] * disp[1] + disp[2] * disp[2]) < (4.0 * radius * radius));
      }
    }
    if (tries == 1000) return 1;
  }
  for (int c = 0; c < 2; c++)
    for (int slice = 0; slice < s->NumSlices; slice++)
      memcpy(s->P(c, slice, 0), R.data(), (size_t)N * 3 * sizeof(double));
  return 0;
}

// PathClass::ShiftPathData (PIMC++/src/PathClass.cc:1026-1110) on one
// process: sendProc == recvProc == 0, so the ring send/receive hands the
// send buffer straight back.  Permutations are the identity (MoveJoin no-op).
int oracle_shift_data(OracleSystem *s, int slicesToShift) {
  const int numPtcls = s->N, numSlices = s->NumSlices;
  if (!(abs(slicesToShift) < numSlices)) return 1;
  auto NEWp = [&](int slice, int ptcl) { return s->P(1, slice, ptcl); };
  auto OLDp = [&](int slice, int ptcl) { return s->P(0, slice, ptcl); };
  if (slicesToShift > 0) {
    for (int slice = numSlices - 1; slice >= slicesToShift; slice--)
      for (int ptcl = 0; ptcl < numPtcls; ptcl++) memcpy(NEWp(slice, ptcl), NEWp(slice - slicesToShift, ptcl), 24);
  } else {
    for (int slice = 0; slice < numSlices + slicesToShift; slice++)
      for (int ptcl = 0; ptcl < numPtcls; ptcl++) memcpy(NEWp(slice, ptcl), NEWp(slice - slicesToShift, ptcl), 24);
  }
  const int count = abs(slicesToShift) * numPtcls;
  std::vector<double> buffer((size_t)count * 3);
  int buffIndex = 0;
  int startSlice = slicesToShift > 0 ? numSlices - slicesToShift : 0;
  for (int slice = startSlice; slice < startSlice + abs(slicesToShift); slice++)
    for (int ptcl = 0; ptcl < numPtcls; ptcl++, buffIndex++)
      memcpy(&buffer[(size_t)buffIndex * 3], OLDp(slicesToShift > 0 ? slice - 1 : slice + 1, ptcl), 24);
  startSlice = slicesToShift > 0 ? 0 : numSlices + slicesToShift;
  buffIndex = 0;
  for (int slice = startSlice; slice < startSlice + abs(slicesToShift); slice++)
    for (int ptcl = 0; ptcl < numPtcls; ptcl++, buffIndex++)
      memcpy(NEWp(slice, ptcl), &buffer[(size_t)buffIndex * 3], 24);
  for (int slice = 0; slice < numSlices; slice++)
    for (int ptcl = 0; ptcl < numPtcls; ptcl++) memcpy(OLDp(slice, ptcl), NEWp(slice, ptcl), 24);
  return 0;
}

double oracle_shortrange_single(OracleSystem *s, int slice1, int slice2, const int *active, int n, int level) {
  return s->ShortRangeSingle(slice1, slice2, active, n, level);
}
double oracle_shortrange_single_abs(OracleSystem *s, int slice1, int slice2, const int *active, int n, int level) {
  return s->ShortRangeSingle(slice1, slice2, active, n, level, true);
}
double oracle_shortrange_dbeta(OracleSystem *s, int slice1, int slice2, int level) {
  return s->ShortRangeDBeta(slice1, slice2, level);
}
double oracle_kinetic_single(OracleSystem *s, int slice1, int slice2, const int *active, int n, int level) {
  return s->KineticSingle(slice1, slice2, active, n, level);
}
double oracle_kinetic_dbeta(OracleSystem *s, int slice1, int slice2, int level) {
  return s->KineticDBeta(slice1, slice2, level);
}

int oracle_setup_kvecs(OracleSystem *s, double kcutoff) {
  s->kCutoff = kcutoff;
  s->SetupkVecs3D();
  return s->nk();
}
int oracle_num_kvecs(OracleSystem *s) { return s->nk(); }
void oracle_get_kvecs(OracleSystem *s, double *kvecs, int *kindices) {
  memcpy(kvecs, s->kVecs.data(), s->kVecs.size() * sizeof(double));
  memcpy(kindices, s->kIndices.data(), s->kIndices.size() * sizeof(int));
}
void oracle_calc_rhok_all(OracleSystem *s) { s->UpdateRho_ksAll(); }
void oracle_update_rhok(OracleSystem *s, int slice1, int slice2, const int *active, int n, int level) {
  s->UpdateRho_ks(slice1, slice2, active, n, level);
}
void oracle_get_rhok(OracleSystem *s, int copy, double *out) {
  memcpy(out, s->Rho_k[copy].data(), s->Rho_k[copy].size() * sizeof(std::complex<double>));
}
void oracle_set_longrange(OracleSystem *s, int num_levels, const double *ulong_k, const double *ulong_r0,
                          const double *ushort_k0, const double *ulong_k0, const double *dulong_k,
                          const double *dulong_r0, const double *dushort_k0, const double *dulong_k0,
                          int use_background) {
  int K = s->nk();
  s->LRLevels = num_levels;
  s->Ulong_k.assign(ulong_k, ulong_k + (size_t)num_levels * K);
  s->dUlong_k.assign(dulong_k, dulong_k + (size_t)num_levels * K);
  s->Ulong_r0.assign(ulong_r0, ulong_r0 + num_levels);
  s->Ushort_k0.assign(ushort_k0, ushort_k0 + num_levels);
  s->Ulong_k0.assign(ulong_k0, ulong_k0 + num_levels);
  s->dUlong_r0.assign(dulong_r0, dulong_r0 + num_levels);
  s->dUshort_k0.assign(dushort_k0, dushort_k0 + num_levels);
  s->dUlong_k0.assign(dulong_k0, dulong_k0 + num_levels);
  s->UseBackground = use_background;
}
double oracle_longrange_single(OracleSystem *s, int slice1, int slice2, const int *active, int n, int level) {
  return s->LongRangeSingle(slice1, slice2, active, n, level);
}
double oracle_longrange_dbeta(OracleSystem *s, int slice1, int slice2, int level) {
  return s->LongRangeDBeta(slice1, slice2, level);
}

int oracle_set_yk(OracleSystem *s, int num_kvals, const double *kvals, const double *uk_long, int rpa) {
  return s->SetYk(num_kvals, kvals, uk_long, rpa);
}
void oracle_get_yk(OracleSystem *s, double *uk, double *duk, double *vlong) {
  memcpy(uk, s->YkU.data(), s->YkU.size() * sizeof(double));
  memcpy(duk, s->YkDU.data(), s->YkDU.size() * sizeof(double));
  memcpy(vlong, s->YkV.data(), s->YkV.size() * sizeof(double));
}
double oracle_yk_single(OracleSystem *s, int slice1, int slice2, const int *active, int n, int level) {
  return s->YkSingle(slice1, slice2, active, n, level);
}
double oracle_yk_dbeta(OracleSystem *s, int slice1, int slice2) { return s->YkSum(slice1, slice2, s->YkDU); }
double oracle_yk_v(OracleSystem *s, int slice1, int slice2) { return s->YkSum(slice1, slice2, s->YkV); }
void oracle_bisection_config(OracleSystem *s, int num_levels, int steps_per_block, int sr_higher, int use_longrange) {
  s->NumLevels = num_levels;
  s->StepsPerBlock = steps_per_block;
  s->SRHigher = sr_higher;
  s->UseLongRange = use_longrange;
}
void oracle_rng_seed(OracleSystem *s, uint64_t seed) {
  s->rng.seed = seed;
  s->rng.stream = STREAM_LOCAL;
  s->rng.nlocal = 0;
  s->rng.one_left = false;
  s->wrng.assign(64 * 16, Random());  // [slot][window]
  for (int w = 0; w < 64 * 16; w++) {
    s->wrng[w].seed = seed;
    s->wrng[w].stream = 0x100u + (uint32_t)w;
  }
  s->rounds = 0;
}
int oracle_run_windows(OracleSystem *s, int n_rounds, OracleMoveRecord *records) {
  const int W = std::min((s->NumSlices - 1) >> s->NumLevels, 64);
  for (int r = 0; r < n_rounds; r++) s->MakeRound(records + (size_t)r * W * s->StepsPerBlock);
  return W;
}
int oracle_run_proposals(OracleSystem *s, int n_rounds, int proposals, OracleMoveRecord *records) {
  const int W = std::min((s->NumSlices - 1) >> s->NumLevels, 64);
  if (proposals < 1 || proposals > 16) return -1;
  for (int r = 0; r < n_rounds; r++)
    s->MakeRound(records + (size_t)r * W * s->StepsPerBlock * proposals, proposals);
  return W;
}
int oracle_run_bisection(OracleSystem *s, int n_blocks, OracleMoveRecord *records) {
  for (int b = 0; b < n_blocks; b++) s->MakeBlock(records + (size_t)b * s->StepsPerBlock);
  return 0;
}
uint64_t oracle_rng_position(OracleSystem *s) { return s->rng.nlocal; }

// Ulong / dUlong quintic tables [levels][points][6] on [0, (points-1) delta];
// turns on Actions.UseLongRange (the short-range subtraction, and the long-range
// action in the bisection's lowest stage when k-vectors are set).
void oracle_set_ulong(OracleSystem *s, int levels, int points, double delta, const double *ulong,
                      const double *dulong) {
  s->ULongTab.assign(ulong, ulong + (size_t)levels * points * 6);
  s->dULongTab.assign(dulong, dulong + (size_t)levels * points * 6);
  s->ULongPoints = points;
  s->ULongDelta = delta;
  s->UseLongRange = 1;
}

// ActionsClass::Energy (ActionsClass.cc:812-871) on the OLD copy: out =
// {kinetic, dUShort, dULong, vShort, vLong (0), total per slice}
void oracle_energy(OracleSystem *s, double *out) {
  const int M = s->NumSlices - 1;
  const int mode = s->mode;
  s->mode = 0;
  const double kinetic = s->KineticDBeta(0, M, 0);
  const double dUShort = s->ShortRangeDBeta(0, M, 0);
  const double dULong = s->LRLevels > 0 ? s->LongRangeDBeta(0, M, 0) : 0.0;
  double vShort = 0.0;
  for (int slice = 0; slice <= M; slice++) {
    double factor = ((slice == 0) || (slice == M)) ? 0.5 : 1.0;
    vShort += factor * s->VSlice(slice);
  }
  s->mode = mode;
  out[0] = kinetic;
  out[1] = dUShort;
  out[2] = dULong;
  out[3] = vShort;
  out[4] = 0.0;
  out[5] = (kinetic + dUShort + dULong) / (double)M;  // ObservableEnergy.cc:45-73
}

// PairCorrelationClass::Accumulate (ObservableCorrelation.cc:191-207), one
// species, on the OLD copy, into hist[num_points-1] on the LinearGrid
// {start, end, num_points} (Grid.h:81-95).
void oracle_gofr_accumulate(OracleSystem *s, double start, double end, int num_points, uint64_t *hist) {
  const double delta = (end - start) / (double)(num_points - 1);
  const double deltainv = 1.0 / delta;
  const int mode = s->mode;
  s->mode = 0;
  for (int slice = 0; slice < s->NumSlices - 1; slice++)
    for (int ptcl1 = 0; ptcl1 < s->N; ptcl1++)
      for (int ptcl2 = ptcl1 + 1; ptcl2 < s->N; ptcl2++) {
        const double dist = s->Dist1(slice, ptcl1, ptcl2);
        if (dist < end) {
          int index = (int)nearbyint((dist - start) * deltainv - 0.5);
          // The reference indexes without a check; a grid starting above 0
          // gives negative bins for closer pairs, which are skipped here.
          if (index >= 0 && index < num_points - 1) hist[index]++;
        }
      }
  s->mode = mode;
}

}  // extern "C"

// Host-side setup of the pair-action tables, in FP64, once per context —
// the work PIMC++ does at Read/Init time before any move runs:
//   * grids (Common/Splines/Grid.h:69-136, :519-575),
//   * cubic-spline second derivatives (Common/Splines/CubicSpline.cc:77-128),
//   * tricubic first-derivative fill (Common/Splines/MyTricubicSpline.cc:19-101),
//   * the ASCII squarer .dm reader (Common/PairAction/DavidPAClass.cc:635-912).
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <new>
#include <stdexcept>
#include <sstream>
#include <string>
#include <vector>

#include "pimc_internal.h"

namespace pimc {

void HostGrid::init_linear(double s, double e, int num) {
  type = PIMC_GRID_LINEAR;
  start = s;
  end = e;
  n = num;
  delta = (end - start) / (double)(n - 1);
  deltainv = 1.0 / delta;
  x.resize(n);
  for (int i = 0; i < n; i++) x[i] = start + (double)i * delta;
}

void HostGrid::init_log(double r0_, double spacing_, int num) {
  type = PIMC_GRID_LOG;
  n = num;
  r0 = r0_;
  spacing = spacing_;
  log_spacing = std::log(spacing);
  start = r0;
  end = r0 * std::pow(spacing, (double)n - 1);
  x.resize(n);
  for (int i = 0; i < n; i++) x[i] = r0 * std::pow(spacing, (double)i);
}

// Second derivatives of the cubic spline through column `col` of y
// ([point][ncols]); start_deriv/end_deriv > 0.99e30 select the natural end.
void spline_second_derivs(const HostGrid &g, const double *y, int ncols, int col, double start_deriv,
                          double end_deriv, double *d2y) {
  const int n = g.n;
  const std::vector<double> &x = g.x;
  auto Y = [&](int j) { return y[(size_t)j * ncols + col]; };
  auto D = [&](int j) -> double & { return d2y[(size_t)j * ncols + col]; };
  std::vector<double> u(n);
  if (start_deriv > 0.99e30) {
    D(0) = 0.0;
    u[0] = 0.0;
  } else {
    D(0) = -0.5;
    u[0] = (3.0 / (x[1] - x[0])) * ((Y(1) - Y(0)) / (x[1] - x[0]) - start_deriv);
  }
  D(n - 1) = 0.0;
  for (int j = 1; j < n - 1; j++) {
    double sig = (x[j] - x[j - 1]) / (x[j + 1] - x[j - 1]);
    double p = sig * D(j - 1) + 2.0;
    D(j) = (sig - 1.0) / p;
    double slope_hi = (Y(j + 1) - Y(j)) / (x[j + 1] - x[j]);
    double slope_lo = (Y(j) - Y(j - 1)) / (x[j] - x[j - 1]);
    u[j] = (6.0 * (slope_hi - slope_lo) / (x[j + 1] - x[j - 1]) - sig * u[j - 1]) / p;
  }
  double un = 0.0, qn = 0.0;
  if (!(end_deriv > 0.99e30)) {
    qn = 0.5;
    un = (3.0 / (x[n - 1] - x[n - 2])) * (end_deriv - (Y(n - 1) - Y(n - 2)) / (x[n - 1] - x[n - 2]));
  }
  D(n - 1) = (un - qn * u[n - 2]) / (qn * D(n - 2) + 1.0);
  for (int k = n - 2; k >= 0; k--) D(k) = D(k) * D(k + 1) + u[k];
}

namespace {
// First derivative along one axis of component `src` into component `dst`
// by the tridiagonal solve with end slopes 1.5*delta/h.
void fill_axis(const HostGrid &g, int axis, int nx, int ny, int nz, int src, int dst, double *F) {
  const int n = g.n;
  const int o1 = axis == 0 ? ny : nx, o2 = axis == 2 ? ny : nz;
  std::vector<double> mu(n);
  for (int a = 0; a < o1; a++)
    for (int b = 0; b < o2; b++) {
      auto at = [&](int j, int c) -> double & {
        size_t node = axis == 0 ? ((size_t)j * ny + a) * nz + b
                      : axis == 1 ? ((size_t)a * ny + j) * nz + b
                                  : ((size_t)a * ny + b) * nz + j;
        return F[node * 8 + c];
      };
      const std::vector<double> &x = g.x;
      at(0, dst) = 1.5 * (at(1, src) - at(0, src)) / (x[1] - x[0]);
      at(n - 1, dst) = 1.5 * (at(n - 1, src) - at(n - 2, src)) / (x[n - 1] - x[n - 2]);
      mu[0] = 0.5;
      for (int j = 1; j < n - 1; j++) {
        double lambda = 0.5 * (x[j + 1] - x[j]) / (x[j + 1] - x[j - 1]);
        mu[j] = 0.5 - lambda;
        at(j, dst) = 3.0 * (lambda * (at(j, src) - at(j - 1, src)) / (x[j] - x[j - 1]) +
                            mu[j] * (at(j + 1, src) - at(j, src)) / (x[j + 1] - x[j]));
        double cj = 1.0 - lambda * mu[j - 1];
        at(j, dst) -= lambda * at(j - 1, dst);
        mu[j] /= cj;
        at(j, dst) /= cj;
      }
      {
        int j = n - 1;
        double lambda = 0.5;
        mu[j] = 0.5 - lambda;
        at(j, dst) = 3.0 * (lambda * (at(j, src) - at(j - 1, src)) / (x[j] - x[j - 1]));
        double cj = 1.0 - lambda * mu[j - 1];
        at(j, dst) -= lambda * at(j - 1, dst);
        mu[j] /= cj;
        at(j, dst) /= cj;
      }
      for (int j = n - 2; j >= 0; j--) at(j, dst) -= mu[j] * at(j + 1, dst);
    }
}
}  // namespace

// values [nx][ny][nz] -> F [nx][ny][nz][8] (F, Fx, Fy, Fz, Fxy, Fxz, Fyz, Fxyz)
void tricubic_fill(const HostGrid &gx, const HostGrid &gy, const HostGrid &gz, const double *values, double *F) {
  const int nx = gx.n, ny = gy.n, nz = gz.n;
  const size_t nodes = (size_t)nx * ny * nz;
  for (size_t i = 0; i < nodes; i++) {
    F[i * 8] = values[i];
    for (int c = 1; c < 8; c++) F[i * 8 + c] = 0.0;
  }
  fill_axis(gx, 0, nx, ny, nz, 0, 1, F);  // dF/dx
  fill_axis(gy, 1, nx, ny, nz, 0, 2, F);  // dF/dy
  fill_axis(gz, 2, nx, ny, nz, 0, 3, F);  // dF/dz
  fill_axis(gy, 1, nx, ny, nz, 1, 4, F);  // d2F/dxdy
  fill_axis(gz, 2, nx, ny, nz, 1, 5, F);  // d2F/dxdz
  fill_axis(gz, 2, nx, ny, nz, 2, 6, F);  // d2F/dydz
  fill_axis(gz, 2, nx, ny, nz, 4, 7, F);  // d3F/dxdydz
}

void build_david(DavidTables &t, const double *ukj, const double *dukj) {
  const size_t per = (size_t)t.grid.n * t.ncols;
  t.uy.assign(ukj, ukj + per * t.num_tau);
  t.duy.assign(dukj, dukj + per * t.num_tau);
  t.ud2.assign(t.uy.size(), 0.0);
  t.dud2.assign(t.duy.size(), 0.0);
  for (int lev = 0; lev < t.num_tau; lev++)
    for (int c = 0; c < t.ncols; c++) {
      // start derivative 5e30 (natural), end derivative 0 (DavidPAClass.cc:760-763)
      spline_second_derivs(t.grid, t.uy.data() + per * lev, t.ncols, c, 5.0e30, 0.0, t.ud2.data() + per * lev);
      spline_second_derivs(t.grid, t.duy.data() + per * lev, t.ncols, c, 5.0e30, 0.0, t.dud2.data() + per * lev);
    }
}

// ---------------------------------------------------------------------------
// ASCII squarer .dm reader.  Field rules (DavidPAClass.h:186-290): a line is
// found by substring; integers are read from the first digit or '-' on;
// doubles from the first digit, '-' or '.'; words are space-delimited.
// ---------------------------------------------------------------------------
namespace {
struct LineCursor {
  std::string s;
  std::string word() {
    size_t c = 0;
    while (c < s.size() && s[c] == ' ') c++;
    size_t b = c;
    while (c < s.size() && s[c] != ' ') c++;
    std::string w = s.substr(b, c - b);
    s.erase(0, c);
    return w;
  }
  long integer() {
    size_t i = 0;
    while (i < s.size() && !((s[i] >= '0' && s[i] <= '9') || s[i] == '-')) i++;
    s.erase(0, i);
    char *end = nullptr;
    long v = std::strtol(s.c_str(), &end, 10);
    s.erase(0, end - s.c_str());
    return v;
  }
  double real() {
    size_t i = 0;
    while (i < s.size() && !((s[i] >= '0' && s[i] <= '9') || s[i] == '-' || s[i] == '.')) i++;
    s.erase(0, i);
    char *end = nullptr;
    double v = std::strtod(s.c_str(), &end);
    s.erase(0, end - s.c_str());
    return v;
  }
};

bool find_line(std::istream &in, const char *key, LineCursor &lc) {
  std::string line;
  while (std::getline(in, line))
    if (line.find(key) != std::string::npos) {
      lc.s = line;
      return true;
    }
  return false;
}

// Sizes a squarer file may declare: anything larger is a damaged file, not
// a table (the reference's reader would allocate it or read past its arrays).
constexpr long kMaxDmGrid = 1L << 24;     // grid points
constexpr long kMaxDmColumns = 4096;      // u_kj columns of one fit
constexpr long kMaxDmTau = 64;            // tau values
constexpr long kMaxDmValues = 1L << 27;   // values in one table block

struct FitBlock {
  int ng = 0, nukj = 0, ntau = 0, nmax = 0, derv = 0;
  double tau_min = 0;
  HostGrid grid;
  std::vector<double> v;  // [grid][ukj][tau]
};

bool read_block(std::istream &in, FitBlock &b, std::string &err) {
  LineCursor lc;
  do {
    if (!find_line(in, "RANK", lc)) { err = "missing RANK 3 block"; return false; }
  } while (lc.integer() != 3);
  const long ng = lc.integer(), nukj = lc.integer(), ntau = lc.integer();
  if (ng < 2 || ng > kMaxDmGrid || nukj < 1 || nukj > kMaxDmColumns || ntau < 1 || ntau > kMaxDmTau ||
      ng * nukj * ntau > kMaxDmValues) {
    err = "RANK 3 block sizes out of range";
    return false;
  }
  b.ng = (int)ng;
  b.nukj = (int)nukj;
  b.ntau = (int)ntau;
  if (!find_line(in, "GRID 1", lc)) { err = "missing GRID 1"; return false; }
  lc.word(); lc.word();
  std::string type = lc.word();
  double g0 = lc.real(), g1 = lc.real();
  if (!(g1 > g0) || !std::isfinite(g0) || !std::isfinite(g1) || (type == "LOG" && !(g0 > 0.0))) {
    err = "bad r grid bounds";
    return false;
  }
  if (type == "LINEAR") {
    b.grid.init_linear(g0, g1, b.ng);
  } else if (type == "LOG") {
    b.grid.init_log(g0, std::pow(g1 / g0, 1.0 / (b.ng - 1.0)), b.ng);
  } else {
    err = "unrecognised grid type " + type;
    return false;
  }
  if (!find_line(in, "GRID   3", lc)) { err = "missing tau grid"; return false; }
  lc.word(); lc.word();
  if (lc.word() != "LOG") { err = "tau grid is not LOG"; return false; }
  b.tau_min = lc.real();
  double tau_max = lc.real();
  if (!(b.tau_min > 0.0) || !(tau_max >= b.tau_min) || !std::isfinite(tau_max)) {
    err = "bad tau grid bounds";
    return false;
  }
  int ntau_calc = (int)std::floor(std::log(tau_max / b.tau_min) / std::log(2.0) + 0.5 + 1.0);
  if (ntau_calc != b.ntau) { err = "tau count inconsistent with tau grid"; return false; }
  if (!find_line(in, "BEGIN density matrix table", lc)) { err = "missing table"; return false; }
  b.nmax = (int)lc.integer();
  b.derv = (int)lc.integer();
  b.v.assign((size_t)b.ng * b.nukj * b.ntau, 0.0);
  for (int t = 0; t < b.ntau; t++)
    for (int u = 0; u < b.nukj; u++)
      for (int g = 0; g < b.ng; g++) {
        double val;
        if (!(in >> val)) { err = "table truncated"; return false; }
        b.v[((size_t)g * b.nukj + u) * b.ntau + t] = val;
      }
  return true;
}
}  // namespace

static int read_dm_file_checked(const char *path, double desired_tau, int num_terms, DavidTables &out,
                                std::string &err) {
  std::ifstream in(path);
  if (!in) {
    err = std::string("cannot open ") + path;
    return PIMC_E_FILE;
  }
  LineCursor lc;
  if (!find_line(in, "SQUARER", lc)) { err = "no SQUARER line"; return PIMC_E_FILE; }
  for (int i = 0; i < 4; i++) lc.word();
  const long num_fits_l = lc.integer();
  if (num_fits_l < 0 || num_fits_l > 64) { err = "bad number of fits"; return PIMC_E_FILE; }
  const int num_fits = (int)num_fits_l;
  if (!find_line(in, "RANK", lc)) { err = "no potential block"; return PIMC_E_FILE; }
  lc.word(); lc.word();
  const long npot_l = lc.integer();
  if (npot_l < 2 || npot_l > kMaxDmGrid) { err = "bad potential size"; return PIMC_E_FILE; }
  const int npot = (int)npot_l;
  std::vector<double> potential(npot);
  if (!find_line(in, "potential", lc)) { err = "no potential table"; return PIMC_E_FILE; }
  for (int i = 0; i < npot; i++)
    if (!(in >> potential[i])) { err = "potential truncated"; return PIMC_E_FILE; }

  std::vector<double> tables[2];
  HostGrid grids[2];
  int nukj = -1, ntau = -1;
  int tau_pos = -1;
  for (int pass = 0; pass < 2; pass++) {
    for (int fit = 0; fit <= num_fits; fit++) {
      FitBlock b;
      if (!read_block(in, b, err)) return PIMC_E_FILE;
      if (b.derv != pass + 1) { err = "unexpected derivative order"; return PIMC_E_FILE; }
      if (b.ng != npot) { err = "grid size differs from potential"; return PIMC_E_FILE; }
      if (pass == 1) {
        double tau = b.tau_min;
        for (int i = 0; i < b.ntau; i++) {
          if (std::fabs(tau - desired_tau) < 1e-4) tau_pos = i;
          tau = tau * 2;
        }
      }
      if (b.nmax != 2) continue;  // only the NMax==2 fit builds the splines
      const int ncol = b.nukj + 1;
      std::vector<double> &t = tables[pass];
      t.assign((size_t)b.ntau * b.ng * ncol, 0.0);
      for (int lev = 0; lev < b.ntau; lev++)
        for (int g = 0; g < b.ng; g++) {
          double *row = &t[((size_t)lev * b.ng + g) * ncol];
          row[0] = potential[g];
          for (int u = 0; u < b.nukj; u++) row[1 + u] = b.v[((size_t)g * b.nukj + u) * b.ntau + lev];
          if (g == b.ng - 1)
            for (int c = 0; c < ncol; c++) row[c] = 0.0;  // last grid row zeroed
        }
      grids[pass] = b.grid;
      nukj = b.nukj;
      ntau = b.ntau;
    }
  }
  if (tables[0].empty() || tables[1].empty()) { err = "no NMax==2 fit"; return PIMC_E_FILE; }
  if (tau_pos < 0) { err = "desired tau not on the file's tau grid"; return PIMC_E_FILE; }
  out.grid = grids[0];
  out.ncols = nukj + 1;
  out.num_tau = ntau;
  out.tau_pos = tau_pos;
  out.num_terms = num_terms;
  build_david(out, tables[0].data(), tables[1].data());
  return PIMC_OK;
}

// No exception crosses the C ABI: a file that still makes the reader throw
// (an allocation it cannot get) is reported as a status.
int read_dm_file(const char *path, double desired_tau, int num_terms, DavidTables &out, std::string &err) {
  try {
    return read_dm_file_checked(path, desired_tau, num_terms, out, err);
  } catch (const std::bad_alloc &) {
    err = std::string("out of host memory reading ") + path;
    return PIMC_E_NOMEM;
  } catch (const std::exception &e) {
    err = std::string("reading ") + path + ": " + e.what();
    return PIMC_E_FILE;
  }
}

}  // namespace pimc

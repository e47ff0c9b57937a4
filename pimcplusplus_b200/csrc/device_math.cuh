// Device-side restatement of the PIMC++ pair-action arithmetic, templated on
// the evaluation precision R (double for the plain path, float for the mixed
// path).  Wherever the result feeds a discrete choice (grid interval, image
// index) the arithmetic uses explicitly rounded intrinsics so no fused
// multiply-add changes the choice relative to the source-order evaluation.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "pimc_internal.h"

namespace pimc {

// ---- explicitly rounded arithmetic (no contraction) ----
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rint_r(double a) { return rint(a); }
__device__ __forceinline__ float rint_r(float a) { return rintf(a); }
__device__ __forceinline__ double log_r(double a) { return log(a); }
__device__ __forceinline__ float log_r(float a) { return logf(a); }
__device__ __forceinline__ double floor_r(double a) { return floor(a); }
__device__ __forceinline__ float floor_r(float a) { return floorf(a); }
__device__ __forceinline__ double sqrt_r(double a) { return sqrt(a); }
__device__ __forceinline__ float sqrt_r(float a) { return sqrtf(a); }
__device__ __forceinline__ double fabs_r(double a) { return fabs(a); }
__device__ __forceinline__ float fabs_r(float a) { return fabsf(a); }

// ---- Grid (Common/Splines/Grid.h:69-136 LinearGrid, :519-575 LogGrid) ----
// LinearGrid::ReverseMap = (int)nearbyint((r-Start)*deltainv - 0.5);
// LogGrid::ReverseMap = (int)floor(log(r/r0)/log(Spacing)).
template <typename R>
__device__ __forceinline__ int reverse_map(const DGrid<R> &g, R r) {
  if (g.type == PIMC_GRID_LINEAR) return (int)rint_r(rsub(rmul(rsub(r, g.start), g.deltainv), R(0.5)));
  return (int)floor_r(log_r(r / g.r0) / g.log_spacing);
}
// Grid node i: LinearGrid stores Start + (double)i*delta (Grid.h:93-95).
template <typename R>
__device__ __forceinline__ R grid_x(const DGrid<R> &g, int i) {
  if (g.type == PIMC_GRID_LINEAR) return radd(g.start, rmul((R)i, g.delta));
  return g.x[i];
}

// Interval of a cubic spline evaluation with the clamps of
// MultiCubicSpline::operator() (CubicSpline.h:485-501).
template <typename R>
struct SplineCell {
  int low, hi;
  R a, b, a3, b3, h26;
};
// Round to nearest even by the magic-constant addition (exact for
// |t| < 2^22 in FP32, 2^51 in FP64; larger |t| only feeds the clamps below,
// which send it to the first or last cell like the integer path does), and
// the integer of an integral value in [0, 2^22).  These keep the cell search
// on the FMA pipe instead of float-int conversions.
__device__ __forceinline__ float round_even_magic(float t) {
  return __fadd_rn(__fadd_rn(t, 12582912.0f), -12582912.0f);
}
__device__ __forceinline__ double round_even_magic(double t) {
  return __dadd_rn(__dadd_rn(t, 6755399441055744.0), -6755399441055744.0);
}
__device__ __forceinline__ int int_of_integral(float v) { return __float_as_int(__fadd_rn(v, 12582912.0f)) - 0x4B400000; }
__device__ __forceinline__ int int_of_integral(double v) {
  return (int)(__double_as_longlong(__dadd_rn(v, 6755399441055744.0)) - 0x4338000000000000LL);
}
__device__ __forceinline__ float fmax_r(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double fmax_r(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float fmin_r(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double fmin_r(double a, double b) { return fmin(a, b); }

template <typename R>
__device__ __forceinline__ SplineCell<R> spline_cell(const DGrid<R> &g, R x) {
  SplineCell<R> c;
  int low, hi;
  R xl, xh;
  if (g.type == PIMC_GRID_LINEAR) {
    // low = clamp(ReverseMap(x), 0, n-2), hi = low + 1, as integers held in R
    const R rm = round_even_magic(rsub(rmul(rsub(x, g.start), g.deltainv), R(0.5)));
    const R lowf = fmin_r(fmax_r(rm, R(0)), (R)(g.n - 2));
    low = int_of_integral(lowf);
    hi = low + 1;
    xl = radd(g.start, rmul(lowf, g.delta));
    xh = radd(g.start, rmul(radd(lowf, R(1)), g.delta));
  } else {
    hi = reverse_map(g, x) + 1;
    low = hi - 1;
    if (low < 0) { low = 0; hi = 1; }
    if (hi > (g.n - 1)) { hi = g.n - 1; low = hi - 1; }
    xl = grid_x(g, low);
    xh = grid_x(g, hi);
  }
  // A linear grid's cell width is delta (X(hi) - X(low) differs from it by a
  // rounding), so its inverse is the precomputed deltainv; a = 1 - b keeps the
  // two weights summing to one in either precision.
  const bool lin = g.type == PIMC_GRID_LINEAR;
  R h = lin ? g.delta : xh - xl;
  R hinv = lin ? g.deltainv : R(1.0) / h;
  c.b = (x - xl) * hinv;
  c.a = lin ? R(1.0) - c.b : (xh - x) * hinv;
  c.a3 = c.a * c.a * c.a - c.a;
  c.b3 = c.b * c.b * c.b - c.b;
  c.h26 = h * h * R(0.1666666666666666666);
  c.low = low;
  c.hi = hi;
  return c;
}
template <typename R>
__device__ __forceinline__ R spline_apply(const SplineCell<R> &c, R yl, R yh, R dl, R dh) {
  return c.a * yl + c.b * yh + (c.a3 * dl + c.b3 * dh) * c.h26;
}
// Column `col` of a [point][ncols] table pair.
template <typename R>
__device__ __forceinline__ R spline_col(const DGrid<R> &g, const R *__restrict__ y, const R *__restrict__ d2,
                                        int ncols, int col, R x) {
  SplineCell<R> c = spline_cell(g, x);
  return spline_apply(c, __ldg(&y[c.low * ncols + col]), __ldg(&y[c.hi * ncols + col]),
                      __ldg(&d2[c.low * ncols + col]), __ldg(&d2[c.hi * ncols + col]));
}

template <typename R>
struct Pair2;
template <>
struct Pair2<double> { typedef double2 T; };
template <>
struct Pair2<float> { typedef float2 T; };

// Column stored as interleaved (y, d2y) pairs, e.g. staged in shared memory.
template <typename R>
__device__ __forceinline__ R spline_pairs(const DGrid<R> &g, const typename Pair2<R>::T *tab, R x) {
  SplineCell<R> c = spline_cell(g, x);
  typename Pair2<R>::T lo = tab[c.low], hi = tab[c.hi];
  return spline_apply(c, lo.x, hi.x, lo.y, hi.y);
}

// ---- DavidPAClass::calcUsqzFast (DavidPAClass.cc:468-511) ----
// U plus the off-diagonal terms Ucof_kj(q) z^2j s^(2k-2j), k = 1..NumTerms,
// j = 0..k, added one by one in the reference's order.  Out of line: the
// diagonal-only tables never take it and the hot item loops stay compact.
// Arguments are plain values so that no parameter-space struct is copied to
// local memory for the call.
template <typename R>
__device__ __noinline__ R david_offdiag_add(DGrid<R> g, const R *y, const R *d2, int ncols, int num_terms, R U, R s2,
                                            R q, R z) {
  const R s = sqrt_r(s2);
  SplineCell<R> c = spline_cell(g, q);
  R zsquared = z * z;
  R ssquared = s * s;
  R ssquaredinverse = R(1.0) / ssquared;
  R Sto2k = ssquared;
  for (int k = 1; k <= num_terms; k++) {
    R Zto2j = 1;
    R currS = Sto2k;
    for (int j = 0; j <= k; j++) {
      int col = k * (k + 1) / 2 + j + 1;
      R Ucof = spline_apply(c, __ldg(&y[c.low * ncols + col]), __ldg(&y[c.hi * ncols + col]),
                            __ldg(&d2[c.low * ncols + col]), __ldg(&d2[c.hi * ncols + col]));
      U += Ucof * Zto2j * currS;
      Zto2j *= zsquared;
      currS = currS * ssquaredinverse;
    }
    Sto2k = Sto2k * ssquared;
  }
  return U;
}

// diag: column 1 of ukj(level+TauPos) as (y, d2y) pairs (global or shared).
template <typename R>
__device__ __forceinline__ R david_U(const DDavid<R> &d, const typename Pair2<R>::T *diag, R s2, R q, R z,
                                     int level) {
  level = level + d.tau_pos;
  const DGrid<R> &g = d.grid;
  R rmin = g.start;
  R r = q + R(0.5) * z;
  R rprime = q - R(0.5) * z;
  if (r > g.end) r = g.end;
  if (rprime > g.end) rprime = g.end;
  if ((rprime < rmin) || (r < rmin)) return spline_pairs(g, diag, rmin);
  R U = R(0.5) * (spline_pairs(g, diag, r) + spline_pairs(g, diag, rprime));
  if (d.num_terms > 0 && s2 > R(0) && q < g.end)
    U = david_offdiag_add<R>(g, d.uy + (size_t)level * g.n * d.ncols, d.ud2 + (size_t)level * g.n * d.ncols, d.ncols,
                             d.num_terms, U, s2, q, z);
  return U;
}

// ---- DavidPAClass::calcUsqz, dU output (DavidPAClass.cc:291-463) ----
template <typename R>
__device__ __forceinline__ R david_dU(const DDavid<R> &d, R s2, R q, R z, int level) {
  level = level + d.tau_pos;
  const DGrid<R> &g = d.grid;
  const R *uy = d.uy + (size_t)level * g.n * d.ncols;
  const R *ud2 = d.ud2 + (size_t)level * g.n * d.ncols;
  const R *dy = d.duy + (size_t)level * g.n * d.ncols;
  const R *dd2 = d.dud2 + (size_t)level * g.n * d.ncols;
  R rmin = g.start;
  R r = q + R(0.5) * z;
  R rprime = q - R(0.5) * z;
  if (r > g.end) r = g.end;
  if (rprime > g.end) rprime = g.end;
  if (rprime < rmin) rprime = rmin;
  if (r < rmin) r = rmin;
  R V = R(0.5) * (spline_col(g, uy, ud2, d.ncols, 0, r) + spline_col(g, uy, ud2, d.ncols, 0, rprime));
  R dU = R(0.5) * (spline_col(g, dy, dd2, d.ncols, 1, r) + spline_col(g, dy, dd2, d.ncols, 1, rprime));
  dU += V;
  if (d.num_terms > 0 && s2 > R(0) && q < g.end) {
    const R s = sqrt_r(s2);
    SplineCell<R> c = spline_cell(g, q);
    R zsquared = z * z;
    R ssquared = s * s;
    R ssquaredinverse = R(1.0) / ssquared;
    R Sto2k = ssquared;
    for (int k = 1; k <= d.num_terms; k++) {
      R Zto2j = 1;
      R currS = Sto2k;
      for (int j = 0; j <= k; j++) {
        int col = k * (k + 1) / 2 + j + 1;
        R dUcof = spline_apply(c, __ldg(&dy[c.low * d.ncols + col]), __ldg(&dy[c.hi * d.ncols + col]),
                               __ldg(&dd2[c.low * d.ncols + col]), __ldg(&dd2[c.hi * d.ncols + col]));
        dU += dUcof * Zto2j * currS;
        Zto2j *= zsquared;
        currS = currS * ssquaredinverse;
      }
      Sto2k = Sto2k * ssquared;
    }
  }
  return dU;
}

// ---- MyTricubicSpline::operator() (MyTricubicSpline.h:197-334) ----
// Hermite basis p1, p2, q1, q2 (MyTricubicSpline.h:38-45).
template <typename R>
__device__ __forceinline__ void hermite4(R t, R h, R out[4]) {
  R tm1 = t - R(1.0);
  out[0] = tm1 * tm1 * (R(1.0) + R(2.0) * t);
  out[1] = t * t * (R(3.0) - R(2.0) * t);
  out[2] = h * (t * tm1 * tm1);
  out[3] = h * (t * t * tm1);
}

// One node's 8 components by 256-bit read-only loads (sm_100: 32 bytes per
// thread per load).  The tables are cudaMalloc'ed (256-byte aligned) and
// every node starts at a multiple of 8 components, so a node is 64-byte
// (FP64) / 32-byte (FP32) aligned.  A cell's scattered gather is bound by
// the L1 requests of its loads, one per lane and load: 32-byte loads halve
// them against 16-byte ones.
template <typename R>
struct Node8;
template <>
struct Node8<double> {
  double v[8];
  __device__ __forceinline__ void load(const double *p) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
        : "l"(p));
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(v[4]), "=d"(v[5]), "=d"(v[6]), "=d"(v[7])
        : "l"(p + 4));
  }
};
template <>
struct Node8<float> {
  float v[8];
  __device__ __forceinline__ void load(const float *p) {
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
        : "l"(p));
  }
};

// F: [nx][ny][nz][8] with components F, Fx, Fy, Fz, Fxy, Fxz, Fyz, Fxyz.
// The cell's (x-node, y-node) pairs k = 2 dx + dy in [k0, k1) are summed, so
// lanes of a team can split one evaluation; [0, 4) is the whole spline.  The
// grids are linear: the cell widths are delta and u = (x - x0) deltainv.
template <typename R>
__device__ __forceinline__ R tricubic_eval(const R *__restrict__ F, const DGrid<R> &gx, const DGrid<R> &gy,
                                           const DGrid<R> &gz, R x, R y, R z, int k0 = 0, int k1 = 4) {
  int ix = reverse_map(gx, x), iy = reverse_map(gy, y), iz = reverse_map(gz, z);
  ix = max(0, ix); ix = min(ix, gx.n - 2);
  iy = max(0, iy); iy = min(iy, gy.n - 2);
  iz = max(0, iz); iz = min(iz, gz.n - 2);
  R a[4], b[4], c[4];
  hermite4((x - grid_x(gx, ix)) * gx.deltainv, gx.delta, a);
  hermite4((y - grid_x(gy, iy)) * gy.deltainv, gy.delta, b);
  hermite4((z - grid_x(gz, iz)) * gz.deltainv, gz.delta, c);
  const size_t sy = (size_t)gz.n * 8, sx = (size_t)gy.n * sy;
  const R *base = F + (size_t)ix * sx + (size_t)iy * sy + (size_t)iz * 8;
  R val = R(0);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    if (k < k0 || k >= k1) continue;
    const int dx = k >> 1, dy = k & 1;
    const R *p = base + dx * sx + dy * sy;
    Node8<R> n0, n1;
    n0.load(p);
    n1.load(p + 8);
    const R A0 = a[dx], A1 = a[2 + dx], B0 = b[dy], B1 = b[2 + dy];
    const R C00 = c[0], C01 = c[2], C10 = c[1], C11 = c[3];  // (z-node, z-derivative)
    const R s00 = n0.v[0] * C00 + n0.v[3] * C01 + n1.v[0] * C10 + n1.v[3] * C11;  // F, Fz
    const R s01 = n0.v[2] * C00 + n0.v[6] * C01 + n1.v[2] * C10 + n1.v[6] * C11;  // Fy, Fyz
    const R s10 = n0.v[1] * C00 + n0.v[5] * C01 + n1.v[1] * C10 + n1.v[5] * C11;  // Fx, Fxz
    const R s11 = n0.v[4] * C00 + n0.v[7] * C01 + n1.v[4] * C10 + n1.v[7] * C11;  // Fxy, Fxyz
    val += A0 * (B0 * s00 + B1 * s01) + A1 * (B0 * s10 + B1 * s11);
  }
  return val;
}

// SplinePot::V (Common/PH/SplinePot.cc:19-31) with no Vouter: the natural
// cubic spline up to the grid end, zero beyond.  Branch-free: the spline is
// evaluated at min(r, End) and the result selected.
template <typename R>
__device__ __forceinline__ R pot_V(const DTricubic<R> &t, R r) {
  const R v = spline_col(t.pot_grid, t.pot_y, t.pot_d2, 1, 0, r <= t.pot_grid.end ? r : t.pot_grid.end);
  return r <= t.pot_grid.end ? v : R(0);
}

// ---- PAtricubicFitClass::U / dU (PAtricubicFit.cc:659-721) ----
// Inside the fitted region (q <= qmax, z < 2q, s < 2q) the tricubic spline at
// (q, z/2q, (s-z)/(2q-z)) (at (0,0,0) when q == 0); outside it the primitive
// action 1/2 beta_l (V(r) + V(r')) (dU: 1/2 (V(r) + V(r'))).
template <typename R, bool DERIV>
__device__ __forceinline__ R tricubic_pa(const DTricubic<R> &t, R q, R z, R s2, int level, int part = 0,
                                         int nparts = 1) {
  const DGrid<R> &qg = t.qg, &yg = t.yg, &tg = t.tg;
  z = fabs_r(z);
  const R smax = R(2.0) * q;
  const R zmax = smax;
  const R s = sqrt_r(s2);
  const bool inside = (q <= t.qmax) && (z < zmax) && (s < smax);
  const bool nonzero = inside && q != R(0);
  const R xq = nonzero ? q : R(0);
  const R xy = nonzero ? z / zmax : R(0);
  const R xt = nonzero ? (s - z) / (smax - z) : R(0);
  const R *F = (DERIV ? t.dU : t.U) + (size_t)level * t.nq * t.ny * t.nt * 8;
  const int k0 = (4 * part) / nparts, k1 = (4 * (part + 1)) / nparts;
  const R r = q + R(0.5) * z;
  const R rp = q - R(0.5) * z;
  R beta = R(0.5);
  if (!DERIV) {
    beta = t.smallest_beta;
    for (int i = 0; i < level; i++) beta *= R(2.0);
    beta = R(0.5) * beta;
  }
  if (nparts == 1) {
    // One lane, one term: a lane inside the fit gathers its cell, a lane
    // outside reads the two potential splines; in a warp with both, each
    // side's loads issue for its own lanes only.
    if (inside) return tricubic_eval(F, qg, yg, tg, xq, xy, xt, k0, k1);
    return beta * (pot_V(t, r) + pot_V(t, rp));
  }
  // A team's parts: every lane takes both candidates and selects, so the
  // parts of one term stay in step.  Part 0 takes V(r), part 1 V(r').
  const R tri = tricubic_eval(F, qg, yg, tg, xq, xy, xt, k0, k1);
  const R prim = part < 2 ? beta * pot_V(t, part == 0 ? r : rp) : R(0);
  return inside ? tri : prim;
}

// ---- PathClass::DistDisp two-slice form (PathClass.h:696-746) ----
// Positions of ptcl1 and ptcl2 at slices A and B; returns dispA = r2-r1 at A
// wrapped to the minimum image and dispB at B taking the image consistent
// with dispA.  Always FP64 (the path is FP64).
__device__ __forceinline__ void dist_disp(const double a1[3], const double a2[3], const double b1[3],
                                          const double b2[3], const DevSystem &s, double dA[3], double dB[3]) {
#pragma unroll
  for (int i = 0; i < 3; i++) {
    double da = a2[i] - a1[i];
    double db = b2[i] - b1[i];
    double n = -rint(rmul(da, s.boxinv[i]));
    da = radd(da, rmul(n, s.box[i]));
    double m = rint(rmul(rsub(da, db), s.boxinv[i]));
    db = radd(db, rmul(m, s.box[i]));
    dA[i] = da;
    dB[i] = db;
  }
}

// PathClass::PutInBox (PathClass.h:897-921)
__device__ __forceinline__ void put_in_box(double v[3], const DevSystem &s) {
#pragma unroll
  for (int i = 0; i < 3; i++) {
    double n = -floor(radd(rmul(v[i], s.boxinv[i]), 0.5));
    v[i] = radd(v[i], rmul(n, s.box[i]));
  }
}
// PathClass::PutInBoxFast (PathClass.cc:1389-1407)
__device__ __forceinline__ void put_in_box_fast(double v[3], const DevSystem &s) {
#pragma unroll
  for (int dim = 0; dim < 3; dim++) {
    double halfBox = s.box[dim] / 2;
    if (v[dim] > halfBox) v[dim] -= s.box[dim];
    if (v[dim] < -halfBox) v[dim] += s.box[dim];
  }
}

// Pair geometry of one link: q, z, s^2 as ShortRangeClass::SingleAction
// forms them (ShortRangeClass.cc:217-220).
template <typename R>
struct LinkGeom {
  R q, z, s2, rmag, rpmag;
};
template <typename R>
__device__ __forceinline__ LinkGeom<R> link_geom(const double dA[3], const double dB[3]) {
  LinkGeom<R> g;
  R ax = (R)dA[0], ay = (R)dA[1], az = (R)dA[2];
  R bx = (R)dB[0], by = (R)dB[1], bz = (R)dB[2];
  R rmag = sqrt_r(ax * ax + ay * ay + az * az);
  R rpmag = sqrt_r(bx * bx + by * by + bz * bz);
  R d0 = ax - bx, d1 = ay - by, d2 = az - bz;
  g.s2 = d0 * d0 + d1 * d1 + d2 * d2;
  g.q = R(0.5) * (rmag + rpmag);
  g.z = (rmag - rpmag);
  g.rmag = rmag;
  g.rpmag = rpmag;
  return g;
}

template <typename R>
__device__ __forceinline__ const DTricubic<R> &tricubic_of(const DevPA &pa);
template <>
__device__ __forceinline__ const DTricubic<double> &tricubic_of<double>(const DevPA &pa) { return pa.t64; }
template <>
__device__ __forceinline__ const DTricubic<float> &tricubic_of<float>(const DevPA &pa) { return pa.t32; }

// U(q, z, s^2, level) of the pair action (ActionBaseClass's PA.U).
// QuinticSpline::operator() (QuinticSpline.h:204-221) on the LongGrid:
// interval ReverseMap(x) clamped to [0, np-2], Horner in P = x - x_I.
template <typename R>
__device__ __forceinline__ R quintic_at(const DCoulomb<R> &c, const R *tab, R x) {
  const R rm = round_even_magic(rsub(rmul(x, c.hinv), R(0.5)));
  const R lowf = fmin_r(fmax_r(rm, R(0)), (R)(c.np - 2));
  const int i = int_of_integral(lowf);
  const R *t = tab + (size_t)i * 6;
  const R P = x - rmul(lowf, c.h);
  return ((((t[5] * P + t[4]) * P + t[3]) * P + t[2]) * P + t[1]) * P + t[0];
}
// PAclassicalFitClass::U with the long-range part taken out as
// ShortRangeClass::SingleAction does (ShortRangeClass.cc:211-214).
template <typename R>
__device__ __forceinline__ R coulomb_U(const DCoulomb<R> &c, const LinkGeom<R> &g, int level) {
  R beta = c.smallest_beta;
  for (int i = 0; i < level; i++) beta *= R(2);
  R U = beta * (c.z1z2 / g.q);
  if (c.long_range) {
    const R *tab = c.ulong + (size_t)level * c.np * 6;
    U -= R(0.5) * (quintic_at(c, tab, g.rmag) + quintic_at(c, tab, g.rpmag));
  }
  return U;
}
// PAclassicalFitClass::dU with dUlong taken out (ShortRangeClass.cc:282-286).
__device__ __forceinline__ double coulomb_dU(const DCoulomb<double> &c, const LinkGeom<double> &g, int level) {
  double dU = c.z1z2 / g.q;
  if (c.long_range) {
    const double *tab = c.dulong + (size_t)level * c.np * 6;
    dU -= 0.5 * (quintic_at(c, tab, g.rmag) + quintic_at(c, tab, g.rpmag));
  }
  return dU;
}

template <typename R, int KIND>
__device__ __forceinline__ R pa_U(const DevPA &pa, const typename Pair2<R>::T *diag, const LinkGeom<R> &g,
                                  int level);
template <>
__device__ __forceinline__ double pa_U<double, PA_COULOMB>(const DevPA &pa, const double2 *,
                                                           const LinkGeom<double> &g, int level) {
  return coulomb_U<double>(pa.c64, g, level);
}
template <>
__device__ __forceinline__ float pa_U<float, PA_COULOMB>(const DevPA &pa, const float2 *, const LinkGeom<float> &g,
                                                         int level) {
  return coulomb_U<float>(pa.c32, g, level);
}
template <>
__device__ __forceinline__ double pa_U<double, PA_DAVID>(const DevPA &pa, const double2 *diag,
                                                         const LinkGeom<double> &g, int level) {
  return david_U<double>(pa.d64, diag, g.s2, g.q, g.z, level);
}
template <>
__device__ __forceinline__ float pa_U<float, PA_DAVID>(const DevPA &pa, const float2 *diag,
                                                       const LinkGeom<float> &g, int level) {
  return david_U<float>(pa.d32, diag, g.s2, g.q, g.z, level);
}
template <>
__device__ __forceinline__ double pa_U<double, PA_TRICUBIC>(const DevPA &pa, const double2 *,
                                                            const LinkGeom<double> &g, int level) {
  const DTricubic<double> &t = pa.t64;
  return tricubic_pa<double, false>(t, g.q, g.z, g.s2, level);
}
template <>
__device__ __forceinline__ float pa_U<float, PA_TRICUBIC>(const DevPA &pa, const float2 *,
                                                          const LinkGeom<float> &g, int level) {
  const DTricubic<float> &t = pa.t32;
  return tricubic_pa<float, false>(t, g.q, g.z, g.s2, level);
}

// Part `part` of `nparts` of U for a team of lanes sharing one evaluation;
// the parts sum to U (up to rounding).  The 1-D DavidPA action is not split.
template <typename R, int KIND>
__device__ __forceinline__ R pa_U_part(const DevPA &pa, const typename Pair2<R>::T *diag, const LinkGeom<R> &g,
                                       int level, int part, int nparts) {
  if (KIND == PA_TRICUBIC) return tricubic_pa<R, false>(tricubic_of<R>(pa), g.q, g.z, g.s2, level, part, nparts);
  return part == 0 ? pa_U<R, KIND>(pa, diag, g, level) : R(0);
}

template <typename R>
__device__ __forceinline__ const DDavid<R> &david_of(const DevPA &pa);
template <>
__device__ __forceinline__ const DDavid<double> &david_of<double>(const DevPA &pa) { return pa.d64; }
template <>
__device__ __forceinline__ const DDavid<float> &david_of<float>(const DevPA &pa) { return pa.d32; }

// ---- mixed precision: FP64 geometry and cell search, FP32 table arithmetic ----
// The mixed path forms r, r', s, q, z, the grid cell and the position inside
// the cell in FP64 — the same operations as the FP64 path, so the same cell
// and bit-identical in-cell coordinates — and rounds only the in-cell
// coordinate (a number in [0, 1]) to FP32.  The spline / tricubic polynomial
// then runs in FP32 on the FP32 copy of the table.  Each term comes with a
// magnitude m >= sum_j |c_j| |b_j| over its coefficients c_j and basis values
// b_j, so that |v - U| <= kMixedErr * m, U the FP64 evaluation of the same
// term: table rounding (2^-24 each), the FP32 rounding of the in-cell
// coordinate and of the basis, and the O(10) FP32 operations of the
// polynomial add up to fewer than 64 units of 2^-24 relative to m.
struct MixedU {
  double v;  // FP32 result (plus any FP64-evaluated addend)
  float m;   // magnitude bound
};
constexpr double kMixedErr = 64.0 * 5.9604644775390625e-8;  // 64 * 2^-24

// Cell and in-cell weight b = (x - x_low) / h of MultiCubicSpline::operator()
// in FP64, as spline_cell<double>; then the cubic in FP32 on (y, d2y) pairs.
__device__ __forceinline__ MixedU spline_pairs_mixed(const DGrid<double> &g, const float2 *tab, double x) {
  int low, hi;
  double xl, xh, h;
  if (g.type == PIMC_GRID_LINEAR) {
    const double rm = round_even_magic(rsub(rmul(rsub(x, g.start), g.deltainv), 0.5));
    const double lowf = fmin(fmax(rm, 0.0), (double)(g.n - 2));
    low = int_of_integral(lowf);
    hi = low + 1;
    xl = radd(g.start, rmul(lowf, g.delta));
    xh = 0.0;
    h = g.delta;
  } else {
    hi = reverse_map(g, x) + 1;
    low = hi - 1;
    if (low < 0) { low = 0; hi = 1; }
    if (hi > (g.n - 1)) { hi = g.n - 1; low = hi - 1; }
    xl = grid_x(g, low);
    xh = grid_x(g, hi);
    h = xh - xl;
  }
  const bool lin = g.type == PIMC_GRID_LINEAR;
  const double hinv = lin ? g.deltainv : 1.0 / h;
  const float b = (float)((x - xl) * hinv);
  const float a = lin ? 1.0f - b : (float)((xh - x) * hinv);
  const float h26 = (float)(h * h * 0.1666666666666666666);
  const float a3 = a * a * a - a, b3 = b * b * b - b;
  const float2 lo = tab[low], hv = tab[hi];
  MixedU r;
  r.v = (double)(a * lo.x + b * hv.x + (a3 * lo.y + b3 * hv.y) * h26);
  // |a|, |b| <= 1 and |a^3 - a|, |b^3 - b| <= 0.385 on the cell
  r.m = fabsf(lo.x) + fabsf(hv.x) + h26 * (fabsf(lo.y) + fabsf(hv.y));
  return r;
}

// DavidPAClass::calcUsqzFast (DavidPAClass.cc:468-511) on the mixed path:
// the diagonal u_00 columns in FP32 (diag: FP32 (y, d2y) pairs of this
// level), the clamps on FP64 r, r'; off-diagonal u_kj terms, when the fit has
// them, in FP64 on the FP64 tables.
__device__ __forceinline__ MixedU david_U_mixed(const DDavid<double> &d, const float2 *diag, double s2, double q,
                                                double z, int level) {
  level = level + d.tau_pos;
  const DGrid<double> &g = d.grid;
  const double rmin = g.start;
  double r = q + 0.5 * z;
  double rprime = q - 0.5 * z;
  if (r > g.end) r = g.end;
  if (rprime > g.end) rprime = g.end;
  if ((rprime < rmin) || (r < rmin)) return spline_pairs_mixed(g, diag, rmin);
  const MixedU a = spline_pairs_mixed(g, diag, r), b = spline_pairs_mixed(g, diag, rprime);
  MixedU U;
  U.v = (double)(0.5f * ((float)a.v + (float)b.v));
  U.m = 0.5f * (a.m + b.m);
  if (d.num_terms > 0 && s2 > 0.0 && q < g.end) {
    const double off = david_offdiag_add<double>(g, d.uy + (size_t)level * g.n * d.ncols,
                                                 d.ud2 + (size_t)level * g.n * d.ncols, d.ncols, d.num_terms, 0.0,
                                                 s2, q, z);
    U.v += off;
    // The FP64 path adds the same terms onto its diagonal value: the two
    // FP64 sums differ by a few 2^-53 of |off|, far below 1e-9 kMixedErr |off|.
    U.m += (float)(1e-9 * fabs(off));
  }
  return U;
}

// MyTricubicSpline::operator() (MyTricubicSpline.h:197-334) with the cell and
// the in-cell coordinates in FP64 and the Hermite basis and contraction in
// FP32 over (x-node, y-node) pairs [k0, k1) of the cell.
__device__ __forceinline__ float tricubic_eval_mixed(const float *__restrict__ F, const DGrid<double> &gx,
                                                     const DGrid<double> &gy, const DGrid<double> &gz, double x,
                                                     double y, double z, int ny, int nt, int &cell, int k0 = 0,
                                                     int k1 = 4) {
  int ix = reverse_map(gx, x), iy = reverse_map(gy, y), iz = reverse_map(gz, z);
  ix = max(0, ix); ix = min(ix, gx.n - 2);
  iy = max(0, iy); iy = min(iy, gy.n - 2);
  iz = max(0, iz); iz = min(iz, gz.n - 2);
  float a[4], b[4], c[4];
  hermite4((float)((x - grid_x(gx, ix)) * gx.deltainv), (float)gx.delta, a);
  hermite4((float)((y - grid_x(gy, iy)) * gy.deltainv), (float)gy.delta, b);
  hermite4((float)((z - grid_x(gz, iz)) * gz.deltainv), (float)gz.delta, c);
  cell = (ix * ny + iy) * nt + iz;
  const size_t sy = (size_t)nt * 8, sx = (size_t)ny * sy;
  const float *base = F + (size_t)cell * 8;
  float val = 0.0f;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    if (k < k0 || k >= k1) continue;
    const int dx = k >> 1, dy = k & 1;
    const float *p = base + dx * sx + dy * sy;
    Node8<float> n0, n1;
    n0.load(p);
    n1.load(p + 8);
    const float A0 = a[dx], A1 = a[2 + dx], B0 = b[dy], B1 = b[2 + dy];
    const float C00 = c[0], C01 = c[2], C10 = c[1], C11 = c[3];
    const float s00 = n0.v[0] * C00 + n0.v[3] * C01 + n1.v[0] * C10 + n1.v[3] * C11;
    const float s01 = n0.v[2] * C00 + n0.v[6] * C01 + n1.v[2] * C10 + n1.v[6] * C11;
    const float s10 = n0.v[1] * C00 + n0.v[5] * C01 + n1.v[1] * C10 + n1.v[5] * C11;
    const float s11 = n0.v[4] * C00 + n0.v[7] * C01 + n1.v[4] * C10 + n1.v[7] * C11;
    val += A0 * (B0 * s00 + B1 * s01) + A1 * (B0 * s10 + B1 * s11);
  }
  return val;
}

// SplinePot::V on the mixed path (cell in FP64, cubic in FP32); zero beyond End.
__device__ __forceinline__ MixedU pot_V_mixed(const DTricubic<double> &t64, const DTricubic<float> &t32, double r) {
  const DGrid<double> &g = t64.pot_grid;
  const double x = r <= g.end ? r : g.end;
  const double rm = round_even_magic(rsub(rmul(rsub(x, g.start), g.deltainv), 0.5));
  const double lowf = fmin(fmax(rm, 0.0), (double)(g.n - 2));
  const int low = int_of_integral(lowf);
  const double xl = radd(g.start, rmul(lowf, g.delta));
  const float b = (float)((x - xl) * g.deltainv), a = 1.0f - b;
  const float h26 = (float)(g.delta * g.delta * 0.1666666666666666666);
  const float a3 = a * a * a - a, b3 = b * b * b - b;
  const float yl = __ldg(&t32.pot_y[low]), yh = __ldg(&t32.pot_y[low + 1]);
  const float dl = __ldg(&t32.pot_d2[low]), dh = __ldg(&t32.pot_d2[low + 1]);
  MixedU u;
  const bool in = r <= g.end;
  u.v = in ? (double)(a * yl + b * yh + (a3 * dl + b3 * dh) * h26) : 0.0;
  u.m = in ? fabsf(yl) + fabsf(yh) + h26 * (fabsf(dl) + fabsf(dh)) : 0.0f;
  return u;
}

// PAtricubicFitClass::U (PAtricubicFit.cc:659-721) on the mixed path; the
// region test, (q, y, t) and the primitive's r, r' in FP64.  The magnitude of
// a tricubic term is the cell's precomputed bound (t32.mbound: the sum over
// the cell's 8 nodes of |F| + h|F_x| + ... + h_x h_y h_z |F_xyz|, which
// bounds sum_j |c_j||b_j| anywhere in the cell since the Hermite basis
// satisfies |p| <= 1, |q| <= 4h/27).  Parts as tricubic_pa.
__device__ __forceinline__ MixedU tricubic_pa_mixed(const DTricubic<double> &t64, const DTricubic<float> &t32,
                                                    double q, double z, double s2, int level, int part = 0,
                                                    int nparts = 1) {
  z = fabs(z);
  const double smax = 2.0 * q;
  const double s = sqrt(s2);
  const bool inside = (q <= t64.qmax) && (z < smax) && (s < smax);
  const bool nonzero = inside && q != 0.0;
  const double xq = nonzero ? q : 0.0;
  const double xy = nonzero ? z / smax : 0.0;
  const double xt = nonzero ? (s - z) / (smax - z) : 0.0;
  const size_t lvl = (size_t)level * t32.nq * t32.ny * t32.nt;
  const int k0 = (4 * part) / nparts, k1 = (4 * (part + 1)) / nparts;
  const double r = q + 0.5 * z, rp = q - 0.5 * z;
  double beta = t64.smallest_beta;
  for (int i = 0; i < level; i++) beta *= 2.0;
  const float hb = (float)(0.5 * beta);
  MixedU prim;
  if (nparts == 1) {  // one lane, one term: only the side the lane needs (as tricubic_pa)
    if (inside) {
      int cell;
      const float tri = tricubic_eval_mixed(t32.U + lvl * 8, t64.qg, t64.yg, t64.tg, xq, xy, xt, t32.ny, t32.nt,
                                            cell, k0, k1);
      return MixedU{(double)tri, __ldg(&t32.mbound[lvl + cell])};
    }
    const MixedU va = pot_V_mixed(t64, t32, r), vb = pot_V_mixed(t64, t32, rp);
    prim.v = (double)(hb * ((float)va.v + (float)vb.v));
    prim.m = hb * (va.m + vb.m);
    return prim;
  }
  int cell;
  const float tri = tricubic_eval_mixed(t32.U + lvl * 8, t64.qg, t64.yg, t64.tg, xq, xy, xt, t32.ny, t32.nt, cell,
                                        k0, k1);
  const float trim = part == 0 ? __ldg(&t32.mbound[lvl + cell]) : 0.0f;
  if (part < 2) {
    const MixedU va = pot_V_mixed(t64, t32, part == 0 ? r : rp);
    prim.v = (double)(hb * (float)va.v);
    prim.m = hb * va.m;
  } else {
    prim.v = 0.0;
    prim.m = 0.0f;
  }
  MixedU u;
  u.v = inside ? (double)tri : prim.v;
  u.m = inside ? trim : prim.m;
  return u;
}

// ---- PAtricubicFitClass::U by lane teams (the device moves' stage sums) ----
// tricubic_prep: the FP64 part of one term as tricubic_pa / tricubic_pa_mixed
// form it — the fit-region test, the cell (index of its low node among the
// level's [q][y][t] nodes), the in-cell coordinates (x - x_low) / h (the FP64
// values on the FP64 path, rounded to FP32 on the mixed path) and r, r' of
// the primitive fallback.
template <typename R>
struct TriPrep {
  R u[3];
  int cell;
  bool inside;
  double r, rp;
};
template <typename R>
__device__ __forceinline__ TriPrep<R> tricubic_prep(const DTricubic<double> &t, double q, double z, double s2) {
  TriPrep<R> p;
  z = fabs(z);
  const double smax = 2.0 * q;
  const double s = sqrt(s2);
  p.inside = (q <= t.qmax) && (z < smax) && (s < smax);
  const bool nonzero = p.inside && q != 0.0;
  const double x[3] = {nonzero ? q : 0.0, nonzero ? z / smax : 0.0, nonzero ? (s - z) / (smax - z) : 0.0};
  const DGrid<double> *g[3] = {&t.qg, &t.yg, &t.tg};
  int i3[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    int i = reverse_map(*g[d], x[d]);
    i = max(0, i);
    i = min(i, g[d]->n - 2);
    i3[d] = i;
    p.u[d] = (R)((x[d] - grid_x(*g[d], i)) * g[d]->deltainv);
  }
  p.cell = (i3[0] * t.ny + i3[1]) * t.nt + i3[2];
  p.r = q + 0.5 * z;
  p.rp = q - 0.5 * z;
  return p;
}

__device__ __forceinline__ void ld4_nc(const double *p, double v[4]) {
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3]) : "l"(p));
}

// One lane's part of a term evaluated by a team of 4 lanes (the FP64 path).
// The cell's four (x, y) node pairs k = 2 dx + dy each hold the nodes iz and
// iz + 1 back to back (128 bytes); part pt takes components 4 (pt & 1) ..
// 4 (pt & 1) + 3 of node iz + (pt >> 1) of every pair.  A lane loads 4 x 32
// bytes per term and the team's lanes load the same pairs together, so a
// warp-wide load touches one or two cache lines per team instead of one per
// lane.  The parts add up to tricubic_eval's value (summed in another order).
// F: this level's nodes.
__device__ __forceinline__ double tricubic_team_part(const double *F, const DTricubic<double> &t, int cell,
                                                     const double u[3], int pt) {
  double a[4], b[4], c[4];
  hermite4(u[0], t.qg.delta, a);
  hermite4(u[1], t.yg.delta, b);
  hermite4(u[2], t.tg.delta, c);
  const size_t sy = (size_t)t.nt * 8, sx = (size_t)t.ny * sy;
  const int nz = pt >> 1, hi = pt & 1;
  const double *p = F + (size_t)cell * 8 + nz * 8 + hi * 4;
  double v[4][4];
#pragma unroll
  for (int k = 0; k < 4; k++) ld4_nc(p + (k >> 1) * sx + (k & 1) * sy, v[k]);
  // components (F, Fx, Fy, Fz) weigh (A0 B0 Cv, A1 B0 Cv, A0 B1 Cv, A0 B0 Cd),
  // (Fxy, Fxz, Fyz, Fxyz) weigh (A1 B1 Cv, A1 B0 Cd, A0 B1 Cd, A1 B1 Cd)
  const double Cv = nz ? c[1] : c[0], Cd = nz ? c[3] : c[2], Ce = hi ? Cd : Cv;
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int dx = k >> 1, dy = k & 1;
    const double A0 = a[dx], A1 = a[2 + dx], B0 = b[dy], B1 = b[2 + dy];
    const double Pd = hi ? A1 * B1 : A0 * B0;
    s += Pd * (Cv * v[k][0] + Cd * v[k][3]) + Ce * (A1 * B0 * v[k][1] + A0 * B1 * v[k][2]);
  }
  return s;
}
// SplinePot::V from (y, d2y) pairs (a shared-memory copy): the same
// arithmetic as pot_V, zero beyond the grid end.
__device__ __forceinline__ double pot_V_pairs(const DGrid<double> &g, const double2 *pp, double r) {
  const double v = spline_pairs(g, pp, r <= g.end ? r : g.end);
  return r <= g.end ? v : 0.0;
}

// QuinticSpline::operator() on the mixed path: interval and P = x - x_I in
// FP64, Horner in FP32; the magnitude is Horner on |coefficients| and |P|.
__device__ __forceinline__ MixedU quintic_mixed(const DCoulomb<double> &c, const float *tab, double x) {
  const double rm = round_even_magic(rsub(rmul(x, c.hinv), 0.5));
  const double lowf = fmin(fmax(rm, 0.0), (double)(c.np - 2));
  const int i = int_of_integral(lowf);
  const float *t = tab + (size_t)i * 6;
  const float P = (float)(x - rmul(lowf, c.h)), aP = fabsf(P);
  MixedU u;
  u.v = (double)(((((t[5] * P + t[4]) * P + t[3]) * P + t[2]) * P + t[1]) * P + t[0]);
  u.m = ((((fabsf(t[5]) * aP + fabsf(t[4])) * aP + fabsf(t[3])) * aP + fabsf(t[2])) * aP + fabsf(t[1])) * aP +
        fabsf(t[0]);
  return u;
}
// PAclassicalFitClass::U minus the long-range part (ShortRangeClass.cc:211-214)
// on the mixed path: beta Z1Z2 / q by one FP32 division of FP64-formed operands.
__device__ __forceinline__ MixedU coulomb_U_mixed(const DCoulomb<double> &c64, const DCoulomb<float> &c32,
                                                  const LinkGeom<double> &g, int level) {
  double beta = c64.smallest_beta;
  for (int i = 0; i < level; i++) beta *= 2.0;
  const float t0 = (float)(beta * c64.z1z2) / (float)g.q;
  MixedU u;
  u.v = (double)t0;
  u.m = fabsf(t0);
  if (c64.long_range) {
    const float *tab = c32.ulong + (size_t)level * c32.np * 6;
    const MixedU a = quintic_mixed(c64, tab, g.rmag), b = quintic_mixed(c64, tab, g.rpmag);
    u.v = (double)(t0 - 0.5f * ((float)a.v + (float)b.v));
    u.m += 0.5f * (a.m + b.m);
  }
  return u;
}

// U of one pair-link on the mixed path from the FP64 geometry; diag: the FP32
// (y, d2y) pairs of this level's u_00 column (DavidPA).  Part `part` of
// `nparts` as pa_U_part.
template <int KIND>
__device__ __forceinline__ MixedU pa_U_mixed(const DevPA &pa, const float2 *diag, const LinkGeom<double> &g,
                                             int level, int part = 0, int nparts = 1) {
  if (KIND == PA_TRICUBIC) return tricubic_pa_mixed(pa.t64, pa.t32, g.q, g.z, g.s2, level, part, nparts);
  if (part != 0) return MixedU{0.0, 0.0f};
  if (KIND == PA_DAVID) return david_U_mixed(pa.d64, diag, g.s2, g.q, g.z, level);
  return coulomb_U_mixed(pa.c64, pa.c32, g, level);
}

// Two-sum accumulation (Knuth): s + c carries the running sum of the terms
// with the exact rounding error of each FP64 addition gathered in c (FP32
// suffices for c: each error is below 2^-53 |s|).
__device__ __forceinline__ void two_sum_add(double &s, float &c, double x) {
  const double t = s + x;
  const double bp = t - s;
  c += (float)((s - (t - bp)) + (x - bp));
  s = t;
}

// dU (energy estimator), FP64 only.
template <int KIND>
__device__ __forceinline__ double pa_dU(const DevPA &pa, const LinkGeom<double> &g, int level);
template <>
__device__ __forceinline__ double pa_dU<PA_DAVID>(const DevPA &pa, const LinkGeom<double> &g, int level) {
  return david_dU<double>(pa.d64, g.s2, g.q, g.z, level);
}
template <>
__device__ __forceinline__ double pa_dU<PA_COULOMB>(const DevPA &pa, const LinkGeom<double> &g, int level) {
  return coulomb_dU(pa.c64, g, level);
}
template <>
__device__ __forceinline__ double pa_dU<PA_TRICUBIC>(const DevPA &pa, const LinkGeom<double> &g, int level) {
  const DTricubic<double> &t = pa.t64;
  return tricubic_pa<double, true>(t, g.q, g.z, g.s2, level);
}

// ---- KineticClass::SingleAction link term (KineticClass.cc:45-78) ----
// vel = Velocity(slice, slice+skip): the PutInBox'ed link vector.
__device__ __forceinline__ double kinetic_link(const double vel[3], double four_lambda_tau_inv, int num_images,
                                               const DevSystem &s) {
  if (num_images == 0) {
    // -log(prod_d exp(-v_d^2 F)) = sum_d v_d^2 F, exact up to rounding while
    // no factor underflows (the reference would then return +inf).
    const double e0 = vel[0] * vel[0] * four_lambda_tau_inv, e1 = vel[1] * vel[1] * four_lambda_tau_inv,
                 e2 = vel[2] * vel[2] * four_lambda_tau_inv;
    if (e0 < 700.0 && e1 < 700.0 && e2 < 700.0) return e0 + e1 + e2;
  }
  double GaussProd = 1.0;
  for (int dim = 0; dim < 3; dim++) {
    double GaussSum = 0.0;
    for (int image = -num_images; image <= num_images; image++) {
      double dist = vel[dim] + (double)image * s.box[dim];
      GaussSum += exp(-dist * dist * four_lambda_tau_inv);
    }
    GaussProd *= GaussSum;
  }
  return -log(GaussProd);
}

// ---- Philox-4x32-10 (Salmon et al., SC'11): the Local/Common/World streams ----
__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
    uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
    uint32_t n0 = hi1 ^ c[1] ^ k0;
    uint32_t n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    k0 += W0; k1 += W1;
  }
}
// Element `index` of stream `stream`: two 53-bit doubles per Philox block.
static __device__ __noinline__ double philox_uniform(uint64_t seed, uint32_t stream, uint64_t index) {
  uint64_t block = index >> 1;
  uint32_t c[4] = {(uint32_t)block, (uint32_t)(block >> 32), stream, 0x50494D43u};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  int h = (int)(index & 1);
  uint32_t a = (h ? c[2] : c[0]) >> 5, b = (h ? c[3] : c[1]) >> 6;
  return ((double)a * 67108864.0 + (double)b) * (1.0 / 9007199254740992.0);
}

// Stream values precomputed for the positions [tb, tb + W) of one Local
// stream (an even tb): the uniform u (u also holds position tb + W), log u,
// and the polar-method pair (X1, X2, accepted) of the candidate pair starting
// at each position.  A CTA fills it with all of its threads at once, so the
// sampler warps, which draw sequentially, read these values instead of
// computing Philox blocks, logarithms and square roots on their critical
// path.  Entries are what the direct computation gives, bit for bit.
struct RngTab {
  double *u, *lu, *x1, *x2;
  unsigned char *acc;
  uint64_t tb;
  int W;  // 0: no table
};

// RandomClass (Common/Random/Random.h:33-49,156-180): Local(), LocalInt(),
// LocalGaussian() with the polar-method pair cache.  Every lane of a warp
// holds the same copy and draws the same values (warp-uniform state).
struct DevRandom {
  uint64_t seed, n;
  uint32_t stream;
  int one_left;
  double x2;
  const RngTab *tab;
  __device__ __forceinline__ double Local() {
    if (tab) {
      const uint64_t k = n - tab->tb;
      if (k < (uint64_t)tab->W) {
        n++;
        return tab->u[k];
      }
    }
    return philox_uniform(seed, stream, n++);
  }
  // log(Local()), the acceptance draw of a stage.
  __device__ __forceinline__ double LocalLog() {
    if (tab) {
      const uint64_t k = n - tab->tb;
      if (k < (uint64_t)tab->W) {
        n++;
        return tab->lu[k];
      }
    }
    return log(philox_uniform(seed, stream, n++));
  }
  __device__ __forceinline__ int LocalInt(int max) { return (int)floor(Local() * max); }
};

// The polar-method transform of one candidate pair (u1, u2).
__device__ __forceinline__ void polar_pair(double u1, double u2, bool &acc, double &X1, double &X2) {
  const double V1 = 2.0 * u1 - 1.0;
  const double V2 = 2.0 * u2 - 1.0;
  const double S = V1 * V1 + V2 * V2;
  acc = !(S >= 1.0);
  const double temp = sqrt((-2.0 * log(S)) / S);
  X1 = V1 * temp;
  X2 = V2 * temp;
}

// Fills t for the positions from (from & ~1), by the `size` threads whose
// index in the group is `gtid`; `sync` is the group's barrier.
template <typename Sync>
__device__ __noinline__ void rng_tab_fill(RngTab &t, int W, uint64_t seed, uint32_t stream, uint64_t from, int gtid, int size,
                             const Sync &sync) {
  const uint64_t tb = from & ~1ull;
  for (int i = gtid; i <= (W >> 1); i += size) {
    const uint64_t blk = (tb >> 1) + (uint64_t)i;
    uint32_t c[4] = {(uint32_t)blk, (uint32_t)(blk >> 32), stream, 0x50494D43u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    t.u[2 * i] = ((double)(c[0] >> 5) * 67108864.0 + (double)(c[1] >> 6)) * (1.0 / 9007199254740992.0);
    t.u[2 * i + 1] = ((double)(c[2] >> 5) * 67108864.0 + (double)(c[3] >> 6)) * (1.0 / 9007199254740992.0);
  }
  sync();
  for (int k = gtid; k < W; k += size) {
    const double u1 = t.u[k], u2 = t.u[k + 1];
    t.lu[k] = log(u1);
    bool acc;
    double X1, X2;
    polar_pair(u1, u2, acc, X1, X2);
    t.acc[k] = acc ? 1 : 0;
    t.x1[k] = X1;
    t.x2[k] = X2;
  }
  if (gtid == 0) {
    t.tb = tb;
    t.W = W;
  }
  sync();
}

// G unit Gaussians in stream order into out[0..G-1], drawn by one full warp.
// Sequentially, LocalGaussian returns the cached X2 if one is left, else
// draws uniform pairs (V1, V2) until S = V1^2 + V2^2 < 1 and returns
// X1 = V1 t, caching X2 = V2 t, t = sqrt(-2 ln S / S).  Here lane j tests the
// candidate pair at stream offset 2j; a ballot orders the accepted pairs, so
// the values, the cache and the stream position come out exactly as the
// sequential loop leaves them.  Candidate pairs inside the precomputed table
// are read from it.  Bounded: at most 4096 rounds of 32 pairs.
static __device__ __noinline__ void warp_gaussians(DevRandom &rng, int G, double *out, int lane) {
  int k = 0;
  if (G > 0 && rng.one_left) {
    if (lane == 0) out[0] = rng.x2;
    rng.one_left = 0;
    k = 1;
  }
  for (int guard = 0; k < G && guard < 4096; guard++) {
    const int need = (G - k + 1) >> 1;
    bool acc;
    double X1, X2;
    const uint64_t kt = rng.tab ? rng.n + 2ull * (uint64_t)lane - rng.tab->tb : ~0ull;
    const bool in_tab = rng.tab && kt < (uint64_t)rng.tab->W;
    if (__all_sync(0xffffffffu, in_tab)) {
      acc = rng.tab->acc[kt] != 0;
      X1 = rng.tab->x1[kt];
      X2 = rng.tab->x2[kt];
    } else {
      // Candidate pair j uses uniforms n+2j and n+2j+1.  Lane j computes the
      // Philox block holding uniform n+2j (two uniforms per block); when n is
      // odd the second uniform is the first half of the next lane's block.
      const uint64_t b0 = (rng.n >> 1) + (uint64_t)lane;
      uint32_t c[4] = {(uint32_t)b0, (uint32_t)(b0 >> 32), rng.stream, 0x50494D43u};
      philox4x32_10(c, (uint32_t)rng.seed, (uint32_t)(rng.seed >> 32));
      const double h0 = ((double)(c[0] >> 5) * 67108864.0 + (double)(c[1] >> 6)) * (1.0 / 9007199254740992.0);
      const double h1 = ((double)(c[2] >> 5) * 67108864.0 + (double)(c[3] >> 6)) * (1.0 / 9007199254740992.0);
      double u1, u2;
      if ((rng.n & 1) == 0) {
        u1 = h0;
        u2 = h1;
      } else {
        u1 = h1;
        u2 = __shfl_down_sync(0xffffffffu, h0, 1);
        if (lane == 31) u2 = philox_uniform(rng.seed, rng.stream, rng.n + 2ull * 31 + 1);
      }
      polar_pair(u1, u2, acc, X1, X2);
    }
    const unsigned m = __ballot_sync(0xffffffffu, acc);
    const int before = __popc(m & ((1u << lane) - 1u));
    const int navail = __popc(m);
    if (acc && before < need) {
      const int idx = k + 2 * before;
      out[idx] = X1;
      if (idx + 1 < G) out[idx + 1] = X2;
    }
    if (navail >= need) {
      const unsigned lastm = __ballot_sync(0xffffffffu, acc && before == need - 1);
      const int p = __ffs(lastm) - 1;
      const double x2p = __shfl_sync(0xffffffffu, X2, p);
      if ((G - k) & 1) {
        rng.x2 = x2p;
        rng.one_left = 1;
      }
      rng.n += 2ull * (uint64_t)(p + 1);
      k = G;
    } else {
      rng.n += 64;
      k += 2 * navail;
    }
  }
}

}  // namespace pimc

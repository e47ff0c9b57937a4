// Internal types of the B200 PIMC action library: host-side tables, the
// device descriptors handed to kernels by value, and the context.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/pimc_b200.h"

namespace pimc {

constexpr int kMaxLevels = 8;        // bisection levels a move may use (2^8 slices)
constexpr int kMaxWindow = (1 << 6) + 1;  // slices of a move window held in shared memory (NumLevels <= 6)
constexpr int kMaxCluster = 16;
constexpr int kMaxActive = 64;       // active particles of one SingleAction call
constexpr int kPartialSlots = 8192;  // per-block partial sums of the reduction kernels

// ---------------------------------------------------------------------------
// Host tables (FP64, built once on the host like the reference's setup).
// ---------------------------------------------------------------------------
struct HostGrid {
  int type = PIMC_GRID_LINEAR;
  int n = 0;
  double start = 0, end = 0, delta = 0, deltainv = 0, r0 = 0, spacing = 1, log_spacing = 0;
  std::vector<double> x;
  void init_linear(double s, double e, int num);
  void init_log(double r0_, double spacing_, int num);
};

// Natural/clamped cubic-spline second derivatives over columns (Numerical
// Recipes tridiagonal solve).  y, d2y row-major [point][column].
void spline_second_derivs(const HostGrid &g, const double *y, int ncols, int col, double start_deriv,
                          double end_deriv, double *d2y);
// First-derivative tricubic coefficient fill of 8 components per node.
void tricubic_fill(const HostGrid &gx, const HostGrid &gy, const HostGrid &gz, const double *values,
                   double *F);

struct DavidTables {
  HostGrid grid;
  int ncols = 0, num_tau = 0, tau_pos = 0, num_terms = 0;
  std::vector<double> uy, ud2, duy, dud2;  // [tau][point][col]
};
int read_dm_file(const char *path, double desired_tau, int num_terms, DavidTables &out, std::string &err);
void build_david(DavidTables &t, const double *ukj, const double *dukj);

// ---------------------------------------------------------------------------
// Device descriptors (passed to kernels by value).
// ---------------------------------------------------------------------------
template <typename R>
struct DGrid {
  int type, n;
  R start, end, delta, deltainv, r0, log_spacing;
  const R *x;  // node coordinates [n]
};

// DavidPAClass tables for one species pair, one precision.
template <typename R>
struct DDavid {
  DGrid<R> grid;
  int ncols, num_tau, tau_pos, num_terms;
  const R *uy, *ud2;    // ukj  [tau][point][col]
  const R *duy, *dud2;  // dukj [tau][point][col]
  const R *diag;        // column 1 of ukj as (y, d2y) pairs [tau][diag_stride][2]
  int diag_stride;      // points per level of diag, rounded up to an even count
};

// PAtricubicFitClass tables for one species pair, one precision.
template <typename R>
struct DTricubic {
  int nq, ny, nt, num_betas;
  DGrid<R> qg, yg, tg;       // linear q, y, t grids
  R qmax;                    // qgrid End
  R smallest_beta;
  const R *U;   // [beta][nq][ny][nt][8]
  const R *dU;  // same
  DGrid<R> pot_grid;
  const R *pot_y, *pot_d2;  // SplinePot natural cubic spline
  const R *pot_pairs;        // FP64: the same as interleaved (y, d2y) pairs [pot_pairs_n][2] (FP32: null)
  int pot_pairs_n;           // pot_grid.n rounded up to an even count (16-byte rows)
  // Mixed path: per level and cell (indexed by the cell's low node, [beta][nq][ny][nt])
  // a bound on sum_j |c_j| |b_j| of the U evaluation anywhere in the cell
  const float *mbound;
};

enum PAKind : int { PA_NONE = 0, PA_DAVID = 1, PA_TRICUBIC = 2, PA_COULOMB = 3 };

// Points of the long-range r grid, LongGrid of LongRangeClass (LongRangeClass.cc:547-549).
constexpr int kLongGridPoints = 1000;

// PAclassicalFitClass with a CoulombPot (PAclassicalFit.cc:57-75, 175-288):
// U = beta_l Z1Z2 / q, dU = Z1Z2 / q, beta_l = smallest_beta 2^l.  With the
// long-range breakup set, ShortRangeClass subtracts 1/2 (Ulong_l(r) +
// Ulong_l(r')) (dUlong for d_dBeta), Ulong_l a natural quintic spline on the
// LongGrid stored as the Taylor coefficients of each interval at its left
// knot, {y, y', y''/2, y^(3)/6, y^(4)/24, y^(5)/120}: ulong[level][point][6].
template <typename R>
struct DCoulomb {
  R z1z2, smallest_beta;
  int num_levels;
  int long_range;  // 1: subtract the long-range part
  int np;
  R h, hinv;       // LongGrid spacing (start 0)
  const R *ulong, *dulong;
};

struct DevPA {
  int kind;
  DDavid<double> d64;
  DDavid<float> d32;
  DTricubic<double> t64;
  DTricubic<float> t32;
  DCoulomb<double> c64;
  DCoulomb<float> c32;
};

// The optimized breakup of a Coulomb pair action (breakup.cc).
struct BreakupTables {
  double rc = 0, rmax = 0, knots_delta = 0;
  int levels = 0, num_k = 0, kpoints = 0;
  std::vector<double> ulong_k, dulong_k;          // [level][k]
  std::vector<double> ulong_r0, dulong_r0, ushort_k0, dushort_k0, ulong_k0, dulong_k0;  // [level]
  std::vector<double> ulong_r, dulong_r;          // [level][kLongGridPoints][6]
};
int coulomb_breakup(const double box[3], double z1z2, double smallest_beta, int num_levels, int num_knots,
                    double kcut, int num_k, const double *kvecs, BreakupTables &out);
bool quintic_natural(int n, double h, const double *y, double *coef);
double quintic_eval(int n, double start, double h, const double *coef, double x);

struct DevSystem {
  int N, S;  // particles, path rows
  double box[3], boxinv[3];
  double tau, lambda;
  int num_images;
};

constexpr int kMaxWindows = 64;      // concurrent slice windows of one chain
constexpr uint32_t kStreamLocal = 0, kStreamCommon = 1, kStreamWorld = 2;
// Local stream of window w, proposal slot p (slot 0 without proposals) is
// kStreamWindow0 + p * kMaxWindows + w, in ChainState p * kMaxWindows + w
constexpr uint32_t kStreamWindow0 = 0x100;
constexpr int kMaxChainStates = kMaxWindows * kMaxCluster;

// Device state of one Local RNG stream and its move counters: the chain in
// the sequential schedule, or one slice window in the concurrent schedule.
struct ChainState {
  uint64_t seed;
  uint64_t nlocal;     // position in the stream
  uint32_t stream;     // Philox stream id
  int32_t one_left;    // LocalGaussian cache flag (Random.h:159-160)
  double x2;           // cached second Gaussian
  int32_t status;
  int32_t pad;
  unsigned long long moves, accepted, stages, pair_evals, flips;
  unsigned long long redone;  // concurrent proposals: moves discarded and made again
  unsigned long long reevals; // mixed path: stages decided on their FP64 re-evaluation
};

struct DeviceBuffer {
  void *p = nullptr;
  size_t bytes = 0;
};

}  // namespace pimc

struct pimc_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  pimc::DevSystem sys{};
  std::vector<int> species_of;
  std::vector<double> lambda;
  int num_species = 1;
  double *d_path[2] = {nullptr, nullptr};
  size_t path_elems = 0;
  // pair action (single species pair)
  pimc::DevPA pa{};
  std::vector<void *> owned;  // device allocations of the tables
  // reduction scratch
  double *d_partials = nullptr;
  unsigned int *d_counter = nullptr;
  double *d_out = nullptr;
  double *h_out = nullptr;  // pinned
  int *d_active = nullptr;
  // bisection
  pimc_bisection_desc bis{};
  bool bis_ready = false;
  pimc::ChainState *d_chain = nullptr;  // kMaxWindows states
  unsigned long long rounds = 0;         // concurrent-window rounds run so far
  uint64_t seed = 0;                     // the key pimc_rng_seed set
  unsigned long long shift_draws = 0;    // ShiftMove draws taken from stream 3
  pimc_move_record *d_trace = nullptr;
  size_t trace_cap = 0;
  int sm_count = 0;
  // long range (one species): k-vectors, rho_k [copy][slice][k], breakup tables
  int num_k = 0;
  double kcutoff = 0;
  int kmax[3] = {0, 0, 0};
  double kbox[3] = {0, 0, 0};
  std::vector<double> kvecs;  // [k][3]
  int3 *d_kidx = nullptr;
  double2 *d_rhok[2] = {nullptr, nullptr};
  double *d_kvec = nullptr;  // [k][3] for the device moves
  // neighbour lists of the device moves
  double4 *d_nbr_cb = nullptr;
  int *d_nbr_cnt = nullptr, *d_nbr_idx = nullptr, *d_nbr_dirty = nullptr;
  int nbr_kmax = 0;
  double nbr_range = 0.0;
  bool rhok_valid = false;   // d_rhok[OLD] holds rho_k of the OLD path
  bool lr_ready = false;
  int lr_levels = 0, use_background = 0;
  double *d_ulong_k = nullptr, *d_dulong_k = nullptr;  // [levels][k]
  std::vector<double> ulong_r0, ushort_k0, ulong_k0, dulong_r0, dushort_k0, dulong_k0;
  // DavidLongRangeClassYk: uk, duk, Vlong_k of the k-vectors ([3][k])
  double *d_yk = nullptr;
  bool yk_ready = false;
  // pair correlation accumulator (PairCorrelationClass)
  unsigned long long *d_gofr = nullptr;
  int gofr_points = 0;
  double gofr_start = 0, gofr_end = 0, gofr_delta = 0, gofr_deltainv = 0;
  long long gofr_counts = 0;
  std::string last_error;
};

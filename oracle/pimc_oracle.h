/*
 * ORACLE — TEST INFRASTRUCTURE ONLY.
 *
 * A plain FP64 CPU restatement of the PIMC++ action-evaluation hot path,
 * written loop for loop after the reference sources it cites.  It is the
 * checker for the CUDA library in pimcplusplus_b200/: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg (and the
 * `--impl reference` arm) may load it.  The product never links or calls it.
 *
 * The reference itself cannot be compiled here (it needs Blitz++, SPRNG2, GSL,
 * HDF5 and LAPACK, none of which is installed), so this restatement stands in
 * for it.  Parity pins: the reference's own fixture PIMC++/examples/testcoul.dm
 * (through tests/golden/), the analytic tricubic test of
 * Common/Splines/TestMyTricubic.cc, and the identities the reference checks in
 * debug builds (incremental rho_k == full recompute, LongRangeClass.cc:283-305;
 * DistDisp == while-loop wrap, PathClass.h:664-676).  No reference-generated
 * SingleAction value exists anywhere, so action values are pinned through
 * those pieces and through second, independent numpy/Python statements of the
 * reference's formulas (tests/test_oracle_composition_cpu.py,
 * test_oracle_tricubic_cpu.py, test_oracle_bisection_cpu.py), not against
 * outputs of the reference itself.
 *
 * The RNG: the reference draws from SPRNG 2 (unpinned version, absent here),
 * so the random stream is parity unpinned.  Both this oracle and the CUDA
 * library use the Philox-4x32-10 stream defined in oracle_philox_uniform()
 * instead (pinned by its published known answers), consumed in the
 * reference's order.
 */
#ifndef PIMC_ORACLE_H
#define PIMC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleSystem OracleSystem;
typedef struct OraclePA OraclePA;

/* ---- RNG (Philox-4x32-10, Salmon et al. SC'11) ---- */
double oracle_philox_uniform(uint64_t seed, uint32_t stream, uint64_t index);
void oracle_philox_block(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* ---- Pair actions ---- */
/* Reads an ASCII squarer .dm file (DavidPAClass::ReadDavidSquarerFile). */
OraclePA *oracle_pa_david_from_dm(const char *path, double desired_tau, int num_offdiag_terms);
/* DavidPAClass tables from arrays on a LINEAR grid: ukj/dukj [tau][grid][ncols]. */
OraclePA *oracle_pa_david_arrays(double grid_start, double grid_end, int n, int ncols, int ntau, const double *ukj,
                                 const double *dukj, int tau_pos, int num_terms);
/* PAtricubicFitClass with a SplinePot potential (PAtricubicFit.cc:794-865). */
OraclePA *oracle_pa_tricubic(double q0, double q1, int nq, double y0, double y1, int ny,
                             double t0, double t1, int nt, int num_betas, double smallest_beta,
                             const double *umat, const double *dumat,
                             double pot_start, double pot_end, int pot_n, const double *pot_data);
/* PAclassicalFitClass with a Coulomb potential Z1Z2/r (PAclassicalFit.cc:57-75). */
OraclePA *oracle_pa_classical_coulomb(double smallest_beta, int num_betas, double z1z2);
void oracle_pa_free(OraclePA *pa);
double oracle_pa_U(OraclePA *pa, double q, double z, double s2, int level);
double oracle_pa_dU(OraclePA *pa, double q, double z, double s2, int level);
int oracle_pa_info(OraclePA *pa, int *num_tau, int *tau_pos, int *num_grid, int *num_cols,
                   double *grid_start, double *grid_end, int *grid_type);
/* Raw spline data of the David tables: which=0 ukj y, 1 ukj d2y, 2 dukj y, 3 dukj d2y. */
int oracle_pa_david_table(OraclePA *pa, int which, int level, double *out);
double oracle_pa_david_spline(OraclePA *pa, int which, int level, int col, double x);
/* Sets Ulong(level)(r) for a long-range pair action as a cubic-spline table. */

/* ---- Tricubic spline (MyTricubicSpline) standalone, for the analytic test ---- */
typedef struct OracleTricubic OracleTricubic;
OracleTricubic *oracle_tricubic_create(double x0, double x1, int nx, double y0, double y1, int ny,
                                       double z0, double z1, int nz, const double *f);
double oracle_tricubic_eval(OracleTricubic *t, double x, double y, double z);
int oracle_tricubic_coefs(OracleTricubic *t, double *out /* nx*ny*nz*8 */);
void oracle_tricubic_free(OracleTricubic *t);

/* ---- The path-integral system (PathDataClass + PathClass + ActionsClass) ---- */
OracleSystem *oracle_system_create(int num_particles, int num_time_slices, const double *box,
                                   double tau, double lambda, int num_images);
void oracle_system_free(OracleSystem *s);
/* Pair action for the (single) species pair; the system does not own it. */
void oracle_system_set_pa(OracleSystem *s, OraclePA *pa);
void oracle_system_set_path(OracleSystem *s, int copy, const double *path);
void oracle_system_get_path(OracleSystem *s, int copy, double *path);
void oracle_system_set_mode(OracleSystem *s, int copy);
/* InitRandomFixed (InitPaths.cc:966-999) from the World stream of `seed`. */
int oracle_init_random_fixed(OracleSystem *s, uint64_t seed, double radius);
int oracle_shift_data(OracleSystem *s, int slicesToShift);

double oracle_shortrange_single(OracleSystem *s, int slice1, int slice2, const int *active,
                                int n_active, int level);
/* Sum of |U| over the same terms: the scale of the summation error. */
double oracle_shortrange_single_abs(OracleSystem *s, int slice1, int slice2, const int *active,
                                    int n_active, int level);
double oracle_shortrange_dbeta(OracleSystem *s, int slice1, int slice2, int level);
double oracle_kinetic_single(OracleSystem *s, int slice1, int slice2, const int *active,
                             int n_active, int level);
double oracle_kinetic_dbeta(OracleSystem *s, int slice1, int slice2, int level);

/* ---- Long range: k-vectors, rho_k, LongRangeClass ---- */
int oracle_setup_kvecs(OracleSystem *s, double kcutoff);
int oracle_num_kvecs(OracleSystem *s);
void oracle_get_kvecs(OracleSystem *s, double *kvecs /* nk*3 */, int *kindices /* nk*3 */);
void oracle_calc_rhok_all(OracleSystem *s);            /* UpdateRho_ks() full recompute */
void oracle_update_rhok(OracleSystem *s, int slice1, int slice2, const int *active, int n, int level);
void oracle_get_rhok(OracleSystem *s, int copy, double *out /* slices*nk*2 */);
void oracle_set_longrange(OracleSystem *s, int num_levels, const double *ulong_k /* levels*nk */,
                          const double *ulong_r0, const double *ushort_k0, const double *ulong_k0,
                          const double *dulong_k, const double *dulong_r0,
                          const double *dushort_k0, const double *dulong_k0, int use_background);
double oracle_longrange_single(OracleSystem *s, int slice1, int slice2, const int *active,
                               int n_active, int level);
double oracle_longrange_dbeta(OracleSystem *s, int slice1, int slice2, int level);

/* ---- Bisection moves (BisectionBlockClass / MultiStageClass / LocalStageClass) ---- */
typedef struct {
  int32_t slice1;
  int32_t ptcl;
  int32_t accepted;       /* 1 if the whole move was accepted */
  int32_t stages_passed;  /* number of bisection stages accepted */
  double dS[8];           /* S_new - S_old of each bisection stage attempted, highest level first */
  double log_sample_ratio[8];
} OracleMoveRecord;

void oracle_bisection_config(OracleSystem *s, int num_levels, int steps_per_block,
                             int shortrange_at_higher_levels, int use_longrange);
void oracle_rng_seed(OracleSystem *s, uint64_t seed);
/* Runs n_blocks BisectionBlock moves; fills n_blocks*steps_per_block records. */
int oracle_run_bisection(OracleSystem *s, int n_blocks, OracleMoveRecord *records);
/* Concurrent-window schedule replayed sequentially: n_rounds rounds, each
 * windows*steps_per_block records (slice1 = -1 for a window that does not
 * fit); returns windows = floor((slices-1)/2^L). */
/* DavidLongRangeClassYk on the k-vectors of oracle_setup_kvecs: tables from
 * the squarer's k-space action uk_long(kvals) (rpa: the single-type RPA
 * construction), -1 if a k-vector's |k| is not among kvals; the actions on
 * the active copy (oracle_system_set_mode). */
int oracle_set_yk(OracleSystem *s, int num_kvals, const double *kvals, const double *uk_long, int rpa);
void oracle_get_yk(OracleSystem *s, double *uk, double *duk, double *vlong);
double oracle_yk_single(OracleSystem *s, int slice1, int slice2, const int *active, int n, int level);
double oracle_yk_dbeta(OracleSystem *s, int slice1, int slice2);
double oracle_yk_v(OracleSystem *s, int slice1, int slice2);
int oracle_run_windows(OracleSystem *s, int n_rounds, OracleMoveRecord *records);
/* The same with `proposals` (1..16) slots per window: every step of a window
 * is slots 0..proposals-1 making one move each, in slot order, slot p from
 * Local stream 0x100 + 64 p + w; records [round][window][step][slot]. */
int oracle_run_proposals(OracleSystem *s, int n_rounds, int proposals, OracleMoveRecord *records);
uint64_t oracle_rng_position(OracleSystem *s);
/* Ulong / dUlong quintic tables [levels][points][6]; sets UseLongRange. */
void oracle_set_ulong(OracleSystem *s, int levels, int points, double delta, const double *ulong,
                      const double *dulong);
/* ActionsClass::Energy terms on the OLD copy: {kinetic, dUShort, dULong,
 * vShort, vLong (0), (kinetic+dUShort+dULong)/M}. */
void oracle_energy(OracleSystem *s, double *out);
/* PairCorrelationClass::Accumulate on the OLD copy into hist[num_points-1]. */
void oracle_gofr_accumulate(OracleSystem *s, double start, double end, int num_points, uint64_t *hist);

#ifdef __cplusplus
}
#endif
#endif

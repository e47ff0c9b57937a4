/*
 * pimc_b200.h — C ABI of the B200 (sm_100a) action-evaluation library for
 * PIMC++ path-integral Monte Carlo.
 *
 * The library owns device copies of the path (OLD/NEW mirrored, like
 * MirroredClass), the pair-action tables and the rho_k cache, and evaluates
 * the actions a bisection move needs.  Plain pointers and sizes only; every
 * entry point returns an int status (0 = PIMC_OK) instead of throwing.  The
 * one failure not turned into a status is a set-up call running out of host
 * memory for the tables it builds, which ends the process; the file readers
 * return PIMC_E_NOMEM for that too.  A context is not thread-safe: one
 * context per host thread, one CUDA stream per context.
 *
 * Path layout everywhere: row-major [slice][particle][3] doubles, with
 * num_time_slices = M+1 rows, the layout of PathClass::Path (Blitz
 * Array<dVec,2>, PathClass.cc:295-443).
 *
 * Reference interfaces replaced (paths relative to the reference root):
 *   ActionBaseClass::SingleAction / d_dBeta      PIMC++/src/Actions/ActionBase.h:43,57
 *   ShortRangeClass::SingleAction / d_dBeta      PIMC++/src/Actions/ShortRangeClass.cc:191,316
 *   KineticClass::SingleAction / d_dBeta         PIMC++/src/Actions/KineticClass.cc:33,187
 *   LongRangeClass::SingleAction / d_dBeta       PIMC++/src/Actions/LongRangeClass.cc:273,374
 *   PathClass::UpdateRho_ks                      PIMC++/src/PathClass.cc:649
 *   PathClass::AcceptCopy / RejectCopy           PIMC++/src/PathClass.cc:797,865
 *   DavidPAClass::Read(…Daviddmfile…)            Common/PairAction/DavidPAClass.h:144
 *   PAtricubicFitClass::Read                     Common/PairAction/PAtricubicFit.cc:794
 *   BisectionBlockClass::MakeMove                PIMC++/src/Moves/BisectionBlock.cc:380
 */
#ifndef PIMC_B200_H
#define PIMC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define PIMC_OK 0
#define PIMC_E_ARG 1      /* invalid argument (sizes, indices, null pointers) */
#define PIMC_E_CUDA 2     /* a CUDA runtime call failed */
#define PIMC_E_NAN 3      /* a kernel produced a non-finite action */
#define PIMC_E_INDEX 4    /* a kernel saw an out-of-range index and skipped it */
#define PIMC_E_CAP 5      /* a bounded device loop hit its iteration cap */
#define PIMC_E_FILE 6     /* an input file is missing or malformed */
#define PIMC_E_STATE 7    /* call out of order (e.g. no pair action set) */
#define PIMC_E_NOMEM 8    /* device or host allocation failed */
#define PIMC_E_STAGING 9  /* |S| > 1e50 on an accepted stage (StageClass.cc:74-85) */

/* ---- enumerations ---- */
#define PIMC_OLD 0
#define PIMC_NEW 1
#define PIMC_BOTH 2

#define PIMC_FP64 0   /* plain FP64 evaluation */
#define PIMC_MIXED 1  /* FP32 pair terms and phases, FP64 accumulation and Metropolis */

/* Guard of the mixed path (pimc_bisection_desc.mixed_guard, pimc_batch_set_guard).
 * Every mixed stage sum carries a rigorous bound E on its distance from the
 * FP64 sums.  DECISION: a stage whose Metropolis decision could come out
 * differently on the FP64 sums (|logAcceptProb - log u| <= E plus the
 * previous stage's bound) is evaluated again in FP64 and decided on those
 * sums, so decisions, trace and path are the FP64 path's.  RELATIVE: as
 * DECISION, and also every stage with E > 1e-6 |dS| is decided on its FP64
 * sums, so every dS a decision uses is within 1e-6 relative of FP64's.
 * NONE: the mixed sums alone. */
#define PIMC_GUARD_DECISION 0
#define PIMC_GUARD_NONE 1
#define PIMC_GUARD_RELATIVE 2

#define PIMC_ACTION_SHORTRANGE 0
#define PIMC_ACTION_KINETIC 1
#define PIMC_ACTION_LONGRANGE 2
#define PIMC_ACTION_DAVIDLONGRANGE 3 /* DavidLongRangeClassYk (pimc_davidlongrange_yk) */

#define PIMC_GRID_LINEAR 0
#define PIMC_GRID_LOG 1

typedef struct pimc_context pimc_context;

/* The system a context simulates: PathClass::Read (PathClass.cc:123-278) and
 * SpeciesClass::Read (SpeciesClass.cc:19-60) after input parsing. */
typedef struct pimc_system_desc {
  int num_particles;        /* N over all species */
  int num_time_slices;      /* path rows, M+1 on one process (PathClass.cc:305) */
  double box[3];            /* periodic box (all three dimensions periodic) */
  double tau;               /* imaginary-time step */
  int num_species;
  const int *species_of;    /* [num_particles] species of each particle */
  const double *lambda;     /* [num_species] hbar^2/(2m) */
  int num_images;           /* Action{NumImages} for kinetic/sampling image sums */
  int device;               /* CUDA device ordinal */
} pimc_system_desc;

const char *pimc_status_string(int status);
int pimc_version(void);

/* Creates a context on desc->device: allocates the path copies and a stream. */
int pimc_create(const pimc_system_desc *desc, pimc_context **out);
int pimc_destroy(pimc_context *ctx);
/* Copies the last error message of this context into buf (NUL-terminated). */
int pimc_last_error(pimc_context *ctx, char *buf, int len);

/* ---- pair actions: PairMatrix(sp1,sp2) of ActionsClass (ActionsClass.cc:147-211) ---- */

/* A DavidPAClass fit from an ASCII squarer .dm file (DavidPAClass.cc:635-912):
 * the NMax==2 fit, column 0 = potential, last grid row zeroed, natural start /
 * zero-slope end splines, TauPos chosen from desc->tau.  num_offdiag_terms is
 * Fits{NumOffDiagonalTerms} of the PairAction section. */
int pimc_pa_david_from_dm(pimc_context *ctx, int sp1, int sp2, const char *dm_path,
                          int num_offdiag_terms);

/* Host-only (no GPU needed): the reader behind pimc_pa_david_from_dm.
 * pimc_dm_read_info reports the table shape; pimc_dm_read_tables fills
 * [num_tau][num_grid][num_cols] arrays: ukj values and second derivatives,
 * dukj values and second derivatives (any pointer may be NULL). */
int pimc_dm_read_info(const char *dm_path, double desired_tau, int *num_grid, int *num_cols, int *num_tau,
                      int *tau_pos, int *grid_type, double *grid_start, double *grid_end);
int pimc_dm_read_tables(const char *dm_path, double desired_tau, double *ukj, double *ukj_d2, double *dukj,
                        double *dukj_d2);

/* The same fit from arrays already read: ukj and dukj are
 * [num_tau][num_grid][num_cols] with column 0 the potential (the tempUkj2 /
 * tempdUkj2 arrays of ReadDavidSquarerFile). */
int pimc_pa_david(pimc_context *ctx, int sp1, int sp2, int grid_type, double grid_start,
                  double grid_end, int num_grid, int num_cols, int num_tau, const double *ukj,
                  const double *dukj, int tau_pos, int num_offdiag_terms);

/* A PAtricubicFitClass fit (PAtricubicFit.cc:659-721,794-865): linear q, y, t
 * grids given as {start, end, n}; umat/dumat are [num_betas][nq][ny][nt] node
 * values for beta = smallest_beta * 2^level; the potential for the primitive
 * fallback is a natural cubic spline (SplinePot, Common/PH/SplinePot.cc) on a
 * linear grid {pot_start, pot_end, pot_n}, zero beyond pot_end. */
int pimc_pa_tricubic(pimc_context *ctx, int sp1, int sp2, const double qgrid[3],
                     const double ygrid[3], const double tgrid[3], int num_betas,
                     double smallest_beta, const double *umat, const double *dumat, double pot_start,
                     double pot_end, int pot_n, const double *pot_data);

/* ---- path state (PathClass / MirroredClass) ---- */
int pimc_set_path(pimc_context *ctx, int copy, const double *path);
int pimc_get_path(pimc_context *ctx, int copy, double *path);

/* Host-only (no GPU needed): PathClass::InitRandomFixed
 * (PIMC++/src/InitPaths.cc:966-999).  Places num_particles points uniformly
 * in the box from the World stream of `seed` (Philox-4x32-10, stream 2,
 * drawn in the reference's order), each at least 2*radius (minimum image)
 * from the earlier ones; writes positions[num_particles][3].  Returns
 * PIMC_E_CAP where the reference aborts: a particle that took 1000 tries. */
int pimc_init_random_fixed(const double box[3], int num_particles, double radius, uint64_t seed,
                           double *positions);

/* Host-only: element `index` of the library's Philox-4x32-10 stream `stream`
 * under `seed`, a double in [0, 1) (the draw RandomClass::Local/Common/World
 * make, Common/Random/Random.h:33-49).  Streams 0, 1, 2 are Local, Common,
 * World; 3 serves host-side ShiftMove draws; 0x100 + 64p + w are the windows'
 * and proposal slots' Local streams. */
int pimc_stream_uniform(uint64_t seed, uint32_t stream, uint64_t index, double *out);

/* PathClass::ShiftPathData on one process (PIMC++/src/PathClass.cc:1026-1110),
 * the data step of ShiftMoveClass::MakeMove (PIMC++/src/Moves/MetaMoves.cc:39-65):
 * row j of both copies becomes row (j - slices_to_shift) mod M of OLD,
 * M = num_time_slices - 1.  Call between moves (OLD == NEW); rho_k and the
 * neighbour lists are rebuilt by the next device moves. */
int pimc_shift_data(pimc_context *ctx, int slices_to_shift);

/* ShiftMoveClass::MakeMove (PIMC++/src/Moves/MetaMoves.cc:39-65): draws
 * CommonInt(M) = floor(u * M) slices, u from stream 3 of the pimc_rng_seed key
 * at the context's own draw counter, and calls pimc_shift_data.  Writes the
 * shift to *slices_shifted (may be NULL). */
int pimc_shift_move(pimc_context *ctx, int *slices_shifted);

/* Flat-binary checkpoint of a chain: both path copies, every Local/window
 * RNG stream position with its Gaussian cache, the move counters and the
 * concurrent-window round counter, the seed and the ShiftMove draw counter.  Replaces the reference's HDF5 path dump
 * and InitPaths = "RESTART" (PIMC++/src/InitPaths.cc:826-845).  Reading
 * checks that N, slices, box, tau and lambda equal the context's
 * (PIMC_E_ARG otherwise, PIMC_E_FILE for a missing or malformed file); a
 * chain continued from its checkpoint makes the same moves as the chain
 * that wrote it.  Read it after pimc_bisection_setup and pimc_rng_seed: setup
 * clears the move counters and seeding resets the streams. */
int pimc_checkpoint_write(pimc_context *ctx, const char *filename);
int pimc_checkpoint_read(pimc_context *ctx, const char *filename);

/* ---- ActionBaseClass drop-in ---- */

/* ActionBaseClass::SingleAction(slice1, slice2, activeParticles, level) of the
 * action `action` on path copy `copy` (the reference's global ActiveCopy made
 * explicit).  Short-range and kinetic sum links [slice1, slice2) with step
 * 2^level; the long-range action sums slices [slice1, slice2] and, on the NEW
 * copy, first updates rho_k like LongRangeClass::SingleAction. */
int pimc_single_action(pimc_context *ctx, int action, int copy, int slice1, int slice2,
                       const int *active, int n_active, int level, int precision, double *out);

/* ActionBaseClass::d_dBeta(slice1, slice2, level) on the OLD copy. */
int pimc_d_dbeta(pimc_context *ctx, int action, int slice1, int slice2, int level, double *out);

/* PathClass::AcceptCopy / RejectCopy for slices [slice1, slice2] of the active
 * particles (PutInBoxFast on NEW, then NEW->OLD; or OLD->NEW), rho_k included. */
int pimc_accept_copy(pimc_context *ctx, int slice1, int slice2, const int *active, int n_active);
int pimc_reject_copy(pimc_context *ctx, int slice1, int slice2, const int *active, int n_active);

/* ---- long range (PathClass k-vectors, rho_k; LongRangeClass tables) ---- */

/* PathClass::SetupkVecs3D (PathClass.cc:534-586); returns the count in *num_k. */
int pimc_setup_kvecs(pimc_context *ctx, double kcutoff, int *num_k);
int pimc_get_kvecs(pimc_context *ctx, double *kvecs /* [num_k][3] */);
/* The breakup output of LongRangeClass::Init for the single species pair:
 * arrays over levels (and k for *_k, [num_levels][num_k]). */
int pimc_set_longrange(pimc_context *ctx, int num_levels, const double *ulong_k,
                       const double *ulong_r0, const double *ushort_k0, const double *ulong_k0,
                       const double *dulong_k, const double *dulong_r0, const double *dushort_k0,
                       const double *dulong_k0, int use_background);
/* PathClass::UpdateRho_ks() full recompute (PathClass.cc:710-718), and the
 * incremental UpdateRho_ks(slice1, slice2, active, level) (:649-707). */
int pimc_calc_rhok(pimc_context *ctx);
int pimc_update_rhok(pimc_context *ctx, int slice1, int slice2, const int *active, int n_active,
                     int level);
int pimc_get_rhok(pimc_context *ctx, int copy, double *out /* [slices][num_k][2] */);
/* DavidLongRangeClassYk (Actions/DavidLongRangeClassYk.cc:38-126), one
 * species: uk, duk and Vlong_k of the k-vectors from the squarer's k-space
 * action uk_long at the magnitudes kvals (the .dm LongRange section read by
 * DavidPAClass::ReadLongRangeHDF5, DavidPAClass.cc:914-950).  rpa = 1: the
 * single-type RPA construction (BuildRPA_SingleType), 0: Build_MultipleSpecies
 * (uk = tau uk_long/Omega, duk = Vlong_k = uk_long/Omega).  Every k-vector's
 * |k| must be in kvals (within 1e-10).  Then PIMC_ACTION_DAVIDLONGRANGE in
 * pimc_single_action / pimc_d_dbeta (d_dBeta ignores the level, as the
 * reference), and DavidLongRangeClassYk::V (:367-389): */
int pimc_davidlongrange_yk(pimc_context *ctx, int num_kvals, const double *kvals, const double *uk_long,
                           int rpa);
int pimc_davidlongrange_v(pimc_context *ctx, int slice1, int slice2, double *out);

/* ---- device-resident bisection moves (BisectionBlockClass::MakeMove) ---- */

/* Move schedules.  SEQUENTIAL is the reference's: one move at a time, the
 * window start drawn from the Local stream (ChooseTimeSlices).  WINDOWS runs
 * one round per block: a Common-stream offset o in [0, 2^L) and concurrent
 * BisectionBlocks on the disjoint windows [o + w 2^L, o + (w+1) 2^L], each
 * with its own Local stream (PIMC++'s time-slice parallelism on one GPU).
 * PROPOSALS is WINDOWS with P = cluster_ctas concurrent moved-particle
 * proposals per window: every step of a window is slots 0..P-1 each making
 * one move from its own Local stream, with the result of making them one
 * after another in slot order (a slot whose move read a particle that an
 * earlier slot's accepted move changed is made again).  Short range only
 * (use_longrange 0); with neighbour lists most slots are independent. */
#define PIMC_SCHEDULE_SEQUENTIAL 0
#define PIMC_SCHEDULE_WINDOWS 1
#define PIMC_SCHEDULE_PROPOSALS 2

typedef struct pimc_bisection_desc {
  int num_levels;                   /* Move{NumLevels} */
  int steps_per_block;              /* Move{StepsPerBlock} */
  int shortrange_at_higher_levels;  /* ShortRange in HigherLevelActions */
  int use_longrange;                /* LongRange pushed at the lowest level */
  int precision;                    /* PIMC_FP64 or PIMC_MIXED */
  int shadow;                       /* also evaluate the other precision, for dS error */
  int cluster_ctas;                 /* CTAs cooperating on one chain (1..16), 0 = auto;
                                       PROPOSALS: proposal slots per window (2..16), one CTA each */
  int threads_per_cta;              /* 0 = auto */
  int schedule;                     /* PIMC_SCHEDULE_SEQUENTIAL, _WINDOWS or _PROPOSALS */
  /* Neighbour lists for the short-range sum (the role of ShortRangeOnClass's
   * cells, Actions/ShortRangeOnClass.cc:35-240), DavidPA only: > 0 turns
   * them on with this skin (length units of the box) around each particle's
   * path; results equal the all-partner sum, since a DavidPA table is zero
   * beyond its grid end.  neighbor_max: list capacity per particle (0 = 1024);
   * a particle with more partners uses all of them. */
  double neighbor_skin;
  int neighbor_max;
  /* PIMC_MIXED only: PIMC_GUARD_DECISION (0, default), PIMC_GUARD_NONE or
   * PIMC_GUARD_RELATIVE; stats.reevaluated counts the stages decided on
   * their FP64 re-evaluation. */
  int mixed_guard;
  /* Tries of the table-staging wait (a bounded spin on an mbarrier) before a
   * launch gives up with PIMC_E_CAP; 0 = 2^22.  test_wait > 0 additionally
   * waits that many tries on a barrier that nothing arrives at, after the
   * table copy has landed, so the give-up path and its status can be tested
   * without a fault; 0 in normal use. */
  int wait_cap;
  int test_wait;
} pimc_bisection_desc;

/* One move: the fields the accept trace is compared on. */
typedef struct pimc_move_record {
  int32_t slice1;
  int32_t ptcl;
  int32_t accepted;       /* whole move accepted */
  int32_t stages_passed;  /* bisection stages accepted */
  double dS[8];           /* S_new - S_old per stage attempted, highest level first, in the
                             run's precision (PIMC_MIXED: the mixed sums) */
  double dS_shadow[8];    /* the same in the other precision (shadow mode), else 0 */
  float dS_bound[8];      /* PIMC_MIXED: bound on |dS - dS of the FP64 sums|, else 0 */
  int32_t reevaluated;    /* bit i: stage i was decided on its FP64 re-evaluation */
  int32_t pad;
} pimc_move_record;

typedef struct pimc_bisection_stats {
  int64_t moves;
  int64_t accepted;
  int64_t stages_attempted;
  int64_t pair_evals;     /* U(q,z,s^2) evaluations, old+new, all stages attempted */
  int64_t flips;          /* shadow mode: stage decisions the other precision would flip */
  int32_t status;         /* device status word: 0, PIMC_E_NAN, PIMC_E_STAGING, PIMC_E_CAP */
  int32_t pad;
  int64_t redone;         /* PROPOSALS: moves discarded and made again (not in moves) */
  int64_t reevaluated;    /* PIMC_MIXED: stages decided on their FP64 re-evaluation */
} pimc_bisection_stats;

int pimc_bisection_setup(pimc_context *ctx, const pimc_bisection_desc *desc);
/* Seeds the chain's streams (Philox-4x32-10 key; counters reset): the Local
 * stream of the sequential schedule and the per-window streams. */
int pimc_rng_seed(pimc_context *ctx, uint64_t seed);
/* Window slots per round of the WINDOWS and PROPOSALS schedules:
 * min(floor((slices-1) / 2^L), 64). */
int pimc_bisection_windows(pimc_context *ctx, int *windows);
/* Runs n_blocks BisectionBlocks on the device (OLD copy is the state; NEW is
 * brought back in sync afterwards).  SEQUENTIAL: n_blocks*steps_per_block
 * moves.  WINDOWS: n_blocks rounds of windows*steps_per_block moves; the
 * trace slots of windows that do not fit a round have slice1 = -1.
 * PROPOSALS: n_blocks rounds of windows*steps_per_block*P moves, records
 * [round][window][step][slot].
 * trace: that many records or NULL.  stats: accumulated since setup. */
int pimc_run_bisection(pimc_context *ctx, int n_blocks, pimc_move_record *trace,
                       pimc_bisection_stats *stats);
/* Enqueues n_blocks moves on the context stream without synchronising or
 * copying anything back (for timing); pimc_bisection_stats reads the totals. */
int pimc_run_bisection_async(pimc_context *ctx, int n_blocks);
int pimc_bisection_get_stats(pimc_context *ctx, pimc_bisection_stats *stats);
/* Clusters of the configured shape that can be resident at once (window
 * clusters beyond this run in a second wave). */
int pimc_bisection_occupancy(pimc_context *ctx, int *max_active_clusters);
int pimc_synchronize(pimc_context *ctx);
/* The CUDA stream of the context (cudaStream_t as void*). */
void *pimc_stream(pimc_context *ctx);

/* ---- many independent chains in one persistent launch ----
 * The reference runs independent Markov chains as clones, one per MPI
 * group (PathDataClass.cc:244-268).  Here a batch holds chains of uneven
 * N, M and tau, each a sequential-schedule BisectionBlock driver with a
 * DavidPA diagonal action u_00(r; tau_l) (no off-diagonal terms) on its own
 * linear grid; one launch runs n_blocks blocks of moves on every chain, the
 * chains taken by CTAs from an atomic queue, largest first. */
typedef struct pimc_batch pimc_batch;

typedef struct pimc_chain_desc {
  int num_particles;        /* N */
  int num_time_slices;      /* path rows, M+1 */
  double box[3];
  double tau;
  double lambda;            /* hbar^2/(2m), one species */
  int num_images;
  int num_levels;           /* Move{NumLevels} */
  int steps_per_block;      /* Move{StepsPerBlock} */
  uint64_t seed;            /* Local stream key */
  double grid_start, grid_end;
  int num_grid;
  int num_tau;              /* tables for tau * 2^l, l = 0..num_tau-1 */
  int tau_pos;              /* level of this chain's tau in the tables */
  const double *u00;        /* [num_tau][num_grid] diagonal action (host) */
  const double *path;       /* [num_time_slices][N][3] initial path (host) */
} pimc_chain_desc;

int pimc_batch_create(int device, int n_chains, const pimc_chain_desc *chains, pimc_batch **out);
int pimc_batch_destroy(pimc_batch *b);
int pimc_batch_last_error(pimc_batch *b, char *buf, int len);
/* precision: PIMC_FP64 or PIMC_MIXED; threads_per_cta 64..512 (0 = 256);
 * ctas: persistent CTAs (0 = every CTA that fits, capped at the chain count).
 * Chains run largest first (cost N * 2^levels * steps_per_block).  A CTA
 * runs the costliest chains with all its threads; with max_split = 1 or 2 it
 * divides into 2 or 4 groups, each running its own chain, for the chains
 * whose cost is at most split_ratio (split_ratio^2) of the largest.  Groups
 * must keep 64+ threads, a multiple of 32. */
int pimc_batch_config(pimc_batch *b, int precision, int shadow, int threads_per_cta, int ctas, int max_split,
                      double split_ratio);
/* n_blocks blocks of moves on every chain; trace: [chain][n_blocks*steps]
 * records (chains with fewer steps leave zeros) or NULL; stats: totals. */
int pimc_batch_run(pimc_batch *b, int n_blocks, pimc_move_record *trace, pimc_bisection_stats *stats);
/* Enqueues n_blocks blocks of moves on every chain, no sync.  The launch is
 * captured once as a CUDA graph and replayed while n_blocks and the
 * configuration stay the same. */
int pimc_batch_run_async(pimc_batch *b, int n_blocks);
/* Times n_blocks blocks under each candidate threads_per_cta (128, 256,
 * 384, 512) x max_split (0..2) x split_ratio (1/2, 1/4) with every CTA that
 * fits, keeps the fastest with the current precision and shadow setting,
 * and puts the chains back in their state from before the probes.  Outputs
 * may be NULL. */
int pimc_batch_autotune(pimc_batch *b, int n_blocks, int *threads_per_cta, int *ctas, int *max_split,
                        double *split_ratio, double *ms);
int pimc_batch_get_stats(pimc_batch *b, int chain /* -1: all */, pimc_bisection_stats *stats);
/* PIMC_MIXED: the guard of the batch's chains, PIMC_GUARD_DECISION (the
 * default), PIMC_GUARD_NONE or PIMC_GUARD_RELATIVE. */
int pimc_batch_set_guard(pimc_batch *b, int guard);
int pimc_batch_get_path(pimc_batch *b, int chain, double *path);
int pimc_batch_synchronize(pimc_batch *b);
/* The batch's CUDA stream (cudaStream_t) for event timing and ordering. */
void *pimc_batch_stream(pimc_batch *b);

/* ---- classical Coulomb pair action and the optimized Ewald breakup ---- */

/* PAclassicalFitClass with a CoulombPot (Common/PairAction/PAclassicalFit.cc:
 * 57-75, 175-288): U = beta_l Z1Z2 / q, dU = Z1Z2 / q, beta_l = tau 2^l for
 * l < num_levels.  Without pimc_longrange_coulomb nothing is subtracted. */
int pimc_pa_coulomb(pimc_context *ctx, int sp1, int sp2, double z1z2, int num_levels);

/* LongRangeClass::Init's OptimizedBreakup_U and _dU (PIMC++/src/Actions/
 * LongRangeClass.cc:482-868) for the Coulomb pair action: LPQHI basis on
 * num_knots knots to r_c = L/2, the k-space fit beyond the pimc_setup_kvecs
 * cutoff, Ulong(r) / dUlong(r) natural quintic splines on the 1000-point
 * LongGrid, and the k = 0 integrals (host, FP64).  Loads the long-range
 * tables (as pimc_set_longrange) and turns on the 1/2 (Ulong(r) + Ulong(r'))
 * subtraction in ShortRange (ShortRangeClass.cc:211-214, 282-286). */
int pimc_longrange_coulomb(pimc_context *ctx, int num_knots, int use_background);

/* The same breakup without a context (host only): tables for num_k
 * k-vectors [num_k][3]; ulong_k/dulong_k [levels][num_k]; the per-level
 * scalars [levels]; ulong_r/dulong_r [levels][1000][6] Taylor coefficients of
 * the quintic splines on the grid [0, *rmax]. Any output may be NULL. */
int pimc_coulomb_breakup(const double box[3], double z1z2, double smallest_beta, int num_levels, int num_knots,
                         double kcutoff, int num_k, const double *kvecs, double *ulong_k, double *dulong_k,
                         double *ulong_r0, double *dulong_r0, double *ushort_k0, double *dushort_k0,
                         double *ulong_k0, double *dulong_k0, double *rmax, double *ulong_r, double *dulong_r);
/* Natural quintic interpolating spline (third and fourth derivatives zero at
 * both ends; QuinticSpline without end derivatives) of y[n] on a uniform
 * grid of spacing h: coef[n][6] Taylor coefficients of each interval at its
 * left knot, host only. */
int pimc_quintic_spline(int n, double h, const double *y, double *coef);

/* ---- observables (on the OLD copy) ---- */

/* The terms of ActionsClass::Energy (ActionsClass.cc:812-871) for the whole
 * path: kinetic = KineticClass::d_dBeta(0, M, 0), du_short =
 * ShortRangeClass::d_dBeta(0, M, 0), du_long = LongRangeClass::d_dBeta
 * (0 without pimc_set_longrange), v_short = sum over slices 0..M of
 * ShortRangePotClass::V(slice) with weight 1/2 at slices 0 and M
 * (ShortRangePotClass.cc:28-47), v_long = 0 (LongRangePotClass is not
 * built), and total = (kinetic + du_short + du_long) / M, the per-slice
 * sample EnergyClass::Accumulate adds (ObservableEnergy.cc:45-73). */
typedef struct pimc_energy_terms {
  double kinetic, du_short, du_long, v_short, v_long, total;
} pimc_energy_terms;
int pimc_energy(pimc_context *ctx, pimc_energy_terms *out);

/* PairCorrelationClass (ObservableCorrelation.cc:36-224), one species: a
 * linear grid {start, end, num_points} (end <= 0: the box side, the
 * reference's default), num_points - 1 <= 12288 bins.  accumulate adds the
 * OLD path's histogram of pair distances over slices 0..M-1 (enqueued, no
 * sync); get returns the counts, g(r) normalised as WriteBlock does and the
 * number of accumulated samples. */
int pimc_gofr_setup(pimc_context *ctx, double start, double end, int num_points);
int pimc_gofr_accumulate(pimc_context *ctx);
int pimc_gofr_get(pimc_context *ctx, uint64_t *histogram, double *gofr, long long *total_counts);
int pimc_gofr_reset(pimc_context *ctx);

/* ---- measurement ----
 * No counterpart in the reference: the read-bandwidth ceiling used to state
 * the bisection kernels' roofline when their tables and path are
 * L2-resident.  Reads `bytes` (1 MiB .. 8 GiB) of a fresh device buffer with
 * 16-byte loads through L2, once untimed, then `reps` launches of `passes`
 * passes each (1..1024) timed with CUDA events; *gbs = bytes * passes * reps
 * / time.  Below the 126 MB L2 this is the L2 read bandwidth, far above it
 * the HBM read bandwidth.  Allocates and frees its buffer; synchronous. */
int pimc_read_bandwidth(int device, size_t bytes, int passes, int reps, double *gbs);

/* ---- allocation-free ShortRange SingleAction ----
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc (an application whose memory pool owns every device
 * allocation, an embedding that forbids allocation after start-up, a
 * latency-critical loop that must not pay for cudaMalloc's implicit device
 * synchronisation).  It needs no context: every
 * buffer is the caller's device memory — path [num_time_slices][N][3]
 * doubles, diag the (y, d2y) pairs of u_00 for this level [num_grid][2] on a
 * LINEAR grid {grid_start, grid_end, num_grid} (DavidPA, no off-diagonal
 * terms: a table with off-diagonal u_kj terms gives a wrong value, not an
 * error), out one double — and active/box are host arrays.  An empty link
 * range (slice1 == slice2) writes 0.  Its scratch is a
 * fixed file-scope device array (2048 block partials, about 16 KB, held by
 * every GPU that loads the library until exit), so n_active * N * links must
 * not exceed 524288 (PIMC_E_ARG otherwise).  Calls share that scratch: calls
 * that overlap on the GPU race, so keep them on one stream.  The first call
 * on a device looks up the scratch address; make it before any stream
 * capture.  Enqueued on `stream` (cudaStream_t, NULL = default), no sync. */
int pimc_shortrange_single_noalloc(const double *path, int num_particles, int num_time_slices,
                                   const double box[3], const double *diag, double grid_start,
                                   double grid_end, int num_grid, int slice1, int slice2, const int *active,
                                   int n_active, int level, double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif

// Launch interface of the device-resident bisection kernel (bisection.cu).
#pragma once

#include <cuda_runtime.h>

#include "pimc_internal.h"

namespace pimc {

struct BisectionArgs {
  double *path;               // OLD path copy, the chain state
  DevSystem sys;
  DevPA pa;
  ChainState *chains;         // [1] sequential, [windows] concurrent
  pimc_move_record *trace;    // device trace or nullptr
  long long trace_offset;
  int num_levels, steps_per_block, n_blocks, sr_higher;
  int concurrent;             // 0: sequential schedule; 1: concurrent windows, one round per launch
  // Concurrent windows with P > 1 proposal slots per window (DavidPA): the
  // cluster of a window has P CTAs, CTA p runs slot p from ChainState
  // p * kMaxWindows + w.  0 or 1: one proposal per window.
  int proposals;
  double pair_range;          // DavidPA: pair terms are zero from this distance on (the grid end)
  unsigned long long round;   // Common-stream index of this round (concurrent)
  // LongRangeClass::SingleAction in the lowest stage (BisectionBlock.cc:92-103):
  // rho_k of the OLD path [slice][k], the k-vectors [k][3] and Ulong_k of level 0
  double2 *rhok;
  const double *kvec;
  const double *ulong_k0;
  int nk, use_lr;
  // Neighbour lists of the short-range sum (0: all partners): per particle the
  // bounding sphere of its path {c, B} and the partners j with
  // |c_i - c_j| <= range + B_i + B_j in ascending order (count -1: overflow)
  int nbr_on, nbr_kmax;
  const double4 *nbr_cb;
  const int *nbr_cnt, *nbr_idx;
  int *nbr_dirty;
  // Mixed path: kGuardOff, kGuardDecision (decide on the FP64 re-evaluation
  // of a stage whenever the decision could differ from the FP64 sums' within
  // the mixed sums' error bound) or kGuardRelative (also when the bound
  // exceeds 1e-6 |dS|).
  int guard;
  // Tries of the table-staging wait before it gives up with PIMC_E_CAP;
  // test_wait > 0 also waits that many tries on a barrier nothing arrives at
  // (after the copy has landed), to exercise the give-up path.
  int wait_cap, test_wait;
};

// Neighbour lists for the device moves (neighbors.cu): rebuilt from the
// current path when *dirty is set, then *dirty cleared.
cudaError_t launch_nbr_rebuild(cudaStream_t st, const double *path, const DevSystem &sys, double range, double skin,
                               int kmax, double4 *cb, int *cnt, int *idx, int *dirty);

constexpr int kGuardOff = 0, kGuardDecision = 1, kGuardRelative = 2;
// The kernel's guard mode of a PIMC_GUARD_* value.
inline int guard_mode(int pimc_guard) {
  return pimc_guard == PIMC_GUARD_NONE ? kGuardOff : pimc_guard == PIMC_GUARD_RELATIVE ? kGuardRelative : kGuardDecision;
}

cudaError_t bisection_occupancy(const BisectionArgs &a, int precision, int shadow, int cluster_ctas, int threads,
                                int *max_clusters);
// Many chains in one persistent launch: jobs[] (one sequential-schedule job
// per chain, each with its own path, tables and ChainState), taken in the
// order order[] through the atomic counter *queue (zero at launch).
constexpr int kMaxSplit = 2;  // a CTA runs up to 2^kMaxSplit chains side by side

struct BatchArgs {
  const BisectionArgs *jobs;
  const int *order;
  unsigned int *queue;
  int n_chains;
  int n_blocks;                 // blocks of moves each chain runs in this launch
  pimc_move_record *trace;      // [chain][n_blocks * steps_per_block] or nullptr
  long long trace_per_chain;
  int max_split;                // finest group level used, 0..kMaxSplit
  int split[kMaxSplit];         // queue positions from which level k+1 groups run the chains
  unsigned dyn_per_slot;        // shared-memory bytes of one slot's staged tables (multiple of 16)
};

cudaError_t launch_batch(const BatchArgs &b, int precision, int shadow, int blocks, int threads, size_t dyn,
                         cudaStream_t st);
cudaError_t batch_occupancy(int precision, int shadow, int threads, size_t dyn, int *blocks_per_sm);

size_t bisection_dyn_smem(const BisectionArgs &a, int precision, int shadow);
cudaError_t launch_bisection(const BisectionArgs &a, int precision, int shadow, int cluster_ctas, int clusters,
                             int threads, cudaStream_t st);

}  // namespace pimc

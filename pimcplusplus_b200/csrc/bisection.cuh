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
  unsigned long long round;   // Common-stream index of this round (concurrent)
};

cudaError_t bisection_occupancy(const BisectionArgs &a, int precision, int shadow, int cluster_ctas, int threads,
                                int *max_clusters);
size_t bisection_dyn_smem(const BisectionArgs &a, int precision, int shadow);
cudaError_t launch_bisection(const BisectionArgs &a, int precision, int shadow, int cluster_ctas, int clusters,
                             int threads, cudaStream_t st);

}  // namespace pimc

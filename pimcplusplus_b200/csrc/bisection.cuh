// Launch interface of the device-resident bisection kernel (bisection.cu).
#pragma once

#include <cuda_runtime.h>

#include "pimc_internal.h"

namespace pimc {

struct BisectionArgs {
  double *path;               // OLD path copy, the chain state
  DevSystem sys;
  DevPA pa;
  ChainState *chain;
  pimc_move_record *trace;    // device trace or nullptr
  long long trace_offset;
  int num_levels, steps_per_block, n_blocks, sr_higher;
};

cudaError_t launch_bisection(const BisectionArgs &a, int precision, int shadow, int cluster_ctas, int threads,
                             cudaStream_t st);

}  // namespace pimc

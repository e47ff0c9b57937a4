// Launch interface of the action-level kernels (action_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "pimc_internal.h"

namespace pimc {

// Active particles of one call, passed by value.
struct ActiveList {
  int n;
  int p[kMaxActive];
};

// Where a reduction kernel leaves its result: per-block partials, a
// completion counter (left at zero) and the scalar output, all on the device.
struct ReduceTarget {
  cudaStream_t stream;
  double *partials;
  unsigned int *counter;
  double *out;
};

cudaError_t launch_sr_single(const ReduceTarget &t, const double *path, const DevSystem &sys, const DevPA &pa,
                             const ActiveList &act, int slice1, int skip, int nlinks, int level, int precision,
                             int sm_count);
cudaError_t launch_sr_dbeta(const ReduceTarget &t, const double *path, const DevSystem &sys, const DevPA &pa,
                            int slice1, int skip, int nlinks, int level, int sm_count);
cudaError_t launch_kin_single(const ReduceTarget &t, const double *path, const DevSystem &sys, const ActiveList &act,
                              int slice1, int skip, int nlinks, int level, int sm_count);
cudaError_t launch_kin_dbeta(const ReduceTarget &t, const double *path, const DevSystem &sys, int slice1, int skip,
                             int nlinks, int level, int sm_count);
// Linear histogram grid of the pair correlation (num_points - 1 bins).
struct GofrGrid {
  double start, end, deltainv;
  int nbins;
};
// Pair observables of the OLD path: V summed into t.out (do_v) and/or the
// g(r) histogram added to hist (gg non-null, <= 12288 bins).
cudaError_t launch_pair_obs(const ReduceTarget &t, const double *path, const DevSystem &sys, const DevPA &pa,
                            bool do_v, const GofrGrid *gg, unsigned long long *hist, int sm_count);
cudaError_t launch_accept(cudaStream_t st, double *path_old, double *path_new, const DevSystem &sys,
                          const ActiveList &act, int slice1, int slice2);
cudaError_t launch_reject(cudaStream_t st, const double *path_old, double *path_new, const DevSystem &sys,
                          const ActiveList &act, int slice1, int slice2);

}  // namespace pimc

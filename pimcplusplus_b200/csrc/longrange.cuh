// Long-range (k-space) kernels: launch interface (longrange.cu).
#pragma once

#include <cuda_runtime.h>

#include "action_kernels.cuh"
#include "pimc_internal.h"

namespace pimc {

// k-vectors of PathClass::SetupkVecs3D for the kernels: indices into the
// per-dimension phase tables, offset by kmax (PathClass.cc:567-585).
struct LRDesc {
  int nk;
  int kmax[3];
  int coff[3];     // offset of dimension d's table in the packed phase tables
  double kbox[3];  // 2 pi / L_d
  const int3 *kidx;
};

cudaError_t launch_rhok_full(cudaStream_t st, const double *path, int N, int S, const LRDesc &lr, double2 *rhok);
cudaError_t launch_rhok_update(cudaStream_t st, const double *path_old, const double *path_new, int N,
                               const LRDesc &lr, const ActiveList &act, int slice1, int slice2, int skip,
                               const double2 *rho_old, double2 *rho_new);
// sum over slices slice1, slice1 + skip, ..., slice2 and k of w |rho_k|^2 uk[k],
// w = end_weight at slice1 and slice2 and 1 between
cudaError_t launch_lr_sum(const ReduceTarget &t, const double2 *rhok, const LRDesc &lr, const double *uk, int slice1,
                          int slice2, int skip, int sm_count, double end_weight = 0.5);
cudaError_t launch_rhok_copy(cudaStream_t st, const double2 *src, double2 *dst, int nk, int slice1, int slice2);

}  // namespace pimc

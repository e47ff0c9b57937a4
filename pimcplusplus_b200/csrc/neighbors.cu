// Neighbour lists for the short-range sum of the device moves (the role of
// ShortRangeOnClass's cell lists, PIMC++/src/Actions/ShortRangeOnClass.cc:35-240,
// with the grid of GridClass.cc:52-121).
//
// A DavidPA table is zero at and beyond its grid end (the reader zeroes the
// last row), so a pair contributes only while one of its link distances is
// below that range.  Every particle's path is bounded by a sphere: centre c =
// its slice-0 position, radius B = the largest minimum-image distance of its
// positions from c, plus a skin.  The list of particle i holds every j with
// |c_i - c_j| <= range + B_i + B_j (minimum image), in ascending order, so the
// partners it omits add exact zeros to the sum.  The moves check their NEW
// positions against the sphere and fall back to all partners when they leave
// it; the lists are rebuilt (here) before the next launch.
#include <cuda_runtime.h>

#include "bisection.cuh"

namespace pimc {

namespace {

__device__ __forceinline__ double min_image2(double dx, double dy, double dz, const DevSystem &s) {
  dx -= rint(dx * s.boxinv[0]) * s.box[0];
  dy -= rint(dy * s.boxinv[1]) * s.box[1];
  dz -= rint(dz * s.boxinv[2]) * s.box[2];
  return dx * dx + dy * dy + dz * dz;
}

__global__ void __launch_bounds__(256) nbr_bounds_kernel(const double *__restrict__ path, DevSystem sys, double skin,
                                                         double4 *cb, const int *dirty) {
  if (*dirty == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sys.N) return;
  const double *c = path + (size_t)i * 3;
  double r2 = 0.0;
  for (int s = 1; s < sys.S; s++) {
    const double *q = path + ((size_t)s * sys.N + i) * 3;
    r2 = fmax(r2, min_image2(q[0] - c[0], q[1] - c[1], q[2] - c[2], sys));
  }
  cb[i] = make_double4(c[0], c[1], c[2], sqrt(r2) + skin);
}

// One warp per particle i: the partners in ascending j, compacted by ballot.
__global__ void __launch_bounds__(256) nbr_fill_kernel(DevSystem sys, double range, int kmax,
                                                       const double4 *__restrict__ cb, int *cnt, int *idx,
                                                       const int *dirty) {
  if (*dirty == 0) return;
  const int lane = threadIdx.x & 31;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= sys.N) return;
  const double4 ci = cb[i];
  int n = 0;
  int *out = idx + (size_t)i * kmax;
  for (int j0 = 0; j0 < sys.N; j0 += 32) {
    const int j = j0 + lane;
    bool take = false;
    if (j < sys.N && j != i) {
      const double4 cj = cb[j];
      const double lim = range + ci.w + cj.w;
      take = min_image2(cj.x - ci.x, cj.y - ci.y, cj.z - ci.z, sys) <= lim * lim;
    }
    const unsigned m = __ballot_sync(0xffffffffu, take);
    const int pos = n + __popc(m & ((1u << lane) - 1u));
    if (take && pos < kmax) out[pos] = j;
    n += __popc(m);
  }
  if (lane == 0) cnt[i] = n <= kmax ? n : -1;  // -1: list overflow, all partners for i
}

__global__ void nbr_clear_kernel(int *dirty) { *dirty = 0; }

}  // namespace

cudaError_t launch_nbr_rebuild(cudaStream_t st, const double *path, const DevSystem &sys, double range, double skin,
                               int kmax, double4 *cb, int *cnt, int *idx, int *dirty) {
  nbr_bounds_kernel<<<(sys.N + 255) / 256, 256, 0, st>>>(path, sys, skin, cb, dirty);
  nbr_fill_kernel<<<(sys.N + 7) / 8, 256, 0, st>>>(sys, range, kmax, cb, cnt, idx, dirty);
  nbr_clear_kernel<<<1, 1, 0, st>>>(dirty);
  return cudaGetLastError();
}

}  // namespace pimc

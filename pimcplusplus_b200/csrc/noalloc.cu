// ShortRange SingleAction for callers that cannot allocate device memory.
//
// Some callers may not call cudaMalloc at all: code running inside a
// host-side memory pool or arena that owns every device allocation, an
// embedding that forbids allocation after start-up, or a latency-critical
// loop that must not pay for cudaMalloc's implicit device synchronisation.
// For them,
// pimc_shortrange_single_noalloc evaluates ShortRangeClass::SingleAction for
// a DavidPA pair action on a linear grid with no off-diagonal terms, from
// device buffers the caller already owns (the path, the (y, d2y) table of
// u_00 for the level, the output scalar), and allocates nothing.  Its
// scratch — one partial sum per thread block and a completion counter — is a
// file-scope __device__ array of fixed size that every GPU loading this
// library holds until the process exits.
//
// Limits and sharing:
//  * At most kNoAllocBlocks blocks of 256 threads, i.e. n_active x particles
//    x links <= kNoAllocMaxTerms pair terms per call; larger calls are
//    rejected with PIMC_E_ARG.
//  * Every call on a device uses the same scratch.  Calls whose kernels
//    overlap on the GPU (different streams, or host threads without
//    ordering) race on it; serialise them on one stream.
//  * The first call on a device looks up the scratch's device address with
//    cudaGetSymbolAddress (with that device current) and caches it; make
//    that first call before any stream capture.
#include <cuda_runtime.h>

#include <mutex>

#include "action_kernels.cuh"
#include "device_math.cuh"

namespace pimc {

constexpr int kNoAllocBlocks = 2048;
constexpr long long kNoAllocMaxTerms = (long long)kNoAllocBlocks * 256;
constexpr int kNoAllocDevices = 64;

struct NoAllocScratch {
  double partials[kNoAllocBlocks];
  unsigned int counter;
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

namespace {

__device__ __forceinline__ double na_block_sum(double v, double *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) r += sh[i];
  return r;
}

// The same terms as the context-based entry point, in a fixed reduction
// order; the order is that entry point's only while both launch the same
// number of blocks (it caps its grid at 8 blocks per SM, this kernel launches
// one block per 256 terms), so large calls may differ from it in the last
// bits.
__global__ void __launch_bounds__(256) sr_single_noalloc_kernel(const double *__restrict__ path, DevSystem sys,
                                                                DDavid<double> d, ActiveList act, int slice1,
                                                                int skip, int nlinks, int level,
                                                                NoAllocScratch *scratch, double *out) {
  __shared__ double sh[32];
  __shared__ int s_last;
  const double2 *diag = reinterpret_cast<const double2 *>(d.diag);
  const int N = sys.N;
  const long long per_active = (long long)N * nlinks;
  const long long total = per_active * act.n;
  double acc = 0.0;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int pi = (int)(idx / per_active);
    const long long rem = idx - pi * per_active;
    const int link = (int)(rem / N);
    const int p2 = (int)(rem - (long long)link * N);
    const int p1 = act.p[pi];
    bool visited = false;
    for (int k = 0; k <= pi; k++) visited |= (act.p[k] == p2);
    if (visited) continue;
    const int slice = slice1 + link * skip;
    double a1[3], a2[3], b1[3], b2[3], dA[3], dB[3];
    for (int i = 0; i < 3; i++) {
      a1[i] = __ldg(path + ((size_t)slice * N + p1) * 3 + i);
      a2[i] = __ldg(path + ((size_t)slice * N + p2) * 3 + i);
      b1[i] = __ldg(path + ((size_t)(slice + skip) * N + p1) * 3 + i);
      b2[i] = __ldg(path + ((size_t)(slice + skip) * N + p2) * 3 + i);
    }
    dist_disp(a1, a2, b1, b2, sys, dA, dB);
    const LinkGeom<double> g = link_geom<double>(dA, dB);
    acc += david_U<double>(d, diag, g.s2, g.q, g.z, level);
  }
  const double r = na_block_sum(acc, sh);
  if (threadIdx.x == 0) {
    scratch->partials[blockIdx.x] = r;
    __threadfence();
    s_last = (atomicAdd(&scratch->counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double v = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) v += __ldcg(&scratch->partials[i]);
  const double tot = na_block_sum(v, sh);
  if (threadIdx.x == 0) {
    *out = tot;
    scratch->counter = 0u;
  }
}

std::mutex g_noalloc_mu;
NoAllocScratch *g_noalloc_ptr[kNoAllocDevices] = {};

}  // namespace
}  // namespace pimc

using namespace pimc;

extern "C" int pimc_shortrange_single_noalloc(const double *path, int num_particles, int num_time_slices,
                                              const double box[3], const double *diag, double grid_start,
                                              double grid_end, int num_grid, int slice1, int slice2,
                                              const int *active, int n_active, int level, double *out,
                                              void *stream) {
  if (!path || !box || !diag || !out || !active) return PIMC_E_ARG;
  if (num_particles < 2 || num_time_slices < 2 || num_grid < 2 || !(grid_end > grid_start)) return PIMC_E_ARG;
  if (level < 0 || level >= kMaxLevels || slice1 < 0 || slice2 < slice1 || slice2 >= num_time_slices)
    return PIMC_E_ARG;
  if (n_active < 1 || n_active > kMaxActive) return PIMC_E_ARG;
  for (int i = 0; i < 3; i++)
    if (!(box[i] > 0.0)) return PIMC_E_ARG;
  ActiveList act;
  act.n = n_active;
  for (int i = 0; i < n_active; i++) {
    if (active[i] < 0 || active[i] >= num_particles) return PIMC_E_ARG;
    act.p[i] = active[i];
  }
  const int skip = 1 << level;
  const int nlinks = (slice2 - slice1 + skip - 1) / skip;
  if (nlinks == 0) {
    // an empty link range sums no term: 0, as pimc_single_action returns
    return cudaMemsetAsync(out, 0, sizeof(double), static_cast<cudaStream_t>(stream)) == cudaSuccess ? PIMC_OK
                                                                                                    : PIMC_E_CUDA;
  }
  if (slice1 + nlinks * skip >= num_time_slices) return PIMC_E_ARG;
  const long long items = (long long)n_active * num_particles * nlinks;
  if (items > kNoAllocMaxTerms) return PIMC_E_ARG;  // beyond the fixed scratch (2048 blocks x 256 threads)

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocDevices) return PIMC_E_CUDA;
  NoAllocScratch *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void *p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return PIMC_E_CUDA;
      g_noalloc_ptr[dev] = static_cast<NoAllocScratch *>(p);
    }
    scratch = g_noalloc_ptr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // The counter must start at zero; a previous call leaves it at zero, but a
  // call cut short would not, so clear it on the caller's stream.
  if (cudaMemsetAsync(&scratch->counter, 0, sizeof(unsigned int), st) != cudaSuccess) return PIMC_E_CUDA;

  DevSystem sys{};
  sys.N = num_particles;
  sys.S = num_time_slices;
  for (int i = 0; i < 3; i++) {
    sys.box[i] = box[i];
    sys.boxinv[i] = 1.0 / box[i];
  }
  DDavid<double> d{};
  d.grid.type = PIMC_GRID_LINEAR;
  d.grid.n = num_grid;
  d.grid.start = grid_start;
  d.grid.end = grid_end;
  d.grid.delta = (grid_end - grid_start) / (double)(num_grid - 1);
  d.grid.deltainv = 1.0 / d.grid.delta;
  d.grid.x = nullptr;
  d.ncols = 2;
  d.num_tau = 1;
  d.tau_pos = -level;  // `diag` is already the level's column
  d.num_terms = 0;
  d.diag = diag;
  d.diag_stride = num_grid;
  const int blocks = (int)((items + 255) / 256);
  sr_single_noalloc_kernel<<<blocks, 256, 0, st>>>(path, sys, d, act, slice1, skip, nlinks, level, scratch, out);
  return cudaGetLastError() == cudaSuccess ? PIMC_OK : PIMC_E_CUDA;
}

// Action-level kernels behind the ActionBaseClass drop-in entry points:
// SingleAction and d_dBeta of ShortRangeClass and KineticClass, and the
// PathClass accept/reject copies.  One launch per call; each reduces its
// terms in a fixed order (warp shuffle tree, block tree, then the last block
// over the per-block partials), so results are bitwise reproducible.
#include <cuda_runtime.h>

#include "action_kernels.cuh"
#include "device_math.cuh"

namespace pimc {

// Block-wide sum; the result is valid in thread 0.  `sh` holds >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    for (int i = 0; i < nw; i++) r += sh[i];
  }
  return r;
}

// Writes this block's partial and lets the last block to finish add all
// partials in block order into *out.
__device__ __forceinline__ void finish_sum(double partial, double *partials, unsigned int *counter, double *out,
                                           double *sh) {
  __shared__ int s_last;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = partial;
    __threadfence();
    unsigned int t = atomicAdd(counter, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double v = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) v += __ldcg(&partials[i]);
  double total = block_sum(v, sh);
  if (threadIdx.x == 0) {
    *out = total;
    *counter = 0u;
  }
}

__device__ __forceinline__ void load3(const double *__restrict__ p, double v[3]) {
  v[0] = __ldg(p);
  v[1] = __ldg(p + 1);
  v[2] = __ldg(p + 2);
}

// ShortRangeClass::SingleAction (ShortRangeClass.cc:191-236).  Item order:
// active particle, link, partner (partner fastest, for coalesced path reads).
template <int KIND, typename R>
__global__ void __launch_bounds__(256) sr_single_kernel(const double *__restrict__ path, DevSystem sys, DevPA pa,
                                                        ActiveList act, int slice1, int skip, int nlinks, int level,
                                                        double *partials, unsigned int *counter, double *out) {
  __shared__ double sh[32];
  typedef typename Pair2<R>::T P2;
  const P2 *diag = nullptr;
  if (KIND == PA_DAVID) {
    const DDavid<R> &d = david_of<R>(pa);
    diag = reinterpret_cast<const P2 *>(d.diag) + (size_t)(level + d.tau_pos) * d.diag_stride;
  }
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
    bool visited = false;  // Path.DoPtcl: moved particles count once
    for (int k = 0; k <= pi; k++) visited |= (act.p[k] == p2);
    if (visited) continue;
    const int slice = slice1 + link * skip;
    double a1[3], a2[3], b1[3], b2[3], dA[3], dB[3];
    load3(path + ((size_t)slice * N + p1) * 3, a1);
    load3(path + ((size_t)slice * N + p2) * 3, a2);
    load3(path + ((size_t)(slice + skip) * N + p1) * 3, b1);
    load3(path + ((size_t)(slice + skip) * N + p2) * 3, b2);
    dist_disp(a1, a2, b1, b2, sys, dA, dB);
    LinkGeom<R> g = link_geom<R>(dA, dB);
    acc += (double)pa_U<R, KIND>(pa, diag, g, level);
  }
  double r = block_sum(acc, sh);
  finish_sum(r, partials, counter, out, sh);
}

// Triangular pair index k -> (p1, p2) with p2 < p1.
__device__ __forceinline__ void tri_decode(long long k, int &p1, int &p2) {
  long long a = (long long)((1.0 + sqrt(1.0 + 8.0 * (double)k)) * 0.5);
  while (a * (a - 1) / 2 > k) a--;
  while ((a + 1) * a / 2 <= k) a++;
  p1 = (int)a;
  p2 = (int)(k - a * (a - 1) / 2);
}

// ShortRangeClass::d_dBeta (ShortRangeClass.cc:316-355), FP64.
template <int KIND>
__global__ void __launch_bounds__(256) sr_dbeta_kernel(const double *__restrict__ path, DevSystem sys, DevPA pa,
                                                       int slice1, int skip, int nlinks, int level, double *partials,
                                                       unsigned int *counter, double *out) {
  __shared__ double sh[32];
  const int N = sys.N;
  const long long npairs = (long long)N * (N - 1) / 2;
  const long long total = npairs * nlinks;
  double acc = 0.0;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int link = (int)(idx / npairs);
    int p1, p2;
    tri_decode(idx - (long long)link * npairs, p1, p2);
    const int slice = slice1 + link * skip;
    double a1[3], a2[3], b1[3], b2[3], dA[3], dB[3];
    load3(path + ((size_t)slice * N + p1) * 3, a1);
    load3(path + ((size_t)slice * N + p2) * 3, a2);
    load3(path + ((size_t)(slice + skip) * N + p1) * 3, b1);
    load3(path + ((size_t)(slice + skip) * N + p2) * 3, b2);
    dist_disp(a1, a2, b1, b2, sys, dA, dB);
    LinkGeom<double> g = link_geom<double>(dA, dB);
    acc += pa_dU<KIND>(pa, g, level);
  }
  double r = block_sum(acc, sh);
  finish_sum(r, partials, counter, out, sh);
}

// ---- observables: ShortRangePotClass::V and PairCorrelationClass::Accumulate ----
// PathClass::DistDisp one-slice form (PathClass.h:637-660): minimum image by
// nearbyint(disp / L), then |disp|.
__device__ __forceinline__ double dist_one_slice(const double a[3], const double b[3], const DevSystem &s) {
  double d2 = 0.0;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    double d = b[i] - a[i];
    const double n = rint(rmul(d, s.boxinv[i]));
    d = rsub(d, rmul(n, s.box[i]));
    d2 = radd(d2, rmul(d, d));
  }
  return sqrt(d2);
}

// V(r) of the pair action: DavidPAClass::V (DavidPAClass.cc:104-113), column 0
// of the first tau table with r clamped to the grid; PAtricubicFit's
// potential spline (PAFitBase.h:82).
template <int KIND>
__device__ __forceinline__ double pa_V(const DevPA &pa, double r) {
  if (KIND == PA_DAVID) {
    const DDavid<double> &d = pa.d64;
    const DGrid<double> &g = d.grid;
    if (r > g.end) r = g.end;
    if (r < g.start) r = g.start;
    return spline_col(g, d.uy, d.ud2, d.ncols, 0, r);
  }
  if (KIND == PA_COULOMB) {
    // CoulombPot V = Z1Z2 / r, less Vlong with the long-range breakup
    // (ShortRangePotClass.cc:41-43); for the classical Coulomb action the V
    // breakup fits the same X_k as the dU one, so Vlong is dUlong.
    const DCoulomb<double> &c = pa.c64;
    double v = c.z1z2 / r;
    if (c.long_range) v -= quintic_at(c, c.dulong, r);
    return v;
  }
  return pot_V(pa.t64, r);
}

// One pass over slices [0, S-1] x pairs p2 < p1 of the OLD path.
//  DO_V: sum over slices of factor * sum_pairs V(r), factor 1/2 at the end
//        slices (ActionsClass.cc:852-857 with ShortRangePotClass.cc:28-47).
//  DO_G: histogram of the pair distances at slices [0, S-2] below the grid
//        end, bin (int)nearbyint((r - start) * deltainv - 0.5)
//        (ObservableCorrelation.cc:191-207, Grid.h:81-84); bins counted per
//        block in shared memory, then added to the 64-bit histogram.
template <int KIND, bool DO_V, bool DO_G>
__global__ void __launch_bounds__(256) pair_obs_kernel(const double *__restrict__ path, DevSystem sys, DevPA pa,
                                                       GofrGrid gg, unsigned long long *hist, double *partials,
                                                       unsigned int *counter, double *out) {
  extern __shared__ unsigned int s_hist[];
  __shared__ double sh[32];
  const int N = sys.N, S = sys.S;
  const long long npairs = (long long)N * (N - 1) / 2;
  const long long total = npairs * S;
  if (DO_G) {
    for (int i = threadIdx.x; i < gg.nbins; i += blockDim.x) s_hist[i] = 0u;
    __syncthreads();
  }
  double acc = 0.0;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int slice = (int)(idx / npairs);
    int p1, p2;
    tri_decode(idx - (long long)slice * npairs, p1, p2);
    if (!DO_V && slice == S - 1) continue;
    double a[3], b[3];
    load3(path + ((size_t)slice * N + p1) * 3, a);
    load3(path + ((size_t)slice * N + p2) * 3, b);
    const double dist = dist_one_slice(a, b, sys);
    if (DO_V) {
      const double f = (slice == 0 || slice == S - 1) ? 0.5 : 1.0;
      acc += f * pa_V<KIND>(pa, dist);
    }
    if (DO_G && slice < S - 1 && dist < gg.end) {
      const int bin = (int)rint(rsub(rmul(rsub(dist, gg.start), gg.deltainv), 0.5));
      if (bin >= 0 && bin < gg.nbins) atomicAdd(&s_hist[bin], 1u);
    }
  }
  if (DO_G) {
    __syncthreads();
    for (int i = threadIdx.x; i < gg.nbins; i += blockDim.x)
      if (s_hist[i]) atomicAdd(&hist[i], (unsigned long long)s_hist[i]);
  }
  if (DO_V) {
    const double r = block_sum(acc, sh);
    finish_sum(r, partials, counter, out, sh);
  }
}

__device__ __forceinline__ void velocity(const double *__restrict__ path, int N, int sa, int sb, int p,
                                         const DevSystem &sys, double v[3]) {
  double a[3], b[3];
  load3(path + ((size_t)sa * N + p) * 3, a);
  load3(path + ((size_t)sb * N + p) * 3, b);
  for (int i = 0; i < 3; i++) v[i] = b[i] - a[i];
  put_in_box(v, sys);
}

// KineticClass::SingleAction (KineticClass.cc:33-90)
__global__ void __launch_bounds__(256) kin_single_kernel(const double *__restrict__ path, DevSystem sys,
                                                         ActiveList act, int slice1, int skip, int nlinks, int level,
                                                         double *partials, unsigned int *counter, double *out) {
  __shared__ double sh[32];
  const double levelTau = sys.tau * (1 << level);
  const double F = 1.0 / (4.0 * sys.lambda * levelTau);
  const int total = act.n * nlinks;
  double acc = 0.0;
  if (sys.lambda != 0.0)
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
      const int pi = idx / nlinks, link = idx - pi * nlinks;
      const int slice = slice1 + link * skip;
      double vel[3];
      velocity(path, sys.N, slice, slice + skip, act.p[pi], sys, vel);
      acc += kinetic_link(vel, F, sys.num_images, sys);
    }
  double r = block_sum(acc, sh);
  finish_sum(r, partials, counter, out, sh);
}

// KineticClass::d_dBeta (KineticClass.cc:187-256)
__global__ void __launch_bounds__(256) kin_dbeta_kernel(const double *__restrict__ path, DevSystem sys, int slice1,
                                                        int skip, int nlinks, int level, double *partials,
                                                        unsigned int *counter, double *out) {
  __shared__ double sh[32];
  const double levelTau = ldexp(sys.tau, level);
  const double F = 1.0 / (4.0 * sys.lambda * levelTau);
  const int total = sys.N * nlinks;
  double acc = 0.0;
  if (sys.lambda != 0.0)
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
      const int link = idx / sys.N, p = idx - link * sys.N;
      const int slice = slice1 + link * skip;
      double vel[3];
      velocity(path, sys.N, slice, slice + skip, p, sys, vel);
      double spring = (0.5 * 3) / levelTau;
      double Z = 1.0, GaussSum[3] = {0, 0, 0}, numSum[3] = {0, 0, 0};
      for (int dim = 0; dim < 3; dim++) {
        for (int image = -sys.num_images; image <= sys.num_images; image++) {
          double dist = vel[dim] + (double)image * sys.box[dim];
          double d2overFLT = dist * dist * F;
          double expPart = exp(-d2overFLT);
          GaussSum[dim] += expPart;
          numSum[dim] += -d2overFLT / levelTau * expPart;
        }
        Z *= GaussSum[dim];
      }
      double scalarnumSum = 0.0;
      for (int dim = 0; dim < 3; dim++) {
        double numProd = 1.0;
        for (int dim2 = 0; dim2 < 3; dim2++) numProd *= (dim2 != dim) ? GaussSum[dim2] : numSum[dim2];
        scalarnumSum += numProd;
      }
      acc += spring + scalarnumSum / Z;
    }
  double r = block_sum(acc, sh);
  finish_sum(r, partials, counter, out, sh);
}

// PathClass::AcceptCopy (PathClass.cc:797-863): PutInBoxFast on NEW, NEW -> OLD.
__global__ void accept_kernel(double *path_old, double *path_new, DevSystem sys, ActiveList act, int slice1,
                              int nslices) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= act.n * nslices) return;
  int pi = idx / nslices, slice = slice1 + (idx - pi * nslices);
  size_t o = ((size_t)slice * sys.N + act.p[pi]) * 3;
  double v[3] = {path_new[o], path_new[o + 1], path_new[o + 2]};
  put_in_box_fast(v, sys);
  for (int i = 0; i < 3; i++) {
    path_new[o + i] = v[i];
    path_old[o + i] = v[i];
  }
}

// PathClass::RejectCopy (PathClass.cc:865-899): OLD -> NEW.
__global__ void reject_kernel(const double *path_old, double *path_new, DevSystem sys, ActiveList act, int slice1,
                              int nslices) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= act.n * nslices) return;
  int pi = idx / nslices, slice = slice1 + (idx - pi * nslices);
  size_t o = ((size_t)slice * sys.N + act.p[pi]) * 3;
  for (int i = 0; i < 3; i++) path_new[o + i] = path_old[o + i];
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
static int grid_for(long long items, int threads, int sm_count) {
  long long b = (items + threads - 1) / threads;
  long long cap = (long long)sm_count * 8;
  if (b > cap) b = cap;
  if (b > kPartialSlots) b = kPartialSlots;
  if (b < 1) b = 1;
  return (int)b;
}

cudaError_t launch_sr_single(const ReduceTarget &t, const double *path, const DevSystem &sys, const DevPA &pa,
                             const ActiveList &act, int slice1, int skip, int nlinks, int level, int precision,
                             int sm_count) {
  long long items = (long long)act.n * sys.N * nlinks;
  int blocks = grid_for(items, 256, sm_count);
  if (pa.kind == PA_DAVID) {
    if (precision == PIMC_MIXED)
      sr_single_kernel<PA_DAVID, float><<<blocks, 256, 0, t.stream>>>(path, sys, pa, act, slice1, skip, nlinks, level,
                                                                       t.partials, t.counter, t.out);
    else
      sr_single_kernel<PA_DAVID, double><<<blocks, 256, 0, t.stream>>>(path, sys, pa, act, slice1, skip, nlinks, level,
                                                                        t.partials, t.counter, t.out);
  } else if (pa.kind == PA_COULOMB) {
    if (precision == PIMC_MIXED)
      sr_single_kernel<PA_COULOMB, float><<<blocks, 256, 0, t.stream>>>(path, sys, pa, act, slice1, skip, nlinks,
                                                                         level, t.partials, t.counter, t.out);
    else
      sr_single_kernel<PA_COULOMB, double><<<blocks, 256, 0, t.stream>>>(path, sys, pa, act, slice1, skip, nlinks,
                                                                          level, t.partials, t.counter, t.out);
  } else {
    if (precision == PIMC_MIXED)
      sr_single_kernel<PA_TRICUBIC, float><<<blocks, 256, 0, t.stream>>>(path, sys, pa, act, slice1, skip, nlinks,
                                                                          level, t.partials, t.counter, t.out);
    else
      sr_single_kernel<PA_TRICUBIC, double><<<blocks, 256, 0, t.stream>>>(path, sys, pa, act, slice1, skip, nlinks,
                                                                           level, t.partials, t.counter, t.out);
  }
  return cudaGetLastError();
}

cudaError_t launch_sr_dbeta(const ReduceTarget &t, const double *path, const DevSystem &sys, const DevPA &pa,
                            int slice1, int skip, int nlinks, int level, int sm_count) {
  long long items = (long long)sys.N * (sys.N - 1) / 2 * nlinks;
  int blocks = grid_for(items, 256, sm_count);
  if (pa.kind == PA_DAVID)
    sr_dbeta_kernel<PA_DAVID><<<blocks, 256, 0, t.stream>>>(path, sys, pa, slice1, skip, nlinks, level, t.partials,
                                                            t.counter, t.out);
  else if (pa.kind == PA_COULOMB)
    sr_dbeta_kernel<PA_COULOMB><<<blocks, 256, 0, t.stream>>>(path, sys, pa, slice1, skip, nlinks, level, t.partials,
                                                              t.counter, t.out);
  else
    sr_dbeta_kernel<PA_TRICUBIC><<<blocks, 256, 0, t.stream>>>(path, sys, pa, slice1, skip, nlinks, level, t.partials,
                                                               t.counter, t.out);
  return cudaGetLastError();
}

cudaError_t launch_kin_single(const ReduceTarget &t, const double *path, const DevSystem &sys, const ActiveList &act,
                              int slice1, int skip, int nlinks, int level, int sm_count) {
  int blocks = grid_for((long long)act.n * nlinks, 256, sm_count);
  kin_single_kernel<<<blocks, 256, 0, t.stream>>>(path, sys, act, slice1, skip, nlinks, level, t.partials, t.counter,
                                                  t.out);
  return cudaGetLastError();
}

cudaError_t launch_kin_dbeta(const ReduceTarget &t, const double *path, const DevSystem &sys, int slice1, int skip,
                             int nlinks, int level, int sm_count) {
  int blocks = grid_for((long long)sys.N * nlinks, 256, sm_count);
  kin_dbeta_kernel<<<blocks, 256, 0, t.stream>>>(path, sys, slice1, skip, nlinks, level, t.partials, t.counter,
                                                 t.out);
  return cudaGetLastError();
}

cudaError_t launch_pair_obs(const ReduceTarget &t, const double *path, const DevSystem &sys, const DevPA &pa,
                            bool do_v, const GofrGrid *gg, unsigned long long *hist, int sm_count) {
  const long long items = (long long)sys.N * (sys.N - 1) / 2 * sys.S;
  const int blocks = grid_for(items, 256, sm_count);
  const size_t dyn = gg ? (size_t)gg->nbins * sizeof(unsigned int) : 0;
  const GofrGrid g0 = gg ? *gg : GofrGrid{0.0, 0.0, 0.0, 0};
  const bool dav = pa.kind == PA_DAVID;
  if (do_v && pa.kind == PA_COULOMB) {
    if (gg)
      pair_obs_kernel<PA_COULOMB, true, true><<<blocks, 256, dyn, t.stream>>>(path, sys, pa, g0, hist, t.partials,
                                                                              t.counter, t.out);
    else
      pair_obs_kernel<PA_COULOMB, true, false><<<blocks, 256, 0, t.stream>>>(path, sys, pa, g0, hist, t.partials,
                                                                             t.counter, t.out);
  } else if (do_v && gg) {
    if (dav)
      pair_obs_kernel<PA_DAVID, true, true><<<blocks, 256, dyn, t.stream>>>(path, sys, pa, g0, hist, t.partials,
                                                                            t.counter, t.out);
    else
      pair_obs_kernel<PA_TRICUBIC, true, true><<<blocks, 256, dyn, t.stream>>>(path, sys, pa, g0, hist, t.partials,
                                                                               t.counter, t.out);
  } else if (do_v) {
    if (dav)
      pair_obs_kernel<PA_DAVID, true, false><<<blocks, 256, 0, t.stream>>>(path, sys, pa, g0, hist, t.partials,
                                                                           t.counter, t.out);
    else
      pair_obs_kernel<PA_TRICUBIC, true, false><<<blocks, 256, 0, t.stream>>>(path, sys, pa, g0, hist, t.partials,
                                                                              t.counter, t.out);
  } else if (gg) {
    pair_obs_kernel<PA_DAVID, false, true><<<blocks, 256, dyn, t.stream>>>(path, sys, pa, g0, hist, t.partials,
                                                                          t.counter, t.out);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_accept(cudaStream_t st, double *path_old, double *path_new, const DevSystem &sys,
                          const ActiveList &act, int slice1, int slice2) {
  int nslices = slice2 - slice1 + 1;
  int items = act.n * nslices;
  accept_kernel<<<(items + 127) / 128, 128, 0, st>>>(path_old, path_new, sys, act, slice1, nslices);
  return cudaGetLastError();
}

cudaError_t launch_reject(cudaStream_t st, const double *path_old, double *path_new, const DevSystem &sys,
                          const ActiveList &act, int slice1, int slice2) {
  int nslices = slice2 - slice1 + 1;
  int items = act.n * nslices;
  reject_kernel<<<(items + 127) / 128, 128, 0, st>>>(path_old, path_new, sys, act, slice1, nslices);
  return cudaGetLastError();
}

}  // namespace pimc

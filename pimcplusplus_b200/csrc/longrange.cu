// Long-range (Ewald breakup) k-space pieces on the device:
//   PathClass::SetupkVecs3D       (PathClass.cc:534-586)  — host, in capi
//   PathClass::CalcRho_ks_Fast    (PathClass.cc:616-647)  — rhok_full_kernel
//   PathClass::UpdateRho_ks       (PathClass.cc:649-707)  — rhok_update_kernel
//   LongRangeClass::SingleAction  (LongRangeClass.cc:273-371) and
//   LongRangeClass::d_dBeta       (LongRangeClass.cc:374-442) — lr_sum_kernel
//   DavidLongRangeClassYk::SingleAction / d_dBeta / V
//                                 (DavidLongRangeClassYk.cc:230-389) — lr_sum_kernel
//
// rho_k is stored [slice][k] as double2 (re, im), one species.  The phase
// factors follow the reference exactly: per particle and dimension,
// C_d(n) = e^{i n kBox_d x_d} is built by repeated multiplication from
// C_d(1) = (cos, sin)(kBox_d x_d), C_d(-n) = conj(C_d(n)), and a k-vector's
// term is (C_0(kx) C_1(ky)) C_2(kz).  The tables of the particles a block
// handles are built cooperatively in shared memory.
#include <cuda_runtime.h>

#include "action_kernels.cuh"
#include "device_math.cuh"
#include "longrange.cuh"

namespace pimc {

namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Fills C[d][n + kmax_d] for one position into shared memory (called by
// threads 0..2, one dimension each).
__device__ __forceinline__ void fill_phase_table(const double *r, int d, const LRDesc &lr, double2 *C) {
  const int m = lr.kmax[d];
  const double phi = r[d] * lr.kbox[d];
  double s, c;
  sincos(phi, &s, &c);
  const double2 t = make_double2(c, s);
  double2 *Cd = C + lr.coff[d];
  Cd[m] = make_double2(1.0, 0.0);
  for (int n = 1; n <= m; n++) {
    Cd[m + n] = cmul(t, Cd[m + n - 1]);
    Cd[m - n] = make_double2(Cd[m + n].x, -Cd[m + n].y);
  }
}

__device__ __forceinline__ double2 k_term(const double2 *C, const LRDesc &lr, int3 ki) {
  const double2 a = C[lr.coff[0] + ki.x], b = C[lr.coff[1] + ki.y], c = C[lr.coff[2] + ki.z];
  return cmul(cmul(a, b), c);
}

constexpr int kMaxPhase = 3 * (2 * 64 + 1);  // kmax <= 64 per dimension

// One block per slice: rho_k(slice) = sum over particles of the k terms.
__global__ void __launch_bounds__(256) rhok_full_kernel(const double *__restrict__ path, int N, LRDesc lr,
                                                        double2 *rhok) {
  __shared__ double2 C[kMaxPhase];
  const int slice = blockIdx.x;
  double2 acc[4];
  const int per = (lr.nk + blockDim.x - 1) / blockDim.x;  // <= 4 (nk <= 1024)
  for (int j = 0; j < 4; j++) acc[j] = make_double2(0.0, 0.0);
  for (int p = 0; p < N; p++) {
    __syncthreads();
    if (threadIdx.x < 3) {
      const double *r = path + ((size_t)slice * N + p) * 3;
      double rr[3] = {r[0], r[1], r[2]};
      fill_phase_table(rr, threadIdx.x, lr, C);
    }
    __syncthreads();
    for (int j = 0; j < per; j++) {
      const int k = threadIdx.x + j * blockDim.x;
      if (k < lr.nk) {
        const double2 t = k_term(C, lr, lr.kidx[k]);
        acc[j].x += t.x;
        acc[j].y += t.y;
      }
    }
  }
  for (int j = 0; j < per; j++) {
    const int k = threadIdx.x + j * blockDim.x;
    if (k < lr.nk) rhok[(size_t)slice * lr.nk + k] = acc[j];
  }
}

// One block per updated slice (slice1 + b*skip): NEW = OLD, then per active
// particle NEW += C(r_new), NEW -= C(r_old), in the reference's order.
__global__ void __launch_bounds__(256) rhok_update_kernel(const double *__restrict__ path_old,
                                                          const double *__restrict__ path_new, int N, LRDesc lr,
                                                          ActiveList act, int slice1, int skip,
                                                          const double2 *__restrict__ rho_old, double2 *rho_new) {
  __shared__ double2 Cn[kMaxPhase], Co[kMaxPhase];
  const int slice = slice1 + blockIdx.x * skip;
  const int per = (lr.nk + blockDim.x - 1) / blockDim.x;
  double2 acc[4];
  for (int j = 0; j < per; j++) {
    const int k = threadIdx.x + j * blockDim.x;
    if (k < lr.nk) acc[j] = rho_old[(size_t)slice * lr.nk + k];
  }
  for (int pi = 0; pi < act.n; pi++) {
    __syncthreads();
    const int p = act.p[pi];
    if (threadIdx.x < 3) {
      const double *r = path_new + ((size_t)slice * N + p) * 3;
      double rr[3] = {r[0], r[1], r[2]};
      fill_phase_table(rr, threadIdx.x, lr, Cn);
    } else if (threadIdx.x >= 32 && threadIdx.x < 35) {
      const double *r = path_old + ((size_t)slice * N + p) * 3;
      double rr[3] = {r[0], r[1], r[2]};
      fill_phase_table(rr, threadIdx.x - 32, lr, Co);
    }
    __syncthreads();
    for (int j = 0; j < per; j++) {
      const int k = threadIdx.x + j * blockDim.x;
      if (k < lr.nk) {
        const int3 ki = lr.kidx[k];
        const double2 tn = k_term(Cn, lr, ki);
        acc[j].x += tn.x;
        acc[j].y += tn.y;
        const double2 to = k_term(Co, lr, ki);
        acc[j].x -= to.x;
        acc[j].y -= to.y;
      }
    }
  }
  for (int j = 0; j < per; j++) {
    const int k = threadIdx.x + j * blockDim.x;
    if (k < lr.nk) rho_new[(size_t)slice * lr.nk + k] = acc[j];
  }
}

__device__ __forceinline__ double lr_block_sum(double v, double *sh) {
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

// sum over slices [slice1, slice2] step skip of factor * sum_k |rho_k|^2 u_k
// (the homologous k-space term); factor 1/2 at the two ends.
__global__ void __launch_bounds__(256) lr_sum_kernel(const double2 *__restrict__ rhok, LRDesc lr,
                                                     const double *__restrict__ uk, int slice1, int slice2, int skip,
                                                     double end_weight, double *partials, unsigned int *counter,
                                                     double *out) {
  __shared__ double sh[32];
  __shared__ int s_last;
  const int nsl = (slice2 - slice1) / skip + 1;
  const long long total = (long long)nsl * lr.nk;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(i / lr.nk), k = (int)(i - (long long)b * lr.nk);
    const int slice = slice1 + b * skip;
    const double factor = (slice == slice1 || slice == slice2) ? end_weight : 1.0;
    const double2 r = rhok[(size_t)slice * lr.nk + k];
    const double rhok2 = r.x * r.x + r.y * r.y;
    acc += factor * 0.5 * 2.0 * rhok2 * uk[k];
  }
  const double v = lr_block_sum(acc, sh);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = v;
    __threadfence();
    s_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double w = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) w += __ldcg(&partials[i]);
  const double tot = lr_block_sum(w, sh);
  if (threadIdx.x == 0) {
    *out = tot;
    *counter = 0u;
  }
}

__global__ void rhok_copy_kernel(const double2 *__restrict__ src, double2 *dst, int nk, int slice1, int nslices) {
  const long long total = (long long)nslices * nk;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const size_t o = (size_t)slice1 * nk + (size_t)i;
    dst[o] = src[o];
  }
}

}  // namespace

cudaError_t launch_rhok_full(cudaStream_t st, const double *path, int N, int S, const LRDesc &lr, double2 *rhok) {
  rhok_full_kernel<<<S, 256, 0, st>>>(path, N, lr, rhok);
  return cudaGetLastError();
}

cudaError_t launch_rhok_update(cudaStream_t st, const double *path_old, const double *path_new, int N,
                               const LRDesc &lr, const ActiveList &act, int slice1, int slice2, int skip,
                               const double2 *rho_old, double2 *rho_new) {
  const int nsl = (slice2 - slice1) / skip + 1;
  rhok_update_kernel<<<nsl, 256, 0, st>>>(path_old, path_new, N, lr, act, slice1, skip, rho_old, rho_new);
  return cudaGetLastError();
}

cudaError_t launch_lr_sum(const ReduceTarget &t, const double2 *rhok, const LRDesc &lr, const double *uk, int slice1,
                          int slice2, int skip, int sm_count, double end_weight) {
  const int nsl = (slice2 - slice1) / skip + 1;
  long long items = (long long)nsl * lr.nk;
  long long blocks = (items + 255) / 256;
  if (blocks > sm_count * 4) blocks = sm_count * 4;
  if (blocks > kPartialSlots) blocks = kPartialSlots;
  if (blocks < 1) blocks = 1;
  lr_sum_kernel<<<(int)blocks, 256, 0, t.stream>>>(rhok, lr, uk, slice1, slice2, skip, end_weight, t.partials,
                                                   t.counter, t.out);
  return cudaGetLastError();
}

cudaError_t launch_rhok_copy(cudaStream_t st, const double2 *src, double2 *dst, int nk, int slice1, int slice2) {
  const int nsl = slice2 - slice1 + 1;
  const long long items = (long long)nsl * nk;
  rhok_copy_kernel<<<(int)((items + 255) / 256), 256, 0, st>>>(src, dst, nk, slice1, nsl);
  return cudaGetLastError();
}

}  // namespace pimc

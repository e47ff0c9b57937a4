// Read-bandwidth probe: the ceiling against which the bisection kernels'
// table and path gathers are compared when their working set is
// L2-resident (the tables of every benchmark configuration fit the 126 MB L2,
// so HBM bandwidth is not the bound that applies to them).
//
// One launch streams `bytes` of a device buffer `passes` times with 16-byte
// loads through L2 (ld.global.cg, bypassing L1) and folds the words into one
// value per thread, so no load can be dropped.  The buffer is read once
// untimed (it is then resident when it fits L2), then `reps` launches are
// timed with CUDA events on one stream; the result is bytes * passes * reps /
// elapsed time.  Several passes per launch keep the launch gaps out of an
// L2-speed figure.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/pimc_b200.h"

namespace {

__global__ void __launch_bounds__(512) read_kernel(const uint4 *__restrict__ p, size_t n16, int passes,
                                                   unsigned *sink) {
  unsigned acc = 0;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (int ps = 0; ps < passes; ps++) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    // four independent loads in flight per thread per iteration
    for (; i + 3 * stride < n16; i += 4 * stride) {
      const uint4 a = __ldcg(p + i), b = __ldcg(p + i + stride), c = __ldcg(p + i + 2 * stride),
                  d = __ldcg(p + i + 3 * stride);
      acc ^= a.x ^ a.y ^ a.z ^ a.w ^ b.x ^ b.y ^ b.z ^ b.w ^ c.x ^ c.y ^ c.z ^ c.w ^ d.x ^ d.y ^ d.z ^ d.w;
    }
    for (; i < n16; i += stride) {
      const uint4 a = __ldcg(p + i);
      acc ^= a.x ^ a.y ^ a.z ^ a.w;
    }
    acc = acc * 2654435761u + (unsigned)ps;
  }
  if (acc == 0x9e3779b9u) atomicAdd(sink, 1u);  // data dependent: the loads stay
}

}  // namespace

extern "C" int pimc_read_bandwidth(int device, size_t bytes, int passes, int reps, double *gbs) {
  if (!gbs || reps < 1 || passes < 1 || passes > 1024 || bytes < ((size_t)1 << 20) || bytes > ((size_t)8 << 30))
    return PIMC_E_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return PIMC_E_CUDA;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return PIMC_E_CUDA;
  const size_t n16 = bytes / 16;
  uint4 *buf = nullptr;
  unsigned *sink = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = PIMC_OK;
  float ms = 0.0f;
  if (cudaMalloc(&buf, n16 * 16) != cudaSuccess || cudaMalloc(&sink, sizeof(unsigned)) != cudaSuccess) {
    rc = PIMC_E_NOMEM;
  } else if (cudaMemset(buf, 0x5a, n16 * 16) != cudaSuccess || cudaStreamCreate(&st) != cudaSuccess ||
             cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    rc = PIMC_E_CUDA;
  } else {
    const int blocks = sms * 4, threads = 512;  // 4 CTAs x 512 threads per SM: a full SM
    read_kernel<<<blocks, threads, 0, st>>>(buf, n16, 1, sink);  // make the buffer resident
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps; r++) read_kernel<<<blocks, threads, 0, st>>>(buf, n16, passes, sink);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || !(ms > 0.0f))
      rc = PIMC_E_CUDA;
    else
      *gbs = (double)(n16 * 16) * passes * reps / (ms * 1e-3) / 1e9;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  cudaFree(buf);
  cudaFree(sink);
  return rc;
}

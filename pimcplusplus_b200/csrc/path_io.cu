// Path set-up and path files: InitRandomFixed, ShiftPathData, and a
// flat-binary checkpoint of the chain (both path copies plus every RNG
// stream position and move counter).
//
//   pimc_init_random_fixed  PathClass::InitRandomFixed   PIMC++/src/InitPaths.cc:966-999
//   pimc_shift_data         PathClass::ShiftPathData     PIMC++/src/PathClass.cc:1026-1110
//                           (one process: the ring send/receive is a copy to itself)
//   pimc_checkpoint_write/  the reference's path dump / RESTART read
//   pimc_checkpoint_read    (PIMC++/src/InitPaths.cc:826-845 reads an HDF5 "Path"
//                           variable; this build reads no HDF5 and keeps a flat file)
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pimc_internal.h"

using namespace pimc;

namespace {

int io_fail(pimc_context *c, int code, const std::string &msg) {
  if (c) c->last_error = msg;
  return code;
}

#define IOCK(call)                                                                        \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) return io_fail(ctx, PIMC_E_CUDA, std::string(#call) + ": " +   \
                                          cudaGetErrorString(e_));                        \
  } while (0)

// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) on the host; the World
// stream element `index` as the device and the oracle draw it: two 53-bit
// doubles per block, counter (block lo, block hi, stream, 0x50494D43).
void philox_host(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
    c[1] = (uint32_t)p1;
    c[3] = (uint32_t)p0;
    c[0] = n0;
    c[2] = n2;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

double stream_uniform(uint64_t seed, uint32_t stream, uint64_t index) {
  const uint64_t block = index >> 1;
  uint32_t c[4] = {(uint32_t)block, (uint32_t)(block >> 32), stream, 0x50494D43u};
  philox_host(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const int h = (int)(index & 1);
  const uint32_t a = c[2 * h] >> 5, b = c[2 * h + 1] >> 6;
  return ((double)a * 67108864.0 + (double)b) * (1.0 / 9007199254740992.0);
}

// PathClass::PutInBox (PathClass.h:897-921): x -= L * floor(x/L + 0.5).
void put_in_box_host(const double box[3], double v[3]) {
  for (int d = 0; d < 3; d++) {
    const double n = -std::floor(v[d] * (1.0 / box[d]) + 0.5);
    v[d] += n * box[d];
  }
}

// new[j] = old[(j - shift) mod M] for j = 0..M, M = S - 1 (row M repeats row 0).
__global__ void shift_rows_kernel(const double *__restrict__ old_path, double *__restrict__ new_path, int N, int S,
                                  int shift) {
  const int M = S - 1;
  const size_t row = (size_t)N * 3;
  const size_t total = (size_t)S * row;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(i / row);
    int src = (j - shift) % M;
    if (src < 0) src += M;
    new_path[i] = old_path[(size_t)src * row + (i - (size_t)j * row)];
  }
}

// Checkpoint record of one RNG stream and its counters (ChainState without
// the transient status word).
struct StreamRecord {
  uint64_t seed, nlocal;
  uint32_t stream;
  int32_t one_left;
  double x2;
  uint64_t moves, accepted, stages, pair_evals, flips, redone;
};

constexpr char kMagic[8] = {'P', 'I', 'M', 'C', 'C', 'K', 'P', '1'};
constexpr int32_t kVersion = 1;
constexpr uint32_t kStreamShift = 3;  // host-side ShiftMove draws

struct FileCloser {
  FILE *f;
  ~FileCloser() {
    if (f) fclose(f);
  }
};

}  // namespace

extern "C" {

int pimc_init_random_fixed(const double box[3], int num_particles, double radius, uint64_t seed, double *positions) {
  if (!box || !positions || num_particles < 0 || !(radius >= 0.0)) return PIMC_E_ARG;
  for (int d = 0; d < 3; d++)
    if (!(box[d] > 0.0)) return PIMC_E_ARG;
  uint64_t nworld = 0;
  for (int i = 0; i < num_particles; i++) {
    bool overlap = true;
    int tries = 0;
    while (overlap && tries < 1000) {
      tries++;
      for (int d = 0; d < 3; d++) positions[i * 3 + d] = box[d] * (stream_uniform(seed, kStreamWorld, nworld++) - 0.5);
      overlap = false;
      for (int j = 0; j < i; j++) {
        double disp[3];
        for (int d = 0; d < 3; d++) disp[d] = positions[j * 3 + d] - positions[i * 3 + d];
        put_in_box_host(box, disp);
        overlap = overlap || ((disp[0] * disp[0] + disp[1] * disp[1] + disp[2] * disp[2]) < (4.0 * radius * radius));
      }
    }
    // InitRandomFixed aborts once a particle took 1000 tries, even when the
    // last one fitted ("Decrease excluded radius").
    if (tries == 1000) return PIMC_E_CAP;
  }
  return PIMC_OK;
}

int pimc_stream_uniform(uint64_t seed, uint32_t stream, uint64_t index, double *out) {
  if (!out) return PIMC_E_ARG;
  *out = stream_uniform(seed, stream, index);
  return PIMC_OK;
}

int pimc_shift_data(pimc_context *ctx, int slices_to_shift) {
  if (!ctx) return PIMC_E_ARG;
  const int S = ctx->sys.S, N = ctx->sys.N;
  if (S < 2 || std::abs(slices_to_shift) >= S)
    return io_fail(ctx, PIMC_E_ARG, "pimc_shift_data: |slices_to_shift| must be below num_time_slices");
  IOCK(cudaSetDevice(ctx->device));
  const size_t total = (size_t)S * N * 3;
  const int threads = 256;
  const int blocks = (int)std::min<size_t>((total + threads - 1) / threads, (size_t)ctx->sm_count * 8 + 1);
  shift_rows_kernel<<<blocks, threads, 0, ctx->stream>>>(ctx->d_path[0], ctx->d_path[1], N, S, slices_to_shift);
  IOCK(cudaGetLastError());
  IOCK(cudaMemcpyAsync(ctx->d_path[0], ctx->d_path[1], total * sizeof(double), cudaMemcpyDeviceToDevice,
                       ctx->stream));
  ctx->rhok_valid = false;  // ShiftRho_kData: the device moves recompute rho_k of the shifted path
  if (ctx->d_nbr_dirty) IOCK(cudaMemsetAsync(ctx->d_nbr_dirty, 0xff, sizeof(int), ctx->stream));
  IOCK(cudaStreamSynchronize(ctx->stream));
  return PIMC_OK;
}

int pimc_shift_move(pimc_context *ctx, int *slices_shifted) {
  if (!ctx) return PIMC_E_ARG;
  const int M = ctx->sys.S - 1;
  // CommonInt(M) = floor(Common() * M), MetaMoves.cc:54-57, from stream 3
  const int n = (int)std::floor(stream_uniform(ctx->seed, kStreamShift, ctx->shift_draws) * M);
  const int rc = pimc_shift_data(ctx, n);
  if (rc) return rc;
  ctx->shift_draws++;
  if (slices_shifted) *slices_shifted = n;
  return PIMC_OK;
}

int pimc_checkpoint_write(pimc_context *ctx, const char *filename) {
  if (!ctx || !filename) return PIMC_E_ARG;
  IOCK(cudaSetDevice(ctx->device));
  const size_t elems = ctx->path_elems;
  std::vector<double> paths(2 * elems);
  std::vector<ChainState> cs(kMaxChainStates);
  IOCK(cudaMemcpyAsync(paths.data(), ctx->d_path[0], elems * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  IOCK(cudaMemcpyAsync(paths.data() + elems, ctx->d_path[1], elems * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->stream));
  IOCK(cudaMemcpyAsync(cs.data(), ctx->d_chain, cs.size() * sizeof(ChainState), cudaMemcpyDeviceToHost, ctx->stream));
  IOCK(cudaStreamSynchronize(ctx->stream));
  FileCloser fc{fopen(filename, "wb")};
  if (!fc.f) return io_fail(ctx, PIMC_E_FILE, std::string("cannot create ") + filename);
  const int32_t hdr[4] = {kVersion, ctx->sys.N, ctx->sys.S, (int32_t)kMaxChainStates};
  const double sysd[5] = {ctx->sys.box[0], ctx->sys.box[1], ctx->sys.box[2], ctx->sys.tau, ctx->sys.lambda};
  const uint64_t counters[3] = {(uint64_t)ctx->rounds, ctx->seed, (uint64_t)ctx->shift_draws};
  bool ok = fwrite(kMagic, 1, 8, fc.f) == 8 && fwrite(hdr, sizeof(hdr), 1, fc.f) == 1 &&
            fwrite(sysd, sizeof(sysd), 1, fc.f) == 1 && fwrite(counters, sizeof(counters), 1, fc.f) == 1 &&
            fwrite(paths.data(), sizeof(double), paths.size(), fc.f) == paths.size();
  for (int w = 0; ok && w < kMaxChainStates; w++) {
    const ChainState &c = cs[w];
    const StreamRecord r{c.seed, c.nlocal, c.stream, c.one_left, c.x2, c.moves, c.accepted,
                         c.stages, c.pair_evals, c.flips, c.redone};
    ok = fwrite(&r, sizeof(r), 1, fc.f) == 1;
  }
  if (!ok) return io_fail(ctx, PIMC_E_FILE, std::string("short write to ") + filename);
  return PIMC_OK;
}

int pimc_checkpoint_read(pimc_context *ctx, const char *filename) {
  if (!ctx || !filename) return PIMC_E_ARG;
  FileCloser fc{fopen(filename, "rb")};
  if (!fc.f) return io_fail(ctx, PIMC_E_FILE, std::string("cannot open ") + filename);
  char magic[8];
  int32_t hdr[4];
  double sysd[5];
  uint64_t counters[3];
  if (fread(magic, 1, 8, fc.f) != 8 || std::memcmp(magic, kMagic, 8) != 0 || fread(hdr, sizeof(hdr), 1, fc.f) != 1 ||
      fread(sysd, sizeof(sysd), 1, fc.f) != 1 || fread(counters, sizeof(counters), 1, fc.f) != 1)
    return io_fail(ctx, PIMC_E_FILE, std::string(filename) + " is not a pimc_b200 checkpoint");
  if (hdr[0] != kVersion || hdr[3] != (int32_t)kMaxChainStates)
    return io_fail(ctx, PIMC_E_FILE, std::string(filename) + ": unsupported checkpoint version");
  // The chain must be the same system: sizes, box and tau bit for bit.
  if (hdr[1] != ctx->sys.N || hdr[2] != ctx->sys.S || sysd[0] != ctx->sys.box[0] || sysd[1] != ctx->sys.box[1] ||
      sysd[2] != ctx->sys.box[2] || sysd[3] != ctx->sys.tau || sysd[4] != ctx->sys.lambda)
    return io_fail(ctx, PIMC_E_ARG, std::string(filename) + ": checkpoint of a different system (N, slices, box, tau "
                                    "or lambda)");
  const size_t elems = ctx->path_elems;
  std::vector<double> paths(2 * elems);
  if (fread(paths.data(), sizeof(double), paths.size(), fc.f) != paths.size())
    return io_fail(ctx, PIMC_E_FILE, std::string(filename) + ": truncated path data");
  std::vector<ChainState> cs(kMaxChainStates);
  for (int w = 0; w < kMaxChainStates; w++) {
    StreamRecord r;
    if (fread(&r, sizeof(r), 1, fc.f) != 1)
      return io_fail(ctx, PIMC_E_FILE, std::string(filename) + ": truncated stream records");
    ChainState &c = cs[w];
    std::memset(&c, 0, sizeof(c));
    c.seed = r.seed;
    c.nlocal = r.nlocal;
    c.stream = r.stream;
    c.one_left = r.one_left;
    c.x2 = r.x2;
    c.moves = r.moves;
    c.accepted = r.accepted;
    c.stages = r.stages;
    c.pair_evals = r.pair_evals;
    c.flips = r.flips;
    c.redone = r.redone;
  }
  IOCK(cudaSetDevice(ctx->device));
  IOCK(cudaMemcpyAsync(ctx->d_path[0], paths.data(), elems * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  IOCK(cudaMemcpyAsync(ctx->d_path[1], paths.data() + elems, elems * sizeof(double), cudaMemcpyHostToDevice,
                       ctx->stream));
  IOCK(cudaMemcpyAsync(ctx->d_chain, cs.data(), cs.size() * sizeof(ChainState), cudaMemcpyHostToDevice, ctx->stream));
  ctx->rounds = counters[0];
  ctx->seed = counters[1];
  ctx->shift_draws = counters[2];
  ctx->rhok_valid = false;
  if (ctx->d_nbr_dirty) IOCK(cudaMemsetAsync(ctx->d_nbr_dirty, 0xff, sizeof(int), ctx->stream));
  IOCK(cudaStreamSynchronize(ctx->stream));
  return PIMC_OK;
}

}  // extern "C"

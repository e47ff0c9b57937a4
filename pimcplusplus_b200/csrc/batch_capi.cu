// Batched independent chains (the reference's clone parallelism,
// PathDataClass.cc:244-268, on one GPU): C ABI over batch_kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "bisection.cuh"
#include "pimc_internal.h"

using namespace pimc;

struct pimc_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  int n_chains = 0;
  std::vector<pimc_chain_desc> desc;
  std::vector<size_t> path_off;  // doubles
  std::vector<BisectionArgs> jobs;
  double *d_paths = nullptr;
  size_t path_doubles = 0;
  std::vector<void *> owned;
  BisectionArgs *d_jobs = nullptr;
  int *d_order = nullptr;
  unsigned int *d_queue = nullptr;
  ChainState *d_chains = nullptr;
  pimc_move_record *d_trace = nullptr;
  size_t trace_cap = 0;
  int precision = PIMC_MIXED, shadow = 0, threads = 256;
  int max_split = 0;
  int split[kMaxSplit] = {};
  std::vector<double> cost_sorted;  // estimated cost of each queue position
  size_t dyn = 0;
  int blocks = 0;
  int sm_count = 0;
  // the launch (queue reset + persistent kernel) captured as a CUDA graph,
  // valid for graph_blocks blocks of moves under configuration cfg_version
  cudaGraphExec_t graph = nullptr;
  int graph_blocks = -1;
  int cfg_version = 0, graph_version = -1;
  std::string last_error;
};

namespace {

int bfail(pimc_batch *b, int code, const std::string &msg) {
  if (b) b->last_error = msg;
  return code;
}

#define BCK(call)                                                                               \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) return bfail(b, PIMC_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
int bupload(pimc_batch *b, const std::vector<T> &host, const T **dev) {
  void *p = nullptr;
  BCK(cudaMalloc(&p, host.size() * sizeof(T) + 16));
  b->owned.push_back(p);
  BCK(cudaMemset(p, 0, host.size() * sizeof(T) + 16));
  BCK(cudaMemcpy(p, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice));
  *dev = static_cast<const T *>(p);
  return PIMC_OK;
}

// The diagonal DavidPA column of one chain, appended to `host` (R pairs):
// (y, d2y) per grid point and level, the natural-start / zero-end-slope
// spline of DavidPAClass (DavidPAClass.cc:760-763).  Every chain's block
// starts at a multiple of 2 pairs so a level's bulk copy stays 16-byte
// aligned.  d.diag receives the OFFSET in pairs; it is rebased once the
// packed array is on the device.
template <typename R>
void build_diag(const pimc_chain_desc &c, const HostGrid &g, std::vector<R> &host, DDavid<R> &d) {
  d.grid.type = PIMC_GRID_LINEAR;
  d.grid.n = g.n;
  d.grid.start = (R)g.start;
  d.grid.end = (R)g.end;
  d.grid.delta = (R)g.delta;
  d.grid.deltainv = (R)g.deltainv;
  d.grid.r0 = 0;
  d.grid.log_spacing = 0;
  d.grid.x = nullptr;
  d.ncols = 2;
  d.num_tau = c.num_tau;
  d.tau_pos = c.tau_pos;
  d.num_terms = 0;
  d.uy = d.ud2 = d.duy = d.dud2 = nullptr;
  d.diag_stride = (g.n + 1) & ~1;
  const size_t base = host.size() / 2;  // pairs
  host.resize(host.size() + (size_t)c.num_tau * d.diag_stride * 2, (R)0);
  std::vector<double> d2(g.n);
  for (int lev = 0; lev < c.num_tau; lev++) {
    const double *y = c.u00 + (size_t)lev * g.n;
    spline_second_derivs(g, y, 1, 0, 5.0e30, 0.0, d2.data());
    R *o = host.data() + (base + (size_t)lev * d.diag_stride) * 2;
    for (int i = 0; i < g.n; i++) {
      o[2 * i] = (R)y[i];
      o[2 * i + 1] = (R)d2[i];
    }
  }
  d.diag = reinterpret_cast<const R *>(base);
}

template <typename R>
void rebase_diag(DDavid<R> &d, const R *dev) {
  d.diag = dev + 2 * reinterpret_cast<size_t>(d.diag);
}

void drop_graph(pimc_batch *b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  b->graph_blocks = -1;
}

// Shared memory for the staged tables: the working precision's column plus,
// with the shadow evaluation, the other precision's (FP32 pairs are half the
// FP64 bytes).
// One slot's share; the launch holds 2^max_split slots.
size_t batch_dyn_slot(const pimc_batch *b) {
  const size_t b64 = b->dyn, b32 = b->dyn / 2;
  size_t d = b->precision == PIMC_MIXED ? b32 : b64;
  if (b->shadow) d += b->precision == PIMC_MIXED ? b64 : b32;
  return (d + 15) & ~(size_t)15;
}
size_t batch_dyn(const pimc_batch *b) { return batch_dyn_slot(b) << b->max_split; }

}  // namespace

extern "C" {

int pimc_batch_create(int device, int n_chains, const pimc_chain_desc *chains, pimc_batch **out) {
  if (!out || !chains || n_chains < 1) return PIMC_E_ARG;
  *out = nullptr;
  pimc_batch *b = new (std::nothrow) pimc_batch();
  if (!b) return PIMC_E_NOMEM;
  b->device = device;
  b->n_chains = n_chains;
  b->desc.assign(chains, chains + n_chains);
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) {
    pimc_batch_destroy(b);
    return PIMC_E_CUDA;
  }
  // validate and lay out the paths
  size_t total = 0;
  size_t maxdyn = 0;
  for (int i = 0; i < n_chains; i++) {
    const pimc_chain_desc &c = chains[i];
    if (c.num_particles < 2 || c.num_particles > (1 << 20) || c.num_time_slices < 3 || !c.path || !c.u00 ||
        !(c.tau > 0.0) || c.num_images < 0 || c.num_levels < 1 || c.num_levels > 6 ||
        (1 << c.num_levels) >= c.num_time_slices || c.steps_per_block < 1 || c.num_grid < 3 ||
        !(c.grid_end > c.grid_start) || c.num_tau < 1 || c.tau_pos < 0 || c.tau_pos + c.num_levels > c.num_tau) {
      int rc = bfail(b, PIMC_E_ARG, "chain " + std::to_string(i) + ": bad description");
      pimc_batch_destroy(b);
      return rc;
    }
    for (int d = 0; d < 3; d++)
      if (!(c.box[d] > 0.0)) {
        pimc_batch_destroy(b);
        return PIMC_E_ARG;
      }
    b->path_off.push_back(total);
    total += (size_t)c.num_time_slices * c.num_particles * 3;
    const size_t stride = (size_t)((c.num_grid + 1) & ~1);
    maxdyn = std::max(maxdyn, (size_t)c.num_levels * stride * sizeof(double2));
  }
  b->path_doubles = total;
  b->dyn = maxdyn;  // FP64 pairs; see batch_dyn for the other configurations
  e = cudaMalloc(&b->d_paths, total * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_chains, n_chains * sizeof(ChainState));
  if (e == cudaSuccess) e = cudaMemset(b->d_chains, 0, n_chains * sizeof(ChainState));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_jobs, n_chains * sizeof(BisectionArgs));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_order, n_chains * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_queue, sizeof(unsigned int));
  if (e != cudaSuccess) {
    pimc_batch_destroy(b);
    return PIMC_E_CUDA;
  }
  std::vector<ChainState> cs(n_chains);
  std::vector<double> diag64;
  std::vector<float> diag32;
  b->jobs.resize(n_chains);
  for (int i = 0; i < n_chains; i++) {
    const pimc_chain_desc &c = chains[i];
    e = cudaMemcpy(b->d_paths + b->path_off[i], c.path,
                   (size_t)c.num_time_slices * c.num_particles * 3 * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      pimc_batch_destroy(b);
      return PIMC_E_CUDA;
    }
    HostGrid g;
    g.init_linear(c.grid_start, c.grid_end, c.num_grid);
    BisectionArgs &j = b->jobs[i];
    std::memset(&j, 0, sizeof(j));
    j.path = b->d_paths + b->path_off[i];
    DevSystem &s = j.sys;
    s.N = c.num_particles;
    s.S = c.num_time_slices;
    for (int d = 0; d < 3; d++) {
      s.box[d] = c.box[d];
      s.boxinv[d] = 1.0 / c.box[d];
    }
    s.tau = c.tau;
    s.lambda = c.lambda;
    s.num_images = c.num_images;
    j.pa.kind = PA_DAVID;
    build_diag<double>(c, g, diag64, j.pa.d64);
    build_diag<float>(c, g, diag32, j.pa.d32);
    j.chains = b->d_chains + i;
    j.num_levels = c.num_levels;
    j.steps_per_block = c.steps_per_block;
    j.sr_higher = 1;
    j.concurrent = 0;
    j.guard = guard_mode(PIMC_GUARD_DECISION);
    cs[i].seed = c.seed;
    cs[i].stream = kStreamLocal;
  }
  {
    const double *p64 = nullptr;
    const float *p32 = nullptr;
    int rc = bupload(b, diag64, &p64);
    if (!rc) rc = bupload(b, diag32, &p32);
    if (rc) {
      pimc_batch_destroy(b);
      return rc;
    }
    for (auto &j : b->jobs) {
      rebase_diag(j.pa.d64, p64);
      rebase_diag(j.pa.d32, p32);
    }
  }
  // largest chains first: cost ~ N * 2^L * StepsPerBlock
  std::vector<int> order(n_chains);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    const double cx = (double)chains[x].num_particles * (1 << chains[x].num_levels) * chains[x].steps_per_block;
    const double cy = (double)chains[y].num_particles * (1 << chains[y].num_levels) * chains[y].steps_per_block;
    return cx > cy;
  });
  b->cost_sorted.resize(n_chains);
  for (int i = 0; i < n_chains; i++)
    b->cost_sorted[i] =
        (double)chains[order[i]].num_particles * (1 << chains[order[i]].num_levels) * chains[order[i]].steps_per_block;
  e = cudaMemcpy(b->d_jobs, b->jobs.data(), n_chains * sizeof(BisectionArgs), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_order, order.data(), n_chains * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_chains, cs.data(), n_chains * sizeof(ChainState), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    pimc_batch_destroy(b);
    return PIMC_E_CUDA;
  }
  *out = b;
  return PIMC_OK;
}

int pimc_batch_destroy(pimc_batch *b) {
  if (!b) return PIMC_E_ARG;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  for (void *p : b->owned) cudaFree(p);
  cudaFree(b->d_paths);
  cudaFree(b->d_chains);
  cudaFree(b->d_jobs);
  cudaFree(b->d_order);
  cudaFree(b->d_queue);
  cudaFree(b->d_trace);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return PIMC_OK;
}

int pimc_batch_last_error(pimc_batch *b, char *buf, int len) {
  if (!b || !buf || len <= 0) return PIMC_E_ARG;
  std::snprintf(buf, (size_t)len, "%s", b->last_error.c_str());
  return PIMC_OK;
}

int pimc_batch_config(pimc_batch *b, int precision, int shadow, int threads_per_cta, int ctas, int max_split,
                      double split_ratio) {
  if (!b) return PIMC_E_ARG;
  if (precision != PIMC_FP64 && precision != PIMC_MIXED) return bfail(b, PIMC_E_ARG, "bad precision");
  const int threads = threads_per_cta ? threads_per_cta : 256;
  if (max_split < 0 || max_split > kMaxSplit) return bfail(b, PIMC_E_ARG, "max_split must be in 0..2");
  if (threads < 64 || threads > 512 || (threads >> max_split) % 32 || (threads >> max_split) < 64)
    return bfail(b, PIMC_E_ARG, "threads_per_cta must be in 64..512 and split into groups of 64+ (multiples of 32)");
  if (max_split > 0 && !(split_ratio > 0.0 && split_ratio < 1.0))
    return bfail(b, PIMC_E_ARG, "split_ratio must be in (0, 1)");
  if (ctas < 0) return bfail(b, PIMC_E_ARG, "ctas must be >= 0");
  BCK(cudaSetDevice(b->device));
  const int old_split = b->max_split;
  b->precision = precision;
  b->shadow = shadow;
  b->threads = threads;
  b->max_split = max_split;
  // level k+1 groups take the chains from the first queue position whose
  // cost is at most ratio^(k+1) of the largest
  for (int k = 0; k < kMaxSplit; k++) {
    int pos = b->n_chains;
    if (k < max_split) {
      const double lim = b->cost_sorted[0] * std::pow(split_ratio, k + 1);
      pos = 0;
      while (pos < b->n_chains && b->cost_sorted[pos] > lim) pos++;
    }
    b->split[k] = pos;
  }
  const size_t dyn = batch_dyn(b);
  int per_sm = 0;
  cudaError_t e = dyn > (size_t)140 * 1024 ? cudaErrorInvalidValue
                                           : batch_occupancy(precision, shadow, b->threads, dyn, &per_sm);
  if (e != cudaSuccess || per_sm < 1) {
    b->max_split = old_split;
    cudaGetLastError();
    return bfail(b, PIMC_E_ARG, "configuration does not fit on an SM");
  }
  b->blocks = ctas ? ctas : std::min(b->n_chains, per_sm * b->sm_count);
  b->cfg_version++;
  return PIMC_OK;
}

static int batch_launch(pimc_batch *b, int n_blocks, pimc_move_record *dtrace, long long per_chain) {
  if (b->blocks == 0) {
    int rc = pimc_batch_config(b, b->precision, b->shadow, b->threads, 0, 0, 0.5);
    if (rc) return rc;
  }
  BCK(cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned int), b->stream));
  BatchArgs a;
  a.jobs = b->d_jobs;
  a.order = b->d_order;
  a.queue = b->d_queue;
  a.n_chains = b->n_chains;
  a.n_blocks = n_blocks;
  a.trace = dtrace;
  a.trace_per_chain = per_chain;
  a.max_split = b->max_split;
  for (int k = 0; k < kMaxSplit; k++) a.split[k] = b->split[k];
  a.dyn_per_slot = (unsigned)batch_dyn_slot(b);
  const size_t dyn = batch_dyn(b);
  BCK(launch_batch(a, b->precision, b->shadow, b->blocks, b->threads, dyn, b->stream));
  return PIMC_OK;
}

int pimc_batch_run_async(pimc_batch *b, int n_blocks) {
  if (!b || n_blocks < 0) return PIMC_E_ARG;
  BCK(cudaSetDevice(b->device));
  if (b->blocks == 0) {
    int rc = pimc_batch_config(b, b->precision, b->shadow, b->threads, 0, 0, 0.5);
    if (rc) return rc;
  }
  if (!b->graph || b->graph_blocks != n_blocks || b->graph_version != b->cfg_version) {
    drop_graph(b);
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
    const int rc = batch_launch(b, n_blocks, nullptr, 0);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return bfail(b, PIMC_E_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
      b->graph = nullptr;
      return bfail(b, PIMC_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
    }
    b->graph_blocks = n_blocks;
    b->graph_version = b->cfg_version;
  }
  BCK(cudaGraphLaunch(b->graph, b->stream));
  return PIMC_OK;
}

int pimc_batch_autotune(pimc_batch *b, int n_blocks, int *threads_out, int *ctas_out, int *split_out,
                        double *ratio_out, double *ms_out) {
  if (!b || n_blocks < 1) return PIMC_E_ARG;
  BCK(cudaSetDevice(b->device));
  BCK(cudaStreamSynchronize(b->stream));
  // The probes advance the chains: keep their state and put it back after.
  double *save_paths = nullptr;
  ChainState *save_cs = nullptr;
  BCK(cudaMalloc(&save_paths, b->path_doubles * sizeof(double)));
  cudaError_t e = cudaMalloc(&save_cs, b->n_chains * sizeof(ChainState));
  if (e != cudaSuccess) {
    cudaFree(save_paths);
    return bfail(b, PIMC_E_CUDA, "autotune: no room for the state copy");
  }
  e = cudaMemcpyAsync(save_paths, b->d_paths, b->path_doubles * sizeof(double), cudaMemcpyDeviceToDevice, b->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(save_cs, b->d_chains, b->n_chains * sizeof(ChainState), cudaMemcpyDeviceToDevice, b->stream);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  const int precision = b->precision, shadow = b->shadow;
  int best_t = 0, best_c = 0, best_s = 0, rc = PIMC_OK;
  double best_r = 0.5;
  float best_ms = 0.f;
  const int cand_threads[] = {128, 256, 384, 512};
  const double cand_ratio[] = {0.5, 0.25};
  for (int ti = 0; ti < 4 && e == cudaSuccess && rc == PIMC_OK; ti++)
    for (int ms_ = 0; ms_ <= kMaxSplit && rc == PIMC_OK && e == cudaSuccess; ms_++)
      for (int ri = 0; ri < (ms_ ? 2 : 1) && rc == PIMC_OK && e == cudaSuccess; ri++) {
        rc = pimc_batch_config(b, precision, shadow, cand_threads[ti], 0, ms_, cand_ratio[ri]);
        if (rc == PIMC_E_ARG) {  // does not fit: not a candidate
          rc = PIMC_OK;
          continue;
        }
        if (rc) break;
        rc = batch_launch(b, n_blocks, nullptr, 0);  // warm-up (module load, caches)
        if (rc) break;
        e = cudaEventRecord(e0, b->stream);
        if (e == cudaSuccess) rc = batch_launch(b, n_blocks, nullptr, 0);
        if (e == cudaSuccess && rc == PIMC_OK) e = cudaEventRecord(e1, b->stream);
        if (e == cudaSuccess && rc == PIMC_OK) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess && rc == PIMC_OK) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess || rc) break;
        if (best_t == 0 || ms < best_ms) {
          best_ms = ms;
          best_t = cand_threads[ti];
          best_c = b->blocks;
          best_s = ms_;
          best_r = cand_ratio[ri];
        }
      }
  cudaError_t er = cudaMemcpyAsync(b->d_paths, save_paths, b->path_doubles * sizeof(double),
                                   cudaMemcpyDeviceToDevice, b->stream);
  if (er == cudaSuccess)
    er = cudaMemcpyAsync(b->d_chains, save_cs, b->n_chains * sizeof(ChainState), cudaMemcpyDeviceToDevice, b->stream);
  if (er == cudaSuccess) er = cudaStreamSynchronize(b->stream);
  cudaFree(save_paths);
  cudaFree(save_cs);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (rc) return rc;
  if (e != cudaSuccess) return bfail(b, PIMC_E_CUDA, std::string("autotune: ") + cudaGetErrorString(e));
  if (er != cudaSuccess) return bfail(b, PIMC_E_CUDA, std::string("autotune restore: ") + cudaGetErrorString(er));
  if (best_t == 0) return bfail(b, PIMC_E_ARG, "autotune: no configuration fits");
  rc = pimc_batch_config(b, precision, shadow, best_t, best_c, best_s, best_r);
  if (rc) return rc;
  if (threads_out) *threads_out = best_t;
  if (ctas_out) *ctas_out = best_c;
  if (split_out) *split_out = best_s;
  if (ratio_out) *ratio_out = best_r;
  if (ms_out) *ms_out = best_ms;
  return PIMC_OK;
}

int pimc_batch_run(pimc_batch *b, int n_blocks, pimc_move_record *trace, pimc_bisection_stats *stats) {
  if (!b || n_blocks < 0) return PIMC_E_ARG;
  BCK(cudaSetDevice(b->device));
  int spb = 0;
  for (const auto &c : b->desc) spb = std::max(spb, c.steps_per_block);
  const long long per_chain = (long long)n_blocks * spb;
  const size_t nrec = (size_t)per_chain * b->n_chains;
  if (trace && nrec > b->trace_cap) {
    cudaFree(b->d_trace);
    b->d_trace = nullptr;
    b->trace_cap = 0;
    BCK(cudaMalloc(&b->d_trace, nrec * sizeof(pimc_move_record)));
    b->trace_cap = nrec;
  }
  if (trace) BCK(cudaMemsetAsync(b->d_trace, 0, nrec * sizeof(pimc_move_record), b->stream));
  int rc = batch_launch(b, n_blocks, trace ? b->d_trace : nullptr, per_chain);
  if (rc) return rc;
  if (trace) BCK(cudaMemcpyAsync(trace, b->d_trace, nrec * sizeof(pimc_move_record), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  pimc_bisection_stats st;
  rc = pimc_batch_get_stats(b, -1, &st);
  if (rc) return rc;
  if (stats) *stats = st;
  if (st.status) return bfail(b, st.status, std::string("device status: ") + pimc_status_string(st.status));
  return PIMC_OK;
}

int pimc_batch_get_stats(pimc_batch *b, int chain, pimc_bisection_stats *stats) {
  if (!b || !stats || chain < -1 || chain >= b->n_chains) return PIMC_E_ARG;
  BCK(cudaSetDevice(b->device));
  std::vector<ChainState> cs(b->n_chains);
  BCK(cudaMemcpyAsync(cs.data(), b->d_chains, cs.size() * sizeof(ChainState), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  std::memset(stats, 0, sizeof(*stats));
  for (int i = 0; i < b->n_chains; i++) {
    if (chain >= 0 && i != chain) continue;
    const ChainState &c = cs[i];
    stats->moves += (int64_t)c.moves;
    stats->accepted += (int64_t)c.accepted;
    stats->stages_attempted += (int64_t)c.stages;
    stats->pair_evals += (int64_t)c.pair_evals;
    stats->flips += (int64_t)c.flips;
    stats->reevaluated += (int64_t)c.reevals;
    if (c.status && !stats->status) stats->status = c.status;
  }
  return PIMC_OK;
}

int pimc_batch_set_guard(pimc_batch *b, int guard) {
  if (!b || guard < 0 || guard > 2) return PIMC_E_ARG;
  BCK(cudaSetDevice(b->device));
  BCK(cudaStreamSynchronize(b->stream));
  for (auto &j : b->jobs) j.guard = guard_mode(guard);
  BCK(cudaMemcpy(b->d_jobs, b->jobs.data(), b->jobs.size() * sizeof(BisectionArgs), cudaMemcpyHostToDevice));
  drop_graph(b);
  b->cfg_version++;
  return PIMC_OK;
}

int pimc_batch_get_path(pimc_batch *b, int chain, double *path) {
  if (!b || !path || chain < 0 || chain >= b->n_chains) return PIMC_E_ARG;
  BCK(cudaSetDevice(b->device));
  const pimc_chain_desc &c = b->desc[chain];
  BCK(cudaMemcpy(path, b->d_paths + b->path_off[chain],
                 (size_t)c.num_time_slices * c.num_particles * 3 * sizeof(double), cudaMemcpyDeviceToHost));
  return PIMC_OK;
}

void *pimc_batch_stream(pimc_batch *b) { return b ? (void *)b->stream : nullptr; }

int pimc_batch_synchronize(pimc_batch *b) {
  if (!b) return PIMC_E_ARG;
  BCK(cudaSetDevice(b->device));
  BCK(cudaStreamSynchronize(b->stream));
  return PIMC_OK;
}

}  // extern "C"

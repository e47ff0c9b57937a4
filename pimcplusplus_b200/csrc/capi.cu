// C ABI of the B200 PIMC action library (include/pimc_b200.h).  Host-side
// argument checks mirror the reference's asserts, but report a status code
// instead of aborting; no C++ exception crosses the ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "action_kernels.cuh"
#include "bisection.cuh"
#include "longrange.cuh"
#include "pimc_internal.h"

using namespace pimc;

namespace {

int fail(pimc_context *c, int code, const std::string &msg) {
  if (c) c->last_error = msg;
  return code;
}

int cuda_fail(pimc_context *c, cudaError_t e, const char *where) {
  return fail(c, PIMC_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                        \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

template <typename T>
int upload(pimc_context *ctx, const T *host, size_t n, const T **dev, size_t pad_bytes = 16) {
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, n * sizeof(T) + pad_bytes);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc(table)");
  ctx->owned.push_back(p);
  e = cudaMemset(p, 0, n * sizeof(T) + pad_bytes);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemset(table)");
  e = cudaMemcpy(p, host, n * sizeof(T), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpy(table)");
  *dev = static_cast<const T *>(p);
  return PIMC_OK;
}

template <typename R>
int upload_grid(pimc_context *ctx, const HostGrid &h, DGrid<R> &g) {
  g.type = h.type;
  g.n = h.n;
  g.start = (R)h.start;
  g.end = (R)h.end;
  g.delta = (R)h.delta;
  g.deltainv = (R)h.deltainv;
  g.r0 = (R)h.r0;
  g.log_spacing = (R)h.log_spacing;
  g.x = nullptr;
  if (h.type == PIMC_GRID_LOG) {
    std::vector<R> x(h.x.begin(), h.x.end());
    return upload(ctx, x.data(), x.size(), &g.x);
  }
  return PIMC_OK;
}

template <typename R>
int upload_david(pimc_context *ctx, const DavidTables &t, DDavid<R> &d) {
  int rc = upload_grid(ctx, t.grid, d.grid);
  if (rc) return rc;
  d.ncols = t.ncols;
  d.num_tau = t.num_tau;
  d.tau_pos = t.tau_pos;
  d.num_terms = t.num_terms;
  const size_t n = t.uy.size();
  std::vector<R> buf(n);
  const std::vector<double> *srcs[4] = {&t.uy, &t.ud2, &t.duy, &t.dud2};
  const R **dsts[4] = {&d.uy, &d.ud2, &d.duy, &d.dud2};
  for (int k = 0; k < 4; k++) {
    for (size_t i = 0; i < n; i++) buf[i] = (R)(*srcs[k])[i];
    if ((rc = upload(ctx, buf.data(), n, dsts[k]))) return rc;
  }
  // diagonal column (col 1) as (y, d2y) pairs, levels padded to an even count
  const int np = t.grid.n;
  d.diag_stride = (np + 1) & ~1;
  std::vector<R> diag((size_t)t.num_tau * d.diag_stride * 2, (R)0);
  for (int lev = 0; lev < t.num_tau; lev++)
    for (int i = 0; i < np; i++) {
      size_t src = ((size_t)lev * np + i) * t.ncols + 1;
      diag[((size_t)lev * d.diag_stride + i) * 2] = (R)t.uy[src];
      diag[((size_t)lev * d.diag_stride + i) * 2 + 1] = (R)t.ud2[src];
    }
  return upload(ctx, diag.data(), diag.size(), &d.diag);
}

int check_pair(pimc_context *ctx, int sp1, int sp2) {
  if (!ctx) return PIMC_E_ARG;
  if (sp1 < 0 || sp2 < 0 || sp1 >= ctx->num_species || sp2 >= ctx->num_species)
    return fail(ctx, PIMC_E_ARG, "species index out of range");
  if (ctx->num_species != 1) return fail(ctx, PIMC_E_ARG, "one species per context is supported");
  return PIMC_OK;
}

int set_david(pimc_context *ctx, DavidTables &t) {
  int rc;
  if ((rc = upload_david<double>(ctx, t, ctx->pa.d64))) return rc;
  if ((rc = upload_david<float>(ctx, t, ctx->pa.d32))) return rc;
  ctx->pa.kind = PA_DAVID;
  return PIMC_OK;
}

int check_active(pimc_context *ctx, const int *active, int n, ActiveList &out) {
  if (n < 0 || n > kMaxActive) return fail(ctx, PIMC_E_ARG, "n_active out of range");
  if (n > 0 && !active) return fail(ctx, PIMC_E_ARG, "active is null");
  out.n = n;
  for (int i = 0; i < n; i++) {
    if (active[i] < 0 || active[i] >= ctx->sys.N) return fail(ctx, PIMC_E_ARG, "active particle out of range");
    out.p[i] = active[i];
  }
  return PIMC_OK;
}

int finish_scalar(pimc_context *ctx, double *out) {
  CK(cudaMemcpyAsync(ctx->h_out, ctx->d_out, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *out = *ctx->h_out;
  if (!std::isfinite(*out)) return fail(ctx, PIMC_E_NAN, "non-finite action");
  return PIMC_OK;
}

LRDesc lr_desc(const pimc_context *ctx) {
  LRDesc lr;
  lr.nk = ctx->num_k;
  for (int d = 0; d < 3; d++) {
    lr.kmax[d] = ctx->kmax[d];
    lr.kbox[d] = ctx->kbox[d];
  }
  lr.coff[0] = 0;
  lr.coff[1] = 2 * ctx->kmax[0] + 1;
  lr.coff[2] = lr.coff[1] + 2 * ctx->kmax[1] + 1;
  lr.kidx = ctx->d_kidx;
  return lr;
}

// PairActionFitClass::IsLongRange of the context's pair action.
// PairActionFitClass::IsLongRange: PAtricubicFit (PAtricubicFit.cc:869-872) and
// a classical Coulomb action with Z1Z2 != 0 (PAclassicalFit.cc:112-117).
bool pa_long_range(const pimc_context *ctx) {
  return ctx->pa.kind == PA_TRICUBIC || (ctx->pa.kind == PA_COULOMB && ctx->pa.c64.z1z2 != 0.0);
}

int pa_levels_ok(pimc_context *ctx, int levels_needed) {
  if (ctx->pa.kind == PA_DAVID && levels_needed + ctx->pa.d64.tau_pos > ctx->pa.d64.num_tau)
    return fail(ctx, PIMC_E_ARG, "level beyond the pair action's tau levels");
  if (ctx->pa.kind == PA_TRICUBIC && levels_needed > ctx->pa.t64.num_betas)
    return fail(ctx, PIMC_E_ARG, "level beyond the pair action's beta levels");
  if (ctx->pa.kind == PA_COULOMB && levels_needed > ctx->pa.c64.num_levels)
    return fail(ctx, PIMC_E_ARG, "level beyond the pair action's beta levels");
  return PIMC_OK;
}

// The constant (Madelung, k=0 / background) part of LongRangeClass's sum over
// slices [slice1, slice2] step 2^level (LongRangeClass.cc:320-366).
double lr_constant(const pimc_context *ctx, int slice1, int slice2, int level, bool deriv) {
  const int skip = 1 << level;
  const double N = (double)ctx->sys.N;
  const double r0 = deriv ? ctx->dulong_r0[level] : ctx->ulong_r0[level];
  const double sk0 = deriv ? ctx->dushort_k0[level] : ctx->ushort_k0[level];
  const double lk0 = deriv ? ctx->dulong_k0[level] : ctx->ulong_k0[level];
  double homo = 0.0, background = 0.0, k0Homo = 0.0;
  for (int slice = slice1; slice <= slice2; slice += skip) {
    const double factor = (slice == slice1 || slice == slice2) ? 0.5 : 1.0;
    homo -= factor * 0.5 * N * r0;
    background -= factor * 0.5 * N * N * sk0;
    k0Homo += factor * 0.5 * N * N * lk0;
  }
  return homo + (ctx->use_background ? background : k0Homo);
}

}  // namespace

extern "C" {

const char *pimc_status_string(int status) {
  switch (status) {
    case PIMC_OK: return "ok";
    case PIMC_E_ARG: return "invalid argument";
    case PIMC_E_CUDA: return "CUDA error";
    case PIMC_E_NAN: return "non-finite action";
    case PIMC_E_INDEX: return "index out of range";
    case PIMC_E_CAP: return "device loop cap reached";
    case PIMC_E_FILE: return "file missing or malformed";
    case PIMC_E_STATE: return "call out of order";
    case PIMC_E_NOMEM: return "allocation failed";
    case PIMC_E_STAGING: return "broken staging (|S| > 1e50)";
    default: return "unknown status";
  }
}

int pimc_version(void) { return 100; }

int pimc_create(const pimc_system_desc *d, pimc_context **out) {
  if (!d || !out) return PIMC_E_ARG;
  *out = nullptr;
  if (d->num_particles < 2 || d->num_time_slices < 2 || d->num_species < 1 || !d->species_of || !d->lambda)
    return PIMC_E_ARG;
  for (int i = 0; i < 3; i++)
    if (!(d->box[i] > 0.0)) return PIMC_E_ARG;
  if (!(d->tau > 0.0) || d->num_images < 0) return PIMC_E_ARG;
  pimc_context *ctx = new (std::nothrow) pimc_context();
  if (!ctx) return PIMC_E_NOMEM;
  ctx->device = d->device;
  ctx->num_species = d->num_species;
  ctx->species_of.assign(d->species_of, d->species_of + d->num_particles);
  ctx->lambda.assign(d->lambda, d->lambda + d->num_species);
  for (int s : ctx->species_of)
    if (s < 0 || s >= d->num_species) {
      delete ctx;
      return PIMC_E_ARG;
    }
  DevSystem &s = ctx->sys;
  s.N = d->num_particles;
  s.S = d->num_time_slices;
  for (int i = 0; i < 3; i++) {
    s.box[i] = d->box[i];
    s.boxinv[i] = 1.0 / d->box[i];
  }
  s.tau = d->tau;
  s.lambda = d->lambda[0];
  s.num_images = d->num_images;
  cudaError_t e = cudaSetDevice(d->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  ctx->path_elems = (size_t)s.S * s.N * 3;
  for (int c = 0; c < 2 && e == cudaSuccess; c++) e = cudaMalloc(&ctx->d_path[c], ctx->path_elems * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_partials, kPartialSlots * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_counter, sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset(ctx->d_counter, 0, sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_out, 4 * sizeof(double));
  if (e == cudaSuccess) e = cudaMallocHost(&ctx->h_out, 4 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_chain, kMaxChainStates * sizeof(ChainState));
  if (e == cudaSuccess) e = cudaMemset(ctx->d_chain, 0, kMaxChainStates * sizeof(ChainState));
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, d->device);
  if (e == cudaSuccess) e = cudaMemset(ctx->d_path[0], 0, ctx->path_elems * sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(ctx->d_path[1], 0, ctx->path_elems * sizeof(double));
  if (e != cudaSuccess) {
    pimc_destroy(ctx);
    return PIMC_E_CUDA;
  }
  *out = ctx;
  return PIMC_OK;
}

int pimc_destroy(pimc_context *ctx) {
  if (!ctx) return PIMC_E_ARG;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (void *p : ctx->owned) cudaFree(p);
  for (int c = 0; c < 2; c++) cudaFree(ctx->d_path[c]);
  cudaFree(ctx->d_partials);
  cudaFree(ctx->d_counter);
  cudaFree(ctx->d_out);
  if (ctx->h_out) cudaFreeHost(ctx->h_out);
  cudaFree(ctx->d_chain);
  cudaFree(ctx->d_trace);
  cudaFree(ctx->d_kidx);
  cudaFree(ctx->d_rhok[0]);
  cudaFree(ctx->d_rhok[1]);
  cudaFree(ctx->d_ulong_k);
  cudaFree(ctx->d_dulong_k);
  cudaFree(ctx->d_yk);
  cudaFree(ctx->d_gofr);
  cudaFree(ctx->d_kvec);
  cudaFree(ctx->d_nbr_cb);
  cudaFree(ctx->d_nbr_cnt);
  cudaFree(ctx->d_nbr_idx);
  cudaFree(ctx->d_nbr_dirty);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return PIMC_OK;
}

int pimc_last_error(pimc_context *ctx, char *buf, int len) {
  if (!ctx || !buf || len <= 0) return PIMC_E_ARG;
  std::snprintf(buf, (size_t)len, "%s", ctx->last_error.c_str());
  return PIMC_OK;
}

int pimc_pa_david_from_dm(pimc_context *ctx, int sp1, int sp2, const char *dm_path, int num_offdiag_terms) {
  int rc = check_pair(ctx, sp1, sp2);
  if (rc) return rc;
  if (!dm_path) return fail(ctx, PIMC_E_ARG, "dm_path is null");
  if (num_offdiag_terms < 0) return fail(ctx, PIMC_E_ARG, "negative NumOffDiagonalTerms");
  CK(cudaSetDevice(ctx->device));
  DavidTables t;
  std::string err;
  rc = read_dm_file(dm_path, ctx->sys.tau, num_offdiag_terms, t, err);
  if (rc) return fail(ctx, rc, err);
  if (t.ncols < 2 || (num_offdiag_terms > 0 && (num_offdiag_terms + 1) * (num_offdiag_terms + 2) / 2 > t.ncols - 1))
    return fail(ctx, PIMC_E_FILE, "fit has too few ukj columns for NumOffDiagonalTerms");
  return set_david(ctx, t);
}

int pimc_dm_read_info(const char *dm_path, double desired_tau, int *num_grid, int *num_cols, int *num_tau,
                      int *tau_pos, int *grid_type, double *grid_start, double *grid_end) {
  if (!dm_path) return PIMC_E_ARG;
  DavidTables t;
  std::string err;
  int rc = read_dm_file(dm_path, desired_tau, 0, t, err);
  if (rc) return rc;
  if (num_grid) *num_grid = t.grid.n;
  if (num_cols) *num_cols = t.ncols;
  if (num_tau) *num_tau = t.num_tau;
  if (tau_pos) *tau_pos = t.tau_pos;
  if (grid_type) *grid_type = t.grid.type;
  if (grid_start) *grid_start = t.grid.start;
  if (grid_end) *grid_end = t.grid.end;
  return PIMC_OK;
}

int pimc_dm_read_tables(const char *dm_path, double desired_tau, double *ukj, double *ukj_d2, double *dukj,
                        double *dukj_d2) {
  if (!dm_path) return PIMC_E_ARG;
  DavidTables t;
  std::string err;
  int rc = read_dm_file(dm_path, desired_tau, 0, t, err);
  if (rc) return rc;
  const size_t bytes = t.uy.size() * sizeof(double);
  if (ukj) std::memcpy(ukj, t.uy.data(), bytes);
  if (ukj_d2) std::memcpy(ukj_d2, t.ud2.data(), bytes);
  if (dukj) std::memcpy(dukj, t.duy.data(), bytes);
  if (dukj_d2) std::memcpy(dukj_d2, t.dud2.data(), bytes);
  return PIMC_OK;
}

int pimc_pa_david(pimc_context *ctx, int sp1, int sp2, int grid_type, double grid_start, double grid_end, int num_grid,
                  int num_cols, int num_tau, const double *ukj, const double *dukj, int tau_pos,
                  int num_offdiag_terms) {
  int rc = check_pair(ctx, sp1, sp2);
  if (rc) return rc;
  if (!ukj || !dukj || num_grid < 2 || num_cols < 2 || num_tau < 1 || tau_pos < 0 || tau_pos >= num_tau ||
      num_offdiag_terms < 0 || (num_offdiag_terms + 1) * (num_offdiag_terms + 2) / 2 > num_cols - 1)
    return fail(ctx, PIMC_E_ARG, "bad DavidPA table arguments");
  if (!(grid_end > grid_start) || (grid_type == PIMC_GRID_LOG && !(grid_start > 0.0)))
    return fail(ctx, PIMC_E_ARG, "bad DavidPA grid");
  CK(cudaSetDevice(ctx->device));
  DavidTables t;
  if (grid_type == PIMC_GRID_LINEAR)
    t.grid.init_linear(grid_start, grid_end, num_grid);
  else if (grid_type == PIMC_GRID_LOG)
    t.grid.init_log(grid_start, std::pow(grid_end / grid_start, 1.0 / (num_grid - 1.0)), num_grid);
  else
    return fail(ctx, PIMC_E_ARG, "bad grid type");
  t.ncols = num_cols;
  t.num_tau = num_tau;
  t.tau_pos = tau_pos;
  t.num_terms = num_offdiag_terms;
  build_david(t, ukj, dukj);
  return set_david(ctx, t);
}

int pimc_pa_tricubic(pimc_context *ctx, int sp1, int sp2, const double qgrid[3], const double ygrid[3],
                     const double tgrid[3], int num_betas, double smallest_beta, const double *umat,
                     const double *dumat, double pot_start, double pot_end, int pot_n, const double *pot_data) {
  int rc = check_pair(ctx, sp1, sp2);
  if (rc) return rc;
  if (!qgrid || !ygrid || !tgrid || !umat || !dumat || !pot_data || num_betas < 1 || pot_n < 3 ||
      !(pot_end > pot_start) || !(smallest_beta > 0.0))
    return fail(ctx, PIMC_E_ARG, "bad tricubic arguments");
  const double *gs[3] = {qgrid, ygrid, tgrid};
  HostGrid hg[3];
  for (int i = 0; i < 3; i++) {
    int n = (int)gs[i][2];
    if (n < 3 || !(gs[i][1] > gs[i][0])) return fail(ctx, PIMC_E_ARG, "bad tricubic grid");
    hg[i].init_linear(gs[i][0], gs[i][1], n);
  }
  CK(cudaSetDevice(ctx->device));
  const size_t nodes = (size_t)hg[0].n * hg[1].n * hg[2].n;
  std::vector<double> F(nodes * 8 * num_betas), dF(nodes * 8 * num_betas);
  for (int b = 0; b < num_betas; b++) {
    tricubic_fill(hg[0], hg[1], hg[2], umat + b * nodes, F.data() + b * nodes * 8);
    tricubic_fill(hg[0], hg[1], hg[2], dumat + b * nodes, dF.data() + b * nodes * 8);
  }
  HostGrid pg;
  pg.init_linear(pot_start, pot_end, pot_n);
  std::vector<double> pd2(pot_n);
  spline_second_derivs(pg, pot_data, 1, 0, 5.0e30, 5.0e30, pd2.data());
  DTricubic<double> &t64 = ctx->pa.t64;
  DTricubic<float> &t32 = ctx->pa.t32;
  t64.nq = t32.nq = hg[0].n;
  t64.ny = t32.ny = hg[1].n;
  t64.nt = t32.nt = hg[2].n;
  t64.num_betas = t32.num_betas = num_betas;
  upload_grid(ctx, hg[0], t64.qg);
  upload_grid(ctx, hg[1], t64.yg);
  upload_grid(ctx, hg[2], t64.tg);
  upload_grid(ctx, hg[0], t32.qg);
  upload_grid(ctx, hg[1], t32.yg);
  upload_grid(ctx, hg[2], t32.tg);
  t64.qmax = hg[0].end;
  t32.qmax = (float)hg[0].end;
  t64.smallest_beta = smallest_beta;
  t32.smallest_beta = (float)smallest_beta;
  if ((rc = upload(ctx, F.data(), F.size(), &t64.U))) return rc;
  if ((rc = upload(ctx, dF.data(), dF.size(), &t64.dU))) return rc;
  {
    std::vector<float> f32(F.begin(), F.end());
    if ((rc = upload(ctx, f32.data(), f32.size(), &t32.U))) return rc;
    std::vector<float> df32(dF.begin(), dF.end());
    if ((rc = upload(ctx, df32.data(), df32.size(), &t32.dU))) return rc;
  }
  {
    // Error bound of the mixed path: per cell (low node ix, iy, iz) the sum
    // over its 8 nodes of |F| + hx|Fx| + hy|Fy| + hz|Fz| + hx hy|Fxy| +
    // hx hz|Fxz| + hy hz|Fyz| + hx hy hz|Fxyz| (component order of the
    // node), rounded up to FP32.
    const int nq = hg[0].n, ny = hg[1].n, nt = hg[2].n;
    const double hx = hg[0].delta, hy = hg[1].delta, hz = hg[2].delta;
    const double hs[8] = {1.0, hx, hy, hz, hx * hy, hx * hz, hy * hz, hx * hy * hz};
    std::vector<float> mb(nodes * num_betas, 0.0f);
    for (int b = 0; b < num_betas; b++)
      for (int ix = 0; ix + 1 < nq; ix++)
        for (int iy = 0; iy + 1 < ny; iy++)
          for (int iz = 0; iz + 1 < nt; iz++) {
            double m = 0.0;
            for (int c = 0; c < 8; c++) {
              const size_t node = ((size_t)(ix + (c >> 2)) * ny + (iy + ((c >> 1) & 1))) * nt + (iz + (c & 1));
              const double *f = F.data() + ((size_t)b * nodes + node) * 8;
              for (int k = 0; k < 8; k++) m += std::fabs(f[k]) * hs[k];
            }
            mb[(size_t)b * nodes + ((size_t)ix * ny + iy) * nt + iz] = (float)(m * (1.0 + 1e-6));
          }
    if ((rc = upload(ctx, mb.data(), mb.size(), &t32.mbound))) return rc;
    t64.mbound = nullptr;
  }
  upload_grid(ctx, pg, t64.pot_grid);
  upload_grid(ctx, pg, t32.pot_grid);
  if ((rc = upload(ctx, pot_data, (size_t)pot_n, &t64.pot_y))) return rc;
  if ((rc = upload(ctx, pd2.data(), pd2.size(), &t64.pot_d2))) return rc;
  {
    std::vector<float> y32(pot_data, pot_data + pot_n), d32(pd2.begin(), pd2.end());
    if ((rc = upload(ctx, y32.data(), y32.size(), &t32.pot_y))) return rc;
    if ((rc = upload(ctx, d32.data(), d32.size(), &t32.pot_d2))) return rc;
  }
  {
    // FP64 (y, d2y) pairs for the device moves' shared-memory copy (the FP64
    // path); the padding row is zero.
    const int np2 = (pot_n + 1) & ~1;
    std::vector<double> p64((size_t)np2 * 2, 0.0);
    for (int i = 0; i < pot_n; i++) {
      p64[2 * i] = pot_data[i];
      p64[2 * i + 1] = pd2[i];
    }
    if ((rc = upload(ctx, p64.data(), p64.size(), &t64.pot_pairs))) return rc;
    t64.pot_pairs_n = np2;
    t32.pot_pairs = nullptr;
    t32.pot_pairs_n = 0;
  }
  ctx->pa.kind = PA_TRICUBIC;
  return PIMC_OK;
}

int pimc_set_path(pimc_context *ctx, int copy, const double *path) {
  if (!ctx || !path || copy < 0 || copy > 2) return fail(ctx, PIMC_E_ARG, "bad set_path arguments");
  CK(cudaSetDevice(ctx->device));
  for (int c = 0; c < 2; c++)
    if (copy == PIMC_BOTH || copy == c)
      CK(cudaMemcpyAsync(ctx->d_path[c], path, ctx->path_elems * sizeof(double), cudaMemcpyHostToDevice,
                         ctx->stream));
  if (copy != PIMC_NEW) {
    ctx->rhok_valid = false;  // the device moves recompute rho_k of the new OLD path
    if (ctx->d_nbr_dirty) CK(cudaMemsetAsync(ctx->d_nbr_dirty, 0xff, sizeof(int), ctx->stream));  // and the lists
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return PIMC_OK;
}

int pimc_get_path(pimc_context *ctx, int copy, double *path) {
  if (!ctx || !path || copy < 0 || copy > 1) return fail(ctx, PIMC_E_ARG, "bad get_path arguments");
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(path, ctx->d_path[copy], ctx->path_elems * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PIMC_OK;
}

static int longrange_single(pimc_context *ctx, int copy, int slice1, int slice2, const ActiveList &act, int level,
                            double *out);
static int yk_single(pimc_context *ctx, int copy, int slice1, int slice2, const ActiveList &act, int level,
                     double *out);
static int yk_sum(pimc_context *ctx, int slice1, int slice2, int table, double *out);

static int check_slices(pimc_context *ctx, int slice1, int slice2, int level, bool inclusive) {
  if (level < 0 || level >= kMaxLevels) return fail(ctx, PIMC_E_ARG, "level out of range");
  if (slice1 < 0 || slice2 < slice1 || slice2 >= ctx->sys.S) return fail(ctx, PIMC_E_ARG, "slice range out of range");
  (void)inclusive;
  return PIMC_OK;
}

int pimc_single_action(pimc_context *ctx, int action, int copy, int slice1, int slice2, const int *active,
                       int n_active, int level, int precision, double *out) {
  if (!ctx || !out) return PIMC_E_ARG;
  if (copy != PIMC_OLD && copy != PIMC_NEW) return fail(ctx, PIMC_E_ARG, "copy must be OLD or NEW");
  if (precision != PIMC_FP64 && precision != PIMC_MIXED) return fail(ctx, PIMC_E_ARG, "bad precision");
  int rc = check_slices(ctx, slice1, slice2, level, action == PIMC_ACTION_LONGRANGE);
  if (rc) return rc;
  ActiveList act;
  if ((rc = check_active(ctx, active, n_active, act))) return rc;
  CK(cudaSetDevice(ctx->device));
  if (action == PIMC_ACTION_LONGRANGE) return longrange_single(ctx, copy, slice1, slice2, act, level, out);
  if (action == PIMC_ACTION_DAVIDLONGRANGE) return yk_single(ctx, copy, slice1, slice2, act, level, out);
  const int skip = 1 << level;
  const int nlinks = (slice2 - slice1 + skip - 1) / skip;
  ReduceTarget t{ctx->stream, ctx->d_partials, ctx->d_counter, ctx->d_out};
  const double *path = ctx->d_path[copy];
  if (nlinks == 0 || n_active == 0) {
    *out = 0.0;
    return PIMC_OK;
  }
  if (slice1 + nlinks * skip > ctx->sys.S - 1 + skip && action != PIMC_ACTION_LONGRANGE)
    return fail(ctx, PIMC_E_ARG, "link runs past the last slice");
  if ((slice1 + (nlinks - 1) * skip + skip) >= ctx->sys.S) return fail(ctx, PIMC_E_ARG, "link runs past the last slice");
  switch (action) {
    case PIMC_ACTION_SHORTRANGE:
      if (ctx->pa.kind == PA_NONE) return fail(ctx, PIMC_E_STATE, "no pair action set");
      if (int rc2 = pa_levels_ok(ctx, level + 1)) return rc2;
      CK(launch_sr_single(t, path, ctx->sys, ctx->pa, act, slice1, skip, nlinks, level, precision, ctx->sm_count));
      break;
    case PIMC_ACTION_KINETIC:
      CK(launch_kin_single(t, path, ctx->sys, act, slice1, skip, nlinks, level, ctx->sm_count));
      break;
    default:
      return fail(ctx, PIMC_E_ARG, "unsupported action");
  }
  return finish_scalar(ctx, out);
}

// LongRangeClass::SingleAction (LongRangeClass.cc:273-371): on the NEW copy
// rho_k is first updated from OLD for the active particles.
static int longrange_single(pimc_context *ctx, int copy, int slice1, int slice2, const ActiveList &act, int level,
                            double *out) {
  if (!ctx->lr_ready) return fail(ctx, PIMC_E_STATE, "pimc_set_longrange not called");
  if (level >= ctx->lr_levels) return fail(ctx, PIMC_E_ARG, "level beyond the long-range tables");
  const int skip = 1 << level;
  if (slice2 > ctx->sys.S - 1) return fail(ctx, PIMC_E_ARG, "slice range out of range");
  const LRDesc lr = lr_desc(ctx);
  if (copy == PIMC_NEW)
    CK(launch_rhok_update(ctx->stream, ctx->d_path[0], ctx->d_path[1], ctx->sys.N, lr, act, slice1, slice2, skip,
                          ctx->d_rhok[0], ctx->d_rhok[1]));
  double ksum = 0.0;
  if (pa_long_range(ctx)) {
    ReduceTarget t{ctx->stream, ctx->d_partials, ctx->d_counter, ctx->d_out};
    CK(launch_lr_sum(t, ctx->d_rhok[copy], lr, ctx->d_ulong_k + (size_t)level * ctx->num_k, slice1, slice2, skip,
                     ctx->sm_count));
    int rc = finish_scalar(ctx, &ksum);
    if (rc) return rc;
  } else {
    CK(cudaStreamSynchronize(ctx->stream));
  }
  *out = ksum + lr_constant(ctx, slice1, slice2, level, false);
  return PIMC_OK;
}

int pimc_d_dbeta(pimc_context *ctx, int action, int slice1, int slice2, int level, double *out) {
  if (!ctx || !out) return PIMC_E_ARG;
  int rc = check_slices(ctx, slice1, slice2, level, false);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  const int skip = 1 << level;
  if (action == PIMC_ACTION_DAVIDLONGRANGE) return yk_sum(ctx, slice1, slice2, 1, out);
  if (action == PIMC_ACTION_LONGRANGE) {
    // LongRangeClass::d_dBeta (LongRangeClass.cc:374-442): rho_k of the OLD
    // copy recomputed (CalcRho_ks_Fast), then the dU tables.
    if (!ctx->lr_ready) return fail(ctx, PIMC_E_STATE, "pimc_set_longrange not called");
    if (level >= ctx->lr_levels) return fail(ctx, PIMC_E_ARG, "level beyond the long-range tables");
    const LRDesc lr = lr_desc(ctx);
    CK(launch_rhok_full(ctx->stream, ctx->d_path[0], ctx->sys.N, ctx->sys.S, lr, ctx->d_rhok[0]));
    double ksum = 0.0;
    if (pa_long_range(ctx)) {
      ReduceTarget t{ctx->stream, ctx->d_partials, ctx->d_counter, ctx->d_out};
      CK(launch_lr_sum(t, ctx->d_rhok[0], lr, ctx->d_dulong_k + (size_t)level * ctx->num_k, slice1, slice2, skip,
                       ctx->sm_count));
      int rc2 = finish_scalar(ctx, &ksum);
      if (rc2) return rc2;
    } else {
      CK(cudaStreamSynchronize(ctx->stream));
    }
    *out = ksum + lr_constant(ctx, slice1, slice2, level, true);
    return PIMC_OK;
  }
  const int nlinks = (slice2 - slice1 + skip - 1) / skip;
  if (nlinks == 0) {
    *out = 0.0;
    return PIMC_OK;
  }
  if ((slice1 + (nlinks - 1) * skip + skip) >= ctx->sys.S) return fail(ctx, PIMC_E_ARG, "link runs past the last slice");
  ReduceTarget t{ctx->stream, ctx->d_partials, ctx->d_counter, ctx->d_out};
  const double *path = ctx->d_path[PIMC_OLD];
  switch (action) {
    case PIMC_ACTION_SHORTRANGE:
      if (ctx->pa.kind == PA_NONE) return fail(ctx, PIMC_E_STATE, "no pair action set");
      if (int rc2 = pa_levels_ok(ctx, level + 1)) return rc2;
      CK(launch_sr_dbeta(t, path, ctx->sys, ctx->pa, slice1, skip, nlinks, level, ctx->sm_count));
      break;
    case PIMC_ACTION_KINETIC:
      CK(launch_kin_dbeta(t, path, ctx->sys, slice1, skip, nlinks, level, ctx->sm_count));
      break;
    default:
      return fail(ctx, PIMC_E_ARG, "unsupported action");
  }
  return finish_scalar(ctx, out);
}

int pimc_accept_copy(pimc_context *ctx, int slice1, int slice2, const int *active, int n_active) {
  if (!ctx) return PIMC_E_ARG;
  int rc = check_slices(ctx, slice1, slice2, 0, true);
  if (rc) return rc;
  ActiveList act;
  if ((rc = check_active(ctx, active, n_active, act))) return rc;
  if (n_active == 0) return PIMC_OK;
  CK(cudaSetDevice(ctx->device));
  CK(launch_accept(ctx->stream, ctx->d_path[0], ctx->d_path[1], ctx->sys, act, slice1, slice2));
  if (ctx->num_k > 0) CK(launch_rhok_copy(ctx->stream, ctx->d_rhok[1], ctx->d_rhok[0], ctx->num_k, slice1, slice2));
  CK(cudaStreamSynchronize(ctx->stream));
  return PIMC_OK;
}

int pimc_reject_copy(pimc_context *ctx, int slice1, int slice2, const int *active, int n_active) {
  if (!ctx) return PIMC_E_ARG;
  int rc = check_slices(ctx, slice1, slice2, 0, true);
  if (rc) return rc;
  ActiveList act;
  if ((rc = check_active(ctx, active, n_active, act))) return rc;
  if (n_active == 0) return PIMC_OK;
  CK(cudaSetDevice(ctx->device));
  CK(launch_reject(ctx->stream, ctx->d_path[0], ctx->d_path[1], ctx->sys, act, slice1, slice2));
  if (ctx->num_k > 0) CK(launch_rhok_copy(ctx->stream, ctx->d_rhok[0], ctx->d_rhok[1], ctx->num_k, slice1, slice2));
  CK(cudaStreamSynchronize(ctx->stream));
  return PIMC_OK;
}

// ---- bisection ----
static int window_slots(const pimc_context *ctx, int num_levels) {
  int w = (ctx->sys.S - 1) >> num_levels;
  return std::max(0, std::min(w, kMaxWindows));
}

int pimc_bisection_setup(pimc_context *ctx, const pimc_bisection_desc *d) {
  if (!ctx || !d) return PIMC_E_ARG;
  if (ctx->pa.kind == PA_NONE) return fail(ctx, PIMC_E_STATE, "no pair action set");
  if (d->num_levels < 1 || d->num_levels > 6) return fail(ctx, PIMC_E_ARG, "NumLevels must be 1..6");
  if ((1 << d->num_levels) >= ctx->sys.S) return fail(ctx, PIMC_E_ARG, "not enough slices for NumLevels");
  if (d->steps_per_block < 1) return fail(ctx, PIMC_E_ARG, "StepsPerBlock must be >= 1");
  if (ctx->sys.N > (1 << 20)) return fail(ctx, PIMC_E_ARG, "device moves support up to 2^20 particles");
  if (d->precision != PIMC_FP64 && d->precision != PIMC_MIXED) return fail(ctx, PIMC_E_ARG, "bad precision");
  if (d->cluster_ctas < 0 || d->cluster_ctas > kMaxCluster) return fail(ctx, PIMC_E_ARG, "cluster_ctas 0..16");
  if (d->threads_per_cta != 0 && (d->threads_per_cta < 64 || d->threads_per_cta > 512 || d->threads_per_cta % 32))
    return fail(ctx, PIMC_E_ARG, "threads_per_cta must be a multiple of 32 in 64..512");
  if (d->schedule != PIMC_SCHEDULE_SEQUENTIAL && d->schedule != PIMC_SCHEDULE_WINDOWS &&
      d->schedule != PIMC_SCHEDULE_PROPOSALS)
    return fail(ctx, PIMC_E_ARG, "bad schedule");
  if (d->schedule != PIMC_SCHEDULE_SEQUENTIAL && window_slots(ctx, d->num_levels) < 1)
    return fail(ctx, PIMC_E_ARG, "no window fits");
  if (d->schedule == PIMC_SCHEDULE_PROPOSALS && d->use_longrange)
    return fail(ctx, PIMC_E_ARG, "concurrent proposals are short-range only (every move changes the window's rho_k)");
  if (d->schedule == PIMC_SCHEDULE_PROPOSALS && ctx->pa.kind != PA_DAVID)
    return fail(ctx, PIMC_E_ARG, "concurrent proposals need a DavidPA table");
  if (d->use_longrange) {
    // LongRange joins the lowest stage (BisectionBlock.cc:92-103); its short-range
    // counterpart must subtract the same Ulong
    if (!ctx->lr_ready || ctx->num_k <= 0) return fail(ctx, PIMC_E_STATE, "long range needs k-vectors and tables");
    if (!(ctx->pa.kind == PA_COULOMB && ctx->pa.c64.long_range))
      return fail(ctx, PIMC_E_ARG, "long range in device moves needs the Coulomb action's breakup (pimc_longrange_coulomb)");
  }
  if (int rc2 = pa_levels_ok(ctx, d->num_levels)) return rc2;
  if (d->neighbor_skin < 0.0 || d->neighbor_max < 0) return fail(ctx, PIMC_E_ARG, "bad neighbour-list settings");
  if (d->mixed_guard < 0 || d->mixed_guard > 2 || d->wait_cap < 0 || d->test_wait < 0)
    return fail(ctx, PIMC_E_ARG, "bad guard / wait settings");
  if (d->neighbor_skin > 0.0) {
    if (ctx->pa.kind != PA_DAVID) return fail(ctx, PIMC_E_ARG, "neighbour lists need a DavidPA table");
    if (ctx->sys.N > 65536) return fail(ctx, PIMC_E_ARG, "neighbour lists support up to 65536 particles");
    CK(cudaSetDevice(ctx->device));
    const int kmax = d->neighbor_max ? std::min(d->neighbor_max, ctx->sys.N) : std::min(1024, ctx->sys.N);
    cudaFree(ctx->d_nbr_cb);
    cudaFree(ctx->d_nbr_cnt);
    cudaFree(ctx->d_nbr_idx);
    cudaFree(ctx->d_nbr_dirty);
    ctx->d_nbr_cb = nullptr;
    ctx->d_nbr_cnt = ctx->d_nbr_idx = ctx->d_nbr_dirty = nullptr;
    CK(cudaMalloc(&ctx->d_nbr_cb, (size_t)ctx->sys.N * sizeof(double4)));
    CK(cudaMalloc(&ctx->d_nbr_cnt, (size_t)ctx->sys.N * sizeof(int)));
    CK(cudaMalloc(&ctx->d_nbr_idx, (size_t)ctx->sys.N * kmax * sizeof(int)));
    CK(cudaMalloc(&ctx->d_nbr_dirty, sizeof(int)));
    CK(cudaMemset(ctx->d_nbr_dirty, 0xff, sizeof(int)));
    ctx->nbr_kmax = kmax;
    ctx->nbr_range = ctx->pa.d64.grid.end;  // the table is zero from its last point on
  }
  CK(cudaSetDevice(ctx->device));
  ctx->bis = *d;
  if (ctx->bis.cluster_ctas == 0)
    ctx->bis.cluster_ctas = (ctx->sys.N >= 256 || d->schedule == PIMC_SCHEDULE_PROPOSALS) ? 8 : 1;
  if (ctx->bis.threads_per_cta == 0) ctx->bis.threads_per_cta = 256;
  std::vector<ChainState> cs(kMaxChainStates);
  CK(cudaMemcpy(cs.data(), ctx->d_chain, cs.size() * sizeof(ChainState), cudaMemcpyDeviceToHost));
  for (auto &c : cs) {
    c.moves = c.accepted = c.stages = c.pair_evals = c.flips = c.redone = c.reevals = 0;
    c.status = 0;
  }
  CK(cudaMemcpy(ctx->d_chain, cs.data(), cs.size() * sizeof(ChainState), cudaMemcpyHostToDevice));
  ctx->bis_ready = true;
  return PIMC_OK;
}

int pimc_rng_seed(pimc_context *ctx, uint64_t seed) {
  if (!ctx) return PIMC_E_ARG;
  CK(cudaSetDevice(ctx->device));
  std::vector<ChainState> cs(kMaxChainStates);
  CK(cudaMemcpy(cs.data(), ctx->d_chain, cs.size() * sizeof(ChainState), cudaMemcpyDeviceToHost));
  for (int w = 0; w < kMaxChainStates; w++) {
    cs[w].seed = seed;
    cs[w].nlocal = 0;
    cs[w].stream = w == 0 && ctx->bis.schedule == PIMC_SCHEDULE_SEQUENTIAL ? kStreamLocal : kStreamWindow0 + w;
    cs[w].one_left = 0;
    cs[w].x2 = 0.0;
  }
  // stream ids are fixed by the schedule at seeding time; window 0 of the
  // concurrent schedule uses kStreamWindow0, the sequential chain kStreamLocal
  cs[0].stream = ctx->bis.schedule == PIMC_SCHEDULE_SEQUENTIAL ? kStreamLocal : kStreamWindow0;
  ctx->rounds = 0;
  ctx->seed = seed;
  ctx->shift_draws = 0;
  CK(cudaMemcpy(ctx->d_chain, cs.data(), cs.size() * sizeof(ChainState), cudaMemcpyHostToDevice));
  return PIMC_OK;
}

int pimc_bisection_windows(pimc_context *ctx, int *windows) {
  if (!ctx || !windows) return PIMC_E_ARG;
  if (!ctx->bis_ready) return fail(ctx, PIMC_E_STATE, "pimc_bisection_setup not called");
  *windows = ctx->bis.schedule != PIMC_SCHEDULE_SEQUENTIAL ? window_slots(ctx, ctx->bis.num_levels) : 1;
  return PIMC_OK;
}

static size_t records_for(const pimc_context *ctx, int n_blocks) {
  size_t per = ctx->bis.schedule != PIMC_SCHEDULE_SEQUENTIAL ? (size_t)window_slots(ctx, ctx->bis.num_levels) : 1;
  if (ctx->bis.schedule == PIMC_SCHEDULE_PROPOSALS) per *= (size_t)ctx->bis.cluster_ctas;
  return (size_t)n_blocks * per * ctx->bis.steps_per_block;
}

static int run_bisection(pimc_context *ctx, int n_blocks, pimc_move_record *device_trace) {
  BisectionArgs a;
  a.path = ctx->d_path[PIMC_OLD];
  a.sys = ctx->sys;
  a.pa = ctx->pa;
  a.chains = ctx->d_chain;
  a.trace = device_trace;
  a.trace_offset = 0;
  a.num_levels = ctx->bis.num_levels;
  a.steps_per_block = ctx->bis.steps_per_block;
  a.n_blocks = n_blocks;
  a.sr_higher = ctx->bis.shortrange_at_higher_levels;
  a.concurrent = ctx->bis.schedule != PIMC_SCHEDULE_SEQUENTIAL;
  a.proposals = ctx->bis.schedule == PIMC_SCHEDULE_PROPOSALS ? ctx->bis.cluster_ctas : 1;
  a.pair_range = ctx->pa.kind == PA_DAVID ? ctx->pa.d64.grid.end : 0.0;
  a.round = ctx->rounds;
  a.use_lr = ctx->bis.use_longrange ? 1 : 0;
  a.rhok = ctx->d_rhok[0];
  a.kvec = ctx->d_kvec;
  a.ulong_k0 = ctx->d_ulong_k;  // level 0 row
  a.nk = ctx->num_k;
  a.nbr_on = ctx->bis.neighbor_skin > 0.0 ? 1 : 0;
  a.nbr_kmax = ctx->nbr_kmax;
  a.nbr_cb = ctx->d_nbr_cb;
  a.nbr_cnt = ctx->d_nbr_cnt;
  a.nbr_idx = ctx->d_nbr_idx;
  a.nbr_dirty = ctx->d_nbr_dirty;
  a.guard = guard_mode(ctx->bis.mixed_guard);
  a.wait_cap = ctx->bis.wait_cap;
  a.test_wait = ctx->bis.test_wait;
  if (a.use_lr && !ctx->rhok_valid) {  // PathClass::UpdateRho_ks() of the current OLD path
    CK(launch_rhok_full(ctx->stream, ctx->d_path[0], ctx->sys.N, ctx->sys.S, lr_desc(ctx), ctx->d_rhok[0]));
    ctx->rhok_valid = true;
  }
  const int cl = ctx->bis.cluster_ctas, thr = ctx->bis.threads_per_cta;
  auto rebuild = [&]() {  // no-op unless a move or set_path marked the lists stale
    return a.nbr_on ? launch_nbr_rebuild(ctx->stream, ctx->d_path[0], ctx->sys, ctx->nbr_range,
                                         ctx->bis.neighbor_skin, ctx->nbr_kmax, ctx->d_nbr_cb, ctx->d_nbr_cnt,
                                         ctx->d_nbr_idx, ctx->d_nbr_dirty)
                    : cudaSuccess;
  };
  if (!a.concurrent) {
    CK(rebuild());
    CK(launch_bisection(a, ctx->bis.precision, ctx->bis.shadow, cl, 1, thr, ctx->stream));
    return PIMC_OK;
  }
  const int W = window_slots(ctx, ctx->bis.num_levels);
  for (int r = 0; r < n_blocks; r++) {
    a.round = ctx->rounds + r;
    a.trace_offset = (long long)r * W * ctx->bis.steps_per_block * a.proposals;
    CK(rebuild());
    CK(launch_bisection(a, ctx->bis.precision, ctx->bis.shadow, cl, W, thr, ctx->stream));
  }
  ctx->rounds += n_blocks;
  return PIMC_OK;
}

int pimc_run_bisection_async(pimc_context *ctx, int n_blocks) {
  if (!ctx || n_blocks < 0) return PIMC_E_ARG;
  if (!ctx->bis_ready) return fail(ctx, PIMC_E_STATE, "pimc_bisection_setup not called");
  CK(cudaSetDevice(ctx->device));
  return run_bisection(ctx, n_blocks, nullptr);
}

int pimc_run_bisection(pimc_context *ctx, int n_blocks, pimc_move_record *trace, pimc_bisection_stats *stats) {
  if (!ctx || n_blocks < 0) return PIMC_E_ARG;
  if (!ctx->bis_ready) return fail(ctx, PIMC_E_STATE, "pimc_bisection_setup not called");
  CK(cudaSetDevice(ctx->device));
  const size_t nrec = records_for(ctx, n_blocks);
  if (trace && nrec > ctx->trace_cap) {
    cudaFree(ctx->d_trace);
    ctx->d_trace = nullptr;
    ctx->trace_cap = 0;
    CK(cudaMalloc(&ctx->d_trace, nrec * sizeof(pimc_move_record)));
    ctx->trace_cap = nrec;
  }
  int rc = run_bisection(ctx, n_blocks, trace ? ctx->d_trace : nullptr);
  if (rc) return rc;
  // The device moves advance OLD only; bring NEW back in sync (MirroredClass invariant).
  CK(cudaMemcpyAsync(ctx->d_path[1], ctx->d_path[0], ctx->path_elems * sizeof(double), cudaMemcpyDeviceToDevice,
                     ctx->stream));
  if (ctx->bis.use_longrange)
    CK(cudaMemcpyAsync(ctx->d_rhok[1], ctx->d_rhok[0], (size_t)ctx->sys.S * ctx->num_k * sizeof(double2),
                       cudaMemcpyDeviceToDevice, ctx->stream));
  if (trace && nrec)
    CK(cudaMemcpyAsync(trace, ctx->d_trace, nrec * sizeof(pimc_move_record), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  pimc_bisection_stats st;
  rc = pimc_bisection_get_stats(ctx, &st);
  if (rc) return rc;
  if (stats) *stats = st;
  if (st.status) {
    // The status belongs to this call: clear it so that the next call on the
    // context starts clean (the chains' counters and streams are kept).
    std::vector<ChainState> cs(kMaxChainStates);
    CK(cudaMemcpy(cs.data(), ctx->d_chain, cs.size() * sizeof(ChainState), cudaMemcpyDeviceToHost));
    for (auto &c : cs) c.status = 0;
    CK(cudaMemcpy(ctx->d_chain, cs.data(), cs.size() * sizeof(ChainState), cudaMemcpyHostToDevice));
    return fail(ctx, st.status, std::string("device status: ") + pimc_status_string(st.status));
  }
  return PIMC_OK;
}

int pimc_bisection_get_stats(pimc_context *ctx, pimc_bisection_stats *stats) {
  if (!ctx || !stats) return PIMC_E_ARG;
  CK(cudaSetDevice(ctx->device));
  std::vector<ChainState> cs(kMaxChainStates);
  CK(cudaMemcpyAsync(cs.data(), ctx->d_chain, cs.size() * sizeof(ChainState), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  std::memset(stats, 0, sizeof(*stats));
  for (const auto &c : cs) {
    stats->moves += (int64_t)c.moves;
    stats->accepted += (int64_t)c.accepted;
    stats->stages_attempted += (int64_t)c.stages;
    stats->pair_evals += (int64_t)c.pair_evals;
    stats->flips += (int64_t)c.flips;
    stats->redone += (int64_t)c.redone;
    stats->reevaluated += (int64_t)c.reevals;
    if (c.status && !stats->status) stats->status = c.status;
  }
  return PIMC_OK;
}

int pimc_bisection_occupancy(pimc_context *ctx, int *max_active_clusters) {
  if (!ctx || !max_active_clusters) return PIMC_E_ARG;
  if (!ctx->bis_ready) return fail(ctx, PIMC_E_STATE, "pimc_bisection_setup not called");
  CK(cudaSetDevice(ctx->device));
  BisectionArgs a{};
  a.pa = ctx->pa;
  a.num_levels = ctx->bis.num_levels;
  a.proposals = ctx->bis.schedule == PIMC_SCHEDULE_PROPOSALS ? ctx->bis.cluster_ctas : 1;
  CK(bisection_occupancy(a, ctx->bis.precision, ctx->bis.shadow, ctx->bis.cluster_ctas, ctx->bis.threads_per_cta,
                         max_active_clusters));
  return PIMC_OK;
}

int pimc_synchronize(pimc_context *ctx) {
  if (!ctx) return PIMC_E_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  return PIMC_OK;
}

void *pimc_stream(pimc_context *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

// PathClass::SetupkVecs3D (PathClass.cc:534-586), one species.
int pimc_setup_kvecs(pimc_context *ctx, double kcutoff, int *num_k) {
  if (!ctx || !num_k || !(kcutoff > 0.0)) return fail(ctx, PIMC_E_ARG, "bad kcutoff");
  CK(cudaSetDevice(ctx->device));
  for (int i = 0; i < 3; i++) ctx->kbox[i] = 2.0 * M_PI / ctx->sys.box[i];
  for (int i = 0; i < 3; i++) ctx->kmax[i] = (int)std::ceil(1.1 * kcutoff / ctx->kbox[i]);
  for (int i = 0; i < 3; i++)
    if (ctx->kmax[i] > 64) return fail(ctx, PIMC_E_ARG, "kCutoff too large (more than 64 k-points per dimension)");
  std::vector<int3> kidx;
  ctx->kvecs.clear();
  for (int ix = -ctx->kmax[0]; ix <= ctx->kmax[0]; ix++) {
    const double k0 = ix * ctx->kbox[0];
    for (int iy = -ctx->kmax[1]; iy <= ctx->kmax[1]; iy++) {
      const double k1 = iy * ctx->kbox[1];
      for (int iz = -ctx->kmax[2]; iz <= ctx->kmax[2]; iz++) {
        const double k2 = iz * ctx->kbox[2];
        // the half-space of PathClass Include() (PathClass.cc:281-292)
        const bool include = (k0 > 0.0) || (k0 == 0.0 && k1 > 0.0) || (k0 == 0.0 && k1 == 0.0 && k2 > 0.0);
        if ((k0 * k0 + k1 * k1 + k2 * k2 < kcutoff * kcutoff) && include) {
          ctx->kvecs.push_back(k0);
          ctx->kvecs.push_back(k1);
          ctx->kvecs.push_back(k2);
          kidx.push_back(make_int3(ix + ctx->kmax[0], iy + ctx->kmax[1], iz + ctx->kmax[2]));
        }
      }
    }
  }
  if (kidx.size() > 1024) return fail(ctx, PIMC_E_ARG, "more than 1024 k-vectors");
  ctx->num_k = (int)kidx.size();
  ctx->kcutoff = kcutoff;
  ctx->rhok_valid = false;
  ctx->yk_ready = false;  // tables are per k-vector
  cudaFree(ctx->d_kvec);
  ctx->d_kvec = nullptr;
  CK(cudaMalloc(&ctx->d_kvec, ctx->kvecs.size() * sizeof(double) + 16));
  CK(cudaMemcpy(ctx->d_kvec, ctx->kvecs.data(), ctx->kvecs.size() * sizeof(double), cudaMemcpyHostToDevice));
  cudaFree(ctx->d_kidx);
  cudaFree(ctx->d_rhok[0]);
  cudaFree(ctx->d_rhok[1]);
  ctx->d_kidx = nullptr;
  ctx->d_rhok[0] = ctx->d_rhok[1] = nullptr;
  if (ctx->num_k > 0) {
    CK(cudaMalloc(&ctx->d_kidx, kidx.size() * sizeof(int3)));
    CK(cudaMemcpy(ctx->d_kidx, kidx.data(), kidx.size() * sizeof(int3), cudaMemcpyHostToDevice));
    for (int c = 0; c < 2; c++) {
      CK(cudaMalloc(&ctx->d_rhok[c], (size_t)ctx->sys.S * ctx->num_k * sizeof(double2)));
      CK(cudaMemset(ctx->d_rhok[c], 0, (size_t)ctx->sys.S * ctx->num_k * sizeof(double2)));
    }
  }
  *num_k = ctx->num_k;
  return PIMC_OK;
}

int pimc_get_kvecs(pimc_context *ctx, double *kvecs) {
  if (!ctx || !kvecs) return PIMC_E_ARG;
  std::memcpy(kvecs, ctx->kvecs.data(), ctx->kvecs.size() * sizeof(double));
  return PIMC_OK;
}

int pimc_set_longrange(pimc_context *ctx, int num_levels, const double *ulong_k, const double *ulong_r0,
                       const double *ushort_k0, const double *ulong_k0, const double *dulong_k,
                       const double *dulong_r0, const double *dushort_k0, const double *dulong_k0,
                       int use_background) {
  if (!ctx) return PIMC_E_ARG;
  if (ctx->num_k <= 0) return fail(ctx, PIMC_E_STATE, "pimc_setup_kvecs not called");
  if (num_levels < 1 || !ulong_k || !ulong_r0 || !ushort_k0 || !ulong_k0 || !dulong_k || !dulong_r0 ||
      !dushort_k0 || !dulong_k0)
    return fail(ctx, PIMC_E_ARG, "bad long-range tables");
  CK(cudaSetDevice(ctx->device));
  const size_t n = (size_t)num_levels * ctx->num_k;
  cudaFree(ctx->d_ulong_k);
  cudaFree(ctx->d_dulong_k);
  ctx->d_ulong_k = ctx->d_dulong_k = nullptr;
  CK(cudaMalloc(&ctx->d_ulong_k, n * sizeof(double)));
  CK(cudaMalloc(&ctx->d_dulong_k, n * sizeof(double)));
  CK(cudaMemcpy(ctx->d_ulong_k, ulong_k, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_dulong_k, dulong_k, n * sizeof(double), cudaMemcpyHostToDevice));
  ctx->ulong_r0.assign(ulong_r0, ulong_r0 + num_levels);
  ctx->ushort_k0.assign(ushort_k0, ushort_k0 + num_levels);
  ctx->ulong_k0.assign(ulong_k0, ulong_k0 + num_levels);
  ctx->dulong_r0.assign(dulong_r0, dulong_r0 + num_levels);
  ctx->dushort_k0.assign(dushort_k0, dushort_k0 + num_levels);
  ctx->dulong_k0.assign(dulong_k0, dulong_k0 + num_levels);
  ctx->lr_levels = num_levels;
  ctx->use_background = use_background;
  ctx->lr_ready = true;
  return PIMC_OK;
}

// ---- DavidLongRangeClassYk (PIMC++/src/Actions/DavidLongRangeClassYk.cc) ----
// BuildRPA_SingleType (:76-126) for one pair type (rpa), else
// Build_MultipleSpecies (:38-74): per k-vector the entry of the squarer's
// k-space table whose k equals its |k| within 1e-10 (:57, :111).
int pimc_davidlongrange_yk(pimc_context *ctx, int num_kvals, const double *kvals, const double *uk_long, int rpa) {
  if (!ctx) return PIMC_E_ARG;
  if (num_kvals < 1 || !kvals || !uk_long) return fail(ctx, PIMC_E_ARG, "bad k-space table");
  if (ctx->num_k <= 0) return fail(ctx, PIMC_E_STATE, "pimc_setup_kvecs not called");
  const int K = ctx->num_k;
  const double vol = ctx->sys.box[0] * ctx->sys.box[1] * ctx->sys.box[2];
  const double ncomps = ctx->sys.N, lambda = ctx->sys.lambda, tau = ctx->sys.tau;
  if (rpa && !(lambda > 0.0)) return fail(ctx, PIMC_E_ARG, "the RPA construction needs lambda > 0");
  std::vector<double> t(3 * (size_t)K, 0.0);
  std::vector<char> set(K, 0);
  for (int i = 0; i < num_kvals; i++) {
    const double k = kvals[i];
    const double v = uk_long[i] / vol;
    double u, du;
    if (rpa) {
      if (std::fabs(k) < 1e-10) continue;  // yk_zero: not used by the action
      const double arg = 1.0 + ncomps * 2.0 * uk_long[i] / (lambda * k * k * vol);
      const double theta = 0.5 * k * k * lambda * tau;
      double sv;
      if (arg < 0) {
        const double q = std::sqrt(-arg), tn = std::tan(q * theta);
        sv = q * (1 - q * tn) / (q + tn);
      } else if (arg == 0) {
        sv = 1.0 / (1.0 + theta);
      } else {
        const double q = std::sqrt(arg), tn = std::tanh(theta * q);
        sv = q * (1.0 + q * tn) / (q + tn);
      }
      u = (-1.0 + sv) / ncomps;
      du = uk_long[i] / vol - lambda * k * k * u * (1.0 + 0.5 * ncomps * u);
    } else {
      u = v * tau;
      du = v;
    }
    for (int j = 0; j < K; j++) {
      const double *kv = &ctx->kvecs[(size_t)j * 3];
      if (std::fabs(std::sqrt(kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2]) - k) < 1e-10) {
        t[j] = u;
        t[K + j] = du;
        t[2 * (size_t)K + j] = v;
        set[j] = 1;
      }
    }
  }
  for (int j = 0; j < K; j++)
    if (!set[j]) return fail(ctx, PIMC_E_ARG, "a k-vector's |k| is not in the k-space table");
  CK(cudaSetDevice(ctx->device));
  cudaFree(ctx->d_yk);
  ctx->d_yk = nullptr;
  ctx->yk_ready = false;
  CK(cudaMalloc(&ctx->d_yk, t.size() * sizeof(double)));
  CK(cudaMemcpy(ctx->d_yk, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice));
  ctx->yk_ready = true;
  return PIMC_OK;
}

// DavidLongRangeClassYk::SingleAction (:230-323).  Away from the whole path
// only the window's interior counts: on NEW, rho_k is updated over
// [slice1 + skip, slice2 - skip] ([slice1, slice2 - skip] for the whole
// path), and sum_k sum_slices |rho_k|^2 uk runs over the same slices with
// weight 1.  No active particle: no species in the sum, 0.
static int yk_single(pimc_context *ctx, int copy, int slice1, int slice2, const ActiveList &act, int level,
                     double *out) {
  if (!ctx->yk_ready) return fail(ctx, PIMC_E_STATE, "pimc_davidlongrange_yk not called");
  const int skip = 1 << level;
  const bool inclusive = !(slice1 == 0 && slice2 == ctx->sys.S - 1);
  const int first = inclusive ? slice1 + skip : slice1, last = slice2 - skip;
  const LRDesc lr = lr_desc(ctx);
  if (copy == PIMC_NEW && first <= last)
    CK(launch_rhok_update(ctx->stream, ctx->d_path[0], ctx->d_path[1], ctx->sys.N, lr, act, first, last, skip,
                          ctx->d_rhok[0], ctx->d_rhok[1]));
  if (act.n == 0 || first > last) {
    CK(cudaStreamSynchronize(ctx->stream));
    *out = 0.0;
    return PIMC_OK;
  }
  ReduceTarget t{ctx->stream, ctx->d_partials, ctx->d_counter, ctx->d_out};
  CK(launch_lr_sum(t, ctx->d_rhok[copy], lr, ctx->d_yk, first, last, skip, ctx->sm_count, 1.0));
  return finish_scalar(ctx, out);
}

// DavidLongRangeClassYk::d_dBeta (:327-363, table 1: duk) and V (:367-389,
// table 2: Vlong_k): rho_k of the OLD copy recomputed, every slice of
// [slice1, slice2] (the level is not used), weight 1/2 at both ends.
static int yk_sum(pimc_context *ctx, int slice1, int slice2, int table, double *out) {
  if (!ctx->yk_ready) return fail(ctx, PIMC_E_STATE, "pimc_davidlongrange_yk not called");
  const LRDesc lr = lr_desc(ctx);
  CK(launch_rhok_full(ctx->stream, ctx->d_path[0], ctx->sys.N, ctx->sys.S, lr, ctx->d_rhok[0]));
  ReduceTarget t{ctx->stream, ctx->d_partials, ctx->d_counter, ctx->d_out};
  CK(launch_lr_sum(t, ctx->d_rhok[0], lr, ctx->d_yk + (size_t)table * ctx->num_k, slice1, slice2, 1, ctx->sm_count,
                   0.5));
  return finish_scalar(ctx, out);
}

int pimc_davidlongrange_v(pimc_context *ctx, int slice1, int slice2, double *out) {
  if (!ctx || !out) return PIMC_E_ARG;
  if (int rc = check_slices(ctx, slice1, slice2, 0, true)) return rc;
  CK(cudaSetDevice(ctx->device));
  return yk_sum(ctx, slice1, slice2, 2, out);
}

// PathClass::UpdateRho_ks() full recompute (PathClass.cc:710-718): OLD, then NEW = OLD.
int pimc_calc_rhok(pimc_context *ctx) {
  if (!ctx) return PIMC_E_ARG;
  if (ctx->num_k <= 0) return fail(ctx, PIMC_E_STATE, "pimc_setup_kvecs not called");
  CK(cudaSetDevice(ctx->device));
  CK(launch_rhok_full(ctx->stream, ctx->d_path[0], ctx->sys.N, ctx->sys.S, lr_desc(ctx), ctx->d_rhok[0]));
  CK(cudaMemcpyAsync(ctx->d_rhok[1], ctx->d_rhok[0], (size_t)ctx->sys.S * ctx->num_k * sizeof(double2),
                     cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->rhok_valid = true;
  return PIMC_OK;
}

int pimc_update_rhok(pimc_context *ctx, int slice1, int slice2, const int *active, int n_active, int level) {
  if (!ctx) return PIMC_E_ARG;
  if (ctx->num_k <= 0) return fail(ctx, PIMC_E_STATE, "pimc_setup_kvecs not called");
  int rc = check_slices(ctx, slice1, slice2, level, true);
  if (rc) return rc;
  ActiveList act;
  if ((rc = check_active(ctx, active, n_active, act))) return rc;
  CK(cudaSetDevice(ctx->device));
  CK(launch_rhok_update(ctx->stream, ctx->d_path[0], ctx->d_path[1], ctx->sys.N, lr_desc(ctx), act, slice1, slice2,
                        1 << level, ctx->d_rhok[0], ctx->d_rhok[1]));
  CK(cudaStreamSynchronize(ctx->stream));
  return PIMC_OK;
}

int pimc_get_rhok(pimc_context *ctx, int copy, double *out) {
  if (!ctx || !out || copy < 0 || copy > 1) return PIMC_E_ARG;
  if (ctx->num_k <= 0) return fail(ctx, PIMC_E_STATE, "pimc_setup_kvecs not called");
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpy(out, ctx->d_rhok[copy], (size_t)ctx->sys.S * ctx->num_k * sizeof(double2), cudaMemcpyDeviceToHost));
  return PIMC_OK;
}

// ---- observables ----

int pimc_energy(pimc_context *ctx, pimc_energy_terms *out) {
  if (!ctx || !out) return PIMC_E_ARG;
  if (ctx->pa.kind == PA_NONE) return fail(ctx, PIMC_E_STATE, "no pair action set");
  CK(cudaSetDevice(ctx->device));
  const int M = ctx->sys.S - 1;
  pimc_energy_terms e = {};
  // ActionsClass::Energy (ActionsClass.cc:812-871) on the OLD path
  int rc = pimc_d_dbeta(ctx, PIMC_ACTION_KINETIC, 0, M, 0, &e.kinetic);
  if (!rc) rc = pimc_d_dbeta(ctx, PIMC_ACTION_SHORTRANGE, 0, M, 0, &e.du_short);
  if (!rc && ctx->lr_ready) rc = pimc_d_dbeta(ctx, PIMC_ACTION_LONGRANGE, 0, M, 0, &e.du_long);
  if (rc) return rc;
  ReduceTarget t{ctx->stream, ctx->d_partials, ctx->d_counter, ctx->d_out};
  CK(launch_pair_obs(t, ctx->d_path[PIMC_OLD], ctx->sys, ctx->pa, true, nullptr, nullptr, ctx->sm_count));
  rc = finish_scalar(ctx, &e.v_short);
  if (rc) return rc;
  e.v_long = 0.0;
  // EnergyClass::Accumulate's sample (ObservableEnergy.cc:45-73): per slice
  e.total = (e.kinetic + e.du_short + e.du_long) / (double)M;
  *out = e;
  return PIMC_OK;
}

int pimc_gofr_setup(pimc_context *ctx, double start, double end, int num_points) {
  if (!ctx) return PIMC_E_ARG;
  if (end <= 0.0) end = ctx->sys.box[0];  // the reference's default grid end (ObservableCorrelation.cc:52-57)
  if (num_points < 2 || num_points - 1 > 12288 || !(start >= 0.0) || !(end > start))
    return fail(ctx, PIMC_E_ARG, "g(r) grid: 0 <= start < end and 2 <= NumPoints <= 12289");
  CK(cudaSetDevice(ctx->device));
  cudaFree(ctx->d_gofr);
  ctx->d_gofr = nullptr;
  CK(cudaMalloc(&ctx->d_gofr, (size_t)(num_points - 1) * sizeof(unsigned long long)));
  CK(cudaMemsetAsync(ctx->d_gofr, 0, (size_t)(num_points - 1) * sizeof(unsigned long long), ctx->stream));
  ctx->gofr_points = num_points;
  ctx->gofr_start = start;
  ctx->gofr_end = end;
  // LinearGrid::Init (Grid.h:87-95)
  ctx->gofr_delta = (end - start) / (double)(num_points - 1);
  ctx->gofr_deltainv = 1.0 / ctx->gofr_delta;
  ctx->gofr_counts = 0;
  return PIMC_OK;
}

int pimc_gofr_accumulate(pimc_context *ctx) {
  if (!ctx) return PIMC_E_ARG;
  if (!ctx->d_gofr) return fail(ctx, PIMC_E_STATE, "pimc_gofr_setup not called");
  CK(cudaSetDevice(ctx->device));
  GofrGrid g{ctx->gofr_start, ctx->gofr_end, ctx->gofr_deltainv, ctx->gofr_points - 1};
  ReduceTarget t{ctx->stream, ctx->d_partials, ctx->d_counter, ctx->d_out};
  CK(launch_pair_obs(t, ctx->d_path[PIMC_OLD], ctx->sys, ctx->pa, false, &g, ctx->d_gofr, ctx->sm_count));
  ctx->gofr_counts++;
  return PIMC_OK;
}

int pimc_gofr_get(pimc_context *ctx, uint64_t *histogram, double *gofr, long long *total_counts) {
  if (!ctx) return PIMC_E_ARG;
  if (!ctx->d_gofr) return fail(ctx, PIMC_E_STATE, "pimc_gofr_setup not called");
  CK(cudaSetDevice(ctx->device));
  const int nb = ctx->gofr_points - 1;
  std::vector<unsigned long long> h(nb);
  CK(cudaMemcpyAsync(h.data(), ctx->d_gofr, nb * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (histogram)
    for (int i = 0; i < nb; i++) histogram[i] = h[i];
  if (total_counts) *total_counts = ctx->gofr_counts;
  if (gofr) {
    // PairCorrelationClass::WriteBlock (ObservableCorrelation.cc:101-135), one species
    const double N = ctx->sys.N, M = ctx->sys.S - 1;
    const double vol = ctx->sys.box[0] * ctx->sys.box[1] * ctx->sys.box[2];
    const double norm = 0.5 * (double)ctx->gofr_counts * M * (N * (N - 1.0)) / vol;
    for (int i = 0; i < nb; i++) {
      const double r1 = ctx->gofr_start + (double)i * ctx->gofr_delta;
      const double r2 = ctx->gofr_start + (double)(i + 1) * ctx->gofr_delta;
      const double binVol = 4.0 * M_PI / 3 * (r2 * r2 * r2 - r1 * r1 * r1);
      gofr[i] = norm > 0.0 ? (double)h[i] / (binVol * norm) : 0.0;
    }
  }
  return PIMC_OK;
}

int pimc_gofr_reset(pimc_context *ctx) {
  if (!ctx) return PIMC_E_ARG;
  if (!ctx->d_gofr) return fail(ctx, PIMC_E_STATE, "pimc_gofr_setup not called");
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemsetAsync(ctx->d_gofr, 0, (size_t)(ctx->gofr_points - 1) * sizeof(unsigned long long), ctx->stream));
  ctx->gofr_counts = 0;
  return PIMC_OK;
}

// ---- classical Coulomb pair action and its optimized breakup ----

int pimc_pa_coulomb(pimc_context *ctx, int sp1, int sp2, double z1z2, int num_levels) {
  if (!ctx) return PIMC_E_ARG;
  if (sp1 != 0 || sp2 != 0) return fail(ctx, PIMC_E_ARG, "one species pair (0, 0) is supported");
  if (num_levels < 1 || num_levels > 16) return fail(ctx, PIMC_E_ARG, "num_levels must be in 1..16");
  DCoulomb<double> c64{};
  DCoulomb<float> c32{};
  c64.z1z2 = z1z2;
  c64.smallest_beta = ctx->sys.tau;
  c64.num_levels = num_levels;
  c64.long_range = 0;
  c64.np = kLongGridPoints;
  c32.z1z2 = (float)z1z2;
  c32.smallest_beta = (float)ctx->sys.tau;
  c32.num_levels = num_levels;
  c32.long_range = 0;
  c32.np = kLongGridPoints;
  ctx->pa = DevPA{};
  ctx->pa.kind = PA_COULOMB;
  ctx->pa.c64 = c64;
  ctx->pa.c32 = c32;
  return PIMC_OK;
}

int pimc_longrange_coulomb(pimc_context *ctx, int num_knots, int use_background) {
  if (!ctx) return PIMC_E_ARG;
  if (ctx->pa.kind != PA_COULOMB) return fail(ctx, PIMC_E_STATE, "pimc_pa_coulomb not called");
  if (ctx->num_k <= 0) return fail(ctx, PIMC_E_STATE, "pimc_setup_kvecs not called");
  if (num_knots < 2 || num_knots > 1000) return fail(ctx, PIMC_E_ARG, "num_knots must be in 2..1000");
  CK(cudaSetDevice(ctx->device));
  DCoulomb<double> &c64 = ctx->pa.c64;
  DCoulomb<float> &c32 = ctx->pa.c32;
  BreakupTables bt;
  int rc = coulomb_breakup(ctx->sys.box, c64.z1z2, c64.smallest_beta, c64.num_levels, num_knots, ctx->kcutoff,
                           ctx->num_k, ctx->kvecs.data(), bt);
  if (rc) return fail(ctx, rc, "breakup failed");
  const double h = bt.rmax / (kLongGridPoints - 1);
  c64.h = h;
  c64.hinv = 1.0 / h;
  c32.h = (float)h;
  c32.hinv = (float)(1.0 / h);
  if ((rc = upload(ctx, bt.ulong_r.data(), bt.ulong_r.size(), &c64.ulong))) return rc;
  if ((rc = upload(ctx, bt.dulong_r.data(), bt.dulong_r.size(), &c64.dulong))) return rc;
  std::vector<float> u32(bt.ulong_r.begin(), bt.ulong_r.end()), du32(bt.dulong_r.begin(), bt.dulong_r.end());
  if ((rc = upload(ctx, u32.data(), u32.size(), &c32.ulong))) return rc;
  if ((rc = upload(ctx, du32.data(), du32.size(), &c32.dulong))) return rc;
  c64.long_range = 1;
  c32.long_range = 1;
  return pimc_set_longrange(ctx, c64.num_levels, bt.ulong_k.data(), bt.ulong_r0.data(), bt.ushort_k0.data(),
                            bt.ulong_k0.data(), bt.dulong_k.data(), bt.dulong_r0.data(), bt.dushort_k0.data(),
                            bt.dulong_k0.data(), use_background);
}

int pimc_coulomb_breakup(const double box[3], double z1z2, double smallest_beta, int num_levels, int num_knots,
                         double kcutoff, int num_k, const double *kvecs, double *ulong_k, double *dulong_k,
                         double *ulong_r0, double *dulong_r0, double *ushort_k0, double *dushort_k0,
                         double *ulong_k0, double *dulong_k0, double *rmax, double *ulong_r, double *dulong_r) {
  if (!box || num_levels < 1 || num_knots < 2 || num_k < 0 || (num_k > 0 && !kvecs)) return PIMC_E_ARG;
  BreakupTables bt;
  const int rc = coulomb_breakup(box, z1z2, smallest_beta, num_levels, num_knots, kcutoff, num_k, kvecs, bt);
  if (rc) return rc;
  auto put = [](double *dst, const std::vector<double> &src) {
    if (dst) std::copy(src.begin(), src.end(), dst);
  };
  put(ulong_k, bt.ulong_k);
  put(dulong_k, bt.dulong_k);
  put(ulong_r0, bt.ulong_r0);
  put(dulong_r0, bt.dulong_r0);
  put(ushort_k0, bt.ushort_k0);
  put(dushort_k0, bt.dushort_k0);
  put(ulong_k0, bt.ulong_k0);
  put(dulong_k0, bt.dulong_k0);
  put(ulong_r, bt.ulong_r);
  put(dulong_r, bt.dulong_r);
  if (rmax) *rmax = bt.rmax;
  return PIMC_OK;
}

int pimc_quintic_spline(int n, double h, const double *y, double *coef) {
  if (n < 3 || !(h > 0.0) || !y || !coef) return PIMC_E_ARG;
  return quintic_natural(n, h, y, coef) ? PIMC_OK : PIMC_E_ARG;
}

}  // extern "C"

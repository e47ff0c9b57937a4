// Device-resident multilevel bisection moves (BisectionBlockClass::MakeMove,
// PIMC++/src/Moves/BisectionBlock.cc:380-451).
//
// Design:
//  * The OLD path copy in HBM is the chain state.  During a move the moved
//    particle's OLD and NEW window positions live in shared memory, so NEW
//    never touches HBM; an accepted move writes the window back once.
//  * A slice window is worked by one thread-block cluster of CL CTAs
//    (CL = 1..16).  Warp 0 of every CTA replays the same Philox stream
//    (slice, particle, Gaussians, acceptance), so sampled positions and
//    decisions are identical in every CTA without communication.  Only the
//    stage action sums cross CTAs: lane r of warp 0 writes this CTA's
//    (S_old, S_new) partial into CTA r's shared memory (DSMEM) and after one
//    cluster barrier every CTA adds the partials in rank order — the same
//    bits everywhere.
//  * Gaussians come from a warp-parallel polar method that reproduces the
//    sequential draw order exactly (warp_gaussians); the per-midpoint work
//    of a level runs one midpoint per lane.
//  * Partners x links of a stage are split over the cluster's threads; each
//    item evaluates the pair action for the OLD and the NEW position of the
//    moved particle against the same partner (partners are identical in
//    both copies), accumulated in FP64.
//  * Two schedules.  Sequential: one window at a time, slice1 drawn from the
//    Local stream exactly as ChooseTimeSlices does (BisectionBlock.cc:362-374).
//    Concurrent windows: one launch is one round; the round draws an offset o
//    from the Common stream and cluster w works the window starting at
//    o + w 2^L with its own Local stream.  Window interiors are disjoint and
//    an action term of one window reads no slice another window moves, so
//    the windows commute: this is PIMC++'s time-slice parallelism (slice
//    blocks moved concurrently, PathClass.h:33-36; the offset plays the role
//    of ShiftMove, MetaMoves.cc:39-65) on the clusters of one GPU.
//  * The 1-D DavidPA diagonal column of every level is staged into shared
//    memory once per launch by a bulk TMA copy (cp.async.bulk) completing on
//    an mbarrier; tricubic tables stay in L2/HBM.
//  * No unbounded waits: the mbarrier wait and the Gaussian rejection loop
//    carry iteration caps that set the status word and stop the run.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "bisection.cuh"
#include "device_math.cuh"

namespace cg = cooperative_groups;

namespace pimc {

namespace {

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
// Bulk (non-tensor) TMA copy global -> this CTA's shared memory.  No multicast.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// BisectionStageClass::Sample (BisectionStage.cc:128-289) for one level on
// the window held in shared memory, run by one full warp: writes the NEW
// midpoints and returns log T_old - log T_new (identical in every lane).
__device__ double sample_level_warp(double (*w_old)[3], double (*w_new)[3], double *gbuf, int num_levels, int level,
                                    const DevSystem &s, DevRandom &rng, int lane) {
  const int skip = 1 << (level + 1);
  const int nmid = (1 << num_levels) >> (level + 1);
  warp_gaussians(rng, 3 * nmid, gbuf, lane);
  __syncwarp();
  const double levelTau = 0.5 * s.tau * skip;
  const double sigma2 = (1.0 * s.lambda * levelTau);
  const double sigma = sqrt(sigma2);
  double lo = 0.0, ln = 0.0;
  if (lane < nmid) {
    const int rel = lane * skip;
    const int mid = rel + (skip >> 1);
    double rdiffOld[3], DeltaOld[3], rdiff[3], rbar[3], Delta[3];
    for (int i = 0; i < 3; i++) rdiffOld[i] = w_old[rel + skip][i] - w_old[rel][i];
    put_in_box(rdiffOld, s);
    for (int i = 0; i < 3; i++) DeltaOld[i] = w_old[mid][i] - (w_old[rel][i] + 0.5 * rdiffOld[i]);
    put_in_box(DeltaOld, s);
    for (int i = 0; i < 3; i++) rdiff[i] = w_new[rel + skip][i] - w_new[rel][i];
    put_in_box(rdiff, s);
    for (int i = 0; i < 3; i++) rbar[i] = w_new[rel][i] + 0.5 * rdiff[i];
    for (int i = 0; i < 3; i++) Delta[i] = gbuf[3 * lane + i] * sigma;
    put_in_box(Delta, s);
    double GaussProd = 1.0, GaussProdOld = 1.0;
    for (int dim = 0; dim < 3; dim++) {
      double GaussSum = 0.0, GaussSumOld = 0.0;
      for (int image = -s.num_images; image <= s.num_images; image++) {
        double dist = Delta[dim] + (double)image * s.box[dim];
        double distOld = DeltaOld[dim] + (double)image * s.box[dim];
        GaussSum += exp(-0.5 * dist * dist / sigma2);
        GaussSumOld += exp(-0.5 * distOld * distOld / sigma2);
      }
      GaussProd *= GaussSum;
      GaussProdOld *= GaussSumOld;
    }
    lo = log(GaussProdOld);
    ln = log(GaussProd);
    for (int i = 0; i < 3; i++) w_new[mid][i] = rbar[i] + Delta[i];
  }
  lo = warp_sum(lo);
  ln = warp_sum(ln);
  __syncwarp();
  return -ln + lo;
}

}  // namespace

// KIND: pair-action type; R: precision of the pair terms; SHADOW: also
// evaluate the pair terms in the other precision for the dS error.
template <int KIND, typename R, bool SHADOW>
__global__ void __launch_bounds__(512, 1) bisection_kernel(BisectionArgs a) {
  typedef typename Pair2<R>::T P2;
  typedef typename std::conditional<std::is_same<R, double>::value, float, double>::type RS;  // shadow precision
  typedef typename Pair2<RS>::T P2S;
  __shared__ double w_old[kMaxWindow][3], w_new[kMaxWindow][3];
  __shared__ double gbuf[3 * 32];
  __shared__ double sh_red[16][4];
  __shared__ double xchg[2][kMaxCluster][4];
  __shared__ int s_ctl[4];  // slice1, ptcl, stage accepted, status
  __shared__ __align__(8) uint64_t s_bar;
  extern __shared__ __align__(16) unsigned char dyn[];

  cg::cluster_group cluster = cg::this_cluster();
  const unsigned rank = cluster.block_rank();
  const unsigned CL = cluster.num_blocks();
  const int window = (int)(blockIdx.x / CL);
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  const DevSystem &sys = a.sys;
  const int N = sys.N;
  const int L = a.num_levels;
  const int span = 1 << L;
  ChainState *cs = a.chains + (a.concurrent ? window : 0);
  const bool lead = (rank == 0 && tid == 0);

  // ---- stage the diagonal DavidPA columns into shared memory (bulk TMA) ----
  // Each level's column is diag_stride pairs long, padded so every level and
  // every copy is a multiple of 16 bytes.  The wait is bounded; the cluster
  // then agrees on the outcome so every CTA takes the same path.
  const P2 *diag_smem = nullptr;
  const P2S *diag_smem_s = nullptr;
  if (KIND == PA_DAVID) {
    const DDavid<R> &d = david_of<R>(a.pa);
    const unsigned bytes = (unsigned)(L * d.diag_stride * sizeof(P2));
    unsigned bytes_s = 0;
    if (SHADOW) bytes_s = (unsigned)(L * david_of<RS>(a.pa).diag_stride * sizeof(P2S));
    if (tid == 0) {
      mbar_init(&s_bar, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&s_bar, bytes + bytes_s);
      bulk_g2s(dyn, reinterpret_cast<const P2 *>(d.diag) + (size_t)d.tau_pos * d.diag_stride, bytes, &s_bar);
      if (SHADOW) {
        const DDavid<RS> &ds = david_of<RS>(a.pa);
        bulk_g2s(dyn + bytes, reinterpret_cast<const P2S *>(ds.diag) + (size_t)ds.tau_pos * ds.diag_stride, bytes_s,
                 &s_bar);
      }
    }
    __syncthreads();
    int ok = 0;
    for (int it = 0; it < (1 << 22); it++)
      if (mbar_try_wait(&s_bar, 0)) {
        ok = 1;
        break;
      }
    ok = __syncthreads_and(ok);
    if (tid < (int)CL) cluster.map_shared_rank(&xchg[1][rank][0], tid)[0] = ok ? 1.0 : 0.0;
    cluster.sync();
    int all_ok = 1;
    for (unsigned r = 0; r < CL; r++) all_ok &= (xchg[1][r][0] != 0.0);
    if (!all_ok) {
      // Give a late copy a second bounded chance to land before this CTA exits.
      for (int it = 0; it < (1 << 22) && !ok; it++) ok = mbar_try_wait(&s_bar, 0);
      if (lead) atomicExch(&cs->status, PIMC_E_CAP);
      cluster.sync();
      return;
    }
    diag_smem = reinterpret_cast<const P2 *>(dyn);
    if (SHADOW) diag_smem_s = reinterpret_cast<const P2S *>(dyn + bytes);
  }

  // ---- RNG state: every lane of warp 0 of every CTA holds the same copy ----
  DevRandom rng;
  rng.seed = cs->seed;
  rng.n = cs->nlocal;
  rng.stream = cs->stream;
  rng.one_left = cs->one_left;
  rng.x2 = cs->x2;
  unsigned long long moves = 0, accepted = 0, stages = 0, pair_evals = 0, flips = 0;
  int status = 0;
  double *path = a.path;
  unsigned xc = 0;  // exchange parity counter

  // Window of this cluster in the concurrent schedule.
  int slice1 = 0;
  if (a.concurrent) {
    const int o = (int)floor(philox_uniform(rng.seed, kStreamCommon, a.round) * span);
    slice1 = o + window * span;
    if (slice1 + span > sys.S - 1) {
      // Inactive this round (uniform over the cluster): mark its trace slots.
      if (a.trace && lead)
        for (int st = 0; st < a.steps_per_block; st++) {
          pimc_move_record r = {};
          r.slice1 = -1;
          r.ptcl = -1;
          a.trace[a.trace_offset + (long long)window * a.steps_per_block + st] = r;
        }
      if (KIND == PA_DAVID) cluster.sync();  // xchg[1] no longer read by peers
      return;
    }
  }
  if (KIND == PA_DAVID) cluster.sync();  // every CTA has read xchg[1]
  const int numLeft = sys.S - span;
  const int n_blocks = a.concurrent ? 1 : a.n_blocks;

  for (int blk = 0; blk < n_blocks; blk++) {
    for (int step = 0; step < a.steps_per_block; step++) {
      // ChooseTimeSlices (BisectionBlock.cc:362-374), ChooseParticle (NoPermuteClass.cc:61-68)
      if (warp == 0) {
        if (!a.concurrent && step == 0) slice1 = rng.LocalInt(numLeft);
        const int p = rng.LocalInt(N);
        if (lane == 0) {
          s_ctl[0] = slice1;
          s_ctl[1] = p;
        }
      }
      __syncthreads();
      slice1 = s_ctl[0];
      const int ptcl = s_ctl[1];
      for (int rel = tid; rel <= span; rel += blockDim.x) {
        const double *p = path + ((size_t)(slice1 + rel) * N + ptcl) * 3;
        for (int i = 0; i < 3; i++) w_old[rel][i] = w_new[rel][i] = p[i];
      }
      __syncthreads();
      double logsr = 0.0;  // meaningful in warp 0
      if (warp == 0) logsr = sample_level_warp(w_old, w_new, gbuf, L, L - 1, sys, rng, lane);
      __syncthreads();

      double prevDS = 0.0, prevDS_s = 0.0;
      bool acc_all = true;
      int passed = 0;
      pimc_move_record rec;
      if (lead) {
        rec.slice1 = slice1;
        rec.ptcl = ptcl;
        for (int i = 0; i < 8; i++) rec.dS[i] = rec.dS_shadow[i] = 0.0;
      }
      int si = 0;
      for (int level = L - 1; level >= 0; level--, si++) {
        // ---- LocalStageClass::Attempt (StageClass.cc:49-95) ----
        const int skip = 1 << level;
        const int nlinks = span >> level;
        double so = 0.0, sn = 0.0, so2 = 0.0, sn2 = 0.0;
        // Kinetic (KineticClass::SingleAction) on the moved particle, CTA 0 only.
        if (rank == 0 && tid < nlinks && sys.lambda != 0.0) {
          const double levelTau = sys.tau * (1 << level);
          const double F = 1.0 / (4.0 * sys.lambda * levelTau);
          const int r0 = tid * skip;
          double vo[3], vn[3];
          for (int i = 0; i < 3; i++) {
            vo[i] = w_old[r0 + skip][i] - w_old[r0][i];
            vn[i] = w_new[r0 + skip][i] - w_new[r0][i];
          }
          put_in_box(vo, sys);
          put_in_box(vn, sys);
          const double ko = kinetic_link(vo, F, sys.num_images, sys), kn = kinetic_link(vn, F, sys.num_images, sys);
          so += ko;
          sn += kn;
          if (SHADOW) {
            so2 += ko;
            sn2 += kn;
          }
        }
        // ShortRange (ShortRangeClass::SingleAction) over partners x links.
        if (level == 0 || a.sr_higher) {
          const int np = N - 1;
          const long long total = (long long)np * nlinks;
          const long long chunk = (total + CL - 1) / CL;
          const long long beg = chunk * rank;
          const long long end = min(total, beg + chunk);
          const P2 *dg = nullptr;
          const P2S *dgs = nullptr;
          if (KIND == PA_DAVID) {
            dg = diag_smem + (size_t)level * david_of<R>(a.pa).diag_stride;
            if (SHADOW) dgs = diag_smem_s + (size_t)level * david_of<RS>(a.pa).diag_stride;
          }
          for (long long it = beg + tid; it < end; it += blockDim.x) {
            const int link = (int)(it / np);
            const int j = (int)(it - (long long)link * np);
            const int p2 = j < ptcl ? j : j + 1;
            const int r0 = link * skip;
            const double *pa_ = path + ((size_t)(slice1 + r0) * N + p2) * 3;
            const double *pb_ = path + ((size_t)(slice1 + r0 + skip) * N + p2) * 3;
            const double a2[3] = {__ldg(pa_), __ldg(pa_ + 1), __ldg(pa_ + 2)};
            const double b2[3] = {__ldg(pb_), __ldg(pb_ + 1), __ldg(pb_ + 2)};
            double dAo[3], dBo[3], dAn[3], dBn[3];
            dist_disp(w_old[r0], a2, w_old[r0 + skip], b2, sys, dAo, dBo);
            dist_disp(w_new[r0], a2, w_new[r0 + skip], b2, sys, dAn, dBn);
            const LinkGeom<R> go = link_geom<R>(dAo, dBo);
            const LinkGeom<R> gn = link_geom<R>(dAn, dBn);
            so += (double)pa_U<R, KIND>(a.pa, dg, go, level);
            sn += (double)pa_U<R, KIND>(a.pa, dg, gn, level);
            if (SHADOW) {
              so2 += (double)pa_U<RS, KIND>(a.pa, dgs, link_geom<RS>(dAo, dBo), level);
              sn2 += (double)pa_U<RS, KIND>(a.pa, dgs, link_geom<RS>(dAn, dBn), level);
            }
          }
          if (lead) pair_evals += 2ull * (unsigned long long)total;
        }
        // ---- reduce: warps -> CTA (warp 0) -> cluster (DSMEM, rank order) ----
        so = warp_sum(so);
        sn = warp_sum(sn);
        if (SHADOW) {
          so2 = warp_sum(so2);
          sn2 = warp_sum(sn2);
        }
        if (lane == 0) {
          sh_red[warp][0] = so;
          sh_red[warp][1] = sn;
          sh_red[warp][2] = so2;
          sh_red[warp][3] = sn2;
        }
        __syncthreads();
        const int par = xc & 1;
        xc++;
        if (warp == 0) {
          double v[4] = {0.0, 0.0, 0.0, 0.0};
          for (int w = 0; w < nwarps; w++)
            for (int c = 0; c < 4; c++) v[c] += sh_red[w][c];
          so = v[0];
          sn = v[1];
          so2 = v[2];
          sn2 = v[3];
          if (CL > 1 && lane < (int)CL) {
            double *dst = cluster.map_shared_rank(&xchg[par][rank][0], lane);
            dst[0] = so;
            dst[1] = sn;
            dst[2] = so2;
            dst[3] = sn2;
          }
        }
        if (CL > 1) {
          cluster.sync();
          if (warp == 0) {
            so = sn = so2 = sn2 = 0.0;
            for (unsigned r = 0; r < CL; r++) {
              so += xchg[par][r][0];
              sn += xchg[par][r][1];
              so2 += xchg[par][r][2];
              sn2 += xchg[par][r][3];
            }
          }
        }
        // ---- Metropolis test (identical in every CTA), then sample the next level ----
        if (warp == 0) {
          const double currActionChange = sn - so;
          const double logAcceptProb = logsr - currActionChange + prevDS;
          const double logu = log(rng.Local());
          bool toAccept = logAcceptProb >= logu;
          if (toAccept && (fabs(sn) > 1e50 || fabs(so) > 1e50)) {  // StageClass.cc:74-85
            toAccept = false;
            status = PIMC_E_STAGING;
          }
          if (!isfinite(currActionChange)) status = PIMC_E_NAN;
          if (SHADOW) {
            const double dss = sn2 - so2;
            const bool other = (logsr - dss + prevDS_s) >= logu;
            if (other != toAccept && lead) flips++;
            prevDS_s = dss;
          }
          prevDS = currActionChange;
          if (lead && si < 8) {
            rec.dS[si] = currActionChange;
            if (SHADOW) rec.dS_shadow[si] = sn2 - so2;
          }
          if (toAccept && level > 0 && status == 0)
            logsr = sample_level_warp(w_old, w_new, gbuf, L, level - 1, sys, rng, lane);
          if (lane == 0) {
            s_ctl[2] = toAccept ? 1 : 0;
            s_ctl[3] = status;
          }
        }
        __syncthreads();
        if (tid == 0) stages++;
        if (!s_ctl[2] || s_ctl[3]) {
          acc_all = false;
          break;
        }
        passed++;
      }
      // ---- AcceptCopy (PathClass.cc:797-863); a rejected move left HBM untouched ----
      if (acc_all) {
        if (rank == 0)
          for (int rel = tid; rel <= span; rel += blockDim.x) {
            double v[3] = {w_new[rel][0], w_new[rel][1], w_new[rel][2]};
            put_in_box_fast(v, sys);
            double *p = path + ((size_t)(slice1 + rel) * N + ptcl) * 3;
            p[0] = v[0];
            p[1] = v[1];
            p[2] = v[2];
          }
        if (CL > 1)
          cluster.sync();
        else
          __syncthreads();
      }
      if (lead) {
        moves++;
        if (acc_all) accepted++;
        if (a.trace) {
          rec.accepted = acc_all ? 1 : 0;
          rec.stages_passed = passed;
          const long long idx = a.concurrent ? a.trace_offset + (long long)window * a.steps_per_block + step
                                             : a.trace_offset + (long long)blk * a.steps_per_block + step;
          a.trace[idx] = rec;
        }
      }
      if (s_ctl[3] != 0) break;
    }
    if (s_ctl[3] != 0) break;
  }
  if (lead) {
    cs->nlocal = rng.n;
    cs->one_left = rng.one_left;
    cs->x2 = rng.x2;
    cs->moves += moves;
    cs->accepted += accepted;
    cs->stages += stages;
    cs->pair_evals += pair_evals;
    cs->flips += flips;
    if (status) cs->status = status;
  }
  if (CL > 1) cluster.sync();
}

template <int KIND, typename R, bool SHADOW>
static cudaError_t launch_t(const BisectionArgs &a, int cl, int clusters, int threads, size_t dyn, cudaStream_t st) {
  auto kfn = bisection_kernel<KIND, R, SHADOW>;
  cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  if (e != cudaSuccess) return e;
  if (cl > 8) {
    e = cudaFuncSetAttribute(kfn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cl * clusters, 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = dyn;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cl;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kfn, a);
}

size_t bisection_dyn_smem(const BisectionArgs &a, int precision, int shadow) {
  if (a.pa.kind != PA_DAVID) return 0;
  const size_t b64 = (size_t)a.num_levels * a.pa.d64.diag_stride * sizeof(double2);
  const size_t b32 = (size_t)a.num_levels * a.pa.d32.diag_stride * sizeof(float2);
  size_t dyn = precision == PIMC_MIXED ? b32 : b64;
  if (shadow) dyn += precision == PIMC_MIXED ? b64 : b32;
  return dyn;
}

cudaError_t launch_bisection(const BisectionArgs &a, int precision, int shadow, int cl, int clusters, int threads,
                             cudaStream_t st) {
  const size_t dyn = bisection_dyn_smem(a, precision, shadow);
  if (dyn > (size_t)200 * 1024) return cudaErrorInvalidValue;  // tables too large for shared memory
  if (threads < 64 || threads > 512 || threads % 32 || cl < 1 || cl > kMaxCluster || clusters < 1 ||
      clusters > kMaxWindows)
    return cudaErrorInvalidValue;
  const bool mixed = precision == PIMC_MIXED;
  if (a.pa.kind == PA_DAVID) {
    if (mixed) return shadow ? launch_t<PA_DAVID, float, true>(a, cl, clusters, threads, dyn, st)
                             : launch_t<PA_DAVID, float, false>(a, cl, clusters, threads, dyn, st);
    return shadow ? launch_t<PA_DAVID, double, true>(a, cl, clusters, threads, dyn, st)
                  : launch_t<PA_DAVID, double, false>(a, cl, clusters, threads, dyn, st);
  }
  if (mixed) return shadow ? launch_t<PA_TRICUBIC, float, true>(a, cl, clusters, threads, dyn, st)
                           : launch_t<PA_TRICUBIC, float, false>(a, cl, clusters, threads, dyn, st);
  return shadow ? launch_t<PA_TRICUBIC, double, true>(a, cl, clusters, threads, dyn, st)
                : launch_t<PA_TRICUBIC, double, false>(a, cl, clusters, threads, dyn, st);
}

}  // namespace pimc

// Device-resident multilevel bisection moves (BisectionBlockClass::MakeMove,
// PIMC++/src/Moves/BisectionBlock.cc:380-451) for one chain.
//
// Design:
//  * The OLD path copy in HBM is the chain state.  During a move the moved
//    particle's OLD and NEW window positions live in shared memory, so NEW
//    never touches HBM; an accepted move writes the window back once.
//  * One chain runs on a thread-block cluster of CL CTAs (CL = 1..16).  Every
//    CTA draws the same Philox stream in thread 0 (slice, particle, Gaussians,
//    acceptance), so the sampled positions and decisions are identical in
//    every CTA without communication.  Only the stage action sums cross CTAs:
//    each CTA writes its (S_old, S_new) partial into every peer's shared
//    memory (DSMEM) and one cluster barrier later all CTAs add the partials in
//    rank order — the same bits everywhere.
//  * Partners x links of a stage are split over the cluster's threads; each
//    item evaluates the pair action for the OLD and the NEW position of the
//    moved particle against the same partner (partners are identical in
//    both copies), accumulated in FP64.
//  * The 1-D DavidPA diagonal column of every level is staged into shared
//    memory once per launch with a bulk TMA copy (cp.async.bulk) completing
//    on an mbarrier; tricubic tables stay in L2/HBM.
//  * No unbounded waits: the mbarrier wait and the Gaussian rejection loop
//    carry iteration caps that set the chain's status word and stop the run.
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

template <typename R>
struct Acc {
  double o, n;
};

// Sum of two doubles over the CTA; result valid in thread 0.
__device__ __forceinline__ void block_sum2(double &a, double &b, double (*sh)[2]) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sh[w][0] = a;
    sh[w][1] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0.0, y = 0.0;
    const int nw = blockDim.x >> 5;
    for (int i = 0; i < nw; i++) {
      x += sh[i][0];
      y += sh[i][1];
    }
    a = x;
    b = y;
  }
}

// BisectionStageClass::Sample (BisectionStage.cc:128-289) on the window held
// in shared memory: writes the NEW midpoints of this level and returns
// log T_old - log T_new.  Runs on one thread (it owns the RNG stream).
__device__ double sample_level(double (*w_old)[3], double (*w_new)[3], int num_levels, int level, const DevSystem &s,
                               DevRandom &rng) {
  const int skip = 1 << (level + 1);
  const double levelTau = 0.5 * s.tau * skip;
  const double sigma2 = (1.0 * s.lambda * levelTau);
  const double sigma = sqrt(sigma2);
  const int span = 1 << num_levels;
  double logSampleProb = 0.0, logOldSampleProb = 0.0;
  for (int rel = 0; rel < span; rel += skip) {
    const int mid = rel + (skip >> 1);
    double rdiffOld[3], DeltaOld[3], rdiff[3], rbar[3], Delta[3];
    for (int i = 0; i < 3; i++) rdiffOld[i] = w_old[rel + skip][i] - w_old[rel][i];
    put_in_box(rdiffOld, s);
    for (int i = 0; i < 3; i++) DeltaOld[i] = w_old[mid][i] - (w_old[rel][i] + 0.5 * rdiffOld[i]);
    put_in_box(DeltaOld, s);
    for (int i = 0; i < 3; i++) rdiff[i] = w_new[rel + skip][i] - w_new[rel][i];
    put_in_box(rdiff, s);
    for (int i = 0; i < 3; i++) rbar[i] = w_new[rel][i] + 0.5 * rdiff[i];
    for (int i = 0; i < 3; i++) Delta[i] = rng.LocalGaussian(sigma);
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
    logOldSampleProb += log(GaussProdOld);
    logSampleProb += log(GaussProd);
    for (int i = 0; i < 3; i++) w_new[mid][i] = rbar[i] + Delta[i];
  }
  return -logSampleProb + logOldSampleProb;
}

}  // namespace

// One launch runs n_blocks BisectionBlock moves (steps_per_block moves each).
// KIND: pair-action type; R: precision of the pair terms; SHADOW: also
// evaluate the pair terms in the other precision for the dS error.
template <int KIND, typename R, bool SHADOW>
__global__ void __launch_bounds__(512) bisection_kernel(BisectionArgs a) {
  typedef typename Pair2<R>::T P2;
  typedef typename std::conditional<std::is_same<R, double>::value, float, double>::type RS;  // shadow precision
  typedef typename Pair2<RS>::T P2S;
  __shared__ double w_old[kMaxWindow][3], w_new[kMaxWindow][3];
  __shared__ double sh_red[16][2];
  __shared__ double sh_red2[16][2];
  __shared__ double xchg[2][kMaxCluster][4];
  __shared__ int s_ctl[4];
  __shared__ __align__(8) uint64_t s_bar;
  extern __shared__ __align__(16) unsigned char dyn[];

  cg::cluster_group cluster = cg::this_cluster();
  const unsigned rank = cluster.block_rank();
  const unsigned CL = cluster.num_blocks();
  const int tid = threadIdx.x;
  const DevSystem &sys = a.sys;
  const int N = sys.N;
  const int L = a.num_levels;
  const int span = 1 << L;

  if (tid == 0) s_ctl[3] = 0;
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
    if (tid == 0)
      for (unsigned r = 0; r < CL; r++) cluster.map_shared_rank(&xchg[0][rank][0], r)[0] = ok ? 1.0 : 0.0;
    cluster.sync();
    int all_ok = 1;
    for (unsigned r = 0; r < CL; r++) all_ok &= (xchg[0][r][0] != 0.0);
    if (!all_ok) {
      // Give a late copy a second bounded chance to land before this CTA exits.
      for (int it = 0; it < (1 << 22) && !ok; it++) ok = mbar_try_wait(&s_bar, 0);
      if (tid == 0 && rank == 0) atomicExch(&a.chain->status, PIMC_E_CAP);
      cluster.sync();
      return;
    }
    cluster.sync();  // every CTA has read xchg[0] before it is reused
    diag_smem = reinterpret_cast<const P2 *>(dyn);
    if (SHADOW) diag_smem_s = reinterpret_cast<const P2S *>(dyn + bytes);
  }
  __syncthreads();

  // ---- chain state: thread 0 of every CTA replays the same stream ----
  DevRandom rng;
  unsigned long long moves = 0, accepted = 0, stages = 0, pair_evals = 0, flips = 0;
  int status = 0;
  if (tid == 0) {
    rng.seed = a.chain->seed;
    rng.n = a.chain->nlocal;
    rng.one_left = a.chain->one_left;
    rng.x2 = a.chain->x2;
  }
  double *path = a.path;
  unsigned xc = 0;  // exchange parity counter
  const int numLeft = sys.S - span;

  for (int blk = 0; blk < a.n_blocks; blk++) {
    for (int step = 0; step < a.steps_per_block; step++) {
      // ChooseTimeSlices (BisectionBlock.cc:362-374) and ChooseParticle (NoPermuteClass.cc:61-68)
      if (tid == 0) {
        if (step == 0) s_ctl[0] = rng.LocalInt(numLeft);
        s_ctl[1] = rng.LocalInt(N);
      }
      __syncthreads();
      const int slice1 = s_ctl[0];
      const int ptcl = s_ctl[1];
      for (int rel = tid; rel <= span; rel += blockDim.x) {
        const double *p = path + ((size_t)(slice1 + rel) * N + ptcl) * 3;
        for (int i = 0; i < 3; i++) w_old[rel][i] = w_new[rel][i] = p[i];
      }
      __syncthreads();

      double prevDS = 0.0, prevDS_s = 0.0;
      bool acc_all = true;
      int passed = 0;
      pimc_move_record rec;
      if (tid == 0 && rank == 0) {
        rec.slice1 = slice1;
        rec.ptcl = ptcl;
        for (int i = 0; i < 8; i++) rec.dS[i] = rec.dS_shadow[i] = 0.0;
      }
      int si = 0;
      for (int level = L - 1; level >= 0; level--, si++) {
        // ---- LocalStageClass::Attempt (StageClass.cc:49-95) ----
        __shared__ double s_logsr;
        if (tid == 0) s_logsr = sample_level(w_old, w_new, L, level, sys, rng);
        __syncthreads();
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
          double ko = kinetic_link(vo, F, sys.num_images, sys), kn = kinetic_link(vn, F, sys.num_images, sys);
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
            double a2[3] = {__ldg(pa_), __ldg(pa_ + 1), __ldg(pa_ + 2)};
            double b2[3] = {__ldg(pb_), __ldg(pb_ + 1), __ldg(pb_ + 2)};
            double dA[3], dB[3];
            dist_disp(w_old[r0], a2, w_old[r0 + skip], b2, sys, dA, dB);
            LinkGeom<R> go = link_geom<R>(dA, dB);
            so += (double)pa_U<R, KIND>(a.pa, dg, go, level);
            if (SHADOW) so2 += (double)pa_U<RS, KIND>(a.pa, dgs, link_geom<RS>(dA, dB), level);
            dist_disp(w_new[r0], a2, w_new[r0 + skip], b2, sys, dA, dB);
            LinkGeom<R> gn = link_geom<R>(dA, dB);
            sn += (double)pa_U<R, KIND>(a.pa, dg, gn, level);
            if (SHADOW) sn2 += (double)pa_U<RS, KIND>(a.pa, dgs, link_geom<RS>(dA, dB), level);
          }
          if (tid == 0 && rank == 0) pair_evals += 2ull * (unsigned long long)total;
        }
        block_sum2(so, sn, sh_red);
        if (SHADOW) block_sum2(so2, sn2, sh_red2);
        // ---- combine the cluster's partials (DSMEM), rank order ----
        const int par = xc & 1;
        xc++;
        if (CL > 1) {
          if (tid == 0) {
            for (unsigned r = 0; r < CL; r++) {
              double *dst = cluster.map_shared_rank(&xchg[par][rank][0], r);
              dst[0] = so;
              dst[1] = sn;
              dst[2] = so2;
              dst[3] = sn2;
            }
          }
          cluster.sync();
          if (tid == 0) {
            so = sn = so2 = sn2 = 0.0;
            for (unsigned r = 0; r < CL; r++) {
              so += xchg[par][r][0];
              sn += xchg[par][r][1];
              so2 += xchg[par][r][2];
              sn2 += xchg[par][r][3];
            }
          }
        }
        // ---- Metropolis test, identical in every CTA ----
        if (tid == 0) {
          const double logSampleRatio = s_logsr;
          const double currActionChange = sn - so;
          const double logAcceptProb = logSampleRatio - currActionChange + prevDS;
          const double u = rng.Local();
          const double logu = log(u);
          bool toAccept = logAcceptProb >= logu;
          if (toAccept && (fabs(sn) > 1e50 || fabs(so) > 1e50)) {  // StageClass.cc:74-85
            toAccept = false;
            status = PIMC_E_STAGING;
          }
          if (!isfinite(currActionChange)) status = PIMC_E_NAN;
          if (SHADOW) {
            const double dss = sn2 - so2;
            const bool other = (logSampleRatio - dss + prevDS_s) >= logu;
            if (other != toAccept) flips++;
            prevDS_s = dss;
          }
          prevDS = currActionChange;
          if (rank == 0 && si < 8) {
            rec.dS[si] = currActionChange;
            if (SHADOW) rec.dS_shadow[si] = sn2 - so2;
          }
          s_ctl[2] = toAccept ? 1 : 0;
          s_ctl[3] = status;
        }
        __syncthreads();
        if (tid == 0) stages++;
        if (!s_ctl[2]) {
          acc_all = false;
          break;
        }
        passed++;
      }
      // ---- AcceptCopy (PathClass.cc:797-863) / RejectCopy ----
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
      if (tid == 0 && rank == 0) {
        moves++;
        if (acc_all) accepted++;
        if (a.trace) {
          rec.accepted = acc_all ? 1 : 0;
          rec.stages_passed = passed;
          a.trace[a.trace_offset + (long long)blk * a.steps_per_block + step] = rec;
        }
      }
      if (s_ctl[3] != 0) break;
    }
    if (s_ctl[3] != 0) break;
  }
  if (tid == 0 && rank == 0) {
    a.chain->nlocal = rng.n;
    a.chain->one_left = rng.one_left;
    a.chain->x2 = rng.x2;
    a.chain->moves += moves;
    a.chain->accepted += accepted;
    a.chain->stages += stages;
    a.chain->pair_evals += pair_evals;
    a.chain->flips += flips;
    if (status) a.chain->status = status;
  }
  if (CL > 1) cluster.sync();
}

template <int KIND, typename R, bool SHADOW>
static cudaError_t launch_t(const BisectionArgs &a, int cl, int threads, size_t dyn, cudaStream_t st) {
  auto kfn = bisection_kernel<KIND, R, SHADOW>;
  cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  if (e != cudaSuccess) return e;
  if (cl > 8) {
    e = cudaFuncSetAttribute(kfn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cl, 1, 1);
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

cudaError_t launch_bisection(const BisectionArgs &a, int precision, int shadow, int cl, int threads,
                             cudaStream_t st) {
  size_t dyn = 0;
  if (a.pa.kind == PA_DAVID) {
    const size_t b64 = (size_t)a.num_levels * a.pa.d64.diag_stride * sizeof(double2);
    const size_t b32 = (size_t)a.num_levels * a.pa.d32.diag_stride * sizeof(float2);
    dyn = precision == PIMC_MIXED ? b32 : b64;
    if (shadow) dyn += precision == PIMC_MIXED ? b64 : b32;
  }
  if (dyn > (size_t)200 * 1024) return cudaErrorInvalidValue;  // tables too large for shared memory
  if (threads < 64 || threads > 512 || threads % 32 || cl < 1 || cl > kMaxCluster) return cudaErrorInvalidValue;
  const bool mixed = precision == PIMC_MIXED;
  if (a.pa.kind == PA_DAVID) {
    if (mixed) return shadow ? launch_t<PA_DAVID, float, true>(a, cl, threads, dyn, st)
                             : launch_t<PA_DAVID, float, false>(a, cl, threads, dyn, st);
    return shadow ? launch_t<PA_DAVID, double, true>(a, cl, threads, dyn, st)
                  : launch_t<PA_DAVID, double, false>(a, cl, threads, dyn, st);
  }
  if (mixed) return shadow ? launch_t<PA_TRICUBIC, float, true>(a, cl, threads, dyn, st)
                           : launch_t<PA_TRICUBIC, float, false>(a, cl, threads, dyn, st);
  return shadow ? launch_t<PA_TRICUBIC, double, true>(a, cl, threads, dyn, st)
                : launch_t<PA_TRICUBIC, double, false>(a, cl, threads, dyn, st);
}

}  // namespace pimc

// Device-resident multilevel bisection moves (BisectionBlockClass::MakeMove,
// PIMC++/src/Moves/BisectionBlock.cc:380-451).
//
// Design:
//  * The OLD path copy in HBM is the chain state.  During a move the moved
//    particle's OLD and NEW window positions live in shared memory, so NEW
//    never touches HBM; an accepted move writes the window back once.
//  * A slice window is worked by one thread-block cluster of CL CTAs
//    (CL = 1..16).  The sampler warp (the last warp) of every CTA replays the
//    same Philox stream (slice, particle, Gaussians, acceptance), so sampled
//    positions and decisions are identical in every CTA without
//    communication.  Only the stage action sums cross CTAs: warp 0 stores
//    this CTA's partials into every peer's shared memory (st.async, each
//    store completing bytes on the peer's mbarrier); once its mbarrier has
//    all CTAs' bytes, warp 0 of every CTA adds the partials in rank order —
//    the same bits everywhere — while the other warps wait at the CTA
//    barrier only, not at a cluster barrier.
//  * Gaussians come from a warp-parallel polar method that reproduces the
//    sequential draw order exactly (warp_gaussians); the per-midpoint work
//    of a level runs one midpoint per lane.
//  * Partners x links of a stage are split over the cluster's threads and
//    accumulated in FP64.  Partners are identical in the OLD and NEW copies,
//    so each item reads its partner once and evaluates the pair action for
//    the OLD and the NEW position of the moved particle, while the sampler
//    warp draws the next level speculatively.  The FP64 tricubic path splits
//    (item, copy) units evenly over the evaluating warps and gathers the
//    terms inside the fit by 4-lane teams (tricubic_stage).  The moved
//    particle's kinetic links are summed by the last evaluating warp.
//  * Three schedules.  Sequential: one window at a time, slice1 drawn from the
//    Local stream exactly as ChooseTimeSlices does (BisectionBlock.cc:362-374).
//    Concurrent windows: one launch is one round; the round draws an offset o
//    from the Common stream and cluster w works the window starting at
//    o + w 2^L with its own Local stream.  Window interiors are disjoint and
//    an action term of one window reads no slice another window moves, so
//    the windows commute: this is PIMC++'s time-slice parallelism (slice
//    blocks moved concurrently, PathClass.h:33-36; the offset plays the role
//    of ShiftMove, MetaMoves.cc:39-65) on the clusters of one GPU.
//    Concurrent proposals: the windows schedule with P CTAs per window, each
//    one proposal slot with its own Local stream evaluating alone; a step of
//    the window has the result of slots 0..P-1 moving one after another, and
//    a slot whose particle an earlier slot's accepted move came near is made
//    again (the in-order commit in run_job).
//  * The 1-D DavidPA diagonal column of every level (tricubic, FP64 path:
//    the potential's (y, d2y) pairs of the primitive fallback) is staged into
//    shared memory once per launch by a bulk TMA copy (cp.async.bulk)
//    completing on an mbarrier; tricubic node tables stay in L2/HBM.
//  * No unbounded waits: the mbarrier waits (table staging, stage
//    reductions) and the Gaussian rejection loop carry iteration caps that
//    set the status word and stop the run.
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
// The same wait with acquire at cluster scope: the phase's bytes were stored
// by other CTAs of the cluster (st.async).
__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t *bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
// Address of the same shared-memory variable in CTA `rank` of the cluster.
__device__ __forceinline__ unsigned mapa_u32(unsigned addr, unsigned rank) {
  unsigned d;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(d) : "r"(addr), "r"(rank));
  return d;
}
// Store of one double into a cluster CTA's shared memory that completes 8
// transaction bytes on that CTA's mbarrier `bar`.
__device__ __forceinline__ void st_async_f64(unsigned addr, double v, unsigned bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f64 [%0], %1, [%2];" ::"r"(addr), "d"(v),
               "r"(bar)
               : "memory");
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
// warp_sum when only lanes [0, n) can hold nonzero values: the butterfly
// starts at the half of the smallest power of two >= n (the steps skipped
// would add exact zeros to lane 0, so lane 0's sum has the same bits), and
// lane 0's sum is broadcast.
__device__ __forceinline__ double warp_sum_n(double v, int n) {
  int o = 16;
  while (o > 1 && o >= n) o >>= 1;
  for (; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return __shfl_sync(0xffffffffu, v, 0);
}

// BisectionStageClass::Sample (BisectionStage.cc:128-289) for one level on
// the window held in shared memory, run by one full warp: writes the NEW
// midpoints and returns log T_old - log T_new (identical in every lane).
__device__ __forceinline__ double sample_level_warp(double (*w_old)[3], double (*w_new)[3], double *gbuf, int num_levels, int level,
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
    // log of the image-summed Gaussian transition densities (BisectionStage.cc:241-256).
    // Without images, log(prod_d exp(-x_d)) = -sum_d x_d up to rounding while no
    // factor underflows; otherwise the reference's product is formed.
    bool direct = s.num_images == 0;
    double eo[3], en[3];
    for (int dim = 0; dim < 3; dim++) {
      en[dim] = 0.5 * Delta[dim] * Delta[dim] / sigma2;
      eo[dim] = 0.5 * DeltaOld[dim] * DeltaOld[dim] / sigma2;
      direct = direct && en[dim] < 700.0 && eo[dim] < 700.0;
    }
    if (direct) {
      lo = -(eo[0] + eo[1] + eo[2]);
      ln = -(en[0] + en[1] + en[2]);
    } else {
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
    }
    for (int i = 0; i < 3; i++) w_new[mid][i] = rbar[i] + Delta[i];
  }
  lo = warp_sum_n(lo, nmid);
  ln = warp_sum_n(ln, nmid);
  __syncwarp();
  return -ln + lo;
}
__device__ __noinline__ double sample_level_warp_outlined(double (*w_old)[3], double (*w_new)[3], double *gbuf,
                                                          int num_levels, int level, const DevSystem &s,
                                                          DevRandom &rng, int lane) {
  return sample_level_warp(w_old, w_new, gbuf, num_levels, level, s, rng, lane);
}
// The level sampler: one out-of-line copy (OUTLINE: fewer cold instruction
// lines per stage when a CTA runs many short jobs) or inlined at each call.
template <bool OUTLINE>
__device__ __forceinline__ double sample_level(double (*w_old)[3], double (*w_new)[3], double *gbuf, int num_levels,
                                               int level, const DevSystem &s, DevRandom &rng, int lane) {
  return OUTLINE ? sample_level_warp_outlined(w_old, w_new, gbuf, num_levels, level, s, rng, lane)
                 : sample_level_warp(w_old, w_new, gbuf, num_levels, level, s, rng, lane);
}

}  // namespace

// e^{i k.r} of one k-vector: the phase in FP64, its sine and cosine in R (the
// FP32 path reduces the phase to [-pi, pi] in FP64 first).
template <typename R>
__device__ __forceinline__ double2 cis_k(const double *kv, const double r[3]);
template <>
__device__ __forceinline__ double2 cis_k<double>(const double *kv, const double r[3]) {
  const double th = radd(radd(rmul(kv[0], r[0]), rmul(kv[1], r[1])), rmul(kv[2], r[2]));
  double sn, cs;
  sincos(th, &sn, &cs);
  return make_double2(cs, sn);
}
template <>
__device__ __forceinline__ double2 cis_k<float>(const double *kv, const double r[3]) {
  const double th = radd(radd(rmul(kv[0], r[0]), rmul(kv[1], r[1])), rmul(kv[2], r[2]));
  const double n = rint(th * 0.15915494309189535);  // 1 / (2 pi)
  const float red = (float)(th - n * 6.283185307179586);
  float sn, cs;
  sincosf(red, &sn, &cs);
  return make_double2((double)cs, (double)sn);
}
// rho_k of the NEW path at one slice after the moved particle's update
// (PathClass::UpdateRho_ks, PathClass.cc:649-707): NEW = OLD, + e^{ik.r_new},
// - e^{ik.r_old}, in that order.
template <typename R>
__device__ __forceinline__ double2 rho_new_k(double2 ro, const double *kv, const double rn[3], const double rold[3]) {
  const double2 cn = cis_k<R>(kv, rn), co = cis_k<R>(kv, rold);
  double2 r = make_double2(ro.x + cn.x, ro.y + cn.y);
  r.x -= co.x;
  r.y -= co.y;
  return r;
}

// OLD and NEW action sums of one stage level over this CTA's share of the
// (partner, link) items (the moved particle's kinetic links are summed by
// the sampler warp, kinetic_sums).  Partner positions are read once and
// serve both copies.
//  * R = double: the FP64 path; SHADOW adds the mixed-path sums alongside.
//  * R = float, the mixed path: FP64 geometry, FP32 table arithmetic
//    (pa_U_mixed), each term two-sum accumulated into FP64, and eb, a bound
//    on |sums - FP64 sums| (kMixedErr times the terms' magnitudes, plus the
//    FP32 phases of the long-range part); SHADOW adds the FP64 sums.
// dg: this level's diagonal (y, d2y) pairs in R (DavidPA), dgs: the same in
// the other precision.
struct StageSums {
  double so, sn, eb, so2, sn2;
};

// One in-fit tricubic term of a pass, listed per warp for its team.
struct TriTerm {
  double u[3];
  int code;  // cell << 1 | copy (1: NEW)
  int pad;
};
// Terms listed per warp and pass (three (item, copy) units per lane).
constexpr int kTriTermsPerWarp = 96;
// Shared memory of the lists: 16 warps.
constexpr unsigned kTriTermBytes = 16u * kTriTermsPerWarp * sizeof(TriTerm);

// The FP64 tricubic short-range sum of one stage over this CTA's items
// [beg, beg + items) (item = link * np + partner index), each item evaluated
// for the OLD and the NEW copy of the moved particle: 2 items (item, copy)
// units.  Per pass every evaluating warp takes an even share of at most 96
// consecutive units, three per lane (C2's 1022 level-0 units of a CTA in one
// pass).  A lane forms its units' geometry
// (DistDisp, q, z, s, the fit-region test, the cell) and adds the primitive
// fallback of the terms outside the fit itself, from the potential's (y, d2y)
// pairs in shared memory (pp; null: the global tables).  The terms inside the
// fit are listed in shared memory (tq: kTriTermsPerWarp per warp) and
// gathered by teams of 4 lanes (tricubic_team_part).  Sums into (so, sn);
// with SHADOW the mixed path's terms into (so2, sn2).
template <bool SHADOW>
__device__ __forceinline__ void tricubic_stage(const BisectionArgs &a, const double (*w_old)[3],
                                               const double (*w_new)[3], const double2 *pp, int lv, int slice1,
                                               int ptcl, int beg, int items, int etid, int ethreads,
                                               const int *plist, int np, TriTerm *tq, double &so, double &sn,
                                               double &so2, double &sn2) {
  constexpr int TS = 4, TPW = 32 / TS;
  const DevSystem &sys = a.sys;
  const DTricubic<double> &t64 = a.pa.t64;
  const int N = sys.N;
  const int skip = 1 << lv;
  const int lane = etid & 31, wi = etid >> 5, nw = ethreads >> 5;
  const int pt = lane & (TS - 1);
  TriTerm *E = tq + wi * kTriTermsPerWarp;
  const size_t lvl = (size_t)lv * t64.nq * t64.ny * t64.nt;
  const double *F = t64.U + lvl * 8;
  double beta = t64.smallest_beta;
  for (int i = 0; i < lv; i++) beta *= 2.0;
  beta = 0.5 * beta;
  const int U = 2 * items;
  const int P = (U + 3 * ethreads - 1) / (3 * ethreads);
  const int cw = P > 0 ? (U + P * nw - 1) / (P * nw) : 0;  // <= 96
  for (int p = 0; p < P; p++) {
    const int ws = (p * nw + wi) * cw, we = min(U, ws + cw);
    bool in[3];
    TriTerm tt[3];
#pragma unroll
    for (int s = 0; s < 3; s++) {
      const int u = ws + lane + 32 * s;
      in[s] = false;
      if (u < we) {
        const int it = beg + (u >> 1);
        const int isn = u & 1;
        const int link = it / np;
        const int j = it - link * np;
        const int p2 = plist ? plist[j] : (j < ptcl ? j : j + 1);
        const int r0 = link * skip;
        const double *pa_ = a.path + ((size_t)(slice1 + r0) * N + p2) * 3;
        const double *pb_ = a.path + ((size_t)(slice1 + r0 + skip) * N + p2) * 3;
        // L2-coherent loads: other CTAs write accepted windows during the launch.
        const double a2[3] = {__ldcg(pa_), __ldcg(pa_ + 1), __ldcg(pa_ + 2)};
        const double b2[3] = {__ldcg(pb_), __ldcg(pb_ + 1), __ldcg(pb_ + 2)};
        const double(*w)[3] = isn ? w_new : w_old;
        double dA[3], dB[3];
        dist_disp(w[r0], a2, w[r0 + skip], b2, sys, dA, dB);
        const LinkGeom<double> g = link_geom<double>(dA, dB);
        const TriPrep<double> pr = tricubic_prep<double>(t64, g.q, g.z, g.s2);
        if (pr.inside) {
          in[s] = true;
          tt[s].u[0] = pr.u[0];
          tt[s].u[1] = pr.u[1];
          tt[s].u[2] = pr.u[2];
          tt[s].code = (pr.cell << 1) | isn;
        } else {  // the primitive action 1/2 beta_l (V(r) + V(r'))
          const double v = pp ? pot_V_pairs(t64.pot_grid, pp, pr.r) + pot_V_pairs(t64.pot_grid, pp, pr.rp)
                              : pot_V(t64, pr.r) + pot_V(t64, pr.rp);
          (isn ? sn : so) += beta * v;
        }
        if (SHADOW) (isn ? sn2 : so2) += tricubic_pa_mixed(t64, a.pa.t32, g.q, g.z, g.s2, lv).v;
      }
    }
    // list the in-fit terms, then each team gathers every TPW-th of them
    const unsigned m0 = __ballot_sync(0xffffffffu, in[0]), m1 = __ballot_sync(0xffffffffu, in[1]);
    const unsigned m2 = __ballot_sync(0xffffffffu, in[2]);
    const unsigned below = (1u << lane) - 1u;
    const int n0 = __popc(m0), n1 = n0 + __popc(m1), n = n1 + __popc(m2);
    if (in[0]) E[__popc(m0 & below)] = tt[0];
    if (in[1]) E[n0 + __popc(m1 & below)] = tt[1];
    if (in[2]) E[n1 + __popc(m2 & below)] = tt[2];
    __syncwarp();
    for (int e = lane / TS; e < n; e += TPW) {
      const TriTerm T = E[e];
      ((T.code & 1) ? sn : so) += tricubic_team_part(F, t64, T.code >> 1, T.u, pt);
    }
    __syncwarp();
  }
}
// Bound on the error of one FP32 e^{ik.r}: the FP64 phase reduced to
// [-pi, pi] and rounded to FP32 (<= 2^-22) and sincosf (2 ulp), doubled.
constexpr double kCisErr = 2.0e-6;

template <int KIND, typename R, bool SHADOW>
__device__ __forceinline__ StageSums stage_sums(const BisectionArgs &a, const double (*w_old)[3],
                                                const double (*w_new)[3], const void *dg, const void *dgs, int lv,
                                                int slice1, int ptcl, unsigned rank, unsigned CL, int etid,
                                                int ethreads, const int *plist, int np, void *tq) {
  constexpr bool MIX = std::is_same<R, float>::value;
  const DevSystem &sys = a.sys;
  const int N = sys.N;
  const int span = 1 << a.num_levels;
  const int skip = 1 << lv;
  const int nlinks = span >> lv;
  const double2 *dg64 = reinterpret_cast<const double2 *>(MIX ? dgs : dg);
  const float2 *dg32 = reinterpret_cast<const float2 *>(MIX ? dg : dgs);
  // mb: sum of the terms' magnitudes m (FP32: a relative shortfall of
  // 2^-24 per addition is far inside the factor kMixedErr leaves spare)
  double so = 0.0, sn = 0.0, so2 = 0.0, sn2 = 0.0, eb = 0.0;
  float co = 0.0f, cn = 0.0f, mb = 0.0f;
  // one term of each copy: the run's precision into (so, sn), the other into the shadow
  auto add_terms = [&](const LinkGeom<double> &g, bool is_new, int part, int nparts) {
    if (MIX) {
      const MixedU t = pa_U_mixed<KIND>(a.pa, dg32, g, lv, part, nparts);
      two_sum_add(is_new ? sn : so, is_new ? cn : co, t.v);
      mb += t.m;
      if (SHADOW) (is_new ? sn2 : so2) += pa_U_part<double, KIND>(a.pa, dg64, g, lv, part, nparts);
    } else {
      (is_new ? sn : so) += pa_U_part<double, KIND>(a.pa, dg64, g, lv, part, nparts);
      if (SHADOW) (is_new ? sn2 : so2) += pa_U_mixed<KIND>(a.pa, dg32, g, lv, part, nparts).v;
    }
  };
  if (KIND == PA_TRICUBIC && !MIX && (lv == 0 || a.sr_higher)) {
    // ShortRangeClass::SingleAction over partners x links with PAtricubicFit
    // terms, by lane teams (tricubic_stage).  The FP64 path only: with FP32
    // nodes (32 bytes) a lane's own 8-node gather is faster on the B200 than
    // a 2-lane team's (4.13e9 vs 3.91e9 C2 evals/s), so the mixed path keeps
    // one lane per term.
    const int total = np * nlinks;
    const int chunk = (total + (int)CL - 1) / (int)CL;
    const int beg = chunk * (int)rank;
    const int end = min(total, beg + chunk);
    if constexpr (!MIX)
      tricubic_stage<SHADOW>(a, w_old, w_new, reinterpret_cast<const double2 *>(dg), lv, slice1, ptcl, beg,
                             max(0, end - beg), etid, ethreads, plist, np, reinterpret_cast<TriTerm *>(tq), so, sn,
                             so2, sn2);
  } else if (lv == 0 || a.sr_higher) {  // ShortRangeClass::SingleAction over partners x links
    // partners: all others (plist null, np = N - 1) or the moved particle's
    // neighbour list (np entries, ascending)
    const int total = np * nlinks;  // < 2^31: N <= 2^20, 2^L <= 64 (host-checked)
    const int chunk = (total + (int)CL - 1) / (int)CL;
    const int beg = chunk * (int)rank;
    const int end = min(total, beg + chunk);
    const double *path = a.path;
    const int items = max(0, end - beg);
    // Team size: when this CTA has fewer items than threads, T lanes share an
    // item — the OLD and the NEW copy on different lanes and, for the tricubic
    // fit, the four (x,y) node pairs split over the rest — which shortens the
    // dependent chain of each lane.  T = 1 keeps one lane per item.
    int T = 1;
    const int tmax = KIND == PA_TRICUBIC ? 8 : 2;
    while (T < tmax && items * T * 2 <= ethreads) T *= 2;
    // When the items outnumber the threads but not twice over, a thread with
    // a second item would evaluate four terms while most evaluate two; as
    // (item, copy) units each thread evaluates at most ceil(2 items / threads)
    // terms (the partner is then read once per copy).
    const int per_item = 2 * ((items + ethreads - 1) / ethreads), per_unit = (2 * items + ethreads - 1) / ethreads;
    if (T == 1 && per_unit < per_item) {
      const int units = 2 * items;
      for (int u0 = etid; u0 < units; u0 += 2 * ethreads) {
        double a2[2][3], b2[2][3];
        int r0s[2];
        bool live[2], isn[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
          const int uu = u0 + u * ethreads;
          live[u] = uu < units;
          const int iu = live[u] ? uu : u0;
          isn[u] = iu >= items;  // units [0, items) are the OLD copies, [items, 2 items) the NEW
          const int it = beg + (isn[u] ? iu - items : iu);
          const int link = it / np;
          const int j = it - link * np;
          const int p2 = plist ? plist[j] : (j < ptcl ? j : j + 1);
          r0s[u] = link * skip;
          const double *pa_ = path + ((size_t)(slice1 + r0s[u]) * N + p2) * 3;
          const double *pb_ = path + ((size_t)(slice1 + r0s[u] + skip) * N + p2) * 3;
          for (int i = 0; i < 3; i++) {
            a2[u][i] = __ldcg(pa_ + i);
            b2[u][i] = __ldcg(pb_ + i);
          }
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
          if (!live[u]) continue;
          const int r0 = r0s[u];
          const double(*w)[3] = isn[u] ? w_new : w_old;
          double dA[3], dB[3];
          dist_disp(w[r0], a2[u], w[r0 + skip], b2[u], sys, dA, dB);
          add_terms(link_geom<double>(dA, dB), isn[u], 0, 1);
        }
      }
    } else if (T == 1) {
      // Two items per pass so a thread's partner and table loads overlap.
      // Item it is (link, j) = (it / np, it % np); both pass items advance
      // by the same stride, so (link, j) is carried instead of divided.
      const int stride = 2 * ethreads;
      const int qs = stride / np, rs = stride - qs * np;
      int lk[2], jj[2];
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const int it = beg + etid + u * ethreads;
        lk[u] = it / np;
        jj[u] = it - lk[u] * np;
      }
      for (int it0 = beg + etid; it0 < end; it0 += stride) {
        double a2[2][3], b2[2][3];
        int r0s[2];
        bool live[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
          const int it = it0 + u * ethreads;
          live[u] = it < end;
          const int link = live[u] ? lk[u] : lk[0];
          const int j = live[u] ? jj[u] : jj[0];
          const int p2 = plist ? plist[j] : (j < ptcl ? j : j + 1);
          r0s[u] = link * skip;
          const double *pa_ = path + ((size_t)(slice1 + r0s[u]) * N + p2) * 3;
          const double *pb_ = path + ((size_t)(slice1 + r0s[u] + skip) * N + p2) * 3;
          // L2-coherent loads: other CTAs write accepted windows during the launch.
          for (int i = 0; i < 3; i++) {
            a2[u][i] = __ldcg(pa_ + i);
            b2[u][i] = __ldcg(pb_ + i);
          }
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
          jj[u] += rs;
          lk[u] += qs;
          if (jj[u] >= np) {
            jj[u] -= np;
            lk[u]++;
          }
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
          if (!live[u]) continue;
          const int r0 = r0s[u];
          double dAo[3], dBo[3], dAn[3], dBn[3];
          dist_disp(w_old[r0], a2[u], w_old[r0 + skip], b2[u], sys, dAo, dBo);
          dist_disp(w_new[r0], a2[u], w_new[r0 + skip], b2[u], sys, dAn, dBn);
          add_terms(link_geom<double>(dAo, dBo), false, 0, 1);
          add_terms(link_geom<double>(dAn, dBn), true, 0, 1);
        }
      }
    } else {
      const int member = etid % T, team = etid / T, nteams = ethreads / T;
      const bool is_new = (member & 1) != 0;
      const int nparts = T >> 1, part = member >> 1;
      const double(*w)[3] = is_new ? w_new : w_old;
      for (int it = beg + team; it < end; it += nteams) {
        const int link = it / np;
        const int j = it - link * np;
        const int p2 = plist ? plist[j] : (j < ptcl ? j : j + 1);
        const int r0 = link * skip;
        const double *pa_ = path + ((size_t)(slice1 + r0) * N + p2) * 3;
        const double *pb_ = path + ((size_t)(slice1 + r0 + skip) * N + p2) * 3;
        const double a2[3] = {__ldcg(pa_), __ldcg(pa_ + 1), __ldcg(pa_ + 2)};
        const double b2[3] = {__ldcg(pb_), __ldcg(pb_ + 1), __ldcg(pb_ + 2)};
        double dA[3], dB[3];
        dist_disp(w[r0], a2, w[r0 + skip], b2, sys, dA, dB);
        add_terms(link_geom<double>(dA, dB), is_new, part, nparts);
      }
    }
  }
  if (a.use_lr && lv == 0) {
    // LongRangeClass::SingleAction (LongRangeClass.cc:273-371) over the
    // window's slices [slice1, slice1 + 2^L] with weight 1/2 at both ends:
    // sum_k Ulong_k |rho_k|^2 of the OLD and of the updated NEW rho_k.  The
    // Madelung and background terms are the same in both and cancel in dS.
    const int nk = a.nk;
    const int total = (span + 1) * nk;
    const int chunk = (total + (int)CL - 1) / (int)CL;
    const int beg = chunk * (int)rank;
    const int end = min(total, beg + chunk);
    for (int it = beg + etid; it < end; it += ethreads) {
      const int rel = it / nk, k = it - rel * nk;
      const double f = (rel == 0 || rel == span) ? 0.5 : 1.0;
      const double2 ro = __ldcg(&a.rhok[(size_t)(slice1 + rel) * nk + k]);
      const double *kv = a.kvec + 3 * k;
      const double u = __ldg(&a.ulong_k0[k]);
      const double2 rn = rho_new_k<R>(ro, kv, w_new[rel], w_old[rel]);
      const double o2 = ro.x * ro.x + ro.y * ro.y, n2 = rn.x * rn.x + rn.y * rn.y;
      if (MIX) {
        two_sum_add(so, co, f * o2 * u);
        two_sum_add(sn, cn, f * n2 * u);
        // |rho_new - its FP64 value| <= 2 kCisErr (one new and one old phase)
        const double dr = 2.0 * kCisErr;
        eb += f * fabs(u) * (2.0 * sqrt(n2) * dr + dr * dr);
      } else {
        so += f * o2 * u;
        sn += f * n2 * u;
      }
      if (SHADOW) {
        const double2 rs = rho_new_k<typename std::conditional<MIX, double, float>::type>(ro, kv, w_new[rel],
                                                                                            w_old[rel]);
        so2 += f * o2 * u;
        sn2 += f * (rs.x * rs.x + rs.y * rs.y) * u;
      }
    }
  }
  StageSums r;
  r.so = so + (double)co;
  r.sn = sn + (double)cn;
  r.eb = eb + kMixedErr * (1.0 + 1e-5) * (double)mb;
  r.so2 = so2;
  r.sn2 = sn2;
  return r;
}

// KineticClass::SingleAction (KineticClass.cc:33-90) of the moved particle's
// links at one level, OLD and NEW, by one full warp (a link per lane, a
// fixed shuffle tree), FP64 on both paths.  The sampler warp computes it
// while the other warps evaluate the pair terms, so no evaluating thread
// starts its partner loads late.  The sums are identical in every lane.
__device__ __forceinline__ double2 kinetic_sums(const double (*w_old)[3], const double (*w_new)[3], int num_levels,
                                                int lv, const DevSystem &sys, int lane) {
  double so = 0.0, sn = 0.0;
  if (sys.lambda != 0.0) {
    const int skip = 1 << lv;
    const int nlinks = (1 << num_levels) >> lv;
    const double levelTau = sys.tau * (1 << lv);
    const double F = 1.0 / (4.0 * sys.lambda * levelTau);
    for (int k = lane; k < nlinks; k += 32) {
      double vo[3], vn[3];
      for (int i = 0; i < 3; i++) {
        vo[i] = w_old[k * skip + skip][i] - w_old[k * skip][i];
        vn[i] = w_new[k * skip + skip][i] - w_new[k * skip][i];
      }
      put_in_box(vo, sys);
      put_in_box(vn, sys);
      so += kinetic_link(vo, F, sys.num_images, sys);
      sn += kinetic_link(vn, F, sys.num_images, sys);
    }
  }
  return make_double2(warp_sum_n(so, (1 << num_levels) >> lv), warp_sum_n(sn, (1 << num_levels) >> lv));
}

// The mixed path's FP64 re-evaluation of a stage (and, with need_prev, of the
// stage before it, at level + 1 with its partner set): the FP64 path's
// stage_sums with its item split, so the sums are the FP64 path's bit for
// bit.  Returns (S_old, S_new, previous S_old, previous S_new) of this CTA.
template <int KIND>
__device__ __forceinline__ double4 stage_sums_reeval(const BisectionArgs &a, const double (*w_old)[3],
                                                     const double (*w_new)[3], int lv, int slice1, int ptcl,
                                                     unsigned rank, unsigned CL, int etid, int ethreads,
                                                     const int *plist, int np, int need_prev,
                                                     const int *prev_plist, int prev_np, void *tq) {
  const DDavid<double> &d64 = a.pa.d64;
  auto dgl = [&](int l) -> const void * {
    return KIND == PA_DAVID ? reinterpret_cast<const double2 *>(d64.diag) + (size_t)(d64.tau_pos + l) * d64.diag_stride
                            : nullptr;
  };
  double4 r = make_double4(0.0, 0.0, 0.0, 0.0);
  for (int k = 0; k < 1 + need_prev; k++) {  // one loop body: the FP64 evaluation is inlined once
    const int l = lv + k;
    const StageSums v = stage_sums<KIND, double, false>(a, w_old, w_new, dgl(l), nullptr, l, slice1, ptcl, rank, CL,
                                                        etid, ethreads, k ? prev_plist : plist, k ? prev_np : np, tq);
    if (k) {
      r.z = v.so;
      r.w = v.sn;
    } else {
      r.x = v.so;
      r.y = v.sn;
    }
  }
  return r;
}

// Committed or speculative position of a chain's Local stream.
struct RngSnap {
  unsigned long long n;
  int one_left;
  double x2;
};

__device__ __forceinline__ DevRandom rng_from(const RngSnap &s, uint64_t seed, uint32_t stream,
                                              const RngTab *tab) {
  DevRandom r;
  r.tab = tab;
  r.seed = seed;
  r.stream = stream;
  r.n = s.n;
  r.one_left = s.one_left;
  r.x2 = s.x2;
  return r;
}
__device__ __forceinline__ void rng_store(RngSnap &s, const DevRandom &r) {
  s.n = r.n;
  s.one_left = r.one_left;
  s.x2 = r.x2;
}

// KIND: pair-action type; R: precision of the pair terms; SHADOW: also
// evaluate the pair terms in the other precision for the dS error.
//
// Two sampler warps own the Local stream; the committed stream position
// lives in shared memory.  While the other warps evaluate the OLD and NEW
// action of stage l:
//  * the level sampler (the last warp) speculatively samples level l-1 from
//    the position that follows stage l's acceptance draw — committed if
//    stage l accepts and the move goes on;
//  * the move speculator (the warp before it) draws the next move's slice
//    window and particle from the same position, loads that particle's
//    window into the spare buffer and samples its top level — committed if
//    the move ends at this stage (a rejection, or acceptance at level 0),
//    unless the accepted particle was drawn again, whose window changes.
// The draw order is therefore exactly the reference's.
// Neighbour-list entries of the moved particle staged in shared memory per
// move (longer lists are read from global memory).
constexpr int kNbrStage = 1024;

// Values reduced over a cluster per stage: S_old, S_new, the mixed bound and
// the two shadow sums.
constexpr int kRed = 5;

// Shared state of one CTA while it runs a job.
struct KernelShared {
  double win_old[2][kMaxWindow][3], win_new[2][kMaxWindow][3];
  double gbuf[2][3 * 32];
  double sh_red[16][kRed];  // per warp: S_old, S_new, the mixed bound, the shadows
  double xchg[2][kMaxCluster][kRed];
  double s_logsr[kMaxLevels], s_logu[kMaxLevels];
  int s_ctl[4];   // slice1, ptcl, stage accepted, status
  int s_next[4];  // next move speculated: valid, slice1, ptcl
  double s_next_f[2];
  RngSnap s_rng, s_spec1, s_spec2;
  int s_ok;
  RngTab tab;
  // neighbour lists: bounding sphere of the moved particle (and of the
  // speculated next one), whether a NEW position of the current stage lies
  // outside it, and whether this job evaluates all partners from now on
  double4 s_cb, s_next_cb;
  int s_far, s_next_far, s_allpairs;
  // concurrent proposals: the stream position at the start of this slot's
  // move (restored when the move is redone), the outcome every slot of the
  // window published for the in-order commit, and the commit's verdict
  RngSnap s_rng0;
  int4 s_pub[kMaxCluster];
  int s_redo[kMaxCluster], s_redo_local;
  int s_commit[4];  // first slot to redo, stop, any committed move left its sphere
  int s_need[2];    // mixed path: re-evaluate this stage in FP64; also the previous stage
  uint64_t test_bar;  // an mbarrier nothing arrives at (the give-up test of the staging wait)
  // Stage reduction across the cluster: per parity an mbarrier that completes
  // when every CTA's partials have landed in xchg[parity] (st.async).
  uint64_t red_bar[2];
};
// Tries of the wait for a stage reduction's partials before PIMC_E_CAP.
constexpr int kRedWaitCap = 1 << 24;

// Whether any of the window's span+1 NEW positions lies outside the moved
// particle's bounding sphere cb (minimum image), by one warp.
__device__ __forceinline__ int window_outside(const double (*w)[3], int span, double4 cb, const DevSystem &sys,
                                              int lane) {
  int out = 0;
  for (int rel = lane; rel <= span; rel += 32) {
    double d[3] = {w[rel][0] - cb.x, w[rel][1] - cb.y, w[rel][2] - cb.z};
    double r2 = 0.0;
    for (int i = 0; i < 3; i++) {
      const double n = rint(d[i] * sys.boxinv[i]);
      d[i] -= n * sys.box[i];
      r2 += d[i] * d[i];
    }
    out |= r2 > cb.w * cb.w;
  }
  return __any_sync(0xffffffffu, out);
}

// Whether a DavidPA pair term of the windows a and b can be nonzero: some
// slice of the window where one of a's OLD/NEW positions and one of b's
// OLD/NEW positions are closer than `range` (minimum image), by one warp.  A
// DavidPA table is zero from its grid end on, and DistDisp's second distance
// is never below the minimum image, so beyond it every link term is zero.
__device__ __forceinline__ bool windows_near(const double (*ao)[3], const double (*an)[3], const double (*bo)[3],
                                             const double (*bn)[3], int span, double range, const DevSystem &sys,
                                             int lane) {
  bool hit = false;
  const double r2 = range * range;
  for (int rel = lane; rel <= span; rel += 32) {
    const double *A[2] = {ao[rel], an[rel]}, *B[2] = {bo[rel], bn[rel]};
    for (int x = 0; x < 2; x++)
      for (int y = 0; y < 2; y++) {
        double d2 = 0.0;
        for (int i = 0; i < 3; i++) {
          double d = A[x][i] - B[y][i];
          d -= rint(d * sys.boxinv[i]) * sys.box[i];
          d2 += d * d;
        }
        hit |= d2 < r2;
      }
  }
  return __any_sync(0xffffffffu, hit);
}

// Storage of the precomputed stream tables of a CTA: NF parts of kTabFine
// positions; a group uses a contiguous run of parts.
constexpr int kTabFine = 256;
template <int NF>
struct RngStore {
  double u[NF * (kTabFine + 2)];
  double lu[NF * kTabFine], x1[NF * kTabFine], x2[NF * kTabFine];
  unsigned char acc[NF * kTabFine];
  template <int NF2>
  __device__ __forceinline__ RngTab part(int first, int count) {
    RngTab t;
    t.u = u + first * (kTabFine + 2);
    t.lu = lu + first * kTabFine;
    t.x1 = x1 + first * kTabFine;
    t.x2 = x2 + first * kTabFine;
    t.acc = acc + first * kTabFine;
    t.tb = 0;
    t.W = count * kTabFine;
    return t;
  }
};

// The threads that run one job: a warp-aligned contiguous range of the CTA
// synchronised by its own named barrier (the whole CTA, or a part of it when
// a CTA runs several small chains side by side).
struct Group {
  int tid;       // thread index within the group
  int size;      // threads in the group, a multiple of 32
  unsigned bar;  // named barrier id
  __device__ __forceinline__ void sync() const {
    asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(size) : "memory");
  }
};

// The moves of one job — one chain, or one window of a chain — on this CTA
// (cluster rank `rank` of `CL`).  `phase` is the parity of the table-staging
// mbarrier `bar`, flipped once per staging.
template <int KIND, typename R, bool SHADOW, bool OUTLINE, bool PROP = false>
__device__ void run_job(const BisectionArgs &a, ChainState *cs, int window, unsigned rank, unsigned CL,
                        cg::cluster_group &cluster, const Group &G, unsigned char *dyn, unsigned dyn_cap,
                        KernelShared &S, uint64_t *bar_ptr, unsigned &phase, const RngTab &tab_mem,
                        int *s_nbr = nullptr) {
  typedef typename Pair2<R>::T P2;
  typedef typename std::conditional<std::is_same<R, double>::value, float, double>::type RS;  // shadow precision
  typedef typename Pair2<RS>::T P2S;
  auto &win_old = S.win_old;
  auto &win_new = S.win_new;
  auto &gbuf = S.gbuf;
  auto &sh_red = S.sh_red;
  auto &xchg = S.xchg;
  auto &s_logsr = S.s_logsr;
  auto &s_logu = S.s_logu;
  auto &s_ctl = S.s_ctl;
  auto &s_next = S.s_next;
  auto &s_next_f = S.s_next_f;
  auto &s_rng = S.s_rng;
  auto &s_spec1 = S.s_spec1;
  auto &s_spec2 = S.s_spec2;
  uint64_t &s_bar = *bar_ptr;
  const int tid = G.tid;
  const int lane = tid & 31, warp = tid >> 5;
  const int nwarps = G.size >> 5;
  const int sampler = nwarps - 1;
  // Concurrent proposals: each CTA of the window's cluster is one proposal
  // slot and evaluates its moves alone (evaluation rank 0 of 1); the cluster
  // only meets to commit the slots' moves in order.
  constexpr bool prop = PROP;
  const unsigned erank = prop ? 0u : rank, ECL = prop ? 1u : CL;
  // next-move speculator (needs >= 4 warps; not with proposals, whose next
  // move may start from a window another slot is about to write)
  const int specwarp = (nwarps >= 4 && !prop) ? nwarps - 2 : -1;
  const int ethreads = (nwarps - (specwarp >= 0 ? 2 : 1)) * 32;  // evaluating threads: warps below the samplers
  // The moved particle's kinetic links: with 8 or more evaluating warps the
  // last of them sums them after its pair terms (the item split leaves it the
  // fewest), so the level sampler's warp only samples; otherwise the sampler.
  const int kinwarp = (ethreads >> 5) >= 8 ? (ethreads >> 5) - 1 : -1;
  const bool evaluator = tid < ethreads;
  const DevSystem &sys = a.sys;
  const int N = sys.N;
  const int L = a.num_levels;
  const int span = 1 << L;
  const bool lead = (erank == 0 && tid == 0);

  // ---- stage 1-D tables into shared memory (bulk TMA) ----
  // DavidPA: the diagonal columns of every level, each diag_stride pairs
  // long, padded so every level and every copy is a multiple of 16 bytes.
  // Tricubic: the potential's (y, d2y) pairs of the primitive fallback when
  // they fit beside the per-warp term lists (kTriTermBytes, after the tables).
  // The wait is bounded; the cluster then agrees on the outcome so every CTA
  // takes the same path.
  const P2 *diag_smem = nullptr;
  const P2S *diag_smem_s = nullptr;
  const void *stage_src = nullptr, *stage_src_s = nullptr;
  unsigned bytes = 0, bytes_s = 0, tail = 0;
  if (KIND == PA_DAVID) {
    const DDavid<R> &d = david_of<R>(a.pa);
    bytes = (unsigned)(L * d.diag_stride * sizeof(P2));
    stage_src = reinterpret_cast<const P2 *>(d.diag) + (size_t)d.tau_pos * d.diag_stride;
    if (SHADOW) {
      const DDavid<RS> &ds = david_of<RS>(a.pa);
      bytes_s = (unsigned)(L * ds.diag_stride * sizeof(P2S));
      stage_src_s = reinterpret_cast<const P2S *>(ds.diag) + (size_t)ds.tau_pos * ds.diag_stride;
    }
  } else if (KIND == PA_TRICUBIC) {
    // the FP64 path's team stage (the mixed path's one-lane terms read the
    // global tables; its FP64 re-evaluation too)
    tail = kTriTermBytes;
    const unsigned b0 = (unsigned)(a.pa.t64.pot_pairs_n * sizeof(double2));
    if (!std::is_same<R, float>::value && b0 + tail <= dyn_cap) {
      bytes = b0;
      stage_src = a.pa.t64.pot_pairs;
    }
  }
  void *tq = dyn + ((bytes + bytes_s + 15u) & ~15u);
  if (bytes + bytes_s + tail > dyn_cap) {  // uniform over the cluster: same job, same launch
    if (lead) atomicExch(&cs->status, PIMC_E_CAP);
    return;
  }
  const bool staged = bytes > 0;
  if (staged) {
    G.sync();  // the previous job's readers of the staged tables are done
    if (tid == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&s_bar, bytes + bytes_s);
      bulk_g2s(dyn, stage_src, bytes, &s_bar);
      if (SHADOW && bytes_s) bulk_g2s(dyn + bytes, stage_src_s, bytes_s, &s_bar);
    }
    G.sync();
    // Bounded wait for the copy; with test_wait, a further bounded wait on a
    // barrier that nothing arrives at once the copy has landed, which always
    // runs out and takes the give-up path below.
    const int cap = a.wait_cap > 0 ? a.wait_cap : (1 << 22);
    int landed = 0;
    for (int it = 0; it < cap; it++)
      if (mbar_try_wait(&s_bar, phase)) {
        landed = 1;
        break;
      }
    int ok = landed;
    if (ok && a.test_wait > 0) {
      ok = 0;
      for (int it = 0; it < a.test_wait; it++)
        if (mbar_try_wait(&S.test_bar, 0)) {
          ok = 1;
          break;
        }
    }
    if (tid == 0) S.s_ok = 1;
    G.sync();
    if (!ok) S.s_ok = 0;
    G.sync();
    ok = S.s_ok;
    int all_ok = ok;
    if (CL > 1) {
      if (tid < (int)CL) cluster.map_shared_rank(&xchg[1][rank][0], tid)[0] = ok ? 1.0 : 0.0;
      cluster.sync();
      for (unsigned r = 0; r < CL; r++) all_ok &= (xchg[1][r][0] != 0.0);
    }
    if (!all_ok) {
      // Let a late copy land (bounded) before this CTA moves on or exits:
      // shared memory must not be left with a copy in flight.
      for (int it = 0; it < (1 << 22) && !landed; it++) landed = mbar_try_wait(&s_bar, phase);
      if (lead) atomicExch(&cs->status, PIMC_E_CAP);
      if (CL > 1) cluster.sync();
      phase ^= 1u;
      return;
    }
    phase ^= 1u;
    diag_smem = reinterpret_cast<const P2 *>(dyn);
    if (SHADOW && bytes_s) diag_smem_s = reinterpret_cast<const P2S *>(dyn + bytes);
  }

  const uint64_t seed = cs->seed;
  const uint32_t stream = cs->stream;
  if (tid == 0) {
    s_rng.n = cs->nlocal;
    s_rng.one_left = cs->one_left;
    s_rng.x2 = cs->x2;
    s_ctl[3] = 0;
    s_next[0] = 0;
    S.s_far = 0;
    S.s_allpairs = 0;
    S.tab = tab_mem;
    S.tab.W = 0;  // filled below
  }
  unsigned long long moves = 0, accepted = 0, stages = 0, pair_evals = 0, flips = 0, redone = 0, reevals = 0;
  int status = 0;
  double *path = a.path;
  unsigned xc = 0;  // exchange parity counter

  // Window of this cluster in the concurrent schedule.
  int slice1 = 0;
  if (a.concurrent) {
    const int o = (int)floor(philox_uniform(seed, kStreamCommon, a.round) * span);
    slice1 = o + window * span;
    if (slice1 + span > sys.S - 1) {
      // Inactive this round (uniform over the cluster): mark its trace slots.
      if (a.trace && lead)
        for (int st = 0; st < a.steps_per_block; st++) {
          pimc_move_record r = {};
          r.slice1 = -1;
          r.ptcl = -1;
          const long long at = (long long)window * a.steps_per_block + st;
          a.trace[a.trace_offset + (prop ? at * a.proposals + rank : at)] = r;
        }
      if (staged && CL > 1) cluster.sync();  // xchg[1] no longer read by peers
      return;
    }
  }
  if (staged && CL > 1) cluster.sync();  // every CTA has read xchg[1]
  // Stage reductions over a cluster: each CTA's red_bar[p] expects the
  // partials of every CTA (kRed doubles each) for its next use; the first
  // uses are posted before the cluster barrier, so before any peer can send.
  const unsigned red_bytes = CL * kRed * (unsigned)sizeof(double);
  unsigned rph = 0;  // phase parity of red_bar[0] (bit 0) and red_bar[1] (bit 1)
  if (ECL > 1) {
    if (tid == 0) {
      mbar_expect_tx(&S.red_bar[0], red_bytes);
      mbar_expect_tx(&S.red_bar[1], red_bytes);
    }
    cluster.sync();
  }
  G.sync();
  auto gsync = [&]() { G.sync(); };
  rng_tab_fill(S.tab, tab_mem.W, seed, stream, s_rng.n, tid, G.size, gsync);
  const int numLeft = sys.S - span;
  const int total_moves = (a.concurrent ? 1 : a.n_blocks) * a.steps_per_block;
  int cur = 0;
  bool have_next = false;
  // Concurrent proposals.  Step `pstep` of the round is slot 0, 1, ..., P-1
  // of the window each making one move from its own Local stream, with the
  // result of making them in that order.  A pass runs slots pfirst..P-1 at
  // once on the positions at the start of the pass; then, in slot order, a
  // slot's move is kept unless an earlier slot of the pass accepted a move
  // of a particle the slot's sums read (or of the slot's own particle).  The
  // first slot that fails this is redone, with the slots after it, in the
  // next pass from the positions the kept moves wrote and from its stream
  // position at the start of the move.
  const int P = prop ? a.proposals : 1;
  int pstep = 0, pfirst = 0;

  for (int m = 0; prop ? pstep < a.steps_per_block : m < total_moves; m++) {
    const int blk = prop ? 0 : m / a.steps_per_block, step = prop ? pstep : m - blk * a.steps_per_block;
    const bool active = !prop || (int)rank >= pfirst;
    // this move's work: counted at once, or with proposals when the move is kept
    unsigned long long mv_stages = 0, mv_pairs = 0, mv_flips = 0, mv_reevals = 0;
    unsigned long long &c_stages = PROP ? mv_stages : stages, &c_pairs = PROP ? mv_pairs : pair_evals,
                       &c_flips = PROP ? mv_flips : flips, &c_reevals = PROP ? mv_reevals : reevals;
    bool acc_all = true;
    int move_far = 0;  // some stage of this move sampled outside the moved particle's sphere
    int mptcl = 0;     // the moved particle
    pimc_move_record rec;
    if (active) {
      if (!have_next) {
        // ChooseTimeSlices (BisectionBlock.cc:362-374), ChooseParticle (NoPermuteClass.cc:61-68)
        if (warp == sampler) {
          DevRandom rng = rng_from(s_rng, seed, stream, &S.tab);
          if (!a.concurrent && step == 0) slice1 = rng.LocalInt(numLeft);
          const int p = rng.LocalInt(N);
          __syncwarp();
          if (lane == 0) {
            if (prop) S.s_rng0 = s_rng;
            s_ctl[0] = slice1;
            s_ctl[1] = p;
            rng_store(s_rng, rng);
          }
        }
        G.sync();
        slice1 = s_ctl[0];
        const int p = s_ctl[1];
        for (int rel = tid; rel <= span; rel += G.size) {
          const double *q = path + ((size_t)(slice1 + rel) * N + p) * 3;
          for (int i = 0; i < 3; i++) win_old[cur][rel][i] = win_new[cur][rel][i] = __ldcg(q + i);
        }
        G.sync();
        if (warp == sampler) {
          DevRandom rng = rng_from(s_rng, seed, stream, &S.tab);
          const double lsr = sample_level<OUTLINE>(win_old[cur], win_new[cur], gbuf[0], L, L - 1, sys, rng, lane);
          const double lu = rng.LocalLog();
          int far = 0;
          double4 cb = make_double4(0.0, 0.0, 0.0, 0.0);
          if (a.nbr_on) {
            cb = a.nbr_cb[s_ctl[1]];
            __syncwarp();
            far = window_outside(win_new[cur], span, cb, sys, lane);
          }
          __syncwarp();
          if (lane == 0) {
            s_logsr[L - 1] = lsr;
            s_logu[L - 1] = lu;
            rng_store(s_rng, rng);
            S.s_cb = cb;
            S.s_far = far;
          }
        }
        G.sync();
      }
      slice1 = s_ctl[0];
      const int ptcl = s_ctl[1];
      mptcl = ptcl;
      const bool more = m + 1 < total_moves;
      const bool next_new_block = !a.concurrent && ((m + 1) % a.steps_per_block == 0);
      double(*w_old)[3] = win_old[cur];
      double(*w_new)[3] = win_new[cur];
      // Neighbour lists: the moved particle's list (fixed for the launch) in
      // shared memory for the whole move, so a stage's item loop starts with
      // the partner loads instead of two dependent reads of the list.
      int mv_cnt = -1;
      if (a.nbr_on && s_nbr) {
        const int cnt = __ldcg(&a.nbr_cnt[ptcl]);
        if (cnt >= 0 && cnt <= kNbrStage) {
          const int *src = a.nbr_idx + (size_t)ptcl * a.nbr_kmax;
          for (int i = tid; i < cnt; i += G.size) s_nbr[i] = __ldcg(src + i);
          mv_cnt = cnt;
        }
        G.sync();
      }

      // prevDS: the previous stage's dS as the decision used it; prevE: a
      // bound on its error against the FP64 sums (0 when it is FP64's)
      double prevDS = 0.0, prevDS_s = 0.0, prevE = 0.0;
      int prev_np = 0;
      const int *prev_plist = nullptr;
      int passed = 0;
      if (lead) {
        rec.slice1 = slice1;
        rec.ptcl = ptcl;
        for (int i = 0; i < 8; i++) {
          rec.dS[i] = rec.dS_shadow[i] = 0.0;
          rec.dS_bound[i] = 0.0f;
        }
        rec.reevaluated = 0;
        rec.pad = 0;
      }
      int si = 0;
      for (int level = L - 1; level >= 0; level--, si++) {
        // ---- LocalStageClass::Attempt (StageClass.cc:49-95) ----
        // Partners: the moved particle's neighbour list while its NEW positions
        // stay inside its sphere and no earlier move of this job left one;
        // otherwise all particles (the same sum: pairs beyond the table's end
        // add exact zeros).
        const int far = S.s_far;
        move_far |= far;
        int np = N - 1;
        const int *plist = nullptr;
        if (a.nbr_on && !far && !S.s_allpairs) {
          if (mv_cnt >= 0) {
            np = mv_cnt;
            plist = s_nbr;
          } else {
            const int cnt = __ldcg(&a.nbr_cnt[ptcl]);
            if (cnt >= 0) {
              np = cnt;
              plist = a.nbr_idx + (size_t)ptcl * a.nbr_kmax;
            }
          }
        }
        if (evaluator) {
          const size_t st = KIND == PA_DAVID ? (size_t)david_of<R>(a.pa).diag_stride : 0;
          const size_t sts = (KIND == PA_DAVID && SHADOW) ? (size_t)david_of<RS>(a.pa).diag_stride : 0;
          const StageSums v = stage_sums<KIND, R, SHADOW>(a, w_old, w_new, diag_smem ? diag_smem + level * st : nullptr,
                                                          diag_smem_s ? diag_smem_s + level * sts : nullptr, level,
                                                          slice1, ptcl, erank, ECL, tid, ethreads, plist, np, tq);
          double r0 = warp_sum(v.so), r1 = warp_sum(v.sn);
          const double r2 = warp_sum(v.eb);
          double r3 = SHADOW ? warp_sum(v.so2) : 0.0, r4 = SHADOW ? warp_sum(v.sn2) : 0.0;
          if (warp == kinwarp && erank == 0) {
            // the moved particle's kinetic links, once per evaluation group
            const double2 k = kinetic_sums(w_old, w_new, L, level, sys, lane);
            r0 += k.x;
            r1 += k.y;
            r3 += k.x;
            r4 += k.y;
          }
          if (lane == 0) {
            sh_red[warp][0] = r0;
            sh_red[warp][1] = r1;
            sh_red[warp][2] = r2;
            sh_red[warp][3] = r3;
            sh_red[warp][4] = r4;
          }
        } else {
          if (warp == sampler && level > 0) {
            // speculative sampling of the next level (BisectionStage::Sample of stage level-1)
            DevRandom spec = rng_from(s_rng, seed, stream, &S.tab);
            const double lsr = sample_level<OUTLINE>(w_old, w_new, gbuf[0], L, level - 1, sys, spec, lane);
            const double lu = spec.LocalLog();
            __syncwarp();
            if (lane == 0) {
              s_logsr[level - 1] = lsr;
              s_logu[level - 1] = lu;
              rng_store(s_spec1, spec);
            }
          }
          if (warp == specwarp && more) {
            // speculative start of the next move, as if this move ends here
            DevRandom spec = rng_from(s_rng, seed, stream, &S.tab);
            const int ns1 = next_new_block ? spec.LocalInt(numLeft) : slice1;
            const int np_ = spec.LocalInt(N);
            // the bounding sphere's load goes out with the window's
            const double4 cb = a.nbr_on ? a.nbr_cb[np_] : make_double4(0.0, 0.0, 0.0, 0.0);
            double(*wo)[3] = win_old[cur ^ 1];
            double(*wn)[3] = win_new[cur ^ 1];
            for (int rel = lane; rel <= span; rel += 32) {
              const double *q = path + ((size_t)(ns1 + rel) * N + np_) * 3;
              for (int i = 0; i < 3; i++) wo[rel][i] = wn[rel][i] = __ldcg(q + i);
            }
            __syncwarp();
            const double lsr = sample_level<OUTLINE>(wo, wn, gbuf[1], L, L - 1, sys, spec, lane);
            const double lu = spec.LocalLog();
            int far = 0;
            if (a.nbr_on) {
              __syncwarp();
              far = window_outside(wn, span, cb, sys, lane);
            }
            __syncwarp();
            if (lane == 0) {
              s_next[1] = ns1;
              s_next[2] = np_;
              s_next_f[0] = lsr;
              s_next_f[1] = lu;
              S.s_next_cb = cb;
              S.s_next_far = far;
              rng_store(s_spec2, spec);
            }
          }
          if (lane < kRed) sh_red[warp][lane] = 0.0;
          if (warp == sampler && erank == 0 && kinwarp < 0) {
            // the moved particle's kinetic links, once per evaluation group
            const double2 k = kinetic_sums(w_old, w_new, L, level, sys, lane);
            __syncwarp();
            if (lane == 0) {
              sh_red[warp][0] = k.x;
              sh_red[warp][1] = k.y;
              sh_red[warp][3] = k.x;
              sh_red[warp][4] = k.y;
            }
          }
        }
        // Counted as the reference performs them: OLD + NEW of the stage's links.
        if (lead && (level == 0 || a.sr_higher)) c_pairs += 2ull * (unsigned long long)np * (span >> level);
        G.sync();
        // ---- reduce: warps -> CTA (warp 0) -> cluster (DSMEM, rank order) ----
        // The sums are bitwise the same in every CTA of the cluster, so every
        // CTA takes the same decision (and the same re-evaluation request).
        auto reduce = [&]() -> double {
          const int par = xc & 1;
          xc++;
          double v = 0.0;
          if (warp != 0) return v;
          if (lane < kRed) {
            // all loads first, then a fixed pairwise tree (16 warps at most)
            double t[16];
#pragma unroll
            for (int w = 0; w < 16; w++) t[w] = w < nwarps ? sh_red[w][lane] : 0.0;
#pragma unroll
            for (int h = 8; h > 0; h >>= 1)
#pragma unroll
              for (int w = 0; w < h; w++) t[w] += t[w + h];
            v = t[0];
            if (ECL > 1) {
              // this CTA's partials into xchg[par][rank] of every CTA of the cluster
              const unsigned dst = smem_addr(&xchg[par][rank][lane]), bar = smem_addr(&S.red_bar[par]);
              for (unsigned r = 0; r < CL; r++) st_async_f64(mapa_u32(dst, r), v, mapa_u32(bar, r));
            } else {
              xchg[par][0][lane] = v;
            }
          }
          if (ECL > 1) {
            // Bounded wait for every CTA's partials.  A peer sends to this
            // buffer again only for the reduction after next, which needs
            // this CTA's next partials, so the next use is posted now.
            bool ok = false;
            for (int it = 0; it < kRedWaitCap && !ok; it++) ok = mbar_try_wait_cluster(&S.red_bar[par], (rph >> par) & 1u);
            rph ^= 1u << par;
            if (!ok) status = PIMC_E_CAP;
            __syncwarp();
            if (lane == 0) mbar_expect_tx(&S.red_bar[par], red_bytes);
          } else {
            __syncwarp();
          }
          v = 0.0;
          if (lane < kRed) {  // rank order, loads first
            double t[kMaxCluster];
#pragma unroll
            for (int r = 0; r < kMaxCluster; r++) t[r] = r < (int)ECL ? xchg[par][r][lane] : 0.0;
#pragma unroll
            for (int r = 0; r < kMaxCluster; r++) v += t[r];
          }
          return v;
        };
        // ---- Metropolis test, identical in every CTA (warp 0) ----
        // exact: so/sn are the FP64 sums (the FP64 path, or the mixed path's
        // re-evaluation).  Otherwise the mixed sums decide when the decision
        // cannot change within their bound E (the stage's bound, the previous
        // stage's, and 1e-12 of the sums for the FP64 path's own rounding);
        // when it could, warp 0 asks for the stage's FP64 re-evaluation (and
        // the previous stage's, if its dS was mixed) and decides on those.
        auto decide = [&](double so, double sn, double eb, double so2, double sn2, bool exact) {
          const double currActionChange = sn - so;
          const double logsr = s_logsr[level];
          const double logu = s_logu[level];
          if (!exact && a.guard) {
            const double logAcceptProb = logsr - currActionChange + prevDS;
            const double E = eb + prevE + 1e-12 * (fabs(so) + fabs(sn));
            // relative gate: |dS_mixed - dS_64| <= eb <= 1e-6 |dS_64| needs eb (1 + 1e-6) <= 1e-6 |dS_mixed|
            const bool rel_fail = a.guard == kGuardRelative && !(eb * (1.0 + 1e-6) <= 1e-6 * fabs(currActionChange));
            if ((rel_fail || !(fabs(logAcceptProb - logu) > E)) && isfinite(currActionChange)) {
              if (lane == 0) {
                S.s_need[0] = 1;
                S.s_need[1] = prevE > 0.0 ? 1 : 0;
              }
              if (lead && si < 8) {
                rec.dS[si] = currActionChange;
                rec.dS_bound[si] = (float)eb;
                rec.reevaluated |= 1 << si;
              }
              return;
            }
          }
          const double logAcceptProb = logsr - currActionChange + prevDS;
          bool toAccept = logAcceptProb >= logu;
          if (toAccept && (fabs(sn) > 1e50 || fabs(so) > 1e50)) {  // StageClass.cc:74-85
            toAccept = false;
            status = PIMC_E_STAGING;
          }
          if (!isfinite(currActionChange)) status = PIMC_E_NAN;
          if (SHADOW) {
            const double dss = sn2 - so2;
            const bool other = (logsr - dss + prevDS_s) >= logu;
            if (other != toAccept && lead) c_flips++;
            prevDS_s = dss;
            if (lead && si < 8) rec.dS_shadow[si] = dss;
          }
          prevDS = currActionChange;
          prevE = exact ? 0.0 : eb;
          if (lead && si < 8) {
            if (!exact || !(rec.reevaluated & (1 << si))) rec.dS[si] = currActionChange;
            if (!exact) rec.dS_bound[si] = (float)eb;
          }
          // commit the stream position the outcome selects
          const bool ends = !toAccept || level == 0 || status != 0;
          // neighbour lists: whether the next stage's NEW positions (the level
          // sampled speculatively into w_new) leave the moved particle's sphere
          const int far_next = (a.nbr_on && !ends) ? window_outside(w_new, span, S.s_cb, sys, lane) : 0;
          if (lane == 0) {
            S.s_need[0] = 0;
            s_ctl[2] = toAccept ? 1 : 0;
            s_ctl[3] = status;
            int nv = 0;
            if (!ends) {
              s_rng = s_spec1;
              S.s_far = far_next;
            } else if (status == 0 && more && specwarp >= 0 && !(toAccept && s_next[2] == ptcl)) {
              s_rng = s_spec2;
              s_ctl[0] = s_next[1];
              s_ctl[1] = s_next[2];
              s_logsr[L - 1] = s_next_f[0];
              s_logu[L - 1] = s_next_f[1];
              S.s_cb = S.s_next_cb;
              S.s_far = S.s_next_far;
              nv = 1;
            }
            s_next[0] = nv;
          }
        };
        {
          const double v = reduce();
          if (warp == 0) {
            const double so = __shfl_sync(0xffffffffu, v, 0), sn = __shfl_sync(0xffffffffu, v, 1);
            const double eb = __shfl_sync(0xffffffffu, v, 2);
            const double so2 = __shfl_sync(0xffffffffu, v, 3), sn2 = __shfl_sync(0xffffffffu, v, 4);
            decide(so, sn, std::is_same<R, float>::value ? eb : 0.0, so2, sn2, !std::is_same<R, float>::value);
          }
        }
        G.sync();
        if (std::is_same<R, float>::value && S.s_need[0]) {
          // FP64 re-evaluation of this stage (and of the previous stage, whose
          // sums read only slices that are multiples of 2^(level+1), unchanged
          // since), with the FP64 path's item split and reduction: its sums are
          // the FP64 path's bit for bit.
          const int need_prev = S.s_need[1];
          if (evaluator) {
            const double4 v = stage_sums_reeval<KIND>(a, w_old, w_new, level, slice1, ptcl, erank, ECL, tid, ethreads,
                                                      plist, np, need_prev, prev_plist, prev_np, tq);
            double r0 = warp_sum(v.x), r1 = warp_sum(v.y), r2 = warp_sum(v.z), r3 = warp_sum(v.w);
            if (warp == kinwarp && erank == 0) {  // the kinetic links, as in the first pass
              const double2 k = kinetic_sums(w_old, w_new, L, level, sys, lane);
              const double2 kp = need_prev ? kinetic_sums(w_old, w_new, L, level + 1, sys, lane)
                                           : make_double2(0.0, 0.0);
              r0 += k.x;
              r1 += k.y;
              r2 += kp.x;
              r3 += kp.y;
            }
            if (lane == 0) {
              sh_red[warp][0] = r0;
              sh_red[warp][1] = r1;
              sh_red[warp][2] = r2;
              sh_red[warp][3] = r3;
              sh_red[warp][4] = 0.0;
            }
          } else {
            if (lane < kRed) sh_red[warp][lane] = 0.0;
            if (warp == sampler && erank == 0 && kinwarp < 0) {  // the kinetic links, as in the first pass
              const double2 k = kinetic_sums(w_old, w_new, L, level, sys, lane);
              const double2 kp = need_prev ? kinetic_sums(w_old, w_new, L, level + 1, sys, lane)
                                           : make_double2(0.0, 0.0);
              __syncwarp();
              if (lane == 0) {
                sh_red[warp][0] = k.x;
                sh_red[warp][1] = k.y;
                sh_red[warp][2] = kp.x;
                sh_red[warp][3] = kp.y;
              }
            }
          }
          if (lead) c_reevals++;
          G.sync();
          const double v = reduce();
          if (warp == 0) {
            const double so = __shfl_sync(0xffffffffu, v, 0), sn = __shfl_sync(0xffffffffu, v, 1);
            const double pso = __shfl_sync(0xffffffffu, v, 2), psn = __shfl_sync(0xffffffffu, v, 3);
            if (need_prev) prevDS = psn - pso;
            decide(so, sn, 0.0, so, sn, true);
          }
          G.sync();
        }
        if (tid == 0) c_stages++;
        prev_np = np;
        prev_plist = plist;
        if (!s_ctl[2] || s_ctl[3]) {
          acc_all = false;
          break;
        }
        passed++;
      }
      have_next = s_next[0] != 0;
      if (lead) {
        rec.accepted = acc_all ? 1 : 0;
        rec.stages_passed = passed;
      }
    }  // active
    // ---- AcceptCopy (PathClass.cc:797-863); a rejected move left HBM untouched ----
    // The moved particle's window (and, with long range, the window's rho_k)
    // by this CTA's threads.
    auto accept_copy = [&](bool write_path) {
      if (a.use_lr) {
        // AcceptCopy of rho_k (PathClass.cc:797-863): the NEW rho_k of the
        // window from the positions before PutInBoxFast as UpdateRho_ks saw
        // them, in FP64 on both paths (the mixed path's FP32 phases serve its
        // decisions only, so the chain state stays the FP64 path's).  Split
        // over the cluster's CTAs; with concurrent windows only interior
        // slices are written (end slices are shared with the neighbouring
        // windows, and their update is rounding only).
        const int lo = a.concurrent ? 1 : 0, hi = a.concurrent ? span - 1 : span;
        const int nk = a.nk, total = (hi - lo + 1) * nk;
        for (int it = (int)erank * G.size + tid; it < total; it += (int)ECL * G.size) {
          const int rel = lo + it / nk, k = it - (it / nk) * nk;
          double2 *p2 = &a.rhok[(size_t)(slice1 + rel) * nk + k];
          const double2 rn = rho_new_k<double>(__ldcg(p2), a.kvec + 3 * k, win_new[cur][rel], win_old[cur][rel]);
          __stcg(p2, rn);
        }
      }
      // With concurrent windows only the interior slices: the end slices are
      // shared with the neighbouring windows and never move, and boxing them
      // here would race with the neighbour's read of the same slice.
      if (write_path)
        for (int rel = (a.concurrent ? 1 : 0) + tid; rel <= (a.concurrent ? span - 1 : span); rel += G.size) {
          double v[3] = {win_new[cur][rel][0], win_new[cur][rel][1], win_new[cur][rel][2]};
          put_in_box_fast(v, sys);
          double *q = path + ((size_t)(slice1 + rel) * N + mptcl) * 3;
          q[0] = v[0];
          q[1] = v[1];
          q[2] = v[2];
        }
    };
    auto count_move = [&](long long at) {  // by the lead thread
      moves++;
      if (acc_all) accepted++;
      if (PROP) {
        stages += mv_stages;
        pair_evals += mv_pairs;
        flips += mv_flips;
        reevals += mv_reevals;
      }
      if (a.trace) a.trace[a.trace_offset + at] = rec;
    };
    if (!PROP) {
      if (acc_all && move_far) {
        // this move left its sphere: the lists no longer bound this job's
        // positions; all partners from here on, and a rebuild before the next launch
        if (tid == 0) S.s_allpairs = 1;
        if (lead) atomicExch(a.nbr_dirty, 1);
      }
      if (acc_all) {
        accept_copy(rank == 0);
        if (CL > 1)
          cluster.sync();
        else
          G.sync();
      }
      if (lead)
        count_move(a.concurrent ? (long long)window * a.steps_per_block + step
                                : (long long)blk * a.steps_per_block + step);
      if (s_ctl[3] != 0) break;
      if (have_next) cur ^= 1;
      G.sync();  // every thread has read s_ctl / s_next before the next move rewrites them
    } else {
      // ---- in-order commit of the pass ----
      // Every slot publishes its outcome to every CTA of the window: accepted,
      // particle, whether it left its sphere, status.
      if (tid == 0) {
        const int4 pub = active ? make_int4(acc_all ? 1 : 0, mptcl, move_far, s_ctl[3]) : make_int4(0, -1, 0, 0);
        for (unsigned r = 0; r < CL; r++) cluster.map_shared_rank(&S.s_pub[rank], r)[0] = pub;
        S.s_redo_local = 0;
      }
      cluster.sync();
      // This slot is made again if an earlier slot q of the pass accepted a
      // move of its particle, or of a particle whose OLD or NEW positions come
      // within the pair range of this slot's OLD or NEW positions at some
      // slice (q's window is read from q's shared memory).  Otherwise every
      // pair term between the two particles is zero before and after q's
      // move, and this slot's sums are those of the in-order move.
      if (active && (int)rank > pfirst)
        for (int q = pfirst + warp; q < (int)rank; q += nwarps) {
          const int4 o = S.s_pub[q];
          if (!o.x) continue;  // a rejected move changed nothing
          bool hit = o.y == mptcl;
          if (!hit) {
            const double(*qo)[3] = cluster.map_shared_rank(&S.win_old[0][0], (unsigned)q);
            const double(*qn)[3] = cluster.map_shared_rank(&S.win_new[0][0], (unsigned)q);
            hit = windows_near(win_old[0], win_new[0], qo, qn, span, a.pair_range, sys, lane);
          }
          if (hit && lane == 0) S.s_redo_local = 1;
        }
      G.sync();
      if (tid == 0)
        for (unsigned r = 0; r < CL; r++) cluster.map_shared_rank(&S.s_redo[rank], r)[0] = S.s_redo_local;
      cluster.sync();
      if (warp == 0) {
        const bool redo = lane > pfirst && lane < P && S.s_redo[lane] != 0;
        const unsigned bad = __ballot_sync(0xffffffffu, redo);
        const int nf = bad ? __ffs(bad) - 1 : P;
        const int4 me = (lane >= pfirst && lane < P) ? S.s_pub[lane] : make_int4(0, -1, 0, 0);
        const bool kept = lane >= pfirst && lane < nf;
        const bool stop = __any_sync(0xffffffffu, me.w != 0);
        const bool far_acc = __any_sync(0xffffffffu, kept && me.x && me.z);
        if (lane == 0) {
          S.s_commit[0] = nf;
          S.s_commit[1] = stop ? 1 : 0;
          S.s_commit[2] = far_acc ? 1 : 0;
        }
      }
      G.sync();
      const int nf = S.s_commit[0];
      if (active && (int)rank < nf) {
        if (acc_all) accept_copy(true);
        if (lead) count_move(((long long)window * a.steps_per_block + step) * P + rank);
      } else if (active) {
        if (tid == 0) {
          s_rng = S.s_rng0;  // the redo draws from the move's first number again
          redone++;
        }
      }
      if (S.s_commit[2]) {
        // a kept move left its sphere: all partners for the rest of the round
        if (tid == 0) S.s_allpairs = 1;
        if (rank == 0 && tid == 0) atomicExch(a.nbr_dirty, 1);
      }
      cluster.sync();  // kept windows are in HBM; every CTA has read s_pub and s_commit
      if (nf >= P) {
        pstep++;
        pfirst = 0;
      } else {
        pfirst = nf;
      }
      if (S.s_commit[1]) break;
    }
    // Refill the stream table once less than half of it is ahead of the
    // committed position (the next move's draws, if any, are committed).
    if ((long long)(S.tab.tb + (uint64_t)S.tab.W) - (long long)s_rng.n < (long long)(tab_mem.W >> 1))
      rng_tab_fill(S.tab, tab_mem.W, seed, stream, s_rng.n, tid, G.size, gsync);
  }
  if (lead) {
    cs->nlocal = s_rng.n;
    cs->one_left = s_rng.one_left;
    cs->x2 = s_rng.x2;
    cs->moves += moves;
    cs->accepted += accepted;
    cs->stages += stages;
    cs->pair_evals += pair_evals;
    cs->flips += flips;
    cs->redone += redone;
    cs->reevals += reevals;
    if (status) cs->status = status;
  }
  if (CL > 1) cluster.sync();
  G.sync();
}

// One chain on a thread-block cluster: the sequential schedule (one launch
// runs n_blocks blocks), or one round of the concurrent-window schedule
// (cluster w works window w).
template <int KIND, typename R, bool SHADOW, bool PROP>
__global__ void __launch_bounds__(512, 1) bisection_kernel(BisectionArgs a) {
  __shared__ KernelShared S;
  __shared__ RngStore<2> store;
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ int s_nbr[kNbrStage];
  extern __shared__ __align__(16) unsigned char dyn[];
  cg::cluster_group cluster = cg::this_cluster();
  const unsigned rank = cluster.block_rank();
  const unsigned CL = cluster.num_blocks();
  const int window = (int)(blockIdx.x / CL);
  if (threadIdx.x == 0) {
    mbar_init(&s_bar, 1);
    mbar_init(&S.test_bar, 1);
    mbar_init(&S.red_bar[0], 1);
    mbar_init(&S.red_bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  unsigned phase = 0;
  ChainState *cs = a.chains + (a.concurrent ? (PROP ? (int)rank * kMaxWindows + window : window) : 0);
  const Group G = {(int)threadIdx.x, (int)blockDim.x, 0u};
  unsigned dyn_size;
  asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn_size));
  const RngTab tab = store.part<2>(0, 2);
  run_job<KIND, R, SHADOW, false, PROP>(a, cs, window, rank, CL, cluster, G, dyn, dyn_size, S, &s_bar, phase, tab,
                                        s_nbr);
}

// Many independent chains in one persistent launch (the reference's clone
// parallelism).  Chains are queued by estimated cost, largest first, behind
// one atomic counter.  A CTA starts as one group of all its threads; a group
// takes the next chain and, when that chain's queue position is at or past
// the split point of its level (split[k]) and a finer level exists, halves:
// the first half keeps the chain, the second half takes a new one.  The
// costliest chains therefore run on the whole CTA and the cheap tail on
// 1/2 or 1/4 of it, so the step is not held up by its largest chains while
// small chains still fill the SMs.  Group (k, p) — level k, position p —
// owns threads [p, p+1) * blockDim/2^k, named barrier 2^k + p, and the
// per-slot shared state of slot p * 2^(max_split-k) (its table copy
// included).
constexpr size_t kBatchStoreBytes = (sizeof(RngStore<1 << kMaxSplit>) + 15) & ~(size_t)15;

template <int KIND, typename R, bool SHADOW>
__global__ void __launch_bounds__(512, 1) batch_kernel(BatchArgs b) {
  constexpr int kSlots = 1 << kMaxSplit;
  __shared__ KernelShared S[kSlots];
  __shared__ BisectionArgs jobs[kSlots];
  __shared__ int s_chain[kSlots];
  __shared__ __align__(8) uint64_t s_bar[kSlots];
  extern __shared__ __align__(16) unsigned char dyn_all[];
  // dynamic shared memory: the stream tables, then the slots' staged tables
  RngStore<kSlots> &store = *reinterpret_cast<RngStore<kSlots> *>(dyn_all);
  unsigned char *dyn = dyn_all + kBatchStoreBytes;
  cg::cluster_group cluster = cg::this_cluster();
  if (threadIdx.x < kSlots) {
    mbar_init(&s_bar[threadIdx.x], 1);
    mbar_init(&S[threadIdx.x].test_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  int k = 0, p = 0;
  int c = -1;  // queue position in hand (group-uniform)
  unsigned phase = 0;
  for (int guard = 0; guard < 2 * b.n_chains + 2 * kSlots + 2; guard++) {
    const int gsize = (int)blockDim.x >> k;
    const Group G = {(int)threadIdx.x - p * gsize, gsize, (1u << k) + (unsigned)p};
    const int slot = p << (b.max_split - k);
    if (c < 0) {
      if (G.tid == 0) s_chain[slot] = (int)atomicAdd(b.queue, 1u);
      G.sync();
      c = s_chain[slot];
      G.sync();  // s_chain[slot] is rewritten only after every thread read it
      if (c >= b.n_chains) break;
    }
    if (k < b.max_split && c >= b.split[k]) {
      const int half = gsize >> 1;
      const int second = G.tid >= half ? 1 : 0;
      k++;
      p = 2 * p + second;
      if (second) {
        c = -1;
        phase = 0;  // this half's slot has an unused mbarrier
      }
      continue;
    }
    const int chain = b.order[c];
    BisectionArgs &job = jobs[slot];
    {
      const int *src = reinterpret_cast<const int *>(b.jobs + chain);
      int *dst = reinterpret_cast<int *>(&job);
      for (int i = G.tid; i < (int)(sizeof(BisectionArgs) / sizeof(int)); i += gsize) dst[i] = src[i];
    }
    G.sync();
    if (G.tid == 0) {
      job.n_blocks = b.n_blocks;
      job.trace = b.trace ? b.trace + (long long)chain * b.trace_per_chain : nullptr;
      job.trace_offset = 0;
    }
    G.sync();
    const RngTab tab = store.part<kSlots>(p << (kMaxSplit - k), 1 << (kMaxSplit - k));
    run_job<KIND, R, SHADOW, true>(job, job.chains, 0, 0, 1, cluster, G, dyn + (size_t)slot * b.dyn_per_slot,
                             b.dyn_per_slot, S[slot], &s_bar[slot], phase, tab);
    c = -1;
  }
}


template <int KIND, typename R, bool SHADOW, bool PROP = false>
static cudaError_t launch_t(const BisectionArgs &a, int cl, int clusters, int threads, size_t dyn, cudaStream_t st) {
  auto kfn = bisection_kernel<KIND, R, SHADOW, PROP>;
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

template <int KIND, typename R, bool SHADOW, bool PROP = false>
static cudaError_t occupancy_t(int cl, int threads, size_t dyn, int *max_clusters) {
  auto kfn = bisection_kernel<KIND, R, SHADOW, PROP>;
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
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cl;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaOccupancyMaxActiveClusters(max_clusters, kfn, &cfg);
}

cudaError_t bisection_occupancy(const BisectionArgs &a, int precision, int shadow, int cl, int threads,
                                int *max_clusters) {
  const size_t dyn = bisection_dyn_smem(a, precision, shadow);
  const bool mixed = precision == PIMC_MIXED;
  if (a.proposals > 1) {
    if (a.pa.kind != PA_DAVID) return cudaErrorInvalidValue;
    if (mixed) return shadow ? occupancy_t<PA_DAVID, float, true, true>(cl, threads, dyn, max_clusters)
                             : occupancy_t<PA_DAVID, float, false, true>(cl, threads, dyn, max_clusters);
    return shadow ? occupancy_t<PA_DAVID, double, true, true>(cl, threads, dyn, max_clusters)
                  : occupancy_t<PA_DAVID, double, false, true>(cl, threads, dyn, max_clusters);
  }
  if (a.pa.kind == PA_DAVID) {
    if (mixed) return shadow ? occupancy_t<PA_DAVID, float, true>(cl, threads, dyn, max_clusters)
                             : occupancy_t<PA_DAVID, float, false>(cl, threads, dyn, max_clusters);
    return shadow ? occupancy_t<PA_DAVID, double, true>(cl, threads, dyn, max_clusters)
                  : occupancy_t<PA_DAVID, double, false>(cl, threads, dyn, max_clusters);
  }
  if (a.pa.kind == PA_COULOMB) {
    if (mixed) return shadow ? occupancy_t<PA_COULOMB, float, true>(cl, threads, dyn, max_clusters)
                             : occupancy_t<PA_COULOMB, float, false>(cl, threads, dyn, max_clusters);
    return shadow ? occupancy_t<PA_COULOMB, double, true>(cl, threads, dyn, max_clusters)
                  : occupancy_t<PA_COULOMB, double, false>(cl, threads, dyn, max_clusters);
  }
  if (mixed) return shadow ? occupancy_t<PA_TRICUBIC, float, true>(cl, threads, dyn, max_clusters)
                           : occupancy_t<PA_TRICUBIC, float, false>(cl, threads, dyn, max_clusters);
  return shadow ? occupancy_t<PA_TRICUBIC, double, true>(cl, threads, dyn, max_clusters)
                : occupancy_t<PA_TRICUBIC, double, false>(cl, threads, dyn, max_clusters);
}

template <int KIND, typename R, bool SHADOW>
static cudaError_t launch_batch_t(const BatchArgs &b, int blocks, int threads, size_t dyn, cudaStream_t st) {
  auto kfn = batch_kernel<KIND, R, SHADOW>;
  dyn += kBatchStoreBytes;
  cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  if (e != cudaSuccess) return e;
  kfn<<<blocks, threads, dyn, st>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_batch(const BatchArgs &b, int precision, int shadow, int blocks, int threads, size_t dyn,
                         cudaStream_t st) {
  if (b.max_split < 0 || b.max_split > kMaxSplit || b.dyn_per_slot % 16 ||
      dyn < ((size_t)b.dyn_per_slot << b.max_split) || dyn + kBatchStoreBytes > (size_t)180 * 1024)
    return cudaErrorInvalidValue;
  if (threads < 64 || threads > 512 || (threads >> b.max_split) % 32 || (threads >> b.max_split) < 64 || blocks < 1)
    return cudaErrorInvalidValue;
  if (precision == PIMC_MIXED)
    return shadow ? launch_batch_t<PA_DAVID, float, true>(b, blocks, threads, dyn, st)
                  : launch_batch_t<PA_DAVID, float, false>(b, blocks, threads, dyn, st);
  return shadow ? launch_batch_t<PA_DAVID, double, true>(b, blocks, threads, dyn, st)
                : launch_batch_t<PA_DAVID, double, false>(b, blocks, threads, dyn, st);
}

template <int KIND, typename R, bool SHADOW>
static cudaError_t batch_occupancy_t(int threads, size_t dyn, int *blocks_per_sm) {
  auto kfn = batch_kernel<KIND, R, SHADOW>;
  dyn += kBatchStoreBytes;
  cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kfn, threads, dyn);
}

cudaError_t batch_occupancy(int precision, int shadow, int threads, size_t dyn, int *blocks_per_sm) {
  if (precision == PIMC_MIXED)
    return shadow ? batch_occupancy_t<PA_DAVID, float, true>(threads, dyn, blocks_per_sm)
                  : batch_occupancy_t<PA_DAVID, float, false>(threads, dyn, blocks_per_sm);
  return shadow ? batch_occupancy_t<PA_DAVID, double, true>(threads, dyn, blocks_per_sm)
                : batch_occupancy_t<PA_DAVID, double, false>(threads, dyn, blocks_per_sm);
}

size_t bisection_dyn_smem(const BisectionArgs &a, int precision, int shadow) {
  if (a.pa.kind == PA_TRICUBIC) {
    // FP64: the potential's pairs when they fit in 160 KB with the term
    // lists; the term lists alone otherwise (and on the mixed path, whose
    // FP64 re-evaluation uses them)
    const size_t pot = precision == PIMC_MIXED ? 0 : (size_t)a.pa.t64.pot_pairs_n * sizeof(double2);
    return pot + kTriTermBytes <= (size_t)160 * 1024 ? pot + kTriTermBytes : (size_t)kTriTermBytes;
  }
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
  if (a.proposals > 1) {  // concurrent proposals: DavidPA tables (the neighbour lists' action)
    if (a.pa.kind != PA_DAVID || !a.concurrent || a.use_lr) return cudaErrorInvalidValue;
    if (mixed) return shadow ? launch_t<PA_DAVID, float, true, true>(a, cl, clusters, threads, dyn, st)
                             : launch_t<PA_DAVID, float, false, true>(a, cl, clusters, threads, dyn, st);
    return shadow ? launch_t<PA_DAVID, double, true, true>(a, cl, clusters, threads, dyn, st)
                  : launch_t<PA_DAVID, double, false, true>(a, cl, clusters, threads, dyn, st);
  }
  if (a.pa.kind == PA_DAVID) {
    if (mixed) return shadow ? launch_t<PA_DAVID, float, true>(a, cl, clusters, threads, dyn, st)
                             : launch_t<PA_DAVID, float, false>(a, cl, clusters, threads, dyn, st);
    return shadow ? launch_t<PA_DAVID, double, true>(a, cl, clusters, threads, dyn, st)
                  : launch_t<PA_DAVID, double, false>(a, cl, clusters, threads, dyn, st);
  }
  if (a.pa.kind == PA_COULOMB) {
    if (mixed) return shadow ? launch_t<PA_COULOMB, float, true>(a, cl, clusters, threads, dyn, st)
                             : launch_t<PA_COULOMB, float, false>(a, cl, clusters, threads, dyn, st);
    return shadow ? launch_t<PA_COULOMB, double, true>(a, cl, clusters, threads, dyn, st)
                  : launch_t<PA_COULOMB, double, false>(a, cl, clusters, threads, dyn, st);
  }
  if (mixed) return shadow ? launch_t<PA_TRICUBIC, float, true>(a, cl, clusters, threads, dyn, st)
                           : launch_t<PA_TRICUBIC, float, false>(a, cl, clusters, threads, dyn, st);
  return shadow ? launch_t<PA_TRICUBIC, double, true>(a, cl, clusters, threads, dyn, st)
                : launch_t<PA_TRICUBIC, double, false>(a, cl, clusters, threads, dyn, st);
}

}  // namespace pimc

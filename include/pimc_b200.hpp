/*
 * pimc_b200.hpp — C++17 host layer over the C ABI in pimc_b200.h, with the
 * reference's class and method names, for PIMC++ code and other C++ callers.
 *
 *   pimc_b200::PathData              PathClass + MirroredClass OLD/NEW copies
 *                                    (PIMC++/src/PathClass.h:37-414, MirroredClass.h:23-200)
 *   pimc_b200::ActionBaseClass       ActionBaseClass::SingleAction / Action / d_dBeta
 *                                    (PIMC++/src/Actions/ActionBase.h:31-75)
 *   pimc_b200::ShortRangeClass       ShortRangeClass (Actions/ShortRangeClass.cc:191-355)
 *   pimc_b200::KineticClass          KineticClass (Actions/KineticClass.cc:33-256)
 *   pimc_b200::LongRangeClass        LongRangeClass (Actions/LongRangeClass.cc:273-442)
 *   pimc_b200::BisectionBlockClass   BisectionBlockClass::MakeMove (Moves/BisectionBlock.cc:380-451)
 *
 * Header-only; link with -lpimc_b200.  A failed call throws pimc_b200::Error
 * carrying the status code and the context's message (the reference
 * asserts or aborts instead; a caller that wants that catches and aborts).
 * Objects are not thread-safe: one PathData per host thread, as the
 * reference is single-threaded per rank.
 */
#ifndef PIMC_B200_HPP
#define PIMC_B200_HPP

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "pimc_b200.h"

namespace pimc_b200 {

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string &what) : std::runtime_error(what), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

enum Mode { OLDMODE = PIMC_OLD, NEWMODE = PIMC_NEW };

/* The chain's device state: path copies, pair action, rho_k. */
class PathData {
 public:
  PathData(int numParticles, int numTimeSlices, const std::array<double, 3> &box, double tau, double lambda,
           int numImages = 0, int device = 0)
      : N_(numParticles), S_(numTimeSlices), lambda_{lambda}, species_(numParticles, 0) {
    pimc_system_desc d{};
    d.num_particles = numParticles;
    d.num_time_slices = numTimeSlices;
    for (int i = 0; i < 3; i++) d.box[i] = box[i];
    d.tau = tau;
    d.num_species = 1;
    d.species_of = species_.data();
    d.lambda = lambda_;
    d.num_images = numImages;
    d.device = device;
    const int rc = pimc_create(&d, &ctx_);
    if (rc != PIMC_OK) throw Error(rc, std::string("pimc_create: ") + pimc_status_string(rc));
  }
  ~PathData() {
    if (ctx_) pimc_destroy(ctx_);
  }
  PathData(const PathData &) = delete;
  PathData &operator=(const PathData &) = delete;

  pimc_context *context() const { return ctx_; }
  int NumParticles() const { return N_; }
  int NumTimeSlices() const { return S_; }

  /* MirroredClass::SetMode: which copy the Action objects evaluate. */
  void SetMode(Mode m) { mode_ = m; }
  Mode GetMode() const { return mode_; }

  /* Path rows [slice][particle][3]; copy PIMC_OLD, PIMC_NEW or PIMC_BOTH. */
  void SetPath(const std::vector<double> &path, int copy = PIMC_BOTH) {
    size_check(path.size());
    check(pimc_set_path(ctx_, copy, path.data()), "pimc_set_path");
  }
  std::vector<double> GetPath(Mode copy = OLDMODE) const {
    std::vector<double> out((size_t)S_ * N_ * 3);
    check(pimc_get_path(ctx_, copy, out.data()), "pimc_get_path");
    return out;
  }

  /* DavidPAClass::Read with Daviddmfile = dmFile (DavidPAClass.h:144-190). */
  void ReadDavidSquarerFile(const std::string &dmFile, int numOffDiagonalTerms = 0) {
    check(pimc_pa_david_from_dm(ctx_, 0, 0, dmFile.c_str(), numOffDiagonalTerms), "pimc_pa_david_from_dm");
  }
  /* PAclassicalFitClass with a Coulomb potential Z1Z2/r. */
  void SetCoulombPairAction(double z1z2, int numLevels) {
    check(pimc_pa_coulomb(ctx_, 0, 0, z1z2, numLevels), "pimc_pa_coulomb");
  }

  void AcceptCopy(int slice1, int slice2, const std::vector<int> &active) {
    check(pimc_accept_copy(ctx_, slice1, slice2, active.data(), (int)active.size()), "pimc_accept_copy");
  }
  void RejectCopy(int slice1, int slice2, const std::vector<int> &active) {
    check(pimc_reject_copy(ctx_, slice1, slice2, active.data(), (int)active.size()), "pimc_reject_copy");
  }
  /* PathClass::ShiftPathData / ShiftMoveClass::MakeMove. */
  void ShiftData(int slicesToShift) { check(pimc_shift_data(ctx_, slicesToShift), "pimc_shift_data"); }
  int ShiftMove() {
    int n = 0;
    check(pimc_shift_move(ctx_, &n), "pimc_shift_move");
    return n;
  }
  void WriteCheckpoint(const std::string &file) const {
    check(pimc_checkpoint_write(ctx_, file.c_str()), "pimc_checkpoint_write");
  }
  /* After BisectionBlockClass set-up and Seed, which clear the counters and streams it restores. */
  void ReadCheckpoint(const std::string &file) { check(pimc_checkpoint_read(ctx_, file.c_str()), "pimc_checkpoint_read"); }

  /* PathClass::SetupkVecs3D and the Coulomb breakup of LongRangeClass::Init. */
  int SetupkVecs(double kCutoff) {
    int nk = 0;
    check(pimc_setup_kvecs(ctx_, kCutoff, &nk), "pimc_setup_kvecs");
    return nk;
  }
  void InitLongRangeCoulomb(int numBreakupKnots, bool useBackground) {
    check(pimc_longrange_coulomb(ctx_, numBreakupKnots, useBackground ? 1 : 0), "pimc_longrange_coulomb");
  }

  void check(int rc, const char *what) const {
    if (rc == PIMC_OK) return;
    char msg[512] = {0};
    if (ctx_) pimc_last_error(ctx_, msg, (int)sizeof msg);
    throw Error(rc, std::string(what) + ": " + pimc_status_string(rc) + (msg[0] ? std::string(": ") + msg : ""));
  }

 private:
  void size_check(size_t n) const {
    if (n != (size_t)S_ * N_ * 3) throw Error(PIMC_E_ARG, "path must hold NumTimeSlices x NumParticles x 3 doubles");
  }
  pimc_context *ctx_ = nullptr;
  int N_, S_;
  double lambda_[1];
  std::vector<int> species_;
  Mode mode_ = OLDMODE;
};

/* ActionBaseClass: SingleAction on the PathData's current mode. */
class ActionBaseClass {
 public:
  explicit ActionBaseClass(PathData &pathData, int precision = PIMC_FP64) : PathData_(pathData), Precision(precision) {}
  virtual ~ActionBaseClass() = default;
  virtual double SingleAction(int slice1, int slice2, const std::vector<int> &activeParticles, int level) {
    double s = 0.0;
    PathData_.check(pimc_single_action(PathData_.context(), kind(), PathData_.GetMode(), slice1, slice2,
                                       activeParticles.data(), (int)activeParticles.size(), level, Precision, &s),
                    "pimc_single_action");
    return s;
  }
  /* ActionBase.cc:147-166: Action forwards to SingleAction. */
  double Action(int slice1, int slice2, const std::vector<int> &activeParticles, int level) {
    return SingleAction(slice1, slice2, activeParticles, level);
  }
  virtual double d_dBeta(int slice1, int slice2, int level) {
    double s = 0.0;
    PathData_.check(pimc_d_dbeta(PathData_.context(), kind(), slice1, slice2, level, &s), "pimc_d_dbeta");
    return s;
  }
  virtual std::string GetName() const = 0;

 protected:
  virtual int kind() const = 0;
  PathData &PathData_;
  int Precision;
};

class ShortRangeClass : public ActionBaseClass {
 public:
  using ActionBaseClass::ActionBaseClass;
  std::string GetName() const override { return "ShortRange"; }

 protected:
  int kind() const override { return PIMC_ACTION_SHORTRANGE; }
};

class KineticClass : public ActionBaseClass {
 public:
  using ActionBaseClass::ActionBaseClass;
  std::string GetName() const override { return "Kinetic"; }

 protected:
  int kind() const override { return PIMC_ACTION_KINETIC; }
};

class LongRangeClass : public ActionBaseClass {
 public:
  using ActionBaseClass::ActionBaseClass;
  std::string GetName() const override { return "LongRange"; }

 protected:
  int kind() const override { return PIMC_ACTION_LONGRANGE; }
};

/* BisectionBlockClass: whole moves on the device.  MakeMoves(n) runs n
 * blocks (n x StepsPerBlock moves in the sequential schedule) and returns
 * their records. */
class BisectionBlockClass {
 public:
  BisectionBlockClass(PathData &pathData, int numLevels, int stepsPerBlock, bool shortRangeAtHigherLevels = true,
                      int precision = PIMC_FP64, int schedule = PIMC_SCHEDULE_SEQUENTIAL, int clusterCtas = 0,
                      int threadsPerCta = 0, bool useLongRange = false)
      : PathData_(pathData) {
    pimc_bisection_desc d{};
    d.num_levels = numLevels;
    d.steps_per_block = stepsPerBlock;
    d.shortrange_at_higher_levels = shortRangeAtHigherLevels ? 1 : 0;
    d.use_longrange = useLongRange ? 1 : 0;
    d.precision = precision;
    d.cluster_ctas = clusterCtas;
    d.threads_per_cta = threadsPerCta;
    d.schedule = schedule;
    PathData_.check(pimc_bisection_setup(PathData_.context(), &d), "pimc_bisection_setup");
    PathData_.check(pimc_bisection_windows(PathData_.context(), &windows_), "pimc_bisection_windows");
    steps_ = stepsPerBlock;
    // PROPOSALS: records [round][window][step][slot], clusterCtas slots (0 = 8)
    if (schedule == PIMC_SCHEDULE_PROPOSALS) steps_ *= clusterCtas ? clusterCtas : 8;
  }
  void Seed(uint64_t seed) { PathData_.check(pimc_rng_seed(PathData_.context(), seed), "pimc_rng_seed"); }
  std::vector<pimc_move_record> MakeMoves(int numBlocks) {
    std::vector<pimc_move_record> rec((size_t)numBlocks * windows_ * steps_);
    pimc_bisection_stats st{};
    PathData_.check(pimc_run_bisection(PathData_.context(), numBlocks, rec.data(), &st), "pimc_run_bisection");
    return rec;
  }
  pimc_bisection_stats Stats() const {
    pimc_bisection_stats st{};
    PathData_.check(pimc_bisection_get_stats(PathData_.context(), &st), "pimc_bisection_get_stats");
    return st;
  }

 private:
  PathData &PathData_;
  int windows_ = 1, steps_ = 1;
};

}  // namespace pimc_b200

#endif  // PIMC_B200_HPP

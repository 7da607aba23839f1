// pic.hpp -- C++ host objects of the PIC step, mirroring gample's classes.
//
//   EMField   src/EMField.{h,mm}   staggered fields, Poisson solve, diagnostics
//   Particle  src/Particle.{h,mm}  one species: push, deposit, reduce
//   Collision src/Collision.{h,mm} initial load and particle sources
//   XmlLogger src/XmlLogger.h      XML log and timeseries CSV
//
// Each object owns its device memory and issues work on one CUDA stream;
// results stay in HBM and are copied back only for diagnostics and I/O.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <fstream>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "device.hpp"
#include "init.hpp"
#include "kernels.hpp"
#include "learned.hpp"
#include "multigrid.hpp"

namespace gample {

// src/XmlLogger.h:89-93 (value rounded to float, std::scientific)
std::string fmtSci(float v, int prec);

// src/XmlLogger.h:8-86
class XmlLogger {
 public:
  XmlLogger(const std::string& logName, const std::string& csvHeader);
  ~XmlLogger();
  void swichLog(bool on) { on_ = on; }
  bool on() const { return on_; }
  void logCycleStart(int cycle, double time);
  void logSection(const std::string& name, const std::map<std::string, std::string>& data);
  void csvOutput(const std::string& data);
  void logCycleEnd();
  void logComment(const std::string& comment);

 private:
  std::ofstream xml_, csv_;
  bool on_ = false;
};

struct SolveStats {
  int iterations = 0;
  double error = 0;         // relative residual
  double meanCathode = 0;   // V
  double energy = 0;        // erg/m (src/EMField.mm:1112: no 1/(4 pi))
  double EEincrement = 0;
  double joule = 0;
  double probe[3] = {0, 0, 0};  // phi1 (statV), Ex1, Ey1 (statV/cm)
  double field_energy_cgs = 0;  // sum E^2/(8 pi) dx dy (physical)
};

struct FlowStats {
  uint32_t particleNumber = 0;
  uint32_t pulledPtclNum = 0;
  int pinum[4] = {0, 0, 0, 0};  // charge-weighted counts per wall
  uint32_t invalid = 0;
  double totalKineticEnergy = 0;  // erg
  double totalKEincrement = 0;
};

class Particle;

class EMField {
 public:
  EMField(const Init& init, cudaStream_t s, int nspecies);  // src/EMField.mm:105-656
  void resetChargeDensity();                               // src/EMField.mm:1363-1378
  SolveStats solvePoisson(double dt, XmlLogger* logger);   // src/EMField.mm:745-1136
  // Combine the fixed-point accumulators (deterministic mode) into rho/jx/jy.
  void finalizeCharge();
  // Learned warm start of the Poisson solve (build addition). mode bits:
  // 1 start the multigrid from previous phi + the network's correction,
  // 2 train the network on (rhs, previous phi) -> (phi - previous phi) after
  // each solve, 4 also solve from the plain warm start for comparison,
  // 8 store each solve's normalised residual in the sample bank, 16 (when
  // the network is created) the residual formulation: a one-channel network
  // (widths 16/32/64/64) maps the residual r = b - A (previous phi), divided
  // by its RMS, to a correction, trained on the mean square of the residual
  // the correction leaves (2 then trains on each solve's sample).
  struct LearnedStats {
    double loss = 0;
    int iters_learned = 0, iters_plain = 0;
    double ms_learned = 0, ms_plain = 0, ms_net = 0;  // solve + network / plain solve / network alone
    double rel0_learned = 0, rel0_plain = 0;          // relative residual of the starting guess
    int trained_steps = 0;
  };
  void setLearned(int mode, float lr, uint64_t seed);
  // Sample bank of the residual formulation (capacity samples on the device)
  // and offline training on it: steps Adam steps on samples drawn at random
  // (seed); out[0], out[1]: mean loss of the first and of the last ten steps,
  // out[2]: samples in the bank.
  void setLearnedBank(int capacity);
  void trainLearned(int steps, float lr, uint64_t seed, double out[3]);
  int learned_mode = 0;
  float learned_lr = 1e-3f;
  std::unique_ptr<nn::WarmStartNet> net;
  LearnedStats last_learned;
  // src/EMField.mm:1138-1361 (Darwin model, FlagForEquation.EMField == 2):
  // Helmholtz split of J, vector potential, delEx/delEy/delBz.
  struct DarwinStats {
    int iters[3] = {0, 0, 0};       // decompose, Ax, Ay
    double errors[3] = {0, 0, 0};   // relative residuals
  };
  DarwinStats solveVectorPotential(double dt, XmlLogger* logger);
  bool darwin = false;
  kern::DarwinGeom dgeom{};
  kern::PoissonLayout dlayout{};
  std::unique_ptr<PoissonMG> dmg;
  DeviceArray<double> psi, Ax, Ay, lastAx, lastAy, drhs, dscr;
  DarwinStats last_darwin;
  void setupDarwin();  // src/EMField.mm:447-651

  kern::GridDims dims{};
  float dx = 0, dy = 0;
  bool det = false;      // deterministic fixed-point deposit
  bool charge_dirty = false;  // fixed-point sums not yet combined into rho/jx/jy
  bool current = false;  // jx, jy deposited (Darwin or FlagForCurDens)
  bool bz_uniform = false;
  float bz_value = 0;
  int fbc[4] = {0, 0, 0, 0};
  double cathodePos = -1;
  kern::PoissonLayout layout{};
  int maxiter = 200;
  double tol = 1e-7;

  DeviceArray<float> rho, jx, jy, Ex, Ey, Ez, Bx, By, Bz;
  DeviceArray<float> delEx, delEy, delBz;  // Darwin corrections (zero in the electrostatic model)
  // Pitched copies of Ex and Ey and their tensor maps, for the field staging
  // of the atomic-mode push in a uniform Bz (the only kernel that reads them).
  // k_gradient writes them with E; any other write of E marks them stale.
  DeviceArray<float> Exp, Eyp;
  kern::FieldMaps maps{};
  bool e_pitched_stale = true;
  // The maps for the push (refreshing stale copies first), or nullptr.
  const kern::FieldMaps* pushMaps();
  DeviceArray<double> phi, sol, b, diag;  // diag: [0..1] rhs sums [2..3] E sums [4] cathode mean [5..7] probe
  // per-species deposit accumulators: int64 fixed point (deterministic mode)
  // or FP64 (fast mode); combined into rho/jx/jy by finalizeCharge()
  std::vector<DeviceArray<long long>> acc_rho, acc_jx, acc_jy;
  std::vector<DeviceArray<double>> f64_rho, f64_jx, f64_jy;
  std::vector<float> species_scale;
  std::unique_ptr<PoissonMG> mg;
  double lastEE = 0;
  MGResult last_mg;
  cudaStream_t stream;

  kern::DepositTargets targets(int s);
  size_t n_rho() const { return size_t(dims.nx + 1) * (dims.ny + 1); }
  size_t n_ex() const { return size_t(dims.nx + 2) * (dims.ny + 1); }
  size_t n_ey() const { return size_t(dims.nx + 1) * (dims.ny + 2); }
  size_t n_bz() const { return size_t(dims.nx + 2) * (dims.ny + 2); }
  size_t n_phi() const { return size_t(dims.nx + 3) * (dims.ny + 3); }

 private:
  PinnedArray<double> host_diag_;
  MGResult poissonSolve(double* d);  // plain or learned warm start
  MGResult residualSolve(double* d);  // learned warm start, residual formulation
  bool learned_residual_ = false;
  DeviceArray<float> bank_;           // normalised residual samples [cap][h][w]
  int bank_cap_ = 0, bank_n_ = 0, bank_next_ = 0;
  DeviceArray<double> nn_sum2_;
  DeviceArray<float> nn_scale_;
  DeviceArray<float> nn_in_, nn_out_, nn_target_, nn_inv_;
  DeviceArray<double> sol_prev_, sol_cmp_, nn_sums_;
  float h_inv_[3] = {0, 0, 0};
  int nn_h_ = 0, nn_w_ = 0;
  void load1dField(const std::string& path, std::vector<float>& out, size_t need) const;  // :658-687
};

class Particle {
 public:
  Particle(const Init& init, int s, cudaStream_t stream);  // src/Particle.mm:407-611
  // src/Particle.mm:615-891; with fused_deposit the new positions are also
  // deposited into fld (next step's charge).
  void update(double dt, EMField& fld, bool fused_deposit);
  FlowStats reduce(XmlLogger* logger);                   // src/Particle.mm:893-1002
  // reduce() in two halves: the compaction and the read-back of the counters
  // enqueued, then (after the caller has synchronised the stream) the flow
  // statistics, the sort decision and the log, so that one synchronisation
  // serves all species of a cycle.
  void reduceLaunch();
  FlowStats reduceFinish(XmlLogger* logger);
  void integrateChargeDensity(EMField& fld, bool injected_only = false);  // src/Particle.mm:1004-1130

  uint32_t pNum();  // synchronous read of the device count
  void setPNum(uint32_t n);
  void upload_aos(const kern::ParticleStateAoS* host, uint32_t n);
  void download_aos(kern::ParticleStateAoS* host, uint32_t n);
  kern::ParticleArrays arrays() const;  // the current buffer
  kern::SpeciesCounters counters();  // synchronous
  // Reorder the particles by cell (counting sort into the spare
  // buffer, then swap). The order of particles is otherwise unspecified.
  // Cell sort. lender: another species on the same stream whose spare buffer
  // is idle during the call (it may be overwritten), or null.
  void sort(Particle* lender = nullptr);
  bool needs_sort = true;
  bool random_order = true;  // particles not yet sorted since loading / upload
  int sort_interval = 0;  // cycles between sorts; 0 = adaptive (below)
  int cycles_since_sort = 0;
  uint32_t slow_after_sort = 0;  // particles pushed outside their window right after the last sort
  // Adaptive re-sort of the atomic mode: the push of the first cycle after a
  // sort sets the base time per particle; each later push adds its time above
  // that base to excess_ms; the species sorts again once excess_ms reaches
  // the time of its last periodic sort (for a push time that grows linearly
  // with the cycles since the sort this is the interval of least total time).
  // Until a periodic sort has been timed its cost is estimated from the
  // particle count. In the deterministic mode, whose cadence must not depend
  // on timings, the species sorts once the particles pushed outside their
  // chunk's window exceed those of the first push after the last sort by 2 %
  // of the live count.
  bool cost_policy = true;
  bool sort_timed = false, sort_pending_timing = false;
  float last_sort_ms = 0;
  double base_ms_per_particle = 0, excess_ms = 0;
  uint32_t n_pushed = 0;
  TimingEvent ev_push[2], ev_sort[2];
  // Autotuner of the atomic-mode push in a uniform Bz. Variants: 2048 or
  // 1024 particles per chunk, and for order 3 the gather tables on or off.
  // The pushes after the first sort run each variant twice, in mirrored
  // order (A B C D D C B A; A B B A for two variants) so that the drift of
  // the push time since the sort weighs on all alike; the fastest per
  // particle is kept for the run. Species with kTuneBelowPpc or more
  // particles per cell keep the defaults (2048, tables) untuned.
  struct PushVariant {
    int per;     // particles per thread (chunk = 256 per)
    int tables;  // 0: gather tables off
  };
  PushVariant push_variant{kern::kPushChunkPer, 1};
  int tune_step = -1;  // -1: not started, then 0 .. 2 * variants - 1, then done
  PushVariant tune_used{kern::kPushChunkPer, 1};
  double tune_ms[4] = {0, 0, 0, 0};  // summed ms per particle per variant
  bool lean_push = false;            // the last push ran the tunable kernel
  int tune_variants() const { return order == 3 ? 4 : 2; }
  static constexpr double kTuneBelowPpc = 128.0;  // tune species with fewer particles per cell
  PushVariant tune_variant(int v) const {
    return PushVariant{v % 2 == 0 ? kern::kPushChunkPer : kern::kPushChunkPer / 2, v < 2 ? 1 : 0};
  }

  std::string pName;
  int index = 0;
  float m = 0, q = 0, w = 0;
  uint32_t pNumMax = 0;
  uint32_t n_bound = 0;  // host-side upper bound of the device count
  uint32_t n_appended = 0;  // host-side upper bound of the particles appended since the last push
                            // (the device's n_injected: reset by every push and by setPNum)
  int order = 1, boris = 2;
  int pbc[4] = {0, 0, 0, 0};
  double lastKE = 0;
  int pinum[4] = {0, 0, 0, 0};
  uint32_t last_pulled = 0;
  double last_dt = 0;

  uint32_t stage_records() const;  // AoS records per upload/download chunk

  struct Buffer {
    DeviceArray<int32_t> cell;
    DeviceArray<float> ox, oy, vx, vy, vz;
    void alloc(size_t n);
    kern::ParticleArrays view() const;
  };
  Buffer buf[2];
  int cur = 0;
  DeviceArray<uint32_t> dead_bits, scratch, sort_scratch;
  DeviceArray<kern::SpeciesCounters> cnt;
  cudaStream_t stream;

 private:
  PinnedArray<kern::SpeciesCounters> host_cnt_;
  double dx_ = 0, dy_ = 0;
  kern::GridDims dims_{};
};

// src/Moment.{h,mm}: velocity moments of one species on the rho nodes.
class Moment {
 public:
  static constexpr int kCount = 10;  // n, ux, uy, uz, Pxx, Pxy, Pxz, Pyy, Pyz, Pzz
  Moment(const Init& init, cudaStream_t s);
  // src/Moment.mm:206-316; the result stays in `out` (device)
  void integrateMoments(Particle& p, const EMField& fld);
  size_t n_rho() const { return n_rho_; }
  DeviceArray<float> out;     // kCount x (nx+1)(ny+1)
  DeviceArray<double> acc;    // FP64 sums, same shape
  int species = -1;           // species of the last integration
  cudaStream_t stream;

 private:
  kern::GridDims dims_{};
  int order_ = 1;
  size_t n_rho_ = 0;
};

class Collision {
 public:
  // src/Collision.mm:189-462: sets up the sources and loads the initial
  // particles of every species (overwriting them) from the splitmix64/PCG32
  // stream.
  Collision(const Init& init, std::vector<Particle*>& ptcls, cudaStream_t stream);
  // Build addition: the initial load again from another master seed (the
  // sources keep their set-up).
  void reload(uint64_t seed, std::vector<Particle*>& ptcls);
  int artificialIonization(double dt, std::vector<Particle*>& ptcls, XmlLogger* logger);  // :464-566
  int hollowCathode(double dt, std::vector<Particle*>& ptcls, XmlLogger* logger);         // :568-678
  // Build addition: re-inject absorbed particles at Xmin (GenerateType
  // fluxMaxwellianAtXmin).
  int fluxReinjection(double dt, std::vector<Particle*>& ptcls, XmlLogger* logger);
  // libc++ minstd_rand + generate_canonical<double, 53> (src/Collision.mm:183, 482-487)
  double uniform01();

  DeviceArray<kern::RNGState> states;
  uint32_t initialized = 0;
  uint64_t master_seed = 0;
  cudaStream_t stream;

 private:
  void ensure_states(uint32_t n);
  void loadInitial(std::vector<Particle*>& ptcls);
  const Init& init_;
  uint64_t minstd_ = 1;
  bool existAI_ = false, existHC_ = false;
  int ai_source_ = -1, hc_source_ = -1;
  std::vector<int> reflux_sources_;
};

}  // namespace gample

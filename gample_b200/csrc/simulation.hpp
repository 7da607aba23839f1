// simulation.hpp -- the reference's main(): object set-up and time loop.
//
// Restates src/main.mm:28-262 in C++ on top of the device objects. Two step
// orders are available:
//   reference order (fused = false): reset, deposit every species, solve,
//     push + reduce each species, sources (src/main.mm:154-254);
//   fused order (default): the charge of the next step is deposited by the
//     push kernel itself (and by one small deposit of the injected
//     particles), so each step reads every particle once. Both orders deposit
//     the same particle states and give the same fields up to the FP32
//     atomic summation order (bit-identical in the deterministic mode).
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "pic.hpp"

namespace gample {

enum Phase { PH_DEPOSIT = 0, PH_SOLVE, PH_PUSH, PH_REDUCE, PH_SOURCE, PH_SORT, PH_COUNT };

class Simulation {
 public:
  // log_name: "<Project>_<tag>" prefix of the XML log and timeseries CSV
  // (src/main.mm:75-85); empty = no files.
  Simulation(const Init& init, const std::string& log_name, bool fused);
  ~Simulation();
  void initialize();  // src/main.mm:114-147 (initial deposit and solve)
  // Build addition: the initial load again from another master seed and the
  // cycle counter back at Start (initialize() follows); fields, solver state
  // and the warm-start network are kept.
  void reload(uint64_t seed);
  void cycle();       // one cycle of src/main.mm:155-253
  void run(int ncycles);
  // Binary outputs under bin/ (src/FileIO.mm) are written only when a log
  // name was given and the bin/ directory exists.
  bool file_output = false;

  Init init;
  cudaStream_t stream = nullptr;
  std::unique_ptr<XmlLogger> logger;
  std::vector<std::unique_ptr<Particle>> particles;
  std::vector<Particle*> ptrs;
  std::unique_ptr<EMField> field;
  std::unique_ptr<Collision> collision;
  std::unique_ptr<Moment> moment;
  bool fused = true;
  int cycle_no = 0;
  double time = 0, comp = 0;
  SolveStats last_solve;
  std::vector<FlowStats> last_flow;
  int last_ai = 0, last_hc = 0, last_reflux = 0;

  // Device time per phase (ms), accumulated while profiling is on.
  void set_profiling(bool on);
  void phase_times(double out[PH_COUNT]);

 private:
  void mark(int phase, bool begin);
  // elapsedTime section of a logged cycle (src/main.mm:167-243): device time
  // of each timed call between two events on the run's stream, in us.
  void tic(const std::string& name);
  void toc();
  void log_resources();
  cudaEvent_t take_event();
  std::vector<std::pair<std::string, std::pair<cudaEvent_t, cudaEvent_t>>> timed_;
  std::vector<cudaEvent_t> event_pool_;
  bool profiling_ = false;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> events_;
  cudaEvent_t open_ = nullptr;
  double acc_[PH_COUNT] = {0, 0, 0, 0, 0, 0};
};

}  // namespace gample

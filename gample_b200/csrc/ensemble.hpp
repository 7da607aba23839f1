// ensemble.hpp -- many independent runs advanced together on one GPU.
//
// Every member is a full Simulation with its own CUDA stream; a pool of host
// threads drives them concurrently, so the kernels of different members
// overlap on the GPU and the host synchronisation points of one member
// (diagnostics, counter reads) do not stall the others. The threads take
// members from a shared queue, largest first (particle capacity times
// species, then grid cells), so that one thread does not end up with several
// large members while the others idle; f receives the member's index. Members share no state: each one's
// results equal the same run alone.
#pragma once

#include <memory>
#include <vector>

#include "simulation.hpp"

namespace gample {

class Ensemble {
 public:
  Ensemble(const std::vector<Init>& inits, int threads);
  void initialize();
  void run(int ncycles);
  // run(ncycles) timed on the device: from the earliest member's first
  // kernel to the latest member's last (CUDA events on the member streams).
  float time_cycles(int ncycles);
  size_t size() const { return members.size(); }
  std::vector<std::unique_ptr<Simulation>> members;

 private:
  template <typename F>
  void parallel(F&& f);
  int threads_ = 1;
  std::vector<size_t> order_;  // members by decreasing size: the pool takes the largest first
};

}  // namespace gample

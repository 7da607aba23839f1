// ensemble.cpp -- thread-pool driver of independent runs (see ensemble.hpp).
#include "ensemble.hpp"

#include <exception>
#include <mutex>
#include <thread>

namespace gample {

Ensemble::Ensemble(const std::vector<Init>& inits, int threads) {
  if (inits.empty()) throw std::invalid_argument("empty ensemble");
  threads_ = threads < 1 ? 1 : threads;
  if (threads_ > int(inits.size())) threads_ = int(inits.size());
  for (const auto& in : inits) members.push_back(std::make_unique<Simulation>(in, "", true));
}

template <typename F>
void Ensemble::parallel(F&& f) {
  std::exception_ptr first;
  std::mutex mu;
  std::vector<std::thread> pool;
  int dev = 0;
  GP_CUDA(cudaGetDevice(&dev));
  for (int t = 0; t < threads_; ++t)
    pool.emplace_back([&, t] {
      try {
        GP_CUDA(cudaSetDevice(dev));
        for (size_t i = size_t(t); i < members.size(); i += size_t(threads_)) f(*members[i]);
      } catch (...) {
        std::lock_guard<std::mutex> lock(mu);
        if (!first) first = std::current_exception();
      }
    });
  for (auto& th : pool) th.join();
  if (first) std::rethrow_exception(first);
}

void Ensemble::initialize() {
  parallel([](Simulation& s) { s.initialize(); });
}

void Ensemble::run(int ncycles) {
  parallel([ncycles](Simulation& s) { s.run(ncycles); });
}

}  // namespace gample

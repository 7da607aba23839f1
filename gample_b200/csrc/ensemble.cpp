// ensemble.cpp -- thread-pool driver of independent runs (see ensemble.hpp).
#include "ensemble.hpp"

#include <algorithm>
#include <atomic>
#include <exception>
#include <mutex>
#include <numeric>
#include <thread>

namespace gample {

Ensemble::Ensemble(const std::vector<Init>& inits, int threads) {
  if (inits.empty()) throw std::invalid_argument("empty ensemble");
  threads_ = threads < 1 ? 1 : threads;
  if (threads_ > int(inits.size())) threads_ = int(inits.size());
  for (const auto& in : inits) members.push_back(std::make_unique<Simulation>(in, "", true));
  std::vector<double> cost(inits.size());
  for (size_t i = 0; i < inits.size(); ++i) {
    const Init& in = inits[i];
    cost[i] = double(in.paramForComputing.pNumMax) * in.flagForEquation.Particle +
              double(in.paramForField.ngx) * in.paramForField.ngy;
  }
  order_.resize(inits.size());
  std::iota(order_.begin(), order_.end(), size_t(0));
  std::stable_sort(order_.begin(), order_.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
}

template <typename F>
void Ensemble::parallel(F&& f) {
  std::exception_ptr first;
  std::mutex mu;
  std::atomic<size_t> next{0};
  std::vector<std::thread> pool;
  int dev = 0;
  GP_CUDA(cudaGetDevice(&dev));
  for (int t = 0; t < threads_; ++t)
    pool.emplace_back([&] {
      try {
        GP_CUDA(cudaSetDevice(dev));
        for (size_t i = next++; i < order_.size(); i = next++) f(*members[order_[i]]);
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

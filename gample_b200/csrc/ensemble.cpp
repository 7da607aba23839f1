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
        for (size_t i = next++; i < order_.size(); i = next++) f(order_[i]);
      } catch (...) {
        std::lock_guard<std::mutex> lock(mu);
        if (!first) first = std::current_exception();
      }
    });
  for (auto& th : pool) th.join();
  if (first) std::rethrow_exception(first);
}

void Ensemble::initialize() {
  parallel([this](size_t i) { members[i]->initialize(); });
}

void Ensemble::run(int ncycles) {
  parallel([this, ncycles](size_t i) { members[i]->run(ncycles); });
}

float Ensemble::time_cycles(int ncycles) {
  const size_t n = members.size();
  std::vector<TimingEvent> t0(n), t1(n);
  for (auto& m : members) GP_CUDA(cudaStreamSynchronize(m->stream));
  parallel([&](size_t i) {
    Simulation& s = *members[i];
    GP_CUDA(cudaEventRecord(t0[i].get(), s.stream));
    s.run(ncycles);
    GP_CUDA(cudaEventRecord(t1[i].get(), s.stream));
  });
  float lo = 0, hi = 0;
  for (size_t i = 0; i < n; ++i) {
    GP_CUDA(cudaEventSynchronize(t1[i].get()));
    float a = 0, b = 0;
    GP_CUDA(cudaEventElapsedTime(&a, t0[0].get(), t0[i].get()));
    GP_CUDA(cudaEventElapsedTime(&b, t0[0].get(), t1[i].get()));
    lo = std::min(lo, a);
    hi = std::max(hi, b);
  }
  return hi - lo;
}

}  // namespace gample

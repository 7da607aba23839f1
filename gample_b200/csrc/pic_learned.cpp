// pic_learned.cpp -- learned warm start of the Poisson solve (build
// addition; no reference counterpart). The multigrid always runs to the same
// relative residual, from either the previous solution (the reference's
// warm start, src/EMField.mm:410, 866) or previous + network correction, so
// the result does not depend on the network; only the number of V-cycles
// does.
#include <cmath>
#include <random>
#include <stdexcept>

#include "pic.hpp"

namespace gample {

namespace {
int rup8(int v) { return (v + 7) / 8 * 8; }

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  explicit Timer(cudaStream_t s) {
    GP_CUDA(cudaEventCreate(&a));
    GP_CUDA(cudaEventCreate(&b));
    GP_CUDA(cudaEventRecord(a, s));
  }
  void stop(cudaStream_t s) { GP_CUDA(cudaEventRecord(b, s)); }
  double ms() {
    float m = 0;
    GP_CUDA(cudaEventSynchronize(b));
    GP_CUDA(cudaEventElapsedTime(&m, a, b));
    return m;
  }
  ~Timer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};
}  // namespace

void EMField::setLearned(int mode, float lr, uint64_t seed) {
  learned_mode = mode;
  learned_lr = lr;
  if (mode == 0 || net) return;
  const int mx = layout.nkx + 1, my = layout.nky + 1;
  nn_h_ = rup8(my);
  nn_w_ = rup8(mx);
  learned_residual_ = (mode & 16) != 0;
  if (learned_residual_) {
    if (layout.fbc[0] == kern::FBC_NEUMANN_C || layout.fbc[2] == kern::FBC_NEUMANN_C)
      throw std::invalid_argument("the residual formulation needs a symmetric operator (no Neumann ends)");
    static constexpr int kResidualWidths[4] = {16, 32, 64, 64};
    net = std::make_unique<nn::WarmStartNet>(nn_h_, nn_w_, seed, stream, 1, kResidualWidths);
    nn_sum2_.resize(1, true);
    nn_scale_.resize(1, true);
  } else {
    net = std::make_unique<nn::WarmStartNet>(nn_h_, nn_w_, seed, stream);
  }
  const size_t hw = size_t(nn_h_) * nn_w_;
  nn_in_.resize(2 * hw, true);
  nn_out_.resize(hw, true);
  nn_target_.resize(hw, true);
  nn_inv_.resize(3, true);
  sol_prev_.resize(size_t(mx) * my, true);
  sol_cmp_.resize(size_t(mx) * my, true);
  nn_sums_.resize(3, true);
  h_inv_[0] = h_inv_[1] = h_inv_[2] = 0.0f;  // set from the first solve
}

void EMField::setLearnedBank(int capacity) {
  if (!net || !learned_residual_) throw std::invalid_argument("the sample bank needs the residual formulation");
  if (capacity < 1) throw std::invalid_argument("bank capacity");
  bank_.resize(size_t(capacity) * nn_h_ * nn_w_, true);
  bank_cap_ = capacity;
  bank_n_ = bank_next_ = 0;
}

void EMField::trainLearned(int steps, float lr, uint64_t seed, double out[3]) {
  if (!net || !learned_residual_ || bank_n_ == 0) throw std::invalid_argument("no samples to train on");
  std::mt19937_64 rng(seed);
  const size_t hw = size_t(nn_h_) * nn_w_;
  double first = 0, last = 0;
  int nf = 0, nl = 0;
  for (int t = 0; t < steps; ++t) {
    const size_t k = size_t(rng() % uint64_t(bank_n_));
    const double loss = net->train_step_residual(bank_.get() + k * hw, layout, lr);
    if (t < 10) first += loss, ++nf;
    if (t >= steps - 10) last += loss, ++nl;
  }
  last_learned.trained_steps += steps;
  out[0] = nf ? first / nf : 0.0;
  out[1] = nl ? last / nl : 0.0;
  out[2] = double(bank_n_);
}

MGResult EMField::residualSolve(double* d) {
  const int mx = layout.nkx + 1, my = layout.nky + 1;
  const size_t n = size_t(mx) * my, hw = size_t(nn_h_) * nn_w_;
  LearnedStats st = last_learned;
  GP_CUDA(cudaMemcpyAsync(sol_prev_.get(), sol.get(), n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  nn::residual_input(b.get(), sol_prev_.get(), layout, nn_h_, nn_w_, nn_in_.get(), nn_sum2_.get(), nn_scale_.get(),
                     stream);
  if ((learned_mode & 8) && bank_cap_ > 0) {
    GP_CUDA(cudaMemcpyAsync(bank_.get() + size_t(bank_next_) * hw, nn_in_.get(), hw * sizeof(float),
                            cudaMemcpyDeviceToDevice, stream));
    bank_next_ = (bank_next_ + 1) % bank_cap_;
    bank_n_ = bank_n_ < bank_cap_ ? bank_n_ + 1 : bank_cap_;
  }
  if (learned_mode & 4) {  // plain warm start on a copy, for comparison
    GP_CUDA(cudaMemcpyAsync(sol_cmp_.get(), sol_prev_.get(), n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    Timer t(stream);
    MGResult rp = mg->solve(b.get(), d, sol_cmp_.get(), tol, maxiter, stream);
    t.stop(stream);
    st.ms_plain = t.ms();
    st.iters_plain = rp.iterations;
    st.rel0_plain = rp.rel0;
  }
  Timer tl(stream);
  if (learned_mode & 1) {
    Timer tn(stream);
    net->forward(nn_in_.get(), nn_out_.get());
    nn::apply_residual_correction(nn_out_.get(), sol_prev_.get(), layout, nn_w_, nn_scale_.get(), sol.get(), stream);
    tn.stop(stream);
    st.ms_net = tn.ms();
  }
  MGResult r = mg->solve(b.get(), d, sol.get(), tol, maxiter, stream);
  tl.stop(stream);
  st.ms_learned = tl.ms();
  st.iters_learned = r.iterations;
  st.rel0_learned = r.rel0;
  if (learned_mode & 2) {
    st.loss = net->train_step_residual(nn_in_.get(), layout, learned_lr);
    ++st.trained_steps;
  }
  last_learned = st;
  return r;
}

MGResult EMField::poissonSolve(double* d) {
  if (!learned_mode || !net) return mg->solve(b.get(), d, sol.get(), tol, maxiter, stream);
  if (learned_residual_) return residualSolve(d);
  const int mx = layout.nkx + 1, my = layout.nky + 1;
  const size_t n = size_t(mx) * my;
  LearnedStats st = last_learned;
  GP_CUDA(cudaMemcpyAsync(sol_prev_.get(), sol.get(), n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  const bool scaled = h_inv_[2] > 0.0f;
  if (scaled) {
    GP_CUDA(cudaMemcpyAsync(nn_inv_.get(), h_inv_, sizeof(h_inv_), cudaMemcpyHostToDevice, stream));
    nn::pack_input(b.get(), sol_prev_.get(), mx, my, nn_h_, nn_w_, nn_inv_.get(), nn_in_.get(), stream);
  }
  if (learned_mode & 4) {  // plain warm start on a copy, for comparison
    GP_CUDA(cudaMemcpyAsync(sol_cmp_.get(), sol_prev_.get(), n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    Timer t(stream);
    MGResult rp = mg->solve(b.get(), d, sol_cmp_.get(), tol, maxiter, stream);
    t.stop(stream);
    st.ms_plain = t.ms();
    st.iters_plain = rp.iterations;
    st.rel0_plain = rp.rel0;
  }
  Timer tl(stream);
  const bool use = (learned_mode & 1) && scaled;
  if (use) {
    Timer tn(stream);
    net->forward(nn_in_.get(), nn_out_.get());
    nn::apply_correction(nn_out_.get(), sol_prev_.get(), mx, my, nn_w_, nn_inv_.get(), sol.get(), stream);
    tn.stop(stream);
    st.ms_net = tn.ms();
  }
  MGResult r = mg->solve(b.get(), d, sol.get(), tol, maxiter, stream);
  tl.stop(stream);
  st.ms_learned = tl.ms();
  st.iters_learned = r.iterations;
  st.rel0_learned = r.rel0;
  if ((learned_mode & 2) || !scaled) {
    // targets in units of the running correction scale; scales from this solve
    const float ones[3] = {1.0f, 1.0f, 1.0f};
    if (!scaled) GP_CUDA(cudaMemcpyAsync(nn_inv_.get(), ones, sizeof(ones), cudaMemcpyHostToDevice, stream));
    nn::make_target(sol.get(), sol_prev_.get(), b.get(), mx, my, nn_h_, nn_w_, nn_inv_.get(), nn_target_.get(),
                    nn_sums_.get(), stream);
    double sums[3];
    GP_CUDA(cudaMemcpyAsync(sums, nn_sums_.get(), sizeof(sums), cudaMemcpyDeviceToHost, stream));
    GP_CUDA(cudaStreamSynchronize(stream));
    if (scaled && (learned_mode & 2)) {
      st.loss = net->train_step(nn_in_.get(), nn_target_.get(), learned_lr);
      ++st.trained_steps;
    }
    for (int q = 0; q < 3; ++q) {  // running 1/RMS (the first solve sets them)
      const float v = sums[q] > 0 ? float(1.0 / std::sqrt(sums[q] / double(n))) : 1.0f;
      h_inv_[q] = scaled ? 0.98f * h_inv_[q] + 0.02f * v : v;
    }
  }
  last_learned = st;
  return r;
}

}  // namespace gample

// multigrid.hpp -- geometric multigrid for the Poisson system of the field.
//
// Replaces AMGCL's SA-AMG + CG (src/EMField.mm:20-28, 412-432, 866) for the
// 5-point system assembled at src/EMField.mm:236-405:
//   Cd u_ij + Cx (u_i-1,j + u_i+1,j) + Cy (u_i,j-1 + u_i,j+1) = b_ij
// with Dirichlet (values folded into b), periodic or Neumann (mirrored: the
// doubled off-diagonal of the Darwin system, src/EMField.mm:527-560)
// directions. Without a Dirichlet direction the system is singular: the
// right-hand side is projected with the left null vector (weight 1/2 at
// Neumann ends) and the solution is returned with zero mean.
//
// Method: flexible conjugate gradients in FP64 (one retained direction,
// FCG(1)) preconditioned by one FP32 V(2,2)-cycle per iteration.
//   x (FP64, warm-started from the previous step like the reference's
//   _phi_sol), r = b - A x in FP64; per iteration z = V-cycle(r) in FP32,
//   p = z + beta p_old with beta = -(z.A p_old) / (p_old.A p_old),
//   alpha = (r.p) / (p.A p), x += alpha p, r -= alpha A p,
//   until ||r||_2 / ||b||_2 <= tol (AMGCL's relative-residual criterion).
// Levels: vertex-centred coarsening (Dirichlet n -> (n-1)/2, periodic
// n -> n/2) while both directions allow it; red-black Gauss-Seidel,
// full-weighting restriction, bilinear prolongation, re-discretised coarse
// operators. Kernels per V-cycle:
//   large levels (> kSmallPoints points): one launch for the pre-smoothing
//     (two red-black sweeps in a shared-memory tile with a 6-point halo), the
//     residual and its restriction, one prolongation + post-smoothing launch;
//   all small levels: one single-CTA kernel running the rest of the V-cycle
//     in shared memory; the coarsest level is solved by a precomputed dense
//     inverse (by CG when it has more than 64 points).
// The FP64 CG passes and the convergence test run on the device (the
// first pass inside the finest post-smoother when its tiles allow, the
// second with the test in its last CTA); the host synchronises once per
// solve (it batches as many V-cycles as the previous solve needed and
// re-checks). Every kernel of the solve is launched with programmatic
// dependent launch (pdl.cuh).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "device.hpp"
#include "kernels.hpp"

namespace gample {

struct MGResult {
  int iterations = 0;        // V-cycles performed
  double rel_residual = 0;   // ||b - A x|| / ||b|| in FP64
  double rel0 = 0;           // the same for the starting guess
  double norm_b = 0;
};

class PoissonMG {
 public:
  PoissonMG(const kern::PoissonLayout& L, int nu_pre = 2, int nu_post = 2);
  ~PoissonMG();
  PoissonMG(const PoissonMG&) = delete;
  PoissonMG& operator=(const PoissonMG&) = delete;
  int unknowns() const { return n_; }
  int levels() const { return int(lv_.size()); }
  // b, x: device FP64 vectors of unknowns(); sums_b[0..1] = sum(b), sum(b^2)
  // already on the device (from kern::build_rhs). x is updated in place by
  // flexible conjugate gradients in FP64 preconditioned with one FP32 V-cycle
  // per iteration, until ||b - A x|| / ||b|| <= tol.
  MGResult solve(const double* b, const double* sums_b, double* x, double tol, int maxiter, cudaStream_t s);

  struct Level {
    int mx, my;
    int bx, by;  // 0 Dirichlet, 1 periodic, 2 Neumann (mirror)
    float cx, cy, cd;
    DeviceArray<float> u, u2, f;  // u2: output of the tiled post-smoother
    bool result_in_u2 = false;    // where the level's final correction is
  };
  const std::vector<Level>& level_info() const { return lv_; }
  int first_small_level() const { return ls_; }

 private:
  // One V-cycle on the finest level's f; with_dots: the finest post-smoother
  // also forms pass A of the flexible-CG iteration when its tiles allow
  // (returns whether it did).
  bool vcycle(cudaStream_t s, bool with_dots = false);
  void enqueue_iteration(int parity, double* x, double tol, int maxiter, cudaStream_t s);
  struct IterationGraphs {
    double* x = nullptr;
    double tol = 0;
    int maxiter = 0;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};  // [0]: one iteration ([1] unused)
    long long kernels = 0;  // kernels per graph launch
  };
  IterationGraphs iteration_graphs(double* x, double tol, int maxiter, cudaStream_t s);
  std::vector<IterationGraphs> graphs_;
  bool graphs_ok_ = true;
  const float* result(int l) const { return lv_[l].result_in_u2 ? lv_[l].u2.get() : lv_[l].u.get(); }
  kern::PoissonLayout L_;
  int n_;
  int nu_pre_, nu_post_;
  int ls_ = 0;              // first level handled by the single-CTA kernel
  size_t small_smem_ = 0;   // its shared-memory bytes
  int last_iters_ = 2;
  int bx_ = 0, by_ = 0;
  bool singular_ = false;  // no Dirichlet direction: solved in the range, zero-mean gauge
  double wsum_ = 0;        // sum of the solvability weights of the finest level
  int mx_top() const { return L_.nkx + 1; }
  int my_top() const { return L_.nky + 1; }
  std::vector<Level> lv_;
  DeviceArray<double> r64_, q_;  // FP64 residual and A p of the flexible CG iteration
  DeviceArray<double> p_[1];      // search direction (updated in place)
  DeviceArray<unsigned> ctr_;     // blocks finished in the flexible-CG update (last one tests convergence)
  DeviceArray<double> acc_;       // slotted partial sums of the flexible-CG passes (7 quantities x 32 slots)
  DeviceArray<float> coarse_inv_;  // dense inverse of the coarsest operator (small coarsest levels)
  DeviceArray<double> state_;   // [0] sum r [1] sum r^2 [2] ||b|| [3] rel res [4] done [5] iterations [6] mean r [7] initial rel res, then the flexible-CG scalars
  PinnedArray<double> host_;
};

}  // namespace gample

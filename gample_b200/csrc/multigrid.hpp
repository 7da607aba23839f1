// multigrid.hpp -- geometric multigrid for the Poisson system of the field.
//
// Replaces AMGCL's SA-AMG + CG (src/EMField.mm:20-28, 412-432, 866) for the
// 5-point system assembled at src/EMField.mm:236-405:
//   Cd u_ij + Cx (u_i-1,j + u_i+1,j) + Cy (u_i,j-1 + u_i,j+1) = b_ij
// with Dirichlet (values folded into b) or periodic directions.
//
// Method: defect correction in FP64 around an FP32 V(2,2)-cycle.
//   x (FP64, warm-started from the previous step like the reference's
//   _phi_sol), r = b - A x in FP64, e = V-cycle(r) in FP32, x += e,
//   until ||r||_2 / ||b||_2 <= tol (AMGCL's relative-residual criterion).
// Levels: vertex-centred coarsening (Dirichlet n -> (n-1)/2, periodic
// n -> n/2) while both directions allow it; red-black Gauss-Seidel
// smoothing, full-weighting restriction, bilinear prolongation,
// re-discretised coarse operators, single-block CG on the coarsest level.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "device.hpp"
#include "kernels.hpp"

namespace gample {

struct MGResult {
  int iterations = 0;        // V-cycles performed
  double rel_residual = 0;   // ||b - A x|| / ||b|| in FP64
  double norm_b = 0;
};

class PoissonMG {
 public:
  PoissonMG(const kern::PoissonLayout& L, int nu_pre = 2, int nu_post = 2);
  int unknowns() const { return n_; }
  int levels() const { return int(lv_.size()); }
  // b, x: device FP64 vectors of unknowns(); sums_b[0..1] = sum(b), sum(b^2)
  // already on the device (from kern::build_rhs). x is updated in place.
  MGResult solve(const double* b, const double* sums_b, double* x, double tol, int maxiter, cudaStream_t s);
  // One V-cycle on the FP32 rhs in level 0's f; result in level 0's u.
  void vcycle(cudaStream_t s);

  struct Level {
    int mx, my;
    bool perx, pery;
    float cx, cy, cd;
    DeviceArray<float> u, f, r;
  };
  const std::vector<Level>& level_info() const { return lv_; }

 private:
  void vcycle_level(int l, cudaStream_t s);
  kern::PoissonLayout L_;
  int n_;
  int nu_pre_, nu_post_;
  std::vector<Level> lv_;
  DeviceArray<double> sums_;     // [0] sum r, [1] sum r^2
  DeviceArray<float> cg_work_;   // coarsest-level CG vectors
  PinnedArray<double> host_;
};

}  // namespace gample

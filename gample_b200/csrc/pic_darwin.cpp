// pic_darwin.cpp -- Darwin model of the field (src/EMField.mm:447-651,
// 1138-1361): the current is split into its longitudinal part (grad psi,
// div grad psi = div J) and the rest, which drives the vector potential
// (lap A = -(4 pi / c)(J - grad psi)); delE = -(A - A_last)/(c dt) and
// delBz = curl_z A. As in the reference the corrections are output and
// diagnostics only: the push uses the electrostatic E (src/Particle.mm:627-635).
//
// The three elliptic solves use the geometric multigrid on the reference's
// operator (5-point Laplacian, doubled off-diagonals on Neumann ends,
// src/EMField.mm:497-618) to ToleranceForPoisson. Differences from the
// reference, whose AMGCL BiCGSTAB result on these singular systems is not
// reproducible (a recorded run diverged): with Neumann ends the right-hand
// side is also projected with the solvability weights (1/2 at the ends) so
// the system is consistent, solutions have zero mean, the solves start from
// the previous solution, the last column (row) of a periodic direction is
// closed through the wrap instead of being left at zero, and delEy is stored
// at the Ay node's own index (i+ngb, j+ngb+1) where the reference writes one
// row higher (src/EMField.mm:1287).
#include "pic.hpp"

namespace gample {

void EMField::setupDarwin() {
  darwin = true;
  kern::DarwinGeom& G = dgeom;
  G.perx = fbc[XMIN] == FBC_PERIODIC;
  G.pery = fbc[YMIN] == FBC_PERIODIC;
  G.nkx = dims.ngx - (G.perx ? 1 : 0);  // src/EMField.mm:484-491
  G.nky = dims.ngy - (G.pery ? 1 : 0);
  G.ngb = dims.ngb;
  G.nx = dims.nx;
  G.ny = dims.ny;
  G.dx = dx;
  G.dy = dy;
  kern::PoissonLayout& L = dlayout;
  L = layout;
  L.nkx = G.nkx;
  L.nky = G.nky;
  L.ikmin = L.jkmin = dims.ngb;
  L.periodic_x = G.perx;
  L.periodic_y = G.pery;
  L.fbc[0] = L.fbc[1] = G.perx ? kern::FBC_PERIODIC_C : kern::FBC_NEUMANN_C;
  L.fbc[2] = L.fbc[3] = G.pery ? kern::FBC_PERIODIC_C : kern::FBC_NEUMANN_C;
  dmg = std::make_unique<PoissonMG>(L);
  const size_t n = size_t(G.nkx + 1) * (G.nky + 1);
  psi.resize(n, true);
  Ax.resize(n, true);
  Ay.resize(n, true);
  lastAx.resize(n, true);
  lastAy.resize(n, true);
  drhs.resize(n, true);
  dscr.resize(8, true);
}

EMField::DarwinStats EMField::solveVectorPotential(double dt, XmlLogger* logger) {
  DarwinStats st;
  if (!darwin) return st;
  finalizeCharge();
  const kern::DarwinGeom& G = dgeom;
  const int n = (G.nkx + 1) * (G.nky + 1);
  double* d = dscr.get();
  auto prepare = [&]() {
    // zero mean as the reference (src/EMField.mm:1186-1191), then the
    // weighted projection that makes a Neumann system consistent
    kern::vec_sums(drhs.get(), n, d, stream);
    kern::subtract_mean(drhs.get(), n, d, stream);
    if (!(G.perx && G.pery)) kern::darwin_weighted_project(drhs.get(), G, d + 2, stream);
    kern::vec_sums(drhs.get(), n, d, stream);
  };
  kern::darwin_div_rhs(jx.get(), jy.get(), G, drhs.get(), stream);
  prepare();
  MGResult r0 = dmg->solve(drhs.get(), d, psi.get(), tol, maxiter, stream);
  kern::darwin_a_rhs(jx.get(), psi.get(), G, 0, drhs.get(), stream);
  prepare();
  MGResult r1 = dmg->solve(drhs.get(), d, Ax.get(), tol, maxiter, stream);
  kern::darwin_a_rhs(jy.get(), psi.get(), G, 1, drhs.get(), stream);
  prepare();
  MGResult r2 = dmg->solve(drhs.get(), d, Ay.get(), tol, maxiter, stream);
  kern::darwin_fields(Ax.get(), Ay.get(), lastAx.get(), lastAy.get(), G, phys::c * dt, delEx.get(), delEy.get(),
                      delBz.get(), stream);
  GP_CUDA(cudaMemcpyAsync(lastAx.get(), Ax.get(), size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  GP_CUDA(cudaMemcpyAsync(lastAy.get(), Ay.get(), size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  const MGResult* r[3] = {&r0, &r1, &r2};
  for (int q = 0; q < 3; ++q) {
    st.iters[q] = r[q]->iterations;
    st.errors[q] = r[q]->rel_residual;
  }
  last_darwin = st;
  if (logger && logger->on())  // src/EMField.mm:1351-1359
    logger->logSection("solveVectorPotential", {{"decompose_iteration", std::to_string(st.iters[0])},
                                                {"decompose_error", fmtSci(float(st.errors[0]), 6)},
                                                {"solveAx_iteration", std::to_string(st.iters[1])},
                                                {"solveAx_error", fmtSci(float(st.errors[1]), 6)},
                                                {"solveAy_iteration", std::to_string(st.iters[2])},
                                                {"solveAy_error", fmtSci(float(st.errors[2]), 6)}});
  return st;
}

}  // namespace gample

// pic_moment.cpp -- Moment host object (src/Moment.{h,mm}).
#include "pic.hpp"

namespace gample {

Moment::Moment(const Init& init, cudaStream_t s) : stream(s) {
  const ParamForField& fp = init.paramForField;
  order_ = fp.weightOrder;
  dims_.ngx = fp.ngx;
  dims_.ngy = fp.ngy;
  dims_.ngb = fp.ngb;
  dims_.nx = fp.ngx + 2 * fp.ngb;
  dims_.ny = fp.ngy + 2 * fp.ngb;
  n_rho_ = size_t(dims_.nx + 1) * (dims_.ny + 1);
  out.resize(kCount * n_rho_, true);
  acc.resize(kCount * n_rho_, true);
}

void Moment::integrateMoments(Particle& p, const EMField& fld) {
  // src/Moment.mm:250-251: scale = w / (dx dy) in FP32
  const float scale = p.w / (fld.dx * fld.dy);
  kern::moments(order_, dims_, p.arrays(), p.cnt.get(), p.n_bound, scale, p.m, acc.get(), out.get(), stream);
  species = p.index;
}

}  // namespace gample

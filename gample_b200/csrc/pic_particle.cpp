// pic_particle.cpp -- Particle host object (one species).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "pic.hpp"

namespace gample {

void Particle::Buffer::alloc(size_t n) {
  cell.resize(n);
  ox.resize(n);
  oy.resize(n);
  vx.resize(n);
  vy.resize(n);
  vz.resize(n);
}

kern::ParticleArrays Particle::Buffer::view() const {
  return kern::ParticleArrays{cell.get(), ox.get(), oy.get(), vx.get(), vy.get(), vz.get()};
}

Particle::Particle(const Init& init, int s, cudaStream_t st) : stream(st), host_cnt_(1) {
  if (s < 0 || s >= int(init.paramForParticle.size())) throw ConfigError("species index out of range");
  const ParamForParticle& pp = init.paramForParticle[s];
  const ParamForField& fp = init.paramForField;
  index = s;
  pName = pp.pName;
  pNumMax = init.paramForComputing.pNumMax;
  m = float(pp.m);
  q = float(pp.q);
  w = float(pp.w);
  order = fp.weightOrder;
  boris = fp.BorisOrder;
  dx_ = fp.dx;
  dy_ = fp.dy;
  sort_interval = init.paramForComputing.sortInterval;
  if (boris != 2 && boris != 4 && boris != 6) throw ConfigError("BorisOrder must be 2, 4 or 6");
  // src/Particle.mm:459-514 (an unknown BC string is fatal there too)
  auto codes = init.particleBCCodes();
  for (int w2 = 0; w2 < 4; ++w2) {
    if (codes[w2] == PBC_INVALID) throw ConfigError("[FatalError] invalid particle boundary");
    pbc[w2] = codes[w2];
  }
  // src/Particle.mm:544-547
  if (pp.pNum > pNumMax) throw ConfigError("pNum > pNumMax for " + pName);
  if (fp.ngx + 2 * fp.ngb + 2 > 65535 || fp.ngy + 2 * fp.ngb + 2 > 32767)
    throw ConfigError("grid too large for the packed cell index");
  dims_.ngx = fp.ngx;
  dims_.ngy = fp.ngy;
  dims_.ngb = fp.ngb;
  dims_.nx = fp.ngx + 2 * fp.ngb;
  dims_.ny = fp.ngy + 2 * fp.ngb;
  const size_t cap = pNumMax;
  buf[0].alloc(cap);
  buf[1].alloc(cap);
  dead_bits.resize((cap + 31) / 32 + 1, true);
  scratch.resize(kern::compact_scratch_words(uint32_t(cap)), true);
  sort_scratch.resize(kern::sort_scratch_words(dims_), true);
  cnt.resize(1, true);
  n_bound = 0;
  // The reference loads pNum particles on the CPU here (src/Particle.mm:568-597)
  // from std::random_device and Collision's init then overwrites them
  // (src/Collision.mm:315-336); the build loads only through Collision.
}

kern::ParticleArrays Particle::arrays() const { return buf[cur].view(); }

kern::SpeciesCounters Particle::counters() {
  GP_CUDA(cudaMemcpyAsync(host_cnt_.get(), cnt.get(), sizeof(kern::SpeciesCounters), cudaMemcpyDeviceToHost,
                          stream));
  GP_CUDA(cudaStreamSynchronize(stream));
  return host_cnt_[0];
}

uint32_t Particle::pNum() {
  uint32_t n = counters().n;
  n_bound = n;
  return n;
}

void Particle::setPNum(uint32_t n) {
  if (n > pNumMax) throw std::invalid_argument("pNum > pNumMax");
  kern::SpeciesCounters c{};
  c.n = n;
  GP_CUDA(cudaMemcpyAsync(cnt.get(), &c, sizeof(c), cudaMemcpyHostToDevice, stream));
  GP_CUDA(cudaStreamSynchronize(stream));
  n_bound = n;
  n_appended = 0;
}

// Host AoS records stream through the spare half of the double buffer (free
// between cycles): chunks that fit in one of its arrays, so that neither
// direction allocates device memory.
namespace {
kern::ParticleArrays offset_view(kern::ParticleArrays p, uint32_t off) {
  return kern::ParticleArrays{p.cell + off, p.ox + off, p.oy + off, p.vx + off, p.vy + off, p.vz + off};
}
}  // namespace

uint32_t Particle::stage_records() const {
  return uint32_t(std::max<size_t>(1, size_t(pNumMax) * sizeof(int32_t) / sizeof(kern::ParticleStateAoS)));
}

// Two staging areas (the spare buffer's cell and ox arrays) alternate, and
// the copies run on a second stream, so that the copy of one chunk overlaps
// the layout conversion of the previous one.
namespace {
struct Staging {
  cudaStream_t xfer = nullptr;
  cudaEvent_t ev[5] = {};  // [0, 2): copy done per area, [2, 4): conversion done per area, [4]: start
  Staging() {
    try {
      GP_CUDA(cudaStreamCreateWithFlags(&xfer, cudaStreamNonBlocking));
      for (auto& e : ev) GP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    } catch (...) {
      release();
      throw;
    }
  }
  ~Staging() { release(); }
  void release() {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (xfer) cudaStreamDestroy(xfer);
  }
};
}  // namespace

void Particle::upload_aos(const kern::ParticleStateAoS* host, uint32_t n) {
  if (n > pNumMax) throw std::invalid_argument("pNum > pNumMax");
  kern::ParticleStateAoS* stage[2] = {reinterpret_cast<kern::ParticleStateAoS*>(buf[1 - cur].cell.get()),
                                      reinterpret_cast<kern::ParticleStateAoS*>(buf[1 - cur].ox.get())};
  const uint32_t chunk = stage_records();
  Staging st;
  GP_CUDA(cudaEventRecord(st.ev[4], stream));  // earlier work on the spare buffer
  GP_CUDA(cudaStreamWaitEvent(st.xfer, st.ev[4], 0));
  int i = 0;
  for (uint32_t off = 0; off < n; off += chunk, ++i) {
    const int a = i & 1;
    const uint32_t m = std::min(chunk, n - off);
    if (i >= 2) GP_CUDA(cudaStreamWaitEvent(st.xfer, st.ev[2 + a], 0));  // area read by the conversion
    GP_CUDA(cudaMemcpyAsync(stage[a], host + off, size_t(m) * sizeof(*host), cudaMemcpyHostToDevice, st.xfer));
    GP_CUDA(cudaEventRecord(st.ev[a], st.xfer));
    GP_CUDA(cudaStreamWaitEvent(stream, st.ev[a], 0));
    kern::aos_to_soa(stage[a], m, offset_view(arrays(), off), dims_.nx, dims_.ny, stream);
    GP_CUDA(cudaEventRecord(st.ev[2 + a], stream));
  }
  GP_CUDA(cudaStreamSynchronize(stream));
  GP_CUDA(cudaStreamSynchronize(st.xfer));
  setPNum(n);
  needs_sort = true;
  random_order = true;
}

void Particle::download_aos(kern::ParticleStateAoS* host, uint32_t n) {
  if (!n) return;
  kern::ParticleStateAoS* stage[2] = {reinterpret_cast<kern::ParticleStateAoS*>(buf[1 - cur].cell.get()),
                                      reinterpret_cast<kern::ParticleStateAoS*>(buf[1 - cur].ox.get())};
  const uint32_t chunk = stage_records();
  Staging st;
  int i = 0;
  for (uint32_t off = 0; off < n; off += chunk, ++i) {
    const int a = i & 1;
    const uint32_t m = std::min(chunk, n - off);
    if (i >= 2) GP_CUDA(cudaStreamWaitEvent(stream, st.ev[a], 0));  // area read by the copy
    kern::soa_to_aos(offset_view(arrays(), off), m, stage[a], stream);
    GP_CUDA(cudaEventRecord(st.ev[2 + a], stream));
    GP_CUDA(cudaStreamWaitEvent(st.xfer, st.ev[2 + a], 0));
    GP_CUDA(cudaMemcpyAsync(host + off, stage[a], size_t(m) * sizeof(*host), cudaMemcpyDeviceToHost, st.xfer));
    GP_CUDA(cudaEventRecord(st.ev[a], st.xfer));
  }
  GP_CUDA(cudaStreamSynchronize(st.xfer));
  GP_CUDA(cudaStreamSynchronize(stream));
}

void Particle::sort(Particle* lender) {
  // freshly loaded or uploaded particles are in random order: staged records
  // (in sector-sized records when another species lends its idle spare buffer)
  const kern::ParticleArrays extra = lender ? lender->buf[1 - lender->cur].view() : kern::ParticleArrays{};
  const uint32_t extra_cap = lender && lender->stream == stream ? lender->pNumMax : 0u;
  if (!(random_order && kern::sort_by_cell_staged(dims_, buf[cur].view(), buf[1 - cur].view(), pNumMax, extra,
                                                  extra_cap, cnt.get(), sort_scratch.get(), n_bound, stream))) {
    GP_CUDA(cudaEventRecord(ev_sort[0].get(), stream));
    kern::sort_by_cell(dims_, buf[cur].view(), buf[1 - cur].view(), cnt.get(), sort_scratch.get(), n_bound, stream);
    GP_CUDA(cudaEventRecord(ev_sort[1].get(), stream));
    sort_pending_timing = !random_order;  // the periodic re-sort of nearly sorted particles
    cur = 1 - cur;
  }
  random_order = false;
  needs_sort = false;
  cycles_since_sort = 0;
}

void Particle::update(double dt, EMField& fld, bool fused_deposit) {
  kern::PushConsts c{};
  // src/Particle.mm:617-621
  c.constE = float(0.5 * double(q) * dt / double(m));
  c.constB = float(0.5 * double(q) * dt / double(m) / phys::c);
  c.constX = float(dt / double(fld.dx));
  c.constY = float(dt / double(fld.dy));
  for (int i = 0; i < 4; ++i) c.bc[i] = pbc[i];
  c.scale = float(double(q * w) / (dx_ * dy_));  // src/Particle.mm:540
  c.bz_uniform = fld.bz_value;
  c.ke_half_m = 0.5 * double(m);
  c.ke_w = double(w);
  fld.species_scale[index] = c.scale;
  if (fused_deposit) fld.charge_dirty = true;
  last_dt = dt;
  kern::FieldPtrs f{fld.Ex.get(), fld.Ey.get(), fld.Bz.get()};
  const kern::FieldMaps* maps = fld.pushMaps();
  lean_push = fused_deposit && !fld.det && !fld.current && fld.bz_uniform;
  const int nv = tune_variants();
  tune_used = push_variant;
  if (lean_push && tune_step >= 0 && tune_step < 2 * nv)  // mirrored order: 0 1 .. nv-1 nv-1 .. 1 0
    tune_used = tune_variant(tune_step < nv ? tune_step : 2 * nv - 1 - tune_step);
  c.no_tables = tune_used.tables ? 0 : 1;
  GP_CUDA(cudaEventRecord(ev_push[0].get(), stream));
  kern::push(order, boris, fused_deposit, fld.det, fld.current, fld.bz_uniform, fld.dims, arrays(), f, c,
             fld.targets(index), cnt.get(), dead_bits.get(), n_bound, stream, maps, tune_used.per);
  GP_CUDA(cudaEventRecord(ev_push[1].get(), stream));
  n_pushed = n_bound;
  n_appended = 0;  // the push zeroed the device's n_injected
  cost_policy = !fld.det;
  ++cycles_since_sort;
}

FlowStats Particle::reduce(XmlLogger* logger) {
  reduceLaunch();
  GP_CUDA(cudaStreamSynchronize(stream));
  return reduceFinish(logger);
}

void Particle::reduceLaunch() {
  kern::compact(arrays(), cnt.get(), dead_bits.get(), scratch.get(), n_bound, stream);
  GP_CUDA(cudaMemcpyAsync(host_cnt_.get(), cnt.get(), sizeof(kern::SpeciesCounters), cudaMemcpyDeviceToHost,
                          stream));
}

FlowStats Particle::reduceFinish(XmlLogger* logger) {
  const kern::SpeciesCounters c = host_cnt_[0];
  if (c.err)
    throw std::runtime_error("push: " + std::to_string(c.err) +
                             " field-staging waits timed out (tiles were loaded per thread instead)");
  FlowStats fs;
  // src/Particle.mm:915: counts in units of the charge sign
  const int unit = int(q / float(phys::ec));
  for (int i = 0; i < 4; ++i) {
    pinum[i] = int(c.wall[i]) * unit;
    fs.pinum[i] = pinum[i];
  }
  fs.particleNumber = c.n;
  fs.pulledPtclNum = c.n_pulled;
  fs.invalid = c.invalid;
  fs.totalKineticEnergy = c.ke;
  fs.totalKEincrement = c.ke - lastKE;
  lastKE = c.ke;
  last_pulled = c.n_pulled;
  n_bound = c.n;
  // Sort policy: a fixed interval, or when the particles pushed outside
  // their chunk's shared-memory window (spread out by drift, compaction and
  // injection) exceed those of the first push after the last sort by 2% of
  // the live count.
  if (cycles_since_sort == 1) slow_after_sort = c.n_slow;
  // the caller synchronised the stream: this cycle's push (and a sort before
  // it) have completed
  if (sort_pending_timing) {
    // a one-off slow sort (a busy GPU) must not stretch the cadence for
    // long: each timing may at most double the previous one
    float t = 0;
    GP_CUDA(cudaEventElapsedTime(&t, ev_sort[0].get(), ev_sort[1].get()));
    last_sort_ms = sort_timed ? std::min(t, 2.0f * last_sort_ms) : t;
    sort_timed = true;
    sort_pending_timing = false;
  }
  if (cycles_since_sort >= 1 && n_pushed > 0) {
    float push_ms = 0;
    GP_CUDA(cudaEventElapsedTime(&push_ms, ev_push[0].get(), ev_push[1].get()));
    const double per = double(push_ms) / double(n_pushed);
    const int nv = tune_variants();
    // the first sort is behind us: tune, unless the cells are so full that the
    // defaults are known to win (at 256 particles per cell the 1024-particle
    // chunks and the table-less order-3 gather were measured slower)
    if (lean_push && tune_step < 0 && cycles_since_sort == 1)
      tune_step = double(n_pushed) < kTuneBelowPpc * double(dims_.ngx) * double(dims_.ngy) ? 0 : (1 << 20);
    if (lean_push && tune_step >= 0 && tune_step < 2 * nv) {
      tune_ms[tune_step < nv ? tune_step : 2 * nv - 1 - tune_step] += per;
      if (++tune_step == 2 * nv) {
        int best = 0;
        for (int v = 1; v < nv; ++v)
          if (tune_ms[v] < tune_ms[best]) best = v;
        push_variant = tune_variant(best);
        // the drift since the sort restarts from the kept variant's mean
        base_ms_per_particle = 0.5 * tune_ms[best];
        excess_ms = 0;
      }
    } else if (cycles_since_sort == 1) {
      base_ms_per_particle = per;
      excess_ms = 0;
    } else if (per < base_ms_per_particle) {
      base_ms_per_particle = per;  // a slow first push must not hide the drift
    } else {
      excess_ms += double(push_ms) - base_ms_per_particle * double(n_pushed);
    }
  }
  if (sort_interval > 0) {
    needs_sort = needs_sort || cycles_since_sort >= sort_interval;
  } else if (cost_policy) {
    // before the first periodic sort has been timed: its cost estimated
    // from the particle count (30 ps per particle, measured: 22-34 ps)
    const double sort_ms = sort_timed ? double(last_sort_ms) : std::max(0.02, 3e-8 * double(c.n));
    needs_sort = needs_sort || excess_ms >= sort_ms;
  } else {
    needs_sort = needs_sort || double(c.n_slow) > double(slow_after_sort) + 0.02 * double(c.n);
  }
  if (logger && logger->on()) {
    // src/Particle.mm:990-1001
    std::map<std::string, std::string> data = {
        {"particleNumber", std::to_string(fs.particleNumber)},
        {"pulledPtclNum", std::to_string(fs.pulledPtclNum)},
        {"Xmin", std::to_string(fs.pinum[0])},
        {"Xmax", std::to_string(fs.pinum[1])},
        {"Ymin", std::to_string(fs.pinum[2])},
        {"Ymax", std::to_string(fs.pinum[3])},
        {"totalKineticEnergy", fmtSci(float(fs.totalKineticEnergy * phys::ergtoev), 6)},
        {"totalKEincrement", fmtSci(float(fs.totalKEincrement * phys::ergtoev), 6)},
    };
    if (fs.invalid) data["invalidPtclNum"] = std::to_string(fs.invalid);
    logger->logSection("flowout_" + pName, data);
  }
  return fs;
}

void Particle::integrateChargeDensity(EMField& fld, bool injected_only) {
  const float scale = float(double(q * w) / (dx_ * dy_));  // src/Particle.mm:540
  fld.species_scale[index] = scale;
  fld.charge_dirty = true;
  // the injected particles' deposit needs blocks for the appended particles only
  kern::deposit(order, fld.det, fld.current, fld.dims, arrays(), scale, fld.targets(index), cnt.get(),
                injected_only ? std::min(n_appended, n_bound) : n_bound, injected_only, stream);
}

}  // namespace gample

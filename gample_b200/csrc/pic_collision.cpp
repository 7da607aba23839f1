// pic_collision.cpp -- Collision host object: initial load and sources.
#include <cmath>
#include <stdexcept>

#include "pic.hpp"

namespace gample {

namespace {

void range_of(const std::vector<double>& gen, double L, float& lo, float& hi) {
  // src/Collision.mm:245-258: a negative first entry means the whole domain.
  if (gen.empty() || gen[0] < 0) {
    lo = 0.0f;
    hi = float(L);
  } else {
    lo = float(gen[0]);
    hi = float(gen.size() > 1 ? gen[1] : gen[0]);
  }
}
float comp(const std::vector<double>& v, int i) { return i < int(v.size()) ? float(v[i]) : 0.0f; }

Particle* find(std::vector<Particle*>& ps, const std::string& name) {
  for (auto* p : ps)
    if (p->pName == name) return p;
  return nullptr;
}

}  // namespace

double Collision::uniform01() {
  // minstd_rand: x <- 48271 x mod (2^31 - 1); generate_canonical with two
  // 30-bit draws, as libc++ implements uniform_real_distribution<double>.
  auto next = [&]() {
    minstd_ = (minstd_ * 48271ULL) % 2147483647ULL;
    return minstd_;
  };
  const double Rp = 2147483646.0;
  double S = double(next() - 1);
  S += double(next() - 1) * Rp;
  return S / (Rp * Rp);
}

void Collision::ensure_states(uint32_t n) {
  if (n <= initialized) return;
  if (n > states.size()) {
    size_t cap = states.size() ? states.size() : 1024;
    while (cap < n) cap *= 2;
    states.grow(cap, initialized, stream);
  }
  kern::seed_rng(states.get(), master_seed, initialized, n, stream);
  initialized = n;
}

// The initial load (src/Collision.mm:189-336): species 0's count of
// electron + ion pairs from the splitmix64/PCG32 streams of master_seed,
// overwriting both species.
void Collision::loadInitial(std::vector<Particle*>& ptcls) {
  const ParamForField& fp = init_.paramForField;
  const auto& pp = init_.paramForParticle;
  Particle* ele = find(ptcls, "electron");
  Particle* ion = nullptr;
  for (auto* p : ptcls)
    if (p->pName != "electron") ion = p;  // the last non-electron species (src/Collision.mm:305-313)
  if (!ele || !ion) throw ConfigError("the initial load needs an \"electron\" species and one ion species");
  // src/Collision.mm:220-233: generator of species 0
  const int genType = Init::loadGenType(pp[0].genType);
  if (genType < 0) throw ConfigError("unknown GenerateType " + pp[0].genType);
  kern::GenParams prm{};
  const uint32_t addn = pp[0].pNum;  // src/Collision.mm:242
  range_of(pp[0].genX, fp.dx * fp.ngx, prm.Xmin, prm.Xmax);
  range_of(pp[0].genY, fp.dy * fp.ngy, prm.Ymin, prm.Ymax);
  for (size_t s = 0; s < pp.size(); ++s) {
    const float vth = float(std::sqrt(2 * phys::kb * pp[s].genT / pp[s].m));
    if (pp[s].pName == "electron") {
      for (int d = 0; d < 3; ++d) prm.ele_genU[d] = comp(pp[s].genU, d);
      for (int d = 0; d < 3; ++d) prm.ele_sinU[d] = comp(pp[s].sinU, d);
      prm.ele_vth = vth;
    } else {
      for (int d = 0; d < 3; ++d) prm.ion_genU[d] = comp(pp[s].genU, d);
      for (int d = 0; d < 3; ++d) prm.ion_sinU[d] = comp(pp[s].sinU, d);
      prm.ion_vth = vth;
    }
  }
  prm.dx = float(fp.dx);
  prm.dy = float(fp.dy);
  prm.ngb = float(fp.ngb);
  for (int d = 0; d < 3; ++d) prm.sin_on |= (prm.ele_sinU[d] != 0.0f || prm.ion_sinU[d] != 0.0f) ? 1 : 0;
  if (addn > ele->pNumMax || addn > ion->pNumMax) throw ConfigError("pNum > pNumMax in the initial load");
  ensure_states(addn);
  ele->setPNum(0);
  ion->setPNum(0);
  kern::ParticleArrays ia = ion->arrays();
  kern::generate(genType, addn, prm, states.get(), ele->arrays(), ele->cnt.get(), &ia, ion->cnt.get(), stream);
  GP_CUDA(cudaStreamSynchronize(stream));
  ele->n_bound = addn;
  ion->n_bound = addn;
  ele->n_appended = addn;
  ion->n_appended = addn;
}

void Collision::reload(uint64_t seed, std::vector<Particle*>& ptcls) {
  master_seed = seed;
  initialized = 0;  // every stream restarts from the new master seed
  minstd_ = 1;
  loadInitial(ptcls);
}

Collision::Collision(const Init& init, std::vector<Particle*>& ptcls, cudaStream_t st) : stream(st), init_(init) {
  master_seed = init.paramForComputing.masterSeed;  // 0 in the reference (src/Collision.mm:283-294)
  const ParamForField& fp = init.paramForField;
  const auto& pp = init.paramForParticle;
  if (pp.empty()) throw ConfigError("no particle species");
  loadInitial(ptcls);

  // Sources: src/Collision.mm:365-458 (one artificial-ionization and one
  // hollow-cathode source; with several, the last one of each kind is used).
  for (size_t i = 0; i < init.particleSources.size(); ++i) {
    const int g = Init::sourceGenType(init.particleSources[i].genType);
    if (g >= 0 && g <= 2) {
      existAI_ = true;
      ai_source_ = int(i);
    } else if (g == 3) {
      existHC_ = true;
      hc_source_ = int(i);
    } else if (g == 7) {
      reflux_sources_.push_back(int(i));
    }
  }
}

int Collision::artificialIonization(double dt, std::vector<Particle*>& ptcls, XmlLogger* logger) {
  if (!existAI_) return 0;
  const SourceForParticle& src = init_.particleSources[ai_source_];
  const ParamForField& fp = init_.paramForField;
  Particle* ele = find(ptcls, "electron");
  Particle* ion = find(ptcls, src.pName);
  if (!ele || !ion) throw ConfigError("artificial ionization needs the electron and " + src.pName + " species");
  kern::GenParams prm{};
  range_of(src.genX, fp.dx * fp.ngx, prm.Xmin, prm.Xmax);
  range_of(src.genY, fp.dy * fp.ngy, prm.Ymin, prm.Ymax);
  for (int d = 0; d < 3; ++d) {
    prm.ele_genU[d] = comp(src.genU_ele, d);
    prm.ion_genU[d] = comp(src.genU, d);
  }
  prm.ele_vth = float(std::sqrt(2 * phys::kb * src.genT_ele / phys::me));
  double mion = 0;
  for (const auto& p : init_.paramForParticle)
    if (p.pName == src.pName) mion = p.m;
  prm.ion_vth = float(std::sqrt(2 * phys::kb * src.genT / mion));
  prm.dx = float(fp.dx);
  prm.dy = float(fp.dy);
  prm.ngb = float(fp.ngb);
  // src/Collision.mm:482-487: stochastic rounding of src/w*dt
  const double addn_d = double(float(src.src) / ele->w) * dt;
  uint32_t addn = (uniform01() < addn_d - int(addn_d)) ? uint32_t(int(addn_d) + 1) : uint32_t(int(addn_d));
  if (logger) logger->logSection("artificialIonization", {{"addn_injected", std::to_string(addn)}});
  if (ele->n_bound + addn > ele->pNumMax || ion->n_bound + addn > ion->pNumMax) {
    // bounds are exact after reduce(); re-read before failing
    if (ele->pNum() + addn > ele->pNumMax || ion->pNum() + addn > ion->pNumMax)
      throw std::runtime_error("[FatalError] pNum+addn > pNumMax");
  }
  ensure_states(addn);
  const int g = Init::sourceGenType(src.genType);
  kern::ParticleArrays ia = ion->arrays();
  kern::generate(g, addn, prm, states.get(), ele->arrays(), ele->cnt.get(), &ia, ion->cnt.get(), stream);
  ele->n_bound += addn;
  ion->n_bound += addn;
  ele->n_appended += addn;
  ion->n_appended += addn;
  return int(addn);
}

int Collision::hollowCathode(double dt, std::vector<Particle*>& ptcls, XmlLogger* logger) {
  (void)dt;
  if (!existHC_) return 0;
  const SourceForParticle& src = init_.particleSources[hc_source_];
  const ParamForField& fp = init_.paramForField;
  Particle* ele = find(ptcls, "electron");
  if (!ele) throw ConfigError("hollow cathode needs the electron species");
  const int wall = int(src.src);
  int addn = 0;
  for (auto* p : ptcls) addn -= p->pinum[wall];  // src/Collision.mm:592-601
  if (ele->n_bound + uint32_t(addn > 0 ? addn : 0) > ele->pNumMax) {
    if (ele->pNum() + uint32_t(addn > 0 ? addn : 0) > ele->pNumMax) throw std::runtime_error("[HC] exceeded maximum pNum");
  }
  if (addn <= 0) {
    if (logger)
      logger->logSection("hollowCathode", {{"addn_neglected", std::to_string(-addn)}, {"addn_injected", "0"}});
    return 0;
  }
  if (logger)
    logger->logSection("hollowCathode", {{"addn_neglected", "0"}, {"addn_injected", std::to_string(addn)}});
  kern::GenParams prm{};
  range_of(src.genX, fp.dx * fp.ngx, prm.Xmin, prm.Xmax);
  range_of(src.genY, fp.dy * fp.ngy, prm.Ymin, prm.Ymax);
  for (int d = 0; d < 3; ++d) prm.ele_genU[d] = comp(src.genU, d);
  prm.ele_vth = float(std::sqrt(2 * phys::kb * src.genT / phys::me));
  prm.dx = float(fp.dx);
  prm.dy = float(fp.dy);
  prm.ngb = float(fp.ngb);
  ensure_states(uint32_t(addn));
  kern::generate(3, uint32_t(addn), prm, states.get(), ele->arrays(), ele->cnt.get(), nullptr, nullptr, stream);
  ele->n_bound += uint32_t(addn);
  ele->n_appended += uint32_t(addn);
  return addn;
}

int Collision::fluxReinjection(double dt, std::vector<Particle*>& ptcls, XmlLogger* logger) {
  int total = 0;
  const ParamForField& fp = init_.paramForField;
  for (int i : reflux_sources_) {
    const SourceForParticle& src = init_.particleSources[i];
    Particle* p = find(ptcls, src.pName);
    if (!p) throw ConfigError("source species " + src.pName + " not found");
    const uint32_t addn = p->last_pulled;
    if (p->n_bound + addn > p->pNumMax) throw std::runtime_error("[FatalError] pNum+addn > pNumMax");
    kern::RefluxParams prm{};
    prm.Xmin = (src.genX.empty() || src.genX[0] < 0) ? 0.0f : float(src.genX[0]);
    range_of(src.genY, fp.dy * fp.ngy, prm.Ymin, prm.Ymax);
    double mass = 0;
    for (const auto& sp : init_.paramForParticle)
      if (sp.pName == src.pName) mass = sp.m;
    prm.vth = float(std::sqrt(2 * phys::kb * src.genT / mass));
    prm.u0 = comp(src.genU, 0);
    prm.u1 = comp(src.genU, 1);
    prm.u2 = comp(src.genU, 2);
    prm.dt = float(dt);
    prm.dx = float(fp.dx);
    prm.dy = float(fp.dy);
    prm.ngb = float(fp.ngb);
    ensure_states(addn);
    kern::reflux(addn, prm, states.get(), p->arrays(), p->cnt.get(), stream);
    p->n_bound += addn;
    p->n_appended += addn;
    total += int(addn);
    if (logger) logger->logSection("fluxReinjection_" + p->pName, {{"addn_injected", std::to_string(addn)}});
  }
  return total;
}

}  // namespace gample

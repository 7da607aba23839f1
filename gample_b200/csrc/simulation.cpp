// simulation.cpp -- time loop of the reference's main() (src/main.mm).
#include "simulation.hpp"

#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <stdexcept>

#include "fileio.hpp"

namespace gample {

Simulation::Simulation(const Init& in, const std::string& log_name, bool fused_step) : init(in), fused(fused_step) {
  GP_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  if (!log_name.empty()) logger = std::make_unique<XmlLogger>(log_name, "cycle,time,phi1,Ex1,Ey1");
  const int ns = init.flagForEquation.Particle;
  if (ns < 1 || ns > int(init.paramForParticle.size()) || ns > 4)
    throw ConfigError("FlagForEquation.Particle must be between 1 and the number of listed species (max 4)");
  for (int s = 0; s < ns; ++s) {  // src/main.mm:96-106
    particles.push_back(std::make_unique<Particle>(init, s, stream));
    ptrs.push_back(particles.back().get());
  }
  field = std::make_unique<EMField>(init, stream, ns);               // src/main.mm:108-113
  moment = std::make_unique<Moment>(init, stream);                   // src/main.mm:114-115
  collision = std::make_unique<Collision>(init, ptrs, stream);        // src/main.mm:117-122
  last_flow.resize(ns);
  cycle_no = init.paramForTimeIntegration.Start;
  struct stat st {};
  file_output = logger && stat("bin", &st) == 0 && S_ISDIR(st.st_mode);
  time = cycle_no * init.paramForTimeIntegration.TimeStep;
}

Simulation::~Simulation() {
  for (auto& e : events_) {
    cudaEventDestroy(e.second.first);
    cudaEventDestroy(e.second.second);
  }
  for (auto& e : timed_) {
    cudaEventDestroy(e.second.first);
    cudaEventDestroy(e.second.second);
  }
  for (auto e : event_pool_) cudaEventDestroy(e);
  particles.clear();
  field.reset();
  collision.reset();
  if (stream) cudaStreamDestroy(stream);
}

void Simulation::set_profiling(bool on) { profiling_ = on; }

void Simulation::mark(int phase, bool begin) {
  if (!profiling_) return;
  if (begin) {
    GP_CUDA(cudaEventCreate(&open_));
    GP_CUDA(cudaEventRecord(open_, stream));
  } else {
    cudaEvent_t e;
    GP_CUDA(cudaEventCreate(&e));
    GP_CUDA(cudaEventRecord(e, stream));
    events_.push_back({phase, {open_, e}});
    open_ = nullptr;
  }
}

cudaEvent_t Simulation::take_event() {
  if (!event_pool_.empty()) {
    cudaEvent_t e = event_pool_.back();
    event_pool_.pop_back();
    return e;
  }
  cudaEvent_t e;
  GP_CUDA(cudaEventCreate(&e));
  return e;
}

void Simulation::tic(const std::string& name) {
  if (!logger || !logger->on()) return;
  cudaEvent_t a = take_event();
  GP_CUDA(cudaEventRecord(a, stream));
  timed_.push_back({name, {a, nullptr}});
}

void Simulation::toc() {
  if (!logger || !logger->on() || timed_.empty() || timed_.back().second.second) return;
  cudaEvent_t b = take_event();
  GP_CUDA(cudaEventRecord(b, stream));
  timed_.back().second.second = b;
}

// elapsedTime (us per timed call) and memoryUsage (kB) of a logged cycle,
// src/main.mm:237-248. The reference's host clock around synchronous Metal
// dispatches measures the device work; here each call is bracketed by events
// on the run's stream. memoryUsage: residentSetSize is the host RSS;
// physicalFootprint adds the device memory the process holds in its pool
// (the reference's unified-memory footprint counts its GPU buffers).
void Simulation::log_resources() {
  if (!logger || !logger->on()) return;
  GP_CUDA(cudaStreamSynchronize(stream));
  std::map<std::string, std::string> et;
  for (auto& e : timed_) {
    float ms = 0;
    if (e.second.second) GP_CUDA(cudaEventElapsedTime(&ms, e.second.first, e.second.second));
    et[e.first] = std::to_string(static_cast<long long>(double(ms) * 1e3));
    event_pool_.push_back(e.second.first);
    if (e.second.second) event_pool_.push_back(e.second.second);
  }
  timed_.clear();
  logger->logSection("elapsedTime", et);
  long rss_pages = 0;
  if (FILE* f = std::fopen("/proc/self/statm", "r")) {
    long total = 0;
    if (std::fscanf(f, "%ld %ld", &total, &rss_pages) != 2) rss_pages = 0;
    std::fclose(f);
  }
  const unsigned long long rss_kb = static_cast<unsigned long long>(rss_pages) * sysconf(_SC_PAGESIZE) / 1024;
  unsigned long long dev_bytes = 0;
  int dev = 0;
  cudaMemPool_t pool;
  if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    size_t used = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess) dev_bytes = used;
  }
  logger->logSection("memoryUsage", {{"physicalFootprint", std::to_string(rss_kb + dev_bytes / 1024)},
                                     {"residentSetSize", std::to_string(rss_kb)}});
}

void Simulation::phase_times(double out[PH_COUNT]) {
  GP_CUDA(cudaStreamSynchronize(stream));
  for (auto& e : events_) {
    float ms = 0;
    GP_CUDA(cudaEventElapsedTime(&ms, e.second.first, e.second.second));
    acc_[e.first] += ms;
    cudaEventDestroy(e.second.first);
    cudaEventDestroy(e.second.second);
  }
  events_.clear();
  for (int i = 0; i < PH_COUNT; ++i) out[i] = acc_[i];
}

void Simulation::initialize() {
  // src/main.mm:124-147: the logger is still switched off here.
  const int start = init.paramForTimeIntegration.Start;
  if (start != 0 && !loadProgress(start, ptrs, init)) throw std::runtime_error("[Fatal] restart failed.");
  // cell order for the freshly loaded particles; the species sort one after
  // the other, so each may use the next one's idle spare buffer
  for (size_t i = 0; i < ptrs.size(); ++i)
    if (ptrs[i]->needs_sort) ptrs[i]->sort(ptrs.size() > 1 ? ptrs[(i + 1) % ptrs.size()] : nullptr);
  field->resetChargeDensity();
  for (auto* p : ptrs) p->integrateChargeDensity(*field);
  last_solve = field->solvePoisson(0.0, logger.get());
  if (file_output) {  // initial field and moments (src/main.mm:142-147)
    outputField(start, *field, init, logger.get());
    for (auto* p : ptrs) {
      moment->integrateMoments(*p, *field);
      outputMoments(start, *moment, p->pName, init, logger.get());
    }
  }
  if (fused) {
    // The first cycle's charge: same particle positions, fresh accumulators.
    field->resetChargeDensity();
    for (auto* p : ptrs) p->integrateChargeDensity(*field);
  }
  GP_CUDA(cudaStreamSynchronize(stream));
}

void Simulation::reload(uint64_t seed) {
  collision->reload(seed, ptrs);
  for (auto* p : ptrs) {
    p->needs_sort = true;
    p->random_order = true;
    p->cycles_since_sort = 0;
  }
  cycle_no = init.paramForTimeIntegration.Start;
  comp = 0;
  time = cycle_no * init.paramForTimeIntegration.TimeStep;
  GP_CUDA(cudaStreamSynchronize(stream));
}

void Simulation::cycle() {
  const auto& T = init.paramForTimeIntegration;
  const double dt = T.TimeStep;
  ++cycle_no;
  if (logger) logger->swichLog(T.LogOutput != 0 && cycle_no % T.LogOutput == 0);  // :157-158 (guarded)
  // Kahan-compensated time (src/main.mm:160-163)
  const double y = dt - comp;
  const double t = time + y;
  comp = (t - time) - y;
  time = t;
  if (logger) logger->logCycleStart(cycle_no, time);
  if (!fused) {
    mark(PH_DEPOSIT, true);
    field->resetChargeDensity();
    for (auto* p : ptrs) {
      tic("integCDens_" + p->pName);
      p->integrateChargeDensity(*field);
      toc();
    }
    mark(PH_DEPOSIT, false);
  }
  const int em = init.flagForEquation.EMField;
  if (em == 1 || em == 2) {
    mark(PH_SOLVE, true);
    tic("solvePoisson");
    last_solve = field->solvePoisson(dt, logger.get());
    toc();
    if (em == 2) {  // src/main.mm:187-190
      tic("solveVectorPotential");
      field->solveVectorPotential(dt, logger.get());
      toc();
    }
    mark(PH_SOLVE, false);
  }
  const bool field_out = file_output && T.FieldOutput != 0 && cycle_no % T.FieldOutput == 0;
  if (field_out) outputField(cycle_no, *field, init, logger.get());  // src/main.mm:193-195
  if (fused) field->resetChargeDensity();
  for (size_t s = 0; s < ptrs.size(); ++s) {
    if (ptrs[s]->needs_sort) {
      mark(PH_SORT, true);
      ptrs[s]->sort();
      mark(PH_SORT, false);
    }
    mark(PH_PUSH, true);
    tic("update_" + ptrs[s]->pName);
    ptrs[s]->update(dt, *field, fused);
    toc();
    mark(PH_PUSH, false);
    mark(PH_REDUCE, true);
    tic("reduce_" + ptrs[s]->pName);
    ptrs[s]->reduceLaunch();
    toc();
    mark(PH_REDUCE, false);
  }
  // one synchronisation for the counters of every species: the next
  // species' push was enqueued behind this one's compaction, not after a
  // host round trip
  GP_CUDA(cudaStreamSynchronize(stream));
  for (size_t s = 0; s < ptrs.size(); ++s) {
    last_flow[s] = ptrs[s]->reduceFinish(logger.get());
    if (file_output && T.ParticleOutput != 0 && cycle_no % T.ParticleOutput == 0)  // :211-214
      outputPhaseSpace(cycle_no, *ptrs[s], init);
    if (field_out) {  // :215-220
      moment->integrateMoments(*ptrs[s], *field);
      outputMoments(cycle_no, *moment, ptrs[s]->pName, init, logger.get());
    }
  }
  mark(PH_SOURCE, true);
  tic("artificialIonization");
  last_ai = collision->artificialIonization(dt, ptrs, logger.get());
  toc();
  tic("hollowCathode");
  last_hc = collision->hollowCathode(dt, ptrs, logger.get());
  toc();
  tic("fluxReinjection");
  last_reflux = collision->fluxReinjection(dt, ptrs, logger.get());
  toc();
  if (fused)  // the injected particles' charge (the rest came with the push)
    for (auto* p : ptrs) {
      tic("integCDens_" + p->pName);
      p->integrateChargeDensity(*field, true);
      toc();
    }
  mark(PH_SOURCE, false);
  // src/main.mm:237-243 (guarded by FieldOutput there; a zero ProgressOutput
  // would divide by zero and is treated as "never")
  if (file_output && T.FieldOutput != 0 && T.ProgressOutput != 0 && cycle_no % T.ProgressOutput == 0)
    if (!saveProgress(cycle_no, ptrs, init)) throw std::runtime_error("output progress failed.");
  log_resources();
  if (logger) logger->logCycleEnd();
}

void Simulation::run(int ncycles) {
  for (int i = 0; i < ncycles; ++i) cycle();
  GP_CUDA(cudaStreamSynchronize(stream));
}

}  // namespace gample

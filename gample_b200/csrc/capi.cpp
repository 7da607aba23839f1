// capi.cpp -- extern "C" entry points declared in include/gample_gpu.h.
#include <cstring>
#include <exception>
#include <string>

#include "../../include/gample_gpu.h"
#include "ensemble.hpp"
#include "fileio.hpp"
#include "learned.hpp"
#include "simulation.hpp"

#include <atomic>
#include <cstdint>
#include <map>
#include <mutex>
#include <set>

namespace gample {
namespace {
std::atomic<unsigned long long> g_launches{0};
}
thread_local unsigned long long t_launches = 0;
void note_kernel_launch() {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  ++t_launches;
}
unsigned long long thread_kernel_launches() { return t_launches; }
void add_kernel_launches(long long n) {
  g_launches.fetch_add(static_cast<unsigned long long>(n), std::memory_order_relaxed);
}
unsigned long long kernel_launches() { return g_launches.load(std::memory_order_relaxed); }

namespace {
std::mutex g_pool_mutex;
std::set<int> g_pool_ready;  // devices whose default pool keeps freed memory
cudaMemPool_t current_pool() {
  int dev = 0;
  GP_CUDA(cudaGetDevice(&dev));
  cudaMemPool_t pool;
  GP_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
  std::lock_guard<std::mutex> lk(g_pool_mutex);
  if (!g_pool_ready.count(dev)) {
    uint64_t keep = UINT64_MAX;
    GP_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    g_pool_ready.insert(dev);
  }
  return pool;
}
}  // namespace

void* device_alloc(size_t bytes) {
  void* p = nullptr;
  GP_CUDA(cudaMallocFromPoolAsync(&p, bytes, current_pool(), 0));
  GP_CUDA(cudaStreamSynchronize(0));
  return p;
}

void device_free(void* p) {
  // as cudaFree: no kernel may still use the block when it is reused
  if (cudaDeviceSynchronize() != cudaSuccess) return;
  cudaFreeAsync(p, 0);
}

namespace {
std::mutex g_pinned_mutex;
std::multimap<size_t, void*> g_pinned_free;  // kept page-locked blocks by size
}  // namespace

void* pinned_alloc(size_t bytes) {
  {
    std::lock_guard<std::mutex> lk(g_pinned_mutex);
    auto it = g_pinned_free.find(bytes);
    if (it != g_pinned_free.end()) {
      void* p = it->second;
      g_pinned_free.erase(it);
      return p;
    }
  }
  void* p = nullptr;
  GP_CUDA(cudaMallocHost(&p, bytes));
  return p;
}

void pinned_free(void* p, size_t bytes) {
  std::lock_guard<std::mutex> lk(g_pinned_mutex);
  g_pinned_free.emplace(bytes, p);
}

void release_cached_device_memory() {
  GP_CUDA(cudaDeviceSynchronize());
  GP_CUDA(cudaMemPoolTrimTo(current_pool(), 0));
  std::lock_guard<std::mutex> lk(g_pinned_mutex);
  for (auto& b : g_pinned_free) cudaFreeHost(b.second);
  g_pinned_free.clear();
}
}  // namespace gample

struct gp_init {
  gample::Init init;
};
struct gp_sim {
  std::unique_ptr<gample::Simulation> sim;
  gample::Simulation* view = nullptr;  // member of an ensemble (not owned)
  gample::Simulation* get() const { return view ? view : sim.get(); }
};
struct gp_ensemble {
  std::unique_ptr<gample::Ensemble> ens;
  std::vector<gp_sim> views;
};
struct gp_nn {
  std::unique_ptr<gample::nn::WarmStartNet> net;
  cudaStream_t stream = nullptr;
  gample::DeviceArray<float> in, out, target;
  ~gp_nn() {
    net.reset();
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

thread_local std::string g_error;

template <typename F>
gp_status guarded(F&& f) {
  try {
    return f();
  } catch (const gample::ConfigError& e) {
    g_error = e.what();
    return GP_ERR_CONFIG;
  } catch (const gample::CudaError& e) {
    g_error = e.what();
    return GP_ERR_CUDA;
  } catch (const std::invalid_argument& e) {
    g_error = e.what();
    return GP_ERR_ARGUMENT;
  } catch (const std::runtime_error& e) {
    g_error = e.what();
    return std::string(e.what()).find("pNum") != std::string::npos ? GP_ERR_CAPACITY : GP_ERR_INTERNAL;
  } catch (const std::exception& e) {
    g_error = e.what();
    return GP_ERR_INTERNAL;
  } catch (...) {
    g_error = "unknown error";
    return GP_ERR_INTERNAL;
  }
}

gample::Particle* species(gp_sim* sim, int s) {
  if (!sim || !sim->get()) throw std::invalid_argument("null simulation handle");
  if (s < 0 || s >= int(sim->get()->ptrs.size())) throw std::invalid_argument("species index out of range");
  return sim->get()->ptrs[s];
}
gample::Simulation& S(gp_sim* sim) {
  if (!sim || !sim->get()) throw std::invalid_argument("null simulation handle");
  return *sim->get();
}
const gample::Simulation& S(const gp_sim* sim) {
  if (!sim || !sim->get()) throw std::invalid_argument("null simulation handle");
  return *sim->get();
}

void fill(gp_solve_stats* out, const gample::SolveStats& st) {
  if (!out) return;
  out->iterations = st.iterations;
  out->error = st.error;
  out->mean_cathode = st.meanCathode;
  out->electric_energy = st.energy;
  out->electric_energy_increment = st.EEincrement;
  out->joule_heating = st.joule;
  for (int i = 0; i < 3; ++i) out->probe[i] = st.probe[i];
  out->field_energy_cgs = st.field_energy_cgs;
}
void fill(gp_flow_stats* out, const gample::FlowStats& fs) {
  if (!out) return;
  out->particle_number = fs.particleNumber;
  out->pulled = fs.pulledPtclNum;
  for (int i = 0; i < 4; ++i) out->pinum[i] = fs.pinum[i];
  out->invalid = fs.invalid;
  out->kinetic_energy = fs.totalKineticEnergy;
  out->kinetic_energy_increment = fs.totalKEincrement;
}

struct FieldBuf {
  void* dev;
  size_t bytes;
};
FieldBuf field_buf(gample::EMField& f, int which) {
  switch (which) {
    case GP_FIELD_RHO: return {f.rho.get(), f.rho.bytes()};
    case GP_FIELD_EX: return {f.Ex.get(), f.Ex.bytes()};
    case GP_FIELD_EY: return {f.Ey.get(), f.Ey.bytes()};
    case GP_FIELD_BZ: return {f.Bz.get(), f.Bz.bytes()};
    case GP_FIELD_JX: return {f.jx.get(), f.jx.bytes()};
    case GP_FIELD_JY: return {f.jy.get(), f.jy.bytes()};
    case GP_FIELD_PHI: return {f.phi.get(), f.phi.bytes()};
    case GP_FIELD_SOL: return {f.sol.get(), f.sol.bytes()};
    case GP_FIELD_DEL_EX: return {f.delEx.get(), f.delEx.bytes()};
    case GP_FIELD_DEL_EY: return {f.delEy.get(), f.delEy.bytes()};
    case GP_FIELD_DEL_BZ: return {f.delBz.get(), f.delBz.bytes()};
    case GP_FIELD_PSI:
    case GP_FIELD_AX:
    case GP_FIELD_AY:
      if (!f.darwin) throw std::invalid_argument("the Darwin solution needs FlagForEquation.EMField = 2");
      if (which == GP_FIELD_PSI) return {f.psi.get(), f.psi.bytes()};
      if (which == GP_FIELD_AX) return {f.Ax.get(), f.Ax.bytes()};
      return {f.Ay.get(), f.Ay.bytes()};
    default: throw std::invalid_argument("unknown field selector");
  }
}

}  // namespace

extern "C" {

gp_status gp_deposit_charge_noalloc(int weighting_order, int ngx, int ngy, const gp_particle_state* particles,
                                    uint32_t n, float scale, float* rho, void* stream) {
  return guarded([&] {
    try {
      gample::kern::deposit_charge_noalloc(weighting_order, ngx, ngy,
                                           reinterpret_cast<const gample::kern::ParticleStateAoS*>(particles), n,
                                           scale, rho, static_cast<cudaStream_t>(stream));
    } catch (const std::length_error& e) {
      g_error = e.what();
      return GP_ERR_CAPACITY;
    }
    return GP_OK;
  });
}

gp_status gp_nn_create(int h, int w, uint64_t seed, gp_nn** out) {
  return guarded([&] {
    if (!out) throw std::invalid_argument("null output handle");
    auto n = std::make_unique<gp_nn>();
    GP_CUDA(cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking));
    n->net = std::make_unique<gample::nn::WarmStartNet>(h, w, seed, n->stream);
    n->in.resize(size_t(h) * w * 2);
    n->out.resize(size_t(h) * w);
    n->target.resize(size_t(h) * w);
    *out = n.release();
    return GP_OK;
  });
}
void gp_nn_free(gp_nn* nn) { delete nn; }

namespace {
gp_nn& NN(gp_nn* nn) {
  if (!nn || !nn->net) throw std::invalid_argument("null network handle");
  return *nn;
}
void put(gample::DeviceArray<float>& d, const float* h, cudaStream_t s) {
  if (!h) throw std::invalid_argument("null host buffer");
  GP_CUDA(cudaMemcpyAsync(d.get(), h, d.bytes(), cudaMemcpyHostToDevice, s));
}
}  // namespace

gp_status gp_nn_forward(gp_nn* nn, const float* in, float* out) {
  return guarded([&] {
    auto& n = NN(nn);
    put(n.in, in, n.stream);
    n.net->forward(n.in.get(), n.out.get());
    GP_CUDA(cudaMemcpyAsync(out, n.out.get(), n.out.bytes(), cudaMemcpyDeviceToHost, n.stream));
    GP_CUDA(cudaStreamSynchronize(n.stream));
    return GP_OK;
  });
}

gp_status gp_nn_loss_grad(gp_nn* nn, const float* in, const float* target, float* loss) {
  return guarded([&] {
    auto& n = NN(nn);
    put(n.in, in, n.stream);
    put(n.target, target, n.stream);
    const float l = n.net->loss_and_grad(n.in.get(), n.target.get());
    if (loss) *loss = l;
    return GP_OK;
  });
}

gp_status gp_nn_train_step(gp_nn* nn, const float* in, const float* target, float lr, float* loss) {
  return guarded([&] {
    auto& n = NN(nn);
    put(n.in, in, n.stream);
    put(n.target, target, n.stream);
    const float l = n.net->train_step(n.in.get(), n.target.get(), lr);
    if (loss) *loss = l;
    return GP_OK;
  });
}

gp_status gp_nn_layer_info(gp_nn* nn, int layer, int* cin, int* cout, int* kpad) {
  return guarded([&] {
    auto& n = NN(nn);
    if (layer < 0 || layer >= n.net->num_layers()) throw std::invalid_argument("layer index out of range");
    const auto& L = n.net->layer(layer);
    if (cin) *cin = L.cin;
    if (cout) *cout = L.cout;
    if (kpad) *kpad = L.kpad;
    return GP_OK;
  });
}

gp_status gp_nn_param(gp_nn* nn, int layer, int which, float* host, size_t count, int set) {
  return guarded([&] {
    auto& n = NN(nn);
    if (layer < 0 || layer >= n.net->num_layers()) throw std::invalid_argument("layer index out of range");
    auto& L = n.net->layer(layer);
    gample::DeviceArray<float>* a = which == 0 ? &L.w : which == 1 ? &L.b : which == 2 ? &L.gw : which == 3 ? &L.gb
                                                                                                           : nullptr;
    if (!a || (set && which >= 2)) throw std::invalid_argument("parameter selector out of range");
    if (!host || count != a->size()) throw std::invalid_argument("host buffer size does not match the parameter");
    if (set) {
      GP_CUDA(cudaMemcpyAsync(a->get(), host, a->bytes(), cudaMemcpyHostToDevice, n.stream));
      n.net->sync_weights();
    } else {
      GP_CUDA(cudaMemcpyAsync(host, a->get(), a->bytes(), cudaMemcpyDeviceToHost, n.stream));
    }
    GP_CUDA(cudaStreamSynchronize(n.stream));
    return GP_OK;
  });
}

const char* gp_last_error(void) { return g_error.c_str(); }
unsigned long long gp_kernel_launches(void) { return gample::kernel_launches(); }
gp_status gp_release_cached_memory(void) {
  return guarded([&] {
    gample::release_cached_device_memory();
    return GP_OK;
  });
}
const char* gp_version(void) { return "gample_b200 0.1 (sm_100a)"; }
int gp_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

gp_status gp_init_parse_file(const char* path, gp_init** out) {
  return guarded([&] {
    if (!path || !out) throw std::invalid_argument("null argument");
    auto* h = new gp_init{gample::Init::parseInputFile(path)};
    *out = h;
    return GP_OK;
  });
}
gp_status gp_init_parse_json(const char* text, gp_init** out) {
  return guarded([&] {
    if (!text || !out) throw std::invalid_argument("null argument");
    auto* h = new gp_init{gample::Init::parseString(text)};
    *out = h;
    return GP_OK;
  });
}
gp_status gp_init_dump(const gp_init* init, char* buf, size_t cap, size_t* len) {
  return guarded([&] {
    if (!init) throw std::invalid_argument("null init");
    std::string s = init->init.dump();
    if (len) *len = s.size() + 1;
    if (buf && cap) {
      size_t n = s.size() < cap - 1 ? s.size() : cap - 1;
      std::memcpy(buf, s.data(), n);
      buf[n] = '\0';
    }
    return GP_OK;
  });
}
void gp_init_free(gp_init* init) { delete init; }

gp_status gp_sim_create(const gp_init* init, const char* log_name, int flags, gp_sim** out) {
  return guarded([&] {
    if (!init || !out) throw std::invalid_argument("null argument");
    auto* h = new gp_sim;
    try {
      h->sim = std::make_unique<gample::Simulation>(init->init, log_name ? log_name : "",
                                                    (flags & GP_SIM_REFERENCE_ORDER) == 0);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return GP_OK;
  });
}
void gp_sim_free(gp_sim* sim) {
  try {
    if (sim && sim->view) return;  // ensemble members are freed with their ensemble
    delete sim;
  } catch (...) {
  }
}

gp_status gp_ensemble_create(const gp_init* const* inits, int n, int threads, gp_ensemble** out) {
  return guarded([&] {
    if (!inits || n <= 0 || !out) throw std::invalid_argument("null or empty ensemble description");
    std::vector<gample::Init> v;
    for (int i = 0; i < n; ++i) {
      if (!inits[i]) throw std::invalid_argument("null condition in the ensemble");
      v.push_back(inits[i]->init);
    }
    auto e = std::make_unique<gp_ensemble>();
    e->ens = std::make_unique<gample::Ensemble>(v, threads);
    e->views.resize(size_t(n));
    for (int i = 0; i < n; ++i) e->views[i].view = e->ens->members[i].get();
    *out = e.release();
    return GP_OK;
  });
}
void gp_ensemble_free(gp_ensemble* e) {
  try {
    delete e;
  } catch (...) {
  }
}
gp_status gp_ensemble_initialize(gp_ensemble* e) {
  return guarded([&] {
    if (!e || !e->ens) throw std::invalid_argument("null ensemble handle");
    e->ens->initialize();
    return GP_OK;
  });
}
gp_status gp_ensemble_run(gp_ensemble* e, int ncycles) {
  return guarded([&] {
    if (!e || !e->ens) throw std::invalid_argument("null ensemble handle");
    if (ncycles < 0) throw std::invalid_argument("negative cycle count");
    e->ens->run(ncycles);
    return GP_OK;
  });
}
gp_status gp_ensemble_time_cycles(gp_ensemble* e, int ncycles, float* ms) {
  return guarded([&] {
    if (!e || !e->ens || !ms) throw std::invalid_argument("null argument");
    if (ncycles < 0) throw std::invalid_argument("negative cycle count");
    *ms = e->ens->time_cycles(ncycles);
    return GP_OK;
  });
}
gp_status gp_ensemble_member(gp_ensemble* e, int i, gp_sim** out) {
  return guarded([&] {
    if (!e || !e->ens || !out) throw std::invalid_argument("null argument");
    if (i < 0 || i >= int(e->views.size())) throw std::invalid_argument("member index out of range");
    *out = &e->views[size_t(i)];
    return GP_OK;
  });
}
gp_status gp_sim_reload(gp_sim* sim, uint64_t seed) {
  return guarded([&] {
    S(sim).reload(seed);
    return GP_OK;
  });
}
gp_status gp_sim_initialize(gp_sim* sim) {
  return guarded([&] {
    S(sim).initialize();
    return GP_OK;
  });
}
gp_status gp_sim_run(gp_sim* sim, int ncycles) {
  return guarded([&] {
    if (ncycles < 0) throw std::invalid_argument("negative cycle count");
    S(sim).run(ncycles);
    return GP_OK;
  });
}
gp_status gp_sim_cycle_number(const gp_sim* sim, int* cycle, double* time) {
  return guarded([&] {
    if (cycle) *cycle = S(sim).cycle_no;
    if (time) *time = S(sim).time;
    return GP_OK;
  });
}
gp_status gp_sim_last_solve(const gp_sim* sim, gp_solve_stats* out) {
  return guarded([&] {
    fill(out, S(sim).last_solve);
    return GP_OK;
  });
}
gp_status gp_sim_last_flow(const gp_sim* sim, int s, gp_flow_stats* out) {
  return guarded([&] {
    const auto& v = S(sim).last_flow;
    if (s < 0 || s >= int(v.size())) throw std::invalid_argument("species index out of range");
    fill(out, v[s]);
    return GP_OK;
  });
}
gp_status gp_sim_synchronize(gp_sim* sim) {
  return guarded([&] {
    GP_CUDA(cudaStreamSynchronize(S(sim).stream));
    return GP_OK;
  });
}
gp_status gp_sim_time_cycles(gp_sim* sim, int ncycles, float* ms) {
  return guarded([&] {
    auto& s = S(sim);
    cudaEvent_t a, b;
    GP_CUDA(cudaEventCreate(&a));
    GP_CUDA(cudaEventCreate(&b));
    GP_CUDA(cudaEventRecord(a, s.stream));
    for (int i = 0; i < ncycles; ++i) s.cycle();
    GP_CUDA(cudaEventRecord(b, s.stream));
    GP_CUDA(cudaEventSynchronize(b));
    float t = 0;
    GP_CUDA(cudaEventElapsedTime(&t, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (ms) *ms = t;
    return GP_OK;
  });
}
gp_status gp_sim_set_profiling(gp_sim* sim, int on) {
  return guarded([&] {
    S(sim).set_profiling(on != 0);
    return GP_OK;
  });
}
gp_status gp_sim_phase_times(gp_sim* sim, double out[6]) {
  return guarded([&] {
    if (!out) throw std::invalid_argument("null output");
    S(sim).phase_times(out);
    return GP_OK;
  });
}

gp_status gp_field_dims(const gp_sim* sim, int* ngx, int* ngy, int* ngb, int* nkx, int* nky) {
  return guarded([&] {
    const auto& f = *S(sim).field;
    if (ngx) *ngx = f.dims.ngx;
    if (ngy) *ngy = f.dims.ngy;
    if (ngb) *ngb = f.dims.ngb;
    if (nkx) *nkx = f.layout.nkx;
    if (nky) *nky = f.layout.nky;
    return GP_OK;
  });
}
gp_status gp_field_reset_charge(gp_sim* sim) {
  return guarded([&] {
    S(sim).field->resetChargeDensity();
    return GP_OK;
  });
}
gp_status gp_field_solve_poisson(gp_sim* sim, double dt, gp_solve_stats* out) {
  return guarded([&] {
    auto& s = S(sim);
    s.last_solve = s.field->solvePoisson(dt, s.logger.get());
    fill(out, s.last_solve);
    return GP_OK;
  });
}
gp_status gp_field_solve_darwin(gp_sim* sim, double dt, int iterations[3], double errors[3]) {
  return guarded([&] {
    auto& s = S(sim);
    if (!s.field->darwin) throw std::invalid_argument("the Darwin solve needs FlagForEquation.EMField = 2");
    const auto st = s.field->solveVectorPotential(dt, s.logger.get());
    for (int q = 0; q < 3; ++q) {
      if (iterations) iterations[q] = st.iters[q];
      if (errors) errors[q] = st.errors[q];
    }
    return GP_OK;
  });
}
gp_status gp_field_learned(gp_sim* sim, int mode, float lr, uint64_t seed) {
  return guarded([&] {
    if (mode < 0 || mode > 31 || !(lr >= 0)) throw std::invalid_argument("learned mode must be 0..31 and lr >= 0");
    S(sim).field->setLearned(mode, lr, seed);
    return GP_OK;
  });
}
gp_status gp_field_learned_bank(gp_sim* sim, int capacity) {
  return guarded([&] {
    S(sim).field->setLearnedBank(capacity);
    return GP_OK;
  });
}
gp_status gp_field_learned_train(gp_sim* sim, int steps, float lr, uint64_t seed, double out[3]) {
  return guarded([&] {
    if (steps < 1 || !(lr > 0) || !out) throw std::invalid_argument("steps >= 1, lr > 0 and an output are needed");
    S(sim).field->trainLearned(steps, lr, seed, out);
    return GP_OK;
  });
}
gp_status gp_field_learned_stats(gp_sim* sim, double out[9]) {
  return guarded([&] {
    if (!out) throw std::invalid_argument("null output");
    const auto& st = S(sim).field->last_learned;
    const double v[9] = {st.loss,      double(st.iters_learned), double(st.iters_plain),
                         st.ms_learned, st.ms_plain,              st.ms_net,
                         st.rel0_learned, st.rel0_plain,          double(st.trained_steps)};
    for (int i = 0; i < 9; ++i) out[i] = v[i];
    return GP_OK;
  });
}
gp_status gp_field_download(gp_sim* sim, int which, void* host, size_t bytes) {
  return guarded([&] {
    auto& s = S(sim);
    if (which == GP_FIELD_RHO || which == GP_FIELD_JX || which == GP_FIELD_JY) {
      // In the deterministic mode rho/jx/jy are combined from the
      // fixed-point sums on demand.
      s.field->finalizeCharge();
    }
    FieldBuf fb = field_buf(*s.field, which);
    if (!host || bytes != fb.bytes) throw std::invalid_argument("buffer size does not match the field extent");
    GP_CUDA(cudaMemcpyAsync(host, fb.dev, bytes, cudaMemcpyDeviceToHost, s.stream));
    GP_CUDA(cudaStreamSynchronize(s.stream));
    return GP_OK;
  });
}
gp_status gp_field_upload(gp_sim* sim, int which, const void* host, size_t bytes) {
  return guarded([&] {
    auto& s = S(sim);
    FieldBuf fb = field_buf(*s.field, which);
    if (!host || bytes != fb.bytes) throw std::invalid_argument("buffer size does not match the field extent");
    GP_CUDA(cudaMemcpyAsync(fb.dev, host, bytes, cudaMemcpyHostToDevice, s.stream));
    GP_CUDA(cudaStreamSynchronize(s.stream));
    if (which == GP_FIELD_BZ) s.field->bz_uniform = false;  // arbitrary Bz: gather it
    s.field->e_pitched_stale = true;
    return GP_OK;
  });
}
gp_status gp_field_set_solver(gp_sim* sim, double tol, int maxiter) {
  return guarded([&] {
    if (!(tol > 0) || maxiter < 0) throw std::invalid_argument("tolerance must be > 0 and maxiter >= 0");
    S(sim).field->tol = tol;
    S(sim).field->maxiter = maxiter;
    return GP_OK;
  });
}

gp_status gp_particle_update(gp_sim* sim, int s, double dt, int fused_deposit) {
  return guarded([&] {
    species(sim, s)->update(dt, *S(sim).field, fused_deposit != 0);
    return GP_OK;
  });
}
gp_status gp_particle_reduce(gp_sim* sim, int s, gp_flow_stats* out) {
  return guarded([&] {
    auto fs = species(sim, s)->reduce(S(sim).logger.get());
    S(sim).last_flow[s] = fs;
    fill(out, fs);
    return GP_OK;
  });
}
gp_status gp_particle_integrate_charge(gp_sim* sim, int s) {
  return guarded([&] {
    species(sim, s)->integrateChargeDensity(*S(sim).field);
    return GP_OK;
  });
}
gp_status gp_particle_count(gp_sim* sim, int s, uint32_t* n) {
  return guarded([&] {
    if (!n) throw std::invalid_argument("null output");
    *n = species(sim, s)->pNum();
    return GP_OK;
  });
}
gp_status gp_particle_sort(gp_sim* sim, int s, int path) {
  return guarded([&] {
    if (path < 0 || path > 2) throw std::invalid_argument("path must be 0, 1 or 2");
    auto* p = species(sim, s);
    if (path) p->random_order = path == 2;
    p->sort();
    GP_CUDA(cudaStreamSynchronize(p->stream));
    return GP_OK;
  });
}
gp_status gp_particle_set_push_variant(gp_sim* sim, int s, int particles, int tables) {
  return guarded([&] {
    auto* p = species(sim, s);
    constexpr int per = gample::kern::kPushChunkPer;
    if (particles == 0) {
      p->tune_step = -1;
      for (double& t : p->tune_ms) t = 0;
      p->push_variant = {per, 1};
    } else if (particles == 256 * per || particles == 128 * per) {
      p->tune_step = 1 << 20;  // no tuning
      p->push_variant = {particles / 256, tables ? 1 : 0};
    } else {
      throw std::invalid_argument("particles per chunk must be 0, 1024 or 2048");
    }
    return GP_OK;
  });
}
gp_status gp_particle_push_stats(gp_sim* sim, int s, uint32_t out[7]) {
  return guarded([&] {
    if (!out) throw std::invalid_argument("null output");
    const auto c = species(sim, s)->counters();
    out[0] = c.n_slow;
    out[1] = c.n_tma;
    out[2] = c.err;
    out[3] = c.n_tab;
    out[4] = c.n_priv;
    out[5] = uint32_t(species(sim, s)->tune_used.per) * 256u;
    out[6] = uint32_t(species(sim, s)->tune_used.tables);
    return GP_OK;
  });
}
gp_status gp_particle_download(gp_sim* sim, int s, gp_particle_state* host, uint32_t capacity, uint32_t* n) {
  return guarded([&] {
    auto* p = species(sim, s);
    const uint32_t cnt = p->pNum();
    if (n) *n = cnt;
    if (host) {
      if (capacity < cnt) throw std::invalid_argument("capacity smaller than pNum");
      static_assert(sizeof(gp_particle_state) == sizeof(gample::kern::ParticleStateAoS), "record size");
      p->download_aos(reinterpret_cast<gample::kern::ParticleStateAoS*>(host), cnt);
    }
    return GP_OK;
  });
}
gp_status gp_particle_upload(gp_sim* sim, int s, const gp_particle_state* host, uint32_t n) {
  return guarded([&] {
    if (n && !host) throw std::invalid_argument("null input");
    species(sim, s)->upload_aos(reinterpret_cast<const gample::kern::ParticleStateAoS*>(host), n);
    return GP_OK;
  });
}
gp_status gp_particle_download_raw(gp_sim* sim, int s, int32_t* cell, float* ox, float* oy, float* vx, float* vy,
                                   float* vz, uint32_t capacity, uint32_t* n) {
  return guarded([&] {
    auto* p = species(sim, s);
    const uint32_t cnt = p->pNum();
    if (n) *n = cnt;
    if (capacity < cnt && (cell || ox || oy || vx || vy || vz))
      throw std::invalid_argument("capacity smaller than pNum");
    auto cp = [&](void* dst, const void* src, size_t elem) {
      if (dst && cnt) GP_CUDA(cudaMemcpyAsync(dst, src, cnt * elem, cudaMemcpyDeviceToHost, p->stream));
    };
    const auto a = p->arrays();
    cp(cell, a.cell, 4);
    cp(ox, a.ox, 4);
    cp(oy, a.oy, 4);
    cp(vx, a.vx, 4);
    cp(vy, a.vy, 4);
    cp(vz, a.vz, 4);
    GP_CUDA(cudaStreamSynchronize(p->stream));
    return GP_OK;
  });
}

gp_status gp_moments_integrate(gp_sim* sim, int s) {
  return guarded([&] {
    auto* p = species(sim, s);
    auto& S_ = S(sim);
    S_.moment->integrateMoments(*p, *S_.field);
    GP_CUDA(cudaStreamSynchronize(S_.stream));
    return GP_OK;
  });
}

gp_status gp_moments_download(gp_sim* sim, int which, float* host, size_t bytes) {
  return guarded([&] {
    auto& S_ = S(sim);
    if (which < 0 || which >= gample::Moment::kCount) throw std::invalid_argument("moment index out of range");
    const size_t n = S_.moment->n_rho();
    if (!host || bytes < n * sizeof(float)) throw std::invalid_argument("host buffer too small");
    GP_CUDA(cudaMemcpyAsync(host, S_.moment->out.get() + size_t(which) * n, n * sizeof(float), cudaMemcpyDeviceToHost,
                            S_.stream));
    GP_CUDA(cudaStreamSynchronize(S_.stream));
    return GP_OK;
  });
}

gp_status gp_sim_output_field(gp_sim* sim, int cycle) {
  return guarded([&] {
    auto& S_ = S(sim);
    gample::outputField(cycle, *S_.field, S_.init, S_.logger.get());
    return GP_OK;
  });
}

gp_status gp_sim_output_moments(gp_sim* sim, int s, int cycle) {
  return guarded([&] {
    auto* p = species(sim, s);
    auto& S_ = S(sim);
    S_.moment->integrateMoments(*p, *S_.field);
    gample::outputMoments(cycle, *S_.moment, p->pName, S_.init, S_.logger.get());
    return GP_OK;
  });
}

gp_status gp_sim_save_progress(gp_sim* sim, int cycle) {
  return guarded([&] {
    auto& S_ = S(sim);
    if (!gample::saveProgress(cycle, S_.ptrs, S_.init)) throw std::runtime_error("output progress failed");
    return GP_OK;
  });
}

gp_status gp_sim_load_progress(gp_sim* sim, int cycle) {
  return guarded([&] {
    auto& S_ = S(sim);
    if (!gample::loadProgress(cycle, S_.ptrs, S_.init)) throw std::runtime_error("restart failed");
    return GP_OK;
  });
}

gp_status gp_collision_artificial_ionization(gp_sim* sim, double dt, int* addn) {
  return guarded([&] {
    auto& s = S(sim);
    int a = s.collision->artificialIonization(dt, s.ptrs, s.logger.get());
    if (addn) *addn = a;
    return GP_OK;
  });
}
gp_status gp_collision_hollow_cathode(gp_sim* sim, double dt, int* addn) {
  return guarded([&] {
    auto& s = S(sim);
    int a = s.collision->hollowCathode(dt, s.ptrs, s.logger.get());
    if (addn) *addn = a;
    return GP_OK;
  });
}
gp_status gp_collision_flux_reinjection(gp_sim* sim, double dt, int* addn) {
  return guarded([&] {
    auto& s = S(sim);
    int a = s.collision->fluxReinjection(dt, s.ptrs, s.logger.get());
    if (addn) *addn = a;
    return GP_OK;
  });
}

}  // extern "C"

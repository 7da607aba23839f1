// oracle_capi.cpp -- time-loop restatement and C API of the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY (see oracle_core.hpp). The Sim class follows the
// reference's object model and call order:
//   Particle  (src/Particle.mm:407-611, 615-891, 893-1002, 1004-1130)
//   EMField   (src/EMField.mm:105-656, 745-1136, 1363-1378)
//   Collision (src/Collision.mm:189-462, 464-566, 568-678)
//   main loop (src/main.mm:114-254)
#include "oracle.h"

#include <cstdio>
#include <memory>

#include "oracle_core.hpp"

using namespace oracle;

namespace {

struct SimBase {
  virtual ~SimBase() = default;
};

template <typename R>
struct Sim : SimBase {
  or_config cfg;
  Grid g;
  int ns = 0;
  // Particle objects
  std::vector<Particles<R>> P;
  std::vector<float> qf, mf, wf;
  std::vector<double> lastKE;
  std::vector<FlowStats> flow;
  // EMField object
  float dxf, dyf;
  std::vector<R> rho, jx, jy, Ex, Ey, Ez, Bx, By, Bz;
  std::vector<double> phi;
  PoissonSystem S;
  std::vector<double> phi_sol;
  double lastEE = 0;
  bool current = false;
  // Collision object
  std::vector<RNGState> states;
  uint64_t master = 0;
  size_t initialized = 0;
  MinstdCanonical rnd_engine;
  int ele = -1, ion = -1;

  explicit Sim(const or_config& c) : cfg(c) {
    master = c.master_seed;
    g.ngx = c.ngx;
    g.ngy = c.ngy;
    g.ngb = c.ngb;
    ns = c.n_species;
    dxf = float(c.dx);
    dyf = float(c.dy);
    P.resize(ns);
    qf.resize(ns);
    mf.resize(ns);
    wf.resize(ns);
    lastKE.assign(ns, 0.0);
    flow.resize(ns);
    for (int s = 0; s < ns; ++s) {
      P[s].resize(c.pnum_max);
      P[s].n = c.sp[s].pnum;
      qf[s] = float(c.sp[s].q);
      mf[s] = float(c.sp[s].m);
      wf[s] = float(c.sp[s].w);
      if (std::string(c.sp[s].name) == "electron")
        ele = s;
      else
        ion = s;
    }
    // src/Particle.mm:523-525: current deposition for FlagForCurDens or Darwin.
    current = (c.cur_dens == 1) || (c.em_field > 1);
    // src/EMField.mm:133-197
    rho.assign(g.n_rho(), R(0));
    jx.assign(g.n_ex(), R(0));
    jy.assign(g.n_ey(), R(0));
    Ex.assign(g.n_ex(), R(0));
    Ey.assign(g.n_ey(), R(0));
    Ez.assign(g.n_rho(), R(0));
    Bx.assign(g.n_ey(), R(0));
    By.assign(g.n_ex(), R(0));
    Bz.assign(g.n_bz(), R(0));
    if (c.initE_uniform) {
      for (auto& v : Ex) v = R(float(c.ampE[0]));
      for (auto& v : Ey) v = R(float(c.ampE[1]));
      for (auto& v : Ez) v = R(float(c.ampE[2]));
    }
    if (c.initB_uniform) {
      for (auto& v : Bx) v = R(float(c.ampB[0]));
      for (auto& v : By) v = R(float(c.ampB[1]));
      for (auto& v : Bz) v = R(float(c.ampB[2]));
    }
    phi.assign(g.n_phi(), 0.0);
    S.g = g;
    for (int w = 0; w < 4; ++w) S.fbc[w] = c.fbc[w];
    S.phiXmin = c.fbc_val[XMIN] * VtosV;
    S.phiXmax = c.fbc_val[XMAX] * VtosV;
    S.phiYmin = c.fbc_val[YMIN] * VtosV;
    S.phiYmax = c.fbc_val[YMAX] * VtosV;
    S.dphidxXmin = c.fbc_val[XMIN];
    S.dphidxXmax = c.fbc_val[XMAX];
    S.dphidyYmin = c.fbc_val[YMIN];
    S.dphidyYmax = c.fbc_val[YMAX];
    S.dx = dxf;
    S.dy = dyf;
    S.build();
    phi_sol.assign(S.A.n, 0.0);
  }

  PushParams push_params(int s, double dt) const {
    PushParams pp;
    pp.ngx = g.ngx;
    pp.ngy = g.ngy;
    pp.ngb = g.ngb;
    pp.order = cfg.weight_order;
    pp.boris_order = cfg.boris_order;
    for (int w = 0; w < 4; ++w) pp.bc[w] = cfg.pbc[w];
    // src/Particle.mm:617-621 (double expressions stored in float members)
    pp.constE = float(0.5 * double(qf[s]) * dt / double(mf[s]));
    pp.constB = float(0.5 * double(qf[s]) * dt / double(mf[s]) / c_light);
    pp.constX = float(dt / double(dxf));
    pp.constY = float(dt / double(dyf));
    return pp;
  }
  float scale(int s) const {  // src/Particle.mm:540
    return float(double(qf[s] * wf[s]) / (cfg.dx * cfg.dy));
  }

  void reset_charge() {
    std::fill(rho.begin(), rho.end(), R(0));
    std::fill(jx.begin(), jx.end(), R(0));
    std::fill(jy.begin(), jy.end(), R(0));
  }
  void deposit(int s) {
    deposit_all_omp<R>(P[s], g, cfg.weight_order, R(scale(s)), current, rho.data(), jx.data(), jy.data());
  }

  void solve_poisson(double dt, double tol_override, or_solve_stats* st) {
    fold_ghosts<R>(rho.data(), g, cfg.fbc);
    std::vector<double> b = S.rhs(rho.data(), true);
    double tol = tol_override > 0 ? tol_override : cfg.tol;
    int maxit = std::max(cfg.maxiter, 50000);
    auto [it, err] = cg_solve(S.A, b, phi_sol, tol, maxit, S.doubly_periodic());
    phi_fill(S, phi_sol, phi);
    double mean = hollow_cathode_shift(S, phi_sol, phi, cfg.cathode_pos);
    gradient<R>(g, dxf, dyf, phi, Ex.data(), Ey.data());
    double energy, joule;
    field_energy<R>(g, dxf, dyf, dt, Ex.data(), Ey.data(), jx.data(), jy.data(), energy, joule);
    lastEE = energy;
    if (st) {
      st->iterations = it;
      st->error = err;
      st->mean_cathode = mean * sVtoV;
      st->energy = energy;
      st->joule = joule;
      // src/EMField.mm:1130-1134
      const int p_i = g.ngx / 4 + g.ngb, p_j = g.ngy / 2 + g.ngb, nx = g.nx();
      st->probe[0] = phi[(p_i + 2) + (p_j + 2) * (nx + 3)];
      st->probe[1] = double(Ex[(p_i + 1) + (p_j)*(nx + 2)]);
      st->probe[2] = double(Ey[(p_i) + (p_j + 1) * (nx + 1)]);
    }
  }

  void push(int s, double dt) {
    PushParams pp = push_params(s, dt);
    push_all<R>(P[s], Ex.data(), Ey.data(), Bz.data(), pp);
  }

  void reduce(int s, bool faithful, or_flow_stats* out) {
    FlowStats fs = reduce_particles<R>(P[s], qf[s], faithful);
    fs.energy = kinetic_energy<R>(P[s], mf[s], wf[s]);
    lastKE[s] = fs.energy;
    flow[s] = fs;
    if (out) {
      for (int w = 0; w < 4; ++w) out->pinum[w] = fs.pinum[w];
      out->pulled = fs.pulled;
      out->pnum = unsigned(P[s].n);
      out->ke = fs.energy;
    }
  }

  void ensure_states(size_t n) {
    if (n > initialized) {
      seed_states(states, initialized, n, master);
      initialized = n;
    }
  }

  // Collision init: src/Collision.mm:220-336.
  int load_initial() {
    const or_species& s0 = cfg.sp[0];
    GenParams prm;
    prm.addn = s0.pnum;
    if (s0.genX[0] < 0) {
      prm.Xmin = 0.0f;
      prm.Xmax = float(cfg.dx * cfg.ngx);
    } else {
      prm.Xmin = float(s0.genX[0]);
      prm.Xmax = float(s0.genX[1]);
    }
    if (s0.genY[0] < 0) {
      prm.Ymin = 0.0f;
      prm.Ymax = float(cfg.dy * cfg.ngy);
    } else {
      prm.Ymin = float(s0.genY[0]);
      prm.Ymax = float(s0.genY[1]);
    }
    for (int s = 0; s < ns; ++s) {
      const or_species& sp = cfg.sp[s];
      float vth = float(std::sqrt(2 * kb * sp.genT / sp.m));
      if (s == ele) {
        for (int d = 0; d < 3; ++d) prm.ele_genU[d] = float(sp.genU[d]);
        prm.ele_vth = vth;
      } else {
        for (int d = 0; d < 3; ++d) prm.ion_genU[d] = float(sp.genU[d]);
        prm.ion_vth = vth;
      }
    }
    prm.dx = float(cfg.dx);
    prm.dy = float(cfg.dy);
    prm.ngb = float(cfg.ngb);
    if (ele < 0 || ion < 0) return -1;
    if (prm.addn > cfg.pnum_max) return -2;
    ensure_states(prm.addn);
    int genType = s0.gen_type;
#pragma omp parallel for schedule(static)
    for (long id = 0; id < long(prm.addn); ++id)
      generate_one<R>(uint32_t(id), genType, prm, states.data(), P[ele], &P[ion]);
    P[ele].n = prm.addn;
    P[ion].n = prm.addn;
    return 0;
  }

  // Artificial ionization: src/Collision.mm:368-416 (parameters) and :464-566.
  // When several artificial-ionization sources are listed the last one's
  // parameters are the ones in effect (src/Collision.mm:368-416 overwrite a
  // single parameter buffer).
  static int last_source(const or_config& c, int lo, int hi) {
    int k = -1;
    for (int i = 0; i < c.n_sources; ++i)
      if (c.src[i].gen_type >= lo && c.src[i].gen_type <= hi) k = i;
    return k;
  }
  int ionize(double dt, int* addn_out) {
    for (int i = last_source(cfg, 0, 2); i >= 0; i = -1) {
      const or_source& src = cfg.src[i];
      int sion = -1;
      for (int s = 0; s < ns; ++s)
        if (std::string(cfg.sp[s].name) == src.pname) sion = s;
      if (sion < 0 || ele < 0) return -1;
      GenParams prm;
      if (src.genX[0] < 0) {
        prm.Xmin = 0.0f;
        prm.Xmax = float(cfg.dx * cfg.ngx);
      } else {
        prm.Xmin = float(src.genX[0]);
        prm.Xmax = float(src.genX[1]);
      }
      if (src.genY[0] < 0) {
        prm.Ymin = 0.0f;
        prm.Ymax = float(cfg.dy * cfg.ngy);
      } else {
        prm.Ymin = float(src.genY[0]);
        prm.Ymax = float(src.genY[1]);
      }
      for (int d = 0; d < 3; ++d) {
        prm.ele_genU[d] = float(src.genU_ele[d]);
        prm.ion_genU[d] = float(src.genU[d]);
      }
      prm.ele_vth = float(std::sqrt(2 * kb * src.genT_ele / me));
      prm.ion_vth = float(std::sqrt(2 * kb * src.genT / cfg.sp[sion].m));
      prm.dx = float(cfg.dx);
      prm.dy = float(cfg.dy);
      prm.ngb = float(cfg.ngb);
      float srcValue = float(src.src);
      double addn_d = double(srcValue / wf[ele]) * dt;
      if (rnd_engine.uniform01() < addn_d - int(addn_d))
        prm.addn = uint32_t(int(addn_d) + 1);
      else
        prm.addn = uint32_t(int(addn_d));
      if (addn_out) *addn_out = int(prm.addn);
      if (P[ele].n + prm.addn > cfg.pnum_max || P[sion].n + prm.addn > cfg.pnum_max) return -2;
      ensure_states(prm.addn);
      prm.ele_pNum = uint32_t(P[ele].n);
      prm.ion_pNum = uint32_t(P[sion].n);
      for (uint32_t id = 0; id < prm.addn; ++id)
        generate_one<R>(id, src.gen_type, prm, states.data(), P[ele], &P[sion]);
      P[ele].n += prm.addn;
      P[sion].n += prm.addn;
      return 0;  // one AI source supported, as the reference (Collision.mm:365)
    }
    if (addn_out) *addn_out = 0;
    return 0;
  }

  // Hollow cathode: src/Collision.mm:418-457 (parameters) and :568-678.
  int hollow_cathode(double dt, int* addn_out) {
    (void)dt;
    for (int i = last_source(cfg, 3, 3); i >= 0; i = -1) {
      const or_source& src = cfg.src[i];
      GenParams prm;
      int wall = int(src.src);
      int addn = 0;
      for (int s = 0; s < ns; ++s) addn -= flow[s].pinum[wall];
      if (addn_out) *addn_out = addn > 0 ? addn : 0;
      if (P[ele].n + (addn > 0 ? addn : 0) > cfg.pnum_max) return -2;
      if (addn <= 0) return 0;
      if (src.genX[0] < 0) {
        prm.Xmin = 0.0f;
        prm.Xmax = float(cfg.dx * cfg.ngx);
      } else {
        prm.Xmin = float(src.genX[0]);
        prm.Xmax = float(src.genX[1]);
      }
      if (src.genY[0] < 0) {
        prm.Ymin = 0.0f;
        prm.Ymax = float(cfg.dy * cfg.ngy);
      } else {
        prm.Ymin = float(src.genY[0]);
        prm.Ymax = float(src.genY[1]);
      }
      for (int d = 0; d < 3; ++d) prm.ele_genU[d] = float(src.genU[d]);
      prm.ele_vth = float(std::sqrt(2 * kb * src.genT / me));
      prm.dx = float(cfg.dx);
      prm.dy = float(cfg.dy);
      prm.ngb = float(cfg.ngb);
      prm.addn = uint32_t(addn);
      ensure_states(prm.addn);
      prm.ele_pNum = uint32_t(P[ele].n);
      for (uint32_t id = 0; id < prm.addn; ++id) generate_one<R>(id, 3, prm, states.data(), P[ele], nullptr);
      P[ele].n += prm.addn;
      return 0;
    }
    if (addn_out) *addn_out = 0;
    return 0;
  }

  // Build addition (no reference counterpart): re-inject at the Xmin wall as
  // many particles of the source's species as its reduce step removed this
  // cycle, with a flux-weighted half-Maxwellian normal velocity.
  int reflux(double dt, int* addn_out) {
    int total = 0;
    for (int i = 0; i < cfg.n_sources; ++i) {
      const or_source& src = cfg.src[i];
      if (src.gen_type != 7) continue;
      int s = -1;
      for (int k = 0; k < ns; ++k)
        if (std::string(cfg.sp[k].name) == src.pname) s = k;
      if (s < 0) return -1;
      uint32_t addn = uint32_t(flow[s].pulled);
      if (P[s].n + addn > cfg.pnum_max) return -2;
      ensure_states(addn);
      float Xmin = src.genX[0] < 0 ? 0.0f : float(src.genX[0]);
      float Ymin = src.genY[0] < 0 ? 0.0f : float(src.genY[0]);
      float Ymax = src.genY[0] < 0 ? float(cfg.dy * cfg.ngy) : float(src.genY[1]);
      float vth = float(std::sqrt(2 * kb * src.genT / cfg.sp[s].m));
      float u0 = float(src.genU[0]), u1 = float(src.genU[1]), u2 = float(src.genU[2]);
      float dtf = float(dt), dxf_ = float(cfg.dx), dyf_ = float(cfg.dy), ngbf = float(cfg.ngb);
      const float twoPI = 2.0f * float(PI);
      size_t base = P[s].n;
      for (uint32_t id = 0; id < addn; ++id) {
        RNGState rng = states[id];
        float r1 = rand01(rng), r2 = rand01(rng), r3 = rand01(rng), r4 = rand01(rng), r5 = rand01(rng);
        float vx = u0 + vth * std::sqrt(-std::log(r1));
        float a = vth * std::sqrt(-std::log(r2));
        float vy = u1 + a * std::cos(twoPI * r3);
        float vz = u2 + a * std::sin(twoPI * r3);
        float x = Xmin + r5 * (vx * dtf);
        float y = Ymin + r4 * (Ymax - Ymin);
        size_t k = base + id;
        P[s].x[k] = R(x / dxf_ + ngbf);
        P[s].y[k] = R(y / dyf_ + ngbf);
        P[s].vx[k] = R(vx);
        P[s].vy[k] = R(vy);
        P[s].vz[k] = R(vz);
        P[s].piflag[k] = 0;
        states[id] = rng;
      }
      P[s].n += addn;
      total += int(addn);
    }
    if (addn_out) *addn_out = total;
    return 0;
  }

  int cycle(int cyc, bool faithful, or_solve_stats* st, or_flow_stats* fs) {
    (void)cyc;
    const double dt = cfg.dt;
    reset_charge();
    for (int s = 0; s < ns; ++s) deposit(s);
    if (cfg.em_field == 1 || cfg.em_field == 2) solve_poisson(dt, -1, st);
    for (int s = 0; s < ns; ++s) {
      push(s, dt);
      reduce(s, faithful, fs ? &fs[s] : nullptr);
    }
    int a;
    if (ionize(dt, &a) != 0) return -1;
    if (hollow_cathode(dt, &a) != 0) return -1;
    if (reflux(dt, &a) != 0) return -1;
    return 0;
  }
};

template <typename F>
auto dispatch(void* h, F&& f) {
  if (auto* s32 = dynamic_cast<Sim<float>*>(static_cast<SimBase*>(h))) return f(*s32);
  return f(*dynamic_cast<Sim<double>*>(static_cast<SimBase*>(h)));
}

}  // namespace

extern "C" {

void* or_sim_create(const or_config* cfg, int real64) {
  if (real64) return static_cast<SimBase*>(new Sim<double>(*cfg));
  return static_cast<SimBase*>(new Sim<float>(*cfg));
}
void or_sim_free(void* h) { delete static_cast<SimBase*>(h); }
int or_sim_load_initial(void* h) {
  return dispatch(h, [](auto& s) { return s.load_initial(); });
}
void or_sim_reset_charge(void* h) {
  dispatch(h, [](auto& s) {
    s.reset_charge();
    return 0;
  });
}
void or_sim_deposit(void* h, int sp) {
  dispatch(h, [&](auto& s) {
    s.deposit(sp);
    return 0;
  });
}
void or_sim_solve_poisson(void* h, double dt, double tol_override, or_solve_stats* st) {
  dispatch(h, [&](auto& s) {
    s.solve_poisson(dt, tol_override, st);
    return 0;
  });
}
void or_sim_push(void* h, int sp, double dt) {
  dispatch(h, [&](auto& s) {
    s.push(sp, dt);
    return 0;
  });
}
void or_sim_reduce(void* h, int sp, int faithful, or_flow_stats* fs) {
  dispatch(h, [&](auto& s) {
    s.reduce(sp, faithful != 0, fs);
    return 0;
  });
}
int or_sim_ionize(void* h, double dt, int* addn) {
  return dispatch(h, [&](auto& s) { return s.ionize(dt, addn); });
}
int or_sim_hollow_cathode(void* h, double dt, int* addn) {
  return dispatch(h, [&](auto& s) { return s.hollow_cathode(dt, addn); });
}
int or_sim_reflux(void* h, double dt, int* addn) {
  return dispatch(h, [&](auto& s) { return s.reflux(dt, addn); });
}
int or_sim_cycle(void* h, int cycle, int faithful, or_solve_stats* st, or_flow_stats* fs) {
  return dispatch(h, [&](auto& s) { return s.cycle(cycle, faithful != 0, st, fs); });
}
unsigned int or_sim_pnum(void* h, int sp) {
  return dispatch(h, [&](auto& s) { return unsigned(s.P[sp].n); });
}
void or_sim_set_pnum(void* h, int sp, unsigned int n) {
  dispatch(h, [&](auto& s) {
    s.P[sp].n = n;
    return 0;
  });
}
void or_sim_get_particles(void* h, int sp, double* x, double* y, double* vx, double* vy, double* vz, int* fl) {
  dispatch(h, [&](auto& s) {
    auto& P = s.P[sp];
    for (size_t k = 0; k < P.n; ++k) {
      x[k] = double(P.x[k]);
      y[k] = double(P.y[k]);
      vx[k] = double(P.vx[k]);
      vy[k] = double(P.vy[k]);
      vz[k] = double(P.vz[k]);
      fl[k] = P.piflag[k];
    }
    return 0;
  });
}
void or_sim_set_particles(void* h, int sp, unsigned int n, const double* x, const double* y, const double* vx,
                          const double* vy, const double* vz, const int* fl) {
  dispatch(h, [&](auto& s) {
    using R = typename std::decay_t<decltype(s.P[0].x)>::value_type;
    auto& P = s.P[sp];
    if (P.x.size() < n) P.resize(n);
    P.n = n;
    for (size_t k = 0; k < n; ++k) {
      P.x[k] = R(x[k]);
      P.y[k] = R(y[k]);
      P.vx[k] = R(vx[k]);
      P.vy[k] = R(vy[k]);
      P.vz[k] = R(vz[k]);
      P.piflag[k] = fl ? fl[k] : 0;
    }
    return 0;
  });
}
void or_sim_get_particles_f32(void* h, int sp, float* x, float* y, float* vx, float* vy, float* vz, int* fl) {
  dispatch(h, [&](auto& s) {
    auto& P = s.P[sp];
    for (size_t k = 0; k < P.n; ++k) {
      x[k] = float(P.x[k]);
      y[k] = float(P.y[k]);
      vx[k] = float(P.vx[k]);
      vy[k] = float(P.vy[k]);
      vz[k] = float(P.vz[k]);
      fl[k] = P.piflag[k];
    }
    return 0;
  });
}
void or_sim_set_particles_f32(void* h, int sp, unsigned int n, const float* x, const float* y, const float* vx,
                              const float* vy, const float* vz, const int* fl) {
  dispatch(h, [&](auto& s) {
    using R = typename std::decay_t<decltype(s.P[0].x)>::value_type;
    auto& P = s.P[sp];
    if (P.x.size() < n) P.resize(n);
    P.n = n;
    for (size_t k = 0; k < n; ++k) {
      P.x[k] = R(x[k]);
      P.y[k] = R(y[k]);
      P.vx[k] = R(vx[k]);
      P.vy[k] = R(vy[k]);
      P.vz[k] = R(vz[k]);
      P.piflag[k] = fl ? fl[k] : 0;
    }
    return 0;
  });
}
void or_sim_get_field(void* h, int which, double* out) {
  dispatch(h, [&](auto& s) {
    if (which == 6) {
      std::copy(s.phi.begin(), s.phi.end(), out);
      return 0;
    }
    auto* v = which == 0 ? &s.rho : which == 1 ? &s.Ex : which == 2 ? &s.Ey : which == 3 ? &s.Bz
            : which == 4 ? &s.jx : &s.jy;
    for (size_t i = 0; i < v->size(); ++i) out[i] = double((*v)[i]);
    return 0;
  });
}
void or_sim_set_field(void* h, int which, const double* in) {
  dispatch(h, [&](auto& s) {
    using R = typename std::decay_t<decltype(s.rho)>::value_type;
    if (which == 6) {
      std::copy(in, in + s.phi.size(), s.phi.begin());
      return 0;
    }
    auto* v = which == 0 ? &s.rho : which == 1 ? &s.Ex : which == 2 ? &s.Ey : which == 3 ? &s.Bz
            : which == 4 ? &s.jx : &s.jy;
    for (size_t i = 0; i < v->size(); ++i) (*v)[i] = R(in[i]);
    return 0;
  });
}
void or_sim_species_consts(void* h, int sp, float* cE, float* cB, float* cX, float* cY, float* scale) {
  dispatch(h, [&](auto& s) {
    PushParams pp = s.push_params(sp, s.cfg.dt);
    *cE = float(pp.constE);
    *cB = float(pp.constB);
    *cX = float(pp.constX);
    *cY = float(pp.constY);
    *scale = s.scale(sp);
    return 0;
  });
}
int or_sim_poisson_size(void* h) {
  return dispatch(h, [](auto& s) { return s.S.A.n; });
}
double or_sim_poisson_residual(void* h, const double* sol) {
  return dispatch(h, [&](auto& s) {
    std::vector<double> b = s.S.rhs(s.rho.data(), true);
    std::vector<double> x(sol, sol + s.S.A.n);
    return s.S.rel_residual(b, x);
  });
}
void or_sim_get_poisson_solution(void* h, double* sol) {
  dispatch(h, [&](auto& s) {
    std::copy(s.phi_sol.begin(), s.phi_sol.end(), sol);
    return 0;
  });
}

// Moments of species sp (src/Moment.mm): out = 10 arrays of n_rho floats.
void or_sim_moments(void* h, int sp, int build, float* out) {
  dispatch(h, [&](auto& s) {
    std::vector<float> m[10];
    const float scale = s.wf[sp] / (s.dxf * s.dyf);
    moments(s.P[sp], s.g, s.cfg.weight_order, scale, s.mf[sp], m, build != 0);
    const size_t ng = s.g.n_rho();
    for (int a = 0; a < 10; ++a) std::copy(m[a].begin(), m[a].end(), out + a * ng);
    return 0;
  });
}

// Darwin model from given currents (see darwin_solve); lastAx/lastAy are
// updated in place; del* must be zero-initialised by the caller.
void or_darwin(int ngx, int ngy, int ngb, int perx, int pery, float dx, float dy, double dt, const float* jx,
               const float* jy, double* lastAx, double* lastAy, double* psi, double* Ax, double* Ay, float* delEx,
               float* delEy, float* delBz) {
  DarwinIn in{ngx, ngy, ngb, perx != 0, pery != 0, dx, dy, dt};
  const int n = (ngx - (perx ? 1 : 0) + 1) * (ngy - (pery ? 1 : 0) + 1);
  std::vector<double> p, ax, ay, lx(lastAx, lastAx + n), ly(lastAy, lastAy + n);
  darwin_solve<float>(in, jx, jy, p, ax, ay, lx, ly, delEx, delEy, delBz);
  std::copy(p.begin(), p.end(), psi);
  std::copy(ax.begin(), ax.end(), Ax);
  std::copy(ay.begin(), ay.end(), Ay);
  std::copy(lx.begin(), lx.end(), lastAx);
  std::copy(ly.begin(), ly.end(), lastAy);
}

static inline int64_t quant40(float w) {
  // w * 2^40 is exact in float (power-of-two scale); round half to even.
  return std::llrint(double(w * 1099511627776.0f));
}

void or_det_deposit_rho(int order, int ngx, int ngy, int ngb, int n, const int32_t* ix, const int32_t* iy,
                        const float* ox, const float* oy, int64_t* acc) {
  const int nx = ngx + 2 * ngb;
  for (int k = 0; k < n; ++k) {
    float wx[6], wy[6];
    shape_build(order, ox[k], wx);
    shape_build(order, oy[k], wy);
    // node-centred x base i2 = ix, y base j1 = iy (src/Particle.mm:360-362)
    const int ny = ngy + 2 * ngb;
    for (int i = 0; i <= order; ++i)
      for (int j = 0; j <= order; ++j) {
        int ii = ix[k] + (i - ngb), jj = iy[k] + (j - ngb);
        // nodes past the array carry weight 0 (particle exactly on the far wall)
        if (ii < 0 || jj < 0 || ii > nx || jj > ny) continue;
        acc[ii + jj * (nx + 1)] += quant40(wx[i] * wy[j]);
      }
  }
}

void or_det_deposit_j(int order, int ngx, int ngy, int ngb, int n, const int32_t* ix, const int32_t* iy,
                      const float* ox, const float* oy, const float* vx, const float* vy, int64_t* accx,
                      int64_t* accy) {
  const int nx = ngx + 2 * ngb;
  const float inv_c = float(1.0 / c_light);
  for (int k = 0; k < n; ++k) {
    // half-shifted bases: i1 = floor(x - 0.5), j2 = floor(y - 0.5)
    int i1 = ox[k] >= 0.5f ? ix[k] : ix[k] - 1;
    float hx1 = ox[k] >= 0.5f ? ox[k] - 0.5f : ox[k] + 0.5f;
    int j2 = oy[k] >= 0.5f ? iy[k] : iy[k] - 1;
    float hy2 = oy[k] >= 0.5f ? oy[k] - 0.5f : oy[k] + 0.5f;
    float wx1[6], wy1[6], wx2[6], wy2[6];
    shape_build(order, hx1, wx1);
    shape_build(order, oy[k], wy1);
    shape_build(order, ox[k], wx2);
    shape_build(order, hy2, wy2);
    const float ux = vx[k] * inv_c, uy = vy[k] * inv_c;
    const int ny = ngy + 2 * ngb;
    for (int i = 0; i <= order; ++i)
      for (int j = 0; j <= order; ++j) {
        int ii = i1 + (i - ngb + 1), jj = iy[k] + (j - ngb);
        if (ii >= 0 && jj >= 0 && ii <= nx + 1 && jj <= ny) accx[ii + jj * (nx + 2)] += quant40((wx1[i] * wy1[j]) * ux);
        ii = ix[k] + (i - ngb);
        jj = j2 + (j - ngb + 1);
        if (ii >= 0 && jj >= 0 && ii <= nx && jj <= ny + 1) accy[ii + jj * (nx + 1)] += quant40((wx2[i] * wy2[j]) * uy);
      }
  }
}

void or_shape_build(int order, float h, float* w) { shape_build(order, h, w); }
void or_shape_ref_f32(int order, float h, float* w) { shape_ref<float>(order, h, w); }
void or_shape_ref_f64(int order, double h, double* w) { shape_ref<double>(order, h, w); }

void or_pcg_stream(uint64_t master_seed, uint64_t first_slot, int nslots, int ndraws, uint32_t* out) {
  std::vector<RNGState> st;
  uint64_t m = master_seed;
  seed_states(st, 0, size_t(first_slot + nslots), m);
  for (int s = 0; s < nslots; ++s) {
    RNGState r = st[first_slot + s];
    for (int d = 0; d < ndraws; ++d) out[size_t(s) * ndraws + d] = pcg32(r);
  }
}

void or_splitmix64_stream(uint64_t seed, int n, uint64_t* out) {
  for (int i = 0; i < n; ++i) out[i] = splitmix64(seed);
}

void or_pcg32_raw(uint64_t state, uint64_t inc, int n, uint32_t* out) {
  RNGState r{state, inc};
  for (int i = 0; i < n; ++i) out[i] = pcg32(r);
}

double or_minstd_uniform(int count, double* out) {
  MinstdCanonical e;
  for (int i = 0; i < count; ++i) out[i] = e.uniform01();
  return count ? out[count - 1] : 0.0;
}

int or_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"

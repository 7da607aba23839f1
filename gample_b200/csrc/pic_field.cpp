// pic_field.cpp -- EMField and XmlLogger host objects.
#include <cmath>
#include <cstdio>
#include <iomanip>
#include <sstream>
#include <stdexcept>

#include "pic.hpp"

namespace gample {

std::string fmtSci(float v, int prec) {
  std::ostringstream oss;
  oss << std::scientific << std::setprecision(prec) << v;
  return oss.str();
}

XmlLogger::XmlLogger(const std::string& logName, const std::string& csvHeader) {
  xml_.open(logName + "_log.xml");
  if (!xml_) throw std::runtime_error("Cannot open log file: " + logName);
  xml_ << "<?xml version=\"1.0\" encoding=\"UTF-8\"?>\n"
       << "<SimulationLog>\n";
  csv_.open(logName + "_timeseries.csv");
  if (!csv_) throw std::runtime_error("Cannot open csv file: " + logName);
  csv_ << csvHeader << "\n";
}
XmlLogger::~XmlLogger() { xml_ << "</SimulationLog>\n"; }
void XmlLogger::logCycleStart(int cycle, double time) {
  if (!on_) return;
  xml_ << " <Cycle ID=\"" << cycle << "\">\n"
       << "  time = " << time << "\n";
  csv_ << cycle << "," << time;
}
void XmlLogger::logSection(const std::string& name, const std::map<std::string, std::string>& data) {
  if (!on_) return;
  xml_ << "  <Section Name=\"" << name << "\">\n";
  for (const auto& kv : data) xml_ << "   <" << kv.first << ">" << kv.second << "</" << kv.first << ">\n";
  xml_ << "  </Section>\n";
}
void XmlLogger::csvOutput(const std::string& data) {
  if (on_) csv_ << "," << data;
}
void XmlLogger::logCycleEnd() {
  if (!on_) return;
  xml_ << " </Cycle>\n";
  csv_ << "\n";
  csv_.flush();
}
void XmlLogger::logComment(const std::string& comment) { xml_ << "<![CDATA[\n" << comment << "]]>\n"; }

// ----------------------------------------------------------------- EMField

EMField::EMField(const Init& init, cudaStream_t s, int nspecies) : stream(s), host_diag_(8) {
  const ParamForField& fp = init.paramForField;
  if (fp.weightOrder != 1 && fp.weightOrder != 3 && fp.weightOrder != 5)
    throw ConfigError("WeightingOrder must be 1, 3 or 5");
  if (fp.ngx < 4 || fp.ngy < 4 || fp.ngx > 16000 || fp.ngy > 16000)
    throw ConfigError("NumberOfGridX/Y must be in [4, 16000]");
  dims.ngx = fp.ngx;
  dims.ngy = fp.ngy;
  dims.ngb = fp.ngb;
  dims.nx = fp.ngx + 2 * fp.ngb;
  dims.ny = fp.ngy + 2 * fp.ngb;
  dx = float(fp.dx);
  dy = float(fp.dy);
  det = init.paramForComputing.depositMode == 1;
  current = fp.checkCurDens == 1 || init.flagForEquation.EMField > 1;  // src/Particle.mm:523-525
  maxiter = init.paramForComputing.maxiter;
  tol = double(init.paramForComputing.tolerance);

  rho.resize(n_rho(), true);
  jx.resize(n_ex(), true);
  jy.resize(n_ey(), true);
  Ex.resize(n_ex(), true);
  Ey.resize(n_ey(), true);
  Ez.resize(n_rho(), true);
  Bx.resize(n_ey(), true);
  By.resize(n_ex(), true);
  Bz.resize(n_bz(), true);
  delEx.resize(n_ex(), true);
  delEy.resize(n_ey(), true);
  delBz.resize(n_bz(), true);
  phi.resize(n_phi(), true);
  diag.resize(8, true);

  // Initial E and B: src/EMField.mm:146-197
  auto amp = [](const std::vector<double>& v, int i) { return i < int(v.size()) ? float(v[i]) : 0.0f; };
  if (fp.InitTypeE == "Uniform") {
    kern::fill_f32(Ex.get(), n_ex(), amp(fp.ampE, 0), s);
    kern::fill_f32(Ey.get(), n_ey(), amp(fp.ampE, 1), s);
    kern::fill_f32(Ez.get(), n_rho(), amp(fp.ampE, 2), s);
  }
  if (fp.InitTypeB == "Uniform") {
    kern::fill_f32(Bx.get(), n_ey(), amp(fp.ampB, 0), s);
    // The reference fills (nx+1)(ny+2) entries of the (nx+2)(ny+1) By buffer
    // (src/EMField.mm:169-171); By is never read by the push, so all of it is
    // filled here.
    kern::fill_f32(By.get(), n_ex(), amp(fp.ampB, 1), s);
    kern::fill_f32(Bz.get(), n_bz(), amp(fp.ampB, 2), s);
    bz_uniform = true;
    bz_value = amp(fp.ampB, 2);
  } else if (fp.InitTypeB == "From1dXFile") {
    const int nx = dims.nx, ny = dims.ny;
    std::vector<float> bx, by, bz;
    load1dField(fp.FilePathBx, bx, size_t(nx) + 1);
    load1dField(fp.FilePathBy, by, size_t(nx) + 2);
    load1dField(fp.FilePathBz, bz, size_t(nx) + 2);
    std::vector<float> hbx(n_ey()), hby(n_ex()), hbz(n_bz());
    for (int i = 0; i <= nx; i++)
      for (int j = 0; j <= ny + 1; j++) hbx[i + j * (nx + 1)] = float(bx[i] * phys::TtoG);
    for (int i = 0; i <= nx + 1; i++)
      for (int j = 0; j <= ny; j++) hby[i + j * (nx + 2)] = float(by[i] * phys::TtoG);
    for (int i = 0; i <= nx + 1; i++)
      for (int j = 0; j <= ny + 1; j++) hbz[i + j * (nx + 2)] = float(bz[i] * phys::TtoG);
    GP_CUDA(cudaMemcpyAsync(Bx.get(), hbx.data(), Bx.bytes(), cudaMemcpyHostToDevice, s));
    GP_CUDA(cudaMemcpyAsync(By.get(), hby.data(), By.bytes(), cudaMemcpyHostToDevice, s));
    GP_CUDA(cudaMemcpyAsync(Bz.get(), hbz.data(), Bz.bytes(), cudaMemcpyHostToDevice, s));
    GP_CUDA(cudaStreamSynchronize(s));
  }

  // Field boundaries and Poisson layout: src/EMField.mm:199-271
  std::array<double, 4> vals{};
  auto codes = init.fieldBCCodes(&vals, &cathodePos);
  for (int w = 0; w < 4; ++w) {
    fbc[w] = codes[w];
    if (codes[w] == FBC_UNDEF) throw ConfigError("field boundary condition missing or unknown");
    if (codes[w] == FBC_NEUMANN)
      throw ConfigError("Neumann boundary condition is included (rejected as in src/EMField.mm:433-436)");
  }
  kern::PoissonLayout& L = layout;
  L.nkx = dims.ngx;
  L.ikmin = dims.ngb;
  if (fbc[XMIN] == FBC_DIRICHLET) {
    L.nkx--;
    L.ikmin++;
  }
  if (fbc[XMAX] == FBC_DIRICHLET) L.nkx--;
  if (fbc[XMIN] == FBC_PERIODIC) L.nkx--;
  L.nky = dims.ngy;
  L.jkmin = dims.ngb;
  if (fbc[YMIN] == FBC_DIRICHLET) {
    L.nky--;
    L.jkmin++;
  }
  if (fbc[YMAX] == FBC_DIRICHLET) L.nky--;
  if (fbc[YMIN] == FBC_PERIODIC) L.nky--;
  for (int w = 0; w < 4; ++w) L.fbc[w] = fbc[w];
  L.Cd = -2 * (1.0 / dx / dx + 1.0 / dy / dy);
  L.Cx = 1.0 / dx / dx;
  L.Cy = 1.0 / dy / dy;
  L.phiXmin = vals[XMIN] * phys::VtosV;
  L.phiXmax = vals[XMAX] * phys::VtosV;
  L.phiYmin = vals[YMIN] * phys::VtosV;
  L.phiYmax = vals[YMAX] * phys::VtosV;
  L.periodic_x = fbc[XMIN] == FBC_PERIODIC;
  L.periodic_y = fbc[YMIN] == FBC_PERIODIC;
  mg = std::make_unique<PoissonMG>(L);
  sol.resize(size_t(mg->unknowns()), true);
  b.resize(size_t(mg->unknowns()), true);
  if (init.flagForEquation.EMField == 2) setupDarwin();
  if (!det && !current && bz_uniform) {
    const size_t pitch = size_t(kern::field_pitch(dims));
    Exp.resize(pitch * (dims.ny + 1), true);
    Eyp.resize(pitch * (dims.ny + 2), true);
    if (!kern::make_field_maps(Exp.get(), Eyp.get(), dims, &maps)) {
      Exp = DeviceArray<float>();
      Eyp = DeviceArray<float>();
    }
  }

  acc_rho.resize(nspecies);
  acc_jx.resize(nspecies);
  acc_jy.resize(nspecies);
  f64_rho.resize(nspecies);
  f64_jx.resize(nspecies);
  f64_jy.resize(nspecies);
  species_scale.assign(nspecies, 0.0f);
  for (int sp = 0; sp < nspecies; ++sp) {
    if (det) {
      acc_rho[sp].resize(n_rho(), true);
      if (current) {
        acc_jx[sp].resize(n_ex(), true);
        acc_jy[sp].resize(n_ey(), true);
      }
    } else {
      f64_rho[sp].resize(n_rho(), true);
      if (current) {
        f64_jx[sp].resize(n_ex(), true);
        f64_jy[sp].resize(n_ey(), true);
      }
    }
  }
  GP_CUDA(cudaStreamSynchronize(s));
}

const kern::FieldMaps* EMField::pushMaps() {
  if (!maps.valid) return nullptr;
  if (e_pitched_stale) {
    kern::pitch_fields(Ex.get(), Ey.get(), dims, Exp.get(), Eyp.get(), stream);
    e_pitched_stale = false;
  }
  return &maps;
}

void EMField::load1dField(const std::string& path, std::vector<float>& out, size_t need) const {
  FILE* fp = std::fopen(path.c_str(), "rb");
  if (!fp) throw ConfigError("Unable to open file " + path + " for reading");
  int n = 0;
  float d = 0;
  if (std::fread(&n, sizeof(int), 1, fp) != 1 || std::fread(&d, sizeof(float), 1, fp) != 1 || n < 0) {
    std::fclose(fp);
    throw ConfigError("Unable to read header of " + path);
  }
  out.resize(size_t(n) + 1);
  if (std::fread(out.data(), sizeof(float), out.size(), fp) != out.size()) {
    std::fclose(fp);
    throw ConfigError("Unable to read data of " + path);
  }
  std::fclose(fp);
  if (out.size() < need) throw ConfigError(path + " holds fewer points than the grid needs");
}

kern::DepositTargets EMField::targets(int s) {
  kern::DepositTargets t{};
  if (s < 0 || s >= int(acc_rho.size())) throw std::invalid_argument("species index out of range");
  if (det) {
    t.acc_rho = acc_rho[s].get();
    t.acc_jx = current ? acc_jx[s].get() : nullptr;
    t.acc_jy = current ? acc_jy[s].get() : nullptr;
  } else {
    t.f64_rho = f64_rho[s].get();
    t.f64_jx = current ? f64_jx[s].get() : nullptr;
    t.f64_jy = current ? f64_jy[s].get() : nullptr;
  }
  return t;
}

void EMField::resetChargeDensity() {
  rho.zero(stream);
  jx.zero(stream);
  jy.zero(stream);
  for (size_t s = 0; s < acc_rho.size(); ++s) {
    acc_rho[s].zero(stream);
    acc_jx[s].zero(stream);
    acc_jy[s].zero(stream);
    f64_rho[s].zero(stream);
    f64_jx[s].zero(stream);
    f64_jy[s].zero(stream);
  }
  charge_dirty = false;
}

void EMField::finalizeCharge() {
  if (!charge_dirty) return;
  charge_dirty = false;
  const int ns = int(acc_rho.size());
  if (det) {
    std::vector<const long long*> pr(ns), px(ns), py(ns);
    for (int s = 0; s < ns; ++s) {
      pr[s] = acc_rho[s].get();
      px[s] = acc_jx[s].get();
      py[s] = acc_jy[s].get();
    }
    kern::combine_fixed_point(pr.data(), species_scale.data(), ns, n_rho(), 1.0, rho.get(), stream);
    if (current) {
      kern::combine_fixed_point(px.data(), species_scale.data(), ns, n_ex(), phys::c, jx.get(), stream);
      kern::combine_fixed_point(py.data(), species_scale.data(), ns, n_ey(), phys::c, jy.get(), stream);
    }
  } else {
    std::vector<const double*> pr(ns), px(ns), py(ns);
    for (int s = 0; s < ns; ++s) {
      pr[s] = f64_rho[s].get();
      px[s] = f64_jx[s].get();
      py[s] = f64_jy[s].get();
    }
    kern::combine_f64(pr.data(), ns, n_rho(), rho.get(), stream);
    if (current) {
      kern::combine_f64(px.data(), ns, n_ex(), jx.get(), stream);
      kern::combine_f64(py.data(), ns, n_ey(), jy.get(), stream);
    }
  }
}

SolveStats EMField::solvePoisson(double dt, XmlLogger* logger) {
  SolveStats st;
  finalizeCharge();
  kern::fold_ghosts(rho.get(), dims, fbc, stream);
  const int n = mg->unknowns();
  double* d = diag.get();
  kern::build_rhs(rho.get(), dims, layout, b.get(), d, stream);
  if (layout.periodic_x && layout.periodic_y) {
    // The doubly periodic system is singular: project the rhs onto the range
    // (zero mean) and fix the gauge (zero-mean solution). The reference skips
    // the projection (src/EMField.mm:852-861).
    kern::subtract_mean(b.get(), n, d, stream);
    kern::vec_sums(b.get(), n, d, stream);
  }
  last_mg = poissonSolve(d);
  kern::phi_fill(sol.get(), dims, layout, dx, cathodePos, d + 4, phi.get(), stream);
  kern::gradient_energy(phi.get(), dims, dx, dy, Ex.get(), Ey.get(), jx.get(), jy.get(), d + 2, stream,
                        maps.valid ? Exp.get() : nullptr, maps.valid ? Eyp.get() : nullptr);
  e_pitched_stale = false;
  kern::probe(phi.get(), Ex.get(), Ey.get(), dims, d + 5, stream);
  GP_CUDA(cudaMemcpyAsync(host_diag_.get(), d, 8 * sizeof(double), cudaMemcpyDeviceToHost, stream));
  GP_CUDA(cudaStreamSynchronize(stream));
  const double* h = host_diag_.get();
  st.iterations = last_mg.iterations;
  st.error = last_mg.rel_residual;
  const double mean = cathodePos > 0.0 ? h[4] : 0.0;
  st.meanCathode = mean * phys::sVtoV;
  // src/EMField.mm:1112-1116
  st.energy = h[2] * (double(dx) * dy / 2);
  st.joule = h[3] * (double(dt) * dx * dy);
  st.EEincrement = st.energy - lastEE;
  lastEE = st.energy;
  st.field_energy_cgs = h[2] * double(dx) * dy / (8 * phys::PI);
  st.probe[0] = h[5];
  st.probe[1] = h[6];
  st.probe[2] = h[7];
  if (logger && logger->on()) {
    logger->logSection("solvePoisson", {{"iteration", std::to_string(st.iterations)},
                                        {"error", fmtSci(float(st.error), 6)},
                                        {"meanCathode", fmtSci(float(st.meanCathode), 6)},
                                        {"totalElectricEnergy", fmtSci(float(st.energy * phys::ergtoev), 6)},
                                        {"totalEEincrement", fmtSci(float(st.EEincrement * phys::ergtoev), 6)},
                                        {"jouleHeating", fmtSci(float(st.joule * phys::ergtoev), 6)}});
    logger->csvOutput(fmtSci(float(st.probe[0]), 6) + "," + fmtSci(float(st.probe[1]), 6) + "," +
                      fmtSci(float(st.probe[2]), 6));
  }
  return st;
}

}  // namespace gample

// fileio.cpp -- binary field/moment/phase-space output and restart files
// (src/FileIO.mm). Device arrays are copied to the host only here.
#include "fileio.hpp"

#include <cstdio>
#include <cstring>
#include <iostream>

namespace gample {

namespace {

constexpr double kGtoV = 1 / (1e6 / phys::c);   // statV/cm -> V/m (src/Constant.h:17)
constexpr double kGtoT = 1e-4;                  // G -> T (src/Constant.h:25)
constexpr double kSJtoJ = 10 / phys::c * 1e4;   // statA/cm^2 -> A/m^2 (src/Constant.h:23)

std::string fmt_cycle(int cycle) {
  char b[16];
  std::snprintf(b, sizeof(b), "%08d", cycle);
  return b;
}

template <typename T>
std::vector<T> fetch(const DeviceArray<T>& a, size_t n, size_t offset, cudaStream_t s) {
  std::vector<T> h(n);
  if (n) {
    GP_CUDA(cudaMemcpyAsync(h.data(), a.get() + offset, n * sizeof(T), cudaMemcpyDeviceToHost, s));
    GP_CUDA(cudaStreamSynchronize(s));
  }
  return h;
}

// src/FileIO.mm:228-248: 32-byte name, type id, array * scale (FP32)
void writeField(FILE* fp, const std::string& name, int type_id, const float* a, size_t n, float scale) {
  char nb[32] = {};
  std::strncpy(nb, name.c_str(), sizeof(nb) - 1);
  std::fwrite(nb, 1, 32, fp);
  std::fwrite(&type_id, sizeof(int), 1, fp);
  std::vector<float> o(n);
  for (size_t i = 0; i < n; ++i) o[i] = a[i] * scale;
  std::fwrite(o.data(), sizeof(float), n, fp);
}

// The reference's min/max scan: `else if`, so a new minimum is not also
// tested as a maximum (src/FileIO.mm:77-95).
void minmax(const std::vector<float>& a, float& mn, float& mx) {
  mn = 1e20f;
  mx = -1e20f;
  for (float v : a) {
    if (v < mn)
      mn = v;
    else if (v > mx)
      mx = v;
  }
}

void header(FILE* fp, int ngx, int ngy, int ngb, float dx, float dy) {
  std::fwrite(&ngx, sizeof(int), 1, fp);
  std::fwrite(&ngy, sizeof(int), 1, fp);
  std::fwrite(&ngb, sizeof(int), 1, fp);
  std::fwrite(&dx, sizeof(float), 1, fp);
  std::fwrite(&dy, sizeof(float), 1, fp);
}

}  // namespace

void outputField(int cycle, EMField& fld, const Init& init, XmlLogger* logger) {
  const auto& T = init.paramForTimeIntegration;
  const std::string path = "bin/" + T.ProjectName + "_EMField_" + fmt_cycle(cycle) + ".bin";
  if (fld.charge_dirty) fld.finalizeCharge();
  cudaStream_t s = fld.stream;
  const auto rho = fetch(fld.rho, fld.n_rho(), 0, s);
  const auto phid = fetch(fld.phi, fld.n_phi(), 0, s);
  std::vector<float> phi(phid.size());
  for (size_t i = 0; i < phid.size(); ++i) phi[i] = float(phid[i]);  // src/EMField.mm:1396-1403
  const auto Ex = fetch(fld.Ex, fld.n_ex(), 0, s);
  const auto Ey = fetch(fld.Ey, fld.n_ey(), 0, s);
  const auto Bz = fetch(fld.Bz, fld.n_bz(), 0, s);
  float a0, a1, b0, b1, c0, c1, d0, d1;
  minmax(rho, a0, a1);
  minmax(Ex, c0, c1);
  minmax(Ey, d0, d1);
  minmax(phi, b0, b1);
  if (logger)
    logger->logSection("outputField", {{"rho_min", fmtSci(a0, 6)},
                                       {"rho_max", fmtSci(a1, 6)},
                                       {"phi_min", fmtSci(float(b0 * phys::sVtoV), 6)},
                                       {"phi_max", fmtSci(float(b1 * phys::sVtoV), 6)},
                                       {"Ex_min", fmtSci(float(c0 * kGtoV), 6)},
                                       {"Ex_max", fmtSci(float(c1 * kGtoV), 6)},
                                       {"Ey_min", fmtSci(float(d0 * kGtoV), 6)},
                                       {"Ey_max", fmtSci(float(d1 * kGtoV), 6)}});
  FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) {
    std::cerr << "Error: Unable to open file " << path << " for writing\n";
    return;
  }
  const int nx = fld.dims.nx, ny = fld.dims.ny;
  header(fp, fld.dims.ngx, fld.dims.ngy, fld.dims.ngb, fld.dx, fld.dy);
  writeField(fp, "rho", 0, rho.data(), size_t(nx + 1) * (ny + 1), 1.0f);
  writeField(fp, "phi", 4, phi.data(), size_t(nx + 3) * (ny + 3), float(phys::sVtoV));
  writeField(fp, "Ex", 1, Ex.data(), size_t(nx + 2) * (ny + 1), float(kGtoV));
  writeField(fp, "Ey", 2, Ey.data(), size_t(nx + 1) * (ny + 2), float(kGtoV));
  writeField(fp, "Bz", 3, Bz.data(), size_t(nx + 2) * (ny + 2), float(kGtoT));
  if (init.flagForEquation.EMField == 2) {
    const auto jx = fetch(fld.jx, fld.n_ex(), 0, s);
    const auto jy = fetch(fld.jy, fld.n_ey(), 0, s);
    const auto dEx = fetch(fld.delEx, fld.n_ex(), 0, s);
    const auto dEy = fetch(fld.delEy, fld.n_ey(), 0, s);
    const auto dBz = fetch(fld.delBz, fld.n_bz(), 0, s);
    writeField(fp, "jx", 1, jx.data(), jx.size(), float(kSJtoJ));
    writeField(fp, "jy", 2, jy.data(), jy.size(), float(kSJtoJ));
    writeField(fp, "delEx", 1, dEx.data(), dEx.size(), float(kGtoV));
    writeField(fp, "delEy", 2, dEy.data(), dEy.size(), float(kGtoV));
    writeField(fp, "delBz", 3, dBz.data(), dBz.size(), float(kGtoT));
  }
  std::fclose(fp);
}

void outputMoments(int cycle, Moment& mom, const std::string& pName, const Init& init, XmlLogger* logger) {
  const auto& T = init.paramForTimeIntegration;
  const auto& F = init.paramForField;
  const std::string path = "bin/" + T.ProjectName + "_Moments_" + pName + "_" + fmt_cycle(cycle) + ".bin";
  const size_t ng = mom.n_rho();
  const auto all = fetch(mom.out, Moment::kCount * ng, 0, mom.stream);
  static const char* names[Moment::kCount] = {"n", "ux", "uy", "uz", "Pxx", "Pxy", "Pxz", "Pyy", "Pyz", "Pzz"};
  float mn[Moment::kCount], mx[Moment::kCount];
  for (int q = 0; q < Moment::kCount; ++q) {
    mn[q] = 1e20f;
    mx[q] = -1e20f;
  }
  // src/FileIO.mm:164-176 (uz is never scanned: the uy line is repeated)
  for (size_t i = 0; i < ng; ++i)
    for (int q = 0; q < Moment::kCount; ++q) {
      if (q == 3) continue;
      const int src = q;
      const float v = all[size_t(src) * ng + i];
      if (v < mn[q])
        mn[q] = v;
      else if (v > mx[q])
        mx[q] = v;
    }
  if (logger) {
    std::map<std::string, std::string> data;
    for (int q = 0; q < Moment::kCount; ++q) {
      const double f = q >= 4 ? 0.1 : 1.0;
      data[std::string(names[q]) + "_min"] = fmtSci(float(mn[q] * f), 6);
      data[std::string(names[q]) + "_max"] = fmtSci(float(mx[q] * f), 6);
    }
    logger->logSection("outputMoment_" + pName, data);
  }
  FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) {
    std::cerr << "Error: Unable to open file " << path << " for writing\n";
    return;
  }
  header(fp, F.ngx, F.ngy, F.ngb, float(F.dx), float(F.dy));
  for (int q = 0; q < Moment::kCount; ++q)
    writeField(fp, pName + "_" + names[q], 0, all.data() + size_t(q) * ng, ng, q >= 4 ? 0.1f : 1.0f);
  std::fclose(fp);
}

void outputPhaseSpace(int cycle, Particle& p, const Init& init) {
  const auto& T = init.paramForTimeIntegration;
  const auto& F = init.paramForField;
  const uint32_t n = p.pNum();
  const uint32_t k = n < 20 ? n : 20;
  std::vector<kern::ParticleStateAoS> h(20);
  if (k) p.download_aos(h.data(), k);
  // src/FileIO.mm:13-35: the reference writes records 0..19 whatever pNum is;
  // slots beyond the live count are written as zeros here.
  for (int idx = 0; idx < 20; ++idx) {
    const std::string path = "bin/" + T.ProjectName + "_PhaseSpace_" + p.pName + "_" + std::to_string(idx) + ".bin";
    FILE* fp = std::fopen(path.c_str(), "ab");
    if (!fp) {
      std::cerr << "Failed to open file: " << path << "\n";
      continue;
    }
    const kern::ParticleStateAoS r = uint32_t(idx) < k ? h[idx] : kern::ParticleStateAoS{};
    const float x = float((r.x - float(F.ngb)) * F.dx);
    const float y = float((r.y - float(F.ngb)) * F.dy);
    std::fwrite(&cycle, sizeof(int), 1, fp);
    std::fwrite(&x, sizeof(float), 1, fp);
    std::fwrite(&y, sizeof(float), 1, fp);
    std::fwrite(&r.vx, sizeof(float), 1, fp);
    std::fwrite(&r.vy, sizeof(float), 1, fp);
    std::fwrite(&r.vz, sizeof(float), 1, fp);
    std::fclose(fp);
  }
}

bool saveProgress(int cycle, std::vector<Particle*>& ptcls, const Init& init) {
  const auto& T = init.paramForTimeIntegration;
  for (auto* p : ptcls) {
    const std::string path = "bin/" + T.ProjectName + "_ProgressData_" + p->pName + "_" + fmt_cycle(cycle) + ".bin";
    const uint32_t n = p->pNum();
    std::vector<kern::ParticleStateAoS> h(n);
    if (n) p->download_aos(h.data(), n);
    FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) {
      std::cerr << "[Error] file open failed: " << path << "\n";
      return false;
    }
    const size_t w = n ? std::fwrite(h.data(), sizeof(kern::ParticleStateAoS), n, fp) : 0;
    std::fclose(fp);
    if (w != n) return false;
  }
  return true;
}

bool loadProgress(int cycle, std::vector<Particle*>& ptcls, const Init& init) {
  const auto& T = init.paramForTimeIntegration;
  const int shift = init.paramForField.diff_ngb;
  for (auto* p : ptcls) {
    const std::string path = "bin/" + T.RestartName + "_ProgressData_" + p->pName + "_" + fmt_cycle(cycle) + ".bin";
    FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) {
      std::cerr << "[Error] file open failed: " << path << "\n";
      return false;
    }
    std::fseek(fp, 0, SEEK_END);
    const long size = std::ftell(fp);
    std::rewind(fp);
    if (size < 0 || size_t(size) > size_t(p->pNumMax) * sizeof(kern::ParticleStateAoS)) {
      std::fclose(fp);
      std::cerr << "[Error] check filesize failed.\n";
      return false;
    }
    const uint32_t n = uint32_t(size_t(size) / sizeof(kern::ParticleStateAoS));
    std::vector<kern::ParticleStateAoS> h(n);
    const size_t r = n ? std::fread(h.data(), sizeof(kern::ParticleStateAoS), n, fp) : 0;
    std::fclose(fp);
    if (r != n) return false;
    if (shift != 0)  // src/FileIO.mm:318-323 (PtclPosOffset)
      for (auto& q : h) {
        q.x += float(shift);
        q.y += float(shift);
      }
    p->upload_aos(h.data(), n);
  }
  return true;
}

}  // namespace gample

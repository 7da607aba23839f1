// init.cpp -- condition-file parser (mirror of src/Init.mm:27-394).
#include "init.hpp"

#include <cmath>
#include <fstream>
#include <iomanip>
#include <limits>
#include <sstream>

#include "json.hpp"

namespace gample {

namespace {

using json::Value;

// NSNumber/NSString integerValue: truncation toward zero; strings parse a
// leading integer; anything else is 0.
long long as_int(const Value* v) {
  if (!v) return 0;
  switch (v->kind) {
    case Value::Bool: return v->b ? 1 : 0;
    case Value::Number:
      if (!std::isfinite(v->num)) return 0;
      if (v->num >= 9.2e18 || v->num <= -9.2e18) return 0;
      return (long long)v->num;
    case Value::String: {
      const std::string& s = v->str;
      size_t i = 0;
      while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
      std::string digits;
      if (i < s.size() && (s[i] == '+' || s[i] == '-')) digits += s[i++];
      while (i < s.size() && std::isdigit((unsigned char)s[i])) digits += s[i++];
      try {
        return digits.empty() ? 0 : std::stoll(digits);
      } catch (...) {
        return 0;
      }
    }
    default: return 0;
  }
}
double as_dbl(const Value* v) {
  if (!v) return 0;
  switch (v->kind) {
    case Value::Bool: return v->b ? 1.0 : 0.0;
    case Value::Number: return v->num;
    case Value::String: {
      try {
        return std::stod(v->str);
      } catch (...) {
        return 0.0;
      }
    }
    default: return 0.0;
  }
}
std::string as_str(const Value* v, const std::string& dflt) {
  if (!v) return dflt;
  if (v->kind == Value::String) return v->str;
  return dflt;
}
std::vector<double> as_vec(const Value* v, const std::vector<double>& dflt) {
  if (!v) return dflt;
  std::vector<double> out;
  if (v->kind == Value::Array)
    for (const auto& e : v->arr) out.push_back(as_dbl(&e));
  return out;
}

// Merged lookup: key present in the section wins, else the default.
struct Section {
  const Value* d;
  const Value* get(const char* k) const { return d ? d->find(k) : nullptr; }
  long long i(const char* k, long long dflt) const {
    const Value* v = get(k);
    return v ? as_int(v) : dflt;
  }
  double f(const char* k, double dflt) const {
    const Value* v = get(k);
    return v ? as_dbl(v) : dflt;
  }
  std::string s(const char* k, const std::string& dflt) const {
    const Value* v = get(k);
    return v ? as_str(v, "") : dflt;
  }
  std::vector<double> vec(const char* k, const std::vector<double>& dflt) const {
    const Value* v = get(k);
    return v ? as_vec(v, dflt) : dflt;
  }
};

const Value& require_object(const Value& root, const char* key) {
  const Value* v = root.find(key);
  if (!v || !v->is_object()) throw ConfigError(std::string(key) + " is not an object");
  return *v;
}
const Value& require_array(const Value& root, const char* key) {
  const Value* v = root.find(key);
  if (!v || !v->is_array()) throw ConfigError(std::string(key) + " is not an array");
  return *v;
}

}  // namespace

Init Init::parseInputFile(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw ConfigError("cannot read " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return parseString(ss.str());
}

Init Init::parseString(const std::string& text) {
  Value root;
  try {
    root = json::parse(text);
  } catch (const json::Error& e) {
    throw ConfigError(e.what());
  }
  if (!root.is_object()) throw ConfigError("top level is not an object");
  Init I;
  {  // FlagForEquation: src/Init.mm:53-66
    Section s{&require_object(root, "FlagForEquation")};
    I.flagForEquation.Particle = int(s.i("Particle", 0));
    I.flagForEquation.EMField = int(s.i("EMField", 0));
    I.flagForEquation.MCCollision = int(s.i("MCCollision", 0));
  }
  {  // ParamForTimeIntegration: src/Init.mm:68-88
    Section s{&require_object(root, "ParamForTimeIntegration")};
    auto& t = I.paramForTimeIntegration;
    t.Start = int(s.i("Start", 0));
    t.End = int(s.i("End", 0));
    t.TimeStep = s.f("TimeStep", 0);
    t.LogOutput = int(s.i("LogOutput", 0));
    t.ParticleOutput = int(s.i("ParticleOutput", 0));
    t.FieldOutput = int(s.i("FieldOutput", 0));
    t.ProgressOutput = int(s.i("ProgressOutput", 0));
    t.ProjectName = s.s("ProjectName", "undefined");
    t.RestartName = s.s("RestartName", "undefined");
  }
  {  // ParamForComputing: src/Init.mm:90-107
    Section s{&require_object(root, "ParamForComputing")};
    auto& c = I.paramForComputing;
    const Value* mp = s.get("MaximumParticleNumber");
    c.pNumMax = uint32_t(mp ? as_int(mp) : 0);  // default @0.08 -> integerValue 0
    c.threadGroupSize = int(s.i("ThreadGroupSize", 256));
    c.integrationChunkSize = int(s.i("IntegrationChunkSize", 256));
    c.aggrThreshold = float(s.f("AggregationThreshold", 0.1));
    c.chebDegree = int(s.i("ChebyshevDegree", 5));
    c.amgCycleType = int(s.i("AMGCycleType", 1));
    c.maxiter = int(s.i("MaxiterForPoisson", 200));
    c.tolerance = float(s.f("ToleranceForPoisson", 1e-7));
    c.depositMode = int(s.i("DepositMode", 0));
    c.sortInterval = int(s.i("SortInterval", 0));
    c.masterSeed = uint64_t(s.i("MasterSeed", 0));
  }
  {  // ParamForField: src/Init.mm:109-146
    Section s{&require_object(root, "ParamForField")};
    auto& f = I.paramForField;
    f.ngx = int(s.i("NumberOfGridX", 0));
    f.ngy = int(s.i("NumberOfGridY", 0));
    f.dx = s.f("GridSizeOfX", 0);
    f.dy = s.f("GridSizeOfY", 0);
    f.InitTypeE = s.s("InitializeTypeOfE", "undefined");
    f.ampE = s.vec("AmplitudeOfE", {0, 0, 0});
    f.FilePathEx = s.s("FilePathOfEx", "undefined");
    f.FilePathEy = s.s("FilePathOfEy", "undefined");
    f.FilePathEz = s.s("FilePathOfEz", "undefined");
    f.InitTypeB = s.s("InitializeTypeOfB", "undefined");
    f.ampB = s.vec("AmplitudeOfB", {0, 0, 0});
    f.FilePathBx = s.s("FilePathOfBx", "undefined");
    f.FilePathBy = s.s("FilePathOfBy", "undefined");
    f.FilePathBz = s.s("FilePathOfBz", "undefined");
    f.weightOrder = int(s.i("WeightingOrder", 5));
    f.ngb = f.weightOrder / 2;
    f.diff_ngb = int(s.i("PtclPosOffset", 0));
    f.BorisOrder = int(s.i("BorisOrder", 2));
    f.checkCurDens = int(s.i("FlagForCurDens", 0));
  }
  {  // BoundaryConditionForField: src/Init.mm:148-167
    const Value& arr = require_array(root, "BoundaryConditionForField");
    for (const auto& e : arr.arr) {
      if (!e.is_object()) continue;
      Section s{&e};
      BoundaryConditionForField bc;
      bc.position = s.s("RegionName", "undefined");
      bc.type = s.s("BCType", "undefined");
      bc.val = s.f("Value", 0);
      I.fieldBoundaries.push_back(bc);
    }
  }
  const int ngx = I.paramForField.ngx, ngy = I.paramForField.ngy;
  {  // ParamForParticle: src/Init.mm:169-226
    const Value& arr = require_array(root, "ParamForParticle");
    for (const auto& e : arr.arr) {
      if (!e.is_object()) continue;
      Section s{&e};
      ParamForParticle p;
      p.pName = s.s("ParticleName", "undefined");
      std::string pm = s.s("pNumSetMethod", "undefined");
      if (pm == "InitialParticleNumber")
        p.pNum = uint32_t(s.i("pNumValue", 0));
      else if (pm == "PtclNumPerCell")
        p.pNum = uint32_t(s.i("pNumValue", 0) * ngx * ngy);
      else
        throw ConfigError("pNumSet failed.");
      p.q = s.f("Charge", 0);
      p.m = s.f("Mass", -1);
      std::string wm = s.s("WeightSetMethod", "undefined");
      if (wm == "WeightValue") {
        p.w = s.f("WeightValue", 0);
      } else if (wm == "InitialNumDens") {
        double ppc = double(p.pNum) / double(ngx * ngy);
        p.w = s.f("WeightValue", 0) * I.paramForField.dx * I.paramForField.dy / ppc;
      } else {
        throw ConfigError("WeightSet failed.");
      }
      p.genType = s.s("GenerateType", "undefined");
      p.genX = s.vec("InitialPosX", {-1, -1});
      p.genY = s.vec("InitialPosY", {-1, -1});
      p.genU = s.vec("InitialVel", {0, 0, 0});
      p.genT = s.f("InitialTemp", 0) * phys::eVtoK;
      p.sinU = s.vec("SinusoidalDriftVel", {0, 0, 0});
      I.paramForParticle.push_back(p);
    }
  }
  {  // SourceForParticle: src/Init.mm:228-282
    const Value& arr = require_array(root, "SourceForParticle");
    for (const auto& e : arr.arr) {
      if (!e.is_object()) continue;
      Section s{&e};
      SourceForParticle src;
      src.pName = s.s("ParticleName", "undefined");
      src.genType = s.s("GenerateType", "undefined");
      std::string m = s.s("SrcSetMethod", "undefined");
      double val = s.f("SrcValue", 0);
      if (m == "Source[1/cm/s]")
        src.src = val;
      else if (m == "CurrentDensity[A/m2]")
        src.src = val * phys::JtosJ * ngy * I.paramForField.dy / phys::ec;
      else if (m == "BoundaryCurrentAtXmin")
        src.src = 0;
      else if (m == "BoundaryCurrentAtXmax")
        src.src = 1;
      else if (m == "BoundaryCurrentAtYmin")
        src.src = 2;
      else if (m == "BoundaryCurrentAtYmax")
        src.src = 3;
      else if (m == "AbsorbedParticleNumber")  // build addition: fluxMaxwellianAtXmin
        src.src = 0;
      else
        throw ConfigError("SrcSet failed.");
      src.genX = s.vec("GeneratePosX", {-1, -1});
      src.genY = s.vec("GeneratePosY", {-1, -1});
      src.genU = s.vec("GenerateVel", {0, 0, 0});
      src.genT = s.f("GenerateTemp", 0) * phys::eVtoK;
      src.genU_ele = s.vec("GenVelForElectron", {0, 0, 0});
      src.genT_ele = s.f("GenTempForElectron", 0) * phys::eVtoK;
      I.particleSources.push_back(src);
    }
  }
  {  // BoundaryConditionForParticle: src/Init.mm:284-298 (no default merge)
    const Value& arr = require_array(root, "BoundaryConditionForParticle");
    for (const auto& e : arr.arr) {
      if (!e.is_object()) continue;
      BoundaryConditionForParticle bc;
      bc.position = as_str(e.find("RegionName"), "");
      bc.type = as_str(e.find("BCType"), "");
      I.particleBoundaries.push_back(bc);
    }
  }
  return I;
}

std::array<int, 4> Init::fieldBCCodes(std::array<double, 4>* values, double* cathodePos) const {
  std::array<int, 4> codes{FBC_UNDEF, FBC_UNDEF, FBC_UNDEF, FBC_UNDEF};
  if (values) values->fill(0.0);
  if (cathodePos) *cathodePos = -1.0;
  static const char* walls[4] = {"Xmin", "Xmax", "Ymin", "Ymax"};
  for (const auto& bc : fieldBoundaries) {
    for (int w = 0; w < 4; ++w) {
      if (bc.position == walls[w]) {
        codes[w] = bc.type == "periodic" ? FBC_PERIODIC
                 : bc.type == "Dirichlet" ? FBC_DIRICHLET
                 : bc.type == "Neumann"   ? FBC_NEUMANN
                                          : FBC_UNDEF;
        if (values) (*values)[w] = bc.val;
      }
    }
    if (bc.position == "hollow-cathode" && cathodePos) *cathodePos = bc.val;
  }
  return codes;
}

std::array<int, 4> Init::particleBCCodes() const {
  std::array<int, 4> codes{PBC_INVALID, PBC_INVALID, PBC_INVALID, PBC_INVALID};
  static const char* walls[4] = {"Xmin", "Xmax", "Ymin", "Ymax"};
  for (const auto& bc : particleBoundaries)
    for (int w = 0; w < 4; ++w)
      if (bc.position == walls[w])
        codes[w] = bc.type == "periodic" ? PBC_PERIODIC
                 : bc.type == "Delete"   ? PBC_DELETE
                 : bc.type == "Reflect"  ? PBC_REFLECT
                                         : PBC_INVALID;
  return codes;
}

int Init::loadGenType(const std::string& s) {
  if (s == "uniform-Gaussian") return 0;
  if (s == "Xsinusoidal-Gaussian") return 1;
  if (s == "Ysinusoidal-Gaussian") return 2;
  if (s == "quietStart") return 4;
  if (s == "Xgaussian-Gaussian") return 5;
  if (s == "Ygaussian-Gaussian") return 6;
  return -1;
}

int Init::sourceGenType(const std::string& s) {
  if (s == "uniformIonization") return 0;
  if (s == "XsinusoidalIonization") return 1;
  if (s == "YsinusoidalIonization") return 2;
  if (s == "hollow-cathode") return 3;
  if (s == "fluxMaxwellianAtXmin") return 7;
  return -1;
}

namespace {
std::string q(const std::string& s) {
  std::string o = "\"";
  for (char c : s) {
    if (c == '"' || c == '\\') o += '\\';
    o += c;
  }
  return o + "\"";
}
std::string num(double v) {
  std::ostringstream os;
  os << std::setprecision(17) << v;
  return os.str();
}
std::string vec(const std::vector<double>& v) {
  std::string o = "[";
  for (size_t i = 0; i < v.size(); ++i) o += (i ? "," : "") + num(v[i]);
  return o + "]";
}
}  // namespace

std::string Init::dump() const {
  std::ostringstream o;
  const auto& f = flagForEquation;
  const auto& t = paramForTimeIntegration;
  const auto& c = paramForComputing;
  const auto& fl = paramForField;
  o << "{\"flag\":{\"Particle\":" << f.Particle << ",\"EMField\":" << f.EMField << ",\"MCCollision\":" << f.MCCollision
    << "},\"time\":{\"Start\":" << t.Start << ",\"End\":" << t.End << ",\"TimeStep\":" << num(t.TimeStep)
    << ",\"LogOutput\":" << t.LogOutput << ",\"ParticleOutput\":" << t.ParticleOutput
    << ",\"FieldOutput\":" << t.FieldOutput << ",\"ProgressOutput\":" << t.ProgressOutput
    << ",\"ProjectName\":" << q(t.ProjectName) << ",\"RestartName\":" << q(t.RestartName) << "}"
    << ",\"comp\":{\"pNumMax\":" << c.pNumMax << ",\"threadGroupSize\":" << c.threadGroupSize
    << ",\"integrationChunkSize\":" << c.integrationChunkSize << ",\"aggrThreshold\":" << num(c.aggrThreshold)
    << ",\"chebDegree\":" << c.chebDegree << ",\"amgCycleType\":" << c.amgCycleType << ",\"maxiter\":" << c.maxiter
    << ",\"tolerance\":" << num(c.tolerance) << "}"
    << ",\"field\":{\"ngx\":" << fl.ngx << ",\"ngy\":" << fl.ngy << ",\"ngb\":" << fl.ngb << ",\"dx\":" << num(fl.dx)
    << ",\"dy\":" << num(fl.dy) << ",\"InitTypeE\":" << q(fl.InitTypeE) << ",\"ampE\":" << vec(fl.ampE)
    << ",\"InitTypeB\":" << q(fl.InitTypeB) << ",\"ampB\":" << vec(fl.ampB) << ",\"FilePathBx\":" << q(fl.FilePathBx)
    << ",\"FilePathBy\":" << q(fl.FilePathBy) << ",\"FilePathBz\":" << q(fl.FilePathBz)
    << ",\"weightOrder\":" << fl.weightOrder << ",\"BorisOrder\":" << fl.BorisOrder
    << ",\"checkCurDens\":" << fl.checkCurDens << ",\"diff_ngb\":" << fl.diff_ngb << "}";
  o << ",\"fieldBCs\":[";
  for (size_t i = 0; i < fieldBoundaries.size(); ++i)
    o << (i ? "," : "") << "{\"position\":" << q(fieldBoundaries[i].position) << ",\"type\":"
      << q(fieldBoundaries[i].type) << ",\"val\":" << num(fieldBoundaries[i].val) << "}";
  o << "],\"particles\":[";
  for (size_t i = 0; i < paramForParticle.size(); ++i) {
    const auto& p = paramForParticle[i];
    o << (i ? "," : "") << "{\"pName\":" << q(p.pName) << ",\"pNum\":" << p.pNum << ",\"q\":" << num(p.q)
      << ",\"m\":" << num(p.m) << ",\"w\":" << num(p.w) << ",\"genType\":" << q(p.genType)
      << ",\"genX\":" << vec(p.genX) << ",\"genY\":" << vec(p.genY) << ",\"genU\":" << vec(p.genU)
      << ",\"genT\":" << num(p.genT) << ",\"sinU\":" << vec(p.sinU) << "}";
  }
  o << "],\"sources\":[";
  for (size_t i = 0; i < particleSources.size(); ++i) {
    const auto& s = particleSources[i];
    o << (i ? "," : "") << "{\"pName\":" << q(s.pName) << ",\"genType\":" << q(s.genType) << ",\"src\":" << num(s.src)
      << ",\"genX\":" << vec(s.genX) << ",\"genY\":" << vec(s.genY) << ",\"genU\":" << vec(s.genU)
      << ",\"genT\":" << num(s.genT) << ",\"genU_ele\":" << vec(s.genU_ele) << ",\"genT_ele\":" << num(s.genT_ele)
      << "}";
  }
  o << "],\"particleBCs\":[";
  for (size_t i = 0; i < particleBoundaries.size(); ++i)
    o << (i ? "," : "") << "{\"position\":" << q(particleBoundaries[i].position) << ",\"type\":"
      << q(particleBoundaries[i].type) << "}";
  o << "]}";
  return o.str();
}

}  // namespace gample

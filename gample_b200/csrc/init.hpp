// init.hpp -- condition-file schema (mirror of gample's Init class).
//
// Same JSON keys, per-section defaults and derived quantities as
// src/Init.h:9-99 and src/Init.mm:27-394 of the reference, with std::string in
// place of NSString. Parse failures throw gample::ConfigError where the
// reference's parser returns nil.
#pragma once

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace gample {

struct ConfigError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// src/Constant.h:3-25 (CGS-Gaussian)
namespace phys {
constexpr double me = 9.10938188e-28;
constexpr double ec = 4.803204197e-10;
constexpr double c = 2.99792458e10;
constexpr double kb = 1.3806503e-16;
constexpr double evtoerg = 1.6021764262e-12;
constexpr double ergtoev = 1 / 1.6021764262e-12;
constexpr double eVtoK = 11604;
constexpr double VtosV = 1e8 / c;
constexpr double sVtoV = 1 / (1e8 / c);
constexpr double JtosJ = 1 / (10 / c * 1e4);
constexpr double TtoG = 1e4;
constexpr double PI = 3.141592653589793;
}  // namespace phys

struct FlagForEquation {  // src/Init.h:9-13
  int Particle = 0;
  int EMField = 0;
  int MCCollision = 0;
};

struct ParamForTimeIntegration {  // src/Init.h:15-25
  int Start = 0, End = 0;
  double TimeStep = 0;
  int LogOutput = 0, ParticleOutput = 0, FieldOutput = 0, ProgressOutput = 0;
  std::string ProjectName = "undefined", RestartName = "undefined";
};

struct ParamForComputing {  // src/Init.h:27-36
  uint32_t pNumMax = 0;
  int threadGroupSize = 256;
  int integrationChunkSize = 256;
  float aggrThreshold = 0.1f;
  int chebDegree = 5;
  int amgCycleType = 1;
  int maxiter = 200;
  float tolerance = 1e-7f;
  // Build additions (no reference key counterpart is required; both default
  // to the reference's behaviour).
  int depositMode = 0;  // "DepositMode": 0 = FP32 atomics, 1 = deterministic fixed point
  int sortInterval = 0; // "SortInterval": cell-sort period in cycles (0 = automatic)
  uint64_t masterSeed = 0;  // "MasterSeed": seed of the splitmix64 -> PCG32 streams (the reference fixes 0)
};

struct ParamForParticle {  // src/Init.h:38-52
  std::string pName;
  uint32_t pNum = 0;
  double q = 0, m = -1, w = 0;
  std::string genType;
  std::vector<double> genX, genY, genU;
  double genT = 0;  // K
  // build addition: amplitude (cm/s, per component) of a drift added to the
  // initial load's velocities with the profile sin(2 pi (x - Xmin) / Lx)
  std::vector<double> sinU;
};

struct BoundaryConditionForParticle {  // src/Init.h:54-57
  std::string position, type;
};

struct SourceForParticle {  // src/Init.h:59-69
  std::string pName, genType;
  double src = 0;
  std::vector<double> genX, genY, genU, genU_ele;
  double genT = 0, genT_ele = 0;
};

struct ParamForField {  // src/Init.h:71-93
  int ngx = 0, ngy = 0, ngb = 0;
  double dx = 0, dy = 0;
  std::string InitTypeE = "undefined", InitTypeB = "undefined";
  std::vector<double> ampE, ampB;
  std::string FilePathEx, FilePathEy, FilePathEz, FilePathBx, FilePathBy, FilePathBz;
  int weightOrder = 5, BorisOrder = 2, checkCurDens = 0;
  int diff_ngb = 0;
};

struct BoundaryConditionForField {  // src/Init.h:95-99
  std::string position, type;
  double val = 0;
};

enum FieldBC { FBC_PERIODIC = 0, FBC_DIRICHLET = 1, FBC_NEUMANN = 2, FBC_UNDEF = -1 };
enum ParticleBC { PBC_PERIODIC = 0, PBC_DELETE = 1, PBC_REFLECT = 2, PBC_INVALID = -1 };
enum Wall { XMIN = 0, XMAX = 1, YMIN = 2, YMAX = 3 };

class Init {
 public:
  FlagForEquation flagForEquation;
  ParamForTimeIntegration paramForTimeIntegration;
  ParamForComputing paramForComputing;
  std::vector<ParamForParticle> paramForParticle;
  std::vector<BoundaryConditionForParticle> particleBoundaries;
  std::vector<SourceForParticle> particleSources;
  ParamForField paramForField;
  std::vector<BoundaryConditionForField> fieldBoundaries;

  // src/Init.mm:27-301
  static Init parseInputFile(const std::string& path);
  static Init parseString(const std::string& json_text);
  // Canonical JSON of the parsed, defaults-merged structs (for tests and logs).
  std::string dump() const;

  // Derived codes used by the device code.
  std::array<int, 4> fieldBCCodes(std::array<double, 4>* values = nullptr, double* cathodePos = nullptr) const;
  std::array<int, 4> particleBCCodes() const;
  static int loadGenType(const std::string& s);    // src/Collision.mm:220-233
  static int sourceGenType(const std::string& s);  // src/Collision.mm:368-377 (+ build code 7)
};

}  // namespace gample

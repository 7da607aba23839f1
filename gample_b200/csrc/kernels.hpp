// kernels.hpp -- host-callable launchers of the sm_100a kernels.
//
// Data layout in HBM:
//  * particles: structure of arrays, one entry per particle slot:
//      cell  int32  packed (iy << 16) | ix of the containing cell in the
//                   reference's ghost-offset grid units; a negative value
//                   -f marks a particle flagged f (1..4 = left through Xmin,
//                   Xmax, Ymin, Ymax; 5 = invalid state) awaiting compaction
//      ox,oy float  offset inside the cell, in [0, 1)
//      vx,vy,vz float velocity in cm/s
//    i.e. x_ref = ix + ox reproduces the reference's grid-unit position
//    (src/Particle.mm:589-594) without its loss of precision far from 0.
//  * fields: the reference's staggered arrays with its extents and strides
//    (rho (nx+1)(ny+1), Ex (nx+2)(ny+1), Ey (nx+1)(ny+2), Bz (nx+2)(ny+2),
//    phi double (nx+3)(ny+3); src/EMField.mm:127-144).
//  * pitched copies of Ex and Ey for the push kernels' TMA staging: the same
//    rows with a row pitch rounded up to 4 floats (a tensor map's row stride
//    must be a multiple of 16 bytes), written with E.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace gample {
namespace kern {

// Field boundary codes (same values as gample::FieldBC).
constexpr int FBC_PERIODIC_C = 0, FBC_DIRICHLET_C = 1, FBC_NEUMANN_C = 2;

struct GridDims {
  int ngx, ngy, ngb;
  int nx, ny;  // ngx + 2 ngb, ngy + 2 ngb
};

struct ParticleArrays {
  int32_t* cell;
  float* ox;
  float* oy;
  float* vx;
  float* vy;
  float* vz;
};

// Per-species counters kept in device memory (written by the push and
// compaction kernels, read by the host only for diagnostics).
struct SpeciesCounters {
  uint32_t n;        // live particle count (pNum)
  uint32_t n_dead;   // particles flagged by the last push
  uint32_t wall[4];  // flagged through Xmin, Xmax, Ymin, Ymax
  uint32_t invalid;  // flagged for a non-finite or out-of-grid state
  uint32_t n_injected;
  uint32_t n_pulled; // removed by the last compaction (which consumes n_dead)
  uint32_t n_slow;   // pushed without a shared-memory window (chunk too spread out)
  uint32_t err;      // chunks whose field staging did not complete in time (staged by loads instead)
  uint32_t n_tma;    // chunks whose Ex / Ey tiles were staged by bulk tensor copies
  uint32_t n_tab;    // chunks that gathered through the per-cell tables (order 3)
  uint32_t n_priv;   // chunks that deposited into the 32 lane-private windows
  double ke;         // sum of 0.5 m v^2 w over particles still live (erg)
};

struct PushConsts {
  float constE, constB, constX, constY;  // src/Particle.mm:617-621
  int bc[4];                             // particle BC code per wall
  float scale;                           // deposit weight q w / (dx dy)
  float bz_uniform;                      // used when the Bz gather is skipped
  double ke_half_m, ke_w;                // 0.5 * m and w for the kinetic energy
  int no_tables;                         // 1: order 3 gathers from the staged windows, not the tables
};

// Per-species charge / current accumulators (reference extents). Fast mode:
// FP64 sums of the FP32 contributions w_x w_y q w / (dx dy) (times v for the
// currents). Deterministic mode: exact int64 sums of the weights quantised to
// 2^-40 (currents: of w_x w_y v / c). combine_* turns them into rho/jx/jy.
struct DepositTargets {
  double* f64_rho;
  double* f64_jx;
  double* f64_jy;
  long long* acc_rho;
  long long* acc_jx;
  long long* acc_jy;
};

struct FieldPtrs {
  const float* Ex;
  const float* Ey;
  const float* Bz;
};

// Tensor maps of the pitched Ex and Ey copies for the push kernels' field
// staging (cp.async.bulk.tensor.2d into shared memory, out-of-range elements
// filled with zero): one map per box size kFieldBoxW[b] x kFieldBoxH[b]
// (columns x rows), so that a chunk copies the smallest box covering its
// window. valid = 0: no maps, the kernels stage with per-thread loads.
constexpr int kFieldBoxes = 3;
constexpr int kFieldBoxW[kFieldBoxes] = {20, 24, 40};
constexpr int kFieldBoxH[kFieldBoxes] = {8, 16, 40};
struct FieldMaps {
  CUtensorMap ex[kFieldBoxes];
  CUtensorMap ey[kFieldBoxes];
  int valid;
};
// Row pitch (floats) of the pitched copies.
inline int field_pitch(const GridDims& g) { return (g.nx + 2 + 3) & ~3; }
// Encode the maps for pitched copies Exp ((ny+1) rows) and Eyp ((ny+2) rows).
// Returns false (maps->valid = 0) when the driver offers no tensor maps.
bool make_field_maps(const float* Exp, const float* Eyp, GridDims g, FieldMaps* maps);
// Ex, Ey -> their pitched copies.
void pitch_fields(const float* Ex, const float* Ey, GridDims g, float* Exp, float* Eyp, cudaStream_t s);

// ------------------------------------------------------------- particles
// Particles per thread of the push's CTAs (256 threads): the atomic-mode
// push in a uniform Bz also runs with half as many (1024-particle chunks),
// chunk_per = kPushChunkPer / 2, for an autotuner to pick per species.
constexpr int kPushChunkPer = 8;
// Gather + Boris + move + boundary conditions for particles [0, n) where n
// is read from counters->n; optionally deposits the new positions (live
// particles only). Writes the dead bitmap (bit k = particle k flagged) and
// the flag counters, and accumulates the kinetic energy of live particles.
// Each CTA takes a chunk of consecutive particles, stages the field window
// covering their stencils in shared memory and accumulates the deposit in a
// shared-memory window flushed with one global atomic per touched node; the
// chunks are compact in space because the particles are cell-sorted.
void push(int order, int boris_order, bool deposit, bool det, bool current, bool bz_uniform, GridDims g,
          ParticleArrays p, FieldPtrs f, PushConsts c, DepositTargets d, SpeciesCounters* counters,
          uint32_t* dead_bits, uint32_t n_bound, cudaStream_t s, const FieldMaps* maps = nullptr,
          int chunk_per = kPushChunkPer);

// Deposit particles [0, counters->n) (src/Particle.mm:281-389), or with
// injected_only the particles appended since the last push,
// [n - n_injected, n).
void deposit(int order, bool det, bool current, GridDims g, ParticleArrays p, float scale, DepositTargets d,
             const SpeciesCounters* counters, uint32_t n_bound, bool injected_only, cudaStream_t s);

// Counting sort of particles [0, counters->n) by cell, in tile-major order
// (8 x 8-cell tiles), from src into dst. Order inside a cell is unspecified.
// scratch holds sort_scratch_words(g) words.
size_t sort_key_count(GridDims g);
size_t sort_scratch_words(GridDims g);
void sort_by_cell(GridDims g, ParticleArrays src, ParticleArrays dst, const SpeciesCounters* counters,
                  uint32_t* scratch, uint32_t n_bound, cudaStream_t s);
// The same order for particles in random order, in place in p: whole records
// are scattered into spare (arrays of capacity words each) and converted
// back. extra is a second idle buffer the call may use (extra_capacity words
// per array, 0 for none); with it the records are sector-sized. Returns false
// (nothing launched) when the records do not fit.
bool sort_by_cell_staged(GridDims g, ParticleArrays p, ParticleArrays spare, uint32_t capacity,
                         ParticleArrays extra, uint32_t extra_capacity, const SpeciesCounters* counters,
                         uint32_t* scratch, uint32_t n_bound, cudaStream_t s);

// Remove flagged particles, filling each hole (ascending) with the last
// live particle (descending) -- the permutation of src/Particle.mm:893-966.
// Updates counters->n. scratch must hold compact_scratch_words(n_bound).
size_t compact_scratch_words(uint32_t n_bound);
void compact(ParticleArrays p, SpeciesCounters* counters, const uint32_t* dead_bits, uint32_t* scratch,
             uint32_t n_bound, cudaStream_t s);

// Reference 24-byte records <-> device SoA.
struct ParticleStateAoS {
  float x, y, vx, vy, vz;
  int piflag;
};
void aos_to_soa(const ParticleStateAoS* in, uint32_t n, ParticleArrays p, int nx, int ny, cudaStream_t s);
void soa_to_aos(ParticleArrays p, uint32_t n, ParticleStateAoS* out, cudaStream_t s);

// ------------------------------------------------------------- generation
struct RNGState {
  unsigned long long state, inc;
};
// Seed slots [from, to) as the reference's host loop does
// (src/Collision.mm:283-294): slot i takes the (2i+1)-th and (2i+2)-th
// outputs of splitmix64 started at master_seed.
void seed_rng(RNGState* states, uint64_t master_seed, uint32_t from, uint32_t to, cudaStream_t s);

struct GenParams {  // src/Collision.h:22-38
  float Xmin, Xmax, Ymin, Ymax;
  float ele_genU[3];
  float ele_vth;
  float ion_genU[3];
  float ion_vth;
  float dx, dy, ngb;
  // build addition (initial load only): drift amplitudes with the profile
  // sin(2 pi (x - Xmin) / Lx); sin_on = 0 leaves the reference's velocities
  float ele_sinU[3], ion_sinU[3];
  int sin_on;
};
// Kernel artificialIonization (src/Collision.mm:63-174): addn particles
// (electron, and a colocated ion unless genType == 3) appended after the
// current counts. Device counts are advanced by addn.
void generate(int gen_type, uint32_t addn, GenParams prm, RNGState* states, ParticleArrays ele,
              SpeciesCounters* ele_cnt, ParticleArrays* ion, SpeciesCounters* ion_cnt, cudaStream_t s);
// Flux-Maxwellian re-injection at Xmin of `addn` particles of one species
// (build addition; no reference counterpart).
struct RefluxParams {
  float Xmin, Ymin, Ymax, vth, u0, u1, u2, dt, dx, dy, ngb;
};
void reflux(uint32_t addn, RefluxParams prm, RNGState* states, ParticleArrays p, SpeciesCounters* cnt,
            cudaStream_t s);

// ------------------------------------------------------------- fields
void zero_f32(float* p, size_t n, cudaStream_t s);
// rho = sum_s double(acc_s) * (scale_s * 2^-40), rounded to float
// (species in order); same for the currents with an extra factor c.
void combine_fixed_point(const long long* const* acc, const float* scales, int nspecies, size_t n, double extra,
                         float* out, cudaStream_t s);
// rho = sum_s acc_s (FP64, species in order), rounded to float.
void combine_f64(const double* const* acc, int nspecies, size_t n, float* out, cudaStream_t s);
// Ghost-charge folding (src/EMField.mm:751-850).
void fold_ghosts(float* rho, GridDims g, const int fbc[4], cudaStream_t s);

struct PoissonLayout {
  int nkx, nky, ikmin, jkmin;  // src/EMField.mm:246-271
  int fbc[4];
  double Cx, Cy, Cd;
  double phiXmin, phiXmax, phiYmin, phiYmax;  // statV
  bool periodic_x, periodic_y;
};
// b = rhs_BC - 4 pi rho (src/EMField.mm:852-861) in FP64; accumulates
// sum(b) and sum(b^2) into sums[0..1].
void build_rhs(const float* rho, GridDims g, PoissonLayout L, double* b, double* sums, cudaStream_t s);
void subtract_mean(double* v, int n, const double* sum, cudaStream_t s);
// sums[0..1] = sum(v), sum(v^2)
void vec_sums(const double* v, int n, double* sums, cudaStream_t s);

// phi (nx+3)(ny+3) from the solution vector (src/EMField.mm:873-1077).
void phi_fill(const double* sol, GridDims g, PoissonLayout L, float dx, double cathode_pos, double* cathode_mean,
              double* phi, cudaStream_t s);
// Ex, Ey = -grad phi (src/EMField.mm:1080-1094) and the energy / Joule
// sums (src/EMField.mm:1096-1111) into sums[0] (sum E^2), sums[1] (sum E.j).
// Exp, Eyp (optional): the pitched copies, written alongside.
void gradient_energy(const double* phi, GridDims g, float dx, float dy, float* Ex, float* Ey, const float* jx,
                     const float* jy, double* sums, cudaStream_t s, float* Exp = nullptr, float* Eyp = nullptr);
// Probe values for the timeseries CSV (src/EMField.mm:1130-1134).
void probe(const double* phi, const float* Ex, const float* Ey, GridDims g, double* out3, cudaStream_t s);

// ------------------------------------------------------------- Darwin
// Vector-potential grid of the Darwin solves (src/EMField.mm:484-492).
struct DarwinGeom {
  int nkx, nky, ngb, nx, ny;
  bool perx, pery;  // otherwise Neumann
  float dx, dy;
};
// rhs = div J with the Neumann boundary terms (src/EMField.mm:1150-1184)
void darwin_div_rhs(const float* jx, const float* jy, DarwinGeom G, double* rhs, cudaStream_t s);
// rhs = -(4 pi / c)(J_a - d_a psi), dir 0: x, 1: y (src/EMField.mm:1201-1275)
void darwin_a_rhs(const float* ja, const double* psi, DarwinGeom G, int dir, double* rhs, cudaStream_t s);
// v -= weighted mean (weights 1/2 at Neumann ends); scratch2: 2 doubles
void darwin_weighted_project(double* v, DarwinGeom G, double* scratch2, cudaStream_t s);
// delEx, delEy, delBz from A and the previous A (src/EMField.mm:1277-1297)
void darwin_fields(const double* Ax, const double* Ay, const double* lastAx, const double* lastAy, DarwinGeom G,
                   double cdt, float* delEx, float* delEy, float* delBz, cudaStream_t s);

// Velocity moments of particles [0, counters->n) (src/Moment.mm:33-135,
// 287-316): out holds 10 arrays of (nx+1)(ny+1) floats (n, ux, uy, uz, Pxx,
// Pxy, Pxz, Pyy, Pyz, Pzz); acc is FP64 scratch of the same size.
void moments(int order, GridDims g, ParticleArrays p, const SpeciesCounters* counters, uint32_t n_bound, float scale,
             float mass, double* acc, float* out, cudaStream_t s);

// Charge density of one species from the reference's 24-byte records in
// device memory into rho ((nx+1)(ny+1) floats), with no allocation: the int64
// accumulator is a file-scope device array of noalloc_max_nodes() entries.
// Throws std::length_error for a larger grid. Calls must not overlap in time.
size_t noalloc_max_nodes();
void deposit_charge_noalloc(int order, int ngx, int ngy, const ParticleStateAoS* particles, uint32_t n, float scale,
                            float* rho, cudaStream_t s);

// ------------------------------------------------------------- utilities
void fill_f32(float* p, size_t n, float v, cudaStream_t s);
void fill_f64(double* p, size_t n, double v, cudaStream_t s);

}  // namespace kern
}  // namespace gample

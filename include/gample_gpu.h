/* gample_gpu.h -- C ABI of the B200-native gample particle-in-cell step.
 *
 * The reference (tnaoki0630/gample) has no plugin API: its boundary is the
 * Objective-C method surface of the Init, Particle, EMField and Collision
 * classes plus the JSON condition schema and the timeseries CSV / XML log.
 * Each entry point below replaces one of those methods (cited as file:line
 * inside the gample repository). Plain pointers and sizes only; every call
 * returns a gp_status (0 = success) and never aborts. gp_last_error() gives
 * the message of the last failure on the calling thread.
 *
 * Threading: a gp_sim owns one CUDA stream on the current device; handles are
 * not thread-safe. Device work is asynchronous; calls that return host values
 * synchronise the stream.
 */
#ifndef GAMPLE_GPU_H
#define GAMPLE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int gp_status;
#define GP_OK 0
#define GP_ERR_ARGUMENT 1     /* bad handle, index or size */
#define GP_ERR_CONFIG 2       /* condition file rejected (Init.mm returns nil) */
#define GP_ERR_CUDA 3         /* CUDA runtime failure (message in gp_last_error) */
#define GP_ERR_CAPACITY 4     /* pNum would exceed MaximumParticleNumber */
#define GP_ERR_INTERNAL 5

typedef struct gp_init gp_init; /* parsed condition (src/Init.h:101-118) */
typedef struct gp_sim gp_sim;   /* Particle[], EMField, Collision, XmlLogger of one run */
typedef struct gp_nn gp_nn;     /* learned warm-start network (build addition) */
typedef struct gp_ensemble gp_ensemble; /* independent runs advanced together (build addition) */

/* Particle record of the reference (src/Particle.h:14-21): x, y in grid units
 * offset by ngb, velocities in cm/s, piflag 0 = live, 1..4 = left through
 * Xmin, Xmax, Ymin, Ymax (5 = invalid state, build addition). */
typedef struct {
  float x, y, vx, vy, vz;
  int32_t piflag;
} gp_particle_state;

typedef struct {
  int32_t iterations;        /* V-cycles (the reference logs AMGCL CG iterations) */
  double error;              /* relative residual ||b - A phi|| / ||b|| */
  double mean_cathode;       /* V */
  double electric_energy;    /* erg/m as logged by the reference (no 1/(4 pi)) */
  double electric_energy_increment;
  double joule_heating;      /* erg/m */
  double probe[3];           /* phi1 (statV), Ex1, Ey1 (statV/cm) of the CSV */
  double field_energy_cgs;   /* sum E^2/(8 pi) dx dy, erg/cm */
} gp_solve_stats;

typedef struct {
  uint32_t particle_number;  /* pNum after removal */
  uint32_t pulled;           /* particles removed */
  int32_t pinum[4];          /* outflow per wall in units of the charge sign */
  uint32_t invalid;          /* removed for a non-finite / off-grid state */
  double kinetic_energy;     /* erg */
  double kinetic_energy_increment;
} gp_flow_stats;

/* Field selectors for gp_field_download / gp_field_upload (reference extents,
 * row-major with the reference's strides, src/EMField.mm:133-144). */
#define GP_FIELD_RHO 0 /* float (nx+1)(ny+1) */
#define GP_FIELD_EX 1  /* float (nx+2)(ny+1) */
#define GP_FIELD_EY 2  /* float (nx+1)(ny+2) */
#define GP_FIELD_BZ 3  /* float (nx+2)(ny+2) */
#define GP_FIELD_JX 4  /* float (nx+2)(ny+1) */
#define GP_FIELD_JY 5  /* float (nx+1)(ny+2) */
#define GP_FIELD_PHI 6 /* double (nx+3)(ny+3) */
#define GP_FIELD_SOL 7 /* double (nkx+1)(nky+1): Poisson solution vector (src/EMField.mm:97, 410) */
#define GP_FIELD_DEL_EX 8  /* float (nx+2)(ny+1): Darwin correction (src/EMField.h, delExBuffer) */
#define GP_FIELD_DEL_EY 9  /* float (nx+1)(ny+2) */
#define GP_FIELD_DEL_BZ 10 /* float (nx+2)(ny+2) */
#define GP_FIELD_PSI 11    /* double (nkx_vec+1)(nky_vec+1): longitudinal potential (src/EMField.mm:1193-1199) */
#define GP_FIELD_AX 12     /* double, same grid: vector potential Ax (src/EMField.mm:1232-1237) */
#define GP_FIELD_AY 13     /* double, same grid: Ay (src/EMField.mm:1270-1275) */

/* ---- Init: -[Init parseInputFile:] (src/Init.mm:27-301) ---- */
gp_status gp_init_parse_file(const char* path, gp_init** out);
gp_status gp_init_parse_json(const char* json_text, gp_init** out);
/* Canonical JSON of the parsed, defaults-merged condition; *len receives the
 * full length (including the terminating NUL) even if cap is too small. */
gp_status gp_init_dump(const gp_init* init, char* buf, size_t cap, size_t* len);
void gp_init_free(gp_init* init);

/* ---- Run objects: src/main.mm:75-122 ----
 * Builds Particle objects (src/Particle.mm:407-611), EMField
 * (src/EMField.mm:105-656) and Collision (src/Collision.mm:189-462, which
 * loads the initial particles). log_name: "<Project>_<tag>" prefix of the
 * XML log and timeseries CSV, or NULL for none. flags: GP_SIM_* below. */
#define GP_SIM_REFERENCE_ORDER 1 /* separate deposit pass (no push-fused deposit) */
gp_status gp_sim_create(const gp_init* init, const char* log_name, int flags, gp_sim** out);
void gp_sim_free(gp_sim* sim);
/* Initial deposit and field solve: src/main.mm:136-141. */
gp_status gp_sim_initialize(gp_sim* sim);
/* The initial load again from master seed `seed` (ParamForComputing
 * MasterSeed; the reference fixes 0) with the cycle counter back at Start;
 * gp_sim_initialize follows. Fields, solver state and any warm-start network
 * are kept. Build addition, no reference counterpart. */
gp_status gp_sim_reload(gp_sim* sim, uint64_t seed);
/* ncycles cycles of the time loop: src/main.mm:155-253. */
gp_status gp_sim_run(gp_sim* sim, int ncycles);
gp_status gp_sim_cycle_number(const gp_sim* sim, int* cycle, double* time);
gp_status gp_sim_last_solve(const gp_sim* sim, gp_solve_stats* out);
gp_status gp_sim_last_flow(const gp_sim* sim, int species, gp_flow_stats* out);
gp_status gp_sim_synchronize(gp_sim* sim);
/* Device-side timing of whole cycles on the run's stream (CUDA events). */
gp_status gp_sim_time_cycles(gp_sim* sim, int ncycles, float* ms);
/* Per-phase device time accumulated while profiling is on (ms):
 * [0] deposit [1] field solve [2] push [3] reduce [4] sources [5] tile sort. */
gp_status gp_sim_set_profiling(gp_sim* sim, int on);
gp_status gp_sim_phase_times(gp_sim* sim, double out[6]);

/* ---- EMField ---- */
gp_status gp_field_dims(const gp_sim* sim, int* ngx, int* ngy, int* ngb, int* nkx, int* nky);
/* -[EMField resetChargeDensity] (src/EMField.mm:1363-1378) */
gp_status gp_field_reset_charge(gp_sim* sim);
/* -[EMField solvePoisson:withLogger:] (src/EMField.mm:745-1136) */
gp_status gp_field_solve_poisson(gp_sim* sim, double dt, gp_solve_stats* out);
/* Buffer accessors (src/EMField.h:22-37, EMField.mm:1396-1424) */
gp_status gp_field_download(gp_sim* sim, int which, void* host, size_t bytes);
gp_status gp_field_upload(gp_sim* sim, int which, const void* host, size_t bytes);
/* -[EMField solveVectorPotential:withLogger:] (src/EMField.mm:1138-1361):
 * Darwin model (FlagForEquation.EMField = 2); iterations / relative
 * residuals of the decomposition, Ax and Ay solves (either may be NULL). */
gp_status gp_field_solve_darwin(gp_sim* sim, double dt, int iterations[3], double errors[3]);
/* Set the Poisson tolerance / iteration cap (ToleranceForPoisson, MaxiterForPoisson). */
gp_status gp_field_set_solver(gp_sim* sim, double tol, int maxiter);

/* ---- Particle (species index s) ---- */
/* -[Particle update:withEMField:withMom:withLogger:] (src/Particle.mm:615-891);
 * fused_deposit != 0 also deposits the new positions into the field's charge. */
gp_status gp_particle_update(gp_sim* sim, int s, double dt, int fused_deposit);
/* -[Particle reduce:] (src/Particle.mm:893-1002) */
gp_status gp_particle_reduce(gp_sim* sim, int s, gp_flow_stats* out);
/* -[Particle integrateChargeDensity:withMoment:withLogger:] (src/Particle.mm:1004-1130) */
gp_status gp_particle_integrate_charge(gp_sim* sim, int s);
/* pNum (src/Particle.mm:451, paramsBuffer) */
gp_status gp_particle_count(gp_sim* sim, int s, uint32_t* n);
/* Sort species s by cell now (build addition; the time loop sorts by
 * itself). path: 0 as the loop would (staged records for particles in
 * random order, the block-local re-sort otherwise), 1 the block-local
 * re-sort of nearly sorted particles, 2 the staged record scatter. */
gp_status gp_particle_sort(gp_sim* sim, int s, int path);
/* Diagnostics of the last push (build addition): out[0] particles pushed
 * without a shared-memory window, out[1] chunks whose Ex / Ey tiles were
 * staged by bulk tensor copies, out[2] staging waits that timed out, out[3]
 * chunks that gathered through the per-cell tables, out[4] chunks that
 * deposited into lane-private windows, out[5] particles per chunk (2048 or
 * 1024), out[6] 1 if order 3 could use the gather tables (out[1], out[3] to
 * out[6]: the atomic mode's push in a uniform Bz). */
gp_status gp_particle_push_stats(gp_sim* sim, int s, uint32_t out[7]);
/* Variant of species s's atomic-mode push in a uniform Bz (build
 * addition): particles per chunk 2048 or 1024 and, for order 3, gather
 * tables on (tables != 0) or off fix it; particles = 0 lets the autotuner
 * pick (the default: the pushes after the first sort time each variant
 * twice, in mirrored order, and keep the fastest). */
gp_status gp_particle_set_push_variant(gp_sim* sim, int s, int particles, int tables);
/* particleBuffer contents as 24-byte records (src/Particle.h:69-78) */
gp_status gp_particle_download(gp_sim* sim, int s, gp_particle_state* host, uint32_t capacity, uint32_t* n);
gp_status gp_particle_upload(gp_sim* sim, int s, const gp_particle_state* host, uint32_t n);
/* Device representation: packed cell ((iy << 16) | ix, negative = -piflag)
 * and in-cell offsets; any pointer may be NULL. */
gp_status gp_particle_download_raw(gp_sim* sim, int s, int32_t* cell, float* ox, float* oy, float* vx, float* vy,
                                   float* vz, uint32_t capacity, uint32_t* n);

/* ---- Moment ---- */
/* -[Moment integrateMoments:withEMField:withLogger:] (src/Moment.mm:206-316)
 * for species s; the ten arrays stay on the device. */
gp_status gp_moments_integrate(gp_sim* sim, int s);
/* One of the ten moment arrays of the last integration, (nx+1)(ny+1) floats:
 * 0 n, 1 ux, 2 uy, 3 uz, 4 Pxx, 5 Pxy, 6 Pxz, 7 Pyy, 8 Pyz, 9 Pzz
 * (src/Moment.h:43-53; CGS units, before the 0.1 Pa scaling of the files). */
gp_status gp_moments_download(gp_sim* sim, int which, float* host, size_t bytes);

/* ---- binary outputs and restart (src/FileIO.mm), under ./bin ---- */
/* outputField (src/FileIO.mm:41-136): bin/<Project>_EMField_%08d.bin */
gp_status gp_sim_output_field(gp_sim* sim, int cycle);
/* integrateMoments + outputMoments (src/FileIO.mm:138-226) of species s */
gp_status gp_sim_output_moments(gp_sim* sim, int s, int cycle);
/* saveProgress (src/FileIO.mm:250-293): bin/<Project>_ProgressData_<name>_%08d.bin */
gp_status gp_sim_save_progress(gp_sim* sim, int cycle);
/* loadProgress (src/FileIO.mm:295-352): reads bin/<RestartName>_ProgressData_...,
 * shifting positions by PtclPosOffset */
gp_status gp_sim_load_progress(gp_sim* sim, int cycle);

/* ---- Collision ---- */
/* -[Collision artificialIonization:withParticles:withLogger:] (src/Collision.mm:464-566) */
gp_status gp_collision_artificial_ionization(gp_sim* sim, double dt, int* addn);
/* -[Collision hollowCathode:withParticles:withLogger:] (src/Collision.mm:568-678) */
gp_status gp_collision_hollow_cathode(gp_sim* sim, double dt, int* addn);
/* Flux-Maxwellian re-injection at Xmin (GenerateType fluxMaxwellianAtXmin);
 * build addition, no reference counterpart. */
gp_status gp_collision_flux_reinjection(gp_sim* sim, double dt, int* addn);

/* ---- allocation-free deposit (no reference counterpart) ----
 * Charge density of one species, for callers that own all device memory and
 * cannot let the library allocate (a fixed device-memory budget or their own
 * pool, or a loop that must not pay cudaMalloc/cudaFree's implicit device
 * synchronisation). No handle is needed and nothing is allocated.
 *   particles  device pointer to n reference records (x, y in grid units
 *              offset by ngb = order / 2, as src/Particle.mm:589-594 stores
 *              them); records with piflag != 0 are skipped
 *   scale      q * w / (dx * dy) of the species (src/Particle.mm:540)
 *   rho        device pointer to (nx+1)(ny+1) floats, nx = ngx + 2 ngb,
 *              ny = ngy + 2 ngb; overwritten (no ghost folding)
 *   stream     cudaStream_t to run on (NULL = default stream)
 * Arithmetic: the deterministic deposit of the handle API (weights quantised
 * to 2^-40, exact int64 sums, one rounding to float), so the result is
 * bit-identical to gp_particle_integrate_charge of the same species with
 * DepositMode 1 in an otherwise empty field.
 * Limit: (nx+1)(ny+1) <= 1048576 nodes (8 MiB of scratch held in a static
 * device array); a larger grid returns GP_ERR_CAPACITY. The scratch is
 * cleared by every call, so nothing needs to start at zero. The scratch is
 * shared by all calls on a device: calls that overlap in time (other streams
 * or host threads without ordering) race, so serialise them. Every call looks
 * up the scratch address in the current context (cudaGetSymbolAddress, no
 * allocation); the first call on a device may load the library's device code
 * and should come before any stream capture on that device. Asynchronous:
 * errors of the kernels themselves surface at the next synchronisation. */
gp_status gp_deposit_charge_noalloc(int weighting_order, int ngx, int ngy, const gp_particle_state* particles,
                                    uint32_t n, float scale, float* rho, void* stream);

/* ---- learned warm start of the Poisson solve (build addition; no
 * reference counterpart): a 4-level convolutional encoder-decoder (3x3,
 * 32/64/128/256 channels, BF16 on the tensor cores). Host buffers: in is
 * [h][w][2] (normalised rhs, previous phi), out/target [h][w]. ---- */
/* Attach the network to a run's Poisson solve. mode bits: 1 start the
 * multigrid from previous phi + network correction, 2 train after each solve
 * on (rhs, previous phi) -> (phi - previous phi), 4 also time a solve from the
 * plain warm start, 8 keep each solve's sample in the sample bank, 16 (when
 * the network is first attached) the residual formulation: a one-channel
 * network (widths 16/32/64/64) maps the residual b - A (previous phi),
 * divided by its RMS, to a correction of previous phi and learns from the
 * mean square of the residual that correction leaves (Dirichlet and periodic
 * field boundaries); the multigrid always reaches ToleranceForPoisson. */
gp_status gp_field_learned(gp_sim* sim, int mode, float lr, uint64_t seed);
/* Sample bank of the residual formulation: room for `capacity` samples on
 * the device, filled by the solves while mode bit 8 is set. */
gp_status gp_field_learned_bank(gp_sim* sim, int capacity);
/* Offline training on the bank: `steps` Adam steps (learning rate lr) on
 * samples drawn at random (seed); out[0], out[1]: mean loss of the first and
 * of the last ten steps, out[2]: samples in the bank. */
gp_status gp_field_learned_train(gp_sim* sim, int steps, float lr, uint64_t seed, double out[3]);
/* last solve: loss, V-cycles (learned, plain), ms (learned incl. network,
 * plain, network alone), starting relative residual (learned, plain),
 * training steps so far */
gp_status gp_field_learned_stats(gp_sim* sim, double out[9]);
gp_status gp_nn_create(int h, int w, uint64_t seed, gp_nn** out);
void gp_nn_free(gp_nn* nn);
gp_status gp_nn_forward(gp_nn* nn, const float* in, float* out);
/* forward + backward (mean-squared error), gradients kept for gp_nn_param */
gp_status gp_nn_loss_grad(gp_nn* nn, const float* in, const float* target, float* loss);
/* one Adam step (learning rate lr) */
gp_status gp_nn_train_step(gp_nn* nn, const float* in, const float* target, float lr, float* loss);
gp_status gp_nn_layer_info(gp_nn* nn, int layer, int* cin, int* cout, int* kpad);
/* which: 0 weights [cout][kpad], 1 bias [cout], 2 weight gradient, 3 bias
 * gradient (FP32); set != 0 writes 0/1 */
gp_status gp_nn_param(gp_nn* nn, int layer, int which, float* host, size_t count, int set);

/* ---- ensemble of independent runs (build addition; no reference
 * counterpart): each member is a full run with its own CUDA stream, driven by
 * a pool of host threads so that members overlap on the GPU; results equal
 * each run alone. ---- */
gp_status gp_ensemble_create(const gp_init* const* inits, int n, int threads, gp_ensemble** out);
void gp_ensemble_free(gp_ensemble* e);
gp_status gp_ensemble_initialize(gp_ensemble* e);
gp_status gp_ensemble_run(gp_ensemble* e, int ncycles);
/* gp_ensemble_run timed on the device (ms): from the earliest member's first
 * kernel to the latest member's last, by CUDA events on the member streams */
gp_status gp_ensemble_time_cycles(gp_ensemble* e, int ncycles, float* ms);
/* a view of member i for the gp_sim_* / gp_particle_* / gp_field_* calls
 * (owned by the ensemble; gp_sim_free on it does nothing) */
gp_status gp_ensemble_member(gp_ensemble* e, int i, gp_sim** out);

/* ---- misc ---- */
const char* gp_last_error(void);
const char* gp_version(void);
/* Number of CUDA devices visible (0 without a GPU); never fails. */
int gp_device_count(void);
/* Kernels this library has launched since it was loaded (all runs). */
unsigned long long gp_kernel_launches(void);
/* Device memory of closed simulations stays cached in the process (the
   current device's stream-ordered pool) so that the next simulation of a
   similar size starts without the driver mapping gigabytes again, and its
   page-locked read-back buffers are kept for reuse; this returns the cached
   memory of the current device to the driver and frees the kept page-locked
   buffers. No counterpart in the reference (it allocates Metal buffers per
   run). */
gp_status gp_release_cached_memory(void);

#ifdef __cplusplus
}
#endif
#endif /* GAMPLE_GPU_H */

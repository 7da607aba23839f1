/* oracle.h -- C API of the CPU oracle (test infrastructure only).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load liboracle.so. It restates gample's particle-in-cell step on the CPU
 * (see oracle_core.hpp for the file:line map) so that the CUDA product can be
 * checked against it.
 */
#ifndef GAMPLE_ORACLE_H
#define GAMPLE_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define OR_MAX_SPECIES 4
#define OR_MAX_SOURCES 4

typedef struct {
  char name[32];
  unsigned int pnum; /* initial particle number (Init.mm:182-190) */
  double q, m, w;    /* statC, g, weight (Init.mm:191-201) */
  int gen_type;      /* Collision.mm:220-233 code of GenerateType, -1 unknown */
  double genX[2], genY[2], genU[3];
  double genT; /* K */
} or_species;

typedef struct {
  char pname[32];
  int gen_type; /* 0 uniformIonization 1 Xsinusoidal 2 Ysinusoidal 3 hollow-cathode 7 fluxMaxwellianAtXmin */
  double src;   /* Init.mm:249-264 */
  double genX[2], genY[2], genU[3], genU_ele[3];
  double genT, genT_ele; /* K */
} or_source;

typedef struct {
  int n_species, em_field, mc_collision;
  int start, end;
  double dt;
  int log_output, particle_output, field_output, progress_output;
  unsigned int pnum_max;
  int maxiter;
  double tol;
  int ngx, ngy, ngb;
  double dx, dy;
  double ampE[3], ampB[3];
  int initE_uniform, initB_uniform;
  int weight_order, boris_order, cur_dens;
  int fbc[4]; /* Xmin Xmax Ymin Ymax: 0 periodic 1 Dirichlet 2 Neumann -1 undefined */
  double fbc_val[4];
  double cathode_pos; /* <0: none */
  int pbc[4];         /* 0 periodic 1 Delete 2 Reflect */
  or_species sp[OR_MAX_SPECIES];
  int n_sources;
  or_source src[OR_MAX_SOURCES];
  uint64_t master_seed; /* build addition: seed of the RNG streams (the reference fixes 0) */
} or_config;

typedef struct {
  int iterations;
  double error;        /* relative residual */
  double mean_cathode; /* statV */
  double energy;       /* erg/m, src/EMField.mm:1112 (no 1/4pi) */
  double joule;
  double probe[3]; /* phi1, Ex1, Ey1 at the CSV probe node */
} or_solve_stats;

typedef struct {
  int pinum[4];
  int pulled;
  unsigned int pnum;
  double ke; /* erg */
} or_flow_stats;

void* or_sim_create(const or_config* cfg, int real64);
void or_sim_free(void* h);
int or_sim_load_initial(void* h);  /* Collision init (Collision.mm:189-336) */
void or_sim_reset_charge(void* h); /* EMField.mm:1363-1378 */
void or_sim_deposit(void* h, int s);
void or_sim_solve_poisson(void* h, double dt, double tol_override, or_solve_stats* st);
void or_sim_push(void* h, int s, double dt);
void or_sim_reduce(void* h, int s, int faithful, or_flow_stats* fs);
int or_sim_ionize(void* h, double dt, int* addn);
int or_sim_hollow_cathode(void* h, double dt, int* addn);
int or_sim_reflux(void* h, double dt, int* addn);
/* One main-loop cycle (main.mm:154-254) without file output; the CSV fields
 * of the cycle are returned through st. */
int or_sim_cycle(void* h, int cycle, int faithful_reduce, or_solve_stats* st, or_flow_stats* fs /* [n_species] */);

unsigned int or_sim_pnum(void* h, int s);
void or_sim_set_pnum(void* h, int s, unsigned int n);
/* Particle arrays in the reference's grid units (x, y) and cm/s. Values are
 * converted to/from the sim's real type. */
void or_sim_get_particles(void* h, int s, double* x, double* y, double* vx, double* vy, double* vz, int* piflag);
void or_sim_set_particles(void* h, int s, unsigned int n, const double* x, const double* y, const double* vx,
                          const double* vy, const double* vz, const int* piflag);
void or_sim_get_particles_f32(void* h, int s, float* x, float* y, float* vx, float* vy, float* vz, int* piflag);
void or_sim_set_particles_f32(void* h, int s, unsigned int n, const float* x, const float* y, const float* vx,
                              const float* vy, const float* vz, const int* piflag);
/* which: 0 rho 1 Ex 2 Ey 3 Bz 4 jx 5 jy (reference extents) ; 6 phi (double) */
void or_sim_get_field(void* h, int which, double* out);
void or_sim_set_field(void* h, int which, const double* in);
void or_sim_species_consts(void* h, int s, float* constE, float* constB, float* constX, float* constY,
                           float* scale);
int or_sim_poisson_size(void* h);
/* Relative residual of a given solution vector against the oracle's CSR
 * system built from the sim's current rho. */
double or_sim_poisson_residual(void* h, const double* sol);
void or_sim_get_poisson_solution(void* h, double* sol);
/* velocity moments of species sp, 10 x n_rho floats (src/Moment.mm); build != 0:
   Horner weights and FP64 sums (the GPU build's summation) */
void or_sim_moments(void* h, int sp, int build, float* out);
/* Darwin model (src/EMField.mm:1138-1361) from given jx, jy (reference extents) */
void or_darwin(int ngx, int ngy, int ngb, int perx, int pery, float dx, float dy, double dt, const float* jx,
               const float* jy, double* lastAx, double* lastAy, double* psi, double* Ax, double* Ay, float* delEx,
               float* delEy, float* delBz);

/* Deterministic-mode deposit of the build restated on the CPU: positions as
 * integer cell (ix, iy) plus float offsets, weights by the build's Horner
 * B-splines, contributions quantised to 2^-40 and summed in int64 per node.
 * acc has (nx+1)(ny+1) entries (rho layout). */
void or_det_deposit_rho(int order, int ngx, int ngy, int ngb, int n, const int32_t* ix, const int32_t* iy,
                        const float* ox, const float* oy, int64_t* acc);
/* Same for the currents: contributions scaled by v / c_light. */
void or_det_deposit_j(int order, int ngx, int ngy, int ngb, int n, const int32_t* ix, const int32_t* iy,
                      const float* ox, const float* oy, const float* vx, const float* vy, int64_t* accx,
                      int64_t* accy);
void or_shape_build(int order, float h, float* w);
void or_shape_ref_f32(int order, float h, float* w);
void or_shape_ref_f64(int order, double h, double* w);
void or_pcg_stream(uint64_t master_seed, uint64_t first_slot, int nslots, int ndraws, uint32_t* out);
double or_minstd_uniform(int count, double* out);
void or_splitmix64_stream(uint64_t seed, int n, uint64_t* out);
void or_pcg32_raw(uint64_t state, uint64_t inc, int n, uint32_t* out);
int or_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif

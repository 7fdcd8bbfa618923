/* CPU restatement of the reference's hydro force path (FP64).
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this; it is
 * the checker that tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg compare the CUDA path against.  Each function cites the reference lines
 * it restates (paths relative to the reference project root).
 *
 * Two families of entry points:
 *  - walk mode  (orc_hydro_walks): the FDPS multiwalk contract of
 *    src/kernel.cu:289-409 / src/force.h:31-60 — every i of a walk is summed
 *    against every j of that walk's (superset) j-list;
 *  - neighbour mode (orc_cells, orc_neighbors, orc_density, orc_hydro,
 *    orc_step): the device-resident path, where the pair set is defined by the
 *    FP32 predicate  0 < r2 < (2h)^2  evaluated exactly as the GPU does.
 */
#ifndef WCSPH_ORACLE_H
#define WCSPH_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* FDPS plugin records, byte-compatible with src/class.h:61-263 (x86-64). */
typedef struct { double pos[3], vel[3], smth, dens, pres, snds, visc; int64_t tag; } orc_epi_hydro;
typedef struct { double pos[3], vel[3], dens, mass, smth, pres, snds, visc; int64_t tag; int32_t type; int32_t pad_; } orc_epj_hydro;
typedef struct { double acc[3], dt, div_v; } orc_result_hydro;

/* Pair-sum variants (see src/force.h:31-60 vs src/kernel.cu:241-280). */
enum { ORC_VSIG_REF_CPU = 0,  /* v_sig = max(v_sig, mu)  (force.h:47)      */
       ORC_VSIG_SIGNAL = 1 }; /* v_sig = max(v_sig, -mu) (kernel.cu:263)   */
enum { ORC_GRAD_HBAR = 0,     /* gradW(dr, (h_i+h_j)/2)  (force.h:49)      */
       ORC_GRAD_SYM = 1 };    /* (gradW(dr,h_i)+gradW(dr,h_j))/2 (kernel.cu:265) */

typedef struct {
  double alpha;    /* artificial-viscosity alpha (force.h:32: 0.01)          */
  double beta;     /* mu^2 coefficient (kernel.cu:262 uses 2*alpha)         */
  double c_cfl;    /* CFL number in the per-particle dt (param.h:5)         */
  double eps;      /* 0.01 in r^2 + eps*h_i*h_j (force.h:45)                 */
  int32_t vsig_mode, grad_mode;
} orc_pair_params;

/* Device-resident (neighbour-mode) configuration. */
typedef struct {
  double h, mass, nu;             /* uniform smoothing length, mass, kinematic viscosity */
  double rho0, gamma, c0;         /* Tait EoS (EoS.h:75-90)                 */
  double g;                       /* gravity along -z (Dam2.h:104-108)      */
  double rho_floor;               /* density floor (Dam2.h:111)             */
  orc_pair_params pair;
  int32_t periodic;               /* 1: periodic box [lo, hi) on all axes   */
  int32_t density_mode;           /* 0 continuity only, 1 summation every step, 2 Shepard every shepard_interval steps */
  int32_t shepard_interval;
  int32_t pad_;
  float lo[3], hi[3];             /* grid (or periodic box) bounds, FP32    */
  float cell[3];                  /* cell edge per axis, FP32 (>= 2h)       */
  int32_t ncell[3];
  float kill_lo[3], kill_hi[3];   /* non-FREEZE particles outside are removed (Dam2.h:117-122) */
} orc_config;

/* ---- kernel function and EoS -------------------------------------------- */
double orc_W(double r, double h);                   /* kernel.h:39-46 */
double orc_gradW_scalar(double r, double h);        /* |gradW| / r factor, kernel.h:47-54 */
void orc_eos(int n, const double* dens, double* pres, double* snds, double gamma, double rho0, double c0);

/* ---- walk mode ----------------------------------------------------------- */
void orc_hydro_walks(int n_walk, const int* ni_displ, const orc_epi_hydro* epi, const int* nj_displ,
                     const orc_epj_hydro* epj, orc_result_hydro* out, const orc_pair_params* pp);
void orc_filter_walks(int n_walk, const int* ni_displ, const double* epi_pos_smth /* 4 per i */,
                      const int* nj_displ, const double* epj_pos_dens_mass /* 5 per j */, double* out_dens);

/* ---- neighbour mode ------------------------------------------------------ */
/* Cell of each particle and its 30-bit Morton key (x in bit 0). */
void orc_cells(int n, const float* pos4, const orc_config* cfg, int32_t* cell_xyz /* 3 per i */, uint32_t* key);
/* Stable sort by key: perm[k] = index of the particle that goes to slot k. */
void orc_sort_perm(int n, const uint32_t* key, int32_t* perm);
/* Neighbour counts under the FP32 predicate; optionally the lists (cap per i,
 * ascending j).  Returns the number of (ordered) pairs, or -1 if some count
 * exceeded cap (lists are then truncated). */
int64_t orc_neighbors(int n, const float* pos4, const orc_config* cfg, int32_t* count, int32_t* list, int cap);
/* Density summation rho_i = sum_{j in N(i) + i} m W (plain) and the Shepard
 * form of force.h:10-30 (sum m W / sum (m/rho_j) W). */
void orc_density(int n, const float* pos4, const float* dens_in, const orc_config* cfg, int shepard, double* dens_out);
/* Hydro pair sum in neighbour mode.  pos4 = (x,y,z,-), vel4 = (vx,vy,vz,-),
 * dens/pres/snds per particle.  acc includes no gravity. */
void orc_hydro(int n, const float* pos4, const float* vel4, const float* dens, const float* pres, const float* snds,
               const orc_config* cfg, double* acc3, double* div_v, double* dt);
/* min over HYDRO particles of {dt_i, 0.25 sqrt(h/|a|), 0.125 h^2/nu} (integral.h:2-12). */
double orc_dt_global(int n, const double* acc3, const double* dt, const int32_t* type, double h, double nu);

/* One full step of the device-resident pipeline in FP64 state
 * (main.cpp:89-133 order).  State arrays (length n, SoA, FP64) are updated in
 * place; acc3/div_v/dt must hold the previous force pass.  Returns the dt used. */
double orc_step(int n, double* pos3, double* vel3, double* vel_half3, double* dens, double* acc3, double* div_v,
                double* dt_i, const int32_t* type, const orc_config* cfg, int64_t step_index);
/* The initial force pass of main.cpp:69-78 (EoS, optional density pass, hydro, gravity, floor). */
void orc_initial_force(int n, const double* pos3, const double* vel3, double* dens, double* acc3, double* div_v,
                       double* dt_i, const orc_config* cfg);

#ifdef __cplusplus
}
#endif
#endif

/* wcsph — B200-native weakly-compressible SPH hydro force path, C ABI.
 *
 * Two surfaces:
 *
 *  1. The FDPS multiwalk plugin pair.  The reference hands
 *       GPU_WC::HydrDispatchKernel / GPU_WC::HydrRetrieveKernel
 *     (src/prototype.h:7-10, src/kernel.cu:289-409) to
 *       calcForceAllAndWriteBackMultiWalk(dispatch, retrieve, tag_max, ...)
 *     (src/main.cpp:71,112,118).  wcsph_hydro_dispatch / wcsph_hydro_retrieve
 *     take exactly those arguments, with the EPI/EPJ/RESULT records described
 *     by a byte-offset layout instead of the reference's C++ types, so that the
 *     library does not depend on the reference's headers.  include/wcsph_fdps.hpp
 *     defines the GPU_WC:: functions with the reference's signatures on top.
 *
 *  2. A device-resident solver (wcsph_sim_*): particle state stays in HBM;
 *     each step runs cell binning + Morton sort, the density pass, the Tait EoS,
 *     the hydro pass, gravity, the KDK update and the CFL dt reduction on the
 *     device (src/main.cpp:89-133 loop order).  One solver object holds any
 *     number of independent simulation instances that step together
 *     (ensembles and the serving loop).
 *
 * Error convention: every int-returning entry point returns 0 (WCSPH_OK) on
 * success and a non-zero wcsph_status otherwise; wcsph_last_error() then holds
 * a message for the calling thread.  (The reference returns 0 always and
 * asserts on overflow, src/kernel.cu:316,367,380,408.)
 *
 * Threading: the plugin state is process-global like the reference's
 * (src/kernel.cu:239-240); call it from one host thread.  Solver objects are
 * independent and may be used from different threads.
 */
#ifndef WCSPH_H
#define WCSPH_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WCSPH_ABI_VERSION 2

typedef enum {
  WCSPH_OK = 0,
  WCSPH_E_INVALID = 1,  /* bad argument or configuration */
  WCSPH_E_CUDA = 2,     /* a CUDA runtime call failed */
  WCSPH_E_CAPACITY = 3, /* a size limit was exceeded (particles, walks, cells, neighbours) */
  WCSPH_E_STATE = 4,    /* call out of order (e.g. retrieve without dispatch) */
  WCSPH_E_NOMEM = 5,    /* device or pinned-host allocation failed */
  WCSPH_E_NODEVICE = 6  /* no CUDA device / the library was not built for it */
} wcsph_status;

int wcsph_abi_version(void);
const char* wcsph_last_error(void);

/* Select the CUDA device the plugin uses (replaces the cudaSetDevice(rank) /
 * stdin prompt of src/kernel.cu:291-299).  Optional: the first dispatch uses
 * the current device when wcsph_init was not called. */
int wcsph_init(int32_t device);
/* Release the plugin's device and pinned buffers (the reference never frees them). */
int wcsph_finalize(void);

/* ------------------------------------------------------------------------- */
/* 1. FDPS multiwalk plugin                                                    */
/* ------------------------------------------------------------------------- */

/* Byte offsets of the FP64 fields inside the caller's plugin records.  Vector
 * fields are three consecutive doubles.  wcsph_fdps_default_layout() fills in
 * STD::EPI::Hydro / STD::EPJ::Hydro / STD::RESULT::Hydro of src/class.h:61-263
 * on x86-64 (96 / 112 / 40 bytes). */
typedef struct wcsph_fdps_layout {
  int32_t epi_size, epi_pos, epi_vel, epi_smth, epi_dens, epi_pres, epi_snds, epi_visc;
  int32_t epj_size, epj_pos, epj_vel, epj_dens, epj_mass, epj_smth, epj_pres, epj_snds, epj_visc;
  int32_t res_size, res_acc, res_dt, res_div_v;
  /* Shepard filter records (EPI::Filter, EPJ::Filter, RESULT::Filter, class.h:75-81,194-208,246-262) */
  int32_t fepi_size, fepi_pos, fepi_smth;
  int32_t fepj_size, fepj_pos, fepj_dens, fepj_mass;
  int32_t fres_size, fres_dens;
} wcsph_fdps_layout;

/* Which pair-sum variant the plugin computes. */
typedef enum {
  WCSPH_VSIG_REF_CPU = 0, /* v_sig = max(v_sig,  mu) as src/force.h:47 (always 0)       */
  WCSPH_VSIG_SIGNAL = 1   /* v_sig = max(v_sig, -mu) as src/kernel.cu:263               */
} wcsph_vsig_mode;
typedef enum {
  WCSPH_GRAD_HBAR = 0, /* gradW(dr, (h_i+h_j)/2)             src/force.h:49   */
  WCSPH_GRAD_SYM = 1   /* (gradW(dr,h_i) + gradW(dr,h_j))/2  src/kernel.cu:265 */
} wcsph_grad_mode;

typedef struct wcsph_pair_params {
  double alpha; /* artificial-viscosity alpha */
  double beta;  /* coefficient of the mu^2 term (kernel.cu:262 has 2*alpha) */
  double c_cfl; /* CFL number of the per-particle dt (param.h:5) */
  double eps;   /* 0.01 in r^2 + eps h_i h_j (force.h:45) */
  int32_t vsig_mode, grad_mode;
} wcsph_pair_params;

void wcsph_fdps_default_layout(wcsph_fdps_layout* out);
/* force.h:31-60 semantics: alpha 0.01, beta 0, C_CFL 0.3, v_sig = max(mu), gradW(hbar). */
void wcsph_pair_params_reference_cpu(wcsph_pair_params* out);
/* kernel.cu:241-280 semantics: alpha 0.01, beta 0.02, C_CFL 0.3, v_sig = max(-mu), symmetrised gradW. */
void wcsph_pair_params_reference_gpu(wcsph_pair_params* out);
/* Set the record layout and pair variant used by later dispatches (defaults:
 * wcsph_fdps_default_layout, wcsph_pair_params_reference_gpu). */
int wcsph_fdps_configure(const wcsph_fdps_layout* layout, const wcsph_pair_params* params);

/* Number of independent tags (buffer sets).  FDPS's tag_max argument
 * (main.cpp:71 passes 1) must not exceed it. */
#define WCSPH_FDPS_MAX_TAGS 4

/* Replaces GPU_WC::HydrDispatchKernel (src/prototype.h:9, src/kernel.cu:289-381).
 * epi[w] points at n_epi[w] EPI records and epj[w] at n_epj[w] EPJ records of
 * walk w.  The records are staged and the pair sum is enqueued; the call
 * returns without waiting for the GPU.  Every i of a walk is summed against
 * every j of the same walk (the FDPS j-list is a superset; pairs outside the
 * kernel support contribute zero, except to v_sig in WCSPH_VSIG_SIGNAL mode,
 * which src/kernel.cu:263 takes over the whole list). */
int wcsph_hydro_dispatch(int32_t tag, int32_t n_walk, const void* const* epi, const int32_t* n_epi,
                         const void* const* epj, const int32_t* n_epj);
/* Replaces GPU_WC::HydrRetrieveKernel (src/prototype.h:10, src/kernel.cu:383-409).
 * Blocks until the walks of the last dispatch with this tag are done and
 * writes acc, dt and div_v of n_i[w] RESULT records at force[w]. */
int wcsph_hydro_retrieve(int32_t tag, int32_t n_walk, const int32_t* n_i, void* const* force);

/* Transfer figures of the last dispatch with this tag (no counterpart in the
 * reference; src/kernel.cu:370-373,388 copy fixed-size half records):
 * out[0] bytes copied host to device (walk records, displacements, work
 * list), out[1] bytes copied device to host (results), out[2] pieces of the
 * batch staged compactly (36-byte records: every record of the piece carried
 * the same h, nu and m, which then travel once, as src/kernel.cu:303-304
 * hoists them), out[3] pieces in all (the rest used 48-byte records). */
int wcsph_fdps_stats(int32_t tag, int64_t* out4);

/* Allocation-free walk pair sum.  No counterpart in the reference: it is for
 * callers that cannot allocate device memory, such as an application that owns
 * all device memory through its own pool allocator or runs under a fixed
 * device-memory budget, or a host loop where a cudaMalloc would synchronise
 * the device in the middle of a step.
 * Everything is device-resident and caller-owned:
 *   d_n_epi, d_n_epj  n_walk int32 walk sizes
 *   d_epi             sum(n_epi) records of three float4:
 *                     (x, y, z, h) (x relative to any origin shared by the walk),
 *                     (vx, vy, vz, rho), (P/rho^2, c, nu, 0)
 *   d_epj             sum(n_epj) records of three float4, the last (P/rho^2, c, nu, m)
 *   d_out             sum(n_epi) results of two float4: (ax, ay, az, div_v), (dt, 0, 0, 0)
 * with the pair variant of params, launched on `stream` (a cudaStream_t,
 * NULL for the legacy stream).  The only scratch, the per-walk displacement
 * tables, is a static device array of WCSPH_NOALLOC_MAX_WALKS walks (about
 * 512 KB per GPU, kept until exit); larger n_walk returns WCSPH_E_CAPACITY.
 * The first call on a device looks the array up (cudaGetSymbolAddress), so
 * make that first call before any stream capture.  All calls share the one
 * array: calls that overlap on the GPU (different streams, no ordering) race.
 * Calls no cudaMalloc, cudaFree or allocating library routine. */
#define WCSPH_NOALLOC_MAX_WALKS 65536
int wcsph_hydro_walks_noalloc(int32_t n_walk, const int32_t* d_n_epi, const int32_t* d_n_epj, const void* d_epi,
                              const void* d_epj, void* d_out, const wcsph_pair_params* params, void* stream);

/* Shepard density filter in the same dispatch/retrieve shape (the reference
 * runs STD::ApplyFilter, src/force.h:10-30, on the CPU through
 * calcForceAllAndWriteBack; its Gather j-lists contain i itself). */
int wcsph_filter_dispatch(int32_t tag, int32_t n_walk, const void* const* epi, const int32_t* n_epi,
                          const void* const* epj, const int32_t* n_epj);
int wcsph_filter_retrieve(int32_t tag, int32_t n_walk, const int32_t* n_i, void* const* result);

/* ------------------------------------------------------------------------- */
/* 2. Device-resident solver                                                   */
/* ------------------------------------------------------------------------- */

typedef enum {
  WCSPH_PREC_FP32 = 0,  /* plain FP32 pair arithmetic, one thread per i-particle          */
  WCSPH_PREC_TILED = 1, /* FP32, shared-memory j-tiles, ballot-compacted pair queues      */
  WCSPH_PREC_HALF2 = 2  /* with neighbour lists: the list pass gathers 16-byte compact
                           j-records (16-bit cell-relative positions and velocities, FP32
                           density), FP32 pair arithmetic and accumulation; without
                           lists the same as WCSPH_PREC_TILED                            */
} wcsph_precision;

typedef enum {
  WCSPH_DENSITY_CONTINUITY = 0, /* d rho/dt = -rho div v only (class.h:151)                */
  WCSPH_DENSITY_SUMMATION = 1,  /* rho_i = sum_j m W_ij (incl. self) every step            */
  WCSPH_DENSITY_SHEPARD = 2     /* continuity + Shepard filter every shepard_interval steps
                                   (force.h:10-30, main.cpp:105, param.h:12)              */
} wcsph_density_mode;

typedef enum { WCSPH_HYDRO = 0, WCSPH_FREEZE = 1 } wcsph_particle_type; /* class.h:33-36 */

/* One simulation instance.  h and mass are uniform within an instance (as the
 * reference assumes when it hoists them, src/kernel.cu:303-304). */
typedef struct wcsph_instance_desc {
  int32_t n;                   /* particles */
  int32_t density_mode;        /* wcsph_density_mode */
  int32_t shepard_interval;    /* steps between Shepard filters (reference: 30) */
  int32_t periodic;            /* 1: periodic box [lo, hi) on all three axes */
  double h, mass, nu;          /* smoothing length, particle mass, kinematic viscosity */
  double rho0, gamma, c0;      /* Tait EoS (EoS.h:75-90) */
  double g;                    /* gravity along -z, added to every particle (Dam2.h:104-108) */
  double rho_floor;            /* density floor applied after each step (Dam2.h:111) */
  wcsph_pair_params pair;      /* alpha, beta, C_CFL, eps, v_sig variant (grad_mode is moot: h uniform) */
  float lo[3], hi[3];          /* cell-grid bounds (the periodic box when periodic) */
  float kill_lo[3], kill_hi[3];/* HYDRO particles leaving this box are removed (Dam2.h:117-122);
                                  ignored when kill_lo >= kill_hi on an axis */
  double t_end;                /* physical end time; 0 = run until removed */
} wcsph_instance_desc;

typedef struct wcsph_sim_options {
  int32_t device;              /* CUDA device ordinal */
  int32_t precision;           /* wcsph_precision */
  int64_t max_particles;       /* capacity over all instances */
  int64_t max_cells;           /* capacity of the cell table over all instances */
  int32_t max_instances;
  int32_t use_graph;           /* capture each step in a CUDA graph (1) or launch eagerly (0) */
  int32_t autotune;            /* 1: time the kernel variants on the live instance set (probe
                                  passes, state untouched) and keep the fastest, re-tuned when the
                                  particle count crosses a power of two; 0: fixed defaults */
  int32_t list_interval;       /* 0: search neighbours every step (exact order of the reference
                                  loop).  K > 0 (tiled and half2 precisions): neighbour lists of
                                  radius 2h + list_skin h, rebuilt at least every K steps and
                                  whenever the instance set changes or the measured drift nears
                                  half the skin; the steps between (density passes included)
                                  read the lists and test 0 < r^2 < (2h)^2 on current positions,
                                  so the pairs summed are the same as with a fresh search (the
                                  summation order differs) */
  float list_skin;             /* skin in units of h (0: 0.3) */
  int32_t list_shape;          /* launch shapes of the neighbour-list passes, 0 in a field for the
                                  autotuner's choice (shape 0 without autotune): bits 0-7 s + 1 fix
                                  the list pass's shape s (wcsph_sim_tuning's out[1]), bits 8-15
                                  b + 1 the list build scan's shape b (out[3]) */
} wcsph_sim_options;

typedef struct wcsph_sim wcsph_sim;

int wcsph_sim_create(const wcsph_sim_options* opt, wcsph_sim** out);
int wcsph_sim_destroy(wcsph_sim* sim);
/* Bytes of device memory the solver allocates for these options (admission
 * control uses it). */
int64_t wcsph_sim_device_bytes(const wcsph_sim_options* opt);

/* Add an instance from host arrays (pos3/vel3: 3 floats per particle, dens:
 * 1 float, type: wcsph_particle_type).  Runs the instance's initial force pass
 * (main.cpp:69-78) before returning.  *slot receives the instance handle. */
int wcsph_sim_add_instance(wcsph_sim* sim, const wcsph_instance_desc* desc, const float* pos3, const float* vel3,
                           const float* dens, const int32_t* type, int32_t* slot);
/* Restore an instance from a restart file's state (io.h:60-84 reads the
 * reference's binary dumps): positions, velocities, densities, types, the
 * last force pass's acc3 and div_v, the physical time, step count and the dt
 * of the next step.  No force pass is run, so stepping continues exactly where
 * the saved run stopped.  alive (may be NULL) drops particles with alive[i] = 0;
 * they keep their original index in reads.  order (may be NULL) is the
 * sequence in which the particles are stored on the device, a permutation of
 * 0..n-1 (wcsph_sim_read_order's perm followed by the dead particles): the
 * binning sort is stable, so with the saved order the neighbour sums run in
 * the same sequence and the continuation is bit-identical. */
int wcsph_sim_restore_instance(wcsph_sim* sim, const wcsph_instance_desc* desc, const float* pos3, const float* vel3,
                               const float* dens, const int32_t* type, const float* acc3, const float* div_v,
                               const int32_t* alive, const int32_t* order, double time, int64_t steps,
                               float dt_next, int32_t* slot);
/* dt the instance's next step will use (its CFL minimum from the last force pass). */
int wcsph_sim_next_dt(wcsph_sim* sim, int32_t slot, float* dt_next);
/* Overwrite it (e.g. with the minimum over the slabs of one simulation). */
int wcsph_sim_set_next_dt(wcsph_sim* sim, int32_t slot, float dt_next);
/* The initial force pass of an instance (main.cpp:69-78) on its current
 * particles: run by wcsph_sim_add_instance itself, and by a slab rank once
 * its first ghost layer is in place. */
int wcsph_sim_force_pass(wcsph_sim* sim, int32_t slot);

/* ---- slab decomposition: one simulation over several solvers ------------
 * Replaces FDPS's domain decomposition and particle exchange
 * (main.cpp:61-62,109-110).  Each rank owns the particles with x in
 * [x_lo, x_hi) as one instance and holds ghost copies of its neighbours'
 * particles within a layer of width wcsph_slab_layer_width() beyond each
 * face.  Per step, on every rank:
 *   wcsph_sim_step(sim, 1);
 *   wcsph_sim_slab_pack(...)   -> records [emigrants L, ghosts L, emigrants R, ghosts R]
 *   (transport: send the L part left and the R part right, receive both)
 *   wcsph_sim_slab_unpack(...) once per received part
 *   dt = min over ranks of wcsph_sim_next_dt(); wcsph_sim_set_next_dt(dt)
 * Records are WCSPH_SLAB_RECORD_BYTES each: float4 (x, y, z, rho),
 * float4 (vx, vy, vz, 0), float4 (ax, ay, az, div v), int32 id,
 * int32 type, 8 bytes padding.  The x axis must not be periodic. */
#define WCSPH_SLAB_RECORD_BYTES 64
typedef struct wcsph_slab {
  float x_lo, x_hi;            /* owned range [x_lo, x_hi); a side without a neighbour extends to the grid */
  float margin;                /* largest drift of a particle in one step that the ghost layer covers (> 0) */
  int32_t has_left, has_right; /* a neighbouring slab exists on that side */
} wcsph_slab;

/* Ghost-layer width W = 2 (2h) (1 + 1e-4) + 2 margin, in FP32. */
float wcsph_slab_layer_width(double h, float margin);
/* Add a slab instance: desc describes the whole simulation (desc->n is the
 * size of the id space, grid bounds are the whole domain's); the count
 * particles given (ids[k] in [0, desc->n)) are the ones the slab owns.  No
 * force pass runs: exchange a first ghost layer, then wcsph_sim_force_pass. */
int wcsph_sim_add_slab(wcsph_sim* sim, const wcsph_instance_desc* desc, const wcsph_slab* slab, int32_t count,
                       const int32_t* ids, const float* pos3, const float* vel3, const float* dens,
                       const int32_t* type, int32_t* slot);
/* Classify, pack into the device buffer send (capacity records) and retire
 * the previous ghost layer.  counts[4] = emigrants left, ghosts left,
 * emigrants right, ghosts right; the records are in that order.  Returns
 * WCSPH_E_STATE when a particle drifted farther than the margin in a step and
 * WCSPH_E_CAPACITY when the records do not fit (nothing changed then). */
int wcsph_sim_slab_pack(wcsph_sim* sim, int32_t slot, void* send, int64_t capacity, int32_t counts[4]);
/* Append n_owned + n_ghost records from the device buffer recv: the first
 * n_owned become owned particles (a neighbour's emigrants), the rest ghosts. */
int wcsph_sim_slab_unpack(wcsph_sim* sim, int32_t slot, const void* recv, int32_t n_owned, int32_t n_ghost);
/* Remove an instance; its particles and cells are reclaimed at the next step. */
int wcsph_sim_remove_instance(wcsph_sim* sim, int32_t slot);

/* Advance every active instance by nsteps steps (each by its own CFL dt).
 * Instances whose time reached t_end stop advancing. */
int wcsph_sim_step(wcsph_sim* sim, int32_t nsteps);
int wcsph_sim_synchronize(wcsph_sim* sim);

/* Instance status: physical time, steps taken, live particle count, finished
 * flag.  With neighbour lists the live count is that of the latest list build
 * (particles removed on the steps between leave the sums and the reads at
 * once, the count at the next build). */
int wcsph_sim_instance_status(wcsph_sim* sim, int32_t slot, double* time, int64_t* steps, int32_t* n_alive,
                              int32_t* finished);
/* Copy an instance's state to host arrays in its ORIGINAL particle order
 * (removed particles keep their last state and get alive[i] = 0).  Any pointer may be NULL. */
int wcsph_sim_read_instance(wcsph_sim* sim, int32_t slot, float* pos3, float* vel3, float* dens, float* acc3,
                            float* div_v, float* dt_i, int32_t* alive);

/* Diagnostics for parity checks on an instance's current state, without
 * advancing it, in ORIGINAL particle order: run the force pass (EoS + hydro)
 * from the current positions, velocities and densities and return the hydro
 * acceleration (no gravity), div v, per-particle dt and the neighbour count of
 * each particle.  density_pass: 0 none, 1 summation, 2 Shepard first. */
int wcsph_sim_probe_forces(wcsph_sim* sim, int32_t slot, int32_t density_pass, float* acc3, float* div_v, float* dt_i,
                           float* dens_out, int32_t* n_neighbors);
/* The same diagnostics computed by the passes a neighbour-list step runs
 * (list_interval > 0): the density pass from the lists (k_density_list) and
 * the pair terms over the lists (k_hydro_list), on the current lists and the
 * current state (the step's refresh of the j-records without its kick).  The
 * sums are those of src/force.h:31-60 (pairs) and src/force.h:12-29 (Shepard)
 * over the in-support entries of each list.  When the solver holds no current
 * lists (none built yet, or the instance set changed), a probe build pass
 * makes them first; the steps that follow read them.  Returns WCSPH_E_STATE
 * when the solver has no lists. */
int wcsph_sim_probe_lists(wcsph_sim* sim, int32_t slot, int32_t density_pass, float* acc3, float* div_v, float* dt_i,
                          float* dens_out, int32_t* n_neighbors);
/* The sorted order of the last binning: perm[k] = original index of the
 * particle in sorted slot k of the instance, and the Morton cell key of each slot. */
int wcsph_sim_read_order(wcsph_sim* sim, int32_t slot, int32_t* perm, uint32_t* cell_key);
/* Conservation sums over an instance's live particles, accumulated on the
 * device in FP64 from the state after the last step (the KDK update of
 * src/class.h:146-163): out[0] mass, out[1..3] momentum, out[4] kinetic
 * energy, out[5] sum m (a_z + g), the vertical total of the pair forces with
 * gravity taken out (zero up to rounding: the pair terms of force.h:38-57
 * are antisymmetric). */
int wcsph_sim_conservation(wcsph_sim* sim, int32_t slot, double* out6);

/* Number of true in-support (ordered) pairs the hydro pass summed in the
 * last step (0 < r^2 < (2h)^2, i != j), over all instances. */
int64_t wcsph_sim_last_pairs(wcsph_sim* sim);
/* Number of kernel launches per step issued by the solver (for accounting). */
int32_t wcsph_sim_kernels_per_step(wcsph_sim* sim);
/* The autotuner's current choice: out[0] block shape of the tiled hydro
 * kernel (0: 4 warps, 1: 2 warps, 2: 8 warps per block, 512-candidate tiles;
 * the shapes share their arithmetic, so results do not depend on the choice),
 * out[1] launch shape of the neighbour-list pass (list_interval > 0; 0: one
 * thread per particle, 5 blocks of 128 per SM; 1: two threads per particle,
 * each taking alternate groups of four list entries, 4 blocks per SM; 2: one
 * thread per particle, 4 blocks per SM; 3: two threads per particle, 5 blocks
 * per SM; 4-6: shape 0 with the half2 pass's neighbour-cell offsets read from
 * a shared table instead of shifted out of the entry (4), P/rho^2 recomputed
 * from the density instead of gathered (5), or both (6); in the FP32 pass
 * shape 0.  Shapes 0,
 * 2 and 4 sum in one order, 1 and 3 in another; 5 and 6 round P/rho^2
 * differently: results agree to FP32 rounding), out[2] log2 particle bucket
 * it was tuned for (-1:
 * defaults, not tuned), out[3] shape of the list build's scan (0-2 as out[0];
 * 3, 4: 4 or 8 warps per block with 256-candidate tiles; 5, 6: one lane per
 * particle walking a 512- or 256-candidate tile, 4 or 8 warps per block; all
 * build the same lists). */
int wcsph_sim_tuning(wcsph_sim* sim, int32_t* out4);
/* Neighbour-list counters (list_interval > 0): out[0] list builds, out[1]
 * steps that read the lists, out[2] builds whose lists overflowed (the next
 * step builds again), out[3] largest list built so far, out[4] kernel
 * launches of a build step, out[5] kernel launches of a list step. */
int wcsph_sim_list_stats(wcsph_sim* sim, int64_t* out6);
/* The neighbour-list schedule (list_interval > 0): out[0] builds, out[1]
 * partial builds among them (only the instances whose particles could reach
 * half the skin re-sorted and rebuilt; the others kept their lists), out[2]
 * steps that read the lists, out[3] steps since the last full build.  No
 * counterpart in the reference (its FDPS call rebuilds every interaction
 * list each step, main.cpp:107-121, param.h:11). */
int wcsph_sim_list_schedule(wcsph_sim* sim, int64_t* out4);
/* Entries of the current neighbour lists over all particles (what one list
 * pass reads: each entry a list word and a j-record), 0 without current
 * lists, -1 on error. */
int64_t wcsph_sim_list_entries(wcsph_sim* sim);
/* Drop the current neighbour lists (list_interval > 0): the next step builds
 * them again, as after a change of the instance set.  For callers that edit
 * state outside the solver, and for timing a build-inclusive sequence of
 * steps.  A no-op without lists. */
int wcsph_sim_invalidate_lists(wcsph_sim* sim);
/* The solver's CUDA stream (a cudaStream_t), so callers can record events on it. */
void* wcsph_sim_stream(wcsph_sim* sim);
/* Run nsteps steps launched one by one (no graph) with CUDA events around each
 * phase and accumulate milliseconds: ms[0] step-begin + kick + binning + sort +
 * permutation, ms[1] density pass + EoS refresh, ms[2] hydro pass, ms[3] whole
 * steps.  Advances the simulation like wcsph_sim_step. */
int wcsph_sim_profile_steps(wcsph_sim* sim, int32_t nsteps, double* ms4);
/* The same eager steps, their phase times split by kind: ms[0..3] summed over
 * the steps that searched (list_interval = 0) or built the neighbour lists,
 * ms[4..7] over the steps that read the lists, ms[8] the builds' list scans
 * alone (a build's hydro phase is its scan plus one list pass, so a list
 * step's ms[6] is one list-pass launch); steps[0], steps[1] count the two
 * kinds.  Times of the per-kernel roofline; no counterpart in the reference
 * (its Timer, class.h:3-17, times whole steps). */
int wcsph_sim_profile_split(wcsph_sim* sim, int32_t nsteps, double* ms9, int32_t* steps2);

#ifdef __cplusplus
}
#endif
#endif /* WCSPH_H */

// Device-resident solver: host orchestration of the step pipeline and the
// wcsph_sim_* C ABI.
//
// Step (one CUDA graph, main.cpp:89-133 order):
//   k_step_begin   dt rotation (integral.h:2-12 result of the previous pass), time += dt
//   k_kick_bin     initialKick + fullDrift + predict (class.h:146-159), Morton cell key
//   radix sort     (keys, slot) pairs, stable
//   memset x2      cell table
//   k_permute      gather main -> alt in sorted order, cell table, EoS j-records
//   k_density/eos  density pass when an instance wants one this step
//   k_hydro        pair sums, gravity, finalKick, density floor, next dt
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <mutex>
#include <vector>

#include "sim_kernels.cuh"
#include "sim_aux.cuh"
#include "sim_tiled.cuh"
#include "sim_slab.cuh"
#include "sim_list.cuh"

namespace wcsph {

struct HostInst {
  bool used = false;     // slot holds an instance (active or draining)
  bool slab = false;     // one slab of a decomposed simulation (wcsph_sim_add_slab)
  SlabGeom geom{};
  bool active = false;   // stepping
  bool drained = false;  // removed, and a pass has been enqueued since (its particles are dead keys)
  wcsph_instance_desc desc{};
  int n = 0;
  int ncell[3] = {0, 0, 0};
  float cell[3] = {0, 0, 0};
  int bits = 0;
};

struct SimImpl {
  wcsph_sim_options opt{};
  cudaStream_t s = nullptr;
  SimArrays buf_main{}, buf_alt{};
  uint32_t *keys_in = nullptr, *keys_out = nullptr;
  int *vals_in = nullptr, *vals_out = nullptr;
  JRec* jr = nullptr;
  float *jC = nullptr, *rho_new = nullptr;
  int *cell_start = nullptr, *cell_end = nullptr;
  InstParams* d_params = nullptr;
  InstDyn* d_dyn = nullptr;
  int* d_phase = nullptr;
  int* d_n_alive = nullptr;
  int* run_list = nullptr;
  int* d_counters = nullptr;  // [0] run_count, [4] density pass in this launch (slab pack: [0..3] between passes)
  unsigned long long* d_pairs = nullptr;
  double* d_cons = nullptr;
  float4* diag_acc = nullptr;
  float *diag_dt = nullptr, *diag_rho = nullptr;
  int* diag_nbr = nullptr;
  void* cub_tmp = nullptr;
  size_t cub_bytes = 0;
  std::vector<void*> allocs;

  std::vector<HostInst> inst;
  std::vector<InstParams> h_params;
  std::vector<int> h_phase;
  int n_host = 0;
  bool appended = false;       // particles were appended after the last pass (its live count is stale)
  int key_bits = 1;
  long long total_cells = 0;
  bool any_density = false;
  int tile_shape = 0;          // tiled pair-kernel shape, chosen by the autotuner
  int list_shape = 0;          // list-pass launch shape (kListShapes), chosen by the autotuner
  int build_shape = 0;         // list build's scan shape (kBuildShapes), chosen by the autotuner
  int tuned_bucket = -1;       // log2 particle bucket of the last tuning
  cudaGraphExec_t gexec = nullptr;
  bool graph_dirty = true;
  int kernels_per_step = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // neighbour lists (opt.list_interval > 0)
  uint32_t* list = nullptr;
  int* list_cnt = nullptr;
  float4* x0 = nullptr;
  uint4* jh = nullptr;  // compact j-records of the half2 list pass (write_h16)
  float* jpo = nullptr;  // P/rho^2 beside them
  int* d_keep = nullptr;  // per instance: keeps its lists in a partial build (k_list_set)
  unsigned* d_lflags = nullptr;       // kLfWords words, see ListFlag
  unsigned* d_motion = nullptr;       // 3 words per instance, see StepArgs::inst_motion
  unsigned* h_lflags = nullptr;       // pinned copy, written at the end of every list-mode step
  cudaEvent_t step_ev[2] = {nullptr, nullptr};
  cudaEvent_t scan_ev = nullptr;  // set while profiling: recorded between a build's scan and its list pass
  bool lists_valid = false;           // false: the next step is asked to build (kLfForce)
  int kernels_reuse = 0;
  long long steps_launched = 0;
};

constexpr int kListMax = kListMaxEntries;  // entries per particle list (2h + 0.3 h holds ~100-115 at h = 1.3 dx)
static float list_skin(const wcsph_sim_options& o) { return o.list_skin > 0.f ? o.list_skin : 0.3f; }
// velocity_quantum (sim_list.cuh) on the host: 2^-15 of the smallest power of
// two above max(vb, c0 2^-12).
static float host_velocity_quantum(float vb, float c0) {
  const float v = std::max(vb, c0 / 4096.0f);
  return std::ldexp(1.0f, std::ilogb(v) + 1 - 15);
}

static int alloc(SimImpl& S, void** p, size_t bytes) {
  WCSPH_CUDA(cudaMalloc(p, bytes ? bytes : 16));
  S.allocs.push_back(*p);
  return 0;
}

static size_t cub_sort_bytes(long long n) {
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr, (const int*)nullptr,
                                  (int*)nullptr, (int)n, 0, 32);
  return bytes;
}

static size_t per_particle_bytes() {
  return 2 * (4 * sizeof(float4) + sizeof(int) + sizeof(uint32_t))  // main + alt state
         + 2 * (sizeof(uint32_t) + sizeof(int))                     // sort keys/values in/out
         + 2 * sizeof(float4) + 2 * sizeof(float)                   // j-records (jr, jC), rho_new
         + sizeof(float4) + 2 * sizeof(float) + sizeof(int)         // diagnostics
         + sizeof(int);                                             // non-empty cell list
}

static bool h16_lists(const wcsph_sim_options& o) { return o.list_interval > 0 && o.precision == WCSPH_PREC_HALF2; }

static int64_t device_bytes(const wcsph_sim_options& o) {
  const int64_t list_bytes =
      o.list_interval > 0 ? (int64_t)(kListMax * 4 + 4 + 16 + (h16_lists(o) ? 20 : 0)) * o.max_particles : 0;
  return (int64_t)per_particle_bytes() * o.max_particles + list_bytes + 2 * sizeof(int) * o.max_cells +
         (sizeof(InstParams) + sizeof(InstDyn) + sizeof(int)) * (int64_t)o.max_instances + (int64_t)cub_sort_bytes(o.max_particles) +
         (1 << 20);
}

static int upload_tables(SimImpl& S) {
  WCSPH_CUDA(cudaMemcpyAsync(S.d_params, S.h_params.data(), sizeof(InstParams) * S.h_params.size(), cudaMemcpyHostToDevice,
                             S.s));
  WCSPH_CUDA(cudaMemcpyAsync(S.d_phase, S.h_phase.data(), sizeof(int) * S.h_phase.size(), cudaMemcpyHostToDevice, S.s));
  return 0;
}

// Instance-major key and cell spaces over the used slots.
static int rebuild_tables(SimImpl& S) {
  uint64_t key = 0;
  long long cells = 0;
  S.any_density = false;
  for (size_t k = 0; k < S.inst.size(); ++k) {
    HostInst& I = S.inst[k];
    InstParams& P = S.h_params[k];
    if (!I.active) {
      P.active = 0;
      continue;
    }
    P.key_base = (uint32_t)key;
    P.cell_base = (int)cells;
    key += (uint64_t)1 << (3 * I.bits);
    cells += (long long)I.ncell[0] * I.ncell[1] * I.ncell[2];
    if (I.desc.density_mode != WCSPH_DENSITY_CONTINUITY) S.any_density = true;
  }
  if (key >= 0xffffffffull) {
    set_error("cell key space of the active instances (%llu) exceeds 32 bits", (unsigned long long)key);
    return WCSPH_E_CAPACITY;
  }
  if (cells > S.opt.max_cells) {
    set_error("active instances need %lld cells, capacity is %lld", cells, (long long)S.opt.max_cells);
    return WCSPH_E_CAPACITY;
  }
  S.total_cells = cells;
  int bits = 1;
  while (bits < 32 && ((uint64_t)1 << bits) <= key) ++bits;  // DeadKey & mask must exceed every live key
  S.key_bits = bits;
  S.graph_dirty = true;
  return upload_tables(S);
}

static StepArgs make_args(SimImpl& S) {
  StepArgs a{};
  a.main = S.buf_main;
  a.alt = S.buf_alt;
  a.params = S.d_params;
  a.dyn = S.d_dyn;
  a.phase = S.d_phase;
  a.keys_in = S.keys_in;
  a.vals_in = S.vals_in;
  a.keys_out = S.keys_out;
  a.vals_out = S.vals_out;
  a.jr = S.jr;
  a.jC = S.jC;
  a.rho_new = S.rho_new;
  a.cell_start = S.cell_start;
  a.cell_end = S.cell_end;
  a.n_alive = S.d_n_alive;
  a.n_host = S.n_host;
  a.n_inst = (int)S.inst.size();
  a.pair_count = S.d_pairs;
  a.run_list = S.run_list;
  a.run_count = S.d_counters;
  a.dens_any = S.d_counters + 4;
  a.diag_acc = S.diag_acc;
  a.diag_dt = S.diag_dt;
  a.diag_nbr = S.diag_nbr;
  a.diag_rho = S.diag_rho;
  if (S.opt.list_interval > 0) {
    a.list = S.list;
    a.list_cnt = S.list_cnt;
    a.list_max = kListMax;
    a.list_flags = S.d_lflags;
    a.inst_motion = S.d_motion;
    a.inst_keep = S.d_keep;
    a.jh = S.jh;
    a.jpo = S.jpo;
    a.list_pad = list_pad_entry((int)S.opt.max_particles, h16_lists(S.opt));
  }
  return a;
}

// A pass was enqueued (captured passes are always launched right after): every removed instance's particles are dead after it.
static void mark_drained(SimImpl& S) {
  for (auto& I : S.inst)
    if (I.used && !I.active) I.drained = true;
}

constexpr int kBlock = 256;
static inline int nblk(long long n) { return (int)std::max<long long>(1, (n + kBlock - 1) / kBlock); }

// Enqueue one pass of the pipeline.  init_filter adds the initial Shepard
// filter after the hydro pass (main.cpp:75).  Returns the kernel-launch count.
// After k_step_begin ran with list_reuse set (the list-step prologue): the
// ranges the binning sets again, and the slot count of a binning pass.
__global__ void k_begin_build(StepArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < a.n_inst) {
    a.dyn[k].range_lo = 0x7fffffff;
    a.dyn[k].range_hi = 0;
  }
  if (k == 0) *a.n_alive = a.n_host;
}

static int enqueue_pass(SimImpl& S, StepArgs a, bool density, bool init_filter, int* launches,
                        cudaEvent_t* ev = nullptr, bool build_lists = false, bool after_prologue = false) {
  int L = 0;
  const int n = S.n_host;
  if (build_lists) a.x0 = S.x0;
  else S.lists_valid = false;  // any other pass re-sorts or changes what the lists refer to
  if (!after_prologue) a.inst_keep = nullptr;  // partial builds happen only in a list step's build branch
  if (after_prologue) {  // a list-mode build branch: the step has begun
    k_begin_build<<<nblk(std::max<int>(1, (int)S.inst.size())), kBlock, 0, S.s>>>(a);
  } else {
    if (ev) WCSPH_CUDA(cudaEventRecord(ev[0], S.s));
    WCSPH_CUDA(cudaMemsetAsync(S.d_counters + 4, 0, sizeof(int), S.s));
    k_step_begin<<<nblk(std::max<int>(1, (int)S.inst.size())), kBlock, 0, S.s>>>(a);
  }
  ++L;
  if (n > 0) {
    k_kick_bin<<<nblk(n), kBlock, 0, S.s>>>(a);
    ++L;
    size_t bytes = S.cub_bytes;
    WCSPH_CUDA(cub::DeviceRadixSort::SortPairs(S.cub_tmp, bytes, S.keys_in, S.keys_out, S.vals_in, S.vals_out, n, 0,
                                               S.key_bits, S.s));
    L += 2 * ((S.key_bits + 7) / 8) + 1;  // onesweep: histogram + one pass per digit (approximate)
    if (S.total_cells > 0) {
      WCSPH_CUDA(cudaMemsetAsync(S.cell_start, 0, sizeof(int) * S.total_cells, S.s));
      WCSPH_CUDA(cudaMemsetAsync(S.cell_end, 0, sizeof(int) * S.total_cells, S.s));
    }
    WCSPH_CUDA(cudaMemsetAsync(S.d_counters, 0, sizeof(int), S.s));
    k_permute<<<nblk(n), kBlock, 0, S.s>>>(a);
    ++L;
    if (ev) WCSPH_CUDA(cudaEventRecord(ev[1], S.s));
    // A list build scans first and takes its density pass from the lists
    // (every instance's are current after the scan: rebuilt or kept); the
    // scan reads positions only, and the EoS records it gathers do not enter
    // the lists.  Other passes search the cells for the density.
    if (density && !build_lists) {
      k_density_plain<<<nblk(n), kBlock, 0, S.s>>>(a);
      k_eos<<<nblk(n), kBlock, 0, S.s>>>(a);
      L += 2;
    }
    if (ev) WCSPH_CUDA(cudaEventRecord(ev[2], S.s));
    if (S.opt.precision == WCSPH_PREC_FP32) {
      k_hydro_plain<true><<<nblk(n), kBlock, 0, S.s>>>(a);
    } else if (build_lists) {  // the scan writes the lists, the list pass sums them
      const bool h16 = S.opt.precision == WCSPH_PREC_HALF2;
      if (int rc = h16 ? launch_hydro_tiled<true, true>(a, n, S.s, S.build_shape)
                       : launch_hydro_tiled<false, true>(a, n, S.s, S.build_shape))
        return rc;
      if (ev && S.scan_ev) WCSPH_CUDA(cudaEventRecord(S.scan_ev, S.s));
      if (density) {
        if (int rc = launch_density_list(a, n, S.s, h16)) return rc;
        StepArgs b = a;  // the particles whose list overflowed: the cell search
        b.density_overflow_only = 1;
        k_density_plain<<<nblk(n), kBlock, 0, S.s>>>(b);
        k_eos<<<nblk(n), kBlock, 0, S.s>>>(a);
        L += 3;
      }
      if (int rc = h16 ? launch_hydro_list<true>(a, n, S.s, S.list_shape)
                       : launch_hydro_list<false>(a, n, S.s, S.list_shape))
        return rc;
      ++L;
    } else if (S.opt.precision == WCSPH_PREC_TILED) {
      if (int rc = launch_hydro_tiled<false>(a, n, S.s, S.tile_shape)) return rc;
    } else {
      if (int rc = launch_hydro_tiled<true>(a, n, S.s, S.tile_shape)) return rc;
    }
    ++L;
    if (ev) WCSPH_CUDA(cudaEventRecord(ev[3], S.s));
    k_copy_dead<<<nblk(n), kBlock, 0, S.s>>>(a);
    ++L;
    if (init_filter) {
      StepArgs b = a;
      b.init_filter = 1;
      k_density_plain<<<nblk(n), kBlock, 0, S.s>>>(b);
      k_apply_init_filter<<<nblk(n), kBlock, 0, S.s>>>(b);
      L += 2;
    }
  }
  WCSPH_CUDA(cudaGetLastError());
  if (launches) *launches = L;
  mark_drained(S);
  S.appended = false;
  return 0;
}

// A step that reads the neighbour lists (sim_list.cuh): no sort, no scan.
// The list-step branch (the step has begun in the prologue).
// The list step.  When dens_body is given (capture of the list-step branch
// of the step graph, whose conditional handle dcond was created on that
// branch's graph), the density pass sits under a conditional node that
// k_kick_refresh opens only when some instance has a density pass due (most
// steps have none, and the two kernels would only return at once); the
// node's body is left in *dens_body for the caller to capture.
static int enqueue_reuse(SimImpl& S, StepArgs a, bool density, int* launches, cudaEvent_t* ev = nullptr,
                         cudaGraphConditionalHandle dcond = 0, cudaGraph_t* dens_body = nullptr) {
  const int n = S.n_host;
  a.list_reuse = 1;
  a.x0 = S.x0;    // read by k_kick_refresh (the displacement since the build)
  a.alt = a.main;  // in place: no re-sort, each particle's state is its own thread's
  int L = 0;
  if (n > 0) {
    const bool cond_density = density && dens_body;
    k_kick_refresh<<<nblk(n), kBlock, 0, S.s>>>(a, dcond, cond_density ? 1 : 0);
    ++L;
    if (ev) WCSPH_CUDA(cudaEventRecord(ev[1], S.s));
    if (cond_density) {
      cudaStreamCaptureStatus st;
      cudaGraph_t cg = nullptr;
      const cudaGraphNode_t* deps = nullptr;
      size_t ndeps = 0;
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = dcond;
      cp.conditional.type = cudaGraphCondTypeIf;
      cp.conditional.size = 1;
      cudaGraphNode_t node = nullptr;
      WCSPH_CUDA(cudaStreamGetCaptureInfo(S.s, &st, nullptr, &cg, &deps, &ndeps));
      WCSPH_CUDA(cudaGraphAddNode(&node, cg, deps, ndeps, &cp));
      WCSPH_CUDA(cudaStreamUpdateCaptureDependencies(S.s, &node, 1, cudaStreamSetCaptureDependencies));
      *dens_body = cp.conditional.phGraph_out[0];
    } else if (density) {  // the kernels return at once for instances with no density pass due
      if (int rc = launch_density_list(a, n, S.s, h16_lists(S.opt))) return rc;
      k_eos<<<nblk(n), kBlock, 0, S.s>>>(a);
      L += 2;
    }
    if (ev) WCSPH_CUDA(cudaEventRecord(ev[2], S.s));
    if (S.opt.precision == WCSPH_PREC_HALF2) {
      if (int rc = launch_hydro_list<true>(a, n, S.s, S.list_shape)) return rc;
    } else {
      if (int rc = launch_hydro_list<false>(a, n, S.s, S.list_shape)) return rc;
    }
    ++L;
    if (ev) WCSPH_CUDA(cudaEventRecord(ev[3], S.s));  // the dead tail stays in place
  }
  WCSPH_CUDA(cudaGetLastError());
  if (launches) *launches = L;
  return 0;
}

// The density pass of a list step (the body of enqueue_reuse's conditional node).
static int enqueue_list_density(SimImpl& S, StepArgs a) {
  const int n = S.n_host;
  a.list_reuse = 1;
  a.x0 = S.x0;
  a.alt = a.main;
  if (int rc = launch_density_list(a, n, S.s, h16_lists(S.opt))) return rc;
  k_eos<<<nblk(n), kBlock, 0, S.s>>>(a);
  WCSPH_CUDA(cudaGetLastError());
  return 0;
}

static int sync_compact(SimImpl& S) {
  WCSPH_CUDA(cudaStreamSynchronize(S.s));
  if (S.appended) return 0;  // no pass has counted the appended particles yet
  int n_alive = 0;
  WCSPH_CUDA(cudaMemcpy(&n_alive, S.d_n_alive, sizeof(int), cudaMemcpyDeviceToHost));
  if (n_alive != S.n_host) {
    S.n_host = n_alive;
    S.graph_dirty = true;
  }
  // Slots of removed instances whose particles a pass has already turned into
  // dead keys can be reused.
  for (auto& I : S.inst)
    if (I.used && !I.active && I.drained) I.used = false;
  return 0;
}



static int set_all_phases(SimImpl& S, int active_phase);

// Milliseconds of `reps` back-to-back launches of fn on the solver stream.
template <typename F>
static int time_launches(SimImpl& S, int reps, F&& fn, float* ms) {
  if (int rc = fn()) return rc;  // warm-up
  WCSPH_CUDA(cudaEventRecord(S.ev0, S.s));
  for (int r = 0; r < reps; ++r)
    if (int rc = fn()) return rc;
  WCSPH_CUDA(cudaEventRecord(S.ev1, S.s));
  WCSPH_CUDA(cudaEventSynchronize(S.ev1));
  WCSPH_CUDA(cudaEventElapsedTime(ms, S.ev0, S.ev1));
  return 0;
}

// Autotuner: on the live instance set, time every block shape of the tiled
// hydro kernel with probe passes (forces go to the diagnostic arrays, the
// state is untouched) and keep the fastest.  The candidates share their
// arithmetic exactly, so the choice never changes a result (an instance is
// bit-identical alone and in a mix).  Re-tuned only when the particle count
// crosses a power of two.
static int autotune(SimImpl& S) {
  if (!S.opt.autotune || S.opt.precision == WCSPH_PREC_FP32 || S.n_host <= 0) return 0;
  int bucket = 0;
  while ((1LL << bucket) < S.n_host) ++bucket;
  if (bucket == S.tuned_bucket) return 0;
  for (size_t q = 0; q < S.inst.size(); ++q) S.h_phase[q] = S.inst[q].active ? PH_PROBE : PH_IDLE;
  if (int rc = upload_tables(S)) return rc;
  StepArgs a = make_args(S);
  a.probe_density = 1;
  // one probe pass bins and sorts; repeated pair-kernel launches are then idempotent
  if (int rc = enqueue_pass(S, a, false, false, nullptr)) return rc;
  const int n = S.n_host;
  const bool h16 = S.opt.precision == WCSPH_PREC_HALF2;
  float best = 1e30f, ms = 0.f;
  int best_shape = 0;
  for (int v = 0; v < kTileShapes; ++v) {
    int rc = time_launches(S, 3, [&]() {
      return h16 ? launch_hydro_tiled<true>(a, n, S.s, v) : launch_hydro_tiled<false>(a, n, S.s, v);
    }, &ms);
    if (rc) return rc;
    if (ms < best) best = ms, best_shape = v;
  }
  S.tile_shape = best_shape;
  if (S.opt.list_interval > 0) {
    // The list pass: a probe build pass makes lists of the current state,
    // then every launch shape is timed on them with probe launches
    // (diagnostics only, state untouched).  The lists are dropped afterwards:
    // the first step builds its own, with the overflow and drift checks of a
    // step's build.
    if (int rc = enqueue_pass(S, a, false, false, nullptr, nullptr, true)) return rc;
    StepArgs b = make_args(S);
    b.list_reuse = 1;
    b.x0 = S.x0;
    b.alt = b.main;
    float best_list = 1e30f;
    const int fixed_list = S.opt.list_shape & 0xff, fixed_build = (S.opt.list_shape >> 8) & 0xff;
    int best_list_shape = fixed_list > 0 ? fixed_list - 1 : 0;
    for (int v = 0; v < kListShapes && fixed_list == 0; ++v) {
      int rc = time_launches(S, 3, [&]() {
        return h16 ? launch_hydro_list<true>(b, n, S.s, v) : launch_hydro_list<false>(b, n, S.s, v);
      }, &ms);
      if (rc) return rc;
      if (ms < best_list) best_list = ms, best_list_shape = v;
    }
    S.list_shape = best_list_shape;
    // the build's scan on the same sorted state (it rewrites the same lists)
    StepArgs c = a;
    c.x0 = S.x0;
    float best_build = 1e30f;
    int best_build_shape = fixed_build > 0 ? fixed_build - 1 : 0;
    for (int v = 0; v < kBuildShapes && fixed_build == 0; ++v) {
      int rc = time_launches(S, 3, [&]() {
        return h16 ? launch_hydro_tiled<true, true>(c, n, S.s, v) : launch_hydro_tiled<false, true>(c, n, S.s, v);
      }, &ms);
      if (rc) return rc;
      if (ms < best_build) best_build = ms, best_build_shape = v;
    }
    S.build_shape = best_build_shape;
    S.lists_valid = false;
    WCSPH_CUDA(cudaMemsetAsync(S.d_lflags + kLfOverflowPending, 0, sizeof(unsigned), S.s));
  }
  S.tuned_bucket = bucket;
  S.graph_dirty = true;
  return set_all_phases(S, PH_STEP);
}

static int set_all_phases(SimImpl& S, int active_phase) {
  for (size_t k = 0; k < S.inst.size(); ++k) S.h_phase[k] = S.inst[k].active ? active_phase : PH_IDLE;
  WCSPH_CUDA(cudaMemcpyAsync(S.d_phase, S.h_phase.data(), sizeof(int) * S.h_phase.size(), cudaMemcpyHostToDevice, S.s));
  return 0;
}

// H_cell: the smallest cell edge, the largest radius any neighbour scan of
// the instance uses (2h; the list radius 2h + skin with neighbour lists), so
// that the 27 cells around a particle's cell hold every particle within it.
static int fill_params(const wcsph_instance_desc& d, float H_cell, HostInst& I, InstParams& P) {
  if (d.n <= 0 || !(d.h > 0) || !(d.mass > 0) || !(d.rho0 > 0) || !(d.gamma > 0) || !(d.c0 > 0) || d.nu < 0) {
    set_error("instance: n, h, mass, rho0, gamma, c0 must be positive and nu >= 0");
    return WCSPH_E_INVALID;
  }
  if (d.density_mode < 0 || d.density_mode > 2 || (d.density_mode == 2 && d.shepard_interval <= 0)) {
    set_error("instance: bad density_mode %d / shepard_interval %d", d.density_mode, d.shepard_interval);
    return WCSPH_E_INVALID;
  }
  if (d.pair.vsig_mode < 0 || d.pair.vsig_mode > 1) {
    set_error("instance: bad vsig_mode %d", d.pair.vsig_mode);
    return WCSPH_E_INVALID;
  }
  P = InstParams{};
  const float H = 2.0f * (float)d.h;             // the support radius
  const float Hc = std::max(H_cell, H);          // the smallest cell edge
  for (int k = 0; k < 3; ++k) {
    const float ext = d.hi[k] - d.lo[k];
    if (!(ext > 0)) {
      set_error("instance: grid bounds must satisfy lo < hi on every axis");
      return WCSPH_E_INVALID;
    }
    int nc = (int)std::floor(ext / (Hc * 1.0001f));
    if (nc < 1) nc = 1;
    if (d.periodic && nc < 3) {
      set_error("instance: periodic box needs at least 3 cells of edge >= 2h (2h + skin with neighbour lists) per "
                "axis (got %d on axis %d)", nc, k);
      return WCSPH_E_INVALID;
    }
    if (nc > 1024) {
      set_error("instance: %d cells on axis %d exceed the 10-bit Morton limit (1024)", nc, k);
      return WCSPH_E_CAPACITY;
    }
    I.ncell[k] = nc;
    I.cell[k] = d.periodic ? ext / (float)nc : std::max(ext / (float)nc, Hc * 1.0001f);
    if (I.cell[k] < Hc) I.cell[k] = Hc * 1.0001f;
    P.lo[k] = d.lo[k];
    P.cell[k] = I.cell[k];
    P.inv_cell[k] = 1.0f / I.cell[k];
    P.ncell[k] = nc;
    P.L[k] = ext;
    P.halfL[k] = 0.5f * ext;
    P.kill_lo[k] = d.kill_lo[k];
    P.kill_hi[k] = d.kill_hi[k];
    if (d.kill_lo[k] < d.kill_hi[k]) P.kill_on = 1;
  }
  int m = std::max(I.ncell[0], std::max(I.ncell[1], I.ncell[2])) - 1;
  int bits = 0;
  while ((1 << bits) <= m) ++bits;
  I.bits = std::max(bits, 1);
  P.periodic = d.periodic;
  P.active = 1;
  P.density_mode = d.density_mode;
  P.shepard_interval = d.shepard_interval;
  P.vsig_mode = d.pair.vsig_mode;
  const double Hd = 2.0 * d.h;
  P.h = (float)d.h;
  P.H2 = H * H;
  P.inv_H = (float)(1.0 / Hd);
  P.Kw = (float)(16.0 / kPi / (Hd * Hd * Hd));
  P.Kg = (float)(16.0 / kPi / (Hd * Hd * Hd * Hd));
  P.W0 = 0.5f * P.Kw;
  P.mass = (float)d.mass;
  P.nu4 = (float)(4.0 * d.nu);
  P.eh2 = (float)(d.pair.eps * d.h * d.h);
  P.alpha = (float)d.pair.alpha;
  P.beta = (float)d.pair.beta;
  P.c_cfl = (float)d.pair.c_cfl;
  P.rho0 = (float)d.rho0;
  P.inv_rho0 = (float)(1.0 / d.rho0);
  const double B = d.c0 * d.c0 * d.rho0 / d.gamma;
  P.B = (float)B;
  P.gamma = (float)d.gamma;
  P.cs2_coef = (float)(B * d.gamma / d.rho0);
  P.c0 = (float)std::sqrt(B * d.gamma / d.rho0);
  P.rho_floor = (float)d.rho_floor;
  P.g = (float)d.g;
  P.dt_nu = d.nu > 0 ? (float)(0.125 * d.h * d.h / d.nu) : INFINITY;
  P.t_end = d.t_end;
  I.desc = d;
  I.n = d.n;
  return 0;
}

// ------------------------------------------------------- neighbour lists
// Sticky errors of the latest completed step, handled after draining the
// stream, so that they are seen and cleared exactly once.
static int read_list_flags(SimImpl& S) {
  volatile unsigned* h = S.h_lflags;
  if (h[kLfErr]) {
    WCSPH_CUDA(cudaStreamSynchronize(S.s));
    h[kLfErr] = 0u;
    WCSPH_CUDA(cudaMemsetAsync(S.d_lflags + kLfErr, 0, sizeof(unsigned), S.s));
    WCSPH_CUDA(cudaStreamSynchronize(S.s));
    S.lists_valid = false;
    set_error("wcsph_sim_step: a particle moved more than half the neighbour-list skin between list builds; "
              "the step's pair sums may be incomplete (raise list_skin or lower list_interval)");
    return WCSPH_E_STATE;
  }
  return 0;
}

// The prologue of a list-mode step: dt rotation (k_step_begin, keeping the
// build's order), then the device's build decision (k_list_set), which sets
// the condition `cond` when use_cond.
static int enqueue_list_prologue(SimImpl& S, const StepArgs& a0, cudaGraphConditionalHandle cond, bool use_cond,
                                 cudaEvent_t* ev) {
  StepArgs a = a0;
  a.list_reuse = 1;
  a.x0 = S.x0;
  if (ev) WCSPH_CUDA(cudaEventRecord(ev[0], S.s));
  WCSPH_CUDA(cudaMemsetAsync(S.d_pairs, 0, sizeof(unsigned long long), S.s));
  WCSPH_CUDA(cudaMemsetAsync(S.d_counters + 4, 0, sizeof(int), S.s));
  k_step_begin<<<nblk(std::max<int>(1, (int)S.inst.size())), kBlock, 0, S.s>>>(a);
  k_list_set<<<1, 1, 0, S.s>>>(a, S.opt.list_interval, cond, use_cond ? 1 : 0);
  WCSPH_CUDA(cudaGetLastError());
  return 0;
}

// One step in list mode.  Stale lists are marked for the device (kLfForce);
// the device decides whether the step builds.  At most two steps are in
// flight; the flags are read one step behind.
static int list_step(SimImpl& S, bool graph, cudaEvent_t* ev, bool* built = nullptr) {
  if (!S.lists_valid) {
    WCSPH_CUDA(cudaMemsetAsync(S.d_lflags + kLfForce, 0x01, sizeof(unsigned), S.s));
    S.lists_valid = true;
  }
  if (graph) {
    WCSPH_CUDA(cudaGraphLaunch(S.gexec, S.s));
  } else {
    StepArgs a = make_args(S);
    if (int rc = enqueue_list_prologue(S, a, 0, false, nullptr)) return rc;
    unsigned build = 0;
    WCSPH_CUDA(cudaMemcpyAsync(&build, S.d_lflags + kLfDecision, sizeof(unsigned), cudaMemcpyDeviceToHost, S.s));
    WCSPH_CUDA(cudaStreamSynchronize(S.s));
    if (built) *built = build != 0;
    if (ev) WCSPH_CUDA(cudaEventRecord(ev[0], S.s));  // after the host read of the decision
    const int rc = build ? enqueue_pass(S, a, S.any_density, false, &S.kernels_per_step, ev, true, true)
                         : enqueue_reuse(S, a, S.any_density, &S.kernels_reuse, ev);
    if (rc) return rc;
    WCSPH_CUDA(cudaMemcpyAsync(S.h_lflags, S.d_lflags, kLfWords * sizeof(unsigned), cudaMemcpyDeviceToHost, S.s));
  }
  const int par = (int)(S.steps_launched & 1);
  WCSPH_CUDA(cudaEventRecord(S.step_ev[par], S.s));
  ++S.steps_launched;
  if (S.steps_launched >= 2) {
    WCSPH_CUDA(cudaEventSynchronize(S.step_ev[par ^ 1]));
    return read_list_flags(S);
  }
  return 0;
}

// The list-mode step graph: the prologue, then a conditional node whose IF
// branch is a build step (binning, sort, scan-only tiled pass, list pass) and
// whose ELSE branch is a list step (kick and refresh in place, list passes),
// then the copy of the flags to the host.
static int capture_list_graph(SimImpl& S) {
  if (S.gexec) {
    cudaGraphExecDestroy(S.gexec);
    S.gexec = nullptr;
  }
  StepArgs a = make_args(S);
  cudaGraph_t g = nullptr;
  WCSPH_CUDA(cudaGraphCreate(&g, 0));
  auto fail = [&](int rc, const char* what) {
    cudaGraphDestroy(g);
    if (rc == WCSPH_E_CUDA || rc == 0) set_error("capturing the neighbour-list step graph failed (%s)", what);
    return rc ? rc : WCSPH_E_CUDA;
  };
  cudaGraphConditionalHandle cond;
  if (cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault) != cudaSuccess)
    return fail(WCSPH_E_CUDA, "conditional handle");
  const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
  if (cudaStreamBeginCaptureToGraph(S.s, g, nullptr, nullptr, 0, mode) != cudaSuccess)
    return fail(WCSPH_E_CUDA, "begin capture");
  int rc = enqueue_list_prologue(S, a, cond, true, nullptr);
  cudaGraphNodeParams cp = {};
  cudaGraphNode_t cnode = nullptr;
  if (!rc) {
    cudaStreamCaptureStatus st;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 2;  // IF: build; ELSE: list step
    if (cudaStreamGetCaptureInfo(S.s, &st, nullptr, &cg, &deps, &ndeps) != cudaSuccess ||
        cudaGraphAddNode(&cnode, cg, deps, ndeps, &cp) != cudaSuccess ||
        cudaStreamUpdateCaptureDependencies(S.s, &cnode, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
      rc = WCSPH_E_CUDA;
  }
  if (!rc && cudaMemcpyAsync(S.h_lflags, S.d_lflags, kLfWords * sizeof(unsigned), cudaMemcpyDeviceToHost, S.s) !=
                 cudaSuccess)
    rc = WCSPH_E_CUDA;
  cudaGraph_t out = nullptr;
  const cudaError_t e = cudaStreamEndCapture(S.s, &out);
  if (rc || e != cudaSuccess) return fail(rc, "prologue");
  // the list-step branch's own conditional (its density pass), set by k_kick_refresh
  cudaGraphConditionalHandle dcond = 0;
  if (S.any_density &&
      cudaGraphConditionalHandleCreate(&dcond, cp.conditional.phGraph_out[1], 0, cudaGraphCondAssignDefault) !=
          cudaSuccess)
    return fail(WCSPH_E_CUDA, "density conditional handle");
  for (int branch = 0; branch < 2; ++branch) {
    if (cudaStreamBeginCaptureToGraph(S.s, cp.conditional.phGraph_out[branch], nullptr, nullptr, 0, mode) !=
        cudaSuccess)
      return fail(WCSPH_E_CUDA, "begin branch capture");
    cudaGraph_t dens_body = nullptr;
    rc = branch == 0 ? enqueue_pass(S, a, S.any_density, false, &S.kernels_per_step, nullptr, true, true)
                     : enqueue_reuse(S, a, S.any_density, &S.kernels_reuse, nullptr, dcond,
                                     S.any_density ? &dens_body : nullptr);
    cudaGraph_t bo = nullptr;
    const cudaError_t eb = cudaStreamEndCapture(S.s, &bo);
    if (rc || eb != cudaSuccess) return fail(rc, branch == 0 ? "build branch" : "list-step branch");
    if (dens_body) {  // the list step's density pass, under its conditional node
      if (cudaStreamBeginCaptureToGraph(S.s, dens_body, nullptr, nullptr, 0, mode) != cudaSuccess)
        return fail(WCSPH_E_CUDA, "begin density capture");
      rc = enqueue_list_density(S, a);
      const cudaError_t ed = cudaStreamEndCapture(S.s, &bo);
      if (rc || ed != cudaSuccess) return fail(rc, "list-step density pass");
    }
  }
  const cudaError_t ei = cudaGraphInstantiate(&S.gexec, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate (list step)", __FILE__, __LINE__);
  S.kernels_per_step += 2;  // the prologue's kernels
  S.kernels_reuse += 2;
  S.graph_dirty = false;
  return 0;
}

}  // namespace wcsph

using namespace wcsph;

struct wcsph_sim {
  SimImpl impl;
};

extern "C" {

int64_t wcsph_sim_device_bytes(const wcsph_sim_options* opt) { return opt ? device_bytes(*opt) : -1; }

int wcsph_sim_create(const wcsph_sim_options* opt, wcsph_sim** out) {
  if (!opt || !out || opt->max_particles <= 0 || opt->max_particles > INT32_MAX - 1 || opt->max_cells <= 0 ||
      opt->max_cells > INT32_MAX || opt->max_instances <= 0 || opt->max_instances > (int)kInstMask ||
      opt->precision < 0 || opt->precision > 2 || opt->list_interval < 0 || !(opt->list_skin >= 0.f) ||
      opt->list_shape < 0 || (opt->list_shape & 0xff) > kListShapes || ((opt->list_shape >> 8) & 0xff) > kBuildShapes ||
      (opt->list_shape >> 16) != 0) {
    set_error("wcsph_sim_create: invalid options");
    return WCSPH_E_INVALID;
  }
  if (opt->list_interval > 0 && opt->precision == WCSPH_PREC_FP32) {
    set_error("wcsph_sim_create: neighbour lists need the tiled or half2 precision");
    return WCSPH_E_INVALID;
  }
  if (h16_lists(*opt) && opt->list_skin > 1.5f) {
    set_error("wcsph_sim_create: the half2 list pass keeps positions within one cell edge of the build cell's "
              "centre, which needs list_skin <= 1.5 h (got %g)", (double)opt->list_skin);
    return WCSPH_E_INVALID;
  }
  if (h16_lists(*opt) && opt->max_particles >= kMaxH16ListParticles) {
    set_error("wcsph_sim_create: half2 list entries hold the slot in %d bits: max_particles < %d (got %d)",
              kH16SlotBits, kMaxH16ListParticles, opt->max_particles);
    return WCSPH_E_INVALID;
  }
  int ndev = 0;
  WCSPH_CUDA(cudaGetDeviceCount(&ndev));
  if (opt->device < 0 || opt->device >= ndev) {
    set_error("wcsph_sim_create: device %d out of range (%d devices)", opt->device, ndev);
    return WCSPH_E_NODEVICE;
  }
  WCSPH_CUDA(cudaSetDevice(opt->device));
  auto* sim = new wcsph_sim();
  SimImpl& S = sim->impl;
  S.opt = *opt;
  S.list_shape = (opt->list_shape & 0xff) > 0 ? (opt->list_shape & 0xff) - 1 : 0;
  S.build_shape = ((opt->list_shape >> 8) & 0xff) > 0 ? ((opt->list_shape >> 8) & 0xff) - 1 : 0;
  auto fail = [&](int rc) {
    for (void* p : S.allocs) cudaFree(p);
    if (S.s) cudaStreamDestroy(S.s);
    delete sim;
    return rc;
  };
  if (cudaStreamCreateWithFlags(&S.s, cudaStreamNonBlocking) != cudaSuccess) return fail(WCSPH_E_CUDA);
  const size_t N = (size_t)opt->max_particles + 1;
  int rc = 0;
  for (SimArrays* A : {&S.buf_main, &S.buf_alt}) {
    rc |= alloc(S, (void**)&A->pos, N * sizeof(float4));
    rc |= alloc(S, (void**)&A->vel, N * sizeof(float4));
    rc |= alloc(S, (void**)&A->vh, N * sizeof(float4));
    rc |= alloc(S, (void**)&A->acc, N * sizeof(float4));
    rc |= alloc(S, (void**)&A->pid, N * sizeof(int));
    rc |= alloc(S, (void**)&A->flags, N * sizeof(uint32_t));
  }
  rc |= alloc(S, (void**)&S.keys_in, N * sizeof(uint32_t));
  rc |= alloc(S, (void**)&S.keys_out, N * sizeof(uint32_t));
  rc |= alloc(S, (void**)&S.vals_in, N * sizeof(int));
  rc |= alloc(S, (void**)&S.vals_out, N * sizeof(int));
  rc |= alloc(S, (void**)&S.jr, N * sizeof(JRec));
  rc |= alloc(S, (void**)&S.jC, N * sizeof(float));
  rc |= alloc(S, (void**)&S.rho_new, N * sizeof(float));
  rc |= alloc(S, (void**)&S.diag_acc, N * sizeof(float4));
  rc |= alloc(S, (void**)&S.diag_dt, N * sizeof(float));
  rc |= alloc(S, (void**)&S.diag_rho, N * sizeof(float));
  rc |= alloc(S, (void**)&S.diag_nbr, N * sizeof(int));
  rc |= alloc(S, (void**)&S.cell_start, (size_t)opt->max_cells * sizeof(int));
  rc |= alloc(S, (void**)&S.cell_end, (size_t)opt->max_cells * sizeof(int));
  rc |= alloc(S, (void**)&S.d_params, (size_t)opt->max_instances * sizeof(InstParams));
  rc |= alloc(S, (void**)&S.d_dyn, (size_t)opt->max_instances * sizeof(InstDyn));
  rc |= alloc(S, (void**)&S.d_phase, (size_t)opt->max_instances * sizeof(int));
  rc |= alloc(S, (void**)&S.d_n_alive, sizeof(int));
  rc |= alloc(S, (void**)&S.run_list, N * sizeof(int));
  rc |= alloc(S, (void**)&S.d_counters, 8 * sizeof(int));
  rc |= alloc(S, (void**)&S.d_pairs, sizeof(unsigned long long));
  rc |= alloc(S, (void**)&S.d_cons, 8 * sizeof(double));
  S.cub_bytes = cub_sort_bytes((long long)N);
  rc |= alloc(S, &S.cub_tmp, S.cub_bytes);
  if (opt->list_interval > 0) {
    rc |= alloc(S, (void**)&S.list, N * kListMax * sizeof(uint32_t));
    rc |= alloc(S, (void**)&S.list_cnt, N * sizeof(int));
    rc |= alloc(S, (void**)&S.x0, N * sizeof(float4));
    rc |= alloc(S, (void**)&S.d_lflags, kLfWords * sizeof(unsigned));
    rc |= alloc(S, (void**)&S.d_motion, 3 * (size_t)opt->max_instances * sizeof(unsigned));
    rc |= alloc(S, (void**)&S.d_keep, (size_t)opt->max_instances * sizeof(int));
    if (h16_lists(*opt)) {
      rc |= alloc(S, (void**)&S.jh, N * sizeof(uint4));
      rc |= alloc(S, (void**)&S.jpo, N * sizeof(float));
    }
    if (!rc && cudaHostAlloc((void**)&S.h_lflags, kLfWords * sizeof(unsigned), cudaHostAllocDefault) != cudaSuccess)
      rc = 1;
  }
  if (rc) {
    if (S.h_lflags) cudaFreeHost(S.h_lflags);
    return fail(WCSPH_E_NOMEM);
  }
  if (cudaMemsetAsync(S.d_dyn, 0, (size_t)opt->max_instances * sizeof(InstDyn), S.s) != cudaSuccess ||
      cudaMemsetAsync(S.d_n_alive, 0, sizeof(int), S.s) != cudaSuccess ||
      cudaMemsetAsync(S.d_pairs, 0, sizeof(unsigned long long), S.s) != cudaSuccess ||
      cudaEventCreate(&S.ev0) != cudaSuccess || cudaEventCreate(&S.ev1) != cudaSuccess ||
      cudaEventCreateWithFlags(&S.step_ev[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&S.step_ev[1], cudaEventDisableTiming) != cudaSuccess)
    return fail(WCSPH_E_CUDA);
  if (S.d_lflags) {
    k_list_pad_slot<<<1, 1, 0, S.s>>>(S.jr, S.jC, S.jpo, S.jh, (int)opt->max_particles);
    if (cudaGetLastError() != cudaSuccess) return fail(WCSPH_E_CUDA);
    memset(S.h_lflags, 0, kLfWords * sizeof(unsigned));
    if (cudaMemsetAsync(S.d_lflags, 0, kLfWords * sizeof(unsigned), S.s) != cudaSuccess ||
        cudaMemsetAsync(S.d_motion, 0, 3 * (size_t)opt->max_instances * sizeof(unsigned), S.s) != cudaSuccess ||
        cudaMemsetAsync(S.d_keep, 0, (size_t)opt->max_instances * sizeof(int), S.s) != cudaSuccess)
      return fail(WCSPH_E_CUDA);
  }
  *out = sim;
  return 0;
}

int wcsph_sim_destroy(wcsph_sim* sim) {
  if (!sim) return 0;
  SimImpl& S = sim->impl;
  cudaSetDevice(S.opt.device);
  cudaStreamSynchronize(S.s);
  if (S.gexec) cudaGraphExecDestroy(S.gexec);
  for (void* p : S.allocs) cudaFree(p);
  if (S.h_lflags) cudaFreeHost(S.h_lflags);
  for (cudaEvent_t e : S.step_ev)
    if (e) cudaEventDestroy(e);
  cudaEventDestroy(S.ev0);
  cudaEventDestroy(S.ev1);
  cudaStreamDestroy(S.s);
  delete sim;
  return 0;
}

}  // extern "C"

namespace wcsph {

// The initial force pass (main.cpp:69-78) of instance k alone.
static int init_force_pass(SimImpl& S, int k) {
  const wcsph_instance_desc& d = S.inst[k].desc;
  for (size_t q = 0; q < S.inst.size(); ++q) S.h_phase[q] = PH_IDLE;
  S.h_phase[k] = PH_INIT;
  if (int rc = upload_tables(S)) return rc;
  StepArgs a = make_args(S);
  WCSPH_CUDA(cudaMemsetAsync(S.d_pairs, 0, sizeof(unsigned long long), S.s));  // last_pairs: this pass
  if (int rc = enqueue_pass(S, a, d.density_mode == WCSPH_DENSITY_SUMMATION, d.density_mode == WCSPH_DENSITY_SHEPARD,
                            nullptr))
    return rc;
  if (int rc = set_all_phases(S, PH_STEP)) return rc;
  WCSPH_CUDA(cudaStreamSynchronize(S.s));
  S.graph_dirty = true;
  return 0;
}

// What an appended instance brings.  Particle q of the storage sequence is
// particle ids[q] with its data at index q (slab), or particle order[q] with
// its data at index order[q] (restart), or particle q (default).
struct AppendSpec {
  const wcsph_instance_desc* desc = nullptr;
  int count = 0;
  const int32_t* ids = nullptr;
  const int32_t* order = nullptr;
  const float *pos3 = nullptr, *vel3 = nullptr, *dens = nullptr, *acc3 = nullptr, *div_v = nullptr;
  const int32_t *type = nullptr, *alive = nullptr;
  const InstDyn* saved = nullptr;  // restart state, else a fresh instance
  enum After { INIT_PASS, BIN_PASS, NO_PASS } after = INIT_PASS;
  const wcsph_slab* slab = nullptr;
};

// Append an instance's particles at [n_host, n_host + count) and register it,
// then run its initial force pass, or one pass with every instance idle that
// only bins (restart), or nothing (slab: the ghost layer comes first).
static int append_instance(SimImpl& S, const AppendSpec& A, int32_t* slot) {
  const wcsph_instance_desc* desc = A.desc;
  const int n = A.count;
  if (int rc = sync_compact(S)) return rc;
  bool draining = false;
  for (auto& I : S.inst) draining |= I.used && !I.active;
  if ((long long)S.n_host + n > S.opt.max_particles && draining) {
    // Removed instances still hold slots: run one pass with every instance
    // idle so their particles become dead keys, then compact.
    for (size_t q = 0; q < S.inst.size(); ++q) S.h_phase[q] = PH_IDLE;
    if (int rc = upload_tables(S)) return rc;
    if (int rc = enqueue_pass(S, make_args(S), false, false, nullptr)) return rc;
    if (int rc = set_all_phases(S, PH_STEP)) return rc;
    if (int rc = sync_compact(S)) return rc;
  }
  if ((long long)S.n_host + n > S.opt.max_particles) {
    set_error("adding an instance: %d + %d particles exceed capacity %lld", S.n_host, n,
              (long long)S.opt.max_particles);
    return WCSPH_E_CAPACITY;
  }
  int k = -1;
  for (size_t q = 0; q < S.inst.size(); ++q)
    if (!S.inst[q].used) {
      k = (int)q;
      break;
    }
  if (k < 0) {
    if ((int)S.inst.size() >= S.opt.max_instances) {
      set_error("adding an instance: all %d instance slots are in use", S.opt.max_instances);
      return WCSPH_E_CAPACITY;
    }
    k = (int)S.inst.size();
    S.inst.emplace_back();
    S.h_params.emplace_back();
    S.h_phase.push_back(PH_IDLE);
  }
  HostInst I;
  InstParams P;
  wcsph_instance_desc d = *desc;
  float W = 0.f;
  if (A.slab) {
    // The slab's grid covers its range and the ghost layers beyond its faces.
    const wcsph_slab& sl = *A.slab;
    W = wcsph_slab_layer_width(d.h, sl.margin);
    if (sl.has_left) d.lo[0] = std::max(d.lo[0], sl.x_lo - W - sl.margin);
    if (sl.has_right) d.hi[0] = std::min(d.hi[0], sl.x_hi + W + sl.margin);
  }
  const float H_cell = 2.0f * (float)d.h + (S.opt.list_interval > 0 ? list_skin(S.opt) * (float)d.h : 0.0f);
  if (int rc = fill_params(d, H_cell, I, P)) return rc;
  if (A.slab) {
    const wcsph_slab& sl = *A.slab;
    I.slab = true;
    I.geom = SlabGeom{sl.x_lo, sl.x_hi, W, sl.has_left ? 1 : 0, sl.has_right ? 1 : 0};
    P.slab_margin2 = sl.margin * sl.margin;
  }
  if (S.opt.list_interval > 0) {
    const float skin = list_skin(S.opt) * (float)d.h, R = 2.0f * (float)d.h + skin;
    P.HL2 = R * R;
    P.inv_skin = 1.0f / skin;
    // Half2 list pass: a rebuilt displacement coordinate is off by at most
    // half a 2^-15 step of the cell edge plus the rounding of the two FP32
    // cell centres; doubled for margin, the squared distance near (2h)^2 is
    // then within band of the exact FP32 value.
    float delta = 0.f;
    for (int k = 0; k < 3; ++k) {
      const float big = std::max(std::fabs(d.lo[k]), std::fabs(d.hi[k])) + 2.0f * I.cell[k];
      const float ulp = std::nextafter(big, INFINITY) - big;
      delta = std::max(delta, 2.0f * (I.cell[k] / 65536.0f + 2.0f * ulp));
    }
    const float H = 2.0f * (float)d.h, H2 = H * H;
    P.h16_band = 4.0f * H * 1.7320508f * delta + 3.0f * delta * delta + 16.0f * (std::nextafter(H2, INFINITY) - H2);
  }
  I.used = I.active = true;
  HostInst prev = S.inst[k];
  InstParams prev_p = S.h_params[k];
  S.inst[k] = I;
  S.h_params[k] = P;
  if (int rc = rebuild_tables(S)) {
    S.inst[k] = prev;
    S.h_params[k] = prev_p;
    rebuild_tables(S);
    return rc;
  }
  const int base = S.n_host;
  std::vector<float4> pos(n), vel(n), acc(n, make_float4(0, 0, 0, 0));
  std::vector<int> pid(n);
  std::vector<uint32_t> flags(n);
  for (int q = 0; q < n; ++q) {
    const int id = A.ids ? A.ids[q] : (A.order ? A.order[q] : q);
    const int i = A.ids ? q : id;  // index of the particle's data in the input arrays
    pos[q] = make_float4(A.pos3[3 * i], A.pos3[3 * i + 1], A.pos3[3 * i + 2], A.dens[i]);
    vel[q] = make_float4(A.vel3[3 * i], A.vel3[3 * i + 1], A.vel3[3 * i + 2], 0.f);
    if (A.acc3)
      acc[q] = make_float4(A.acc3[3 * i], A.acc3[3 * i + 1], A.acc3[3 * i + 2], A.div_v ? A.div_v[i] : 0.f);
    pid[q] = id;
    flags[q] = (uint32_t)k | (A.type[i] == WCSPH_FREEZE ? kFreezeBit : 0u) | (A.alive && !A.alive[i] ? kDeadBit : 0u);
  }
  if (n > 0) {
    WCSPH_CUDA(cudaMemcpyAsync(S.buf_main.pos + base, pos.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, S.s));
    WCSPH_CUDA(cudaMemcpyAsync(S.buf_main.vel + base, vel.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, S.s));
    WCSPH_CUDA(cudaMemcpyAsync(S.buf_main.acc + base, acc.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, S.s));
    WCSPH_CUDA(cudaMemcpyAsync(S.buf_main.pid + base, pid.data(), sizeof(int) * n, cudaMemcpyHostToDevice, S.s));
    WCSPH_CUDA(
        cudaMemcpyAsync(S.buf_main.flags + base, flags.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, S.s));
  }
  InstDyn dyn{};
  dyn.dt_next_bits = 0x7f800000u;
  if (A.saved) dyn = *A.saved;
  {  // velocity quantum of the compact records until the list passes bound the motion (k_list_set)
    float vmax = 0.f;
    for (int q = 0; q < n; ++q)
      vmax = std::max(vmax, std::max(std::fabs(vel[q].x), std::max(std::fabs(vel[q].y), std::fabs(vel[q].z))));
    dyn.vq = host_velocity_quantum(2.0f * vmax, (float)desc->c0);
  }
  WCSPH_CUDA(cudaMemcpyAsync(S.d_dyn + k, &dyn, sizeof(InstDyn), cudaMemcpyHostToDevice, S.s));
  S.n_host = base + n;
  S.appended = true;
  S.lists_valid = false;
  if (slot) *slot = k;
  if (A.after == AppendSpec::INIT_PASS) return init_force_pass(S, k);
  if (A.after == AppendSpec::BIN_PASS) {
    // One pass with every instance idle bins the restored particles (their
    // keys come from the saved positions, so a saved sorted order stays as
    // it is) and sets the instance's range; no state changes.
    for (size_t q = 0; q < S.inst.size(); ++q) S.h_phase[q] = PH_IDLE;
    if (int rc = upload_tables(S)) return rc;
    if (int rc = enqueue_pass(S, make_args(S), false, false, nullptr)) return rc;
    if (int rc = set_all_phases(S, PH_STEP)) return rc;
  }
  WCSPH_CUDA(cudaStreamSynchronize(S.s));
  S.graph_dirty = true;
  return 0;
}

}  // namespace wcsph

extern "C" {

int wcsph_sim_add_instance(wcsph_sim* sim, const wcsph_instance_desc* desc, const float* pos3, const float* vel3,
                           const float* dens, const int32_t* type, int32_t* slot) {
  if (!sim || !desc || !pos3 || !vel3 || !dens || !type) {
    set_error("wcsph_sim_add_instance: null argument");
    return WCSPH_E_INVALID;
  }
  WCSPH_CUDA(cudaSetDevice(sim->impl.opt.device));
  AppendSpec A;
  A.desc = desc;
  A.count = desc->n;
  A.pos3 = pos3, A.vel3 = vel3, A.dens = dens, A.type = type;
  return append_instance(sim->impl, A, slot);
}

int wcsph_sim_restore_instance(wcsph_sim* sim, const wcsph_instance_desc* desc, const float* pos3, const float* vel3,
                               const float* dens, const int32_t* type, const float* acc3, const float* div_v,
                               const int32_t* alive, const int32_t* order, double time, int64_t steps,
                               float dt_next, int32_t* slot) {
  if (!sim || !desc || !pos3 || !vel3 || !dens || !type || !acc3 || !div_v || !(dt_next > 0.f) || time < 0.0 ||
      steps < 0 || desc->n <= 0) {
    set_error("wcsph_sim_restore_instance: null argument, empty instance, non-positive dt_next or negative time");
    return WCSPH_E_INVALID;
  }
  if (order) {
    std::vector<char> seen(desc->n, 0);
    for (int q = 0; q < desc->n; ++q) {
      if (order[q] < 0 || order[q] >= desc->n || seen[order[q]]) {
        set_error("wcsph_sim_restore_instance: order is not a permutation of 0..%d (entry %d)", desc->n - 1, q);
        return WCSPH_E_INVALID;
      }
      seen[order[q]] = 1;
    }
  }
  WCSPH_CUDA(cudaSetDevice(sim->impl.opt.device));
  InstDyn dyn{};
  dyn.time = time;
  dyn.steps = steps;
  memcpy(&dyn.dt_next_bits, &dt_next, sizeof(float));
  dyn.finished = (desc->t_end > 0.0 && time >= desc->t_end) ? 1 : 0;
  dyn.range_lo = 0x7fffffff;
  AppendSpec A;
  A.desc = desc;
  A.count = desc->n;
  A.order = order;
  A.pos3 = pos3, A.vel3 = vel3, A.dens = dens, A.type = type, A.acc3 = acc3, A.div_v = div_v, A.alive = alive;
  A.saved = &dyn;
  A.after = AppendSpec::BIN_PASS;
  return append_instance(sim->impl, A, slot);
}

int wcsph_sim_next_dt(wcsph_sim* sim, int32_t slot, float* dt_next) {
  if (!sim || !dt_next) return WCSPH_E_INVALID;
  SimImpl& S = sim->impl;
  if (slot < 0 || slot >= (int)S.inst.size() || !S.inst[slot].used) {
    set_error("wcsph_sim_next_dt: slot %d is not in use", slot);
    return WCSPH_E_INVALID;
  }
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  WCSPH_CUDA(cudaStreamSynchronize(S.s));
  InstDyn d;
  WCSPH_CUDA(cudaMemcpy(&d, S.d_dyn + slot, sizeof(InstDyn), cudaMemcpyDeviceToHost));
  memcpy(dt_next, &d.dt_next_bits, sizeof(float));
  return 0;
}

int wcsph_sim_set_next_dt(wcsph_sim* sim, int32_t slot, float dt_next) {
  if (!sim || !(dt_next > 0.f)) {
    set_error("wcsph_sim_set_next_dt: dt_next must be positive");
    return WCSPH_E_INVALID;
  }
  SimImpl& S = sim->impl;
  if (slot < 0 || slot >= (int)S.inst.size() || !S.inst[slot].active) {
    set_error("wcsph_sim_set_next_dt: slot %d is not active", slot);
    return WCSPH_E_INVALID;
  }
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  unsigned bits;
  memcpy(&bits, &dt_next, sizeof(bits));
  static_assert(offsetof(InstDyn, dt_next_bits) % 4 == 0, "dt_next_bits alignment");
  WCSPH_CUDA(cudaMemcpyAsync((char*)(S.d_dyn + slot) + offsetof(InstDyn, dt_next_bits), &bits, sizeof(bits),
                             cudaMemcpyHostToDevice, S.s));
  WCSPH_CUDA(cudaStreamSynchronize(S.s));
  return 0;
}

int wcsph_sim_force_pass(wcsph_sim* sim, int32_t slot) {
  if (!sim) return WCSPH_E_INVALID;
  SimImpl& S = sim->impl;
  if (slot < 0 || slot >= (int)S.inst.size() || !S.inst[slot].active) {
    set_error("wcsph_sim_force_pass: slot %d is not active", slot);
    return WCSPH_E_INVALID;
  }
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  return init_force_pass(S, slot);
}

float wcsph_slab_layer_width(double h, float margin) {
  return (float)(2.0 * (2.0 * h) * 1.0001) + 2.0f * margin;
}

int wcsph_sim_add_slab(wcsph_sim* sim, const wcsph_instance_desc* desc, const wcsph_slab* slab, int32_t count,
                       const int32_t* ids, const float* pos3, const float* vel3, const float* dens,
                       const int32_t* type, int32_t* slot) {
  if (!sim || !desc || !slab || count < 0 || (count > 0 && (!ids || !pos3 || !vel3 || !dens || !type))) {
    set_error("wcsph_sim_add_slab: null argument or negative count");
    return WCSPH_E_INVALID;
  }
  if (desc->periodic) {
    set_error("wcsph_sim_add_slab: slabs along a periodic x axis are not supported");
    return WCSPH_E_INVALID;
  }
  const float W = wcsph_slab_layer_width(desc->h, slab->margin);
  const float lo = slab->has_left ? slab->x_lo : desc->lo[0], hi = slab->has_right ? slab->x_hi : desc->hi[0];
  if (!(slab->margin > 0.f) || !(hi > lo) || ((slab->has_left || slab->has_right) && hi - lo < 2.0f * W)) {
    set_error("wcsph_sim_add_slab: need margin > 0 and a slab at least twice the ghost layer (%g) wide", W);
    return WCSPH_E_INVALID;
  }
  for (int q = 0; q < count; ++q)
    if (ids[q] < 0 || ids[q] >= desc->n) {
      set_error("wcsph_sim_add_slab: id %d at %d outside [0, %d)", ids[q], q, desc->n);
      return WCSPH_E_INVALID;
    }
  WCSPH_CUDA(cudaSetDevice(sim->impl.opt.device));
  AppendSpec A;
  A.desc = desc;
  A.count = count;
  A.ids = ids;
  A.pos3 = pos3, A.vel3 = vel3, A.dens = dens, A.type = type;
  A.after = AppendSpec::NO_PASS;
  A.slab = slab;
  return append_instance(sim->impl, A, slot);
}

int wcsph_sim_slab_pack(wcsph_sim* sim, int32_t slot, void* send, int64_t capacity, int32_t counts[4]) {
  if (!sim || !counts || capacity < 0 || (capacity > 0 && !send)) return WCSPH_E_INVALID;
  SimImpl& S = sim->impl;
  if (slot < 0 || slot >= (int)S.inst.size() || !S.inst[slot].active || !S.inst[slot].slab) {
    set_error("wcsph_sim_slab_pack: slot %d is not an active slab", slot);
    return WCSPH_E_INVALID;
  }
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  if (int rc = sync_compact(S)) return rc;
  InstDyn d;
  WCSPH_CUDA(cudaMemcpy(&d, S.d_dyn + slot, sizeof(InstDyn), cudaMemcpyDeviceToHost));
  if (d.errors & kErrDrift) {
    set_error("wcsph_sim_slab_pack: a particle drifted farther than the slab margin (%g) in one step",
              (double)std::sqrt(S.h_params[slot].slab_margin2));
    return WCSPH_E_STATE;
  }
  const int n = S.n_host;
  const SlabGeom G = S.inst[slot].geom;
  S.lists_valid = false;
  int h_counts[4] = {0, 0, 0, 0};
  if (n > 0) {
    // class keys and indices in the step's sort buffers (free between passes)
    WCSPH_CUDA(cudaMemsetAsync(S.d_counters, 0, 4 * sizeof(int), S.s));
    k_slab_classify<<<nblk(n), kBlock, 0, S.s>>>(S.buf_main, n, slot, G, S.keys_in, S.vals_in, S.d_counters);
    WCSPH_CUDA(cudaGetLastError());
    size_t need = 0;
    WCSPH_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, need, S.keys_in, S.keys_out, S.vals_in, S.vals_out, n, 0,
                                               kSlabClassBits, S.s));
    if (need > S.cub_bytes) {
      set_error("wcsph_sim_slab_pack: sort scratch %zu B exceeds %zu B", need, S.cub_bytes);
      return WCSPH_E_CAPACITY;
    }
    size_t bytes = S.cub_bytes;
    WCSPH_CUDA(cub::DeviceRadixSort::SortPairs(S.cub_tmp, bytes, S.keys_in, S.keys_out, S.vals_in, S.vals_out, n, 0,
                                               kSlabClassBits, S.s));
    WCSPH_CUDA(cudaMemcpyAsync(h_counts, S.d_counters, sizeof(h_counts), cudaMemcpyDeviceToHost, S.s));
    WCSPH_CUDA(cudaStreamSynchronize(S.s));
  }
  const long long total = (long long)h_counts[0] + h_counts[1] + h_counts[2] + h_counts[3];
  if (total > capacity) {
    set_error("wcsph_sim_slab_pack: %lld records exceed the send buffer (%lld)", total, (long long)capacity);
    return WCSPH_E_CAPACITY;
  }
  if (total > 0) {
    k_slab_pack<<<nblk(total), kBlock, 0, S.s>>>(S.buf_main, S.vals_out, (int)total, (SlabRecord*)send);
    WCSPH_CUDA(cudaGetLastError());
  }
  if (n > 0) {
    k_slab_commit<<<nblk(n), kBlock, 0, S.s>>>(S.buf_main, n, slot, G);
    WCSPH_CUDA(cudaGetLastError());
  }
  WCSPH_CUDA(cudaStreamSynchronize(S.s));
  for (int c = 0; c < 4; ++c) counts[c] = h_counts[c];
  return 0;
}

int wcsph_sim_slab_unpack(wcsph_sim* sim, int32_t slot, const void* recv, int32_t n_owned, int32_t n_ghost) {
  if (!sim || n_owned < 0 || n_ghost < 0 || (n_owned + n_ghost > 0 && !recv)) return WCSPH_E_INVALID;
  SimImpl& S = sim->impl;
  if (slot < 0 || slot >= (int)S.inst.size() || !S.inst[slot].active || !S.inst[slot].slab) {
    set_error("wcsph_sim_slab_unpack: slot %d is not an active slab", slot);
    return WCSPH_E_INVALID;
  }
  const long long m = (long long)n_owned + n_ghost;
  if (S.n_host + m > S.opt.max_particles) {
    set_error("wcsph_sim_slab_unpack: %d + %lld particles exceed capacity %lld", S.n_host, m,
              (long long)S.opt.max_particles);
    return WCSPH_E_CAPACITY;
  }
  if (m == 0) return 0;
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  k_slab_unpack<<<nblk(m), kBlock, 0, S.s>>>(S.buf_main, S.n_host, (int)m, n_owned, slot, (const SlabRecord*)recv);
  WCSPH_CUDA(cudaGetLastError());
  WCSPH_CUDA(cudaStreamSynchronize(S.s));
  S.n_host += (int)m;
  S.appended = true;
  S.lists_valid = false;
  S.graph_dirty = true;
  return 0;
}

int wcsph_sim_remove_instance(wcsph_sim* sim, int32_t slot) {
  if (!sim) return WCSPH_E_INVALID;
  SimImpl& S = sim->impl;
  if (slot < 0 || slot >= (int)S.inst.size() || !S.inst[slot].active) {
    set_error("wcsph_sim_remove_instance: slot %d is not active", slot);
    return WCSPH_E_INVALID;
  }
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  S.inst[slot].active = false;  // particles are marked dead by the next binning
  S.inst[slot].drained = false;
  S.lists_valid = false;
  S.h_phase[slot] = PH_IDLE;
  return rebuild_tables(S);
}

int wcsph_sim_step(wcsph_sim* sim, int32_t nsteps) {
  if (!sim || nsteps < 0) return WCSPH_E_INVALID;
  SimImpl& S = sim->impl;
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  if (nsteps == 0) return 0;
  if (S.opt.list_interval > 0) {
    if (S.opt.use_graph && (S.graph_dirty || !S.gexec)) {
      if (int rc = autotune(S)) return rc;
      if (int rc = capture_list_graph(S)) return rc;
    }
    for (int t = 0; t < nsteps; ++t)
      if (int rc = list_step(S, S.opt.use_graph != 0, nullptr)) return rc;
    mark_drained(S);
    return 0;
  }
  StepArgs a = make_args(S);
  if (!S.opt.use_graph) {
    WCSPH_CUDA(cudaMemsetAsync(S.d_pairs, 0, sizeof(unsigned long long), S.s));
    for (int t = 0; t < nsteps; ++t) {
      if (t == nsteps - 1) WCSPH_CUDA(cudaMemsetAsync(S.d_pairs, 0, sizeof(unsigned long long), S.s));
      if (int rc = enqueue_pass(S, a, S.any_density, false, &S.kernels_per_step)) return rc;
    }
    return 0;
  }
  if (S.graph_dirty || !S.gexec) {
    if (int rc = autotune(S)) return rc;
    a = make_args(S);
    if (S.gexec) {
      cudaGraphExecDestroy(S.gexec);
      S.gexec = nullptr;
    }
    cudaGraph_t g;
    WCSPH_CUDA(cudaStreamBeginCapture(S.s, cudaStreamCaptureModeThreadLocal));
    WCSPH_CUDA(cudaMemsetAsync(S.d_pairs, 0, sizeof(unsigned long long), S.s));
    int rc = enqueue_pass(S, a, S.any_density, false, &S.kernels_per_step);
    cudaError_t e = cudaStreamEndCapture(S.s, &g);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture", __FILE__, __LINE__);
    e = cudaGraphInstantiate(&S.gexec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate", __FILE__, __LINE__);
    S.graph_dirty = false;
  }
  for (int t = 0; t < nsteps; ++t) WCSPH_CUDA(cudaGraphLaunch(S.gexec, S.s));
  mark_drained(S);
  return 0;
}

int wcsph_sim_synchronize(wcsph_sim* sim) {
  if (!sim) return WCSPH_E_INVALID;
  WCSPH_CUDA(cudaSetDevice(sim->impl.opt.device));
  WCSPH_CUDA(cudaStreamSynchronize(sim->impl.s));
  return 0;
}

int wcsph_sim_instance_status(wcsph_sim* sim, int32_t slot, double* time, int64_t* steps, int32_t* n_alive,
                              int32_t* finished) {
  if (!sim) return WCSPH_E_INVALID;
  SimImpl& S = sim->impl;
  if (slot < 0 || slot >= (int)S.inst.size() || !S.inst[slot].used) {
    set_error("wcsph_sim_instance_status: slot %d is not in use", slot);
    return WCSPH_E_INVALID;
  }
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  WCSPH_CUDA(cudaStreamSynchronize(S.s));
  InstDyn d;
  WCSPH_CUDA(cudaMemcpy(&d, S.d_dyn + slot, sizeof(InstDyn), cudaMemcpyDeviceToHost));
  if (time) *time = d.time;
  if (steps) *steps = d.steps;
  if (n_alive) *n_alive = d.range_hi > d.range_lo ? d.range_hi - d.range_lo : 0;
  if (finished) *finished = d.finished;
  return 0;
}

}  // extern "C"

namespace wcsph {
// Copy the instance's slice [range_lo, range_hi) of `src` arrays to host in
// original order.  Extra tail particles (dead, not yet compacted) are scanned too.
static int read_slice(SimImpl& S, int slot, const SimArrays& A, InstDyn& d, std::vector<float4>& pos,
                      std::vector<float4>& vel, std::vector<float4>& acc, std::vector<int>& pid,
                      std::vector<uint32_t>& flags) {
  WCSPH_CUDA(cudaStreamSynchronize(S.s));
  WCSPH_CUDA(cudaMemcpy(&d, S.d_dyn + slot, sizeof(InstDyn), cudaMemcpyDeviceToHost));
  int n_alive = 0;
  WCSPH_CUDA(cudaMemcpy(&n_alive, S.d_n_alive, sizeof(int), cudaMemcpyDeviceToHost));
  const int lo = d.range_hi > d.range_lo ? d.range_lo : 0, hi = d.range_hi > d.range_lo ? d.range_hi : 0;
  const int nl = hi - lo, nt = S.n_host - n_alive;
  pos.resize(nl + nt);
  vel.resize(nl + nt);
  acc.resize(nl + nt);
  pid.resize(nl + nt);
  flags.resize(nl + nt);
  auto cp = [&](void* dst, const void* src, size_t el, int off, int cnt) -> int {
    if (cnt > 0) WCSPH_CUDA(cudaMemcpy(dst, (const char*)src + el * off, el * cnt, cudaMemcpyDeviceToHost));
    return 0;
  };
  int rc = 0;
  rc |= cp(pos.data(), A.pos, sizeof(float4), lo, nl);
  rc |= cp(vel.data(), A.vel, sizeof(float4), lo, nl);
  rc |= cp(acc.data(), A.acc, sizeof(float4), lo, nl);
  rc |= cp(pid.data(), A.pid, sizeof(int), lo, nl);
  rc |= cp(flags.data(), A.flags, sizeof(uint32_t), lo, nl);
  rc |= cp(pos.data() + nl, A.pos, sizeof(float4), n_alive, nt);
  rc |= cp(vel.data() + nl, A.vel, sizeof(float4), n_alive, nt);
  rc |= cp(acc.data() + nl, A.acc, sizeof(float4), n_alive, nt);
  rc |= cp(pid.data() + nl, A.pid, sizeof(int), n_alive, nt);
  rc |= cp(flags.data() + nl, A.flags, sizeof(uint32_t), n_alive, nt);
  return rc;
}
}  // namespace wcsph

extern "C" {

int wcsph_sim_read_instance(wcsph_sim* sim, int32_t slot, float* pos3, float* vel3, float* dens, float* acc3,
                            float* div_v, float* dt_i, int32_t* alive) {
  if (!sim) return WCSPH_E_INVALID;
  SimImpl& S = sim->impl;
  if (slot < 0 || slot >= (int)S.inst.size() || !S.inst[slot].used) {
    set_error("wcsph_sim_read_instance: slot %d is not in use", slot);
    return WCSPH_E_INVALID;
  }
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  std::vector<float4> pos, vel, acc;
  std::vector<int> pid;
  std::vector<uint32_t> flags;
  InstDyn d;
  if (int rc = read_slice(S, slot, S.buf_main, d, pos, vel, acc, pid, flags)) return rc;
  const int n = S.inst[slot].n;
  if (alive)
    for (int i = 0; i < n; ++i) alive[i] = 0;
  for (size_t q = 0; q < pid.size(); ++q) {
    if ((int)(flags[q] & kInstMask) != slot || (flags[q] & kGhostBit)) continue;  // ghosts: their owner reports them
    const int i = pid[q];
    if (i < 0 || i >= n) continue;
    if (pos3) pos3[3 * i] = pos[q].x, pos3[3 * i + 1] = pos[q].y, pos3[3 * i + 2] = pos[q].z;
    if (vel3) vel3[3 * i] = vel[q].x, vel3[3 * i + 1] = vel[q].y, vel3[3 * i + 2] = vel[q].z;
    if (dens) dens[i] = pos[q].w;
    if (acc3) acc3[3 * i] = acc[q].x, acc3[3 * i + 1] = acc[q].y, acc3[3 * i + 2] = acc[q].z;
    if (div_v) div_v[i] = acc[q].w;
    if (dt_i) dt_i[i] = 0.0f;
    if (alive) alive[i] = (flags[q] & kDeadBit) ? 0 : 1;
  }
  return 0;
}

}  // extern "C"

namespace wcsph {

// The diagnostic arrays of a probe pass over instance slot, in original order.
static int read_probe(SimImpl& S, int slot, float* acc3, float* div_v, float* dt_i, float* dens_out,
                      int32_t* n_neighbors) {
  WCSPH_CUDA(cudaStreamSynchronize(S.s));
  InstDyn d;
  WCSPH_CUDA(cudaMemcpy(&d, S.d_dyn + slot, sizeof(InstDyn), cudaMemcpyDeviceToHost));
  const int lo = d.range_lo, nl = d.range_hi > d.range_lo ? d.range_hi - d.range_lo : 0;
  std::vector<float4> dacc(nl);
  std::vector<float> ddt(nl), drho(nl);
  std::vector<int> dn(nl), pid(nl);
  if (nl > 0) {
    WCSPH_CUDA(cudaMemcpy(dacc.data(), S.diag_acc + lo, sizeof(float4) * nl, cudaMemcpyDeviceToHost));
    WCSPH_CUDA(cudaMemcpy(ddt.data(), S.diag_dt + lo, sizeof(float) * nl, cudaMemcpyDeviceToHost));
    WCSPH_CUDA(cudaMemcpy(drho.data(), S.diag_rho + lo, sizeof(float) * nl, cudaMemcpyDeviceToHost));
    WCSPH_CUDA(cudaMemcpy(dn.data(), S.diag_nbr + lo, sizeof(int) * nl, cudaMemcpyDeviceToHost));
    WCSPH_CUDA(cudaMemcpy(pid.data(), S.buf_main.pid + lo, sizeof(int) * nl, cudaMemcpyDeviceToHost));
  }
  const int n = S.inst[slot].n;
  for (int q = 0; q < nl; ++q) {
    const int i = pid[q];
    if (i < 0 || i >= n) continue;
    if (acc3) acc3[3 * i] = dacc[q].x, acc3[3 * i + 1] = dacc[q].y, acc3[3 * i + 2] = dacc[q].z;
    if (div_v) div_v[i] = dacc[q].w;
    if (dt_i) dt_i[i] = ddt[q];
    if (dens_out) dens_out[i] = drho[q];
    if (n_neighbors) n_neighbors[i] = dn[q];
  }
  return 0;
}

// Probe passes over the neighbour lists (sim_list.cuh) of the current build,
// with the probed instance in PH_PROBE and every other one idle: the list
// step's refresh without its kick (j-records from the current state), the
// density pass from the lists when asked, and the list pass, whose epilogue
// writes the diagnostic arrays.  Positions, order and lists are untouched.
static int enqueue_probe_lists(SimImpl& S, int density_pass) {
  StepArgs a = make_args(S);
  a.probe_density = density_pass;
  a.list_reuse = 1;
  a.x0 = S.x0;
  a.alt = a.main;
  const int n = S.n_host;
  WCSPH_CUDA(cudaMemsetAsync(S.d_pairs, 0, sizeof(unsigned long long), S.s));
  WCSPH_CUDA(cudaMemsetAsync(S.d_counters + 4, 0, sizeof(int), S.s));
  k_step_begin<<<nblk(std::max<int>(1, (int)S.inst.size())), kBlock, 0, S.s>>>(a);
  if (n > 0) {
    k_kick_refresh<<<nblk(n), kBlock, 0, S.s>>>(a, 0, 0);
    if (density_pass) {
      if (int rc = launch_density_list(a, n, S.s, h16_lists(S.opt))) return rc;
      k_eos<<<nblk(n), kBlock, 0, S.s>>>(a);
    }
    const bool h16 = S.opt.precision == WCSPH_PREC_HALF2;
    if (int rc = h16 ? launch_hydro_list<true>(a, n, S.s, S.list_shape)
                     : launch_hydro_list<false>(a, n, S.s, S.list_shape))
      return rc;
  }
  WCSPH_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace wcsph

extern "C" {

int wcsph_sim_probe_forces(wcsph_sim* sim, int32_t slot, int32_t density_pass, float* acc3, float* div_v, float* dt_i,
                           float* dens_out, int32_t* n_neighbors) {
  if (!sim || density_pass < 0 || density_pass > 2) return WCSPH_E_INVALID;
  SimImpl& S = sim->impl;
  if (slot < 0 || slot >= (int)S.inst.size() || !S.inst[slot].active) {
    set_error("wcsph_sim_probe_forces: slot %d is not active", slot);
    return WCSPH_E_INVALID;
  }
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  for (size_t q = 0; q < S.inst.size(); ++q) S.h_phase[q] = PH_IDLE;
  S.h_phase[slot] = PH_PROBE;
  if (int rc = upload_tables(S)) return rc;
  StepArgs a = make_args(S);
  a.probe_density = density_pass;
  int rc = enqueue_pass(S, a, density_pass != 0, false, nullptr);
  int rc2 = set_all_phases(S, PH_STEP);
  if (rc) return rc;
  if (rc2) return rc2;
  S.graph_dirty = true;
  return read_probe(S, slot, acc3, div_v, dt_i, dens_out, n_neighbors);
}

int wcsph_sim_probe_lists(wcsph_sim* sim, int32_t slot, int32_t density_pass, float* acc3, float* div_v, float* dt_i,
                          float* dens_out, int32_t* n_neighbors) {
  if (!sim || density_pass < 0 || density_pass > 2) return WCSPH_E_INVALID;
  SimImpl& S = sim->impl;
  if (S.opt.list_interval <= 0) {
    set_error("wcsph_sim_probe_lists: the solver has no neighbour lists (list_interval = 0)");
    return WCSPH_E_STATE;
  }
  if (slot < 0 || slot >= (int)S.inst.size() || !S.inst[slot].active) {
    set_error("wcsph_sim_probe_lists: slot %d is not active", slot);
    return WCSPH_E_INVALID;
  }
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  if (S.appended && S.n_host > 0) {
    set_error("wcsph_sim_probe_lists: particles were appended since the last pass; step first");
    return WCSPH_E_STATE;
  }
  for (size_t q = 0; q < S.inst.size(); ++q) S.h_phase[q] = PH_IDLE;
  S.h_phase[slot] = PH_PROBE;
  if (int rc = upload_tables(S)) return rc;
  int rc = 0;
  if (S.lists_valid) {
    rc = enqueue_probe_lists(S, density_pass);
  } else {
    // No current lists: a build pass in probe phase (binning at the current
    // positions, the scan writes the lists, the list pass sums them).  Its
    // lists serve the steps that follow like those of a step's build.
    StepArgs a = make_args(S);
    a.probe_density = density_pass;
    rc = enqueue_pass(S, a, density_pass != 0, false, nullptr, nullptr, true);
    if (!rc) {  // the device's schedule starts from these lists
      S.lists_valid = true;
      if (cudaMemsetAsync(S.d_lflags + kLfSince, 0, sizeof(unsigned), S.s) != cudaSuccess ||
          cudaMemsetAsync(S.d_lflags + kLfForce, 0, sizeof(unsigned), S.s) != cudaSuccess)
        rc = WCSPH_E_CUDA;
    }
  }
  int rc2 = set_all_phases(S, PH_STEP);
  if (rc) return rc;
  if (rc2) return rc2;
  return read_probe(S, slot, acc3, div_v, dt_i, dens_out, n_neighbors);
}

int wcsph_sim_read_order(wcsph_sim* sim, int32_t slot, int32_t* perm, uint32_t* cell_key) {
  if (!sim) return WCSPH_E_INVALID;
  SimImpl& S = sim->impl;
  if (slot < 0 || slot >= (int)S.inst.size() || !S.inst[slot].active) {
    set_error("wcsph_sim_read_order: slot %d is not active", slot);
    return WCSPH_E_INVALID;
  }
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  WCSPH_CUDA(cudaStreamSynchronize(S.s));
  InstDyn d;
  WCSPH_CUDA(cudaMemcpy(&d, S.d_dyn + slot, sizeof(InstDyn), cudaMemcpyDeviceToHost));
  const int lo = d.range_lo, nl = d.range_hi > d.range_lo ? d.range_hi - d.range_lo : 0;
  if (nl > 0) {
    if (perm) WCSPH_CUDA(cudaMemcpy(perm, S.buf_main.pid + lo, sizeof(int) * nl, cudaMemcpyDeviceToHost));
    if (cell_key) {
      WCSPH_CUDA(cudaMemcpy(cell_key, S.keys_out + lo, sizeof(uint32_t) * nl, cudaMemcpyDeviceToHost));
      const uint32_t base = S.h_params[slot].key_base;
      for (int q = 0; q < nl; ++q) cell_key[q] -= base;
    }
  }
  return nl;
}

int wcsph_sim_conservation(wcsph_sim* sim, int32_t slot, double* out6) {
  if (!sim || !out6) return WCSPH_E_INVALID;
  SimImpl& S = sim->impl;
  const int n = (slot >= 0 && slot < (int)S.inst.size()) ? S.inst[slot].n : 0;
  if (n <= 0) {
    set_error("wcsph_sim_conservation: slot %d is not in use", slot);
    return WCSPH_E_INVALID;
  }
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  return launch_conservation(S.buf_main, S.d_dyn, S.d_params, slot, S.d_cons, S.s, out6);
}

int64_t wcsph_sim_last_pairs(wcsph_sim* sim) {
  if (!sim) return -1;
  SimImpl& S = sim->impl;
  if (cudaSetDevice(S.opt.device) != cudaSuccess || cudaStreamSynchronize(S.s) != cudaSuccess) return -1;
  unsigned long long c = 0;
  if (cudaMemcpy(&c, S.d_pairs, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  return (int64_t)c;
}

int32_t wcsph_sim_kernels_per_step(wcsph_sim* sim) { return sim ? sim->impl.kernels_per_step : -1; }

void* wcsph_sim_stream(wcsph_sim* sim) { return sim ? (void*)sim->impl.s : nullptr; }

int wcsph_sim_tuning(wcsph_sim* sim, int32_t* out4) {
  if (!sim || !out4) return WCSPH_E_INVALID;
  out4[0] = sim->impl.tile_shape;
  out4[1] = sim->impl.list_shape;
  out4[2] = sim->impl.tuned_bucket;
  out4[3] = sim->impl.build_shape;
  return 0;
}

int wcsph_sim_list_stats(wcsph_sim* sim, int64_t* out6) {
  if (!sim || !out6) return WCSPH_E_INVALID;
  SimImpl& S = sim->impl;
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  WCSPH_CUDA(cudaStreamSynchronize(S.s));
  unsigned lf[kLfWords] = {};
  if (S.d_lflags) WCSPH_CUDA(cudaMemcpy(lf, S.d_lflags, sizeof(lf), cudaMemcpyDeviceToHost));
  out6[0] = lf[kLfBuilds];
  out6[1] = lf[kLfListSteps];
  out6[2] = lf[kLfOverflows] + (lf[kLfOverflowPending] ? 1 : 0);
  out6[3] = (int64_t)lf[kLfLongest];
  out6[4] = S.kernels_per_step;
  out6[5] = S.kernels_reuse;
  return 0;
}

int wcsph_sim_list_schedule(wcsph_sim* sim, int64_t* out4) {
  if (!sim || !out4) return WCSPH_E_INVALID;
  SimImpl& S = sim->impl;
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  WCSPH_CUDA(cudaStreamSynchronize(S.s));
  unsigned lf[kLfWords] = {};
  if (S.d_lflags) WCSPH_CUDA(cudaMemcpy(lf, S.d_lflags, sizeof(lf), cudaMemcpyDeviceToHost));
  out4[0] = lf[kLfBuilds];
  out4[1] = lf[kLfPartials];
  out4[2] = lf[kLfListSteps];
  out4[3] = (int64_t)lf[kLfSince];
  return 0;
}

int64_t wcsph_sim_list_entries(wcsph_sim* sim) {
  if (!sim) return -1;
  SimImpl& S = sim->impl;
  if (S.opt.list_interval <= 0 || !S.lists_valid) return 0;
  if (cudaSetDevice(S.opt.device) != cudaSuccess || cudaStreamSynchronize(S.s) != cudaSuccess) return -1;
  int n_alive = 0;
  if (cudaMemcpy(&n_alive, S.d_n_alive, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  std::vector<int> cnt(std::max(0, n_alive));
  if (n_alive > 0 && cudaMemcpy(cnt.data(), S.list_cnt, sizeof(int) * n_alive, cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  int64_t tot = 0;
  for (int c : cnt) tot += std::min(c, kListMax);
  return tot;
}

int wcsph_sim_invalidate_lists(wcsph_sim* sim) {
  if (!sim) return WCSPH_E_INVALID;
  sim->impl.lists_valid = false;
  return 0;
}

// Eager steps with CUDA events around each phase; ms[0..3] summed over the
// steps that searched or built, ms[4..7] over the steps that read the lists,
// ms[8] the builds' scans; steps[0..1] how many of each.
static int profile_impl(SimImpl& S, int nsteps, double* ms, int32_t* steps) {
  WCSPH_CUDA(cudaSetDevice(S.opt.device));
  cudaEvent_t ev[4];
  for (auto& e : ev) WCSPH_CUDA(cudaEventCreate(&e));
  WCSPH_CUDA(cudaEventCreate(&S.scan_ev));
  for (int k = 0; k < 9; ++k) ms[k] = 0.0;
  steps[0] = steps[1] = 0;
  StepArgs a = make_args(S);
  int rc = 0;
  for (int t = 0; t < nsteps && !rc; ++t) {
    bool built = true;
    if (S.opt.list_interval > 0) {
      rc = list_step(S, false, ev, &built);  // the same build / list-step schedule as wcsph_sim_step
    } else {
      if (cudaMemsetAsync(S.d_pairs, 0, sizeof(unsigned long long), S.s) != cudaSuccess) rc = WCSPH_E_CUDA;
      if (!rc) rc = enqueue_pass(S, a, S.any_density, false, &S.kernels_per_step, ev);
    }
    if (!rc && cudaEventSynchronize(ev[3]) != cudaSuccess) rc = WCSPH_E_CUDA;
    if (!rc) {
      float x[3];
      cudaEventElapsedTime(&x[0], ev[0], ev[1]);
      cudaEventElapsedTime(&x[1], ev[1], ev[2]);
      cudaEventElapsedTime(&x[2], ev[2], ev[3]);
      double* m = ms + (built ? 0 : 4);
      for (int k = 0; k < 3; ++k) m[k] += x[k];
      m[3] += x[0] + x[1] + x[2];
      ++steps[built ? 0 : 1];
      if (built && S.opt.list_interval > 0) {
        float sc = 0.f;
        cudaEventElapsedTime(&sc, ev[2], S.scan_ev);
        ms[8] += sc;
      }
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  cudaEventDestroy(S.scan_ev);
  S.scan_ev = nullptr;
  if (rc == WCSPH_E_CUDA) set_error("profiling steps: CUDA error %s", cudaGetErrorString(cudaGetLastError()));
  return rc;
}

int wcsph_sim_profile_steps(wcsph_sim* sim, int32_t nsteps, double* ms4) {
  if (!sim || !ms4 || nsteps < 0) return WCSPH_E_INVALID;
  double ms[9];
  int32_t steps[2];
  const int rc = profile_impl(sim->impl, nsteps, ms, steps);
  for (int k = 0; k < 4; ++k) ms4[k] = rc ? 0.0 : ms[k] + ms[4 + k];
  return rc;
}

int wcsph_sim_profile_split(wcsph_sim* sim, int32_t nsteps, double* ms9, int32_t* steps2) {
  if (!sim || !ms9 || !steps2 || nsteps < 0) return WCSPH_E_INVALID;
  return profile_impl(sim->impl, nsteps, ms9, steps2);
}

}  // extern "C"

// Device-resident solver kernels: binning, permutation, density, EoS, hydro.
//
// Data layout in HBM (structure of arrays, sorted by cell every step):
//   state "main" and "alt" buffers (float4 each, double-buffered by the sort):
//     pos = (x, y, z, rho)   vel = (vx, vy, vz, -)   vh = (vx_half, ..., -)
//     acc = (ax, ay, az, div v)   pid (original index)   flags (instance | FREEZE | dead)
//   j-records written after the EoS, read by the pair kernels (36 B / particle):
//     jr[p].a = (x, y, z, P/rho^2)   jr[p].b = (vx, vy, vz, rho)   jC = c
//     (a and b interleaved: one 32-byte sector per particle, read by the
//     pair phases with one 256-bit load)
//   cell table: start/end per linear cell, instance-major.
#pragma once
#include <cuda_fp16.h>

#include "wcsph_common.cuh"

namespace wcsph {

struct __align__(32) JRec {
  float4 a, b;
};

// One particle's j-record in a single 256-bit read-only load (sm_100).
__device__ __forceinline__ JRec ld_jrec(const JRec* p) {
  JRec r;
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(r.a.x), "=f"(r.a.y), "=f"(r.a.z), "=f"(r.a.w), "=f"(r.b.x), "=f"(r.b.y), "=f"(r.b.z), "=f"(r.b.w)
      : "l"(p));
  return r;
}

// ---------------------------------------------- compact (half2) j-records
// The half2 list pass gathers one 16-byte record per list entry (two records
// per 32-byte sector), jh[p] = uint4:
//   .x = x | y << 16, .y = z | vx << 16, .z = vy | vz << 16, .w = rho (FP32 bits)
// Positions are 16-bit fixed-point offsets from the centre of the particle's
// cell at the last list build (steps of 2^-15 cell edges, biased by 2^15, so
// one cell edge either side).  Velocities are 16-bit fixed point in steps of
// the instance's velocity quantum vq (a power of two, 2^-15 of a bound on its
// fastest particle this step; InstDyn::vq), biased by 2^15.  P/rho^2 is
// gathered from jpo beside the records and c recomputed from rho by the
// pass.  A particle outside either range (far
// from its build cell, above the grid where cells are clamped, faster than
// the bound) or removed is marked far (rho = kFarRho, 0: finite in every term
// it meets before the entry switches to the FP32 record), and its entries are
// read from the FP32 record.
constexpr uint32_t kFarRho = 0u;
constexpr float kQ16Scale = 32768.0f;

__device__ __forceinline__ float cell_centre(const InstParams& P, int k, int c) {
  return __fmaf_rn((float)c + 0.5f, P.cell[k], P.lo[k]);
}

// Biased 16-bit code (1 .. 65535) of q, in steps, or -1 when |q| > 32767 or q is NaN.
__device__ __forceinline__ int q16(float q) {
  if (!(fabsf(q) <= 32767.0f)) return -1;
  return __float2int_rn(q) + 32768;
}

// Write the compact record of slot p: position x, velocity v, density rho,
// build cell (cx, cy, cz), velocity quantum vq.
__device__ __forceinline__ void write_h16(uint4* jh, const InstParams& P, float vq, int p, const float4& x,
                                          const float4& v, float rho, int cx, int cy, int cz) {
  const int c[3] = {cx, cy, cz};
  const float* xa = &x.x;
  int u[6];
#pragma unroll
  for (int k = 0; k < 3; ++k) u[k] = q16((xa[k] - cell_centre(P, k, c[k])) * P.inv_cell[k] * kQ16Scale);
  const float ivq = 1.0f / vq;  // vq is a power of two: exact
  u[3] = q16(v.x * ivq), u[4] = q16(v.y * ivq), u[5] = q16(v.z * ivq);
  bool far = !(rho > 0.0f);
#pragma unroll
  for (int k = 0; k < 6; ++k) far |= u[k] < 0;
  if (far) {
    jh[p] = make_uint4(0x80008000u, 0x80008000u, 0x80008000u, kFarRho);
    return;
  }
  jh[p] = make_uint4((uint32_t)u[0] | ((uint32_t)u[1] << 16), (uint32_t)u[2] | ((uint32_t)u[3] << 16),
                     (uint32_t)u[4] | ((uint32_t)u[5] << 16), __float_as_uint(rho));
}

// A removed particle: far, so that its entries take the FP32 record (whose
// position is far from everything).
__device__ __forceinline__ void write_h16_dead(uint4* jh, int p) {
  jh[p] = make_uint4(0x80008000u, 0x80008000u, 0x80008000u, kFarRho);
}

// Words of StepArgs::list_flags.
enum ListFlag {
  kLfDeaths = 0,           // a particle was removed since the last full build: the next step builds in full
  kLfPartials = 1,         // partial builds so far (counted in kLfBuilds too)
  kLfErr = 2,              // sticky errors: bit 0 a displacement passed skin / 2 on a list step
  kLfLongest = 3,          // largest list built
  kLfOverflowPending = 4,  // the last build overflowed a list: the next step builds
  kLfBuilds = 5,           // builds so far
  kLfListSteps = 6,        // list steps so far
  kLfOverflows = 7,        // builds whose lists overflowed
  kLfSince = 8,            // steps since the last full build (the build counts 1)
  kLfPartial = 9,          // this step's build is partial: instances with inst_keep set keep their lists
  kLfForce = 10,           // the host asks for a build (lists stale)
  kLfDecision = 11,        // this step builds (1) or reads the lists (0)
  kLfWords = 16
};

struct SimArrays {
  float4 *pos, *vel, *vh, *acc;  // one buffer set
  int* pid;
  uint32_t* flags;
};

struct StepArgs {
  SimArrays main, alt;
  const InstParams* params;
  InstDyn* dyn;
  const int* phase;       // per-instance phase for this launch
  uint32_t* keys_in;
  int* vals_in;
  const uint32_t* keys_out;
  const int* vals_out;
  JRec* jr;
  float* jC;
  float* rho_new;         // density pass output
  int *cell_start, *cell_end;
  int* n_alive;           // device count of live particles after binning
  int n_host;             // particle slots in use (upper bound of live)
  int n_inst;
  unsigned long long* pair_count;
  int* run_list;          // linear index of every non-empty cell (unordered)
  int* run_count;         // number of entries in run_list
  int init_filter;        // initial-pass Shepard filter launch (main.cpp:75)
  // neighbour lists (list_interval > 0)
  uint32_t* list;         // list_max entries per sorted slot: slot | image code << 27
  int* list_cnt;          // entries per slot
  int list_max;
  float4* x0;             // build steps: record the positions the lists were built at
  unsigned* list_flags;   // ListFlag words: sticky errors, largest list, the device's build
                          // decision (full or partial) and the schedule's counters
  int list_reuse;         // this step reads the lists: periodic wrapping waits for the next build
  int* dens_any;          // set by k_step_begin when any instance has a density pass in this launch
  unsigned* inst_motion;  // neighbour lists: per instance, the largest |x - x0|, |v| and |a| over its moving
                          // particles at the end of the step, in units of its skin (float bits)
  int* inst_keep;          // neighbour lists, partial builds: per instance, 1 = keeps its lists (k_list_set)
  // compact j-records of the half2 list pass (WCSPH_PREC_HALF2 with lists; null otherwise)
  uint4* jh;              // 16-bit cell-relative x, y, z, 16-bit velocity, FP32 rho (write_h16)
  float* jpo;             // P/rho^2 of every slot beside jh (jr[p].a.w, gathered in 4 bytes)
  uint32_t list_pad;      // list entry naming the padding slot (k_list_pad_slot): rows are padded with it
                          // to whole groups of four entries
  int density_overflow_only;  // k_density_plain of a list build: only the particles whose list overflowed
  int probe_density;      // density pass of a probe launch: 0 none, 1 summation, 2 Shepard
  // diagnostics (probe phase)
  float4* diag_acc;
  float* diag_dt;
  int* diag_nbr;
  float* diag_rho;
};

__device__ __forceinline__ float bits_f(unsigned b) { return __uint_as_float(b); }

// Density pass of an instance in the current launch: 0 none, 1 summation, 2 Shepard.
__device__ __forceinline__ int density_kind(const StepArgs& a, const InstParams& P, const InstDyn& d, int ph) {
  if (ph == PH_IDLE || !P.active) return 0;
  if (ph == PH_PROBE) return a.probe_density;
  if (ph == PH_INIT) {
    if (a.init_filter) return P.density_mode == WCSPH_DENSITY_SHEPARD ? 2 : 0;
    return P.density_mode == WCSPH_DENSITY_SUMMATION ? 1 : 0;
  }
  if (d.dt_cur <= 0.0f) return 0;  // finished: the state no longer changes
  if (P.density_mode == WCSPH_DENSITY_SUMMATION) return 1;
  if (P.density_mode == WCSPH_DENSITY_SHEPARD && P.shepard_interval > 0 &&
      ((d.steps - 1) % P.shepard_interval) == 0)  // main.cpp:105, step index before increment
    return 2;
  return 0;
}

// ------------------------------------------------------------ step begin
// One thread per instance: rotate dt, advance time, mark finished.
__global__ void k_step_begin(StepArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < a.n_inst) {
    InstDyn& d = a.dyn[k];
    const InstParams& P = a.params[k];
    const int ph = a.phase[k];
    if (!a.list_reuse) {  // the binning sets them again; a list step keeps the build's order
      d.range_lo = 0x7fffffff;
      d.range_hi = 0;
    }
    if (ph == PH_STEP && P.active) {
      const float dt = d.finished ? 0.0f : bits_f(d.dt_next_bits);
      d.dt_cur = dt;
      d.dt_next_bits = 0x7f800000u;  // +inf
      if (dt > 0.0f) {
        d.time += (double)dt;
        d.steps += 1;
        if (P.t_end > 0.0 && d.time >= P.t_end) d.finished = 1;
      }
    } else if (ph == PH_INIT) {
      d.dt_cur = 0.0f;
      d.dt_next_bits = 0x7f800000u;
    } else {
      d.dt_cur = 0.0f;
    }
    if (a.dens_any && (ph == PH_INIT || ph == PH_PROBE || density_kind(a, P, d, ph))) atomicOr(a.dens_any, 1);
  }
  if (k == 0 && !a.list_reuse) *a.n_alive = a.n_host;
}

// ------------------------------------------------------- kick + binning
// Periodic wrap of a position into [lo, lo + L) (one rounded FP32 operation
// per axis); true when a coordinate moved.
__device__ __forceinline__ bool wrap_periodic(const InstParams& P, float4& x) {
  bool moved = false;
  float* c = &x.x;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float hi = P.lo[k] + P.L[k];
    if (c[k] >= hi) c[k] = __fsub_rn(c[k], P.L[k]), moved = true;
    else if (c[k] < P.lo[k]) c[k] = __fadd_rn(c[k], P.L[k]), moved = true;
  }
  return moved;
}

// KDK first half of one live particle p of a stepping instance
// (class.h:146-159 as main.cpp:98-103 runs it), periodic wrap (not on list
// steps), escapee removal (Dam2.h:117-122).  Returns true when the state
// changed; dead is set when the particle left the kill box.
__device__ __forceinline__ bool kick_particle(const StepArgs& a, const InstParams& P, int inst, int p, uint32_t f,
                                              float4& x, float4& v, float4& vh, bool& dead, bool keep = false) {
  const int ph = a.phase[inst];
  const float dt = a.dyn[inst].dt_cur;
  if (!(ph == PH_STEP && dt > 0.0f)) return false;
  const float4 acc = a.main.acc[p];
  x.w += -x.w * dt * acc.w;  // continuity, FREEZE included (class.h:151)
  if (!(f & kFreezeBit)) {
    const float hdt = 0.5f * dt;
    vh = make_float4(v.x + hdt * acc.x, v.y + hdt * acc.y, v.z + hdt * acc.z, 0.f);
    x.x += dt * vh.x;
    x.y += dt * vh.y;
    x.z += dt * vh.z;
    if (P.slab_margin2 > 0.0f && dt * dt * (vh.x * vh.x + vh.y * vh.y + vh.z * vh.z) > P.slab_margin2)
      atomicOr(&a.dyn[inst].errors, kErrDrift);  // the ghost layer no longer covers this drift
    v = make_float4(v.x + dt * acc.x, v.y + dt * acc.y, v.z + dt * acc.z, 0.f);
    if (P.periodic && !a.list_reuse && !keep) wrap_periodic(P, x);  // between list builds positions run on continuously
    if (P.kill_on) {
      const float* c = &x.x;
#pragma unroll
      for (int k = 0; k < 3; ++k)
        if (P.kill_lo[k] < P.kill_hi[k] && (c[k] < P.kill_lo[k] || c[k] > P.kill_hi[k])) dead = true;
    }
  }
  return true;
}

// The kick, the periodic wrap (every binning pass: positions run on
// continuously between neighbour-list builds), then the Morton cell key of
// each particle.  In a partial list build, an instance that keeps its lists
// (inst_keep) is kicked like a list step (no wrap, |x - x0| checked) and keyed
// by its build positions x0, so the stable sort leaves its particles in
// their slots; a particle removed during a partial build keeps the key of
// its build position too (in place, marked dead, far records), and the next
// step builds in full.
__global__ void k_kick_bin(StepArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n_host) return;
  uint32_t f = a.main.flags[p];
  const int inst = f & kInstMask;
  const InstParams& P = a.params[inst];
  const bool was_dead = (f & kDeadBit) || !P.active;
  bool dead = was_dead;
  const bool partial = a.inst_keep && a.list_flags[kLfPartial] != 0u;
  const bool keep = partial && a.inst_keep[inst];
  float4 x = a.main.pos[p];
  float4 v = a.main.vel[p];
  float4 vh = v;
  bool changed = !dead && kick_particle(a, P, inst, p, f, x, v, vh, dead, keep);
  // passes without a kick (probe, initial and binning passes) wrap too, so
  // that positions left outside the box by list steps are binned correctly
  if (!dead && !changed && !keep && P.periodic && wrap_periodic(P, x)) changed = true;
  if (changed) {
    a.main.pos[p] = x;
    a.main.vel[p] = v;
  }
  a.main.vh[p] = vh;
  uint32_t key = kDeadKey;
  if (dead && !(f & kDeadBit)) a.main.flags[p] = f | kDeadBit;
  // (particles removed before this step sit in the tail since the last full
  // build, which every removal forces: they keep the dead key)
  if (partial && !was_dead && (keep || dead)) {
    const float4 o = a.x0[p];  // the build position: the particle keeps its cell and slot
    key = P.key_base + morton3(cell_of(o.x, P.lo[0], P.inv_cell[0], P.ncell[0]),
                               cell_of(o.y, P.lo[1], P.inv_cell[1], P.ncell[1]),
                               cell_of(o.z, P.lo[2], P.inv_cell[2], P.ncell[2]));
    if (dead) atomicOr(&a.list_flags[kLfDeaths], 1u);  // the next step builds in full
    if (keep && !dead) {
      const float dx = x.x - o.x, dy = x.y - o.y, dz = x.z - o.z;
      if (sqrtf(dx * dx + dy * dy + dz * dz) * P.inv_skin > 0.5f) atomicOr(&a.list_flags[kLfErr], 1u);
    }
  } else if (!dead) {
    const int cx = cell_of(x.x, P.lo[0], P.inv_cell[0], P.ncell[0]);
    const int cy = cell_of(x.y, P.lo[1], P.inv_cell[1], P.ncell[1]);
    const int cz = cell_of(x.z, P.lo[2], P.inv_cell[2], P.ncell[2]);
    key = P.key_base + morton3(cx, cy, cz);
  }
  a.keys_in[p] = key;
  a.vals_in[p] = p;
}

// ------------------------------------------------- permutation + tables
// Gather the state into sorted order (main -> alt), fill the cell table and
// the instance ranges, count live particles, and write the j-records with the
// Tait EoS (EoS.h:80-86) of the current density.
__global__ void k_permute(StepArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n_host) return;
  const int src = a.vals_out[p];
  const uint32_t key = a.keys_out[p];
  const float4 x = a.main.pos[src];
  const float4 v = a.main.vel[src];
  a.alt.pos[p] = x;
  a.alt.vel[p] = v;
  a.alt.vh[p] = a.main.vh[src];
  a.alt.acc[p] = a.main.acc[src];
  a.alt.pid[p] = a.main.pid[src];
  const uint32_t f = a.main.flags[src];
  a.alt.flags[p] = f;
  const uint32_t kprev = p > 0 ? a.keys_out[p - 1] : 0u;
  const uint32_t knext = p + 1 < a.n_host ? a.keys_out[p + 1] : kDeadKey;
  if (key == kDeadKey) {
    if (p == 0 || kprev != kDeadKey) *a.n_alive = p;
    return;
  }
  const int inst = f & kInstMask;
  const InstParams& P = a.params[inst];
  const uint32_t local = key - P.key_base;
  const int cx = compact3(local), cy = compact3(local >> 1), cz = compact3(local >> 2);
  const int lin = P.cell_base + (cz * P.ncell[1] + cy) * P.ncell[0] + cx;
  if (p == 0 || kprev != key) {
    a.cell_start[lin] = p;
    a.run_list[atomicAdd(a.run_count, 1)] = lin;
  }
  if (knext != key) a.cell_end[lin] = p + 1;
  // instance ranges (keys are instance-major, so each instance is contiguous)
  if (p == 0 || kprev == kDeadKey || (int)(a.main.flags[a.vals_out[p - 1]] & kInstMask) != inst)
    a.dyn[inst].range_lo = p;
  if (knext == kDeadKey || (int)(a.main.flags[a.vals_out[p + 1]] & kInstMask) != inst) a.dyn[inst].range_hi = p + 1;
  // list build: the positions the lists refer to (kept by an instance that
  // keeps its lists in a partial build)
  const bool keep = a.inst_keep && a.list_flags[kLfPartial] != 0u && a.inst_keep[inst];
  if (a.x0 && !keep) a.x0[p] = make_float4(x.x, x.y, x.z, 0.f);
  if (f & kDeadBit) {  // removed during a partial build: in place until the next full build, far from all
    a.jr[p].a = make_float4(1.0e30f, 1.0e30f, 1.0e30f, 0.f);
    a.jr[p].b = make_float4(0.f, 0.f, 0.f, 1.f);
    a.jC[p] = 0.f;
    if (a.jh) write_h16_dead(a.jh, p);
    if (a.jpo) a.jpo[p] = 0.f;
    return;
  }
  float pres, snds;
  tait(P, x.w, pres, snds);
  const float po = pres / (x.w * x.w);
  a.jr[p].a = make_float4(x.x, x.y, x.z, po);
  a.jr[p].b = make_float4(v.x, v.y, v.z, x.w);
  a.jC[p] = snds;
  if (a.jh) write_h16(a.jh, P, a.dyn[inst].vq, p, x, v, x.w, cx, cy, cz);
  if (a.jpo) a.jpo[p] = po;
}

// Does the hydro pass run for an instance in the current launch?
__device__ __forceinline__ bool wants_force(const InstParams& P, const InstDyn& d, int ph) {
  if (!P.active) return false;
  return ph == PH_INIT || ph == PH_PROBE || (ph == PH_STEP && d.dt_cur > 0.0f);
}

// Neighbour-cell iteration shared by the plain kernels.  Calls
// body(q, J, dx, dy, dz, r2, code) for every in-support j (0 < r2 < (2h)^2,
// FP32 predicate of the oracle); code is the periodic image code of the tiled
// kernel's queue entries ((sx+1) + 3 (sy+1) + 9 (sz+1) in units of the box).
template <typename Body>
__device__ __forceinline__ void for_each_neighbor(const StepArgs& a, const InstParams& P, float xi, float yi, float zi,
                                                  Body&& body) {
  const int cx = cell_of(xi, P.lo[0], P.inv_cell[0], P.ncell[0]);
  const int cy = cell_of(yi, P.lo[1], P.inv_cell[1], P.ncell[1]);
  const int cz = cell_of(zi, P.lo[2], P.inv_cell[2], P.ncell[2]);
  const float H2 = P.H2;
  for (int oz = -1; oz <= 1; ++oz) {
    int z;
    float sz;
    if (!neighbor_cell(P, 2, cz + oz, z, sz)) continue;
    for (int oy = -1; oy <= 1; ++oy) {
      int y;
      float sy;
      if (!neighbor_cell(P, 1, cy + oy, y, sy)) continue;
      const int row = P.cell_base + (z * P.ncell[1] + y) * P.ncell[0];
      for (int ox = -1; ox <= 1; ++ox) {
        int x;
        float sx;
        if (!neighbor_cell(P, 0, cx + ox, x, sx)) continue;
        const int lin = row + x;
        const int s = a.cell_start[lin], e = a.cell_end[lin];
        const uint32_t code = (uint32_t)((sx > 0.f) - (sx < 0.f) + 1 + 3 * ((sy > 0.f) - (sy < 0.f) + 1) +
                                         9 * ((sz > 0.f) - (sz < 0.f) + 1));
        for (int q = s; q < e; ++q) {
          const float4 J = __ldg(&a.jr[q].a);
          const float dx = __fsub_rn(xi, __fadd_rn(J.x, sx));
          const float dy = __fsub_rn(yi, __fadd_rn(J.y, sy));
          const float dz = __fsub_rn(zi, __fadd_rn(J.z, sz));
          const float r2 = dist2(dx, dy, dz);
          if (r2 > 0.0f && r2 < H2) body(q, J, dx, dy, dz, r2, code);
        }
      }
    }
  }
}

// ---------------------------------------------------------- density pass
// Summation rho_i = m sum_j W_ij (self included) or the Shepard filter of
// force.h:12-29, sum m W / sum (m/rho_j) W, from the pre-filter densities.
__global__ void k_density_plain(StepArgs a) {
  if (a.dens_any && !*a.dens_any) return;  // no density pass in this launch
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= *a.n_alive) return;
  if (a.density_overflow_only && a.list_cnt[p] <= a.list_max) return;  // k_density_list has it
  const int inst = a.alt.flags[p] & kInstMask;
  const InstParams& P = a.params[inst];
  const int kind = density_kind(a, P, a.dyn[inst], a.phase[inst]);
  if (!kind) return;
  // an instance that keeps its lists in a partial build: its cells are those
  // of its build positions, so its density pass reads the lists (k_density_list)
  if (a.inst_keep && a.list_flags[kLfPartial] != 0u && a.inst_keep[inst]) return;
  const float4 I = a.jr[p].a;
  const float rho_i = a.jr[p].b.w;
  float sum = 0.5f, one = 0.5f / rho_i;  // self term: w(0) = 1/2
  const float iH = P.inv_H;
  const bool shep = kind == 2;
  for_each_neighbor(a, P, I.x, I.y, I.z, [&](int q, const float4&, float, float, float, float r2, uint32_t) {
    const float w = spline_w(sqrtf(r2) * iH);
    sum += w;
    if (shep) one += w / __ldg(&a.jr[q].b.w);
  });
  a.rho_new[p] = shep ? sum / one : P.mass * P.Kw * sum;
}

// Refresh the j-records of particles whose density was just recomputed.
__global__ void k_eos(StepArgs a) {
  if (a.dens_any && !*a.dens_any) return;  // no density pass in this launch
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= *a.n_alive) return;
  const int inst = a.alt.flags[p] & kInstMask;
  const InstParams& P = a.params[inst];
  const int ph = a.phase[inst];
  if (!density_kind(a, P, a.dyn[inst], ph)) return;
  const float rho = a.rho_new[p];
  float pres, snds;
  tait(P, rho, pres, snds);
  const float po = pres / (rho * rho);
  a.jr[p].a.w = po;
  if (a.jpo) a.jpo[p] = po;
  a.jr[p].b.w = rho;
  a.jC[p] = snds;
  if (a.jh && a.jh[p].w != kFarRho) a.jh[p].w = __float_as_uint(rho);  // the compact record's density
  if (ph != PH_PROBE) a.alt.pos[p].w = rho;
}

// Warp-aggregated atomic min of a positive float into dt_next of an instance.
__device__ __forceinline__ void dt_min(InstDyn* dyn, int inst, float v, bool valid) {
  const unsigned full = 0xffffffffu;
  const int inst0 = __shfl_sync(full, inst, 0);
  const bool uniform = __all_sync(full, inst == inst0 || !valid);
  if (uniform) {
    float m = valid ? v : __int_as_float(0x7f800000);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(full, m, o));
    if ((threadIdx.x & 31) == 0 && m < __int_as_float(0x7f800000))
      atomicMin(&dyn[inst0].dt_next_bits, __float_as_uint(m));
  } else if (valid) {
    atomicMin(&dyn[inst].dt_next_bits, __float_as_uint(v));
  }
}

// Epilogue shared by the hydro kernels: finish particle p from its pair sums
// (acc sums without the mass factor, sum g (dr.dv), v_sig, pair count).
// Adds gravity to every particle (Dam2.h:104-108), does the final kick of
// HYDRO particles (class.h:160-163), the density floor (Dam2.h:111), and
// folds the CFL limits of integral.h:2-12 into dt_cand.  Writes main[p].
// Motion of a particle at the end of a step, in units of its instance's skin:
// |x - x0| (x0: its position at the last list build), |v| and |a|.  The next
// step's drift is dt (v + dt/2 a), so its displacement from x0 is at most
// d + dt s + dt^2/2 acc (k_list_set).
struct Motion {
  float d = 0.f, s = 0.f, acc = 0.f;
};

__device__ __forceinline__ void finish_hydro(const StepArgs& a, int p, const InstParams& P, int inst, int ph,
                                             uint32_t f, float ax, float ay, float az, float dsum, float vsig,
                                             unsigned cnt, float& dt_cand, bool& dt_valid, Motion* mo = nullptr) {
  float4 x = a.alt.pos[p];
  float4 v = a.alt.vel[p];
  float4 acc;
  const float rho_i = a.jr[p].b.w, ci = a.jC[p];
  const float m = P.mass, h = P.h;
  ax *= m;
  ay *= m;
  az *= m;
  const float divv = -m * dsum / rho_i;
  const float dt_i = P.c_cfl * h / (ci + vsig);
  if (ph == PH_PROBE) {
    a.diag_acc[p] = make_float4(ax, ay, az, divv);
    a.diag_dt[p] = dt_i;
    a.diag_nbr[p] = (int)cnt;
    a.diag_rho[p] = rho_i;
    acc = a.alt.acc[p];
  } else {
    az -= P.g;
    if (!(f & kFreezeBit)) {
      if (!(f & kGhostBit)) {  // ghosts: their owner folds their dt
        const float amag = sqrtf(ax * ax + ay * ay + az * az);
        const float c = fminf(fminf(dt_i, 0.25f * sqrtf(h / amag)), P.dt_nu);
        dt_cand = dt_valid ? fminf(dt_cand, c) : c;
        dt_valid = true;
      }
      if (ph == PH_STEP) {
        const float hdt = 0.5f * a.dyn[inst].dt_cur;
        const float4 vh = a.alt.vh[p];
        v = make_float4(vh.x + hdt * ax, vh.y + hdt * ay, vh.z + hdt * az, 0.f);
      }
    }
    acc = make_float4(ax, ay, az, divv);
    x.w = fmaxf(x.w, P.rho_floor);
    if (mo && !(f & kFreezeBit) && ph == PH_STEP) {
      const float4 o = a.x0[p];
      const float dx = x.x - o.x, dy = x.y - o.y, dz = x.z - o.z;
      mo->d = sqrtf(dx * dx + dy * dy + dz * dz) * P.inv_skin;
      mo->s = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z) * P.inv_skin;
      mo->acc = sqrtf(ax * ax + ay * ay + az * az) * P.inv_skin;
    }
  }
  a.main.pos[p] = x;
  a.main.vel[p] = v;
  a.main.acc[p] = acc;
  a.main.pid[p] = a.alt.pid[p];
  a.main.flags[p] = f;
}

__device__ __forceinline__ void copy_state(const StepArgs& a, int p) {
  a.main.pos[p] = a.alt.pos[p];
  a.main.vel[p] = a.alt.vel[p];
  a.main.acc[p] = a.alt.acc[p];
  a.main.pid[p] = a.alt.pid[p];
  a.main.flags[p] = a.alt.flags[p];
}

// ------------------------------------------------------------ hydro pass
// One thread per i-particle (the plain FP32 path).  Restates force.h:38-57
// for uniform h, m, nu within an instance:
//   a_i  = m sum_j [ -(P_i/rho_i^2 + P_j/rho_j^2 + Pi_ij) g + 4 nu g r^2 / ((rho_i+rho_j)(r^2+eps h^2)) dv ] ...
// with gradW = g dr; div v_i = -m/rho_i sum_j g (dr.dv); dt_i = C h / (c_i + v_sig).
// The epilogue adds gravity (Dam2.h:104-108), does the final kick
// (class.h:160-163), the density floor (Dam2.h:111), and folds the CFL limits
// of integral.h:2-12 into the instance's next dt.
template <bool COUNT>
__global__ void __launch_bounds__(256) k_hydro_plain(StepArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = *a.n_alive;
  const bool in = p < n;
  int inst = 0;
  float dt_cand = 0.0f;
  bool dt_valid = false;
  unsigned cnt = 0;
  if (in) {
    const uint32_t f = a.alt.flags[p];
    inst = f & kInstMask;
    const InstParams& P = a.params[inst];
    const int ph = a.phase[inst];
    if (wants_force(P, a.dyn[inst], ph)) {
      const float4 I = a.jr[p].a;
      const float4 IB = a.jr[p].b;
      const float ci = a.jC[p];
      const float rho_i = IB.w, po_i = I.w;
      float ax = 0.f, ay = 0.f, az = 0.f, dsum = 0.f, vsig = 0.f;
      const float h = P.h, eh2 = P.eh2, Kg = P.Kg, iH = P.inv_H, alpha = P.alpha, beta = P.beta, nu4 = P.nu4;
      const int vs = P.vsig_mode;
      for_each_neighbor(a, P, I.x, I.y, I.z, [&](int q, const float4& J, float dx, float dy, float dz, float r2,
                                                  uint32_t) {
        ++cnt;
        const float4 JB = __ldg(&a.jr[q].b);
        const float cj = __ldg(&a.jC[q]);
        const float rinv = rsqrtf(r2);
        const float g = spline_F(r2 * rinv * iH) * Kg * rinv;
        const float dvx = IB.x - JB.x, dvy = IB.y - JB.y, dvz = IB.z - JB.z;
        const float drdv = dx * dvx + dy * dvy + dz * dvz;
        const float rden = __frcp_rn(r2 + eh2);
        const float mu = drdv < 0.0f ? h * drdv * rden : 0.0f;
        const float rs = __frcp_rn(rho_i + JB.w);
        const float av = (beta * mu - alpha * 0.5f * (ci + cj)) * mu * 2.0f * rs;
        vsig = vs ? fmaxf(vsig, -mu) : fmaxf(vsig, mu);
        const float pg = (po_i + J.w + av) * g;
        const float visc = nu4 * g * r2 * rs * rden;
        ax += visc * dvx - pg * dx;
        ay += visc * dvy - pg * dy;
        az += visc * dvz - pg * dz;
        dsum += g * drdv;
      });
      finish_hydro(a, p, P, inst, ph, f, ax, ay, az, dsum, vsig, cnt, dt_cand, dt_valid);
      if (f & kGhostBit) cnt = 0;  // pairs are counted for owned particles only
    } else {
      copy_state(a, p);
    }
  }
  dt_min(a.dyn, inst, dt_cand, dt_valid);
  if (COUNT) {
    unsigned long long c = cnt;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(a.pair_count, c);
  }
}

// Dead tail [n_alive, n_host): carry the slots over to main unchanged so that
// removed particles keep their last state until the host compacts.
__global__ void k_copy_dead(StepArgs a) {
  const int p = *a.n_alive + blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n_host) return;
  a.main.pos[p] = a.alt.pos[p];
  a.main.vel[p] = a.alt.vel[p];
  a.main.acc[p] = a.alt.acc[p];
  a.main.pid[p] = a.alt.pid[p];
  a.main.flags[p] = a.alt.flags[p];
}

// Initial Shepard filter of main.cpp:75 (after the initial hydro pass).
__global__ void k_apply_init_filter(StepArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= *a.n_alive) return;
  const int inst = a.main.flags[p] & kInstMask;
  const InstParams& P = a.params[inst];
  if (a.phase[inst] != PH_INIT || P.density_mode != WCSPH_DENSITY_SHEPARD) return;
  a.main.pos[p].w = fmaxf(a.rho_new[p], P.rho_floor);
}

}  // namespace wcsph

// Neighbour-list steps (wcsph_sim_options.list_interval > 0).
//
// A build step is an ordinary step whose tiled kernel only scans: it writes,
// for every particle, the candidates within 2h + skin (the list radius), and
// the pair terms are summed by the list pass (k_hydro_list); its permutation
// records the positions x0 the lists refer to.  The steps up to the next
// build skip the binning sort and the candidate scan:
//   k_kick_refresh  KDK first half in place (periodic wrapping waits for the
//                 next build, so that the lists' image shifts stay valid),
//                 EoS j-records refreshed, |x - x0| checked
//   k_density_list, k_eos   the density pass from the lists, when one is due
//   k_hydro_list  the pair terms over each particle's list (thread per
//                 particle), every entry tested for 0 < r^2 < (2h)^2 on the
//                 current positions, then the shared epilogue
// A pair within the support now was within 2h + |dx_i| + |dx_j| at the
// build, so the lists hold every pair the support test can accept while no
// particle has moved more than skin / 2 since the build.  Whether a step
// builds is decided on the device at the start of the step (k_list_set): a
// build is due when the lists are stale (the host asks), the last build
// overflowed, list_interval steps have passed, or a particle could end this
// step's drift 0.45 skin or more from where the lists were built (bounded
// from the motion the last list pass recorded and the step's dt).  In the
// step's CUDA graph the decision selects one branch of a conditional node;
// without a graph the host reads it.  A displacement beyond skin / 2 at a list
// step would still set a sticky error that the next wcsph_sim_step reports.
#pragma once
#include "sim_tiled.cuh"

namespace wcsph {

constexpr int kListMaxEntries = 192;  // entries per list (the solver's list_max; the dam break needs up to ~140)
static_assert(kListMaxEntries % 4 == 0, "list rows are padded to whole groups of four entries");

// The padding slot (index max_particles, past every particle's slot) that
// list rows are padded with: records that no support test accepts and that
// no band or far test sends to the FP32 record.  FP32 position 1e30 (r^2
// overflows to inf, as for a removed particle), compact position one cell
// edge into the (+1, +1, +1) neighbour cell of the padding entry's offset
// (more than 1.4 cell edges from any i on every axis), zero velocity,
// density 1, P/rho^2 and c 0.
__global__ void k_list_pad_slot(JRec* jr, float* jC, float* jpo, uint4* jh, int d) {
  jr[d].a = make_float4(1.0e30f, 1.0e30f, 1.0e30f, 0.f);
  jr[d].b = make_float4(0.f, 0.f, 0.f, 1.f);
  jC[d] = 0.f;
  if (jpo) jpo[d] = 0.f;
  if (jh) jh[d] = make_uint4(0xffffffffu, 0x8000ffffu, 0x80008000u, __float_as_uint(1.0f));
}
// List entries naming the padding slot d: the FP32 list's image code 13 (no
// shift), or the half2 list's neighbour-cell offset (+1, +1, +1).
inline uint32_t list_pad_entry(int d, bool h16) {
  return h16 ? (uint32_t)d | (42u << kH16SlotBits) : (uint32_t)d | (13u << 27);
}

constexpr float kListRebuildAt = 0.45f;  // predicted displacement / skin that makes a step build
// In a build that happens anyway, an instance that has used this much of its
// skin gets new lists too: instances rebuild together instead of one build
// (and one sort of every particle) per instance.
constexpr float kListJoinAt = 0.225f;

// Warp-aggregated maxima of a particle's motion into its instance's words.
__device__ __forceinline__ void motion_max(unsigned* w, int inst, const Motion& m) {
  const unsigned full = 0xffffffffu;
  const unsigned bd = __float_as_uint(m.d), bs = __float_as_uint(m.s), ba = __float_as_uint(m.acc);
  const int inst0 = __shfl_sync(full, inst, 0);
  if (__all_sync(full, inst == inst0 || (bd | bs | ba) == 0u)) {
    const unsigned md = __reduce_max_sync(full, bd), ms = __reduce_max_sync(full, bs), ma = __reduce_max_sync(full, ba);
    if ((threadIdx.x & 31) == 0 && (md | ms | ma)) {
      atomicMax(&w[3 * inst0], md);
      atomicMax(&w[3 * inst0 + 1], ms);
      atomicMax(&w[3 * inst0 + 2], ma);
    }
  } else if (bd | bs | ba) {
    atomicMax(&w[3 * inst], bd);
    atomicMax(&w[3 * inst + 1], bs);
    atomicMax(&w[3 * inst + 2], ba);
  }
}

// Velocity quantum of the compact records for speeds below vb: 2^-15 of the
// smallest power of two above max(vb, c0 2^-12).
__device__ __forceinline__ float velocity_quantum(float vb, float c0) {
  const float v = fmaxf(vb, c0 * (1.0f / 4096.0f));
  return __uint_as_float(((__float_as_uint(v) >> 23) + 1u - 15u) << 23);
}

// One thread, after k_step_begin: the step's build decision, the counters,
// and (in a graph) the condition of the node that selects the build or the
// list-step branch.  An instance needs new lists when the largest
// displacement its particles can reach in this step, d + dt s + dt^2/2 acc
// from the motion the last list pass recorded, reaches kListRebuildAt skins.
// The build is full (every instance, removed particles compacted) when the
// host asks for it, the last build overflowed, list_interval steps have
// passed since the last full build, a particle was removed since, or every
// instance needs new lists; otherwise it is partial: the instances that do
// not need new lists keep them (inst_keep), their particles keep their cells
// and slots, and the step re-sorts and scans the others.  With compact
// records the same motion bounds this step's velocities, s + dt acc, which
// sets the instance's velocity quantum (kept when there is no motion yet).
__global__ void k_list_set(StepArgs a, int interval, cudaGraphConditionalHandle cond, int use_cond) {
  unsigned* lf = a.list_flags;
  int need = 0, live = 0;
  for (int k = 0; k < a.n_inst; ++k) {
    const InstParams& P = a.params[k];
    const float dt = a.dyn[k].dt_cur;
    unsigned* w = a.inst_motion + 3 * k;
    bool moved = false, near = false;
    if (P.active && P.inv_skin > 0.0f && a.phase[k] == PH_STEP && dt > 0.0f) {
      const float reach = __uint_as_float(w[0]) + dt * __uint_as_float(w[1]) + 0.5f * dt * dt * __uint_as_float(w[2]);
      moved = reach >= kListRebuildAt;
      near = reach >= kListJoinAt;
      if (a.jh && (w[1] | w[2])) {
        const float vb = (__uint_as_float(w[1]) + dt * __uint_as_float(w[2])) / P.inv_skin;
        a.dyn[k].vq = velocity_quantum(vb * 1.001f, P.c0);
      }
    }
    if (P.active) {
      ++live;
      need += moved;
    }
    a.inst_keep[k] = moved ? 0 : (near ? 2 : 1);  // read only in a partial build (2: joins one)
    w[0] = w[1] = w[2] = 0u;  // refilled by this step's list pass
  }
  const bool overflowed = lf[kLfOverflowPending] != 0u;
  const bool full = lf[kLfForce] != 0u || overflowed || (int)lf[kLfSince] >= interval || lf[kLfDeaths] != 0u ||
                    (need > 0 && need == live);
  const bool build = full || need > 0;
  if (overflowed) ++lf[kLfOverflows];
  if (build) {
    ++lf[kLfBuilds];
    lf[kLfForce] = 0u;
    lf[kLfOverflowPending] = 0u;
  } else {
    ++lf[kLfListSteps];
  }
  if (full) {
    lf[kLfSince] = 1u;
    lf[kLfDeaths] = 0u;
  } else {
    ++lf[kLfSince];
  }
  if (build && !full) ++lf[kLfPartials];
  for (int k = 0; k < a.n_inst; ++k)  // only a partial build keeps lists, and the instances near the bound join it
    a.inst_keep[k] = (!build || full || a.inst_keep[k] == 2) ? 0 : a.inst_keep[k];
  lf[kLfPartial] = (build && !full) ? 1u : 0u;
  lf[kLfDecision] = build ? 1u : 0u;
  if (use_cond) cudaGraphSetConditional(cond, build ? 1u : 0u);
}

// A list step's kick (kick_particle, no wrapping), in place in the build's
// order, with the EoS j-records refreshed and |x - x0| checked.  List steps
// run on one buffer set (alt = main): every particle's state is read and
// written by its own thread only, so the list pass updates it in place too.
__global__ void k_kick_refresh(StepArgs a, cudaGraphConditionalHandle dens_cond, int use_dens_cond) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  // in the step graph: open the density pass's conditional node when some
  // instance has a density pass due (k_step_begin set dens_any)
  if (p == 0 && use_dens_cond) cudaGraphSetConditional(dens_cond, *a.dens_any ? 1u : 0u);
  if (p >= a.n_host) return;
  uint32_t f = a.main.flags[p];
  const int inst = f & kInstMask;
  const InstParams& P = a.params[inst];
  bool dead = (f & kDeadBit) || !P.active;
  float4 x = a.main.pos[p];
  float4 v = a.main.vel[p];
  float4 vh = v;
  if (!dead && kick_particle(a, P, inst, p, f, x, v, vh, dead)) {
    a.main.pos[p] = x;
    a.main.vel[p] = v;
  }
  a.main.vh[p] = vh;
  if (dead && !(f & kDeadBit)) {
    a.main.flags[p] = f | kDeadBit;
    atomicOr(&a.list_flags[kLfDeaths], 1u);  // the next build compacts it: in full
  }
  if (!dead) {
    float pres, snds;
    tait(P, x.w, pres, snds);
    const float po = pres / (x.w * x.w);
    a.jr[p].a = make_float4(x.x, x.y, x.z, po);
    a.jr[p].b = make_float4(v.x, v.y, v.z, x.w);
    a.jC[p] = snds;
    if (a.jpo) a.jpo[p] = po;
    const float4 o = a.x0[p];
    if (a.jh)  // compact record relative to the particle's cell at the build
      write_h16(a.jh, P, a.dyn[inst].vq, p, x, v, x.w, cell_of(o.x, P.lo[0], P.inv_cell[0], P.ncell[0]),
                cell_of(o.y, P.lo[1], P.inv_cell[1], P.ncell[1]), cell_of(o.z, P.lo[2], P.inv_cell[2], P.ncell[2]));
    const float dx = x.x - o.x, dy = x.y - o.y, dz = x.z - o.z;
    const float r = sqrtf(dx * dx + dy * dy + dz * dz) * P.inv_skin;
    if (r > 0.5f) atomicOr(&a.list_flags[kLfErr], 1u);  // a pair may be missing from the lists
  } else {  // removed: never in anyone's support again
    a.jr[p].a = make_float4(1.0e30f, 1.0e30f, 1.0e30f, 0.f);
    a.jr[p].b = make_float4(0.f, 0.f, 0.f, 1.f);
    a.jC[p] = 0.f;
    if (a.jh) write_h16_dead(a.jh, p);
    if (a.jpo) a.jpo[p] = 0.f;
  }
}

// The build cell of slot p (its position x0 at the last list build).
__device__ __forceinline__ void build_cell(const StepArgs& a, const InstParams& P, int p, int c[3]) {
  const float4 o = a.x0[p];
  c[0] = cell_of(o.x, P.lo[0], P.inv_cell[0], P.ncell[0]);
  c[1] = cell_of(o.y, P.lo[1], P.inv_cell[1], P.ncell[1]);
  c[2] = cell_of(o.z, P.lo[2], P.inv_cell[2], P.ncell[2]);
}

// Neighbour-cell offsets + 1 (0, 1, 2 per axis) of a half2 list entry.
__device__ __forceinline__ void h16_offsets(uint32_t e, uint32_t& ox1, uint32_t& oy1, uint32_t& oz1) {
  ox1 = (e >> kH16SlotBits) & 3u;
  oy1 = (e >> (kH16SlotBits + 2)) & 3u;
  oz1 = e >> (kH16SlotBits + 4);
}

// Periodic image shift of a half2 list entry for a particle in build cell c:
// the neighbour cell c + o wraps past an edge on an axis exactly where the
// image code of the FP32 list build would name a shift.
__device__ __forceinline__ void offset_shift(const InstParams& P, const int c[3], uint32_t e, float& sx, float& sy,
                                             float& sz) {
  uint32_t o1[3];
  h16_offsets(e, o1[0], o1[1], o1[2]);
  float sh[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int q = c[d] + (int)o1[d] - 1;
    sh[d] = q < 0 ? -P.L[d] : (q >= P.ncell[d] ? P.L[d] : 0.0f);
  }
  sx = sh[0], sy = sh[1], sz = sh[2];
}

// Density pass over the lists: k_density_plain's sums (summation, or the
// Shepard filter of force.h:12-29) over each particle's list entries that are
// within the support now, one thread per particle walking its own list row
// four entries per 16-byte load.  Particles removed since the build keep
// their density.  H16: the entries carry offset codes (half2 list build).
template <bool H16>
__global__ void __launch_bounds__(128) k_density_list(StepArgs a) {
  if (a.dens_any && !*a.dens_any) return;  // no density pass in this launch
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= *a.n_alive) return;
  const uint32_t fp = a.alt.flags[p];
  const int inst = fp & kInstMask;
  const InstParams& P = a.params[inst];
  const int kind = density_kind(a, P, a.dyn[inst], a.phase[inst]);
  if (!kind) return;
  if (fp & kDeadBit) {
    a.rho_new[p] = a.alt.pos[p].w;
    return;
  }
  const bool shep = kind == 2;
  const float iH = P.inv_H, H2 = P.H2;
  const float4 I = a.jr[p].a;
  const float rho_i = a.jr[p].b.w;
  // a list that overflowed at this step's build: k_density_plain sums it over
  // the cell search (density_overflow_only), and the next step builds again
  if (a.list_cnt[p] > a.list_max) return;
  const int n = min(a.list_cnt[p], a.list_max);
  const uint4* row = reinterpret_cast<const uint4*>(a.list + (size_t)p * a.list_max);
  int ci[3] = {0, 0, 0};
  if (H16 && P.periodic) build_cell(a, P, p, ci);
  float sum = 0.f, one = 0.f;
  for (int k = 0; k < n; k += 4) {
    const uint4 e4 = __ldg(&row[k >> 2]);
    const uint32_t ent[4] = {e4.x, e4.y, e4.z, e4.w};
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (k + u < n) {
        const int q = ent[u] & (H16 ? kH16SlotMask : kSlotMask);
        const float4 J = __ldg(&a.jr[q].a);
        float sx = 0.f, sy = 0.f, sz = 0.f;
        if (P.periodic) {
          if (H16) offset_shift(P, ci, ent[u], sx, sy, sz);
          else entry_shift(P, ent[u] >> 27, sx, sy, sz);
        }
        const float dx = __fsub_rn(I.x, __fadd_rn(J.x, sx));
        const float dy = __fsub_rn(I.y, __fadd_rn(J.y, sy));
        const float dz = __fsub_rn(I.z, __fadd_rn(J.z, sz));
        const float r2 = dist2(dx, dy, dz);
        if (r2 > 0.0f && r2 < H2) {
          const float w = spline_w(sqrtf(r2) * iH);
          sum += w;
          if (shep) one += w / __ldg(&a.jr[q].b.w);
        }
      }
    }
  }
  const float t = 0.5f + sum;  // self term: w(0) = 1/2
  a.rho_new[p] = shep ? t / (0.5f / rho_i + one) : P.mass * P.Kw * t;
}

inline int launch_density_list(const StepArgs& a, int n, cudaStream_t s, bool h16) {
  if (n <= 0) return 0;
  if (h16) k_density_list<true><<<(n + 127) / 128, 128, 0, s>>>(a);
  else k_density_list<false><<<(n + 127) / 128, 128, 0, s>>>(a);
  WCSPH_CUDA(cudaGetLastError());
  return 0;
}

// snds7 of the two densities in the f32x2 halves, bit-identical to snds7.
__device__ __forceinline__ f2 snds7_2(f2 RHO, f2 RHO0, f2 IRHO0, f2 C0) {
  const f2 X = add2(dup(1.0f), mul2(sub2(RHO, RHO0), IRHO0));
  const f2 T = mul2(C0, mul2(mul2(X, X), X));
  return pk(fmaxf(fabsf(lo(T)), 1.0e-8f), fmaxf(fabsf(hi(T)), 1.0e-8f));
}

// i-side operands of the half2 list pass: i's position relative to the
// centre of its build cell (FP32, exact: the two are within a factor of two),
// the scales -cell / 2^15 that turn the 16-bit offsets into lengths, the
// instance's velocity quantum, the band of squared distances that take the
// FP32 record, half of (2h)^2, and i's slot (the rare FP32-record entries
// read i's FP32 position and build cell again instead of holding them).
struct H16I {
  f2 QX, QY, QZ, SX, SY, SZ, VQ, B;
  float band, hm;
  int slot;
};

// (rho / rho0)^7 - 1 in Horner form and P / rho^2 of the two densities
// (the Tait pressure of tait(), clamped at 0; rho^-2 by the fast quotient, so
// within FP32 rounding of the stored value).
__device__ __forceinline__ f2 po7_2(f2 RHO, f2 RHO0, f2 IRHO0, f2 B) {
  const f2 D = mul2(sub2(RHO, RHO0), IRHO0);
  f2 X = add2(D, dup(7.0f));
  X = fma2(D, X, dup(21.0f));
  X = fma2(D, X, dup(35.0f));
  X = fma2(D, X, dup(35.0f));
  X = fma2(D, X, dup(21.0f));
  X = fma2(D, X, dup(7.0f));
  X = mul2(mul2(D, X), B);
  const f2 R2 = mul2(RHO, RHO);
  return pk(__fdividef(fmaxf(lo(X), 0.0f), lo(R2)), __fdividef(fmaxf(hi(X), 0.0f), hi(R2)));
}

// Neighbour-cell offsets + 1 of a half2 list entry's 6-bit code (entry >> 26),
// each shifted to bits 15-16 as h16_pair2 adds them: (x, y, z, 0).  Filled by
// each block of the half2 list pass's table shapes (OFT).
__shared__ uint4 s_h16_off[64];

// 2^23 + the 16 bits of w selected by s (0x7610 low, 0x7632 high) as a float:
// byte-permuted under the exponent of 2^23.
__device__ __forceinline__ float h16_magic(uint32_t w, uint32_t s) { return __uint_as_float(__byte_perm(w, 0x4B000000u, s)); }

// Two list entries (halves a, b) of the half2 list pass, from their 16-byte
// records Qa, Qb.  The displacement of j from i is rebuilt from the 16-bit
// offsets: x_i - x_j = q_i - (o + q_j) cell, with o the entry's neighbour-cell
// offset; the biased offset and o + 1 (shifted to 2^15) are added as integers
// under the exponent of 2^23, so one packed subtraction turns them into an
// exact (q_j + o) 2^15.  Velocities come the same way, times the velocity
// quantum (exact); P/rho^2 is gathered from its 4-byte array (jpo: the
// FP32 record's value) and c recomputed from the FP32 density.  An
// entry takes the FP32 record instead (the displacement exactly as the FP32
// path and the oracle round it, and j's FP32 velocity and density) when its
// squared distance lies within the band where the 16-bit positions cannot
// decide 0 < r^2 < (2h)^2, or when j is marked far: the pairs summed, and the
// neighbour counts, are exactly those of the FP32 support test.  OFT: the
// offsets from s_h16_off (one shared load) instead of shifts and masks of the
// entry; POR: P/rho^2 recomputed from the density for gamma = 7 instead of
// gathered.  Which costs less depends on whether the L1 data pipe (shared and
// global loads) or instruction issue binds, so both are launch shapes.
template <bool OFT, bool POR>
__device__ __forceinline__ void h16_pair2(const StepArgs& a, const InstParams& P, const PairC& C, const PairI& I,
                                          const H16I& H, const uint4& Qa, const uint4& Qb, uint32_t ea, uint32_t eb,
                                          bool qva, bool qvb, bool g7, f2 RHO0, f2 IRHO0, f2 C0, f2& AX, f2& AY,
                                          f2& AZ, f2& DS, float& vsa, float& vsb, unsigned& na, unsigned& nb) {
  const f2 MAG = dup(8388608.0f + 65536.0f), MAGV = dup(8388608.0f + 32768.0f);
  constexpr uint32_t kLo = 0x7610u, kHi = 0x7632u, kO = 0x18000u;  // o + 1 at bits 15-16
  uint4 Oa, Ob;
  if (OFT) {
    Oa = s_h16_off[ea >> kH16SlotBits], Ob = s_h16_off[eb >> kH16SlotBits];
  } else {
    Oa = make_uint4((ea >> (kH16SlotBits - 15)) & kO, (ea >> (kH16SlotBits - 13)) & kO,
                    (ea >> (kH16SlotBits - 11)) & kO, 0u);
    Ob = make_uint4((eb >> (kH16SlotBits - 15)) & kO, (eb >> (kH16SlotBits - 13)) & kO,
                    (eb >> (kH16SlotBits - 11)) & kO, 0u);
  }
  const f2 TX = sub2(pk(__uint_as_float(__float_as_uint(h16_magic(Qa.x, kLo)) + Oa.x),
                        __uint_as_float(__float_as_uint(h16_magic(Qb.x, kLo)) + Ob.x)),
                     MAG);
  const f2 TY = sub2(pk(__uint_as_float(__float_as_uint(h16_magic(Qa.x, kHi)) + Oa.y),
                        __uint_as_float(__float_as_uint(h16_magic(Qb.x, kHi)) + Ob.y)),
                     MAG);
  const f2 TZ = sub2(pk(__uint_as_float(__float_as_uint(h16_magic(Qa.y, kLo)) + Oa.z),
                        __uint_as_float(__float_as_uint(h16_magic(Qb.y, kLo)) + Ob.z)),
                     MAG);
  f2 DX = fma2(TX, H.SX, H.QX), DY = fma2(TY, H.SY, H.QY), DZ = fma2(TZ, H.SZ, H.QZ);
  f2 R2raw = fma2(DZ, DZ, fma2(DY, DY, mul2(DX, DX)));
  f2 VXJ = mul2(sub2(pk(h16_magic(Qa.y, kHi), h16_magic(Qb.y, kHi)), MAGV), H.VQ);
  f2 VYJ = mul2(sub2(pk(h16_magic(Qa.z, kLo), h16_magic(Qb.z, kLo)), MAGV), H.VQ);
  f2 VZJ = mul2(sub2(pk(h16_magic(Qa.z, kHi), h16_magic(Qb.z, kHi)), MAGV), H.VQ);
  const bool fa = Qa.w == kFarRho, fb = Qb.w == kFarRho;
  float r2a = lo(R2raw), r2b = hi(R2raw);
  // |(|r^2 - (2h)^2/2|) - (2h)^2/2| < band: r^2 within the band of 0 or of
  // (2h)^2 (two roundings of at most ulp((2h)^2) / 4, inside the band's margin)
  const bool xa = qva && (fa || fabsf(fabsf(r2a - H.hm) - H.hm) < H.band);
  const bool xb = qvb && (fb || fabsf(fabsf(r2b - H.hm) - H.hm) < H.band);
  // a far record's density (0) is replaced by its FP32 record's (exact path)
  float rja = __uint_as_float(Qa.w), rjb = __uint_as_float(Qb.w);
  if (xa || xb) {  // rare: the exact FP32 record, as the FP32 path reads it
    float dx[2] = {lo(DX), hi(DX)}, dy[2] = {lo(DY), hi(DY)}, dz[2] = {lo(DZ), hi(DZ)}, r2[2] = {r2a, r2b};
    float rj[2] = {rja, rjb}, vx[2] = {lo(VXJ), hi(VXJ)}, vy[2] = {lo(VYJ), hi(VYJ)}, vz[2] = {lo(VZJ), hi(VZJ)};
    const bool ex[2] = {xa, xb};
    const uint32_t e[2] = {ea, eb};
    const float4 Xi = __ldg(&a.jr[H.slot].a);
    int c[3] = {0, 0, 0};
    if (P.periodic) build_cell(a, P, H.slot, c);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (!ex[h]) continue;
      const JRec R = ld_jrec(&a.jr[e[h] & kH16SlotMask]);
      float sx = 0.f, sy = 0.f, sz = 0.f;
      if (P.periodic) offset_shift(P, c, e[h], sx, sy, sz);
      dx[h] = __fsub_rn(Xi.x, __fadd_rn(R.a.x, sx));
      dy[h] = __fsub_rn(Xi.y, __fadd_rn(R.a.y, sy));
      dz[h] = __fsub_rn(Xi.z, __fadd_rn(R.a.z, sz));
      r2[h] = dist2(dx[h], dy[h], dz[h]);
      rj[h] = R.b.w;
      vx[h] = R.b.x, vy[h] = R.b.y, vz[h] = R.b.z;
    }
    DX = pk(dx[0], dx[1]), DY = pk(dy[0], dy[1]), DZ = pk(dz[0], dz[1]);
    R2raw = pk(r2[0], r2[1]);
    r2a = r2[0], r2b = r2[1];
    rja = rj[0], rjb = rj[1];
    VXJ = pk(vx[0], vx[1]), VYJ = pk(vy[0], vy[1]), VZJ = pk(vz[0], vz[1]);
  }
  const bool va = qva && r2a > 0.0f && r2a < C.H2;
  const bool vb = qvb && r2b > 0.0f && r2b < C.H2;
  na += va, nb += vb;
  const f2 RHOJ = pk(rja, rjb);
  const uint32_t ga = ea & kH16SlotMask, gb = eb & kH16SlotMask;
  const f2 POJ = POR && g7 ? po7_2(RHOJ, RHO0, IRHO0, H.B)
                           : pk(__ldg(&a.jpo[ga]), __ldg(&a.jpo[gb]));  // P/rho^2 as the FP32 records hold it
  const f2 CJ = g7 ? snds7_2(RHOJ, RHO0, IRHO0, C0) : pk(__ldg(&a.jC[ga]), __ldg(&a.jC[gb]));
  pair_terms2(C, I, DX, DY, DZ, R2raw, va, vb, VXJ, VYJ, VZJ, POJ, RHOJ, CJ, AX, AY, AZ, DS, vsa, vsb);
}

// The list pass over particle slots below the build's live count (the
// particles of the build's cell table; the dead tail is k_copy_dead's), on
// list steps and right after the scan of a build step: TPI threads per
// particle walk its list row, each taking every TPI-th group of four entries
// (one 16-byte load), and sum two entries at a time in the f32x2 halves of
// pair2, support tested per entry; the TPI partial sums are combined with
// shuffles, and no shared memory is used.  For gamma = 7 the sound speed of j
// is recomputed from its density (snds7_2, the stored value bit for bit)
// instead of gathered: one gather per entry fewer.  MINB is the launch
// bound's blocks per SM (it sets the register budget).  With TPI = 1 every
// sum runs in list order; TPI = 2 changes the summation order (the results
// agree to FP32 rounding).  The half2 pass (H16) reads every group of four
// whole: rows are padded with the padding slot's entry (k_list_pad_slot);
// OFT and POR choose how it gets the neighbour-cell offsets and P/rho^2
// (h16_pair2).  The FP32 pass keeps its per-entry selects of i's own record
// for the entries past n, which fit its 96 registers without spilling.
template <bool H16, int TPI, bool OFT = false, bool POR = false>
__device__ __forceinline__ void hydro_list_body(const StepArgs& a) {
  const unsigned full = 0xffffffffu;
  if (H16 && OFT) {  // before any thread leaves: the offset table of the half2 entries
    if (threadIdx.x < 64) {
      const uint32_t c = threadIdx.x;
      s_h16_off[c] = make_uint4((c & 3u) << 15, ((c >> 2) & 3u) << 15, (c >> 4) << 15, 0u);
    }
    __syncthreads();
  }
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int p = t / TPI, sub = t % TPI;
  float dt_cand = 0.f;
  bool dt_valid = false;
  int inst = 0;
  unsigned owned = 0;
  bool work = false;
  uint32_t fp = 0;
  float sx = 0.f, sy = 0.f, sz = 0.f, sd = 0.f, sv = 0.f;
  unsigned scnt = 0;
  if (p < *a.n_alive) {
    fp = a.alt.flags[p];
    inst = fp & kInstMask;
    const InstParams& P = a.params[inst];
    const int ph = a.phase[inst];
    if ((fp & kDeadBit) || !wants_force(P, a.dyn[inst], ph)) {
      if (sub == 0) copy_state(a, p);
    } else {
      work = true;
      const JRec R = a.jr[p];
      PairI I;
      I.X = dup(R.a.x), I.Y = dup(R.a.y), I.Z = dup(R.a.z), I.PO = dup(R.a.w);
      I.VX = dup(R.b.x), I.VY = dup(R.b.y), I.VZ = dup(R.b.z), I.RHO = dup(R.b.w);
      I.CI = dup(a.jC[p]);
      const PairC C = pair_consts(P);
      const bool g7 = P.gamma == 7.0f;
      const f2 RHO0 = dup(P.rho0), IRHO0 = dup(P.inv_rho0), C0 = dup(P.c0);
      const int cnt_build = a.list_cnt[p];
      const int n = cnt_build <= a.list_max ? cnt_build : 0;
      const uint4* row = reinterpret_cast<const uint4*>(a.list + (size_t)p * a.list_max);
      f2 AX = 0ull, AY = 0ull, AZ = 0ull, DS = 0ull;
      float vsa = 0.f, vsb = 0.f;
      unsigned ca = 0, cb = 0;
      if (cnt_build > a.list_max && sub == 0) {
        // The list overflowed at this step's build (the host rebuilds at the
        // next step, so no list step ever sees it): sum over the cell search
        // of the build's cell table instead, one j at a time.
        for_each_neighbor(a, P, R.a.x, R.a.y, R.a.z,
                          [&](int q, const float4&, float, float, float, float, uint32_t code) {
                            const JRec Rq = ld_jrec(&a.jr[q]);
                            const float cq = g7 ? lo(snds7_2(dup(Rq.b.w), RHO0, IRHO0, C0)) : __ldg(&a.jC[q]);
                            pair2<false>(P, C, I, Rq, R, code, 13u, dup(cq), true, false, AX, AY, AZ, DS, vsa, vsb,
                                         ca, cb);
                            ++ca;
                          });
      }
      if (H16) {  // compact records
        H16I H;
        int bc[3];
        build_cell(a, P, p, bc);
        H.QX = dup(R.a.x - cell_centre(P, 0, bc[0]));
        H.QY = dup(R.a.y - cell_centre(P, 1, bc[1]));
        H.QZ = dup(R.a.z - cell_centre(P, 2, bc[2]));
        H.SX = dup(-P.cell[0] / kQ16Scale), H.SY = dup(-P.cell[1] / kQ16Scale), H.SZ = dup(-P.cell[2] / kQ16Scale);
        H.VQ = dup(a.dyn[inst].vq);
        H.band = P.h16_band;
        H.hm = 0.5f * C.H2;
        H.slot = p;
        H.B = dup(P.B);
        // entries past n up to the end of the group of four name the padding
        // slot, which no support, band or far test accepts
        for (int k = 4 * sub; k < n; k += 4 * TPI) {
          const uint4 e = __ldg(&row[k >> 2]);
          const uint4 Q0 = __ldg(&a.jh[e.x & kH16SlotMask]), Q1 = __ldg(&a.jh[e.y & kH16SlotMask]);
          const uint4 Q2 = __ldg(&a.jh[e.z & kH16SlotMask]), Q3 = __ldg(&a.jh[e.w & kH16SlotMask]);
          h16_pair2<OFT, POR>(a, P, C, I, H, Q0, Q1, e.x, e.y, true, true, g7, RHO0, IRHO0, C0, AX, AY, AZ, DS, vsa,
                              vsb, ca, cb);
          h16_pair2<OFT, POR>(a, P, C, I, H, Q2, Q3, e.z, e.w, true, true, g7, RHO0, IRHO0, C0, AX, AY, AZ, DS, vsa,
                              vsb, ca, cb);
        }
      } else {
        // idle halves past n read i's own record (weight 0): this loop keeps
        // its selects, which leave the FP32 pass within 96 registers
        const uint32_t self = (uint32_t)p | (13u << 27);
        for (int k = 4 * sub; k < n; k += 4 * TPI) {
          const uint4 e = __ldg(&row[k >> 2]);
          const uint32_t e0 = e.x, e1 = k + 1 < n ? e.y : self, e2 = k + 2 < n ? e.z : self,
                         e3 = k + 3 < n ? e.w : self;
          const int g0 = e0 & kSlotMask, g1 = e1 & kSlotMask, g2 = e2 & kSlotMask, g3 = e3 & kSlotMask;
          const JRec R0 = ld_jrec(&a.jr[g0]), R1 = ld_jrec(&a.jr[g1]);
          const JRec R2 = ld_jrec(&a.jr[g2]), R3 = ld_jrec(&a.jr[g3]);
          f2 C01, C23;
          if (g7) {  // c_j from rho_j: no gather of c
            C01 = snds7_2(pk(R0.b.w, R1.b.w), RHO0, IRHO0, C0);
            C23 = snds7_2(pk(R2.b.w, R3.b.w), RHO0, IRHO0, C0);
          } else {
            C01 = pk(__ldg(&a.jC[g0]), __ldg(&a.jC[g1])), C23 = pk(__ldg(&a.jC[g2]), __ldg(&a.jC[g3]));
          }
          pair2<true>(P, C, I, R0, R1, e0 >> 27, e1 >> 27, C01, true, k + 1 < n, AX, AY, AZ, DS, vsa, vsb, ca, cb);
          pair2<true>(P, C, I, R2, R3, e2 >> 27, e3 >> 27, C23, k + 2 < n, k + 3 < n, AX, AY, AZ, DS, vsa, vsb, ca,
                      cb);
        }
      }
      sx = lo(AX) + hi(AX), sy = lo(AY) + hi(AY), sz = lo(AZ) + hi(AZ), sd = -(lo(DS) + hi(DS));  // DS: -sum g dr.dv
      sv = fmaxf(vsa, vsb);
      scnt = ca + cb;
    }
  }
#pragma unroll
  for (int o = 1; o < TPI; o <<= 1) {  // every lane takes part; a particle's TPI lanes are adjacent
    sx += __shfl_xor_sync(full, sx, o);
    sy += __shfl_xor_sync(full, sy, o);
    sz += __shfl_xor_sync(full, sz, o);
    sd += __shfl_xor_sync(full, sd, o);
    sv = fmaxf(sv, __shfl_xor_sync(full, sv, o));
    scnt += __shfl_xor_sync(full, scnt, o);
  }
  Motion mo;
  if (work && sub == 0) {
    const InstParams& P = a.params[inst];
    if (!(fp & kGhostBit)) owned = scnt;  // owned particles only
    finish_hydro(a, p, P, inst, a.phase[inst], fp, sx, sy, sz, sd, sv, scnt, dt_cand, dt_valid, &mo);
  }
  dt_min(a.dyn, inst, dt_cand, dt_valid);
  motion_max(a.inst_motion, inst, mo);
  const unsigned tot = __reduce_add_sync(full, owned);
  if ((threadIdx.x & 31) == 0 && tot) atomicAdd(a.pair_count, (unsigned long long)tot);
}

template <bool H16, int TPI, int MINB, bool OFT = false, bool POR = false>
__global__ void __launch_bounds__(128, MINB) k_hydro_list(StepArgs a) {
  hydro_list_body<H16, TPI, OFT, POR>(a);
}

// Launch shapes of the list pass the autotuner chooses among: (threads per
// particle, blocks of 128 per SM of the launch bound, which sets the register
// budget: 96 or 128).  Shapes 0 and 2 sum in one order (bit-identical
// results), shapes 1 and 3 in another.  Shapes 4-6 are shape 0 with the half2
// pass's other ways to the offsets and P/rho^2 (h16_pair2 OFT, POR): 4 the
// shared offset table, bit-identical to 0; 5 and 6 recompute P/rho^2 (FP32
// rounding of 0), with shifts or with the table.  In the FP32 pass they are
// shape 0.  (On the 1.6M dam break the half2 pass takes 0.566 ms in shape 0,
// 0.615 with the table, 0.578 and 0.589 recomputing P/rho^2.)
constexpr int kListShapes = 7;
constexpr int kListShapeTPI[kListShapes] = {1, 2, 1, 2, 1, 1, 1};
constexpr int kListShapeBlock[kListShapes] = {128, 128, 128, 128, 128, 128, 128};

template <bool H16>
inline int launch_hydro_list(const StepArgs& a, int n, cudaStream_t s, int shape = 0) {
  if (n <= 0) return 0;
  const int sh = shape < 0 || shape >= kListShapes ? 0 : shape;
  const long long threads = (long long)n * kListShapeTPI[sh];
  const int B = kListShapeBlock[sh];
  const int grid = (int)((threads + B - 1) / B);
  switch (sh) {
    case 1: k_hydro_list<H16, 2, 4><<<grid, 128, 0, s>>>(a); break;
    case 2: k_hydro_list<H16, 1, 4><<<grid, 128, 0, s>>>(a); break;
    case 3: k_hydro_list<H16, 2, 5><<<grid, 128, 0, s>>>(a); break;
    case 4:
      if (H16) k_hydro_list<true, 1, 5, true, false><<<grid, 128, 0, s>>>(a);
      else k_hydro_list<false, 1, 5><<<grid, 128, 0, s>>>(a);
      break;
    case 5:
      if (H16) k_hydro_list<true, 1, 5, false, true><<<grid, 128, 0, s>>>(a);
      else k_hydro_list<false, 1, 5><<<grid, 128, 0, s>>>(a);
      break;
    case 6:
      if (H16) k_hydro_list<true, 1, 5, true, true><<<grid, 128, 0, s>>>(a);
      else k_hydro_list<false, 1, 5><<<grid, 128, 0, s>>>(a);
      break;
    default: k_hydro_list<H16, 1, 5><<<grid, 128, 0, s>>>(a); break;
  }
  WCSPH_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace wcsph

// Tiled hydro kernel (WCSPH_PREC_TILED, WCSPH_PREC_HALF2; the two differ only
// in the entries a list build writes): one warp per non-empty cell.
//
//   1. The 27 neighbour cells of the warp's cell are flattened into one
//      candidate list and staged into the warp's shared-memory tile as
//      structure-of-arrays x[], y[], z[] (pre-shifted by the periodic image)
//      and e[] (global slot | image code << 27; the half2 list build writes
//      the neighbour-cell offset code instead), with coalesced loads (a
//      cell's particles are contiguous after the sort).
//   2. The cell's i-particles are taken two at a time.  Each lane tests two
//      adjacent candidates against both i: one 64-bit shared load yields the
//      candidate pair already packed, and the four FP32 support predicates are
//      evaluated with packed f32x2 arithmetic (bit-identical to the scalar
//      predicate).  In-support candidates are ballot-compacted into one queue
//      per i.
//   3. The two queues are consumed together, lane k taking pair k of each
//      queue (dense lanes, no predicate divergence), with the pair terms of the
//      two i-particles evaluated in packed f32x2 arithmetic; j records are
//      gathered from global memory by the slot in the queue entry (a few
//      contiguous runs, so the loads coalesce).  Partial sums are combined
//      with a butterfly reduce-scatter (9 shuffles for 8 sums) and accumulated
//      per i in shared memory.
//   4. Lane l finishes i = batch + l with the epilogue shared with the plain
//      kernel (gravity, final kick, density floor, next-dt fold, state write).
// Work distribution: a persistent grid; warp w takes the non-empty cells
// w, w + W, w + 2W, ... of the cell list (W warps in the grid), whose order
// follows the Morton sort, so neighbouring warps share L2-resident records.
// Staging is latency-bound, so it is flattened: each lane locates the source
// cell of its candidates by a binary search over the 27 range offsets and
// keeps several independent loads in flight.
#pragma once
#include <cuda_fp16.h>

#include "f32x2.cuh"
#include "sim_kernels.cuh"

namespace wcsph {

constexpr int kStageUnroll = 4;            // staging loads in flight per lane
constexpr uint32_t kSlotMask = (1u << 27) - 1;
constexpr int kMaxTiledParticles = 1 << 27;  // queue entries hold the slot in 27 bits
// Half2 list entries: the slot in the low 26 bits, the neighbour cell's offset
// + 1 per axis (0, 1, 2) in bits 26-27 (x), 28-29 (y), 30-31 (z).
constexpr int kH16SlotBits = 26;
constexpr uint32_t kH16SlotMask = (1u << kH16SlotBits) - 1;
constexpr int kMaxH16ListParticles = 1 << kH16SlotBits;

// Shared memory of a block of WARPS warps with TILE-candidate tiles
// (TILE a multiple of 64).
template <int WARPS, int TILE>
struct TiledSmem {
  float x[WARPS][TILE], y[WARPS][TILE], z[WARPS][TILE];  // staged candidates
  uint32_t e[WARPS][TILE];                   // slot | image code << 27
  uint32_t q[WARPS][2][TILE];                // per-i compacted queues of entries
  float res[WARPS][32][6];                   // per-i accumulators of the current batch
};

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Butterfly reduce-scatter of 8 per-lane sums: returns, in every lane, the
// warp total of slot ((lane >> 2) & 7).  9 shuffles instead of 40.
__device__ __forceinline__ float butterfly8(const float v[8], int lane) {
  const unsigned full = 0xffffffffu;
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
  float w[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float send = b4 ? v[k] : v[k + 4];
    const float keep = b4 ? v[k + 4] : v[k];
    w[k] = keep + __shfl_xor_sync(full, send, 16);
  }
  float x[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const float send = b3 ? w[k] : w[k + 2];
    const float keep = b3 ? w[k + 2] : w[k];
    x[k] = keep + __shfl_xor_sync(full, send, 8);
  }
  const float send = b2 ? x[0] : x[1];
  float y = (b2 ? x[1] : x[0]) + __shfl_xor_sync(full, send, 4);
  y += __shfl_xor_sync(full, y, 2);
  y += __shfl_xor_sync(full, y, 1);
  return y;
}

// Image shift of a queue entry's code ((sx+1) + 3 (sy+1) + 9 (sz+1)).
__device__ __forceinline__ void entry_shift(const InstParams& P, uint32_t code, float& sx, float& sy, float& sz) {
  sx = (float)((int)(code % 3u) - 1) * P.L[0];
  sy = (float)((int)((code / 3u) % 3u) - 1) * P.L[1];
  sz = (float)((int)(code / 9u) - 1) * P.L[2];
}

// Operands of pair2.  PairI: the i-side of the two halves (two i-particles,
// or one i duplicated); PairC: the instance constants, built once per i.
struct PairI {
  f2 X, Y, Z, VX, VY, VZ, RHO, PO, CI;
};
// The constants carry factors of pair_terms2: 3 Kg (the spline gradient,
// negated), -4 nu, 2 beta and -alpha (the factor 2 of Pi_ij moved in: exact).
struct PairC {
  float H2, iH, KgiH;
  f2 IH, KG3, EH2, HH, NNU4, BETA2, MALPHA;
  int vs;
  bool per;
};
__device__ __forceinline__ PairC pair_consts(const InstParams& P) {
  PairC c;
  c.H2 = P.H2, c.iH = P.inv_H, c.KgiH = P.Kg * P.inv_H;
  c.IH = dup(P.inv_H), c.KG3 = dup(3.0f * P.Kg), c.EH2 = dup(P.eh2), c.HH = dup(P.h);
  c.NNU4 = dup(-P.nu4), c.BETA2 = dup(2.0f * P.beta), c.MALPHA = dup(-P.alpha);
  c.vs = P.vsig_mode, c.per = P.periodic;
  return c;
}

// Pair terms of two (i, j) pairs at once, one per f32x2 half (force.h:38-57
// for uniform h, m, nu within an instance), from the displacements DX, DY,
// DZ = x_i - x_j with R2raw their squared length, j's velocity VJX..VJZ,
// P_j/rho_j^2 POJ, density RHOJ and sound speed CJ; va, vb say whether a half
// holds an in-support pair (idle halves add exactly zero).  Accumulates a_x,
// a_y, a_z, MINUS sum g dr.dv (the gradient factor is carried negated) and the
// v_sig maximum per half.
__device__ __forceinline__ void pair_terms2(const PairC& C, const PairI& I, f2 DX, f2 DY, f2 DZ, f2 R2raw, bool va,
                                            bool vb, f2 VJX, f2 VJY, f2 VJZ, f2 POJ, f2 RHOJ, f2 CJ, f2& AX, f2& AY,
                                            f2& AZ, f2& DS, float& vsa, float& vsb) {
  const f2 ONE = dup(1.0f), HALF = dup(0.5f);
  const f2 R2 = pk(va ? lo(R2raw) : C.H2, vb ? hi(R2raw) : C.H2);  // finite stand-in for idle halves
  const f2 W = pk(va ? 1.0f : 0.0f, vb ? 1.0f : 0.0f);
  // gradW = g dr with g = (12 (1/2-s)+^2 - 3 (1-s)^2) Kg / r; NG = -g = 3 Kg ((1-s)^2 - 4 (1/2-s)+^2) / r
  const f2 RINV = rsqrt2(R2);
  const f2 S = mul2(mul2(R2, RINV), C.IH);
  // 1 - s needs no clamp: s <= 1 in support and for the stand-in up to
  // rounding, and a rounding residue squared is far below FP32 resolution
  const f2 A = sub2(ONE, S), B = max0_2(sub2(HALF, S));
  const f2 NG = mul2(mul2(fma2(dup(-4.0f), mul2(B, B), mul2(A, A)), C.KG3), mul2(RINV, W));
  const f2 DVX = sub2(I.VX, VJX), DVY = sub2(I.VY, VJY), DVZ = sub2(I.VZ, VJZ);
  const f2 DRDV = fma2(DZ, DVZ, fma2(DY, DVY, mul2(DX, DVX)));
  const f2 RDEN = rcp2(add2(R2, C.EH2));
  const f2 MUr = mul2(mul2(DRDV, RDEN), C.HH);
  // mu = h dr.dv / (r^2 + eps h^2) where dr.dv < 0 (the sign of MUr), 0
  // otherwise and for idle halves (W = 0; MUr is finite there)
  const f2 MU = pk(va ? fminf(lo(MUr), 0.0f) : 0.0f, vb ? fminf(hi(MUr), 0.0f) : 0.0f);
  const f2 RS = rcp2(add2(I.RHO, RHOJ));
  // Pi_ij = (beta mu - alpha/2 (c_i + c_j)) mu 2 / (rho_i + rho_j)
  const f2 AV = mul2(mul2(fma2(C.BETA2, MU, mul2(C.MALPHA, add2(I.CI, CJ))), MU), RS);
  if (C.vs) {
    vsa = fmaxf(vsa, -lo(MU));
    vsb = fmaxf(vsb, -hi(MU));
  } else {
    vsa = fmaxf(vsa, lo(MU));
    vsb = fmaxf(vsb, hi(MU));
  }
  const f2 NPG = mul2(add2(add2(I.PO, POJ), AV), NG);                  // -(P_i/rho_i^2 + P_j/rho_j^2 + Pi_ij) g
  const f2 VISC = mul2(mul2(mul2(C.NNU4, NG), R2), mul2(RS, RDEN));  // 4 nu g r^2 / ((rho_i+rho_j)(r^2+eps h^2))
  AX = fma2(NPG, DX, fma2(VISC, DVX, AX));
  AY = fma2(NPG, DY, fma2(VISC, DVY, AY));
  AZ = fma2(NPG, DZ, fma2(VISC, DVZ, AZ));
  DS = fma2(NG, DRDV, DS);
}

// Pair terms of two (i, j) pairs at once from FP32 j-records Ra, Rb with
// image codes ea, eb (entry >> 27) and sound speeds CJ; qva, qvb say whether a
// half holds a pair (idle halves must still name a valid record; they add
// exactly zero).  CHECK: halves outside 0 < r^2 < (2h)^2 add exactly zero,
// and na, nb count the halves summed.
template <bool CHECK>
__device__ __forceinline__ void pair2(const InstParams& P, const PairC& C, const PairI& I, const JRec& Ra,
                                      const JRec& Rb, uint32_t ea, uint32_t eb, f2 CJ, bool qva, bool qvb, f2& AX,
                                      f2& AY, f2& AZ, f2& DS, float& vsa, float& vsb, unsigned& na, unsigned& nb) {
  const float4 &Ja = Ra.a, &Jb = Rb.a, &JBa = Ra.b, &JBb = Rb.b;
  float jxa = Ja.x, jya = Ja.y, jza = Ja.z, jxb = Jb.x, jyb = Jb.y, jzb = Jb.z;
  if (C.per) {  // the same rounded image position the scan tested
    float sx, sy, sz;
    entry_shift(P, ea, sx, sy, sz);
    jxa = __fadd_rn(jxa, sx), jya = __fadd_rn(jya, sy), jza = __fadd_rn(jza, sz);
    entry_shift(P, eb, sx, sy, sz);
    jxb = __fadd_rn(jxb, sx), jyb = __fadd_rn(jyb, sy), jzb = __fadd_rn(jzb, sz);
  }
  const f2 DX = sub2(I.X, pk(jxa, jxb)), DY = sub2(I.Y, pk(jya, jyb)), DZ = sub2(I.Z, pk(jza, jzb));
  const f2 R2raw = fma2(DZ, DZ, fma2(DY, DY, mul2(DX, DX)));
  const bool va = CHECK ? qva && lo(R2raw) > 0.0f && lo(R2raw) < C.H2 : qva;
  const bool vb = CHECK ? qvb && hi(R2raw) > 0.0f && hi(R2raw) < C.H2 : qvb;
  if (CHECK) na += va, nb += vb;
  pair_terms2(C, I, DX, DY, DZ, R2raw, va, vb, pk(JBa.x, JBb.x), pk(JBa.y, JBb.y), pk(JBa.z, JBb.z), pk(Ja.w, Jb.w),
              pk(JBa.w, JBb.w), CJ, AX, AY, AZ, DS, vsa, vsb);
}

// Pair terms of i_a (low half) and i_b (high half) over their queues; adds
// the warp totals into res[0] (i_a) and res[1] (i_b): ax, ay, az, sum g drdv,
// v_sig, count.  Lanes past a queue's end contribute exactly zero.
__device__ __forceinline__ void hydro_queues2(const StepArgs& a, const InstParams& P, int ia, int ib, bool has_b,
                                              const float4& IA, const float4& IBp, const uint32_t* qa, int na,
                                              const uint32_t* qb, int nb, float (*res)[6], int lane) {
  const float4 VA = __ldg(&a.jr[ia].b), VB = __ldg(&a.jr[ib].b);
  PairI I;
  I.X = pk(IA.x, IBp.x), I.Y = pk(IA.y, IBp.y), I.Z = pk(IA.z, IBp.z);
  I.VX = pk(VA.x, VB.x), I.VY = pk(VA.y, VB.y), I.VZ = pk(VA.z, VB.z);
  I.RHO = pk(VA.w, VB.w), I.PO = pk(IA.w, IBp.w);
  I.CI = pk(__ldg(&a.jC[ia]), __ldg(&a.jC[ib]));
  const PairC C = pair_consts(P);
  const int nbq = has_b ? nb : 0;
  const int n = max(na, nbq);
  f2 AX = 0ull, AY = 0ull, AZ = 0ull, DS = 0ull;
  float vsa = 0.f, vsb = 0.f;
  unsigned ca = 0, cb = 0;  // unused: every queue entry is in support
  for (int k = lane; k < n; k += 32) {
    const bool qva = k < na, qvb = k < nbq;
    // idle halves read i_a's own record (always a valid slot; weight 0 below)
    const uint32_t self = (uint32_t)ia | (13u << 27);
    const uint32_t ea = qva ? qa[k] : self, eb = qvb ? qb[k] : self;
    const int ga = ea & kSlotMask, gb = eb & kSlotMask;
    const JRec Ra = ld_jrec(&a.jr[ga]), Rb = ld_jrec(&a.jr[gb]);
    const f2 CJ = pk(__ldg(&a.jC[ga]), __ldg(&a.jC[gb]));
    pair2<false>(P, C, I, Ra, Rb, ea >> 27, eb >> 27, CJ, qva, qvb, AX, AY, AZ, DS, vsa, vsb, ca, cb);
  }
  const float v8[8] = {lo(AX), lo(AY), lo(AZ), -lo(DS), hi(AX), hi(AY), hi(AZ), -hi(DS)};  // DS holds -sum g dr.dv
  const float y = butterfly8(v8, lane);
  vsa = warp_max(vsa);
  vsb = warp_max(vsb);
  if ((lane & 3) == 0) {
    const int slot = lane >> 2;
    if (slot < 4) res[0][slot] += y;
    else if (has_b) res[1][slot - 4] += y;
  }
  if (lane == 0) {
    res[0][4] = fmaxf(res[0][4], vsa);
    res[0][5] += (float)na;
    if (has_b) {
      res[1][4] = fmaxf(res[1][4], vsb);
      res[1][5] += (float)nb;
    }
  }
}

// Append the in-support candidates (even/odd halves of the lane's pair) to a queue.
__device__ __forceinline__ void append2(uint32_t* q, int& n, bool he, bool ho, uint32_t ee, uint32_t eo, unsigned lt) {
  const unsigned me = __ballot_sync(0xffffffffu, he), mo = __ballot_sync(0xffffffffu, ho);
  const int p = n + __popc(me & lt) + __popc(mo & lt);
  if (he) q[p] = ee;
  if (ho) q[p + (he ? 1 : 0)] = eo;
  n += __popc(me) + __popc(mo);
}

// The 27 neighbour-cell ranges of cell (cx, cy, cz) of instance P, one per
// lane k < 27 (offset (k%3-1, k/3%3-1, k/9-1)): first slot, count, periodic
// image shift and entry code (the image code k, or with HL, the half2 list
// build, the neighbour-cell offset + 1 in two bits per axis: its compact
// records are relative to the build's cells), the exclusive prefix of the
// counts over the lanes and, in every lane, their total.
struct NbRanges {
  int start, excl, total;
  float shx, shy, shz;
  uint32_t code;
};
template <bool HL>
__device__ __forceinline__ NbRanges nb_ranges(const StepArgs& a, const InstParams& P, int cx, int cy, int cz,
                                              int lane) {
  const unsigned full = 0xffffffffu;
  const int nx = P.ncell[0], ny = P.ncell[1];
  NbRanges R;
  int cnt = 0;
  R.start = 0, R.shx = 0.f, R.shy = 0.f, R.shz = 0.f, R.code = 13;
  if (lane < 27) {
    int x, y, z;
    if (neighbor_cell(P, 0, cx + lane % 3 - 1, x, R.shx) && neighbor_cell(P, 1, cy + (lane / 3) % 3 - 1, y, R.shy) &&
        neighbor_cell(P, 2, cz + lane / 9 - 1, z, R.shz)) {
      const int l2 = P.cell_base + (z * ny + y) * nx + x;
      R.start = a.cell_start[l2];
      cnt = a.cell_end[l2] - R.start;
      R.code = (uint32_t)((R.shx > 0.f) - (R.shx < 0.f) + 1) + 3u * (uint32_t)((R.shy > 0.f) - (R.shy < 0.f) + 1) +
               9u * (uint32_t)((R.shz > 0.f) - (R.shz < 0.f) + 1);
    }
    if (HL) R.code = (uint32_t)(lane % 3) | ((uint32_t)((lane / 3) % 3) << 2) | ((uint32_t)(lane / 9) << 4);
  }
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(full, incl, o);
    if (lane >= o) incl += t;
  }
  R.total = __shfl_sync(full, incl, 31);
  R.excl = incl - cnt;
  return R;
}

// Stage candidates [t0, t0 + tn) of a cell's flattened neighbour ranges into
// a warp's tile: positions pre-shifted by the periodic image, entries slot |
// code (at bit 27, or with HL at bit 26), padded to a multiple of 64 with
// positions that no support test accepts.  Candidate u comes from the last
// neighbour cell k with excl_k <= u (binary search over lanes 0..26);
// kStageUnroll independent loads per lane are in flight before any store.
template <bool HL>
__device__ __forceinline__ void stage_tile(const StepArgs& a, const NbRanges& R, int t0, int tn, float* tx,
                                           float* ty, float* tz, uint32_t* te, int lane) {
  const unsigned full = 0xffffffffu;
  const int tn64 = (tn + 63) & ~63;
  for (int ub = t0; ub < t0 + tn; ub += 32 * kStageUnroll) {
    float4 J[kStageUnroll];
    int gk[kStageUnroll], kk[kStageUnroll];
#pragma unroll
    for (int r = 0; r < kStageUnroll; ++r) {
      const int u = ub + 32 * r + lane;
      int k = 0;
#pragma unroll
      for (int step = 16; step; step >>= 1) {
        const int cand = k + step;
        const int ec = __shfl_sync(full, R.excl, cand < 27 ? cand : 26);
        if (cand < 27 && ec <= u) k = cand;
      }
      const int sk = __shfl_sync(full, R.start, k), ek = __shfl_sync(full, R.excl, k);
      kk[r] = k;
      gk[r] = sk + (u - ek);
      if (u < t0 + tn) J[r] = __ldg(&a.jr[gk[r]].a);
    }
#pragma unroll
    for (int r = 0; r < kStageUnroll; ++r) {
      const int u = ub + 32 * r + lane;
      const int k = kk[r];
      const float sx = __shfl_sync(full, R.shx, k), sy = __shfl_sync(full, R.shy, k), sz = __shfl_sync(full, R.shz, k);
      const uint32_t ck = __shfl_sync(full, R.code, k) << (HL ? kH16SlotBits : 27);
      if (u < t0 + tn) {
        tx[u - t0] = __fadd_rn(J[r].x, sx);
        ty[u - t0] = __fadd_rn(J[r].y, sy);
        tz[u - t0] = __fadd_rn(J[r].z, sz);
        te[u - t0] = (uint32_t)gk[r] | ck;
      }
    }
  }
  for (int u = tn + lane; u < tn64; u += 32) {  // pad to a multiple of 64: never in support
    tx[u] = 1.0e30f;
    ty[u] = 1.0e30f;
    tz[u] = 1.0e30f;
    te[u] = 0u;
  }
}

// k_hydro_tiled keeps its own copy of the neighbour-range and staging code:
// written through these helpers it allocated registers differently and
// spilled in its 4- and 8-warp list-build shapes.

// LB (neighbour-list build): scan only.  The scan keeps the candidates
// within the list radius 2h + skin and each i's queue is written to its list
// (list_cnt holds the full count, also past the list's capacity); the pair
// terms and the epilogue are left to the list pass (k_hydro_list) that
// follows, as on the steps that reuse the lists.
template <bool H16, int WARPS, int TILE, bool LB = false>
__global__ void __launch_bounds__(WARPS * 32) k_hydro_tiled(StepArgs a) {
  constexpr int kTiledWarps = WARPS;
  constexpr int kTile = TILE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TiledSmem<WARPS, TILE>& S = *reinterpret_cast<TiledSmem<WARPS, TILE>*>(smem_raw);
  const unsigned full = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* tx = S.x[warp];
  float* ty = S.y[warp];
  float* tz = S.z[warp];
  uint32_t* te = S.e[warp];
  uint32_t* qa = S.q[warp][0];
  uint32_t* qb = S.q[warp][1];
  float(*res)[6] = S.res[warp];
  const int nrun = *a.run_count;
  const unsigned lt = lanemask_lt();
  unsigned long long pairs = 0;
  // Static round-robin over the non-empty cells (no contended counter); the
  // next cell's index is loaded one iteration ahead.
  const int stride = gridDim.x * kTiledWarps;
  int c = blockIdx.x * kTiledWarps + warp;
  int lin_next = c < nrun ? a.run_list[c] : 0;
  for (; c < nrun; c += stride) {
    const int lin = lin_next;
    if (c + stride < nrun) lin_next = a.run_list[c + stride];
    const int s = a.cell_start[lin], e = a.cell_end[lin];
    const uint32_t f0 = a.alt.flags[s];
    const int inst = f0 & kInstMask;
    if (LB && a.inst_keep && a.list_flags[kLfPartial] != 0u && a.inst_keep[inst]) continue;  // keeps its lists
    const InstParams& P = a.params[inst];
    const int ph = a.phase[inst];
    if (!wants_force(P, a.dyn[inst], ph)) {
      for (int p = s + lane; p < e; p += 32) {
        if (LB) a.list_cnt[p] = 0;
        else copy_state(a, p);
      }
      continue;
    }
    const int nx = P.ncell[0], ny = P.ncell[1];
    const int local = lin - P.cell_base;
    const int cx = local % nx, cy = (local / nx) % ny, cz = local / (nx * ny);
    // neighbour cells: lane k < 27 owns offset (k%3-1, k/3%3-1, k/9-1), image code k
    int nb_start = 0, nb_cnt = 0;
    float shx = 0.f, shy = 0.f, shz = 0.f;
    uint32_t code = 13;
    if (lane < 27) {
      int x, y, z;
      if (neighbor_cell(P, 0, cx + lane % 3 - 1, x, shx) && neighbor_cell(P, 1, cy + (lane / 3) % 3 - 1, y, shy) &&
          neighbor_cell(P, 2, cz + lane / 9 - 1, z, shz)) {
        const int l2 = P.cell_base + (z * ny + y) * nx + x;
        nb_start = a.cell_start[l2];
        nb_cnt = a.cell_end[l2] - nb_start;
        code = (uint32_t)((shx > 0.f) - (shx < 0.f) + 1) + 3u * (uint32_t)((shy > 0.f) - (shy < 0.f) + 1) +
               9u * (uint32_t)((shz > 0.f) - (shz < 0.f) + 1);
      }
      // the half2 list build writes the neighbour-cell offset instead, two
      // bits per axis (its compact records are relative to the build's cells)
      if (H16 && LB) code = (uint32_t)(lane % 3) | ((uint32_t)((lane / 3) % 3) << 2) | ((uint32_t)(lane / 9) << 4);
    }
    int incl = nb_cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(full, incl, o);
      if (lane >= o) incl += t;
    }
    const int T = __shfl_sync(full, incl, 31);
    const int excl = incl - nb_cnt;
    const int own = __shfl_sync(full, excl, 13);  // tile offset of the cell's own particles
    const float HS = LB ? P.HL2 : P.H2;  // scan bound
    float dt_cand = 0.f;
    bool dt_valid = false;
    for (int ib = s; ib < e; ib += 32) {
      const int nbat = min(32, e - ib);
      int lcount = 0;  // LB: list entries written so far for i = ib + lane
#pragma unroll
      for (int k = 0; k < 6; ++k) res[lane][k] = 0.f;
      for (int t0 = 0; t0 < T; t0 += kTile) {
        const int tn = min(kTile, T - t0);
        const int tn64 = (tn + 63) & ~63;
        __syncwarp();
        // Flattened staging: candidate u comes from the last neighbour cell k
        // with excl_k <= u (binary search over lanes 0..26); kStageUnroll
        // independent loads per lane are in flight before any store.
        for (int ub = t0; ub < t0 + tn; ub += 32 * kStageUnroll) {
          float4 J[kStageUnroll];
          int gk[kStageUnroll], kk[kStageUnroll];
#pragma unroll
          for (int r = 0; r < kStageUnroll; ++r) {
            const int u = ub + 32 * r + lane;
            int k = 0;
#pragma unroll
            for (int step = 16; step; step >>= 1) {
              const int cand = k + step;
              const int ec = __shfl_sync(full, excl, cand < 27 ? cand : 26);
              if (cand < 27 && ec <= u) k = cand;
            }
            const int sk = __shfl_sync(full, nb_start, k), ek = __shfl_sync(full, excl, k);
            kk[r] = k;
            gk[r] = sk + (u - ek);
            if (u < t0 + tn) J[r] = __ldg(&a.jr[gk[r]].a);
          }
#pragma unroll
          for (int r = 0; r < kStageUnroll; ++r) {
            const int u = ub + 32 * r + lane;
            const int k = kk[r];
            const float sx = __shfl_sync(full, shx, k), sy = __shfl_sync(full, shy, k), sz = __shfl_sync(full, shz, k);
            // entries carry the image code, or for the half2 list pass the
            // neighbour-cell offset (h16_entry)
            const uint32_t ck27 = __shfl_sync(full, code, k) << (H16 && LB ? kH16SlotBits : 27);
            if (u < t0 + tn) {
              tx[u - t0] = __fadd_rn(J[r].x, sx);
              ty[u - t0] = __fadd_rn(J[r].y, sy);
              tz[u - t0] = __fadd_rn(J[r].z, sz);
              te[u - t0] = (uint32_t)gk[r] | ck27;
            }
          }
        }
        for (int u = tn + lane; u < tn64; u += 32) {  // pad to a multiple of 64: never in support
          tx[u] = 1.0e30f;
          ty[u] = 1.0e30f;
          tz[u] = 1.0e30f;
          te[u] = 0u;
        }
        __syncwarp();
        for (int ii = 0; ii < nbat; ii += 2) {
          const int ia = ib + ii;
          const bool has_b = ii + 1 < nbat;
          const int ibb = has_b ? ia + 1 : ia;
          // i positions from the tile when the own cell (lane 13) is staged in this pass
          const int oa = own + (ia - s) - t0, ob = own + (ibb - s) - t0;
          const float4 IA = (oa >= 0 && oa < tn) ? make_float4(tx[oa], ty[oa], tz[oa], __ldg(&a.jr[ia].a.w))
                                                 : __ldg(&a.jr[ia].a);
          const float4 IB = (ob >= 0 && ob < tn) ? make_float4(tx[ob], ty[ob], tz[ob], __ldg(&a.jr[ibb].a.w))
                                                 : __ldg(&a.jr[ibb].a);
          const f2 XA = dup(IA.x), YA = dup(IA.y), ZA = dup(IA.z);
          const f2 XB = dup(IB.x), YB = dup(IB.y), ZB = dup(IB.z);
          int na = 0, nb = 0;
          for (int tb = 2 * lane; tb < tn64; tb += 64) {
            const f2 CX = *reinterpret_cast<const f2*>(&tx[tb]);
            const f2 CY = *reinterpret_cast<const f2*>(&ty[tb]);
            const f2 CZ = *reinterpret_cast<const f2*>(&tz[tb]);
            const uint2 E = *reinterpret_cast<const uint2*>(&te[tb]);
            f2 DX = sub2(XA, CX), DY = sub2(YA, CY), DZ = sub2(ZA, CZ);
            const f2 RA = fma2(DZ, DZ, fma2(DY, DY, mul2(DX, DX)));  // == dist2 per half
            DX = sub2(XB, CX), DY = sub2(YB, CY), DZ = sub2(ZB, CZ);
            const f2 RB = fma2(DZ, DZ, fma2(DY, DY, mul2(DX, DX)));
            const float ra0 = lo(RA), ra1 = hi(RA), rb0 = lo(RB), rb1 = hi(RB);
            append2(qa, na, ra0 > 0.0f && ra0 < HS, ra1 > 0.0f && ra1 < HS, E.x, E.y, lt);
            append2(qb, nb, has_b && rb0 > 0.0f && rb0 < HS, has_b && rb1 > 0.0f && rb1 < HS, E.x, E.y, lt);
          }
          __syncwarp();
          if (LB) {  // append this tile pass's queue entries to the lists of ia and ibb
            const int L = a.list_max;
            const int oa = __shfl_sync(full, lcount, ii), ob = __shfl_sync(full, lcount, ii + 1);
            uint32_t* la = a.list + (size_t)ia * L;
            for (int k = lane; k < na; k += 32)
              if (oa + k < L) la[oa + k] = qa[k];
            if (has_b) {
              uint32_t* lb = a.list + (size_t)ibb * L;
              for (int k = lane; k < nb; k += 32)
                if (ob + k < L) lb[ob + k] = qb[k];
            }
            if (lane == ii) lcount += na;
            if (has_b && lane == ii + 1) lcount += nb;
          }
          if (!LB) hydro_queues2(a, P, ia, ibb, has_b, IA, IB, qa, na, qb, nb, &res[ii], lane);
          __syncwarp();
        }
      }
      __syncwarp();
      if (LB) {
        if (lane < nbat) {
          a.list_cnt[ib + lane] = lcount;
          if (lcount > a.list_max) {
            a.list_flags[kLfOverflowPending] = 1u;  // the next step rebuilds
          } else {  // pad the row to a whole group of four (list_max is a multiple of four)
            uint32_t* row = a.list + (size_t)(ib + lane) * a.list_max;
            for (int k = lcount; k < ((lcount + 3) & ~3); ++k) row[k] = a.list_pad;
          }
        }
        const int mx = __reduce_max_sync(full, lane < nbat ? lcount : 0);
        if (lane == 0) atomicMax(&a.list_flags[kLfLongest], (unsigned)mx);
      }
      if (!LB && lane < nbat) {
        const int p = ib + lane;
        const float* r = res[lane];
        const uint32_t fp = a.alt.flags[p];
        if (!(fp & kGhostBit)) pairs += (unsigned long long)r[5];  // owned particles only
        finish_hydro(a, p, P, inst, ph, fp, r[0], r[1], r[2], r[3], r[4], (unsigned)r[5], dt_cand, dt_valid);
      }
    }
    dt_min(a.dyn, inst, dt_cand, dt_valid);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(full, pairs, o);
  if (lane == 0 && pairs) atomicAdd(a.pair_count, pairs);
}

// List build, lane per particle: a warp per non-empty cell stages the
// cell's candidates as k_hydro_tiled does (stage_tile); then each lane takes
// one particle i of the cell and walks the tile eight candidates per step
// (shared-memory broadcasts, four f32x2 distances), appending each candidate
// within the list radius (0 < r^2 < (2h + skin)^2) to its own list row.  No
// ballots and no queues: the entries are those of k_hydro_tiled's scan in the
// same (candidate) order, so the lists are bit-identical.
template <int WARPS, int TILE>
struct ScanSmem {
  float x[WARPS][TILE], y[WARPS][TILE], z[WARPS][TILE];
  uint32_t e[WARPS][TILE];
};

template <bool H16, int WARPS, int TILE>
__global__ void __launch_bounds__(WARPS * 32) k_list_scan(StepArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ScanSmem<WARPS, TILE>& S = *reinterpret_cast<ScanSmem<WARPS, TILE>*>(smem_raw);
  const unsigned full = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* tx = S.x[warp];
  float* ty = S.y[warp];
  float* tz = S.z[warp];
  uint32_t* te = S.e[warp];
  const int nrun = *a.run_count;
  const int L = a.list_max;
  const int stride = gridDim.x * WARPS;
  int c = blockIdx.x * WARPS + warp;
  int lin_next = c < nrun ? a.run_list[c] : 0;
  for (; c < nrun; c += stride) {
    const int lin = lin_next;
    if (c + stride < nrun) lin_next = a.run_list[c + stride];
    const int s = a.cell_start[lin], e = a.cell_end[lin];
    const int inst = a.alt.flags[s] & kInstMask;
    if (a.inst_keep && a.list_flags[kLfPartial] != 0u && a.inst_keep[inst]) continue;  // keeps its lists
    const InstParams& P = a.params[inst];
    if (!wants_force(P, a.dyn[inst], a.phase[inst])) {
      for (int p = s + lane; p < e; p += 32) a.list_cnt[p] = 0;
      continue;
    }
    const int nx = P.ncell[0], ny = P.ncell[1];
    const int local = lin - P.cell_base;
    const NbRanges R = nb_ranges<H16>(a, P, local % nx, (local / nx) % ny, local / (nx * ny), lane);
    // 0 < r^2 < (2h + skin)^2 as one unsigned compare of the bit patterns
    // (r^2 is a sum of squares, never negative or NaN)
    const uint32_t hb = __float_as_uint(P.HL2) - 1u;
    for (int ib = s; ib < e; ib += 32) {
      const int p = ib + lane;
      const bool mine = p < e;
      const float4 I = __ldg(&a.jr[mine ? p : s].a);
      const f2 IX = dup(I.x), IY = dup(I.y), IZ = dup(I.z);
      uint32_t* row = a.list + (size_t)(mine ? p : s) * L;
      int cnt = 0;
      for (int t0 = 0; t0 < R.total; t0 += TILE) {
        const int tn = min(TILE, R.total - t0);
        __syncwarp();
        stage_tile<H16>(a, R, t0, tn, tx, ty, tz, te, lane);
        __syncwarp();
        if (mine) {
          for (int u = 0; u < tn; u += 8) {  // the tile is padded to a multiple of 64
            const f2* x2 = reinterpret_cast<const f2*>(&tx[u]);
            const f2* y2 = reinterpret_cast<const f2*>(&ty[u]);
            const f2* z2 = reinterpret_cast<const f2*>(&tz[u]);
            const uint4 E0 = *reinterpret_cast<const uint4*>(&te[u]);
            const uint4 E1 = *reinterpret_cast<const uint4*>(&te[u + 4]);
            float r2[8];
#pragma unroll
            for (int h = 0; h < 4; ++h) {
              const f2 DX = sub2(IX, x2[h]), DY = sub2(IY, y2[h]), DZ = sub2(IZ, z2[h]);
              const f2 R2 = fma2(DZ, DZ, fma2(DY, DY, mul2(DX, DX)));  // == dist2 per half
              r2[2 * h] = lo(R2), r2[2 * h + 1] = hi(R2);
            }
            const uint32_t ev[8] = {E0.x, E0.y, E0.z, E0.w, E1.x, E1.y, E1.z, E1.w};
#pragma unroll
            for (int k = 0; k < 8; ++k) {
              if (__float_as_uint(r2[k]) - 1u < hb) {
                if (cnt < L) row[cnt] = ev[k];
                ++cnt;
              }
            }
          }
        }
      }
      if (mine) {
        a.list_cnt[p] = cnt;
        if (cnt > L) {
          a.list_flags[kLfOverflowPending] = 1u;  // the next step rebuilds
        } else {  // pad the row to a whole group of four (list_max is a multiple of four)
          for (int k = cnt; k < ((cnt + 3) & ~3); ++k) row[k] = a.list_pad;
        }
      }
      const int mx = __reduce_max_sync(full, mine ? cnt : 0);
      if (lane == 0) atomicMax(&a.list_flags[kLfLongest], (unsigned)mx);
    }
  }
}

struct TiledLaunch {
  int device = -1;
  int blocks = 0;
};

template <bool H16, int WARPS, int TILE, bool LB>
inline int launch_pair_tiled_v(const StepArgs& a, cudaStream_t s) {
  static TiledLaunch L[16];
  int dev = 0;
  WCSPH_CUDA(cudaGetDevice(&dev));
  TiledLaunch& T = L[dev & 15];
  auto kern = k_hydro_tiled<H16, WARPS, TILE, LB>;
  const int bytes = (int)sizeof(TiledSmem<WARPS, TILE>);
  if (T.device != dev) {
    WCSPH_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    int per_sm = 0, sms = 0;
    WCSPH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WARPS * 32, bytes));
    WCSPH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    T.blocks = std::max(1, per_sm) * sms;
    T.device = dev;
  }
  kern<<<T.blocks, WARPS * 32, bytes, s>>>(a);
  WCSPH_CUDA(cudaGetLastError());
  return 0;
}

template <bool H16, int WARPS, int TILE>
inline int launch_list_scan_v(const StepArgs& a, cudaStream_t s) {
  static TiledLaunch L[16];
  int dev = 0;
  WCSPH_CUDA(cudaGetDevice(&dev));
  TiledLaunch& T = L[dev & 15];
  auto kern = k_list_scan<H16, WARPS, TILE>;
  const int bytes = (int)sizeof(ScanSmem<WARPS, TILE>);
  if (T.device != dev) {
    WCSPH_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    int per_sm = 0, sms = 0;
    WCSPH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WARPS * 32, bytes));
    WCSPH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    T.blocks = std::max(1, per_sm) * sms;
    T.device = dev;
  }
  kern<<<T.blocks, WARPS * 32, bytes, s>>>(a);
  WCSPH_CUDA(cudaGetLastError());
  return 0;
}

// Block shapes the autotuner chooses among (warps per block, at a fixed
// 512-candidate tile).  They change only how cells map to blocks, never the
// order of any sum, so results are bit-identical whichever is chosen.
constexpr int kTileShapes = 3;

template <bool H16, bool LB = false>
inline int launch_hydro_tiled(const StepArgs& a, int n, cudaStream_t s, int shape = 0) {
  if (n > kMaxTiledParticles) {
    set_error("the tiled path holds at most %d particles per solver (got %d)", kMaxTiledParticles, n);
    return WCSPH_E_CAPACITY;
  }
  if constexpr (LB) {  // list builds only: smaller tiles, more warps per SM (the scan writes no sums)
    if (shape == 3) return launch_pair_tiled_v<H16, 4, 256, LB>(a, s);
    if (shape == 4) return launch_pair_tiled_v<H16, 8, 256, LB>(a, s);
    if (shape == 5) return launch_list_scan_v<H16, 4, 512>(a, s);
    if (shape == 6) return launch_list_scan_v<H16, 8, 256>(a, s);
  }
  switch (shape) {
    case 1: return launch_pair_tiled_v<H16, 2, 512, LB>(a, s);
    case 2: return launch_pair_tiled_v<H16, 8, 512, LB>(a, s);
    default: return launch_pair_tiled_v<H16, 4, 512, LB>(a, s);
  }
}

// Shapes of the list build's scan-only pass: the three above and two with
// 256-candidate tiles (half the shared memory a warp, so up to twice the
// warps per SM; a cell's candidates then take two tile passes, which changes
// only the order in which its list entries are found within each pass), and
// the lane-per-particle scan k_list_scan with 4 warps x 512 or 8 warps x 256
// candidates (the same entries in the same order).
constexpr int kBuildShapes = 7;

}  // namespace wcsph

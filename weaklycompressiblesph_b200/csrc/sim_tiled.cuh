// Tiled pair kernels (WCSPH_PREC_TILED): one warp per non-empty cell.
//
//   1. The 27 neighbour cells of the warp's cell are flattened into one
//      candidate list and their complete j-records are staged into the warp's
//      shared-memory tile: x[], y[], z[] (pre-shifted by the periodic image,
//      structure of arrays for the scan), v[] = (vx, vy, vz, rho) and
//      pc[] = (P/rho^2, c).  Each lane locates the source cell of its
//      candidates by a binary search over the 27 range offsets, so every load
//      is coalesced and several are in flight per lane.
//   2. The cell's i-particles are taken two at a time.  Each lane tests two
//      adjacent candidates against both i: one 64-bit shared load yields the
//      candidate pair already packed, and the four FP32 support predicates are
//      evaluated with packed f32x2 arithmetic (bit-identical to the scalar
//      predicate).  In-support candidates are ballot-compacted into one queue
//      of tile indices per i.
//   3. The two queues are consumed together, lane k taking pair k of each
//      queue (dense lanes, no predicate divergence), with the pair terms of the
//      two i-particles evaluated in packed f32x2 arithmetic from the tile
//      (shared memory only: no global gathers per pair).  Partial sums are
//      combined with a butterfly reduce-scatter (9 shuffles for 8 sums) and
//      accumulated per i in shared memory.
//   4. Lane l finishes i = batch + l with the epilogue shared with the plain
//      kernel (gravity, final kick, density floor, next-dt fold, state write).
// Work distribution: a persistent grid; warp w takes the non-empty cells
// w, w + W, w + 2W, ... of the cell list (W warps in the grid), whose order
// follows the Morton sort, so neighbouring warps share L2-resident records.
#pragma once
#include "f32x2.cuh"
#include "sim_kernels.cuh"

namespace wcsph {

constexpr int kTiledWarps = 2;
constexpr int kTile = 512;       // candidates staged per pass (multiple of 64)
constexpr int kStageUnroll = 2;  // staging candidates in flight per lane

struct TiledSmem {
  float x[kTiledWarps][kTile], y[kTiledWarps][kTile], z[kTiledWarps][kTile];  // shifted positions
  float4 v[kTiledWarps][kTile];                 // vx, vy, vz, rho
  float2 pc[kTiledWarps][kTile];                // P/rho^2, c
  unsigned short q[kTiledWarps][2][kTile];      // per-i queues of tile indices
  float res[kTiledWarps][32][6];                // per-i accumulators of the current batch
};

struct Tile {
  const float *x, *y, *z;
  const float4* v;
  const float2* pc;
};

// The i-side record of a pair group.
struct IRec {
  float x, y, z, po, vx, vy, vz, rho, c;
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

// i-record from the tile slot o (when 0 <= o < tn) or from global memory.
__device__ __forceinline__ IRec load_i(const StepArgs& a, const Tile& T, int o, int tn, int i) {
  IRec r;
  if (o >= 0 && o < tn) {
    const float4 v = T.v[o];
    const float2 pc = T.pc[o];
    r = IRec{T.x[o], T.y[o], T.z[o], pc.x, v.x, v.y, v.z, v.w, pc.y};
  } else {
    const float4 A = __ldg(&a.jA[i]), v = __ldg(&a.jB[i]);
    r = IRec{A.x, A.y, A.z, A.w, v.x, v.y, v.z, v.w, __ldg(&a.jC[i])};
  }
  return r;
}

// Pair terms of i_a (low half) and i_b (high half) over their queues; adds
// the warp totals into res[0] (i_a) and res[1] (i_b): ax, ay, az, sum g drdv,
// v_sig, count.  Lanes past a queue's end contribute exactly zero.
__device__ __forceinline__ void hydro_queues2(const InstParams& P, const Tile& T, const IRec& A_, const IRec& B_,
                                              bool has_b, const unsigned short* qa, int na, const unsigned short* qb,
                                              int nb, int self_a, float (*res)[6], int lane) {
  const f2 X = pk(A_.x, B_.x), Y = pk(A_.y, B_.y), Z = pk(A_.z, B_.z);
  const f2 VX = pk(A_.vx, B_.vx), VY = pk(A_.vy, B_.vy), VZ = pk(A_.vz, B_.vz);
  const f2 RHO = pk(A_.rho, B_.rho), PO = pk(A_.po, B_.po), CI = pk(A_.c, B_.c);
  const float H2 = P.H2;
  const f2 IH = dup(P.inv_H), KG = dup(P.Kg), EH2 = dup(P.eh2), HH = dup(P.h), NU4 = dup(P.nu4);
  const f2 ONE = dup(1.0f), HALF = dup(0.5f), TWELVE = dup(12.0f), MTHREE = dup(-3.0f), TWO = dup(2.0f);
  const f2 BETA = dup(P.beta), MHALPHA = dup(-0.5f * P.alpha), MONE = dup(-1.0f);
  const int vs = P.vsig_mode;
  const int nbq = has_b ? nb : 0;
  const int n = max(na, nbq);
  f2 AX = 0ull, AY = 0ull, AZ = 0ull, DS = 0ull;
  float vsa = 0.f, vsb = 0.f;
  for (int k = lane; k < n; k += 32) {
    const bool va = k < na, vb = k < nbq;
    // idle halves read a valid slot (weight 0 below)
    const int ta = va ? qa[k] : self_a, tb = vb ? qb[k] : self_a;
    const float4 Va = T.v[ta], Vb = T.v[tb];
    const float2 Ca = T.pc[ta], Cb = T.pc[tb];
    const f2 DX = sub2(X, pk(T.x[ta], T.x[tb])), DY = sub2(Y, pk(T.y[ta], T.y[tb])),
             DZ = sub2(Z, pk(T.z[ta], T.z[tb]));
    const f2 R2raw = fma2(DZ, DZ, fma2(DY, DY, mul2(DX, DX)));
    const f2 R2 = pk(va ? lo(R2raw) : H2, vb ? hi(R2raw) : H2);  // finite stand-in for idle halves
    const f2 W = pk(va ? 1.0f : 0.0f, vb ? 1.0f : 0.0f);
    const f2 RINV = rsqrt2(R2);
    const f2 S = mul2(mul2(R2, RINV), IH);
    const f2 A = max0_2(sub2(ONE, S)), B = max0_2(sub2(HALF, S));
    const f2 F = fma2(TWELVE, mul2(B, B), mul2(MTHREE, mul2(A, A)));  // 12 (1/2-s)+^2 - 3 (1-s)+^2
    const f2 G = mul2(mul2(F, KG), mul2(RINV, W));                     // gradW = G * dr
    const f2 DVX = sub2(VX, pk(Va.x, Vb.x)), DVY = sub2(VY, pk(Va.y, Vb.y)), DVZ = sub2(VZ, pk(Va.z, Vb.z));
    const f2 DRDV = fma2(DZ, DVZ, fma2(DY, DVY, mul2(DX, DVX)));
    const f2 RDEN = rcp2(add2(R2, EH2));
    const f2 MUr = mul2(mul2(DRDV, RDEN), HH);
    const f2 MU = pk(va && lo(DRDV) < 0.0f ? lo(MUr) : 0.0f, vb && hi(DRDV) < 0.0f ? hi(MUr) : 0.0f);
    const f2 RS = rcp2(add2(RHO, pk(Va.w, Vb.w)));
    const f2 AV = mul2(mul2(fma2(BETA, MU, mul2(MHALPHA, add2(CI, pk(Ca.y, Cb.y)))), MU), mul2(RS, TWO));
    if (vs) {
      vsa = fmaxf(vsa, -lo(MU));
      vsb = fmaxf(vsb, -hi(MU));
    } else {
      vsa = fmaxf(vsa, lo(MU));
      vsb = fmaxf(vsb, hi(MU));
    }
    const f2 NPG = mul2(mul2(add2(add2(PO, pk(Ca.x, Cb.x)), AV), G), MONE);
    const f2 VISC = mul2(mul2(mul2(NU4, G), R2), mul2(RS, RDEN));
    AX = fma2(NPG, DX, fma2(VISC, DVX, AX));
    AY = fma2(NPG, DY, fma2(VISC, DVY, AY));
    AZ = fma2(NPG, DZ, fma2(VISC, DVZ, AZ));
    DS = fma2(G, DRDV, DS);
  }
  const float v8[8] = {lo(AX), lo(AY), lo(AZ), lo(DS), hi(AX), hi(AY), hi(AZ), hi(DS)};
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

// Density sums of i_a / i_b over their queues: sum w and sum w / rho_j
// (w = (1-s)+^3 - 4 (1/2-s)+^3, the cubic spline without its normalisation),
// added into res[.][0], res[.][1]; count into res[.][5].
__device__ __forceinline__ void density_queues2(const InstParams& P, const Tile& T, const IRec& A_, const IRec& B_,
                                                bool has_b, const unsigned short* qa, int na,
                                                const unsigned short* qb, int nb, int self_a, float (*res)[6],
                                                int lane) {
  const f2 X = pk(A_.x, B_.x), Y = pk(A_.y, B_.y), Z = pk(A_.z, B_.z);
  const float H2 = P.H2;
  const f2 IH = dup(P.inv_H), ONE = dup(1.0f), HALF = dup(0.5f), MFOUR = dup(-4.0f);
  const int nbq = has_b ? nb : 0;
  const int n = max(na, nbq);
  f2 SW = 0ull, SO = 0ull;
  for (int k = lane; k < n; k += 32) {
    const bool va = k < na, vb = k < nbq;
    const int ta = va ? qa[k] : self_a, tb = vb ? qb[k] : self_a;
    const f2 DX = sub2(X, pk(T.x[ta], T.x[tb])), DY = sub2(Y, pk(T.y[ta], T.y[tb])),
             DZ = sub2(Z, pk(T.z[ta], T.z[tb]));
    const f2 R2raw = fma2(DZ, DZ, fma2(DY, DY, mul2(DX, DX)));
    const f2 R2 = pk(va ? lo(R2raw) : H2, vb ? hi(R2raw) : H2);
    const f2 S = mul2(mul2(R2, rsqrt2(R2)), IH);
    const f2 A = max0_2(sub2(ONE, S)), B = max0_2(sub2(HALF, S));
    const f2 Wf = mul2(fma2(MFOUR, mul2(B, mul2(B, B)), mul2(A, mul2(A, A))), pk(va ? 1.0f : 0.0f, vb ? 1.0f : 0.0f));
    SW = add2(SW, Wf);
    SO = fma2(Wf, rcp2(pk(T.v[ta].w, T.v[tb].w)), SO);
  }
  const float v8[8] = {lo(SW), lo(SO), 0.f, 0.f, hi(SW), hi(SO), 0.f, 0.f};
  const float y = butterfly8(v8, lane);
  if ((lane & 3) == 0) {
    const int slot = lane >> 2;
    if (slot < 2) res[0][slot] += y;
    else if (slot >= 4 && slot < 6 && has_b) res[1][slot - 4] += y;
  }
  if (lane == 0) {
    res[0][5] += (float)na;
    if (has_b) res[1][5] += (float)nb;
  }
}

// Append the in-support candidates (even/odd halves of the lane's pair) to a queue.
__device__ __forceinline__ void append2(unsigned short* q, int& n, bool he, bool ho, int t, unsigned lt) {
  const unsigned me = __ballot_sync(0xffffffffu, he), mo = __ballot_sync(0xffffffffu, ho);
  const int p = n + __popc(me & lt) + __popc(mo & lt);
  if (he) q[p] = (unsigned short)t;
  if (ho) q[p + (he ? 1 : 0)] = (unsigned short)(t + 1);
  n += __popc(me) + __popc(mo);
}

enum PairPass { PASS_HYDRO = 0, PASS_DENSITY = 1 };

template <int PASS>
__global__ void __launch_bounds__(kTiledWarps * 32) k_pair_tiled(StepArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TiledSmem& S = *reinterpret_cast<TiledSmem*>(smem_raw);
  const unsigned full = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* tx = S.x[warp];
  float* ty = S.y[warp];
  float* tz = S.z[warp];
  float4* tv = S.v[warp];
  float2* tpc = S.pc[warp];
  const Tile T{tx, ty, tz, tv, tpc};
  unsigned short* qa = S.q[warp][0];
  unsigned short* qb = S.q[warp][1];
  float(*res)[6] = S.res[warp];
  const int nrun = *a.run_count;
  const unsigned lt = lanemask_lt();
  unsigned long long pairs = 0;
  const int stride = gridDim.x * kTiledWarps;
  int c = blockIdx.x * kTiledWarps + warp;
  int lin_next = c < nrun ? a.run_list[c] : 0;
  for (; c < nrun; c += stride) {
    const int lin = lin_next;
    if (c + stride < nrun) lin_next = a.run_list[c + stride];
    const int s = a.cell_start[lin], e = a.cell_end[lin];
    const uint32_t f0 = a.alt.flags[s];
    const int inst = f0 & kInstMask;
    const InstParams& P = a.params[inst];
    const int ph = a.phase[inst];
    const int dkind = PASS == PASS_DENSITY ? density_kind(a, P, a.dyn[inst], ph) : 0;
    if (PASS == PASS_HYDRO && !wants_force(P, a.dyn[inst], ph)) {
      for (int p = s + lane; p < e; p += 32) copy_state(a, p);
      continue;
    }
    if (PASS == PASS_DENSITY && !dkind) continue;
    const int nx = P.ncell[0], ny = P.ncell[1];
    const int local = lin - P.cell_base;
    const int cx = local % nx, cy = (local / nx) % ny, cz = local / (nx * ny);
    // neighbour cells: lane k < 27 owns offset (k%3-1, k/3%3-1, k/9-1)
    int nb_start = 0, nb_cnt = 0;
    float shx = 0.f, shy = 0.f, shz = 0.f;
    if (lane < 27) {
      int x, y, z;
      if (neighbor_cell(P, 0, cx + lane % 3 - 1, x, shx) && neighbor_cell(P, 1, cy + (lane / 3) % 3 - 1, y, shy) &&
          neighbor_cell(P, 2, cz + lane / 9 - 1, z, shz)) {
        const int l2 = P.cell_base + (z * ny + y) * nx + x;
        nb_start = a.cell_start[l2];
        nb_cnt = a.cell_end[l2] - nb_start;
      }
    }
    int incl = nb_cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(full, incl, o);
      if (lane >= o) incl += t;
    }
    const int Tn = __shfl_sync(full, incl, 31);
    const int excl = incl - nb_cnt;
    const int own = __shfl_sync(full, excl, 13);  // tile offset of the cell's own particles
    const float H2 = P.H2;
    float dt_cand = 0.f;
    bool dt_valid = false;
    for (int ib = s; ib < e; ib += 32) {
      const int nbat = min(32, e - ib);
#pragma unroll
      for (int k = 0; k < 6; ++k) res[lane][k] = 0.f;
      for (int t0 = 0; t0 < Tn; t0 += kTile) {
        const int tn = min(kTile, Tn - t0);
        const int tn64 = (tn + 63) & ~63;
        __syncwarp();
        // Staging: candidate u comes from the last neighbour cell k with
        // excl_k <= u (binary search over lanes 0..26).
        for (int ub = t0; ub < t0 + tn; ub += 32 * kStageUnroll) {
          float4 JA[kStageUnroll], JB[kStageUnroll];
          float JC[kStageUnroll];
          int kk[kStageUnroll];
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
            if (u < t0 + tn) {
              const int g = sk + (u - ek);
              JA[r] = __ldg(&a.jA[g]);
              JB[r] = __ldg(&a.jB[g]);
              JC[r] = __ldg(&a.jC[g]);
            }
          }
#pragma unroll
          for (int r = 0; r < kStageUnroll; ++r) {
            const int u = ub + 32 * r + lane;
            const int k = kk[r];
            const float sx = __shfl_sync(full, shx, k), sy = __shfl_sync(full, shy, k), sz = __shfl_sync(full, shz, k);
            if (u < t0 + tn) {
              const int o = u - t0;
              tx[o] = __fadd_rn(JA[r].x, sx);
              ty[o] = __fadd_rn(JA[r].y, sy);
              tz[o] = __fadd_rn(JA[r].z, sz);
              tv[o] = JB[r];
              tpc[o] = make_float2(JA[r].w, JC[r]);
            }
          }
        }
        for (int u = tn + lane; u < tn64; u += 32) {  // pad to a multiple of 64: never in support
          tx[u] = 1.0e30f;
          ty[u] = 1.0e30f;
          tz[u] = 1.0e30f;
        }
        __syncwarp();
        for (int ii = 0; ii < nbat; ii += 2) {
          const int ia = ib + ii;
          const bool has_b = ii + 1 < nbat;
          const int ibb = has_b ? ia + 1 : ia;
          const int oa = own + (ia - s) - t0, ob = own + (ibb - s) - t0;
          const IRec RA_ = load_i(a, T, oa, tn, ia), RB_ = load_i(a, T, ob, tn, ibb);
          const f2 XA = dup(RA_.x), YA = dup(RA_.y), ZA = dup(RA_.z);
          const f2 XB = dup(RB_.x), YB = dup(RB_.y), ZB = dup(RB_.z);
          int na = 0, nb = 0;
          for (int tb = 2 * lane; tb < tn64; tb += 64) {
            const f2 CX = *reinterpret_cast<const f2*>(&tx[tb]);
            const f2 CY = *reinterpret_cast<const f2*>(&ty[tb]);
            const f2 CZ = *reinterpret_cast<const f2*>(&tz[tb]);
            f2 DX = sub2(XA, CX), DY = sub2(YA, CY), DZ = sub2(ZA, CZ);
            const f2 RA = fma2(DZ, DZ, fma2(DY, DY, mul2(DX, DX)));  // == dist2 per half
            DX = sub2(XB, CX), DY = sub2(YB, CY), DZ = sub2(ZB, CZ);
            const f2 RB = fma2(DZ, DZ, fma2(DY, DY, mul2(DX, DX)));
            const float ra0 = lo(RA), ra1 = hi(RA), rb0 = lo(RB), rb1 = hi(RB);
            append2(qa, na, ra0 > 0.0f && ra0 < H2, ra1 > 0.0f && ra1 < H2, tb, lt);
            append2(qb, nb, has_b && rb0 > 0.0f && rb0 < H2, has_b && rb1 > 0.0f && rb1 < H2, tb, lt);
          }
          __syncwarp();
          const int self_a = (oa >= 0 && oa < tn) ? oa : 0;
          if (PASS == PASS_HYDRO) hydro_queues2(P, T, RA_, RB_, has_b, qa, na, qb, nb, self_a, &res[ii], lane);
          else density_queues2(P, T, RA_, RB_, has_b, qa, na, qb, nb, self_a, &res[ii], lane);
          __syncwarp();
        }
      }
      __syncwarp();
      if (lane < nbat) {
        const int p = ib + lane;
        const float* r = res[lane];
        if (PASS == PASS_HYDRO) {
          pairs += (unsigned long long)r[5];
          finish_hydro(a, p, P, inst, ph, a.alt.flags[p], r[0], r[1], r[2], r[3], r[4], (unsigned)r[5], dt_cand,
                       dt_valid);
        } else {  // self term w(0) = 1/2 (force.h:16-20 lists contain i)
          const float sum = 0.5f + r[0];
          a.rho_new[p] = dkind == 2 ? sum / (0.5f / a.jB[p].w + r[1]) : P.mass * P.Kw * sum;
        }
      }
    }
    if (PASS == PASS_HYDRO) dt_min(a.dyn, inst, dt_cand, dt_valid);
  }
  if (PASS == PASS_HYDRO) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(full, pairs, o);
    if (lane == 0 && pairs) atomicAdd(a.pair_count, pairs);
  }
}

struct TiledLaunch {
  int device = -1;
  int blocks = 0;
};

template <int PASS>
inline int launch_pair_tiled(const StepArgs& a, int n, cudaStream_t s) {
  (void)n;
  static TiledLaunch L[16];
  int dev = 0;
  WCSPH_CUDA(cudaGetDevice(&dev));
  TiledLaunch& T = L[dev & 15];
  if (T.device != dev) {
    const int bytes = (int)sizeof(TiledSmem);
    WCSPH_CUDA(cudaFuncSetAttribute(k_pair_tiled<PASS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    int per_sm = 0, sms = 0;
    WCSPH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pair_tiled<PASS>, kTiledWarps * 32, bytes));
    WCSPH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    T.blocks = std::max(1, per_sm) * sms;
    T.device = dev;
  }
  k_pair_tiled<PASS><<<T.blocks, kTiledWarps * 32, sizeof(TiledSmem), s>>>(a);
  WCSPH_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace wcsph

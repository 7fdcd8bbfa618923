// Tiled pair kernels (WCSPH_PREC_TILED): one warp per non-empty cell.
//
//   1. The 27 neighbour cells of the warp's cell are flattened into one
//      candidate list; their j-records (x, y, z pre-shifted by the periodic
//      image, P/rho^2) are staged into the warp's shared-memory tile with
//      coalesced loads (a cell's particles are contiguous after the sort).
//   2. For every i of the cell (two at a time) the warp scans the tile with
//      one candidate per lane, evaluates the FP32 support predicate, and
//      ballot-compacts the in-support candidates into a per-i queue.
//   3. The queue is consumed 32 pairs at a time (dense lanes, no predicate
//      divergence); velocities, densities and sound speeds of those j are
//      gathered from global memory by index (they lie in a few contiguous
//      runs, so the loads coalesce well); partial sums are reduced with warp
//      shuffles and accumulated per i in shared memory.
//   4. Lane l finishes i = batch + l: gravity, final kick, density floor,
//      next-dt fold, state write (the same epilogue as the plain kernel).
// Work is distributed dynamically: warps take cells from the list of
// non-empty cells through a global counter (persistent grid).
#pragma once
#include "sim_kernels.cuh"

namespace wcsph {

constexpr int kTiledWarps = 4;
constexpr int kTile = 512;

struct TiledSmem {
  float4 pos[kTiledWarps][kTile];                // staged j: shifted x, y, z and P/rho^2
  int gidx[kTiledWarps][kTile];                  // global slot of each staged j
  unsigned short q[kTiledWarps][2][kTile];       // per-i compacted candidate queues
  float res[kTiledWarps][32][6];                 // per-i accumulators of the current batch
};

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sum the pair terms of one i over its compacted queue (lane-strided) and
// add the warp totals into res (ax, ay, az, sum g drdv, v_sig, count).
__device__ __forceinline__ void hydro_queue(const StepArgs& a, const InstParams& P, int i, const float4& I,
                                            const unsigned short* q, int nq, const float4* tp, const int* tg,
                                            float* res, int lane) {
  const float4 IB = __ldg(&a.jB[i]);
  const float ci = __ldg(&a.jC[i]);
  const float rho_i = IB.w, po_i = I.w;
  const float h = P.h, eh2 = P.eh2, Kg = P.Kg, iH = P.inv_H, alpha = P.alpha, beta = P.beta, nu4 = P.nu4;
  const int vs = P.vsig_mode;
  float ax = 0.f, ay = 0.f, az = 0.f, dsum = 0.f, vsig = 0.f;
  for (int k = lane; k < nq; k += 32) {
    const int t = q[k];
    const float4 J = tp[t];
    const int g = tg[t];
    const float4 JB = __ldg(&a.jB[g]);
    const float cj = __ldg(&a.jC[g]);
    const float dx = __fsub_rn(I.x, J.x), dy = __fsub_rn(I.y, J.y), dz = __fsub_rn(I.z, J.z);
    const float r2 = dist2(dx, dy, dz);
    const float rinv = rsqrtf(r2);
    const float gr = spline_F(r2 * rinv * iH) * Kg * rinv;
    const float dvx = IB.x - JB.x, dvy = IB.y - JB.y, dvz = IB.z - JB.z;
    const float drdv = dx * dvx + dy * dvy + dz * dvz;
    const float rden = __frcp_rn(r2 + eh2);
    const float mu = drdv < 0.0f ? h * drdv * rden : 0.0f;
    const float rs = __frcp_rn(rho_i + JB.w);
    const float av = (beta * mu - alpha * 0.5f * (ci + cj)) * mu * 2.0f * rs;
    vsig = vs ? fmaxf(vsig, -mu) : fmaxf(vsig, mu);
    const float pg = (po_i + J.w + av) * gr;
    const float visc = nu4 * gr * r2 * rs * rden;
    ax += visc * dvx - pg * dx;
    ay += visc * dvy - pg * dy;
    az += visc * dvz - pg * dz;
    dsum += gr * drdv;
  }
  ax = warp_sum(ax);
  ay = warp_sum(ay);
  az = warp_sum(az);
  dsum = warp_sum(dsum);
  vsig = warp_max(vsig);
  if (lane == 0) {
    res[0] += ax;
    res[1] += ay;
    res[2] += az;
    res[3] += dsum;
    res[4] = fmaxf(res[4], vsig);
    res[5] += (float)nq;
  }
}

__global__ void __launch_bounds__(kTiledWarps * 32) k_hydro_tiled(StepArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TiledSmem& S = *reinterpret_cast<TiledSmem*>(smem_raw);
  const unsigned full = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float4* tp = S.pos[warp];
  int* tg = S.gidx[warp];
  unsigned short* qa = S.q[warp][0];
  unsigned short* qb = S.q[warp][1];
  float(*res)[6] = S.res[warp];
  const int nrun = *a.run_count;
  const unsigned lt = lanemask_lt();
  unsigned long long pairs = 0;
  for (;;) {
    int c = 0;
    if (lane == 0) c = atomicAdd(a.work_counter, 1);
    c = __shfl_sync(full, c, 0);
    if (c >= nrun) break;
    const int lin = a.run_list[c];
    const int s = a.cell_start[lin], e = a.cell_end[lin];
    const uint32_t f0 = a.alt.flags[s];
    const int inst = f0 & kInstMask;
    const InstParams& P = a.params[inst];
    const int ph = a.phase[inst];
    if (!wants_force(P, a.dyn[inst], ph)) {
      for (int p = s + lane; p < e; p += 32) copy_state(a, p);
      continue;
    }
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
    const int T = __shfl_sync(full, incl, 31);
    const int excl = incl - nb_cnt;
    const float H2 = P.H2;
    float dt_cand = 0.f;
    bool dt_valid = false;
    for (int ib = s; ib < e; ib += 32) {
      const int nbat = min(32, e - ib);
#pragma unroll
      for (int k = 0; k < 6; ++k) res[lane][k] = 0.f;
      for (int t0 = 0; t0 < T; t0 += kTile) {
        const int tn = min(kTile, T - t0);
        __syncwarp();
        for (int k = 0; k < 27; ++k) {
          const int ck = __shfl_sync(full, nb_cnt, k);
          const int sk = __shfl_sync(full, nb_start, k);
          const int ek = __shfl_sync(full, excl, k);
          const float sx = __shfl_sync(full, shx, k), sy = __shfl_sync(full, shy, k), sz = __shfl_sync(full, shz, k);
          const int lo = max(ek, t0), hi = min(ek + ck, t0 + tn);
          for (int u = lo + lane; u < hi; u += 32) {
            const int g = sk + (u - ek);
            const float4 J = __ldg(&a.jA[g]);
            tp[u - t0] = make_float4(__fadd_rn(J.x, sx), __fadd_rn(J.y, sy), __fadd_rn(J.z, sz), J.w);
            tg[u - t0] = g;
          }
        }
        __syncwarp();
        for (int ii = 0; ii < nbat; ii += 2) {
          const int ia = ib + ii;
          const bool has_b = ii + 1 < nbat;
          const int ibb = has_b ? ia + 1 : ia;
          const float4 IA = __ldg(&a.jA[ia]);
          const float4 IB = __ldg(&a.jA[ibb]);
          int na = 0, nb = 0;
          for (int tb = 0; tb < tn; tb += 32) {
            const int t = tb + lane;
            bool ina = false, inb = false;
            if (t < tn) {
              const float4 J = tp[t];
              const float r2a = dist2(__fsub_rn(IA.x, J.x), __fsub_rn(IA.y, J.y), __fsub_rn(IA.z, J.z));
              const float r2b = dist2(__fsub_rn(IB.x, J.x), __fsub_rn(IB.y, J.y), __fsub_rn(IB.z, J.z));
              ina = r2a > 0.0f && r2a < H2;
              inb = has_b && r2b > 0.0f && r2b < H2;
            }
            const unsigned ba = __ballot_sync(full, ina), bb = __ballot_sync(full, inb);
            if (ina) qa[na + __popc(ba & lt)] = (unsigned short)t;
            if (inb) qb[nb + __popc(bb & lt)] = (unsigned short)t;
            na += __popc(ba);
            nb += __popc(bb);
          }
          __syncwarp();
          hydro_queue(a, P, ia, IA, qa, na, tp, tg, res[ii], lane);
          if (has_b) hydro_queue(a, P, ibb, IB, qb, nb, tp, tg, res[ii + 1], lane);
          __syncwarp();
        }
      }
      __syncwarp();
      if (lane < nbat) {
        const int p = ib + lane;
        const float* r = res[lane];
        pairs += (unsigned long long)r[5];
        finish_hydro(a, p, P, inst, ph, a.alt.flags[p], r[0], r[1], r[2], r[3], r[4], (unsigned)r[5], dt_cand,
                     dt_valid);
      }
    }
    dt_min(a.dyn, inst, dt_cand, dt_valid);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(full, pairs, o);
  if (lane == 0 && pairs) atomicAdd(a.pair_count, pairs);
}

struct TiledLaunch {
  int device = -1;
  int blocks = 0;
};

inline int launch_hydro_tiled(const StepArgs& a, int n, int precision, cudaStream_t s) {
  (void)n;
  if (precision != WCSPH_PREC_TILED) {
    set_error("precision %d is not built in this library", precision);
    return WCSPH_E_INVALID;
  }
  static TiledLaunch L[16];
  int dev = 0;
  WCSPH_CUDA(cudaGetDevice(&dev));
  TiledLaunch& T = L[dev & 15];
  if (T.device != dev) {
    const int bytes = (int)sizeof(TiledSmem);
    WCSPH_CUDA(cudaFuncSetAttribute(k_hydro_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    int per_sm = 0, sms = 0;
    WCSPH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hydro_tiled, kTiledWarps * 32, bytes));
    WCSPH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    T.blocks = std::max(1, per_sm) * sms;
    T.device = dev;
  }
  k_hydro_tiled<<<T.blocks, kTiledWarps * 32, sizeof(TiledSmem), s>>>(a);
  WCSPH_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace wcsph

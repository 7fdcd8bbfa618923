// Neighbour-list steps (wcsph_sim_options.list_interval > 0).
//
// A build step is an ordinary step whose tiled hydro kernel also writes, for
// every particle, the candidates within 2h + skin (the list radius) and whose
// permutation records the positions x0 the lists refer to.  The steps up to
// the next build skip the binning sort and the candidate scan:
//   k_kick_refresh  KDK first half (periodic wrapping waits for the next
//                 build, so that the lists' image shifts stay valid), state
//                 written in the build's order, EoS j-records refreshed,
//                 |x - x0| checked
//   k_density_list, k_eos   the density pass from the lists, when one is due
//   k_hydro_list  the tiled kernel's pair phase over each particle's list
//                 (warp per cell of the build's cell table), every entry
//                 tested for 0 < r^2 < (2h)^2 on the current positions, then
//                 the shared epilogue
// A pair within the support now was within 2h + |dx_i| + |dx_j| at the
// build, so the lists hold every pair the support test can accept while no
// particle has moved more than skin / 2 since the build.  The host rebuilds
// before that (k_kick_refresh reports each step's largest drift and the
// largest displacement); a displacement beyond skin / 2 sets a sticky error
// that the next wcsph_sim_step reports.
#pragma once
#include "sim_tiled.cuh"

namespace wcsph {

constexpr int kListWarps = 4;
constexpr int kListMaxEntries = 192;  // entries per list (the solver's list_max; the dam break needs up to ~120)

// A list step's kick (kick_particle, no wrapping) with the state written
// straight to the alt buffers in the build's order, the EoS j-records
// refreshed, and |x - x0| checked.  The main buffers are rewritten from alt by
// the list pass (every particle below the live count is in a cell of the
// build's table) and by k_copy_dead (the tail).
__global__ void k_kick_refresh(StepArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n_host) return;
  uint32_t f = a.main.flags[p];
  const int inst = f & kInstMask;
  const InstParams& P = a.params[inst];
  bool dead = (f & kDeadBit) || !P.active;
  float4 x = a.main.pos[p];
  float4 v = a.main.vel[p];
  float4 vh = v;
  unsigned drift_bits = 0u, disp_bits = 0u;
  if (!dead) kick_particle(a, P, inst, p, f, x, v, vh, dead, drift_bits);
  if (dead) f |= kDeadBit;
  a.alt.pos[p] = x;
  a.alt.vel[p] = v;
  a.alt.vh[p] = vh;
  a.alt.acc[p] = a.main.acc[p];
  a.alt.pid[p] = a.main.pid[p];
  a.alt.flags[p] = f;
  if (!dead) {
    float pres, snds;
    tait(P, x.w, pres, snds);
    a.jr[p].a = make_float4(x.x, x.y, x.z, pres / (x.w * x.w));
    a.jr[p].b = make_float4(v.x, v.y, v.z, x.w);
    a.jC[p] = snds;
    const float4 o = a.x0[p];
    const float dx = x.x - o.x, dy = x.y - o.y, dz = x.z - o.z;
    const float r = sqrtf(dx * dx + dy * dy + dz * dz) * P.inv_skin;
    disp_bits = __float_as_uint(r);
    if (r > 0.5f) atomicOr(&a.list_flags[2], 1u);  // a pair may be missing from the lists
  } else {  // removed: never in anyone's support again
    a.jr[p].a = make_float4(1.0e30f, 1.0e30f, 1.0e30f, 0.f);
    a.jr[p].b = make_float4(0.f, 0.f, 0.f, 1.f);
    a.jC[p] = 0.f;
  }
  list_flag_max(&a.list_flags[0], disp_bits);
  list_flag_max(&a.list_flags[1], drift_bits);
}

// Density pass over the lists: k_density_plain's sums (summation, or the
// Shepard filter of force.h:12-29) over each particle's list entries that are
// within the support now.  Warp per cell of the build's cell table, four
// particles at a time, eight lanes per particle walking its list (coalesced
// list loads), the eight partial sums combined by shuffles.  Particles
// removed since the build keep their density.
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_density_list(StepArgs a) {
  if (a.dens_any && !*a.dens_any) return;  // no density pass in this launch
  const unsigned full = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane & 7, grp = lane >> 3;
  const int nrun = *a.run_count;
  const int stride = gridDim.x * WARPS;
  for (int c = blockIdx.x * WARPS + warp; c < nrun; c += stride) {
    const int lin = a.run_list[c];
    const int s = a.cell_start[lin], e = a.cell_end[lin];
    const int inst = a.alt.flags[s] & kInstMask;
    const InstParams& P = a.params[inst];
    const int kind = density_kind(a, P, a.dyn[inst], a.phase[inst]);
    if (!kind) continue;
    const bool shep = kind == 2;
    const float iH = P.inv_H, H2 = P.H2;
    for (int ib = s; ib < e; ib += 4) {
      const int p = ib + grp;
      const bool valid = p < e;
      const bool dead = valid && (a.alt.flags[p] & kDeadBit);
      const int n = valid && !dead ? min(a.list_cnt[p], a.list_max) : 0;
      const float4 I = valid ? __ldg(&a.jr[p].a) : make_float4(0.f, 0.f, 0.f, 0.f);
      const uint32_t* l = a.list + (size_t)(valid ? p : s) * a.list_max;
      float sum = 0.f, one = 0.f;
      for (int k = sub; k < n; k += 8) {
        const uint32_t ent = __ldg(&l[k]);
        const int q = ent & kSlotMask;
        const float4 J = __ldg(&a.jr[q].a);
        float sx = 0.f, sy = 0.f, sz = 0.f;
        if (P.periodic) entry_shift(P, ent >> 27, sx, sy, sz);
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
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) {
        sum += __shfl_xor_sync(full, sum, o);
        one += __shfl_xor_sync(full, one, o);
      }
      if (valid && sub == 0) {
        if (dead) {
          a.rho_new[p] = a.alt.pos[p].w;
        } else {
          const float rho_i = __ldg(&a.jr[p].b.w);
          const float t = 0.5f + sum;  // self term: w(0) = 1/2
          a.rho_new[p] = shep ? t / (0.5f / rho_i + one) : P.mass * P.Kw * t;
        }
      }
    }
  }
}

template <int WARPS>
inline int launch_density_list(const StepArgs& a, cudaStream_t s) {
  static int blocks[16] = {0};
  int dev = 0;
  WCSPH_CUDA(cudaGetDevice(&dev));
  auto kern = k_density_list<WARPS>;
  if (!blocks[dev & 15]) {
    int per_sm = 0, sms = 0;
    WCSPH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WARPS * 32, 0));
    WCSPH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    blocks[dev & 15] = std::max(1, per_sm) * sms;
  }
  kern<<<blocks[dev & 15], WARPS * 32, 0, s>>>(a);
  WCSPH_CUDA(cudaGetLastError());
  return 0;
}

// The pair phase of the tiled kernel over the lists.  The cell table of the
// last build is still valid (list steps do not re-sort), so the work is laid
// out as in k_hydro_tiled: warp per non-empty cell, batches of 32 particles,
// pairs of i at a time; each pair's two list rows are brought into
// shared-memory queues by TMA bulk copies one pair ahead, into the other of
// two buffers, each with its own mbarrier; the shared pair routine tests the
// support per entry, and lane l finishes particle batch + l with the shared
// epilogue.
// Bulk copies global -> shared (TMA, cp.async.bulk, no multicast) completing
// on a shared-memory mbarrier, and the barrier operations they need.
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
// Order this thread's earlier generic accesses of shared memory before later
// async-proxy (bulk copy) writes to it.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  unsigned long long state;
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;\n"
               : "=l"(state)
               : "r"(smem_addr(bar)), "r"(bytes)
               : "memory");
  (void)state;
}
// bytes: a multiple of 16; dst and src 16-byte aligned.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
constexpr unsigned kListErrCopy = 4u;     // list_flags[2]: a bulk copy of a list did not complete
constexpr int kMbarSpinLimit = 1 << 22;   // try_wait rounds before giving up on a copy

template <bool H16, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 5) k_hydro_list(StepArgs a) {
  // [warp][buffer][i of the pair][entry]; a list row is 768 bytes, 16-byte aligned
  __shared__ __align__(16) uint32_t s_q[WARPS][2][2][kListMaxEntries];
  __shared__ __align__(8) unsigned long long s_bar[WARPS][2];  // one mbarrier per buffer
  __shared__ float s_res[WARPS][32][6];
  const unsigned full = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float(*res)[6] = s_res[warp];
  const int L = a.list_max;
  const int nrun = *a.run_count;
  unsigned long long pairs = 0;
  if (lane == 0) {
    mbar_init(&s_bar[warp][0], 1);
    mbar_init(&s_bar[warp][1], 1);
    fence_mbar_init();
  }
  __syncwarp();
  unsigned parity = 0u;  // bit b: parity of buffer b's next completion
  bool copy_failed = false;
  const int stride = gridDim.x * WARPS;
  for (int c = blockIdx.x * WARPS + warp; c < nrun; c += stride) {
    const int lin = a.run_list[c];
    const int s = a.cell_start[lin], e = a.cell_end[lin];
    const int inst = a.alt.flags[s] & kInstMask;
    const InstParams& P = a.params[inst];
    const int ph = a.phase[inst];
    if (!wants_force(P, a.dyn[inst], ph)) {
      for (int p = s + lane; p < e; p += 32) copy_state(a, p);
      continue;
    }
    float dt_cand = 0.f;
    bool dt_valid = false;
    for (int ib = s; ib < e; ib += 32) {
      const int nbat = min(32, e - ib);
#pragma unroll
      for (int k = 0; k < 6; ++k) res[lane][k] = 0.f;
      // list lengths of the batch in one load (particles removed since the
      // build keep their state and sum nothing)
      const int my_n = lane < nbat && !(a.alt.flags[ib + lane] & kDeadBit) ? min(a.list_cnt[ib + lane], L) : 0;
      // lane 0 copies the next pair's two list rows into the other buffer
      // (bulk copies rounded up to 16 bytes, within the 768-byte rows) while
      // the current pair is summed
      auto fetch = [&](int ii, int buf) {
        const int na = __shfl_sync(full, my_n, ii), nb = __shfl_sync(full, my_n, min(ii + 1, 31));
        if (lane == 0 && !copy_failed) {
          const bool has_b = ii + 1 < nbat;
          const unsigned ba = (unsigned)(na * 4 + 15) & ~15u, bb = has_b ? (unsigned)(nb * 4 + 15) & ~15u : 0u;
          fence_proxy_async();  // the buffer's previous reads come first
          mbar_arrive_expect_tx(&s_bar[warp][buf], ba + bb);
          if (ba) bulk_g2s(&s_q[warp][buf][0][0], a.list + (size_t)(ib + ii) * L, ba, &s_bar[warp][buf]);
          if (bb) bulk_g2s(&s_q[warp][buf][1][0], a.list + (size_t)(ib + ii + 1) * L, bb, &s_bar[warp][buf]);
        }
      };
      fetch(0, 0);
      for (int ii = 0, buf = 0; ii < nbat; ii += 2, buf ^= 1) {
        const int ia = ib + ii;
        const bool has_b = ii + 1 < nbat;
        const int ibb = has_b ? ia + 1 : ia;
        int na = __shfl_sync(full, my_n, ii), nb = has_b ? __shfl_sync(full, my_n, ii + 1) : 0;
        // every lane waits for the copies, boundedly: after a copy that never
        // lands the warp issues and waits for no more copies, sums nothing for
        // its remaining particles and reports the failure (kListErrCopy)
        if (!copy_failed) {
          bool ok = false;
          for (int t = 0; t < kMbarSpinLimit && !ok; ++t) ok = mbar_try_wait(&s_bar[warp][buf], (parity >> buf) & 1u);
          parity ^= 1u << buf;
          copy_failed = !__all_sync(full, ok);
        }
        if (copy_failed) na = nb = 0;
        __syncwarp();
        if (ii + 2 < nbat) fetch(ii + 2, buf ^ 1);
        hydro_queues2<H16, true>(a, P, ia, ibb, has_b, __ldg(&a.jr[ia].a), __ldg(&a.jr[ibb].a), s_q[warp][buf][0], na,
                                 s_q[warp][buf][1], nb, &res[ii], lane);
        fence_proxy_async();  // this buffer is refilled by a bulk copy two pairs on
        __syncwarp();
      }
      __syncwarp();
      if (lane < nbat) {
        const int p = ib + lane;
        const uint32_t fp = a.alt.flags[p];
        if (fp & kDeadBit) {
          copy_state(a, p);
        } else {
          const float* r = res[lane];
          if (!(fp & kGhostBit)) pairs += (unsigned long long)r[5];
          finish_hydro(a, p, P, inst, ph, fp, r[0], r[1], r[2], r[3], r[4], (unsigned)r[5], dt_cand, dt_valid);
        }
      }
      __syncwarp();
    }
    dt_min(a.dyn, inst, dt_cand, dt_valid);
  }
  if (copy_failed && lane == 0) atomicOr(&a.list_flags[2], kListErrCopy);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(full, pairs, o);
  if (lane == 0 && pairs) atomicAdd(a.pair_count, pairs);
}

template <bool H16>
inline int launch_hydro_list(const StepArgs& a, int n, cudaStream_t s) {
  (void)n;
  static int blocks[16] = {0};
  int dev = 0;
  WCSPH_CUDA(cudaGetDevice(&dev));
  auto kern = k_hydro_list<H16, kListWarps>;
  if (!blocks[dev & 15]) {
    int per_sm = 0, sms = 0;
    WCSPH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kListWarps * 32, 0));
    WCSPH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    blocks[dev & 15] = std::max(1, per_sm) * sms;
  }
  kern<<<blocks[dev & 15], kListWarps * 32, 0, s>>>(a);
  WCSPH_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace wcsph

// Neighbour-list steps (wcsph_sim_options.list_interval > 0).
//
// A build step is an ordinary step whose tiled hydro kernel also writes, for
// every particle, the candidates within 2h + skin (the list radius) and whose
// permutation records the positions x0 the lists refer to.  The steps up to
// the next build skip the binning sort and the candidate scan:
//   k_kick_bin    KDK first half (periodic wrapping waits for the next build,
//                 so that the lists' image shifts stay valid)
//   k_refresh     state copied in place (the sorted order of the build is
//                 kept), EoS j-records refreshed, |x - x0| checked
//   k_hydro_list  the tiled kernel's pair phase over each particle's list,
//                 every entry tested for 0 < r^2 < (2h)^2 on the current
//                 positions, then the shared epilogue
// A pair within the support now was within 2h + |dx_i| + |dx_j| at the
// build, so the lists hold every pair the support test can accept while no
// particle has moved more than skin / 2 since the build.  The host rebuilds
// before that (the kick reports each step's largest drift, k_refresh the
// largest displacement); a displacement beyond skin / 2 sets a sticky error
// that the next wcsph_sim_step reports.
#pragma once
#include "sim_tiled.cuh"

namespace wcsph {

constexpr int kListWarps = 8;

// Copy main -> alt in place, refresh the j-records, check the displacement.
__global__ void k_refresh(StepArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n_host) return;
  const uint32_t f = a.main.flags[p];
  const float4 x = a.main.pos[p];
  const float4 v = a.main.vel[p];
  a.alt.pos[p] = x;
  a.alt.vel[p] = v;
  a.alt.vh[p] = a.main.vh[p];
  a.alt.acc[p] = a.main.acc[p];
  a.alt.pid[p] = a.main.pid[p];
  a.alt.flags[p] = f;
  const int inst = f & kInstMask;
  const InstParams& P = a.params[inst];
  unsigned disp_bits = 0u;
  if (!(f & kDeadBit) && P.active) {
    float pres, snds;
    tait(P, x.w, pres, snds);
    a.jA[p] = make_float4(x.x, x.y, x.z, pres / (x.w * x.w));
    a.jB[p] = make_float4(v.x, v.y, v.z, x.w);
    a.jC[p] = snds;
    const float4 o = a.x0[p];
    const float dx = x.x - o.x, dy = x.y - o.y, dz = x.z - o.z;
    const float r = sqrtf(dx * dx + dy * dy + dz * dz) * P.inv_skin;
    disp_bits = __float_as_uint(r);
    if (r > 0.5f) atomicOr(&a.list_flags[2], 1u);  // a pair may be missing from the lists
  } else {  // removed this step: never in anyone's support again
    a.jA[p] = make_float4(1.0e30f, 1.0e30f, 1.0e30f, 0.f);
    a.jB[p] = make_float4(0.f, 0.f, 0.f, 1.f);
    a.jC[p] = 0.f;
  }
  const unsigned m = __activemask();
  const unsigned mx = __reduce_max_sync(m, disp_bits);
  if ((int)(threadIdx.x & 31) == __ffs(m) - 1 && mx) atomicMax(&a.list_flags[0], mx);
}

// Pair sums of ia (and ib = ia + 1 when has_b: same instance) from their lists.
template <bool H16>
__device__ __forceinline__ void list_group(const StepArgs& a, int ia, bool has_b, float (*res)[6], int lane,
                                           unsigned long long& pairs) {
  const int ib = has_b ? ia + 1 : ia;
  const uint32_t fa = a.alt.flags[ia], fb = a.alt.flags[ib];
  const int inst = fa & kInstMask;
  const InstParams& P = a.params[inst];
  const int ph = a.phase[inst];
  if (!wants_force(P, a.dyn[inst], ph)) {
    if (lane == 0) copy_state(a, ia);
    if (lane == 1 && has_b) copy_state(a, ib);
    return;
  }
  const bool da = fa & kDeadBit, db = fb & kDeadBit;
  const int na = da ? 0 : a.list_cnt[ia];
  const int nb = (!has_b || db) ? 0 : a.list_cnt[ib];
  if (lane < 12) (&res[0][0])[lane] = 0.f;
  __syncwarp();
  const uint32_t* qa = a.list + (size_t)ia * a.list_max;
  const uint32_t* qb = a.list + (size_t)ib * a.list_max;
  hydro_queues2<H16, true>(a, P, ia, ib, has_b, a.jA[ia], a.jA[ib], qa, na, qb, nb, res, lane);
  __syncwarp();
  float dt_cand = 0.f;
  bool dt_valid = false;
  if (lane < (has_b ? 2 : 1)) {
    const int p = ia + lane;
    const uint32_t fp = lane ? fb : fa;
    const float* r = res[lane];
    if (fp & kDeadBit) {
      copy_state(a, p);
    } else {
      if (!(fp & kGhostBit)) pairs += (unsigned long long)r[5];
      finish_hydro(a, p, P, inst, ph, fp, r[0], r[1], r[2], r[3], r[4], (unsigned)r[5], dt_cand, dt_valid);
    }
  }
  dt_min(a.dyn, inst, dt_cand, dt_valid);
}

// One warp per pair of consecutive sorted slots (a pair split across two
// instances is summed one particle at a time).
template <bool H16>
__global__ void __launch_bounds__(kListWarps * 32) k_hydro_list(StepArgs a) {
  __shared__ float s_res[kListWarps][2][6];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float(*res)[6] = s_res[warp];
  const int n = *a.n_alive;
  unsigned long long pairs = 0;
  for (int q = blockIdx.x * kListWarps + warp; 2 * q < n; q += gridDim.x * kListWarps) {
    const int ia = 2 * q, ib = ia + 1;
    const bool two = ib < n;
    const bool same = two && (a.alt.flags[ia] & kInstMask) == (a.alt.flags[ib] & kInstMask);
    list_group<H16>(a, ia, same, res, lane, pairs);
    if (two && !same) {
      __syncwarp();
      list_group<H16>(a, ib, false, res, lane, pairs);
    }
    __syncwarp();
  }
  pairs = __reduce_add_sync(0xffffffffu, (unsigned)pairs);
  if (lane == 0 && pairs) atomicAdd(a.pair_count, pairs);
}

template <bool H16>
inline int launch_hydro_list(const StepArgs& a, int n, cudaStream_t s) {
  static int blocks[16] = {0};
  int dev = 0;
  WCSPH_CUDA(cudaGetDevice(&dev));
  if (!blocks[dev & 15]) {
    int per_sm = 0, sms = 0;
    WCSPH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hydro_list<H16>, kListWarps * 32, 0));
    WCSPH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    blocks[dev & 15] = std::max(1, per_sm) * sms;
  }
  const int need = (n / 2 + kListWarps) / kListWarps + 1;
  k_hydro_list<H16><<<std::min(need, blocks[dev & 15]), kListWarps * 32, 0, s>>>(a);
  WCSPH_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace wcsph

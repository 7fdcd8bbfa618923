// FDPS multiwalk plugin: wcsph_hydro_dispatch / wcsph_hydro_retrieve and the
// Shepard-filter pair, the drop-in for GPU_WC::HydrDispatchKernel /
// GPU_WC::HydrRetrieveKernel (src/kernel.cu:289-409, src/prototype.h:7-10).
//
// Data path per dispatch (one CUDA stream per tag):
//   host:   gather the FP64 fields of each walk's EPI/EPJ records (byte offsets
//           from wcsph_fdps_layout) into pinned FP32 staging records, with
//           positions taken relative to the walk's first i-particle (so FP32
//           keeps full relative precision; the reference instead scales by
//           L, v0, rho0 into half, src/kernel.cu:317-368).  OpenMP over walks.
//   H2D:    one async copy per chunk of walks, overlapping the packing of the
//           next chunk.
//   device: one CTA per walk; the walk's j-records are staged through shared
//           memory in tiles and every i of the walk (one thread each) sums over
//           all of them (walk semantics of src/kernel.cu:251-274 and
//           src/force.h:38-55).
//   D2H:    results (FP32 acc, div v, dt) copied back per chunk; retrieve
//           waits on the tag's event and scatters into the caller's RESULT
//           records in FP64.
#include <cuda_runtime.h>
#include <omp.h>
#include <algorithm>
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <vector>

#include "f32x2.cuh"
#include "wcsph_common.cuh"
#if defined(__x86_64__)
#include <immintrin.h>
#endif

namespace wcsph {

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}

int cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
  set_error("CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what, file, line);
  return (e == cudaErrorMemoryAllocation) ? WCSPH_E_NOMEM
         : (e == cudaErrorNoDevice || e == cudaErrorNoKernelImageForDevice || e == cudaErrorInsufficientDriver)
             ? WCSPH_E_NODEVICE
             : WCSPH_E_CUDA;
}

// ---------------------------------------------------------- walk kernels
// Staged records (FP32, 48 B): A = (x, y, z, h) relative to the walk origin,
// B = (vx, vy, vz, rho), C = (P/rho^2, c, nu, m).  i-records use the same
// shape (m unused).  Compact staging (36 B), used for a piece of the batch
// whose records all carry the same h, nu and m (the reference hoists them
// from the first particle, src/kernel.cu:303-304,400-401): A = (x, y, z,
// P/rho^2), B as above, and c alone in the C block; h, nu, m travel in
// WalkPair.  The kernels rebuild the full records, so both stagings give the
// same results bit for bit.
struct WalkPair {
  float alpha, beta, c_cfl, eps;
  int vsig_mode, grad_mode;
  float h, nu, m;  // compact staging: the piece's uniform h, nu, m
};

constexpr int kWalkThreads = 128;  // one thread per i; FDPS Ngroup = 128 (param.h:9)
constexpr int kWalkTile = 256;     // j-records per shared-memory tile

__device__ __forceinline__ float grad_factor(float r, float h) {  // g(r,h) with gradW = g * dr
  const float H = 2.0f * h;
  const float iH = __frcp_rn(H);
  const float K = (float)(16.0 / kPi) * iH * iH * iH * iH;
  return spline_F(r * iH) * K / r;
}

// Hydro pair sum over FDPS walks (force.h:38-57; GPU variant kernel.cu:241-280
// when VSIG/GRAD select it).  A walk's j-list is a superset of every one of
// its i's neighbours (a few per cent of the (i, j) combinations are in
// support), so the pass is split in two, per pair of i-particles and
// 1024-record tile of the j-list:
//   scan  — the tile is staged as structure-of-arrays (padded to a multiple
//           of 64 with far-away sentinels); each lane tests two adjacent
//           candidates against both i with packed f32x2 arithmetic and a
//           squared-radius bound that covers every pair of the tile (2 max h),
//           and the in-bound candidates are ballot-compacted into one queue
//           of tile indices per i.  The GPU variant's v_sig (max of -mu over
//           the whole walk, kernel.cu:263) is taken here over every j with
//           r^2 > 0, with the rounding of the pair terms;
//   pairs — lanes take consecutive queue entries (dense, no predicate
//           divergence) and evaluate the exact support test and pair terms.
// Partial sums are combined per warp with a butterfly reduce-scatter and kept
// per i in shared memory.  A block of kWQWarps warps takes kWQChunk i of one
// walk and shares the staged tile; warp w always takes the same i-pairs, so
// every sum runs in a fixed order.  The blocks come from a host-built work
// list of (walk, first i) ordered by decreasing n_i n_j: a tree walk can
// collect j-lists tens of times the median (a group whose Morton run spans
// distant regions), and those blocks start first instead of ending last.
constexpr int kWQWarps = 4;
constexpr int kWQTile = 1024;   // j-records per staged tile (queue entries are 16-bit tile indices)
constexpr int kWQChunk = 32;    // i-particles per block: a walk is split into blocks of this many i

// Dynamic shared memory of a walk block: staged j as SoA (x, y, z, h and, for
// the GPU-variant v_sig, vx, vy, vz, rho), per-i queues, per-i accumulators
// (ax, ay, az, -sum m g dr.dv, v_sig), the tile's largest h.
template <int VSIG>
struct WalkQLayout {
  static constexpr int nsoa = VSIG ? 8 : 4;
  static constexpr size_t soa = 0;
  static constexpr size_t q = soa + sizeof(float) * nsoa * kWQTile;
  static constexpr size_t res = q + sizeof(uint16_t) * kWQWarps * 2 * kWQTile;
  static constexpr size_t hmax = res + sizeof(float) * kWQChunk * 5;
  static constexpr size_t bytes = hmax + 16;
};

__device__ __forceinline__ float wq_butterfly8(const float v[8], int lane) {
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
  return y;  // warp total of slot (lane >> 2) & 7
}

// Pair terms of i (records a, b, c) with j (A, B, C): adds to
// acc = (ax, ay, az, -sum m g dr.dv) as force.h:42-54 / kernel.cu:251-273
// evaluate them (FP32).
template <int GRAD>
__device__ __forceinline__ void walk_pair(const float4& a, const float4& b, const float4& c, const float4& A,
                                          const float4& B, const float4& C, const WalkPair& pp, float acc[4]) {
  const float dx = a.x - A.x, dy = a.y - A.y, dz = a.z - A.z;
  const float r2 = dist2(dx, dy, dz);
  const float hi = a.w, hj = A.w;
  const float dvx = b.x - B.x, dvy = b.y - B.y, dvz = b.z - B.z;
  const float drdv = __fmaf_rn(dz, dvz, __fmaf_rn(dy, dvy, __fmul_rn(dx, dvx)));
  const float den = r2 + pp.eps * hi * hj;
  const float mu = drdv < 0.0f ? 0.5f * (hi + hj) * drdv / den : 0.0f;
  const float r = sqrtf(r2);
  float g;
  if (GRAD == WCSPH_GRAD_SYM) {
    g = 0.0f;
    if (r < 2.0f * hi) g += grad_factor(r, hi);
    if (r < 2.0f * hj) g += grad_factor(r, hj);
    g *= 0.5f;
  } else {
    const float hb = 0.5f * (hi + hj);
    g = (r < 2.0f * hb) ? grad_factor(r, hb) : 0.0f;
  }
  if (g == 0.0f) return;  // outside the support every term is zero
  const float rho_sum = b.w + B.w;
  const float av = (-pp.alpha * 0.5f * (c.y + C.y) * mu + pp.beta * mu * mu) * 2.0f / rho_sum;
  const float pterm = c.x + C.x + av;
  const float visc = 2.0f * (c.z + C.z) * (g * r2) / rho_sum / den;
  const float m = C.w;
  acc[0] += m * (visc * dvx - pterm * g * dx);
  acc[1] += m * (visc * dvy - pterm * g * dy);
  acc[2] += m * (visc * dvz - pterm * g * dz);
  acc[3] -= m * g * drdv;
}

// max(vs, -mu) over one more j (r2 > 0, drdv as walk_pair rounds it).  The
// running maximum is screened with a fast approximate quotient (relative
// error far below 1e-6); the exact quotient of walk_pair is taken only where
// it can raise the maximum, so the result is the maximum of the exact values.
__device__ __forceinline__ float walk_vsig(float vs, float hi, float hj, float r2, float drdv, float eps) {
  if (!(drdv < 0.0f) || !(r2 > 0.0f)) return vs;
  const float num = 0.5f * (hi + hj) * drdv;
  const float den = r2 + eps * hi * hj;
  if (__fdividef(-num, den) < vs * 0.999999f) return vs;
  return fmaxf(vs, -(num / den));
}

__device__ __forceinline__ void wq_append2(uint16_t* q, int& n, bool he, bool ho, int u, unsigned lt) {
  const unsigned me = __ballot_sync(0xffffffffu, he), mo = __ballot_sync(0xffffffffu, ho);
  const int p = n + __popc(me & lt) + __popc(mo & lt);
  if (he) q[p] = (uint16_t)u;
  if (ho) q[p + (he ? 1 : 0)] = (uint16_t)(u + 1);
  n += __popc(me) + __popc(mo);
}

// Full (A, C) records of staged record q under either staging.
template <bool COMPACT>
__device__ __forceinline__ float4 walk_rec_a(const float4* __restrict__ A, int q, const WalkPair& pp) {
  float4 r = A[q];
  if (COMPACT) r.w = pp.h;
  return r;
}
template <bool COMPACT>
__device__ __forceinline__ float4 walk_rec_c(const float4* __restrict__ A, const float4* __restrict__ C,
                                             const float* __restrict__ c, int q, const WalkPair& pp) {
  if (COMPACT) return make_float4(A[q].w, c[q], pp.nu, pp.m);
  return C[q];
}

template <int VSIG, int GRAD, bool COMPACT>
__global__ void __launch_bounds__(kWQWarps * 32, 4) k_walk_hydro(const float4* __restrict__ iA, const float4* __restrict__ iB,
                                                              const float4* __restrict__ iC, const float4* __restrict__ jA,
                                                              const float4* __restrict__ jB, const float4* __restrict__ jC,
                                                              const int* __restrict__ ni_displ,
                                                              const int* __restrict__ nj_displ,
                                                              const int2* __restrict__ items, WalkPair pp,
                                                              float4* __restrict__ out4, float* __restrict__ out_dt,
                                                              const float* __restrict__ ic,
                                                              const float* __restrict__ jc) {
  using Lay = WalkQLayout<VSIG>;
  extern __shared__ __align__(16) unsigned char wq_smem[];
  float* tx = reinterpret_cast<float*>(wq_smem + Lay::soa);
  float* ty = tx + kWQTile;
  float* tz = ty + kWQTile;
  float* th = tz + kWQTile;
  float* tvx = th + kWQTile;  // VSIG only
  float* tvy = tvx + kWQTile;
  float* tvz = tvy + kWQTile;
  float* trho = tvz + kWQTile;
  uint16_t(*sq)[2][kWQTile] = reinterpret_cast<uint16_t(*)[2][kWQTile]>(wq_smem + Lay::q);
  float(*res)[5] = reinterpret_cast<float(*)[5]>(wq_smem + Lay::res);
  unsigned* s_hmax = reinterpret_cast<unsigned*>(wq_smem + Lay::hmax);
  const unsigned full = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned lt;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
  const int2 item = items[blockIdx.x];  // (walk, first i of this block)
  const int w = item.x;
  const int i1 = ni_displ[w + 1];
  const int j0 = nj_displ[w], j1 = nj_displ[w + 1];
  uint16_t* qa = sq[warp][0];
  uint16_t* qb = sq[warp][1];
  {
    const int ib = item.y;
    const int nb = min(kWQChunk, i1 - ib);
    for (int t = threadIdx.x; t < kWQChunk * 5; t += blockDim.x) (&res[0][0])[t] = 0.0f;
    // largest h of the batch's i (h > 0: its bits order like the values)
    float hm = 0.0f;
    for (int t = threadIdx.x; t < nb; t += blockDim.x) hm = fmaxf(hm, walk_rec_a<COMPACT>(iA, ib + t, pp).w);
    for (int jb = j0; jb < j1; jb += kWQTile) {
      const int nt = min(kWQTile, j1 - jb), nt64 = (nt + 63) & ~63;
      __syncthreads();  // the previous tile's readers are done; res zeroed
      if (threadIdx.x == 0) s_hmax[0] = 0u;
      __syncthreads();
      float hj_max = hm;
      for (int k = threadIdx.x; k < nt64; k += blockDim.x) {
        if (k < nt) {
          const float4 J = walk_rec_a<COMPACT>(jA, jb + k, pp);
          tx[k] = J.x, ty[k] = J.y, tz[k] = J.z, th[k] = J.w;
          hj_max = fmaxf(hj_max, J.w);
          if (VSIG) {
            const float4 V = jB[jb + k];
            tvx[k] = V.x, tvy[k] = V.y, tvz[k] = V.z, trho[k] = V.w;
          }
        } else {  // padding: never within any bound, never approaching
          tx[k] = 1.0e30f, ty[k] = 1.0e30f, tz[k] = 1.0e30f, th[k] = 0.0f;
          if (VSIG) tvx[k] = tvy[k] = tvz[k] = trho[k] = 0.0f;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) hj_max = fmaxf(hj_max, __shfl_xor_sync(full, hj_max, o));
      if (lane == 0) atomicMax(s_hmax, __float_as_uint(hj_max));
      __syncthreads();
      // every pair of the tile lies within 2 max h (both variants), with margin
      const float Rb = 2.0f * __uint_as_float(s_hmax[0]);
      const float B2 = Rb * Rb * 1.0001f;
      for (int ip = 2 * warp; ip < nb; ip += 2 * kWQWarps) {
        const int ia = ib + ip;
        const bool has_b = ip + 1 < nb;
        const int ibb = has_b ? ia + 1 : ia;
        const float4 Aa = walk_rec_a<COMPACT>(iA, ia, pp), Ab = walk_rec_a<COMPACT>(iA, ibb, pp);
        const float4 Ba = iB[ia], Bb = iB[ibb];
        const f2 XA = dup(Aa.x), YA = dup(Aa.y), ZA = dup(Aa.z);
        const f2 XB = dup(Ab.x), YB = dup(Ab.y), ZB = dup(Ab.z);
        int na = 0, nq = 0;
        float vsa = 0.0f, vsb = 0.0f;
        for (int tb = 2 * lane; tb < nt64; tb += 64) {
          const f2 CX = *reinterpret_cast<const f2*>(&tx[tb]);
          const f2 CY = *reinterpret_cast<const f2*>(&ty[tb]);
          const f2 CZ = *reinterpret_cast<const f2*>(&tz[tb]);
          const f2 DXA = sub2(XA, CX), DYA = sub2(YA, CY), DZA = sub2(ZA, CZ);
          const f2 DXB = sub2(XB, CX), DYB = sub2(YB, CY), DZB = sub2(ZB, CZ);
          const f2 RA = fma2(DZA, DZA, fma2(DYA, DYA, mul2(DXA, DXA)));  // == dist2 per half
          const f2 RB = fma2(DZB, DZB, fma2(DYB, DYB, mul2(DXB, DXB)));
          const float ra0 = lo(RA), ra1 = hi(RA), rb0 = lo(RB), rb1 = hi(RB);
          wq_append2(qa, na, ra0 > 0.0f && ra0 < B2, ra1 > 0.0f && ra1 < B2, tb, lt);
          wq_append2(qb, nq, has_b && rb0 > 0.0f && rb0 < B2, has_b && rb1 > 0.0f && rb1 < B2, tb, lt);
          if (VSIG) {
            const f2 CVX = *reinterpret_cast<const f2*>(&tvx[tb]);
            const f2 CVY = *reinterpret_cast<const f2*>(&tvy[tb]);
            const f2 CVZ = *reinterpret_cast<const f2*>(&tvz[tb]);
            const f2 DA = fma2(DZA, sub2(dup(Ba.z), CVZ), fma2(DYA, sub2(dup(Ba.y), CVY), mul2(DXA, sub2(dup(Ba.x), CVX))));
            const f2 DB = fma2(DZB, sub2(dup(Bb.z), CVZ), fma2(DYB, sub2(dup(Bb.y), CVY), mul2(DXB, sub2(dup(Bb.x), CVX))));
            const float h0 = th[tb], h1 = th[tb + 1];
            const bool real0 = tb < nt, real1 = tb + 1 < nt;
            if (real0) vsa = walk_vsig(vsa, Aa.w, h0, ra0, lo(DA), pp.eps);
            if (real1) vsa = walk_vsig(vsa, Aa.w, h1, ra1, hi(DA), pp.eps);
            if (has_b && real0) vsb = walk_vsig(vsb, Ab.w, h0, rb0, lo(DB), pp.eps);
            if (has_b && real1) vsb = walk_vsig(vsb, Ab.w, h1, rb1, hi(DB), pp.eps);
          }
        }
        __syncwarp();
        const float4 Ca = walk_rec_c<COMPACT>(iA, iC, ic, ia, pp), Cb = walk_rec_c<COMPACT>(iA, iC, ic, ibb, pp);
        float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        const int n = max(na, nq);
        for (int k = lane; k < n; k += 32) {
          if (k < na) {
            const int u = qa[k];
            const float4 J = make_float4(tx[u], ty[u], tz[u], th[u]);
            const float4 V = VSIG ? make_float4(tvx[u], tvy[u], tvz[u], trho[u]) : jB[jb + u];
            walk_pair<GRAD>(Aa, Ba, Ca, J, V, walk_rec_c<COMPACT>(jA, jC, jc, jb + u, pp), pp, acc);
          }
          if (k < nq) {
            const int u = qb[k];
            const float4 J = make_float4(tx[u], ty[u], tz[u], th[u]);
            const float4 V = VSIG ? make_float4(tvx[u], tvy[u], tvz[u], trho[u]) : jB[jb + u];
            walk_pair<GRAD>(Ab, Bb, Cb, J, V, walk_rec_c<COMPACT>(jA, jC, jc, jb + u, pp), pp, acc + 4);
          }
        }
        const float y = wq_butterfly8(acc, lane);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          vsa = fmaxf(vsa, __shfl_xor_sync(full, vsa, o));
          vsb = fmaxf(vsb, __shfl_xor_sync(full, vsb, o));
        }
        if ((lane & 3) == 0) {
          const int slot = lane >> 2;
          if (slot < 4) res[ip][slot] += y;
          else if (has_b) res[ip + 1][slot - 4] += y;
        }
        if (lane == 0) {
          res[ip][4] = fmaxf(res[ip][4], vsa);
          if (has_b) res[ip + 1][4] = fmaxf(res[ip + 1][4], vsb);
        }
        __syncwarp();
      }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nb; t += blockDim.x) {
      const int i = ib + t;
      const float* r = res[t];
      out4[i] = make_float4(r[0], r[1], r[2], r[3] / iB[i].w);
      out_dt[i] = pp.c_cfl * walk_rec_a<COMPACT>(iA, i, pp).w /
                  (walk_rec_c<COMPACT>(iA, iC, ic, i, pp).y + r[4]);  // force.h:56 / kernel.cu:279
    }
    __syncthreads();
  }
}

// Shepard filter (force.h:12-29): rho_i = sum m W / sum (m/rho_j) W over the
// walk's j-list (which contains i itself).  iA = (x,y,z,h); jA = (x,y,z,m/rho), jB.x = m.
__global__ void __launch_bounds__(kWalkThreads) k_walk_filter(const float4* __restrict__ iA, const float4* __restrict__ jA,
                                                             const float* __restrict__ jm,
                                                             const int* __restrict__ ni_displ,
                                                             const int* __restrict__ nj_displ, int walk0,
                                                             float* __restrict__ out_dens) {
  __shared__ float4 sA[kWalkTile];
  __shared__ float sM[kWalkTile];
  const int w = walk0 + blockIdx.x;
  const int i0 = ni_displ[w], i1 = ni_displ[w + 1];
  const int j0 = nj_displ[w], j1 = nj_displ[w + 1];
  for (int ib = i0; ib < i1; ib += kWalkThreads) {
    const int i = ib + threadIdx.x;
    const bool valid = i < i1;
    const float4 a = valid ? iA[i] : make_float4(0.f, 0.f, 0.f, 1.f);
    const float H = 2.0f * a.w, iH = __frcp_rn(H);
    float one = 0.f, sum = 0.f;
    for (int jb = j0; jb < j1; jb += kWalkTile) {
      const int nt = min(kWalkTile, j1 - jb);
      __syncthreads();
      for (int k = threadIdx.x; k < nt; k += kWalkThreads) {
        sA[k] = jA[jb + k];
        sM[k] = jm[jb + k];
      }
      __syncthreads();
      if (!valid) continue;
      for (int k = 0; k < nt; ++k) {
        const float4 A = sA[k];
        const float dx = a.x - A.x, dy = a.y - A.y, dz = a.z - A.z;
        const float w_ = spline_w(sqrtf(dist2(dx, dy, dz)) * iH);
        one += w_ * A.w;
        sum += w_ * sM[k];
      }
    }
    if (valid) out_dens[i] = sum / one;  // the normalisation Kw cancels
  }
}

// ------------------------------------------------------------ plugin state
struct PinnedBuf {
  void* p = nullptr;
  size_t bytes = 0;
};
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

static int ensure_pinned(PinnedBuf& b, size_t bytes) {
  if (b.bytes >= bytes) return 0;
  const size_t want = std::max(bytes, b.bytes * 3 / 2);
  if (b.p) cudaFreeHost(b.p);
  b.p = nullptr;
  b.bytes = 0;
  WCSPH_CUDA(cudaMallocHost(&b.p, want));
  b.bytes = want;
  return 0;
}
static int ensure_dev(DevBuf& b, size_t bytes) {
  if (b.bytes >= bytes) return 0;
  const size_t want = std::max(bytes, b.bytes * 3 / 2);
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
  WCSPH_CUDA(cudaMalloc(&b.p, want));
  b.bytes = want;
  return 0;
}

enum Kind { K_NONE = 0, K_HYDRO = 1, K_FILTER = 2 };

struct TagState {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  int kind = K_NONE;  // what the last dispatch enqueued
  int n_walk = 0;
  long long ni_total = 0;
  long long h2d_bytes = 0, d2h_bytes = 0;  // of the last dispatch
  int pieces = 0, pieces_compact = 0;
  PinnedBuf h_i, h_j, h_off, h_out;
  DevBuf d_i, d_j, d_off, d_out;
};

struct Plugin {
  bool ready = false;
  int device = -1;
  wcsph_fdps_layout layout{};
  wcsph_pair_params pair{};
  TagState tags[WCSPH_FDPS_MAX_TAGS];
};

static Plugin g_plugin;
static std::mutex g_plugin_mu;

static int plugin_ready() {
  if (g_plugin.ready) return 0;
  if (g_plugin.device < 0) {
    int dev = 0;
    WCSPH_CUDA(cudaGetDevice(&dev));
    g_plugin.device = dev;
  }
  WCSPH_CUDA(cudaSetDevice(g_plugin.device));
  for (auto& t : g_plugin.tags) {
    WCSPH_CUDA(cudaStreamCreateWithFlags(&t.stream, cudaStreamNonBlocking));
    WCSPH_CUDA(cudaEventCreateWithFlags(&t.done, cudaEventDisableTiming));
  }
  g_plugin.ready = true;
  return 0;
}

// Store into the pinned staging buffers.  On x86-64 a streaming store: the
// staging is written once and read only by the copy engine, so the lines are
// not fetched into the cache first (about a fifth less host memory traffic).
static inline void st_stage(float4* dst, float x, float y, float z, float w) {
#if defined(__x86_64__)
  _mm_stream_ps(reinterpret_cast<float*>(dst), _mm_set_ps(w, z, y, x));
#else
  *dst = make_float4(x, y, z, w);
#endif
}
static inline void stage_fence() {
#if defined(__x86_64__)
  _mm_sfence();  // streaming stores are weakly ordered: complete them before the copy reads them
#endif
}

static inline double rd(const void* base, int off) {
  double v;
  memcpy(&v, (const char*)base + off, sizeof(double));
  return v;
}
static inline void wr(void* base, int off, double v) { memcpy((char*)base + off, &v, sizeof(double)); }

constexpr int kChunks = 4;  // walks are staged and copied in this many pieces

}  // namespace wcsph

using namespace wcsph;

extern "C" {

int wcsph_abi_version(void) { return WCSPH_ABI_VERSION; }
const char* wcsph_last_error(void) { return g_err.c_str(); }

void wcsph_fdps_default_layout(wcsph_fdps_layout* o) {
  // src/class.h:61-263 on x86-64 with PS::F64vec = 3 doubles.
  *o = wcsph_fdps_layout{96, 0, 24, 48, 56, 64, 72, 80,       // EPI::Hydro
                         112, 0, 24, 48, 56, 64, 72, 80, 88,  // EPJ::Hydro
                         40, 0, 24, 32,                       // RESULT::Hydro
                         32, 0, 24,                           // EPI::Filter
                         40, 0, 24, 32,                       // EPJ::Filter
                         8, 0};                               // RESULT::Filter
}

void wcsph_pair_params_reference_cpu(wcsph_pair_params* o) {
  *o = wcsph_pair_params{0.01, 0.0, 0.3, 0.01, WCSPH_VSIG_REF_CPU, WCSPH_GRAD_HBAR};
}
void wcsph_pair_params_reference_gpu(wcsph_pair_params* o) {
  *o = wcsph_pair_params{0.01, 0.02, 0.3, 0.01, WCSPH_VSIG_SIGNAL, WCSPH_GRAD_SYM};
}

int wcsph_init(int32_t device) {
  std::lock_guard<std::mutex> lk(g_plugin_mu);
  int n = 0;
  WCSPH_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) {
    set_error("wcsph_init: device %d out of range (%d devices)", device, n);
    return WCSPH_E_INVALID;
  }
  if (g_plugin.ready && g_plugin.device != device) {
    set_error("wcsph_init: plugin already bound to device %d", g_plugin.device);
    return WCSPH_E_STATE;
  }
  g_plugin.device = device;
  return plugin_ready();
}

int wcsph_finalize(void) {
  std::lock_guard<std::mutex> lk(g_plugin_mu);
  if (!g_plugin.ready) return 0;
  cudaSetDevice(g_plugin.device);
  for (auto& t : g_plugin.tags) {
    cudaStreamSynchronize(t.stream);
    for (PinnedBuf* b : {&t.h_i, &t.h_j, &t.h_off, &t.h_out})
      if (b->p) cudaFreeHost(b->p), b->p = nullptr, b->bytes = 0;
    for (DevBuf* b : {&t.d_i, &t.d_j, &t.d_off, &t.d_out})
      if (b->p) cudaFree(b->p), b->p = nullptr, b->bytes = 0;
    cudaEventDestroy(t.done);
    cudaStreamDestroy(t.stream);
    t = TagState{};
  }
  g_plugin.ready = false;
  return 0;
}

}  // extern "C"

namespace wcsph {
// Defaults (class.h layout, kernel.cu pair semantics) are installed once,
// before the first explicit configuration or dispatch, never after.
static bool g_configured_once = false;
static void default_config() {
  if (g_configured_once) return;
  wcsph_fdps_default_layout(&g_plugin.layout);
  wcsph_pair_params_reference_gpu(&g_plugin.pair);
  g_configured_once = true;
}
}  // namespace wcsph

extern "C" {

int wcsph_fdps_configure(const wcsph_fdps_layout* layout, const wcsph_pair_params* params) {
  std::lock_guard<std::mutex> lk(g_plugin_mu);
  default_config();
  if (layout) {
    const wcsph_fdps_layout& L = *layout;
    const int sz[3] = {L.epi_size, L.epj_size, L.res_size};
    if (sz[0] <= 0 || sz[1] <= 0 || sz[2] <= 0) {
      set_error("wcsph_fdps_configure: record sizes must be positive");
      return WCSPH_E_INVALID;
    }
    g_plugin.layout = L;
  }
  if (params) {
    if (params->vsig_mode < 0 || params->vsig_mode > 1 || params->grad_mode < 0 || params->grad_mode > 1) {
      set_error("wcsph_fdps_configure: bad vsig_mode/grad_mode");
      return WCSPH_E_INVALID;
    }
    g_plugin.pair = *params;
  }
  return 0;
}

}  // extern "C"

namespace wcsph {

static int check_walk_args(const char* fn, int32_t tag, int32_t n_walk, const void* const* epi, const int32_t* n_epi,
                           const void* const* epj, const int32_t* n_epj) {
  if (tag < 0 || tag >= WCSPH_FDPS_MAX_TAGS) {
    set_error("%s: tag %d outside [0, %d)", fn, tag, WCSPH_FDPS_MAX_TAGS);
    return WCSPH_E_INVALID;
  }
  if (n_walk < 0 || (n_walk > 0 && (!epi || !n_epi || !epj || !n_epj))) {
    set_error("%s: n_walk %d with null arrays", fn, n_walk);
    return WCSPH_E_INVALID;
  }
  for (int w = 0; w < n_walk; ++w)
    if (n_epi[w] < 0 || n_epj[w] < 0 || (n_epi[w] > 0 && !epi[w]) || (n_epj[w] > 0 && !epj[w])) {
      set_error("%s: walk %d has a negative count or a null record pointer", fn, w);
      return WCSPH_E_INVALID;
    }
  return 0;
}

// Where the hydro records of one dispatch are staged (SoA blocks of the
// pinned buffers) and what one piece of it is packed with.
struct HydroPack {
  const wcsph_fdps_layout* L;
  const void* const* epi;
  const void* const* epj;
  const int32_t* n_epi;
  const int32_t* n_epj;
  const long long* ni_d;
  const long long* nj_d;
  float4 *hiA, *hiB, *hiC, *hjA, *hjB, *hjC;
  bool compact;
  double h0, nu0, m0;  // compact: the piece's uniform values
  float *hic, *hjc;    // compact: c of record q at hic[q] / hjc[q], inside the piece's own part of the C blocks
};

// Origin of walk w: its first i-particle's position (or j when it has no i).
// Staged positions are relative to it.
static void walk_origin(const HydroPack& K, int w, double o[3]) {
  const wcsph_fdps_layout& L = *K.L;
  o[0] = o[1] = o[2] = 0.0;
  if (K.n_epi[w] > 0) {
    for (int k = 0; k < 3; ++k) o[k] = rd(K.epi[w], L.epi_pos + 8 * k);
  } else if (K.n_epj[w] > 0) {
    for (int k = 0; k < 3; ++k) o[k] = rd(K.epj[w], L.epj_pos + 8 * k);
  }
}

// Pack staged records [q0, q1) of one side (i or j) of walks w0.. (the walk
// of q0 found by bisection of the displacements), positions relative to each
// walk's origin org[w - w_first].  Full staging: A = (x, y, z, h),
// B = (v, rho), C = (P/rho^2, c, nu, m).  Compact: A = (x, y, z, P/rho^2), B,
// c alone.  Returns false when a record's h, nu or m differs from the piece's
// (the piece is then packed again in full).  Record-parallel: walks of very
// different sizes (a few carry 40-80x the median j-list) split evenly.
template <bool J>
static bool pack_hydro_range(const HydroPack& K, long long q0, long long q1, int w_first, int w_last,
                             const double* org) {
  const wcsph_fdps_layout& L = *K.L;
  const long long* d = J ? K.nj_d : K.ni_d;
  const void* const* base = J ? K.epj : K.epi;
  const int size = J ? L.epj_size : L.epi_size;
  const int o_pos = J ? L.epj_pos : L.epi_pos, o_vel = J ? L.epj_vel : L.epi_vel, o_dens = J ? L.epj_dens : L.epi_dens,
            o_pres = J ? L.epj_pres : L.epi_pres, o_snds = J ? L.epj_snds : L.epi_snds,
            o_smth = J ? L.epj_smth : L.epi_smth, o_visc = J ? L.epj_visc : L.epi_visc;
  float4* A = J ? K.hjA : K.hiA;
  float4* B = J ? K.hjB : K.hiB;
  float4* C = J ? K.hjC : K.hiC;
  float* c1 = J ? K.hjc : K.hic;
  // the walk holding record q0: last w with d[w] <= q0 (empty walks skipped)
  int lo = w_first, hi = w_last;  // invariant: d[lo] <= q0 < d[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) / 2;
    if (d[mid] <= q0) lo = mid;
    else hi = mid;
  }
  int w = lo;
  bool uniform = true;
  for (long long q = q0; q < q1; ++q) {
    while (q >= d[w + 1]) ++w;
    const char* r = (const char*)base[w] + (size_t)(q - d[w]) * size;
    const double* o = org + 3 * (w - w_first);
    const double dens = rd(r, o_dens);
    const float po = (float)(rd(r, o_pres) / (dens * dens));
    const float x = (float)(rd(r, o_pos) - o[0]), y = (float)(rd(r, o_pos + 8) - o[1]),
                z = (float)(rd(r, o_pos + 16) - o[2]);
    st_stage(&B[q], (float)rd(r, o_vel), (float)rd(r, o_vel + 8), (float)rd(r, o_vel + 16), (float)dens);
    if (K.compact) {
      uniform &= rd(r, o_smth) == K.h0 && rd(r, o_visc) == K.nu0 && (!J || rd(r, L.epj_mass) == K.m0);
      st_stage(&A[q], x, y, z, po);
      c1[q] = (float)rd(r, o_snds);
    } else {
      st_stage(&A[q], x, y, z, (float)rd(r, o_smth));
      st_stage(&C[q], po, (float)rd(r, o_snds), (float)rd(r, o_visc), J ? (float)rd(r, L.epj_mass) : 0.f);
    }
  }
  stage_fence();
  return uniform;
}

// Pack the i- and j-records of walks [w0, w1) on all host threads, in blocks
// of kPackBlock records.  Returns false when the piece's records are not
// uniform in h, nu and m (compact staging only).
constexpr long long kPackBlock = 2048;
static bool pack_hydro_piece(const HydroPack& K, int w0, int w1) {
  std::vector<double> org(3 * (size_t)(w1 - w0));
#pragma omp parallel for schedule(static)
  for (int w = w0; w < w1; ++w) walk_origin(K, w, &org[3 * (size_t)(w - w0)]);
  const long long a0 = K.ni_d[w0], a1 = K.ni_d[w1], b0 = K.nj_d[w0], b1 = K.nj_d[w1];
  const long long ni_blk = (a1 - a0 + kPackBlock - 1) / kPackBlock, nj_blk = (b1 - b0 + kPackBlock - 1) / kPackBlock;
  int mixed = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(| : mixed)
  for (long long t = 0; t < ni_blk + nj_blk; ++t) {
    bool u;
    if (t < nj_blk) {
      const long long q0 = b0 + t * kPackBlock;
      u = pack_hydro_range<true>(K, q0, std::min(b1, q0 + kPackBlock), w0, w1, org.data());
    } else {
      const long long q0 = a0 + (t - nj_blk) * kPackBlock;
      u = pack_hydro_range<false>(K, q0, std::min(a1, q0 + kPackBlock), w0, w1, org.data());
    }
    mixed |= u ? 0 : 1;
  }
  return !mixed;
}

// Shared dispatch body.  kind selects the record shapes and the kernel.
static int dispatch_common(int kind, int32_t tag, int32_t n_walk, const void* const* epi, const int32_t* n_epi,
                           const void* const* epj, const int32_t* n_epj) {
  const char* fn = kind == K_HYDRO ? "wcsph_hydro_dispatch" : "wcsph_filter_dispatch";
  default_config();
  if (int rc = check_walk_args(fn, tag, n_walk, epi, n_epi, epj, n_epj)) return rc;
  if (int rc = plugin_ready()) return rc;
  WCSPH_CUDA(cudaSetDevice(g_plugin.device));
  TagState& T = g_plugin.tags[tag];
  WCSPH_CUDA(cudaStreamSynchronize(T.stream));  // the tag's previous batch owns the buffers until done
  const wcsph_fdps_layout& L = g_plugin.layout;

  // Displacements (src/kernel.cu:306-310), 64-bit so huge batches cannot wrap.
  std::vector<long long> ni_d(n_walk + 1), nj_d(n_walk + 1);
  ni_d[0] = nj_d[0] = 0;
  for (int w = 0; w < n_walk; ++w) {
    ni_d[w + 1] = ni_d[w] + n_epi[w];
    nj_d[w + 1] = nj_d[w] + n_epj[w];
  }
  const long long NI = ni_d[n_walk], NJ = nj_d[n_walk];
  if (NI > INT32_MAX || NJ > INT32_MAX) {
    set_error("%s: %lld i / %lld j records exceed the 2^31 limit of one batch", fn, NI, NJ);
    return WCSPH_E_CAPACITY;
  }
  const size_t i_rec = kind == K_HYDRO ? 3 * sizeof(float4) : sizeof(float4);
  const size_t j_rec = kind == K_HYDRO ? 3 * sizeof(float4) : sizeof(float4) + sizeof(float);
  const size_t o_rec = kind == K_HYDRO ? sizeof(float4) + sizeof(float) : sizeof(float);
  if (int rc = ensure_pinned(T.h_i, i_rec * (NI + 1))) return rc;
  if (int rc = ensure_pinned(T.h_j, j_rec * (NJ + 1))) return rc;
  // Work list of the hydro kernel: (walk, first i) per block of kWQChunk i.
  long long n_items = 0;
  if (kind == K_HYDRO)
    for (int w = 0; w < n_walk; ++w) n_items += (n_epi[w] + kWQChunk - 1) / kWQChunk;
  const size_t off_bytes = sizeof(int) * 2 * (n_walk + 1) + sizeof(int2) * (size_t)n_items;
  if (int rc = ensure_pinned(T.h_off, off_bytes)) return rc;
  if (int rc = ensure_pinned(T.h_out, o_rec * (NI + 1))) return rc;
  if (int rc = ensure_dev(T.d_i, i_rec * (NI + 1))) return rc;
  if (int rc = ensure_dev(T.d_j, j_rec * (NJ + 1))) return rc;
  if (int rc = ensure_dev(T.d_off, off_bytes)) return rc;
  if (int rc = ensure_dev(T.d_out, o_rec * (NI + 1))) return rc;

  int* h_ni = (int*)T.h_off.p;
  int* h_nj = h_ni + (n_walk + 1);
  for (int w = 0; w <= n_walk; ++w) {
    h_ni[w] = (int)ni_d[w];
    h_nj[w] = (int)nj_d[w];
  }
  int* d_ni = (int*)T.d_off.p;
  int* d_nj = d_ni + (n_walk + 1);
  const int chunks = n_walk < kChunks * 64 ? 1 : kChunks;
  // Per dispatch chunk, its blocks in decreasing order of work n_i n_j (ties
  // by position, so the list is reproducible; the order never changes a result).
  int2* h_items = reinterpret_cast<int2*>(h_nj + (n_walk + 1));
  std::vector<long long> item_off(chunks + 1, 0);
  if (kind == K_HYDRO) {
    std::vector<std::pair<long long, long long>> key;  // (-work, position)
    long long pos = 0;
    for (int ch = 0; ch < chunks; ++ch) {
      const int w0 = (int)((long long)n_walk * ch / chunks), w1 = (int)((long long)n_walk * (ch + 1) / chunks);
      key.clear();
      std::vector<int2> its;
      for (int w = w0; w < w1; ++w)
        for (int i = 0; i < n_epi[w]; i += kWQChunk) {
          const long long work = (long long)std::min(kWQChunk, n_epi[w] - i) * std::max(1, n_epj[w]);
          key.emplace_back(-work, (long long)its.size());
          its.push_back(make_int2(w, (int)(ni_d[w] + i)));
        }
      std::sort(key.begin(), key.end());
      for (const auto& k : key) h_items[pos++] = its[k.second];
      item_off[ch + 1] = pos;
    }
  }
  WCSPH_CUDA(cudaMemcpyAsync(d_ni, h_ni, off_bytes, cudaMemcpyHostToDevice, T.stream));
  T.h2d_bytes = (long long)off_bytes;
  T.d2h_bytes = 0;
  T.pieces = T.pieces_compact = 0;
  const int2* d_items = reinterpret_cast<const int2*>(d_nj + (n_walk + 1));

  // SoA sub-arrays inside the staging buffers.
  float4* hiA = (float4*)T.h_i.p;
  float4* hiB = hiA + NI;
  float4* hiC = hiB + NI;
  float4* hjA = (float4*)T.h_j.p;
  float4* hjB = hjA + NJ;
  float4* hjC = hjB + NJ;
  float* hjm = (float*)(hjA + NJ);  // filter: m after the A block
  float4* diA = (float4*)T.d_i.p;
  float4* djA = (float4*)T.d_j.p;

  for (int ch = 0; ch < chunks; ++ch) {
    const int w0 = (int)((long long)n_walk * ch / chunks), w1 = (int)((long long)n_walk * (ch + 1) / chunks);
    if (w0 == w1) continue;
    bool compact = false;
    WalkPair pp{(float)g_plugin.pair.alpha, (float)g_plugin.pair.beta, (float)g_plugin.pair.c_cfl,
                (float)g_plugin.pair.eps, g_plugin.pair.vsig_mode, g_plugin.pair.grad_mode, 0.f, 0.f, 0.f};
    if (kind == K_HYDRO) {
      // A compact piece keeps c of record q at float 3 a0 + q of the C block:
      // bytes [16 a0, 16 a0 + 4 (a1 - a0)), inside the piece's own part
      // [16 a0, 16 a1) (the copies of earlier pieces may still be reading
      // theirs).
      HydroPack K{&L, epi, epj, n_epi, n_epj, ni_d.data(), nj_d.data(), hiA, hiB, hiC, hjA, hjB, hjC, false, 0, 0, 0,
                  reinterpret_cast<float*>(hiC) + 3 * ni_d[w0], reinterpret_cast<float*>(hjC) + 3 * nj_d[w0]};
      // Compact staging when every record of the piece carries the h, nu and
      // m of its first j-record (checked while packing).
      for (int w = w0; w < w1 && !K.compact; ++w)
        if (n_epj[w] > 0) {
          const char* r = (const char*)epj[w];
          K.compact = true;
          K.h0 = rd(r, L.epj_smth), K.nu0 = rd(r, L.epj_visc), K.m0 = rd(r, L.epj_mass);
        }
      if (!pack_hydro_piece(K, w0, w1) && K.compact) {
        K.compact = false;
        pack_hydro_piece(K, w0, w1);
      }
      compact = K.compact;
      if (compact) pp.h = (float)K.h0, pp.nu = (float)K.nu0, pp.m = (float)K.m0;
      ++T.pieces;
      T.pieces_compact += compact ? 1 : 0;
    } else {
#pragma omp parallel for schedule(dynamic, 16)
      for (int w = w0; w < w1; ++w) {
        const char* pi = (const char*)epi[w];
        const char* pj = (const char*)epj[w];
        double o[3] = {0, 0, 0};
        if (n_epi[w] > 0) {
          for (int k = 0; k < 3; ++k) o[k] = rd(pi, L.fepi_pos + 8 * k);
        } else if (n_epj[w] > 0) {
          for (int k = 0; k < 3; ++k) o[k] = rd(pj, L.fepj_pos + 8 * k);
        }
        for (int i = 0; i < n_epi[w]; ++i) {
          const char* r = pi + (size_t)i * L.fepi_size;
          hiA[ni_d[w] + i] = make_float4((float)(rd(r, L.fepi_pos) - o[0]), (float)(rd(r, L.fepi_pos + 8) - o[1]),
                                         (float)(rd(r, L.fepi_pos + 16) - o[2]), (float)rd(r, L.fepi_smth));
        }
        for (int j = 0; j < n_epj[w]; ++j) {
          const char* r = pj + (size_t)j * L.fepj_size;
          const double m = rd(r, L.fepj_mass);
          hjA[nj_d[w] + j] = make_float4((float)(rd(r, L.fepj_pos) - o[0]), (float)(rd(r, L.fepj_pos + 8) - o[1]),
                                         (float)(rd(r, L.fepj_pos + 16) - o[2]), (float)(m / rd(r, L.fepj_dens)));
          hjm[nj_d[w] + j] = (float)m;
        }
      }
    }
    // H2D of this chunk's records (SoA blocks copied piecewise).
    const long long a0 = ni_d[w0], a1 = ni_d[w1], b0 = nj_d[w0], b1 = nj_d[w1];
    // the third block carries full float4 records, or only c (compact staging,
    // at the start of the piece's part of the block)
    auto h2d = [&](void* dst, const void* src, size_t bytes) -> int {
      if (bytes == 0) return 0;
      WCSPH_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, T.stream));
      T.h2d_bytes += (long long)bytes;
      return 0;
    };
    int rc = 0;
    if (kind == K_HYDRO) {
      if (a1 > a0) {
        rc |= h2d(diA + a0, hiA + a0, sizeof(float4) * (a1 - a0));
        rc |= h2d(diA + NI + a0, hiB + a0, sizeof(float4) * (a1 - a0));
        rc |= h2d(diA + 2 * NI + a0, hiC + a0, (compact ? sizeof(float) : sizeof(float4)) * (a1 - a0));
      }
      if (b1 > b0) {
        rc |= h2d(djA + b0, hjA + b0, sizeof(float4) * (b1 - b0));
        rc |= h2d(djA + NJ + b0, hjB + b0, sizeof(float4) * (b1 - b0));
        rc |= h2d(djA + 2 * NJ + b0, hjC + b0, (compact ? sizeof(float) : sizeof(float4)) * (b1 - b0));
      }
    } else {
      if (a1 > a0) rc |= h2d(diA + a0, hiA + a0, sizeof(float4) * (a1 - a0));
      if (b1 > b0) {
        rc |= h2d(djA + b0, hjA + b0, sizeof(float4) * (b1 - b0));
        rc |= h2d((float*)(djA + NJ) + b0, hjm + b0, sizeof(float) * (b1 - b0));
      }
    }
    if (rc) return rc;
    // One CTA per walk.
    if (kind == K_HYDRO) {
      float4* out4 = (float4*)T.d_out.p;
      float* out_dt = (float*)(out4 + NI);
      auto kern = compact ? (pp.vsig_mode ? (pp.grad_mode ? k_walk_hydro<1, 1, true> : k_walk_hydro<1, 0, true>)
                                          : (pp.grad_mode ? k_walk_hydro<0, 1, true> : k_walk_hydro<0, 0, true>))
                          : (pp.vsig_mode ? (pp.grad_mode ? k_walk_hydro<1, 1, false> : k_walk_hydro<1, 0, false>)
                                          : (pp.grad_mode ? k_walk_hydro<0, 1, false> : k_walk_hydro<0, 0, false>));
      const int smem = (int)(pp.vsig_mode ? WalkQLayout<1>::bytes : WalkQLayout<0>::bytes);
      WCSPH_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      const long long nblk = item_off[ch + 1] - item_off[ch];
      if (nblk > 0) {
        kern<<<(unsigned)nblk, kWQWarps * 32, smem, T.stream>>>(diA, diA + NI, diA + 2 * NI, djA, djA + NJ,
                                                                djA + 2 * NJ, d_ni, d_nj, d_items + item_off[ch], pp,
                                                                out4, out_dt,
                                                                reinterpret_cast<const float*>(diA + 2 * NI) + 3 * a0,
                                                                reinterpret_cast<const float*>(djA + 2 * NJ) + 3 * b0);
        WCSPH_CUDA(cudaGetLastError());
      }
      if (a1 > a0) {
        WCSPH_CUDA(cudaMemcpyAsync((float4*)T.h_out.p + a0, out4 + a0, sizeof(float4) * (a1 - a0),
                                   cudaMemcpyDeviceToHost, T.stream));
        WCSPH_CUDA(cudaMemcpyAsync((float*)((float4*)T.h_out.p + NI) + a0, out_dt + a0, sizeof(float) * (a1 - a0),
                                   cudaMemcpyDeviceToHost, T.stream));
        T.d2h_bytes += (long long)(sizeof(float4) + sizeof(float)) * (a1 - a0);
      }
    } else {
      float* out = (float*)T.d_out.p;
      k_walk_filter<<<w1 - w0, kWalkThreads, 0, T.stream>>>(diA, djA, (const float*)(djA + NJ), d_ni, d_nj, w0, out);
      WCSPH_CUDA(cudaGetLastError());
      if (a1 > a0) {
        WCSPH_CUDA(cudaMemcpyAsync((float*)T.h_out.p + a0, out + a0, sizeof(float) * (a1 - a0), cudaMemcpyDeviceToHost,
                                   T.stream));
        T.d2h_bytes += (long long)sizeof(float) * (a1 - a0);
      }
    }
  }
  WCSPH_CUDA(cudaEventRecord(T.done, T.stream));
  T.kind = kind;
  T.n_walk = n_walk;
  T.ni_total = NI;
  return 0;
}

static int retrieve_common(int kind, int32_t tag, int32_t n_walk, const int32_t* n_i, void* const* force) {
  const char* fn = kind == K_HYDRO ? "wcsph_hydro_retrieve" : "wcsph_filter_retrieve";
  if (tag < 0 || tag >= WCSPH_FDPS_MAX_TAGS) {
    set_error("%s: tag %d outside [0, %d)", fn, tag, WCSPH_FDPS_MAX_TAGS);
    return WCSPH_E_INVALID;
  }
  TagState& T = g_plugin.tags[tag];
  if (!g_plugin.ready || T.kind != kind) {
    set_error("%s: no pending dispatch of this kind for tag %d", fn, tag);
    return WCSPH_E_STATE;
  }
  if (n_walk != T.n_walk || (n_walk > 0 && (!n_i || !force))) {
    set_error("%s: n_walk %d does not match the dispatch (%d) or null arrays", fn, n_walk, T.n_walk);
    return WCSPH_E_INVALID;
  }
  std::vector<long long> off(n_walk + 1);
  off[0] = 0;
  for (int w = 0; w < n_walk; ++w) off[w + 1] = off[w] + n_i[w];
  if (off[n_walk] != T.ni_total) {
    set_error("%s: %lld i-particles requested, %lld dispatched", fn, off[n_walk], T.ni_total);
    return WCSPH_E_INVALID;
  }
  WCSPH_CUDA(cudaEventSynchronize(T.done));
  const wcsph_fdps_layout& L = g_plugin.layout;
  const long long NI = T.ni_total;
  if (kind == K_HYDRO) {
    const float4* o4 = (const float4*)T.h_out.p;
    const float* odt = (const float*)(o4 + NI);
#pragma omp parallel for schedule(dynamic, 64)
    for (int w = 0; w < n_walk; ++w) {
      char* base = (char*)force[w];
      for (int i = 0; i < n_i[w]; ++i) {
        const float4 a = o4[off[w] + i];
        char* r = base + (size_t)i * L.res_size;
        wr(r, L.res_acc, a.x);
        wr(r, L.res_acc + 8, a.y);
        wr(r, L.res_acc + 16, a.z);
        wr(r, L.res_div_v, a.w);
        wr(r, L.res_dt, odt[off[w] + i]);
      }
    }
  } else {
    const float* od = (const float*)T.h_out.p;
#pragma omp parallel for schedule(dynamic, 64)
    for (int w = 0; w < n_walk; ++w) {
      char* base = (char*)force[w];
      for (int i = 0; i < n_i[w]; ++i) wr(base + (size_t)i * L.fres_size, L.fres_dens, od[off[w] + i]);
    }
  }
  T.kind = K_NONE;
  return 0;
}
}  // namespace wcsph

extern "C" {
int wcsph_hydro_dispatch(int32_t tag, int32_t n_walk, const void* const* epi, const int32_t* n_epi,
                         const void* const* epj, const int32_t* n_epj) {
  std::lock_guard<std::mutex> lk(g_plugin_mu);
  return dispatch_common(K_HYDRO, tag, n_walk, epi, n_epi, epj, n_epj);
}
int wcsph_hydro_retrieve(int32_t tag, int32_t n_walk, const int32_t* n_i, void* const* force) {
  std::lock_guard<std::mutex> lk(g_plugin_mu);
  return retrieve_common(K_HYDRO, tag, n_walk, n_i, force);
}
int wcsph_filter_dispatch(int32_t tag, int32_t n_walk, const void* const* epi, const int32_t* n_epi,
                          const void* const* epj, const int32_t* n_epj) {
  std::lock_guard<std::mutex> lk(g_plugin_mu);
  return dispatch_common(K_FILTER, tag, n_walk, epi, n_epi, epj, n_epj);
}
int wcsph_filter_retrieve(int32_t tag, int32_t n_walk, const int32_t* n_i, void* const* result) {
  std::lock_guard<std::mutex> lk(g_plugin_mu);
  return retrieve_common(K_FILTER, tag, n_walk, n_i, result);
}
int wcsph_fdps_stats(int32_t tag, int64_t* out4) {
  if (tag < 0 || tag >= WCSPH_FDPS_MAX_TAGS || !out4) {
    set_error("wcsph_fdps_stats: bad tag %d or null output", tag);
    return WCSPH_E_INVALID;
  }
  std::lock_guard<std::mutex> lk(g_plugin_mu);
  const TagState& T = g_plugin.tags[tag];
  out4[0] = T.h2d_bytes;
  out4[1] = T.d2h_bytes;
  out4[2] = T.pieces_compact;
  out4[3] = T.pieces;
  return 0;
}
}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free walk pair sum.
//
// For callers that cannot allocate device memory: hosts that hand the plugin a
// fixed memory budget and forbid growth, embedders whose allocator owns every
// device byte, and host loops in which a cudaMalloc would synchronise the
// device in the middle of a step.  The caller passes device-resident inputs
// and outputs; the only scratch this path needs, the per-walk displacement
// tables (exclusive prefix sums of the walk sizes), lives in the file-scope
// array below, sized for WCSPH_NOALLOC_MAX_WALKS walks (about 512 KB, held on
// every GPU that loads the library until the process exits).
namespace wcsph {

static __device__ __align__(256) int g_noalloc_displ[2 * (WCSPH_NOALLOC_MAX_WALKS + 1)];

// Exclusive prefix sums of the two count arrays into g_noalloc_displ-shaped
// scratch: displ[0..n] for i-counts, displ[n+1 .. 2n+1] for j-counts.  One
// block; every entry it later reads is written, so nothing needs clearing.
__global__ void __launch_bounds__(1024) k_noalloc_displ(int n, const int* __restrict__ n_epi,
                                                       const int* __restrict__ n_epj, int* displ) {
  __shared__ int warp_tot[2][32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int per = (n + 1023) / 1024;
  const int b = min(n, tid * per), e = min(n, b + per);
  int si = 0, sj = 0;
  for (int k = b; k < e; ++k) {
    si += n_epi[k];
    sj += n_epj[k];
  }
  int ii = si, ij = sj;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int ti = __shfl_up_sync(0xffffffffu, ii, o), tj = __shfl_up_sync(0xffffffffu, ij, o);
    if (lane >= o) ii += ti, ij += tj;
  }
  if (lane == 31) warp_tot[0][warp] = ii, warp_tot[1][warp] = ij;
  __syncthreads();
  if (warp == 0) {
    int wi = warp_tot[0][lane], wj = warp_tot[1][lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int ti = __shfl_up_sync(0xffffffffu, wi, o), tj = __shfl_up_sync(0xffffffffu, wj, o);
      if (lane >= o) wi += ti, wj += tj;
    }
    warp_tot[0][lane] = wi;
    warp_tot[1][lane] = wj;
  }
  __syncthreads();
  int oi = ii - si + (warp > 0 ? warp_tot[0][warp - 1] : 0);
  int oj = ij - sj + (warp > 0 ? warp_tot[1][warp - 1] : 0);
  for (int k = b; k < e; ++k) {
    displ[k] = oi;
    displ[n + 1 + k] = oj;
    oi += n_epi[k];
    oj += n_epj[k];
  }
  if (tid == 1023) {
    displ[n] = oi;
    displ[2 * n + 1] = oj;
  }
}

// The walk pair sum of k_walk_hydro with records interleaved per particle
// (three float4 per record) and results as two float4 per i-particle.
template <int VSIG, int GRAD>
__global__ void __launch_bounds__(kWalkThreads) k_walk_hydro_interleaved(const float4* __restrict__ ei,
                                                                        const float4* __restrict__ ej,
                                                                        const int* __restrict__ displ, int n_walk,
                                                                        WalkPair pp, float4* __restrict__ out) {
  __shared__ float4 sA[kWalkTile], sB[kWalkTile], sC[kWalkTile];
  const int w = blockIdx.x;
  const int i0 = displ[w], i1 = displ[w + 1];
  const int j0 = displ[n_walk + 1 + w], j1 = displ[n_walk + 2 + w];
  for (int ib = i0; ib < i1; ib += kWalkThreads) {
    const int i = ib + threadIdx.x;
    const bool valid = i < i1;
    float4 a = make_float4(0.f, 0.f, 0.f, 1.f), b = make_float4(0.f, 0.f, 0.f, 1.f), c = make_float4(0.f, 1.f, 0.f, 0.f);
    if (valid) {
      a = ei[3 * (size_t)i];
      b = ei[3 * (size_t)i + 1];
      c = ei[3 * (size_t)i + 2];
    }
    float ax = 0.f, ay = 0.f, az = 0.f, dv_acc = 0.f, vsig = 0.f;
    for (int jb = j0; jb < j1; jb += kWalkTile) {
      const int nt = min(kWalkTile, j1 - jb);
      __syncthreads();
      for (int k = threadIdx.x; k < nt; k += kWalkThreads) {
        sA[k] = ej[3 * (size_t)(jb + k)];
        sB[k] = ej[3 * (size_t)(jb + k) + 1];
        sC[k] = ej[3 * (size_t)(jb + k) + 2];
      }
      __syncthreads();
      if (!valid) continue;
      for (int k = 0; k < nt; ++k) {
        const float4 A = sA[k];
        const float dx = a.x - A.x, dy = a.y - A.y, dz = a.z - A.z;
        const float r2 = dist2(dx, dy, dz);
        if (!(r2 > 0.0f)) continue;
        const float4 B = sB[k];
        const float hi = a.w, hj = A.w;
        const float dvx = b.x - B.x, dvy = b.y - B.y, dvz = b.z - B.z;
        const float drdv = dx * dvx + dy * dvy + dz * dvz;
        const float den = r2 + pp.eps * hi * hj;
        const float mu = drdv < 0.0f ? 0.5f * (hi + hj) * drdv / den : 0.0f;
        vsig = VSIG ? fmaxf(vsig, -mu) : fmaxf(vsig, mu);
        const float r = sqrtf(r2);
        float g;
        if (GRAD == WCSPH_GRAD_SYM) {
          g = 0.0f;
          if (r < 2.0f * hi) g += grad_factor(r, hi);
          if (r < 2.0f * hj) g += grad_factor(r, hj);
          g *= 0.5f;
        } else {
          const float hb = 0.5f * (hi + hj);
          g = (r < 2.0f * hb) ? grad_factor(r, hb) : 0.0f;
        }
        if (g == 0.0f) continue;
        const float4 C = sC[k];
        const float rho_sum = b.w + B.w;
        const float av = (-pp.alpha * 0.5f * (c.y + C.y) * mu + pp.beta * mu * mu) * 2.0f / rho_sum;
        const float pterm = c.x + C.x + av;
        const float visc = 2.0f * (c.z + C.z) * (g * r2) / rho_sum / den;
        const float m = C.w;
        ax += m * (visc * dvx - pterm * g * dx);
        ay += m * (visc * dvy - pterm * g * dy);
        az += m * (visc * dvz - pterm * g * dz);
        dv_acc -= m * g * drdv;
      }
    }
    if (valid) {
      out[2 * (size_t)i] = make_float4(ax, ay, az, dv_acc / b.w);
      out[2 * (size_t)i + 1] = make_float4(pp.c_cfl * a.w / (c.y + vsig), 0.f, 0.f, 0.f);
    }
  }
}

// Device address of the scratch array, looked up once per device.
static int* g_noalloc_ptr[64];
static std::mutex g_noalloc_mu;

static int noalloc_scratch(int** out) {
  int dev = 0;
  WCSPH_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("wcsph_hydro_walks_noalloc: device ordinal %d is beyond the supported 64", dev);
    return WCSPH_E_NODEVICE;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_displ);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_displ)", __FILE__, __LINE__);
    g_noalloc_ptr[dev] = (int*)p;
  }
  *out = g_noalloc_ptr[dev];
  return 0;
}

}  // namespace wcsph

extern "C" int wcsph_hydro_walks_noalloc(int32_t n_walk, const int32_t* d_n_epi, const int32_t* d_n_epj,
                                         const void* d_epi, const void* d_epj, void* d_out,
                                         const wcsph_pair_params* params, void* stream) {
  if (n_walk < 0 || !params) {
    set_error("wcsph_hydro_walks_noalloc: n_walk %d < 0 or null params", n_walk);
    return WCSPH_E_INVALID;
  }
  if (n_walk > WCSPH_NOALLOC_MAX_WALKS) {
    set_error("wcsph_hydro_walks_noalloc: %d walks exceed the allocation-free limit of %d walks per call", n_walk,
              WCSPH_NOALLOC_MAX_WALKS);
    return WCSPH_E_CAPACITY;
  }
  if (params->vsig_mode < 0 || params->vsig_mode > 1 || params->grad_mode < 0 || params->grad_mode > 1) {
    set_error("wcsph_hydro_walks_noalloc: bad vsig_mode/grad_mode");
    return WCSPH_E_INVALID;
  }
  if (n_walk == 0) return 0;
  if (!d_n_epi || !d_n_epj || !d_epi || !d_epj || !d_out) {
    set_error("wcsph_hydro_walks_noalloc: null device pointer");
    return WCSPH_E_INVALID;
  }
  int* displ = nullptr;
  if (int rc = noalloc_scratch(&displ)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  k_noalloc_displ<<<1, 1024, 0, s>>>(n_walk, d_n_epi, d_n_epj, displ);
  const WalkPair pp{(float)params->alpha, (float)params->beta, (float)params->c_cfl, (float)params->eps,
                    params->vsig_mode, params->grad_mode};
  auto kern = pp.vsig_mode ? (pp.grad_mode ? k_walk_hydro_interleaved<1, 1> : k_walk_hydro_interleaved<1, 0>)
                           : (pp.grad_mode ? k_walk_hydro_interleaved<0, 1> : k_walk_hydro_interleaved<0, 0>);
  kern<<<n_walk, kWalkThreads, 0, s>>>((const float4*)d_epi, (const float4*)d_epj, displ, n_walk, pp, (float4*)d_out);
  WCSPH_CUDA(cudaGetLastError());
  return 0;
}

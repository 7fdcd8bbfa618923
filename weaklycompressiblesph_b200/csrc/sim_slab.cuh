// Slab decomposition of one simulation over several solvers (one per GPU):
// each rank's instance owns the particles with x in [x_lo, x_hi) and holds
// ghost copies of its neighbours' particles within a layer of width W beyond
// each face.  After every step the rank
//   1. classifies its particles (k_slab_classify): owned particles that left
//      the slab are emigrants, owned particles within W of a face are sent to
//      that neighbour as ghosts, everything else stays;
//   2. orders them by class with a stable radix sort (so the records follow
//      the sorted cell order of the last step and the exchange is
//      deterministic) and packs 64-byte records (k_slab_pack) in the order
//      [emigrants left, ghosts left, emigrants right, ghosts right];
//   3. retires its previous ghosts and turns its emigrants into ghosts
//      (k_slab_commit): an emigrant sits just past the face, where this rank
//      needs it as a ghost until its new owner sends it back as one;
//   4. appends what its neighbours sent (k_slab_unpack): their emigrants as
//      owned particles, their layer as ghosts.
// Ghosts are kicked and drifted by the receiver with the same arithmetic as
// by their owner, so their positions at the next force pass are the owner's.
// W = 2 (2h) + 2 margin covers the pair sums of the owned particles (support
// 2h) and the density passes of the ghosts those sums read (another 2h), with
// every particle drifting at most `margin` in the step; k_kick_bin flags a
// larger drift (kErrDrift) and the next pack reports it.
// This replaces the domain decomposition and particle exchange FDPS runs
// every step (src/main.cpp:61-62,109-110).
#pragma once
#include "sim_kernels.cuh"

namespace wcsph {

struct SlabRecord {
  float4 pos;     // x, y, z, rho
  float4 vel;     // vx, vy, vz, 0
  float4 acc;     // ax, ay, az, div v
  int id;         // index in the instance's id space
  uint32_t type;  // WCSPH_HYDRO or WCSPH_FREEZE
  int pad[2];
};
static_assert(sizeof(SlabRecord) == WCSPH_SLAB_RECORD_BYTES, "slab record size");

enum SlabClass : uint32_t { SL_EMIG_L = 0, SL_GHOST_L = 1, SL_EMIG_R = 2, SL_GHOST_R = 3, SL_STAY = 4 };
constexpr int kSlabClassBits = 3;

struct SlabGeom {
  float x_lo, x_hi, W;
  int has_left, has_right;
};

__device__ __forceinline__ uint32_t slab_class(const SlabGeom& G, uint32_t f, int slot, float x) {
  if ((int)(f & kInstMask) != slot || (f & (kDeadBit | kGhostBit))) return SL_STAY;
  if (G.has_left && x < G.x_lo) return SL_EMIG_L;
  if (G.has_right && x >= G.x_hi) return SL_EMIG_R;
  if (G.has_left && x < G.x_lo + G.W) return SL_GHOST_L;
  if (G.has_right && x >= G.x_hi - G.W) return SL_GHOST_R;
  return SL_STAY;
}

// cls[p] = class, idx[p] = p; counts[c] += 1 for the four sent classes.
__global__ void k_slab_classify(SimArrays A, int n, int slot, SlabGeom G, uint32_t* cls, int* idx, int* counts) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t c = SL_STAY;
  if (p < n) {
    c = slab_class(G, A.flags[p], slot, A.pos[p].x);
    cls[p] = c;
    idx[p] = p;
  }
  const unsigned full = 0xffffffffu;
#pragma unroll
  for (uint32_t k = 0; k < 4; ++k) {
    const unsigned m = __ballot_sync(full, c == k);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(&counts[k], __popc(m));
  }
}

// Record q of the send buffer from sorted entry q (classes 0-3 come first).
__global__ void k_slab_pack(SimArrays A, const int* idx_sorted, int total, SlabRecord* out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= total) return;
  const int p = idx_sorted[q];
  SlabRecord r;
  r.pos = A.pos[p];
  r.vel = A.vel[p];
  r.acc = A.acc[p];
  r.id = A.pid[p];
  r.type = (A.flags[p] & kFreezeBit) ? (uint32_t)WCSPH_FREEZE : (uint32_t)WCSPH_HYDRO;
  r.pad[0] = r.pad[1] = 0;
  out[q] = r;
}

// Retire the previous ghosts; emigrants stay on as ghosts.
__global__ void k_slab_commit(SimArrays A, int n, int slot, SlabGeom G) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const uint32_t f = A.flags[p];
  if ((int)(f & kInstMask) != slot || (f & kDeadBit)) return;
  if (f & kGhostBit) {
    A.flags[p] = f | kDeadBit;
    return;
  }
  const uint32_t c = slab_class(G, f, slot, A.pos[p].x);
  if (c == SL_EMIG_L || c == SL_EMIG_R) A.flags[p] = f | kGhostBit;
}

// Append n records at [base, base + n): the first n_owned as owned particles,
// the rest as ghosts.
__global__ void k_slab_unpack(SimArrays A, int base, int n, int n_owned, int slot, const SlabRecord* in) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const SlabRecord r = in[q];
  const int p = base + q;
  A.pos[p] = r.pos;
  A.vel[p] = r.vel;
  A.vh[p] = r.vel;
  A.acc[p] = r.acc;
  A.pid[p] = r.id;
  A.flags[p] = (uint32_t)slot | (r.type == (uint32_t)WCSPH_FREEZE ? kFreezeBit : 0u) | (q >= n_owned ? kGhostBit : 0u);
}

}  // namespace wcsph

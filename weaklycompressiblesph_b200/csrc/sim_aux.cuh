// Conservation sums of one instance's live particles, accumulated in FP64 on
// the device: out[0] total mass, out[1..3] momentum, out[4] kinetic energy,
// out[5] sum m (a_z + g), the vertical component of the pair forces' total
// (gravity taken out): zero up to rounding, since every pair term enters the
// sums of i and j with opposite signs (force.h:38-57).
#pragma once
#include "sim_kernels.cuh"

namespace wcsph {

__global__ void k_conservation(SimArrays A, const InstDyn* dyn, const InstParams* params, int slot, double* out) {
  const int lo = dyn[slot].range_lo, hi = dyn[slot].range_hi;
  const double m = params[slot].mass, g = params[slot].g;
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (int p = lo + blockIdx.x * blockDim.x + threadIdx.x; p < hi; p += gridDim.x * blockDim.x) {
    // a slab's ghost copies belong to their owner's sums; particles removed
    // since the last neighbour-list build stay in place until the next one
    if (A.flags[p] & (kGhostBit | kDeadBit)) continue;
    const float4 v = A.vel[p];
    const float4 a = A.acc[p];
    s[0] += m;
    s[1] += m * v.x;
    s[2] += m * v.y;
    s[3] += m * v.z;
    s[4] += 0.5 * m * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
    s[5] += m * ((double)a.z + g);
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double x = s[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0 && x != 0.0) atomicAdd(&out[k], x);
  }
}

inline int launch_conservation(const SimArrays& A, const InstDyn* dyn, const InstParams* params, int slot,
                               double* d_scratch, cudaStream_t s, double* out6) {
  WCSPH_CUDA(cudaMemsetAsync(d_scratch, 0, 6 * sizeof(double), s));
  k_conservation<<<296, 256, 0, s>>>(A, dyn, params, slot, d_scratch);
  WCSPH_CUDA(cudaGetLastError());
  WCSPH_CUDA(cudaMemcpyAsync(out6, d_scratch, 6 * sizeof(double), cudaMemcpyDeviceToHost, s));
  WCSPH_CUDA(cudaStreamSynchronize(s));
  return 0;
}

}  // namespace wcsph

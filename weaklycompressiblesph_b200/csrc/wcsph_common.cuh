// Shared device-side definitions: cubic-spline kernel, Tait EoS, instance
// parameter records, Morton keys, error plumbing.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "wcsph.h"

namespace wcsph {

// ---------------------------------------------------------------- errors ---
void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

inline int cuda_fail_if(cudaError_t e) { return e == cudaSuccess ? 0 : cuda_fail(e, "kernel launch", __FILE__, __LINE__); }

#define WCSPH_CUDA(call)                                                 \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) return ::wcsph::cuda_fail(e_, #call, __FILE__, __LINE__); \
  } while (0)

// ------------------------------------------------------- cubic spline ---
// 3-D cubic spline of the reference (kernel.h:27-55), support H = 2h:
//   W(r)     = [(1-s)+^3 - 4 (1/2-s)+^3] * Kw,      Kw = 16 / (pi H^3)
//   gradW(r) = dr * [12 (1/2-s)+^2 - 3 (1-s)+^2] * Kw / (r H) = g * dr
constexpr double kPi = 3.14159265358979323846;

__device__ __forceinline__ float spline_F(float s) {  // 12 (1/2-s)+^2 - 3 (1-s)+^2
  const float a = fmaxf(1.0f - s, 0.0f), b = fmaxf(0.5f - s, 0.0f);
  return 12.0f * b * b - 3.0f * a * a;
}
__device__ __forceinline__ float spline_w(float s) {  // (1-s)+^3 - 4 (1/2-s)+^3
  const float a = fmaxf(1.0f - s, 0.0f), b = fmaxf(0.5f - s, 0.0f);
  return a * a * a - 4.0f * b * b * b;
}

// ------------------------------------------------------------- Morton ---
__host__ __device__ __forceinline__ uint32_t spread3(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
__host__ __device__ __forceinline__ uint32_t compact3(uint32_t v) {
  v &= 0x09249249u;
  v = (v | (v >> 2)) & 0x030C30C3u;
  v = (v | (v >> 4)) & 0x0300F00Fu;
  v = (v | (v >> 8)) & 0x030000FFu;
  v = (v | (v >> 16)) & 0x3ffu;
  return v;
}
__host__ __device__ __forceinline__ uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

// Cell of a coordinate, FP32, clamped (the oracle evaluates the same expression).
__device__ __forceinline__ int cell_of(float x, float lo, float inv, int n) {
  int c = (int)floorf(__fmul_rn(__fsub_rn(x, lo), inv));
  return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

// Periodic images: a candidate j visited through a neighbour cell whose index
// wrapped past the box edge on an axis is taken at x_j + s L (s = +1 past the
// high edge, -1 past the low edge); the displacement is x_i - (x_j + s L),
// two rounded FP32 operations.  The oracle uses the same convention.

// Squared distance as the neighbour predicate defines it.
__device__ __forceinline__ float dist2(float dx, float dy, float dz) {
  return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

// -------------------------------------------------- instance parameters ---
// Static per-instance record (uploaded when the instance set changes).
struct InstParams {
  float lo[3], inv_cell[3];
  float L[3], halfL[3];   // periodic box edge and half edge
  int ncell[3];
  int cell_base;          // first linear cell of this instance in the global table
  uint32_t key_base;      // first Morton key of this instance in the global key space
  int periodic;
  int active;
  int density_mode, shepard_interval, vsig_mode, kill_on;
  // physics in FP32, precomputed
  float h, H2, inv_H, Kg, Kw, W0, mass, nu4, eh2, alpha, beta, c_cfl;
  float rho0, inv_rho0, B, gamma, cs2_coef /* B*gamma/rho0 */, c0 /* sqrt(cs2_coef) */, rho_floor, g;
  float dt_nu;            // 0.125 h^2 / nu (or +inf)
  float kill_lo[3], kill_hi[3];
  float slab_margin2;     // slab instances: squared largest drift a step may make (0: not a slab)
  float cell[3];          // cell edge per axis
  float h16_band;         // half2 list pass: squared-distance band around (2h)^2 and 0 within which the
                          // 16-bit positions cannot decide the support test (exact FP32 test there)
  float HL2;              // neighbour lists: squared list radius (2h + skin)^2
  float inv_skin;         // neighbour lists: 1 / skin (0: lists off)
  double t_end;
};

// Dynamic per-instance record (lives on the device, advanced by kernels).
struct InstDyn {
  double time;
  long long steps;
  float dt_cur;          // dt of the step in flight
  unsigned dt_next_bits; // atomicMin target: bits of a positive float
  int finished;
  int phase;             // 0 idle, 1 step, 2 initial force pass, 3 probe
  int range_lo, range_hi;// [first, last+1) sorted slot of this instance after binning
  int n_alive;
  unsigned errors;       // kErrDrift: a slab particle drifted past the ghost-layer margin
  float vq;              // half2 list records: velocity quantum (a power of two; write_h16)
};

constexpr unsigned kErrDrift = 1u;

enum Phase { PH_IDLE = 0, PH_STEP = 1, PH_INIT = 2, PH_PROBE = 3 };

// Particle flags word: bits 0-15 instance slot, bit 16 FREEZE, bit 17 dead,
// bit 18 ghost (a copy of a particle another slab owns: a neighbour in the
// pair sums, kicked and drifted like its owner's copy, never reported, never
// in the dt minimum or the pair count).
constexpr uint32_t kInstMask = 0xffffu;
constexpr uint32_t kFreezeBit = 1u << 16;
constexpr uint32_t kDeadBit = 1u << 17;
constexpr uint32_t kGhostBit = 1u << 18;
constexpr uint32_t kDeadKey = 0xffffffffu;

// Neighbour cell q (may be out of range by one) on axis k: wrapped index and
// image shift s L; false when it lies outside a non-periodic grid.
__device__ __forceinline__ bool neighbor_cell(const InstParams& P, int k, int q, int& out, float& shift) {
  shift = 0.0f;
  if (q < 0) {
    if (!P.periodic) return false;
    out = q + P.ncell[k];
    shift = -P.L[k];
  } else if (q >= P.ncell[k]) {
    if (!P.periodic) return false;
    out = q - P.ncell[k];
    shift = P.L[k];
  } else {
    out = q;
  }
  return true;
}

// Sound speed of the Tait EoS for gamma = 7: sqrt(B gamma/rho0 x^6) = c0 |x^3|
// with x = 1 + (rho - rho0)/rho0, floored at sqrt(1e-16).  Every step is
// rounded explicitly, so that the packed form in the list pass (snds7_2)
// reproduces it bit for bit from rho alone.
__device__ __forceinline__ float snds7(const InstParams& P, float rho) {
  const float x = __fadd_rn(1.0f, __fmul_rn(__fsub_rn(rho, P.rho0), P.inv_rho0));
  const float x3 = __fmul_rn(__fmul_rn(x, x), x);
  return fmaxf(fabsf(__fmul_rn(P.c0, x3)), 1.0e-8f);
}

// Tait EoS (EoS.h:75-90): P = max(B ((rho/rho0)^gamma - 1), 0),
// c = sqrt(max(B gamma/rho0 (rho/rho0)^(gamma-1), 1e-16)).
// (rho/rho0)^gamma - 1 is evaluated on d = (rho - rho0)/rho0 without the
// cancellation of x^gamma - 1 near rho0 (weakly compressible: |d| ~ 1e-3):
// for gamma = 7 the binomial expansion d (7 + d (21 + d (35 + ...))) in Horner
// form (and c by snds7), otherwise expm1(gamma log1p(d)).
__device__ __forceinline__ void tait(const InstParams& P, float rho, float& pres, float& snds) {
  const float d = (rho - P.rho0) * P.inv_rho0;
  float xgm1;
  if (P.gamma == 7.0f) {
    xgm1 = d * (7.0f + d * (21.0f + d * (35.0f + d * (35.0f + d * (21.0f + d * (7.0f + d))))));
    snds = snds7(P, rho);
  } else {
    const float l = log1pf(d);
    xgm1 = expm1f(P.gamma * l);
    snds = sqrtf(fmaxf(P.cs2_coef * expf((P.gamma - 1.0f) * l), 1.0e-16f));
  }
  pres = fmaxf(P.B * xgm1, 0.0f);
}

}  // namespace wcsph

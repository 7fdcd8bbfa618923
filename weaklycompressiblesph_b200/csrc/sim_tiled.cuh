// Tiled hydro pass (WCSPH_PREC_TILED / WCSPH_PREC_HALF2).
#pragma once
#include "sim_kernels.cuh"

namespace wcsph {

inline int launch_hydro_tiled(const StepArgs&, int, int precision, cudaStream_t) {
  set_error("precision %d is not built in this library", precision);
  return WCSPH_E_INVALID;
}

}  // namespace wcsph

// Header-only FDPS shim: GPU_WC::HydrDispatchKernel / GPU_WC::HydrRetrieveKernel
// with the exact signatures of the reference (src/prototype.h:7-10), forwarding
// to the wcsph C ABI (include/wcsph.h).  Include it in the translation unit
// that defines the plugin types (STD::EPI::Hydro, STD::EPJ::Hydro,
// STD::RESULT::Hydro of src/class.h) after those definitions, link
// libwcsph.so, and hand the two functions to
//   hydr_tree.calcForceAllAndWriteBackMultiWalk(GPU_WC::HydrDispatchKernel,
//       GPU_WC::HydrRetrieveKernel, tag_max, sph_system, dinfo, N_WALK_LIMIT, ...)
// exactly as src/main.cpp:71,112,118 does.  tag_max may be up to
// WCSPH_FDPS_MAX_TAGS; FDPS then keeps that many batches in flight.
//
// The record layout is taken from the caller's own types with offsetof, so the
// shim follows whatever PS::F64vec / field order the build uses.  The pair
// variant defaults to the reference GPU kernel's (kernel.cu:241-280:
// alpha 0.01, beta 2*alpha, v_sig = max(-mu), symmetrised gradW); define
// WCSPH_FDPS_CPU_SEMANTICS before including this header to get the CPU
// functor's (force.h:31-60).
//
// Differences from src/kernel.cu by design: results are FP32-accumulated
// sums over FP32 records with walk-relative positions (the reference computes
// in half after scaling by L, v0, rho0); the device is chosen by wcsph_init
// (the reference reads it from stdin or the MPI rank); CUDA errors are
// reported through the return value and wcsph_last_error().
#pragma once
#include <cstddef>
#include <cstdio>

#include "wcsph.h"

namespace GPU_WC {

namespace detail {
inline int configure_once() {
  static int rc = -1;
  if (rc >= 0) return rc;
  wcsph_fdps_layout L;
  wcsph_fdps_default_layout(&L);
  L.epi_size = (int32_t)sizeof(STD::EPI::Hydro);
  L.epi_pos = (int32_t)offsetof(STD::EPI::Hydro, pos);
  L.epi_vel = (int32_t)offsetof(STD::EPI::Hydro, vel);
  L.epi_smth = (int32_t)offsetof(STD::EPI::Hydro, smth);
  L.epi_dens = (int32_t)offsetof(STD::EPI::Hydro, dens);
  L.epi_pres = (int32_t)offsetof(STD::EPI::Hydro, pres);
  L.epi_snds = (int32_t)offsetof(STD::EPI::Hydro, snds);
  L.epi_visc = (int32_t)offsetof(STD::EPI::Hydro, visc);
  L.epj_size = (int32_t)sizeof(STD::EPJ::Hydro);
  L.epj_pos = (int32_t)offsetof(STD::EPJ::Hydro, pos);
  L.epj_vel = (int32_t)offsetof(STD::EPJ::Hydro, vel);
  L.epj_dens = (int32_t)offsetof(STD::EPJ::Hydro, dens);
  L.epj_mass = (int32_t)offsetof(STD::EPJ::Hydro, mass);
  L.epj_smth = (int32_t)offsetof(STD::EPJ::Hydro, smth);
  L.epj_pres = (int32_t)offsetof(STD::EPJ::Hydro, pres);
  L.epj_snds = (int32_t)offsetof(STD::EPJ::Hydro, snds);
  L.epj_visc = (int32_t)offsetof(STD::EPJ::Hydro, visc);
  L.res_size = (int32_t)sizeof(STD::RESULT::Hydro);
  L.res_acc = (int32_t)offsetof(STD::RESULT::Hydro, acc);
  L.res_dt = (int32_t)offsetof(STD::RESULT::Hydro, dt);
  L.res_div_v = (int32_t)offsetof(STD::RESULT::Hydro, div_v);
  wcsph_pair_params P;
#ifdef WCSPH_FDPS_CPU_SEMANTICS
  wcsph_pair_params_reference_cpu(&P);
#else
  wcsph_pair_params_reference_gpu(&P);
#endif
  rc = wcsph_fdps_configure(&L, &P);
  return rc;
}
inline PS::S32 report(const char* fn, int rc) {
  if (rc != WCSPH_OK) std::fprintf(stderr, "%s: %s\n", fn, wcsph_last_error());
  return rc;
}
}  // namespace detail

inline PS::S32 HydrDispatchKernel(const PS::S32 tag, const PS::S32 n_walk, const STD::EPI::Hydro** epi,
                                  const PS::S32* n_epi, const STD::EPJ::Hydro** epj, const PS::S32* n_epj) {
  if (int rc = detail::configure_once()) return detail::report("GPU_WC::HydrDispatchKernel", rc);
  return detail::report("GPU_WC::HydrDispatchKernel",
                        wcsph_hydro_dispatch(tag, n_walk, reinterpret_cast<const void* const*>(epi), n_epi,
                                             reinterpret_cast<const void* const*>(epj), n_epj));
}

inline PS::S32 HydrRetrieveKernel(const PS::S32 tag, const PS::S32 n_walk, const PS::S32* ni,
                                  STD::RESULT::Hydro** force) {
  return detail::report("GPU_WC::HydrRetrieveKernel",
                        wcsph_hydro_retrieve(tag, n_walk, ni, reinterpret_cast<void* const*>(force)));
}

}  // namespace GPU_WC

// Reference CPU functors exposed through a C ABI.
//
// TEST INFRASTRUCTURE ONLY (the oracle).  This file contains no physics of its
// own: it includes the reference's headers unmodified, from the reference
// source tree given on the compiler command line (-I<reference>/src), and
// forwards plain arrays to the reference's own code:
//   STD::CalcHydroForce<kernel_t>   force.h:31-60   (hydro pair sum per walk)
//   STD::ApplyFilter<kernel_t>      force.h:10-30   (Shepard density filter)
//   STD::CalcPressure               force.h:3-9 -> EoS.h:75-90 (Tait EoS)
//   getTimeStepGlobal               integral.h:2-12 (CFL dt reduction)
//   RealPtcl::initialKick/fullDrift/predict/finalKick  class.h:146-163 (KDK)
//   CubicSpline<3>::W / gradW       kernel.h:27-55
// The FDPS names those headers need come from oracle/ps_standin.
// Built by oracle/Makefile into oracle/_ref/libwcsph_ref.so with the
// reference's own CPU flags (src/Makefile:3-4) minus the 2-D define.
#include <particle_simulator.hpp>
#include <cstddef>
#include <omp.h>
#include "param.h"
#include "kernel.h"
#include "EoS.h"
#include "class.h"
#include "force.h"
#include "integral.h"

using namespace STD;

extern "C" {

// Sizes and field offsets of the FDPS plugin types (class.h:61-263), so the
// tests can prove that the numpy / C-ABI layouts are byte-identical.
int ref_layout(long* out, int cap) {
  long v[] = {
      (long)sizeof(EPI::Hydro), (long)offsetof(EPI::Hydro, pos), (long)offsetof(EPI::Hydro, vel),
      (long)offsetof(EPI::Hydro, smth), (long)offsetof(EPI::Hydro, dens), (long)offsetof(EPI::Hydro, pres),
      (long)offsetof(EPI::Hydro, snds), (long)offsetof(EPI::Hydro, visc), (long)offsetof(EPI::Hydro, tag),
      (long)sizeof(EPJ::Hydro), (long)offsetof(EPJ::Hydro, pos), (long)offsetof(EPJ::Hydro, vel),
      (long)offsetof(EPJ::Hydro, dens), (long)offsetof(EPJ::Hydro, mass), (long)offsetof(EPJ::Hydro, smth),
      (long)offsetof(EPJ::Hydro, pres), (long)offsetof(EPJ::Hydro, snds), (long)offsetof(EPJ::Hydro, visc),
      (long)offsetof(EPJ::Hydro, tag), (long)offsetof(EPJ::Hydro, type),
      (long)sizeof(RESULT::Hydro), (long)offsetof(RESULT::Hydro, acc), (long)offsetof(RESULT::Hydro, dt),
      (long)offsetof(RESULT::Hydro, div_v),
      (long)sizeof(EPI::Filter), (long)offsetof(EPI::Filter, pos), (long)offsetof(EPI::Filter, smth),
      (long)sizeof(EPJ::Filter), (long)offsetof(EPJ::Filter, pos), (long)offsetof(EPJ::Filter, dens),
      (long)offsetof(EPJ::Filter, mass),
      (long)sizeof(RESULT::Filter), (long)offsetof(RESULT::Filter, dens)};
  int n = (int)(sizeof(v) / sizeof(v[0]));
  for (int k = 0; k < n && k < cap; ++k) out[k] = v[k];
  return n;
}

// One FDPS walk: clear the results (class.h:68-72) then run the functor,
// exactly as FDPS's calcForceAllAndWriteBack does per interaction group.
void ref_hydro_walk(const EPI::Hydro* epi, int ni, const EPJ::Hydro* epj, int nj, RESULT::Hydro* out) {
  for (int i = 0; i < ni; ++i) out[i].clear();
  CalcHydroForce<kernel_t>()(epi, ni, epj, nj, out);
}

// Many walks, threaded over walks the way FDPS threads interaction groups.
// ni_displ / nj_displ are exclusive prefix sums (length n_walk + 1).
void ref_hydro_walks(int n_walk, const int* ni_displ, const EPI::Hydro* epi, const int* nj_displ,
                     const EPJ::Hydro* epj, RESULT::Hydro* out, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
  for (int w = 0; w < n_walk; ++w) {
    const int i0 = ni_displ[w], j0 = nj_displ[w];
    ref_hydro_walk(epi + i0, ni_displ[w + 1] - i0, epj + j0, nj_displ[w + 1] - j0, out + i0);
  }
}

void ref_filter_walks(int n_walk, const int* ni_displ, const EPI::Filter* epi, const int* nj_displ,
                      const EPJ::Filter* epj, RESULT::Filter* out, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
  for (int w = 0; w < n_walk; ++w) {
    const int i0 = ni_displ[w], j0 = nj_displ[w];
    const int ni = ni_displ[w + 1] - i0;
    for (int i = 0; i < ni; ++i) out[i0 + i].clear();
    ApplyFilter<kernel_t>()(epi + i0, ni, epj + j0, nj_displ[w + 1] - j0, out + i0);
  }
}

// Tait EoS through the reference's CalcPressure loop (force.h:3-9).
void ref_pressure(int n, const double* dens, double* pres, double* snds, double gmm, double rho0, double c0) {
  EoS::Murnaghan<PS::F64> eos(gmm, rho0, c0);
  PS::ParticleSystem<RealPtcl> sys;
  sys.setNumberOfParticleLocal(n);
  for (int i = 0; i < n; ++i) {
    sys[i].dens = dens[i];
    sys[i].EoS = &eos;
  }
  CalcPressure(sys);
  for (int i = 0; i < n; ++i) {
    pres[i] = sys[i].pres;
    snds[i] = sys[i].snds;
  }
}

static void load(RealPtcl& p, int i, const double* pos, const double* vel, const double* vel_half,
                 const double* acc, const double* dens, const double* smth, const double* div_v,
                 const double* dt, const int* type) {
  p.pos = PS::F64vec(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
  p.vel = PS::F64vec(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
  if (vel_half) p.vel_half = PS::F64vec(vel_half[3 * i], vel_half[3 * i + 1], vel_half[3 * i + 2]);
  p.acc = PS::F64vec(acc[3 * i], acc[3 * i + 1], acc[3 * i + 2]);
  p.dens = dens[i];
  p.smth = smth ? smth[i] : 0.0;
  p.div_v = div_v ? div_v[i] : 0.0;
  p.dt = dt ? dt[i] : 0.0;
  p.type = type[i] ? FREEZE : HYDRO;
}

// Global timestep (integral.h:2-12) with a Newtonian kinematic viscosity nu
// shared by all particles (EoS.h:29-37).
double ref_timestep(int n, const double* smth, const double* acc, const double* dt, const int* type, double nu) {
  Viscosity::Newtonian<PS::F64> visc(nu);
  PS::ParticleSystem<RealPtcl> sys;
  sys.setNumberOfParticleLocal(n);
  for (int i = 0; i < n; ++i) {
    sys[i].smth = smth[i];
    sys[i].acc = PS::F64vec(acc[3 * i], acc[3 * i + 1], acc[3 * i + 2]);
    sys[i].dt = dt[i];
    sys[i].type = type[i] ? FREEZE : HYDRO;
    sys[i].visc = &visc;
  }
  return getTimeStepGlobal<RealPtcl>(sys);
}

// First half of the KDK step as main.cpp:98-103 runs it: initialKick,
// fullDrift, predict.  Arrays are updated in place; vel_half is written.
void ref_kdk_first(int n, double* pos, double* vel, double* vel_half, const double* acc, double* dens,
                   const double* div_v, const int* type, double dt) {
  for (int i = 0; i < n; ++i) {
    RealPtcl p;
    load(p, i, pos, vel, nullptr, acc, dens, nullptr, div_v, nullptr, type);
    p.initialKick(dt);
    p.fullDrift(dt);
    p.predict(dt);
    for (int k = 0; k < 3; ++k) {
      pos[3 * i + k] = (&p.pos.x)[k];
      vel[3 * i + k] = (&p.vel.x)[k];
      if (!type[i]) vel_half[3 * i + k] = (&p.vel_half.x)[k];
    }
    dens[i] = p.dens;
  }
}

// finalKick (class.h:160-163) as main.cpp:124-127 runs it.
void ref_kdk_final(int n, double* vel, const double* vel_half, const double* acc, const int* type, double dt) {
  for (int i = 0; i < n; ++i) {
    RealPtcl p;
    p.vel = PS::F64vec(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    p.vel_half = PS::F64vec(vel_half[3 * i], vel_half[3 * i + 1], vel_half[3 * i + 2]);
    p.acc = PS::F64vec(acc[3 * i], acc[3 * i + 1], acc[3 * i + 2]);
    p.type = type[i] ? FREEZE : HYDRO;
    p.finalKick(dt);
    for (int k = 0; k < 3; ++k) vel[3 * i + k] = (&p.vel.x)[k];
  }
}

double ref_W(double dx, double dy, double dz, double h) { return kernel_t::W(PS::F64vec(dx, dy, dz), h); }

void ref_gradW(double dx, double dy, double dz, double h, double* out) {
  PS::F64vec g = kernel_t::gradW(PS::F64vec(dx, dy, dz), h);
  out[0] = g.x;
  out[1] = g.y;
  out[2] = g.z;
}

// Reference parameters the functors bake in (param.h:4-5, force.h:32).
void ref_params(double* out) {
  out[0] = PARAM::SMTH;
  out[1] = PARAM::C_CFL;
  out[2] = 0.01;  // CalcHydroForce::AV_STRENGTH, force.h:32
  out[3] = (double)PARAM::Ngroup;
  out[4] = (double)PARAM::FILTER_APPLYING_INTERVAL;
}

}  // extern "C"

// Drop-in check of include/wcsph_fdps.hpp against the reference's own types
// and functor.  TEST INFRASTRUCTURE ONLY (built by oracle/Makefile into
// oracle/_ref/ where the reference sources exist, run by tests/test_fdps_shim.py).
//
// It compiles the reference's unmodified src/class.h plugin types and
// src/force.h CalcHydroForce, builds FDPS-style walks over a jittered lattice,
// and runs the same walks through
//   (a) GPU_WC::HydrDispatchKernel / GPU_WC::HydrRetrieveKernel (the shim,
//       CPU-functor pair semantics), and
//   (b) STD::CalcHydroForce<kernel_t> (the reference functor, FP64),
// then prints the relative L2 errors and exits non-zero above 1e-5.
#include <particle_simulator.hpp>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "param.h"
#include "kernel.h"
#include "EoS.h"
#include "class.h"
#include "force.h"

#define WCSPH_FDPS_CPU_SEMANTICS
#include "wcsph_fdps.hpp"

int main(int argc, char** argv) {
  const int side = argc > 1 ? std::atoi(argv[1]) : 12;
  const double dx = 0.01, h = 1.3 * dx, rho0 = 1000.0, c0 = 20.0;
  EoS::Murnaghan<PS::F64> eos(7.0, rho0, c0);
  std::mt19937_64 rng(7);
  std::uniform_real_distribution<double> U(-1.0, 1.0);
  std::vector<STD::RealPtcl> p;
  for (int i = 0; i < side; ++i)
    for (int j = 0; j < side; ++j)
      for (int k = 0; k < side; ++k) {
        STD::RealPtcl r;
        r.pos = PS::F64vec((i + 0.5 + 0.1 * U(rng)) * dx, (j + 0.5 + 0.1 * U(rng)) * dx, (k + 0.5 + 0.1 * U(rng)) * dx);
        r.vel = PS::F64vec(0.2 * U(rng), 0.2 * U(rng), 0.2 * U(rng));
        r.dens = rho0 * (1.0 + 0.01 * U(rng));
        r.mass = rho0 * dx * dx * dx;
        r.smth = h;
        r.pres = eos.Pressure(r.dens, 0.0);
        r.snds = eos.SoundSpeed(r.dens, 0.0);
        r.visc = &Viscosity::Water;
        p.push_back(r);
      }
  const int n = (int)p.size();
  // Walks: consecutive groups of <= 64 i; j-list = every particle within the
  // group's box grown by 2h (a superset, as FDPS hands out).
  std::vector<std::vector<STD::EPI::Hydro>> epi;
  std::vector<std::vector<STD::EPJ::Hydro>> epj;
  for (int g0 = 0; g0 < n; g0 += 64) {
    const int g1 = std::min(n, g0 + 64);
    PS::F64vec lo(1e30), hi(-1e30);
    std::vector<STD::EPI::Hydro> wi;
    for (int i = g0; i < g1; ++i) {
      STD::EPI::Hydro e;
      e.copyFromFP(p[i]);
      wi.push_back(e);
      lo = PS::F64vec(std::min(lo.x, p[i].pos.x), std::min(lo.y, p[i].pos.y), std::min(lo.z, p[i].pos.z));
      hi = PS::F64vec(std::max(hi.x, p[i].pos.x), std::max(hi.y, p[i].pos.y), std::max(hi.z, p[i].pos.z));
    }
    std::vector<STD::EPJ::Hydro> wj;
    for (int j = 0; j < n; ++j) {
      const PS::F64vec& q = p[j].pos;
      if (q.x >= lo.x - 2 * h && q.x <= hi.x + 2 * h && q.y >= lo.y - 2 * h && q.y <= hi.y + 2 * h &&
          q.z >= lo.z - 2 * h && q.z <= hi.z + 2 * h) {
        STD::EPJ::Hydro e;
        e.copyFromFP(p[j]);
        wj.push_back(e);
      }
    }
    epi.push_back(wi);
    epj.push_back(wj);
  }
  const int nw = (int)epi.size();
  std::vector<const STD::EPI::Hydro*> pi(nw);
  std::vector<const STD::EPJ::Hydro*> pj(nw);
  std::vector<PS::S32> ni(nw), nj(nw);
  std::vector<std::vector<STD::RESULT::Hydro>> gpu(nw), ref(nw);
  std::vector<STD::RESULT::Hydro*> pf(nw);
  for (int w = 0; w < nw; ++w) {
    pi[w] = epi[w].data();
    pj[w] = epj[w].data();
    ni[w] = (PS::S32)epi[w].size();
    nj[w] = (PS::S32)epj[w].size();
    gpu[w].resize(ni[w]);
    ref[w].resize(ni[w]);
    pf[w] = gpu[w].data();
    for (auto& r : ref[w]) r.clear();
    STD::CalcHydroForce<kernel_t>()(epi[w].data(), ni[w], epj[w].data(), nj[w], ref[w].data());
  }
  if (GPU_WC::HydrDispatchKernel(0, nw, pi.data(), ni.data(), pj.data(), nj.data()) != 0) return 2;
  if (GPU_WC::HydrRetrieveKernel(0, nw, ni.data(), pf.data()) != 0) return 3;
  double ea = 0, na = 0, ed = 0, nd = 0, edt = 0;
  for (int w = 0; w < nw; ++w)
    for (int i = 0; i < ni[w]; ++i) {
      const auto &a = gpu[w][i], &b = ref[w][i];
      const PS::F64vec d = a.acc - b.acc;
      ea += d * d;
      na += b.acc * b.acc;
      ed += (a.div_v - b.div_v) * (a.div_v - b.div_v);
      nd += b.div_v * b.div_v;
      edt = std::max(edt, std::fabs(a.dt / b.dt - 1.0));
    }
  const double ra = std::sqrt(ea / na), rd = std::sqrt(ed / nd);
  std::printf("walks %d particles %d acc_rel_l2 %.3e divv_rel_l2 %.3e dt_max_rel %.3e\n", nw, n, ra, rd, edt);
  return (ra < 1e-5 && rd < 1e-5 && edt < 1e-5) ? 0 : 1;
}

"""Generate tests/golden/*.npz from the reference's own CPU functors.

Run in a container where the reference source tree exists (oracle/_ref is
built from it):  python tests/golden/make_golden.py

hydro_walks_small.npz: a seeded 810-particle dam break (dx = 0.1, three wall
layers, random velocities), FDPS-style walks of <= 32 i-particles, and the
outputs of STD::CalcHydroForce (src/force.h:31-60) and STD::ApplyFilter
(src/force.h:10-30) over those walks, in FP64.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from tests.helpers import eos_np  # noqa: E402
from weaklycompressiblesph_b200 import cases, fdps  # noqa: E402


def small_case():
    c = cases.dam_break(dx=0.1, column=(0.3, 0.3, 0.4), tank=(0.6, 0.3, 0.5))
    rng = np.random.default_rng(11)
    c.vel = rng.normal(0.0, 0.5, size=c.vel.shape)
    c.vel[c.type == 1] = 0.0
    c.dens = c.dens * (1.0 + rng.uniform(-0.005, 0.005, size=c.n))
    return c


def records(c, w):
    pres, snds = eos_np(c.dens, c.phys)
    epi, epj = fdps.walk_records(w, c.pos, c.vel, c.dens, pres, snds, c.h, c.mass, c.phys.nu, type_=c.type)
    epi_f = np.zeros(len(epi), fdps.EPI_FILTER)
    epi_f["pos"], epi_f["smth"] = epi["pos"], epi["smth"]
    epj_f = np.zeros(len(epj), fdps.EPJ_FILTER)
    epj_f["pos"], epj_f["dens"], epj_f["mass"] = epj["pos"], epj["dens"], epj["mass"]
    return epi, epj, epi_f, epj_f


def main():
    oracle.build()
    assert oracle.ref_available(), "the reference build (oracle/_ref) is required"
    c = small_case()
    w = fdps.build_walks(c.pos, 2.0 * c.h, group_size=32)
    epi, epj, epi_f, epj_f = records(c, w)
    out = oracle.ref_hydro_walks(w.i_off, epi, w.j_off, epj)
    fd = oracle.ref_filter_walks(w.i_off, epi_f, w.j_off, epj_f)
    np.savez_compressed(os.path.join(HERE, "hydro_walks_small.npz"),
                        pos=c.pos, vel=c.vel, dens=c.dens, type=c.type, h=c.h, mass=c.mass,
                        i_idx=w.i_idx, i_off=w.i_off, j_idx=w.j_idx, j_off=w.j_off,
                        acc=out["acc"], div_v=out["div_v"], dt=out["dt"], filter_dens=fd)
    print("wrote", os.path.join(HERE, "hydro_walks_small.npz"), c.n, "particles", w.n_walk, "walks")


if __name__ == "__main__":
    main()

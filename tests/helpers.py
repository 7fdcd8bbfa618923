"""Shared builders for the parity tests (seeded, small)."""
import numpy as np

from weaklycompressiblesph_b200 import cases
from weaklycompressiblesph_b200 import fdps
from weaklycompressiblesph_b200 import _native as N


def small_dam(dx=0.05, seed=0, vel_sigma=0.3, **kw):
    """A coarse dam break with random velocities (exercises the AV branch)."""
    c = cases.dam_break(dx=dx, **kw)
    rng = np.random.default_rng(seed)
    c.vel = rng.normal(0.0, vel_sigma, size=c.vel.shape)
    c.vel[c.type == N.FREEZE] = 0.0
    c.dens = c.dens * (1.0 + rng.uniform(-0.003, 0.003, size=c.n))
    return c


def eos_np(dens, phys):
    B = phys.B
    x = dens / phys.rho0
    pres = np.maximum(B * (x ** phys.gamma - 1.0), 0.0)
    snds = np.sqrt(np.maximum(B * phys.gamma / phys.rho0 * x ** (phys.gamma - 1.0), 1e-16))
    return pres, snds


def walk_setup(case, group_size=128, r_factor=2.0):
    """Walks + FP64 EPI/EPJ records of a case (uniform h, mass, nu)."""
    pres, snds = eos_np(case.dens, case.phys)
    box = np.array(case.hi) - np.array(case.lo) if case.periodic else None
    w = fdps.build_walks(case.pos, r_factor * case.h, group_size=group_size, box=box)
    epi, epj = fdps.walk_records(w, case.pos, case.vel, case.dens, pres, snds, case.h, case.mass, case.phys.nu,
                                 type_=case.type, box=box)
    return w, epi, epj


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))

"""Seeded synthetic problem setups.

* ``dam_break``        the 3-D dam break: a water column at rest with
                       hydrostatic density in an open-top tank with three
                       layers of fixed (FREEZE) wall particles.  The
                       reference's own setup is src/init/Dam2.h:9-103 (a
                       different geometry); the wall semantics, gravity and
                       density floor follow it (Dam2.h:60-63,104-111).
* ``periodic_lattice`` the force-kernel microbenchmark: a jittered cubic
                       lattice in a periodic cube.
* ``ensemble_cases``   uneven dam breaks for the batched ensemble.
* ``serving_requests`` Poisson arrivals of dam-break requests.

Physics defaults follow the dam-break configuration the benchmarks are quoted
on: rho0 = 1000, Tait gamma = 7, c0 = 10 sqrt(g * 0.8), g = 9.81,
h = 1.3 dx, alpha = 0.1, beta = 0, CFL 0.25, nu = 1e-6.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as N


@dataclass
class Physics:
    rho0: float = 1000.0
    gamma: float = 7.0
    c0: float = 10.0 * math.sqrt(9.81 * 0.8)
    g: float = 9.81
    h_over_dx: float = 1.3
    alpha: float = 0.1
    beta: float = 0.0
    c_cfl: float = 0.25
    eps: float = 0.01
    nu: float = 1.0e-6
    vsig_mode: int = N.VSIG_SIGNAL
    rho_floor: float = 100.0          # Dam2.h:111
    density_mode: int = N.DENSITY_SHEPARD
    shepard_interval: int = 30        # param.h:12

    @property
    def B(self):
        return self.c0 * self.c0 * self.rho0 / self.gamma


@dataclass
class Case:
    """Particle arrays (FP64 on the host) plus the instance description."""
    name: str
    pos: np.ndarray            # (n, 3) float64
    vel: np.ndarray            # (n, 3) float64
    dens: np.ndarray           # (n,)   float64
    type: np.ndarray           # (n,)   int32, 0 HYDRO / 1 FREEZE
    dx: float
    h: float
    mass: float
    phys: Physics
    lo: tuple
    hi: tuple
    periodic: bool = False
    kill_lo: tuple = (0.0, 0.0, 0.0)
    kill_hi: tuple = (0.0, 0.0, 0.0)
    t_end: float = 0.0
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return len(self.dens)

    @property
    def n_fluid(self):
        return int(np.sum(self.type == N.HYDRO))

    def eos(self):
        """FP64 Tait pressure and sound speed of the current densities, the
        host-side CalcPressure an FDPS caller runs before the force pass
        (src/force.h:3-9, src/EoS.h:80-86)."""
        p = self.phys
        x = self.dens / p.rho0
        pres = np.maximum(p.B * (x ** p.gamma - 1.0), 0.0)
        snds = np.sqrt(np.maximum(p.B * p.gamma / p.rho0 * x ** (p.gamma - 1.0), 1e-16))
        return pres, snds

    def desc(self, density_mode=None, t_end=None) -> N.InstanceDesc:
        p = self.phys
        d = N.InstanceDesc()
        d.n = self.n
        d.density_mode = p.density_mode if density_mode is None else density_mode
        d.shepard_interval = p.shepard_interval
        d.periodic = 1 if self.periodic else 0
        d.h, d.mass, d.nu = self.h, self.mass, p.nu
        d.rho0, d.gamma, d.c0 = p.rho0, p.gamma, p.c0
        d.g, d.rho_floor = p.g, p.rho_floor
        d.pair = N.PairParams(p.alpha, p.beta, p.c_cfl, p.eps, p.vsig_mode, N.GRAD_HBAR)
        for k in range(3):
            d.lo[k], d.hi[k] = self.lo[k], self.hi[k]
            d.kill_lo[k], d.kill_hi[k] = self.kill_lo[k], self.kill_hi[k]
        d.t_end = self.t_end if t_end is None else t_end
        return d


def _hydrostatic(z, height, phys):
    """rho(z) with P = rho0 g (H - z) = B ((rho/rho0)^gamma - 1)."""
    depth = np.maximum(height - z, 0.0)
    return phys.rho0 * (1.0 + phys.rho0 * phys.g * depth / phys.B) ** (1.0 / phys.gamma)


def dam_break(dx=0.02, column=(0.4, 0.4, 0.8), tank=(1.6, 0.4, 1.0), layers=3, phys=None,
              headroom=0.5, name=None) -> Case:
    """Water column [0,cx]x[0,cy]x[0,cz] in the open-top tank [0,tx]x[0,ty]x[0,tz].

    Particles sit at cell centres (i + 1/2) dx.  Wall particles fill `layers`
    lattice layers outside the tank's bottom and four sides (up to the tank
    top).  Counts at dx = 0.02: 16,000 fluid + 38,508 wall; at dx = 0.005:
    1,024,000 fluid + 571,308 wall.
    """
    phys = phys or Physics()
    cx, cy, cz = (int(round(c / dx)) for c in column)
    tx, ty, tz = (int(round(t / dx)) for t in tank)
    # fluid
    ii, jj, kk = np.meshgrid(np.arange(cx), np.arange(cy), np.arange(cz), indexing="ij")
    fluid = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1)
    # walls: lattice box [-L, t+L) x [-L, t+L) x [-L, tz) minus the interior
    L = layers
    wi, wj, wk = np.meshgrid(np.arange(-L, tx + L), np.arange(-L, ty + L), np.arange(-L, tz), indexing="ij")
    w = np.stack([wi.ravel(), wj.ravel(), wk.ravel()], axis=1)
    interior = (w[:, 0] >= 0) & (w[:, 0] < tx) & (w[:, 1] >= 0) & (w[:, 1] < ty) & (w[:, 2] >= 0)
    wall = w[~interior]
    idx = np.concatenate([fluid, wall], axis=0)
    pos = (idx.astype(np.float64) + 0.5) * dx
    n_f = len(fluid)
    typ = np.zeros(len(idx), np.int32)
    typ[n_f:] = N.FREEZE
    dens = _hydrostatic(pos[:, 2], column[2], phys)
    vel = np.zeros_like(pos)
    h = phys.h_over_dx * dx
    mass = phys.rho0 * dx ** 3
    pad = 2.0 * h
    lo = (-L * dx - pad, -L * dx - pad, -L * dx - pad)
    hi = (tank[0] + L * dx + pad, tank[1] + L * dx + pad, tank[2] + headroom)
    kill_lo = (lo[0], lo[1], lo[2])
    kill_hi = (hi[0], hi[1], tank[2] + 4.0 * headroom)
    return Case(name or f"dam_break_dx{dx:g}", pos, vel, dens, typ, dx, h, mass, phys, lo, hi,
                periodic=False, kill_lo=kill_lo, kill_hi=kill_hi,
                meta=dict(column=column, tank=tank, layers=layers, n_fluid=n_f, n_wall=len(wall)))


def periodic_lattice(n_side=200, dx=0.01, seed=12345, jitter=0.1, phys=None, name=None) -> Case:
    """Jittered cubic lattice in the periodic cube [0, n_side*dx)^3.

    Jitter U(+-jitter*dx) per coordinate, rho = rho0 (1 + U(-0.01, 0.01)),
    v ~ N(0, 0.05 c0) per component, h = 1.3 dx, no gravity.  Seeded PCG64.
    """
    phys = phys or Physics(g=0.0, density_mode=N.DENSITY_SUMMATION)
    rng = np.random.default_rng(seed)
    side = n_side * dx
    ii, jj, kk = np.meshgrid(np.arange(n_side), np.arange(n_side), np.arange(n_side), indexing="ij")
    pos = (np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1).astype(np.float64) + 0.5) * dx
    pos += rng.uniform(-jitter * dx, jitter * dx, size=pos.shape)
    pos = np.mod(pos, side)
    n = len(pos)
    dens = phys.rho0 * (1.0 + rng.uniform(-0.01, 0.01, size=n))
    vel = rng.normal(0.0, 0.05 * phys.c0, size=(n, 3))
    typ = np.zeros(n, np.int32)
    h = phys.h_over_dx * dx
    mass = phys.rho0 * dx ** 3
    return Case(name or f"periodic_{n_side}^3", pos, vel, dens, typ, dx, h, mass, phys,
                (0.0, 0.0, 0.0), (side, side, side), periodic=True, meta=dict(n_side=n_side, seed=seed))


def ensemble_cases(count=64, seed=2024, n_min=1.0e4, n_max=5.0e5, phys=None):
    """Uneven dam breaks: column width W ~ U(0.2, 0.6) (square base), aspect
    ratio A ~ U(1, 3) (height A*W), fluid count log-uniform in [n_min, n_max];
    dx solves W*W*A*W / dx^3 = count; tank 4W x W x 1.25 A W."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        W = rng.uniform(0.2, 0.6)
        A = rng.uniform(1.0, 3.0)
        target = math.exp(rng.uniform(math.log(n_min), math.log(n_max)))
        dx = W * (A / target) ** (1.0 / 3.0)
        # snap so that the column holds an integer number of cells
        nw = max(2, int(round(W / dx)))
        dx = W / nw
        out.append(dam_break(dx=dx, column=(W, W, nw * dx * round(A * nw) / nw),
                             tank=(4 * W, W, 1.25 * A * W), phys=phys, name=f"ens{k:02d}"))
    return out


def serving_requests(count=32, rate=20.0, seed=7, n_min=2.0e4, n_max=2.0e6, t_end=1.0, phys=None):
    """Poisson(rate) arrival times and dam-break requests with fluid counts
    log-uniform in [n_min, n_max] and column aspect ratio U(1, 3)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=count))
    reqs = []
    for k in range(count):
        W = rng.uniform(0.2, 0.6)
        A = rng.uniform(1.0, 3.0)
        target = math.exp(rng.uniform(math.log(n_min), math.log(n_max)))
        dx = W * (A / target) ** (1.0 / 3.0)
        nw = max(2, int(round(W / dx)))
        dx = W / nw
        c = dam_break(dx=dx, column=(W, W, nw * dx * round(A * nw) / nw), tank=(4 * W, W, 1.25 * A * W),
                      phys=phys, name=f"req{k:03d}")
        c.t_end = t_end
        reqs.append((float(t[k]), c))
    return reqs

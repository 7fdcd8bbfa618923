"""Configs 1 and 3 checked against the FP64 oracle at their own size.

    python tests/validate_configs.py --config 1 [--steps 2000] [--every 250]
    python tests/validate_configs.py --config 3

Config 1: the 16k-fluid dam break (dx = 0.02: 16,000 fluid + 38,508 wall
particles), 2000 FP32 steps on the device with neighbour lists (the default
mode) and on the plain FP32 path.  At every checkpoint the device's own state
is read back and one force pass on it (through the list passes for the list
run) is compared with the FP64 oracle: relative L2 of the acceleration, div v
and drho/dt, neighbour counts exactly, plus the device's FP64 conservation
sums.

Config 3: the 8M-particle jittered periodic lattice (200^3, dx = 0.01,
h = 1.3 dx, seeded): one summation-density pass and one hydro pass of the
initial state, per precision (plain FP32, tiled FP32, half2), through a fresh
search and through the neighbour lists, against the FP64 oracle (density,
acceleration, div v, per-particle dt; neighbour counts exactly).

Prints one JSON line.  Not collected by pytest (long); run on a GPU box.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import oracle  # noqa: E402
from weaklycompressiblesph_b200 import _native as N  # noqa: E402
from weaklycompressiblesph_b200 import cases  # noqa: E402
from weaklycompressiblesph_b200.sim import Solver  # noqa: E402

PRECS = {"fp32": N.PREC_FP32, "tiled": N.PREC_TILED, "half2": N.PREC_HALF2}


def rel(a, b):
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def f32(a):
    return np.asarray(a, np.float32)


def oracle_forces(case, pos, vel, dens):
    cfg = oracle.config_from_case(case)
    p4 = oracle.pos4(f32(pos))
    v4 = oracle.pos4(f32(vel))
    d = f32(dens)
    pres, snds = oracle.eos(d.astype(np.float64), case.phys.gamma, case.phys.rho0, case.phys.c0)
    acc, dv, dt = oracle.hydro(p4, v4, d, f32(pres), f32(snds), cfg)
    cnt, tot = oracle.neighbors(p4, cfg)
    return acc, dv, dt, cnt, tot


def compare(case, pr, st, dens_used=None):
    d = f32(st["dens"] if dens_used is None else dens_used)
    acc, dv, dt, cnt, tot = oracle_forces(case, st["pos"], st["vel"], d)
    return {"acc": rel(pr["acc"], acc), "div_v": rel(pr["div_v"], dv),
            "drho_dt": rel(-pr["dens"] * pr["div_v"], -d.astype(np.float64) * dv), "dt": rel(pr["dt"], dt),
            "neighbors_exact": bool(np.array_equal(pr["nbr"], cnt)), "pairs": int(tot)}


def config1(args):
    case = cases.dam_break(dx=0.02)
    out = {"config": 1, "case": case.name, "particles": case.n, "steps": args.steps, "runs": {}}
    for name, prec, li in (("tiled_lists", N.PREC_TILED, 30), ("half2_lists", N.PREC_HALF2, 30),
                           ("plain_fp32", N.PREC_FP32, 0)):
        checks = []
        t0 = time.perf_counter()
        with Solver(case.n + 1024, precision=prec, list_interval=li) as s:
            k = s.add(case)
            done = 0
            while True:
                if done % args.every == 0 or done == args.steps:
                    st = s.read(k)
                    pr = s.probe(k, lists=li > 0)
                    c = compare(case, pr, st)
                    cons = s.conservation(k)
                    c.update(step=done, time=s.status(k)["time"], mass=cons[0],
                             momentum=float(np.linalg.norm(cons[1:4])), kinetic=cons[4])
                    checks.append(c)
                if done >= args.steps:
                    break
                n = min(args.every, args.steps - done)
                s.step(n)
                done += n
            lists = s.list_stats() if li else None
        out["runs"][name] = {"checks": checks, "wall_s": time.perf_counter() - t0, "lists": lists,
                             "max_acc": max(c["acc"] for c in checks), "max_div_v": max(c["div_v"] for c in checks),
                             "neighbors_exact": all(c["neighbors_exact"] for c in checks)}
    return out


def config3(args):
    case = cases.periodic_lattice(n_side=200, dx=0.01, seed=12345)
    out = {"config": 3, "case": case.name, "particles": case.n, "runs": {}}
    cfg = oracle.config_from_case(case)
    p4 = oracle.pos4(f32(case.pos))
    t0 = time.perf_counter()
    rho_ref = oracle.density(p4, f32(case.dens), cfg, False)
    out["oracle_density_s"] = time.perf_counter() - t0
    for name in ("fp32", "tiled", "half2"):
        for lists in ((False, True) if name != "fp32" else (False,)):
            key = name + ("_lists" if lists else "")
            with Solver(case.n + 1024, precision=PRECS[name], list_interval=10 if lists else 0) as s:
                k = s.add(case, density_mode=N.DENSITY_CONTINUITY)
                st = s.read(k)
                pr = s.probe(k, density_pass=1, lists=lists)
                if lists:  # the first probe built the lists (its density pass searched); this one reads them
                    pr = s.probe(k, density_pass=1, lists=True)
            r = {"density": rel(pr["dens"], rho_ref)}
            r.update(compare(case, pr, st, dens_used=pr["dens"]))
            out["runs"][key] = r
            print(key, r, file=sys.stderr, flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, choices=[1, 3], required=True)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--every", type=int, default=250)
    args = ap.parse_args()
    out = config1(args) if args.config == 1 else config3(args)
    print(json.dumps(out))


if __name__ == "__main__":
    main()

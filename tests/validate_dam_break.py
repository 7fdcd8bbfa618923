"""Config-2 validation: the dam break at dx = 0.005 (1,024,000 fluid + 571,308
wall particles) on the FP32 (tiled) and half2 paths, searching every step and
with neighbour lists.

    python tests/validate_dam_break.py [--steps 5000] [--every 500] [--dx 0.005]

At every checkpoint the GPU's own FP32 state is read back and one force pass
is checked against the FP64 oracle on that state: relative L2 of the
acceleration, drho/dt = -rho div v, and div v (runs with lists probe through
the list passes themselves).  The FP64 conservation sums of the device
(mass, momentum, kinetic energy, vertical pair-force total) are recorded at
every checkpoint.  The surge front (largest x of a fluid particle) is recorded
against physical time for every path and compared with the FP32 front.
Prints one JSON line.
Not collected by pytest (long); run on a GPU box.
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


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def check(case, s, k, lists=False):
    """GPU force pass vs FP64 oracle on the GPU's current state; with lists,
    the passes a list step runs (k_hydro_list over the current lists)."""
    st = s.read(k)
    pr = s.probe(k, lists=lists)
    cfg = oracle.config_from_case(case)
    p4 = oracle.pos4(st["pos"])
    v4 = oracle.pos4(st["vel"])
    d = st["dens"].astype(np.float64)
    pres, snds = oracle.eos(d, case.phys.gamma, case.phys.rho0, case.phys.c0)
    acc, dv, _ = oracle.hydro(p4, v4, st["dens"], pres.astype(np.float32), snds.astype(np.float32), cfg)
    cnt, _ = oracle.neighbors(p4, cfg)
    cons = s.conservation(k)
    alive = st["alive"] == 1
    az = st["acc"][alive, 2].astype(np.float64) + case.phys.g
    return {"acc": rel(pr["acc"], acc), "drho_dt": rel(-pr["dens"] * pr["div_v"], -d * dv), "div_v": rel(pr["div_v"], dv),
            "neighbors_exact": bool(np.array_equal(pr["nbr"], cnt)),
            # FP64 sums on the device: mass, |momentum|, kinetic energy, and the
            # vertical pair-force total relative to the sum of its magnitudes
            "mass": cons[0], "momentum": float(np.linalg.norm(cons[1:4])), "kinetic": cons[4],
            "pair_force_z_rel": float(abs(cons[5]) / max(case.mass * np.abs(az).sum(), 1e-300))}


def run(case, precision, steps, every, list_interval=0):
    front = []
    checks = []
    with Solver(case.n + 1024, precision=precision, list_interval=list_interval) as s:
        k = s.add(case)
        fluid = case.type == N.HYDRO
        t0 = time.perf_counter()
        done = 0
        while True:
            st = s.status(k)
            pos = s.read(k)["pos"]
            front.append((st["time"], float(pos[fluid, 0].max())))
            if done % every == 0 or done == steps:
                c = check(case, s, k, lists=list_interval > 0)
                c["step"] = done
                checks.append(c)
            if done >= steps:
                break
            n = min(100, steps - done)
            s.step(n)
            done += n
        wall = time.perf_counter() - t0
        lists = s.list_stats() if list_interval else None
    return {"front": front, "checks": checks, "wall_s": wall, "lists": lists}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--every", type=int, default=1000)
    ap.add_argument("--dx", type=float, default=0.005)
    ap.add_argument("--list-interval", type=int, default=30,
                    help="also run the tiled and half2 paths with neighbour lists rebuilt at least every K steps "
                         "(0: skip)")
    ap.add_argument("--paths", default="", help="comma-separated subset of the paths (fp32_tiled always runs)")
    ap.add_argument("--summary", default="", help="also write the largest error of every path as JSON here")
    args = ap.parse_args()
    case = cases.dam_break(dx=args.dx)
    out = {"case": case.name, "particles": case.n, "steps": args.steps}
    res = {}
    # (half2 without lists runs the FP32 tiled kernel: its compact records
    # belong to the list pass, so it is the fp32_tiled path)
    paths = [("fp32_tiled", N.PREC_TILED, 0)]
    if args.list_interval:
        paths.append(("tiled_lists", N.PREC_TILED, args.list_interval))
        paths.append(("half2_lists", N.PREC_HALF2, args.list_interval))
    if args.paths:
        keep = set(args.paths.split(","))
        paths = [p for p in paths if p[0] in keep or p[0] == "fp32_tiled"]
    for name, prec, k in paths:
        res[name] = run(case, prec, args.steps, args.every, list_interval=k)
        out[name] = {"checks": res[name]["checks"], "sim_time_end": res[name]["front"][-1][0],
                     "front_end": res[name]["front"][-1][1], "lists": res[name]["lists"]}
    f32 = np.array(res["fp32_tiled"]["front"])
    col = 0.4  # initial column length
    out["surge_front"] = {"fp32_samples": [(round(t, 5), round(x, 5)) for t, x in f32[:: max(1, len(f32) // 10)]]}
    for name in res:
        if name == "fp32_tiled":
            continue
        # compare fronts at common physical times (interpolate onto the FP32 run's times)
        other = np.array(res[name]["front"])
        oi = np.interp(f32[:, 0], other[:, 0], other[:, 1])
        out["surge_front"][name + "_vs_fp32"] = {
            "max_abs_diff_m": float(np.abs(oi - f32[:, 1]).max()),
            "max_rel_diff_vs_travel": float(np.abs(oi - f32[:, 1]).max() / max(f32[:, 1].max() - col, 1e-9))}
    print(json.dumps(out))
    if args.summary:
        summ = {"case": case.name, "particles": case.n, "steps": args.steps, "every": args.every, "paths": {}}
        for name in res:
            ch = out[name]["checks"]
            summ["paths"][name] = {"max_acc": max(c["acc"] for c in ch), "max_div_v": max(c["div_v"] for c in ch),
                                   "max_drho_dt": max(c["drho_dt"] for c in ch), "checkpoints": len(ch),
                                   "neighbors_exact": all(c["neighbors_exact"] for c in ch)}
        with open(args.summary, "w") as f:
            json.dump(summ, f, indent=1)


if __name__ == "__main__":
    main()

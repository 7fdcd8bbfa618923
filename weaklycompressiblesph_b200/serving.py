"""Continuous-batching request loop over one device-resident solver.

Requests are dam-break simulations (a `Case` with `t_end`) that arrive over
wall-clock time.  A request is admitted as soon as its particles fit the HBM
budget next to the simulations already on the device and an instance slot is
free; its particle state then stays resident on the GPU.  Every admitted
simulation advances in the same kernels (one CUDA graph per step, each
instance with its own CFL dt); a simulation whose physical time reached
`t_end` stops advancing, is read back, and is removed, which frees room for
queued requests.  Reported: per-request time-to-completion (arrival to result
on the host), its p50/p99, and aggregate particle-steps/s.

    python -m weaklycompressiblesph_b200.serving [--requests 32] [--t-end 1.0] [--budget-gb 150]
"""
from __future__ import annotations

import argparse
import collections
import json
import time

import numpy as np

from . import _native as N
from .cases import serving_requests
from .sim import Solver

BYTES_PER_PARTICLE_ESTIMATE = None


def particle_bytes(list_interval=0):
    """Device bytes per particle of a solver (from the library's own sizing)."""
    a = Solver.device_bytes(1 << 20, max_cells=1, max_instances=1, list_interval=list_interval)
    b = Solver.device_bytes(2 << 20, max_cells=1, max_instances=1, list_interval=list_interval)
    return (b - a) / float(1 << 20)


class Server:
    def __init__(self, budget_bytes=150e9, precision=N.PREC_TILED, max_instances=256, chunk_steps=25, device=0,
                 max_particles=None, read_results=True, list_interval=0):
        """list_interval > 0 steps the requests with neighbour lists (see
        Solver); results then depend on the mix, so a request's result is no
        longer bit-identical to running it alone."""
        per = particle_bytes(list_interval)
        cap = int(budget_bytes / (per + 8.0))  # + 2 cells per particle of table headroom
        if max_particles is not None:
            cap = min(cap, int(max_particles))
        self.capacity = cap
        self.solver = Solver(cap, precision=precision, max_cells=2 * cap, max_instances=max_instances,
                             device=device, list_interval=list_interval)
        self.chunk_steps = chunk_steps
        self.max_instances = max_instances
        self.read_results = read_results

    def close(self):
        self.solver.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self, requests, clock=time.perf_counter):
        """requests: list of (arrival_seconds, Case with t_end).  Returns a
        dict with per-request records and aggregate figures."""
        s = self.solver
        queue = collections.deque(sorted(enumerate(requests), key=lambda r: r[1][0]))
        pending = collections.deque()
        active = {}          # slot -> (req id, case, arrival wall time, admit wall time)
        in_use = 0
        done = {}
        particle_steps = 0
        t0 = clock()
        while queue or pending or active:
            now = clock() - t0
            while queue and queue[0][1][0] <= now:
                pending.append(queue.popleft())
            # admission: FIFO by arrival, as long as memory and slots allow
            while pending and len(active) < self.max_instances:
                rid, (arr, case) = pending[0]
                if case.n > self.capacity:
                    raise ValueError(f"request {rid} ({case.n} particles) exceeds the budget")
                if in_use + case.n > self.capacity:
                    break
                pending.popleft()
                slot = s.add(case, t_end=case.t_end)
                active[slot] = (rid, case, arr, clock() - t0)
                in_use += case.n
            if not active:
                if queue:
                    time.sleep(max(0.0, min(0.01, queue[0][1][0] - (clock() - t0))))
                continue
            s.step(self.chunk_steps)
            for slot in list(active):
                st = s.status(slot)
                rid, case, arr, adm = active[slot]
                if st["finished"]:
                    res = s.read(slot) if self.read_results else None
                    fin = clock() - t0
                    done[rid] = dict(request=rid, n=case.n, arrival=arr, admitted=adm, finished=fin,
                                     latency=fin - arr, steps=st["steps"], sim_time=st["time"], result=res)
                    particle_steps += case.n * st["steps"]
                    s.remove(slot)
                    del active[slot]
                    in_use -= case.n
        wall = clock() - t0
        lat = np.array([d["latency"] for d in done.values()])
        return dict(records=[done[k] for k in sorted(done)], wall_s=wall, particle_steps=particle_steps,
                    particle_steps_per_s=particle_steps / wall if wall > 0 else 0.0,
                    p50_s=float(np.percentile(lat, 50)), p99_s=float(np.percentile(lat, 99)),
                    lists=dict(s.list_stats(), **s.list_schedule()) if s.opt.list_interval else None)


def run_alone(case, precision=N.PREC_TILED, chunk_steps=25, device=0, list_interval=0):
    """One request by itself, stepped to t_end; returns (seconds, steps, result)."""
    with Solver(case.n + 1024, precision=precision, max_instances=2, device=device,
                list_interval=list_interval) as s:
        k = s.add(case, t_end=case.t_end)
        s.synchronize()
        t0 = time.perf_counter()
        while True:
            s.step(chunk_steps)
            st = s.status(k)
            if st["finished"]:
                break
        el = time.perf_counter() - t0
        return el, st["steps"], s.read(k)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=32)
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--n-min", type=float, default=2e4)
    ap.add_argument("--n-max", type=float, default=2e6)
    ap.add_argument("--t-end", type=float, default=1.0)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--serial", action="store_true", help="also time the requests one at a time on plain FP32")
    args = ap.parse_args(argv)
    reqs = serving_requests(count=args.requests, rate=args.rate, seed=args.seed, n_min=args.n_min,
                            n_max=args.n_max, t_end=args.t_end)
    total = sum(c.n for _, c in reqs)
    with Server(budget_bytes=args.budget_gb * 1e9, max_particles=max(total, 1) + 1024) as srv:
        out = srv.run(reqs)
    line = dict(requests=args.requests, particles=total, wall_s=out["wall_s"], p50_s=out["p50_s"],
                p99_s=out["p99_s"], particle_steps_per_s=out["particle_steps_per_s"])
    if args.serial:
        el = 0.0
        ps = 0
        for _, c in reqs:
            t, steps, _ = run_alone(c, precision=N.PREC_FP32)
            el += t
            ps += c.n * steps
        line["serial_plain_particle_steps_per_s"] = ps / el
    print(json.dumps(line))


if __name__ == "__main__":
    main()

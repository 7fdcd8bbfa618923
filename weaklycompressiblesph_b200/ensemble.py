"""Batched ensembles: many independent dam breaks stepping together in one
solver (one graph per step, every kernel launched once over all instances),
and the reference point they are compared with, the same instances run one at
a time on the plain FP32 single-instance path."""
from __future__ import annotations

import time

import numpy as np

from . import _native as N
from .sim import Solver

PRECISIONS = {"fp32": N.PREC_FP32, "tiled": N.PREC_TILED, "half2": N.PREC_HALF2}


def _sync_time(solver, fn):
    solver.synchronize()
    t0 = time.perf_counter()
    fn()
    solver.synchronize()
    return time.perf_counter() - t0


def run_batched(cases, steps, precision="tiled", warmup=3, device=0, list_interval=0, read=False):
    """Step all cases together; returns dict with wall seconds for `steps`
    steps, particle-steps/s and per-instance status (and, with read=True, each
    instance's final state).  list_interval > 0 uses neighbour lists (see
    Solver)."""
    total = sum(c.n for c in cases)
    with Solver(total + 1024, precision=PRECISIONS[precision], max_instances=len(cases) + 1, device=device,
                list_interval=list_interval) as s:
        slots = [s.add(c) for c in cases]
        s.step(warmup)
        el = _sync_time(s, lambda: s.step(steps))
        st = [s.status(k) for k in slots]
        states = [s.read(k) for k in slots] if read else None
        lists = dict(s.list_stats(), **s.list_schedule()) if list_interval else None
        tuning = s.tuning()
    return dict(seconds=el, steps=steps, particles=total, particle_steps_per_s=total * steps / el,
                status=st, states=states, lists=lists, tuning=tuning)


def run_serial(cases, steps, precision="fp32", warmup=3, device=0, list_interval=0, read=False):
    """The same instances one at a time (each in its own solver)."""
    el = 0.0
    total = 0
    states = [] if read else None
    for c in cases:
        with Solver(c.n + 1024, precision=PRECISIONS[precision], max_instances=2, device=device,
                    list_interval=list_interval) as s:
            k = s.add(c)
            s.step(warmup)
            el += _sync_time(s, lambda: s.step(steps))
            total += c.n
            if read:
                states.append(s.read(k))
    return dict(seconds=el, steps=steps, particles=total, particle_steps_per_s=total * steps / el, states=states)


def latency_percentiles(seconds):
    a = np.asarray(seconds, np.float64)
    return dict(p50=float(np.percentile(a, 50)), p99=float(np.percentile(a, 99)), mean=float(a.mean()),
                count=int(a.size))

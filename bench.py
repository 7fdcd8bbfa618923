"""Benchmark: pair interactions/s and steps/s of the WCSPH step on the 1M-fluid
dam break (dx = 0.005: 1,024,000 fluid + 571,308 wall particles), on one B200
per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload dam1m|dam16k|periodic8m] [--precision fp32|tiled|half2]

One JSON line on rank 0.  A "step" is one full device-resident timestep
(binning + Morton sort, density pass when due, EoS, hydro pass, gravity, KDK,
CFL dt) of the whole workload.  `value` counts the hydro pass's true
in-support pairs (0 < r^2 < (2h)^2) per second over the timed steps.
`e2e` is the same metric through the FDPS drop-in C ABI
(wcsph_hydro_dispatch / wcsph_hydro_retrieve) from host walk records, copies
included.  `--impl reference` times the reference's own CPU functor
(STD::CalcHydroForce, built by oracle/) on the same walks, on all host cores.
Multi-GPU: independent replicas by default (weak scaling); `--decomp slab`
cuts the one dam break into x-slabs, one per rank, with ghost-layer and
particle exchange over NCCL after every step (strong scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "pair interactions/s and steps/s (1M dam-break) vs plain FP32; p50/p99 ensemble latency"
UNIT = "pair interactions/s"
BYTES_PER_PAIR = {"fp32": 36, "tiled": 36, "half2": 18}  # hydro j-record per evaluated true pair


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="dam1m", choices=["dam1m", "dam16k", "periodic8m"])
    ap.add_argument("--precision", default="best", choices=["best", "fp32", "tiled", "half2"])
    ap.add_argument("--decomp", default="replicas", choices=["replicas", "slab"],
                    help="N>1: independent replicas (weak scaling) or one dam break cut into x-slabs (strong)")
    ap.add_argument("--list-interval", type=int, default=30,
                    help="neighbour lists rebuilt at least every K steps (0: search every step)")
    ap.add_argument("--list-skin", type=float, default=0.0, help="list skin in units of h (0: 0.3)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-only", action="store_true",
                    help="time only the FDPS drop-in pass (dispatch + retrieve from host records), --steps passes")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-FP32 comparison run")
    ap.add_argument("--no-other-precision", action="store_true",
                    help="skip the run of the other list-mode precision (half2 beside FP32, or the reverse)")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the ensemble and serving samples")
    ap.add_argument("--ensemble-steps", type=int, default=60)
    ap.add_argument("--ensemble-precision", default="half2", choices=["tiled", "half2"],
                    help="precision of the batched ensemble (config: half2 pairs; the FP32 list path is timed beside it)")
    ap.add_argument("--serving-precision", default="tiled", choices=["tiled", "half2"],
                    help="precision of the served requests (the config names none: the default FP32 list path)")
    ap.add_argument("--serving-requests", type=int, default=16)
    ap.add_argument("--serving-nmax", type=float, default=2e5, help="largest request (config: 2e6 particles)")
    ap.add_argument("--serving-tend", type=float, default=0.1, help="physical end time (config: 1.0 s)")
    ap.add_argument("--serving-no-serial", action="store_true",
                    help="time only the served mix (skip the one-at-a-time plain FP32 baseline)")
    ap.add_argument("--ncu-pass", action="store_true",
                    help="only run 12 eager steps in list mode (launch shape 0, no autotuner, no graph) and exit: "
                         "the 7th list-pass launch is a list step, for an ncu capture of one launch")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    return ap.parse_args()


def make_case(workload):
    from weaklycompressiblesph_b200 import cases
    if workload == "dam1m":
        return cases.dam_break(dx=0.005)
    if workload == "dam16k":
        return cases.dam_break(dx=0.02)
    return cases.periodic_lattice(n_side=200, dx=0.01, seed=12345)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML polled every 10 ms on a thread (reads only), the device matched
    by PCI bus id; nvidia-smi at its 200 ms floor when NVML is unavailable.
    Call mark_start() / mark_stop() around the timed work; only samples taken in
    between are summarised."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.samples = []  # (time, sm_mhz, max_mhz, reasons)
        self.t0 = self.t1 = None
        self.stop = threading.Event()
        self.thread = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(self.device)
        try:
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def _poll_nvml(self, nv, h):
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        while not self.stop.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((time.perf_counter(), sm, mx, {k for k, v in bits.items() if r & v}))
            except Exception:
                pass
            self.stop.wait(0.01)

    def _read_smi(self):
        for ln in self.proc.stdout:
            f = [x.strip() for x in ln.strip().split(",")]
            if len(f) < 8:
                continue
            try:
                sm, mx = float(f[1]), float(f[2])
            except ValueError:
                continue
            self.samples.append((time.perf_counter(), sm, mx,
                                 {nm for k, nm in enumerate(self.NAMES) if f[4 + k].lower().startswith("active")}))

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.thread = threading.Thread(target=self._poll_nvml, args=(nv, h), daemon=True)
        except Exception:
            try:
                self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                              "--format=csv,noheader,nounits", "-lms", "200"],
                                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.thread = threading.Thread(target=self._read_smi, daemon=True)
            except Exception:
                self.thread = None
        if self.thread:
            self.thread.start()
        return self

    def mark_start(self):
        self.t0 = time.perf_counter()

    def mark_stop(self):
        self.t1 = time.perf_counter()

    def __exit__(self, *exc):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)

    def summary(self):
        t0 = self.t0 if self.t0 is not None else -math.inf
        t1 = self.t1 if self.t1 is not None else math.inf
        sel = [x for x in self.samples if t0 <= x[0] <= t1]
        if not sel and self.samples:  # a region shorter than one sampling period: the nearest sample
            sel = [min(self.samples, key=lambda x: abs(x[0] - t1))]
        reasons = set()
        for x in sel:
            reasons |= x[3]
        return {"sm_mhz": statistics.median([x[1] for x in sel]) if sel else None,
                "sm_max_mhz": sel[-1][2] if sel else None, "reasons": sorted(reasons), "samples": len(sel),
                "source": "nvml" if self.proc is None else "nvidia-smi"}

def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        # host scalars (barrier, max over ranks) over gloo; the slab mode's
        # exchange buffers (device memory) over NCCL
        backend = "cpu:gloo,cuda:nccl" if getattr(args, "decomp", "replicas") == "slab" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def cuda_events_ms(stream_handle, fn):
    import torch
    s = torch.cuda.ExternalStream(stream_handle)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    fn()
    e1.record(s)
    e1.synchronize()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def precision_code(name):
    from weaklycompressiblesph_b200 import _native as N
    return {"fp32": N.PREC_FP32, "tiled": N.PREC_TILED, "half2": N.PREC_HALF2}[name]


def best_precision():
    from weaklycompressiblesph_b200.sim import BEST_PRECISION
    return BEST_PRECISION


def run_device(case, prec_name, steps, warmup, device, clocks=False, list_interval=0, list_skin=0.0):
    """Timed device-resident steps; returns dict of measurements."""
    from weaklycompressiblesph_b200.sim import Solver
    res = {}
    lists = list_interval > 0 and prec_name != "fp32"
    with Solver(case.n + 1024, precision=precision_code(prec_name), device=device, max_instances=4,
                list_interval=list_interval if lists else 0, list_skin=list_skin) as s:
        k = s.add(case)
        s.step(warmup)
        s.synchronize()
        pairs = s.last_pairs()
        if lists:
            # the timed steps start with a list build, so that they carry their
            # share of builds (one at least, then one every list_interval steps
            # or sooner when the drift rule asks) whatever their number
            s.invalidate_lists()
        ls0 = s.list_stats() if lists else None
        sampler = ClockSampler(device) if clocks else None
        if sampler:
            sampler.__enter__()
            time.sleep(0.05)  # the sampler's first reading comes before the timed region
            sampler.mark_start()
        ms = cuda_events_ms(s.stream(), lambda: s.step(steps))
        if sampler:
            sampler.mark_stop()
            sampler.__exit__()
            res["clocks"] = sampler.summary()
        pairs_end = s.last_pairs()
        res["ms_per_step"] = ms / steps
        res["pairs_per_step"] = 0.5 * (pairs + pairs_end)
        res["kernels_per_step"] = s.kernels_per_step()
        if lists:
            ls1 = s.list_stats()
            b, r = ls1["builds"] - ls0["builds"], ls1["list_steps"] - ls0["list_steps"]
            res["kernels_per_step"] = (b * ls1["kernels_build"] + r * ls1["kernels_list"]) / max(1, b + r)
            res["lists"] = {"interval": list_interval, "skin_h": list_skin or 0.3, "timed_builds": b,
                            "timed_list_steps": r, "overflows": ls1["overflows"], "longest": ls1["longest"],
                            "entries": s.list_entries()}
        # per-phase kernel times (eager launches, CUDA events on the solver
        # stream), split into steps that searched or built and steps that read
        # the lists; with lists the profile starts with a build and spans two
        # rebuild periods, so it carries builds in the timed region's share
        if lists:
            s.invalidate_lists()
            prof_steps = max(3, min(steps, 2 * list_interval))
        else:
            prof_steps = max(3, min(20, steps // 5))
        sp = s.profile_split(prof_steps)
        res["phase_ms"] = ((sp["build"] + sp["list"]) / prof_steps).tolist()
        res["profile"] = sp
        res["status"] = s.status(k)
        res["tuning"] = s.tuning()
    return res


def run_slab(case, prec_name, steps, warmup, rank, world, device, pg, clocks=False):
    """One dam break cut into `world` x-slabs, this rank's slab on its GPU;
    every step is followed by the ghost-layer and particle exchange and the
    dt minimum over the ranks.  Timed with CUDA events on the solver stream
    (the exchange synchronises it, so the interval spans all of it)."""
    from weaklycompressiblesph_b200 import slab
    slabs = slab.plan(case, world)
    dom = slab.SlabDomain(case, slabs, rank, precision=precision_code(prec_name), device=device)
    try:
        drv = slab.DistRank(dom, rank, world) if world > 1 else slab.LocalGroup([dom])
        drv.start()
        drv.step(warmup)
        barrier(pg)
        pairs = dom.last_pairs()
        sampler = ClockSampler(device) if clocks else None
        if sampler:
            sampler.__enter__()
            time.sleep(0.05)
            sampler.mark_start()
        ms = cuda_events_ms(dom.solver.stream(), lambda: drv.step(steps))
        if sampler:
            sampler.mark_stop()
            sampler.__exit__()
        res = {"ms_per_step": ms / steps, "pairs_per_step": 0.5 * (pairs + dom.last_pairs()),
               "kernels_per_step": dom.solver.kernels_per_step() + 3,  # + classify, pack, commit (+ unpacks)
               "status": dom.status(), "tuning": None, "owned": int(dom.read()["alive"].sum())}
        if sampler:
            res["clocks"] = sampler.summary()
        barrier(pg)
        # per-phase kernel times of the slab's own passes (after the timed region; no exchange)
        prof_steps = max(3, min(20, steps // 5))
        res["phase_ms"] = (dom.solver.profile_steps(prof_steps) / prof_steps).tolist()
    finally:
        dom.close()
    return res


def run_e2e(case, steps, warmup, device):
    """FDPS drop-in over host walk records: dispatch + retrieve per pass."""
    import ctypes as C
    from weaklycompressiblesph_b200 import fdps
    from weaklycompressiblesph_b200 import _native as N
    pres, snds = case.eos()
    w = fdps.build_walks(case.pos, 2.0 * case.h, group_size=128)
    epi, epj = fdps.walk_records(w, case.pos, case.vel, case.dens, pres, snds, case.h, case.mass, case.phys.nu,
                                 type_=case.type)
    out = np.zeros(len(epi), fdps.RESULT_HYDRO)
    N.call("wcsph_init", device)
    fdps.configure(fdps.pair_params("reference_cpu", alpha=case.phys.alpha, beta=case.phys.beta,
                                    c_cfl=case.phys.c_cfl, vsig_mode=case.phys.vsig_mode))
    limit = 16384  # N_WALK_LIMIT, kernel.cuh:4
    batches = []
    for w0 in range(0, w.n_walk, limit):
        w1 = min(w.n_walk, w0 + limit)
        pi = (C.c_void_p * (w1 - w0))(*[epi[w.i_off[k]:].ctypes.data for k in range(w0, w1)])
        pj = (C.c_void_p * (w1 - w0))(*[epj[w.j_off[k]:].ctypes.data for k in range(w0, w1)])
        po = (C.c_void_p * (w1 - w0))(*[out[w.i_off[k]:].ctypes.data for k in range(w0, w1)])
        ni = np.ascontiguousarray(np.diff(w.i_off[w0:w1 + 1]), np.int32)
        nj = np.ascontiguousarray(np.diff(w.j_off[w0:w1 + 1]), np.int32)
        batches.append((pi, pj, po, ni, nj, w1 - w0))
    L = N.lib()

    def one_pass():
        for pi, pj, po, ni, nj, nw in batches:
            N.check("dispatch", L.wcsph_hydro_dispatch(0, nw, pi, N.ptr(ni, C.c_int32), pj, N.ptr(nj, C.c_int32)))
            N.check("retrieve", L.wcsph_hydro_retrieve(0, nw, N.ptr(ni, C.c_int32), po))

    for _ in range(warmup):
        one_pass()
    # bytes each pass moves, as the library counts them (wcsph_fdps_stats after each batch)
    h2d = d2h = pieces = compact = 0
    st = (C.c_int64 * 4)()
    for pi, pj, po, ni, nj, nw in batches:
        N.check("dispatch", L.wcsph_hydro_dispatch(0, nw, pi, N.ptr(ni, C.c_int32), pj, N.ptr(nj, C.c_int32)))
        N.check("stats", L.wcsph_fdps_stats(0, st))
        N.check("retrieve", L.wcsph_hydro_retrieve(0, nw, N.ptr(ni, C.c_int32), po))
        h2d, d2h, compact, pieces = h2d + st[0], d2h + st[1], compact + st[2], pieces + st[3]
    split = [0.0, 0.0]  # dispatch (pack + enqueue), retrieve (wait + unpack)

    def timed_pass():
        for pi, pj, po, ni, nj, nw in batches:
            t0 = time.perf_counter()
            N.check("dispatch", L.wcsph_hydro_dispatch(0, nw, pi, N.ptr(ni, C.c_int32), pj, N.ptr(nj, C.c_int32)))
            t1 = time.perf_counter()
            N.check("retrieve", L.wcsph_hydro_retrieve(0, nw, N.ptr(ni, C.c_int32), po))
            split[0] += t1 - t0
            split[1] += time.perf_counter() - t1

    t0 = time.perf_counter()
    for _ in range(steps):
        timed_pass()
    dt = (time.perf_counter() - t0) / steps
    return dict(s_per_pass=dt, h2d=int(h2d), d2h=int(d2h), n_walk=w.n_walk, evaluated=w.n_evaluated, walks=w, epi=epi,
                epj=epj, dispatch_ms=1e3 * split[0] / steps, retrieve_ms=1e3 * split[1] / steps,
                pieces=int(pieces), pieces_compact=int(compact))


def cpu_reference(case, walks, epi, epj, seconds, pairs_total, whole_budget_s=None):
    """The reference's CalcHydroForce (oracle/_ref) over the walks of the
    workload on all host threads.  Whole passes over every walk when one fits
    in whole_budget_s (default: seconds), else repeated passes over a bounded
    sample of the walks (every k-th walk).  Returns (pairs/s, description,
    cores, seconds of one whole pass: measured, or from the sample's rate)."""
    import oracle
    if not oracle.ref_available():
        raise RuntimeError("oracle/_ref/libwcsph_ref.so missing")
    cores = os.cpu_count() or 1
    cfg = oracle.config_from_case(case)
    cnt, tot = oracle.neighbors(oracle.pos4(case.pos.astype(np.float32)), cfg)
    n_walk = walks.n_walk
    stride = max(1, n_walk // 64)
    sel = np.arange(0, n_walk, stride)

    def sample(sel):
        i_off = np.zeros(len(sel) + 1, np.int64)
        j_off = np.zeros(len(sel) + 1, np.int64)
        i_off[1:] = np.cumsum(walks.i_off[sel + 1] - walks.i_off[sel])
        j_off[1:] = np.cumsum(walks.j_off[sel + 1] - walks.j_off[sel])
        ei = np.concatenate([epi[walks.i_off[k]:walks.i_off[k + 1]] for k in sel])
        ej = np.concatenate([epj[walks.j_off[k]:walks.j_off[k + 1]] for k in sel])
        pairs = int(sum(cnt[walks.i_idx[walks.i_off[k]:walks.i_off[k + 1]]].sum() for k in sel))
        return i_off, ei, j_off, ej, pairs

    # probe on the sample to estimate a whole pass
    i_off, ei, j_off, ej, pairs = sample(sel)
    t0 = time.perf_counter()
    oracle.ref_hydro_walks(i_off, ei, j_off, ej, nthreads=cores)
    t1 = max(time.perf_counter() - t0, 1e-4)
    est_whole = t1 * tot / max(pairs, 1)
    budget = seconds if whole_budget_s is None else whole_budget_s
    consts = "(the functor's own alpha 0.01 and C_CFL 0.3, force.h:32, param.h:5: the same pairs and arithmetic as " \
             "the config's alpha 0.1, C_CFL 0.25)"
    if est_whole <= budget:
        reps = max(1, int(seconds / est_whole))
        t0 = time.perf_counter()
        for _ in range(reps):
            oracle.ref_hydro_walks(walks.i_off, epi, walks.j_off, epj, nthreads=cores)
        el = (time.perf_counter() - t0) / reps
        desc = (f"whole passes over all {n_walk} FDPS-style walks (<=128 i each), {tot} true pairs, {reps} "
                f"repetitions, STD::CalcHydroForce -O3 -ffast-math OpenMP {consts}")
        return tot / el, desc, cores, el
    reps = max(1, int(seconds / t1))
    t0 = time.perf_counter()
    for _ in range(reps):
        oracle.ref_hydro_walks(i_off, ei, j_off, ej, nthreads=cores)
    el = (time.perf_counter() - t0) / reps
    desc = (f"{len(sel)} of {n_walk} FDPS-style walks (every {stride}th, <=128 i each), {pairs} true pairs, "
            f"{reps} repetitions, STD::CalcHydroForce -O3 -ffast-math OpenMP {consts}")
    return pairs / el, desc, cores, tot * el / max(pairs, 1)


def measure_ensemble(device, steps=None):
    """Config 4 sample: 64 seeded dam breaks (fluid counts log-uniform in
    [1e4, 5e5]) stepping together, vs the same instances one at a time on the
    plain FP32 path; `steps` timed steps each (the config runs 2000)."""
    from weaklycompressiblesph_b200 import cases, ensemble
    steps = steps or ARGS.ensemble_steps
    ens = cases.ensemble_cases(count=64, seed=2024)
    b = ensemble.run_batched(ens, steps=steps, warmup=3, device=device, list_interval=ARGS.list_interval,
                             precision=ARGS.ensemble_precision)
    s = ensemble.run_serial(ens, steps=steps, warmup=3, precision="fp32", device=device)
    other = None
    if ARGS.ensemble_precision != "tiled":  # the default FP32 list path on the same instances
        o = ensemble.run_batched(ens, steps=steps, warmup=3, device=device, list_interval=ARGS.list_interval,
                                 precision="tiled")
        other = {"precision": "tiled", "batched_particle_steps_per_s": o["particle_steps_per_s"],
                 "speedup_vs_serial_plain": o["particle_steps_per_s"] / s["particle_steps_per_s"],
                 "lists": _list_summary(o.get("lists"))}
    return {"instances": len(ens), "particles": b["particles"], "steps": steps,
            "precision": ARGS.ensemble_precision,
            "batched_particle_steps_per_s": b["particle_steps_per_s"],
            "serial_plain_particle_steps_per_s": s["particle_steps_per_s"],
            "speedup_vs_serial_plain": b["particle_steps_per_s"] / s["particle_steps_per_s"],
            "fp32_lists": other,
            "tuning": b.get("tuning"),
            "lists": _list_summary(b.get("lists")),
            "sample": f"{steps} timed steps per instance" + ("" if steps >= 2000 else " (config: 2000)"),
            "neighbour_search": (f"lists, rebuilt at least every {ARGS.list_interval} steps" if ARGS.list_interval
                                 else "every step") + "; serial baseline: plain FP32, search every step"}


def measure_serving(device):
    """Config 5 sample: Poisson(20/s) dam-break requests, fluid counts
    log-uniform in [2e4, 2e5] (config: up to 2e6), each run to t = 0.1 s
    (config: 1.0 s), admitted by a 150 GB HBM budget; p50/p99
    time-to-completion and aggregate particle-steps/s, vs the same requests
    one at a time on the plain FP32 path."""
    from weaklycompressiblesph_b200 import _native as N
    from weaklycompressiblesph_b200 import cases
    from weaklycompressiblesph_b200.serving import Server, run_alone
    reqs = cases.serving_requests(count=ARGS.serving_requests, rate=20.0, seed=7, n_min=2e4,
                                  n_max=ARGS.serving_nmax, t_end=ARGS.serving_tend)
    total = sum(c.n for _, c in reqs)
    with Server(budget_bytes=150e9, max_particles=total + 1024, device=device, read_results=False,
                list_interval=ARGS.list_interval, precision=precision_code(ARGS.serving_precision)) as srv:
        out = srv.run(reqs)
    el = 0.0
    ps = 0
    for _, c in ([] if ARGS.serving_no_serial else reqs):
        t, steps, _ = run_alone(c, precision=N.PREC_FP32, device=device)
        el += t
        ps += c.n * steps
    serial = ps / el if el > 0 else None
    return {"requests": len(reqs), "particles": total, "p50_s": out["p50_s"], "p99_s": out["p99_s"],
            "wall_s": out["wall_s"], "particle_steps_per_s": out["particle_steps_per_s"],
            "serial_plain_particle_steps_per_s": serial,
            "speedup_vs_serial_plain": out["particle_steps_per_s"] / serial if serial else None,
            "neighbour_search": (f"lists, rebuilt at least every {ARGS.list_interval} steps" if ARGS.list_interval
                                 else "every step") + "; serial baseline: plain FP32, search every step",
            "precision": ARGS.serving_precision,
            "lists": _list_summary(out.get("lists")),
            "sample": f"{len(reqs)} requests, counts log-uniform [2e4, {ARGS.serving_nmax:.0e}], "
                      f"t_end {ARGS.serving_tend:g} s, Poisson 20/s, budget 150 GB"
                      + ("" if ARGS.serving_nmax >= 2e6 and ARGS.serving_tend >= 1.0
                         else " (config: counts to 2e6, t_end 1.0 s)")}


def _list_summary(ls):
    if not ls:
        return None
    steps = ls["builds"] + ls["list_steps"]
    return {"builds": ls["builds"], "partial_builds": ls.get("partial_builds"), "list_steps": ls["list_steps"],
            "overflows": ls["overflows"], "steps_per_build": steps / max(1, ls["builds"])}


ARGS = None


def main():
    global ARGS
    args = parse()
    ARGS = args
    world, rank, local, pg = dist_setup(args)
    if args.impl == "reference":
        if rank != 0:
            return 0
        return main_reference(args)
    import torch
    torch.cuda.set_device(local)
    from weaklycompressiblesph_b200 import build as B
    B.build()
    prec = args.precision if args.precision != "best" else best_precision()
    case = make_case(args.workload)
    if args.ncu_pass:
        if rank == 0:
            from weaklycompressiblesph_b200.sim import Solver
            with Solver(case.n + 1024, precision=precision_code(prec), max_instances=4,
                        list_interval=args.list_interval, list_skin=args.list_skin, list_shape=0, autotune=False,
                        use_graph=False) as s:
                s.add(case)
                s.step(12)
                s.synchronize()
                print(json.dumps({"ncu_pass": True, "precision": prec, "lists": s.list_stats()}))
        return finish(pg)
    if args.e2e_only:
        if rank == 0:
            e = run_e2e(case, args.steps, args.warmup, local)
            print(json.dumps({"e2e_only": True, "workload": args.workload, "passes": args.steps,
                              "warmup": args.warmup, "ms_per_pass": 1e3 * e["s_per_pass"],
                              "dispatch_ms": e["dispatch_ms"], "retrieve_ms": e["retrieve_ms"],
                              "walks": e["n_walk"], "pair_evaluations_per_pass": e["evaluated"],
                              "h2d_bytes_per_pass": e["h2d"], "d2h_bytes_per_pass": e["d2h"],
                              "pieces_compact": f"{e['pieces_compact']} of {e['pieces']}"}))
        barrier(pg)
        finish(pg)
        return 0
    barrier(pg)
    slab_mode = args.decomp == "slab"
    if slab_mode:
        args.no_plain = args.no_e2e = args.no_ensemble = True
        dev = run_slab(case, prec, args.steps, args.warmup, rank, world, local, pg, clocks=(rank == 0))
    else:
        dev = run_device(case, prec, args.steps, args.warmup, local, clocks=(rank == 0),
                         list_interval=args.list_interval, list_skin=args.list_skin)
    ms = max_over_ranks(pg, dev["ms_per_step"])
    pairs_all = sum_over_ranks(pg, dev["pairs_per_step"])
    value = pairs_all / (ms * 1e-3)
    steps_per_s = 1e3 / ms
    plain = search = None
    if prec != "fp32" and not args.no_plain:
        p = run_device(case, "fp32", max(10, args.steps // 4), args.warmup, local)
        plain = {"value": p["pairs_per_step"] / (p["ms_per_step"] * 1e-3), "steps_per_s": 1e3 / p["ms_per_step"],
                 "ms_per_step": p["ms_per_step"]}
        if dev.get("lists"):  # the same path with a neighbour search every step
            q = run_device(case, prec, args.steps, args.warmup, local)
            search = {"value": q["pairs_per_step"] / (q["ms_per_step"] * 1e-3), "steps_per_s": 1e3 / q["ms_per_step"],
                      "ms_per_step": q["ms_per_step"], "hydro_ms": q["phase_ms"][2]}
    other = None
    if not args.no_other_precision and not slab_mode and prec in ("tiled", "half2"):
        oprec = "half2" if prec == "tiled" else "tiled"
        o = run_device(case, oprec, args.steps, args.warmup, local, list_interval=args.list_interval,
                       list_skin=args.list_skin)
        other = {"precision": oprec, "value": o["pairs_per_step"] / (o["ms_per_step"] * 1e-3),
                 "steps_per_s": 1e3 / o["ms_per_step"], "ms_per_step": o["ms_per_step"],
                 "hydro_ms": o["phase_ms"][2], "lists": o.get("lists"), "tuning": o.get("tuning")}
        if plain:
            other["speedup_vs_plain_fp32"] = other["steps_per_s"] / plain["steps_per_s"]
        other["error_vs_fp64"] = validation_errors(args.workload, oprec)
    peak, peak_kind = load_peaks()
    if other:
        other["roofline"] = hbm_roofline(args.workload, other["precision"], case.n, o, peak, peak_kind)
        other["roofline_l1"] = l1_roofline(args.workload, other["precision"], o)
    roof = hbm_roofline(args.workload, prec, case.n, dev, peak, peak_kind)
    l1 = l1_roofline(args.workload, prec, dev)
    e2e = None
    cpu = None
    if rank == 0 and not args.no_e2e and args.workload != "periodic8m":
        e = run_e2e(case, max(1, min(3, args.steps // 50)), 1, local)
        e2e = {"value": dev["pairs_per_step"] / e["s_per_pass"], "unit": UNIT, "h2d_bytes_per_step": e["h2d"],
               "d2h_bytes_per_step": e["d2h"], "path": "wcsph_hydro_dispatch/retrieve, FDPS walks of <=128 i",
               "walks": e["n_walk"], "pair_evaluations_per_pass": e["evaluated"],
               "ms_per_pass": 1e3 * e["s_per_pass"], "dispatch_ms": e["dispatch_ms"], "retrieve_ms": e["retrieve_ms"],
               "pieces_compact": f"{e['pieces_compact']} of {e['pieces']}"}
        if not args.no_cpu:
            v, desc, cores, _ = cpu_reference(case, e["walks"], e["epi"], e["epj"], args.cpu_seconds,
                                              dev["pairs_per_step"])
            cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "reference", "sample": desc}
    ens = srv = None
    if rank == 0 and not args.no_ensemble:
        ens = measure_ensemble(local)
        srv = measure_serving(local)
    if rank != 0:
        barrier(pg)
        finish(pg)
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong" if slab_mode else "weak",
        "vs_baseline": None, "dtype": "f32" if prec != "half2" else "f16x2-pair/f32-accumulate",
        "data": "synthetic (seeded lattice IC, no dataset)",
        "config": bench_config(args, case, prec, world),
        "steps_per_s": steps_per_s * 1.0,
        "pairs_per_step": dev["pairs_per_step"],
        "plain_fp32": plain,
        "speedup_vs_plain_fp32": (steps_per_s / plain["steps_per_s"]) if plain else None,
        "search_every_step": search,
        ("half2" if other and other["precision"] == "half2" else "fp32_tiled"): other,
        "phase_ms": {"bin_sort_permute": dev["phase_ms"][0], "density": dev["phase_ms"][1],
                     "hydro": dev["phase_ms"][2], "total": dev["phase_ms"][3]},
        "roofline": roof,
        "roofline_l1": l1,
        "error_vs_fp64": validation_errors(args.workload, prec),
        "cpu_baseline": cpu,
        "e2e": e2e,
        "autotune": dev.get("tuning"),
        "ensemble": ens,
        "serving": srv,
        "gpu_launches": int(round(dev["kernels_per_step"] * args.steps)),
        "neighbour_lists": dev.get("lists"),
        "clocks": dev.get("clocks"),
        "sim_time_s": dev["status"]["time"],
    }
    if slab_mode:
        line["e2e_note"] = "e2e, cpu_baseline, plain FP32, ensemble and serving are measured in the default mode"
    print(json.dumps(line))
    sys.stdout.flush()
    barrier(pg)
    finish(pg)
    return 0


def _profile_json(name):
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)


def validation_errors(workload, prec):
    """Relative L2 errors against the FP64 oracle of the same path, from the
    committed summary of tests/validate_dam_break.py (largest over its
    checkpoints), or None when that path was not validated on this workload."""
    v = _profile_json("validation_dam1m.json")
    if not v or workload != "dam1m":
        return None
    path = {"tiled": "tiled_lists", "half2": "half2_lists", "fp32": None}.get(prec)
    r = v.get("paths", {}).get(path)
    if not r:
        return None
    return {"acc": r["max_acc"], "div_v": r["max_div_v"], "drho_dt": r["max_drho_dt"], "checkpoints": r["checkpoints"],
            "steps": v["steps"], "source": "tests/validate_dam_break.py (profiles/validation_dam1m.md)"}


# Bytes a hydro pass must move per particle besides the j-records it gathers:
# the epilogue reads position, velocity, half-step velocity, flags and id and
# writes position, velocity, acceleration (+ div v), flags and id (112 B, the
# final kick and the dt candidate are fused into the pass); the particle's own
# FP32 j-record and c (36 B); with lists its entry count (4 B).
PASS_STATE_BYTES = 112
OWN_RECORD_BYTES = 36
COMPACT_RECORD_BYTES = 20   # half2 lists: the particle's compact record and P/rho^2, fetched once as j operands
SURVEY_I_BYTES = 64         # the per-particle i read and write of the per-pair record model


def hbm_roofline(workload, prec, n, dev, peak, peak_kind):
    """The hydro pass against HBM.  Algorithmic bytes per launch = what the
    pass must move at least: every particle's state and own record once, and
    with lists every list word once (4 B per entry); a j-record that a
    particle's neighbours gather again comes from L1 or L2, so it is counted
    once.  Duration = the pass's average launch time over the profiled steps
    (CUDA events on the solver stream): on list steps exactly one list-pass
    launch.  `traffic` is the DRAM bytes of one launch from an ncu capture.
    `pair_record_model` is the per-pair model (36 B per true pair + 64 B per
    particle), an operand rate: the records it counts reach the pair terms
    from L1 and L2, so it is not a DRAM figure and can exceed the HBM peak."""
    sp = dev.get("profile")
    lists = dev.get("lists")
    bpp = BYTES_PER_PAIR[prec]
    if lists and sp and sp["list_steps"] > 0:
        kernel = {"tiled": "k_hydro_list<0> (list pass, FP32 records)",
                  "half2": "k_hydro_list<1> (list pass, half2 compact records)"}[prec]
        launch_ms = sp["list"][2] / sp["list_steps"]
        per_particle = PASS_STATE_BYTES + OWN_RECORD_BYTES + 4 + (COMPACT_RECORD_BYTES if prec == "half2" else 0)
        alg = n * per_particle + 4.0 * lists["entries"]
        units = (f"{per_particle} B per particle (state {PASS_STATE_BYTES}, own record {OWN_RECORD_BYTES}, "
                 f"list count 4" + (f", compact record and P/rho^2 {COMPACT_RECORD_BYTES}" if prec == "half2" else "")
                 + ") + 4 B per list entry")
        key = f"{workload}/{prec}/lists"
    else:
        kernel = {"tiled": "k_hydro_tiled (search every step)", "half2": "k_hydro_tiled (search every step)",
                  "fp32": "k_hydro_plain (search every step)"}[prec]
        tot = (sp["build"][2] + sp["list"][2]) if sp else dev["phase_ms"][2]
        launch_ms = tot / max(1, (sp["build_steps"] + sp["list_steps"]) if sp else 1)
        per_particle = PASS_STATE_BYTES + OWN_RECORD_BYTES
        alg = n * per_particle
        units = f"{per_particle} B per particle (state {PASS_STATE_BYTES}, own record {OWN_RECORD_BYTES})"
        key = f"{workload}/{prec}"
    achieved = alg / (launch_ms * 1e-3) / 1e9
    traffic = None
    limiter = "instruction issue"
    if lists:
        l1 = (_profile_json("hydro_list_l1.json") or {}).get(f"{workload}/{prec}", {})
        limiter = l1.get("limiter", "L1 data pipe") + " (roofline_l1)"
    tp = _profile_json("hydro_traffic.json")
    if tp:
        traffic = tp.get(key, {}).get("bytes_per_launch")
    pair_rate = (dev["pairs_per_step"] * bpp + n * SURVEY_I_BYTES) / (launch_ms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "kernel": kernel, "launch_ms": launch_ms, "algorithmic_bytes": alg,
            "model": units, "peak_kind": peak_kind,
            "limiter": limiter,
            "pair_record_model": {"bytes_per_pair": bpp, "bytes_per_particle": SURVEY_I_BYTES,
                                  "operand_rate_gbs": pair_rate,
                                  "note": "j-records delivered to the pair terms, mostly from L1; not DRAM"}}


def l1_roofline(workload, prec, dev):
    """The FP32 list pass is bound by the L1 data pipe that delivers its
    gathers (the half2 pass about as much by issue).  Per list entry it needs
    one list word and one j-record (half2: the compact record and P/rho^2): at
    128 B per L1 wavefront that is (4 + record bytes) / 128 wavefronts at least.  The
    measured L1 load wavefronts of one launch come from the ncu capture
    summarised in profiles/hydro_list_l1.json; entries and true pairs are this
    run's."""
    t = _profile_json("hydro_list_l1.json")
    lists = dev.get("lists")
    if not t or not lists or not lists.get("entries"):
        return None
    r = t.get(f"{workload}/{prec}")
    if not r:
        return None
    entries, pairs = lists["entries"], dev["pairs_per_step"]
    need = entries * (4 + r["record_bytes"]) / 128.0
    return {"bound": "l1", "wavefronts_per_launch": r["wavefronts"], "min_wavefronts_per_launch": need,
            "frac": need / r["wavefronts"], "wavefronts_per_pair": r["wavefronts"] / pairs,
            "entries_per_pair": entries / pairs, "record_bytes": r["record_bytes"],
            "l1_pipe_util_pct": r.get("l1_pipe_util_pct"),
            "source": "ncu capture of one list-pass launch, profiles/hydro_list_l1.json"}


def bench_config(args, case, prec, world):
    """The workload description, the same in both arms (a function of the
    command line and the case only)."""
    lists = args.list_interval > 0 and prec != "fp32" and args.decomp != "slab"
    return {"workload": {"dam1m": "3-D dam break dx=0.005 (1,024,000 fluid + 571,308 wall particles)",
                         "dam16k": "3-D dam break dx=0.02 (16,000 fluid + 38,508 wall particles)",
                         "periodic8m": "periodic jittered lattice 200^3 dx=0.01"}[args.workload],
            "n_particles": case.n, "precision": prec, "h_over_dx": case.phys.h_over_dx,
            "neighbour_search": (f"lists of radius 2h + {args.list_skin or 0.3:g} h, rebuilt at least every "
                                 f"{args.list_interval} steps" if lists else "every step"),
            "density_mode": case.phys.density_mode,
            "parallelism": f"slab x{world}" if args.decomp == "slab" else f"replicas x{world}",
            "l2": "working set > L2 (126 MB): particle state and records "
                  f"{case.n * 200 / 1e6:.0f} MB, no flush needed"}


def finish(pg):
    if pg is not None:
        pg.destroy_process_group()


def main_reference(args):
    """The reference arm: STD::CalcHydroForce (oracle/_ref) over the walks of the
    same workload on all host cores; each step a bounded sample of walks."""
    import oracle
    case = make_case(args.workload)
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libwcsph_ref.so was not built"}))
        return 0
    from weaklycompressiblesph_b200 import fdps
    pres, snds = case.eos()
    w = fdps.build_walks(case.pos, 2.0 * case.h, group_size=128)
    epi, epj = fdps.walk_records(w, case.pos, case.vel, case.dens, pres, snds, case.h, case.mass, case.phys.nu,
                                 type_=case.type)
    # each step one whole pass over every walk when the whole run stays within
    # about four minutes, else a bounded sample of the walks
    per_step = max(1.0, min(10.0, 240.0 / max(1, args.steps + args.warmup)))
    vals, secs = [], []
    for k in range(args.warmup + args.steps):
        v, desc, cores, whole_s = cpu_reference(case, w, epi, epj, per_step, None, whole_budget_s=per_step)
        if k >= args.warmup:
            vals.append(v)
            secs.append(whole_s)
    value = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "ms_per_step": 1e3 * statistics.median(secs),
            "ms_per_step_note": "one hydro pass of the functor over every walk of the workload (no tree, EoS or KDK)",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lattice IC, no dataset)",
            "config": bench_config(args, case, args.precision if args.precision != "best" else best_precision(),
                                   int(os.environ.get("WORLD_SIZE", "1"))),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())

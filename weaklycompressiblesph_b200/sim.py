"""Device-resident solver: Python mirror of the wcsph_sim_* C ABI.

A ``Solver`` owns device memory for up to ``max_particles`` particles and any
number of independent simulation instances that advance together, each with
its own CFL timestep (the reference's main loop, src/main.cpp:89-133, run on
the device for every instance at once).
"""
from __future__ import annotations

import ctypes as C
from types import SimpleNamespace

import numpy as np

from . import _native as N
from .cases import Case


# The fastest pair-sum variant this build ships (used when callers ask for "best").
BEST_PRECISION = "tiled"


def _f32(a, shape):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(shape))


class Solver:
    def __init__(self, max_particles, precision=N.PREC_FP32, max_cells=None, max_instances=64, device=0,
                 use_graph=True, autotune=True, list_interval=0, list_skin=0.0, list_shape=None,
                 build_shape=None):
        """list_interval > 0 turns on neighbour lists (radius 2h + list_skin h,
        rebuilt at least every list_interval steps; see wcsph_sim_options).
        list_shape / build_shape fix the list pass's and the list build scan's
        launch shapes (None: the autotuner's)."""
        o = N.SimOptions()
        o.device = device
        o.precision = precision
        o.max_particles = int(max_particles)
        o.max_cells = int(max_cells if max_cells is not None else max(1 << 20, 2 * max_particles))
        o.max_instances = int(max_instances)
        o.use_graph = 1 if use_graph else 0
        o.autotune = 1 if autotune else 0
        o.list_interval = int(list_interval)
        o.list_skin = float(list_skin)
        o.list_shape = (0 if list_shape is None else int(list_shape) + 1) | \
            ((0 if build_shape is None else int(build_shape) + 1) << 8)
        self.opt = o
        h = C.c_void_p()
        N.call("wcsph_sim_create", C.byref(o), C.byref(h))
        self._h = h
        self.slots = {}

    @staticmethod
    def device_bytes(max_particles, max_cells=None, max_instances=64, list_interval=0):
        o = N.SimOptions(0, 0, int(max_particles), int(max_cells or max(1 << 20, 2 * max_particles)),
                         int(max_instances), 1, 0, int(list_interval))
        return int(N.lib().wcsph_sim_device_bytes(C.byref(o)))

    def close(self):
        if self._h:
            N.lib().wcsph_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- instances ---------------------------------------------------------
    def add(self, case: Case, density_mode=None, t_end=None) -> int:
        d = case.desc(density_mode=density_mode, t_end=t_end)
        pos = _f32(case.pos, (-1, 3))
        vel = _f32(case.vel, (-1, 3))
        dens = _f32(case.dens, (-1,))
        typ = np.ascontiguousarray(case.type, dtype=np.int32)
        slot = C.c_int32()
        N.call("wcsph_sim_add_instance", self._h, C.byref(d), N.ptr(pos, C.c_float), N.ptr(vel, C.c_float),
               N.ptr(dens, C.c_float), N.ptr(typ, C.c_int32), C.byref(slot))
        self.slots[slot.value] = case
        return slot.value

    def restore(self, case, state, desc=None) -> int:
        """Add an instance from saved state (a dict with pos, vel, dens, acc,
        div_v, time, steps, dt_next and optionally alive, order, type; see
        snapshot.py) without a force pass, so that it continues exactly where
        the saved run stopped.  case may be None when desc and state["type"]
        are given."""
        d = desc if desc is not None else case.desc()
        n = int(d.n)
        typ = state.get("type", None if case is None else case.type)
        f = lambda a, shape: np.ascontiguousarray(np.asarray(a, np.float32).reshape(shape))
        i32 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.int32)
        typ, alive, order = i32(typ), i32(state.get("alive")), i32(state.get("order"))
        if typ is None or len(typ) != n:
            raise ValueError("restore: particle types of length desc.n are required")
        slot = C.c_int32()
        N.call("wcsph_sim_restore_instance", self._h, C.byref(d), N.ptr(f(state["pos"], (n, 3)), C.c_float),
               N.ptr(f(state["vel"], (n, 3)), C.c_float), N.ptr(f(state["dens"], (n,)), C.c_float),
               N.ptr(typ, C.c_int32), N.ptr(f(state["acc"], (n, 3)), C.c_float),
               N.ptr(f(state["div_v"], (n,)), C.c_float), N.ptr(alive, C.c_int32), N.ptr(order, C.c_int32),
               float(state["time"]), int(state["steps"]), float(state["dt_next"]), C.byref(slot))
        self.slots[slot.value] = case if case is not None else SimpleNamespace(n=n, type=typ)
        return slot.value

    def next_dt(self, slot):
        v = C.c_float()
        N.call("wcsph_sim_next_dt", self._h, slot, C.byref(v))
        return v.value

    def set_next_dt(self, slot, dt):
        N.call("wcsph_sim_set_next_dt", self._h, slot, float(dt))

    def force_pass(self, slot):
        N.call("wcsph_sim_force_pass", self._h, slot)

    # -- slab decomposition (see slab.py) ------------------------------------
    def add_slab(self, case: Case, slab: N.Slab, ids, density_mode=None, t_end=None) -> int:
        """Add the particles `ids` of `case` as the slab `slab` of a decomposed
        simulation; no force pass runs (see wcsph_sim_add_slab)."""
        d = case.desc(density_mode=density_mode, t_end=t_end)
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        pos = _f32(case.pos[ids], (-1, 3))
        vel = _f32(case.vel[ids], (-1, 3))
        dens = _f32(case.dens[ids], (-1,))
        typ = np.ascontiguousarray(case.type[ids], dtype=np.int32)
        slot = C.c_int32()
        N.call("wcsph_sim_add_slab", self._h, C.byref(d), C.byref(slab), len(ids), N.ptr(ids, C.c_int32),
               N.ptr(pos, C.c_float), N.ptr(vel, C.c_float), N.ptr(dens, C.c_float), N.ptr(typ, C.c_int32),
               C.byref(slot))
        self.slots[slot.value] = case
        return slot.value

    def slab_pack(self, slot, send_ptr, capacity):
        """Pack into the device buffer at send_ptr (capacity records); returns
        [emigrants left, ghosts left, emigrants right, ghosts right]."""
        counts = (C.c_int32 * 4)()
        N.call("wcsph_sim_slab_pack", self._h, slot, C.c_void_p(send_ptr), int(capacity), counts)
        return [int(c) for c in counts]

    def slab_unpack(self, slot, recv_ptr, n_owned, n_ghost):
        N.call("wcsph_sim_slab_unpack", self._h, slot, C.c_void_p(recv_ptr), int(n_owned), int(n_ghost))

    def remove(self, slot):
        N.call("wcsph_sim_remove_instance", self._h, slot)
        self.slots.pop(slot, None)

    # -- stepping ----------------------------------------------------------
    def step(self, nsteps=1):
        N.call("wcsph_sim_step", self._h, int(nsteps))

    def synchronize(self):
        N.call("wcsph_sim_synchronize", self._h)

    def status(self, slot):
        t = C.c_double()
        s = C.c_int64()
        n = C.c_int32()
        f = C.c_int32()
        N.call("wcsph_sim_instance_status", self._h, slot, C.byref(t), C.byref(s), C.byref(n), C.byref(f))
        return dict(time=t.value, steps=s.value, n_alive=n.value, finished=bool(f.value))

    def read(self, slot):
        n = self.slots[slot].n
        out = dict(pos=np.zeros((n, 3), np.float32), vel=np.zeros((n, 3), np.float32),
                   dens=np.zeros(n, np.float32), acc=np.zeros((n, 3), np.float32),
                   div_v=np.zeros(n, np.float32), alive=np.zeros(n, np.int32))
        N.call("wcsph_sim_read_instance", self._h, slot, N.ptr(out["pos"], C.c_float), N.ptr(out["vel"], C.c_float),
               N.ptr(out["dens"], C.c_float), N.ptr(out["acc"], C.c_float), N.ptr(out["div_v"], C.c_float), None,
               N.ptr(out["alive"], C.c_int32))
        return out

    def probe(self, slot, density_pass=0, lists=False):
        """Force pass on the current state without advancing it (original order).
        Returns acc (hydro only, no gravity), div_v, dt_i, dens used, neighbour counts.
        lists=True runs the passes of a neighbour-list step (wcsph_sim_probe_lists)
        instead of a fresh cell search."""
        n = self.slots[slot].n
        out = dict(acc=np.zeros((n, 3), np.float32), div_v=np.zeros(n, np.float32), dt=np.zeros(n, np.float32),
                   dens=np.zeros(n, np.float32), nbr=np.zeros(n, np.int32))
        fn = "wcsph_sim_probe_lists" if lists else "wcsph_sim_probe_forces"
        N.call(fn, self._h, slot, int(density_pass), N.ptr(out["acc"], C.c_float),
               N.ptr(out["div_v"], C.c_float), N.ptr(out["dt"], C.c_float), N.ptr(out["dens"], C.c_float),
               N.ptr(out["nbr"], C.c_int32))
        return out

    def order(self, slot):
        n = self.slots[slot].n
        perm = np.zeros(n, np.int32)
        key = np.zeros(n, np.uint32)
        m = N.lib().wcsph_sim_read_order(self._h, slot, N.ptr(perm, C.c_int32), N.ptr(key, C.c_uint32))
        if m < 0:
            N.check("wcsph_sim_read_order", m)
        return perm[:m], key[:m]

    def conservation(self, slot):
        out = np.zeros(6, np.float64)
        N.call("wcsph_sim_conservation", self._h, slot, N.ptr(out, C.c_double))
        return out

    def last_pairs(self):
        return int(N.lib().wcsph_sim_last_pairs(self._h))

    def kernels_per_step(self):
        return int(N.lib().wcsph_sim_kernels_per_step(self._h))

    def tuning(self):
        """Autotuner decision: tiled-kernel block shape, list-pass launch shape,
        tuned bucket, list-build scan shape."""
        out = np.zeros(4, np.int32)
        N.call("wcsph_sim_tuning", self._h, N.ptr(out, C.c_int32))
        return dict(tile_shape=int(out[0]), list_shape=int(out[1]), bucket=int(out[2]), build_shape=int(out[3]))

    def stream(self):
        """The solver's cudaStream_t as an integer handle."""
        return int(N.lib().wcsph_sim_stream(self._h) or 0)

    def list_stats(self):
        out = (C.c_int64 * 6)()
        N.call("wcsph_sim_list_stats", self._h, out)
        return dict(builds=int(out[0]), list_steps=int(out[1]), overflows=int(out[2]), longest=int(out[3]),
                    kernels_build=int(out[4]), kernels_list=int(out[5]))

    def list_schedule(self):
        """Builds, partial builds among them, list steps, steps since the last
        full build (wcsph_sim_list_schedule)."""
        out = (C.c_int64 * 4)()
        N.call("wcsph_sim_list_schedule", self._h, out)
        return dict(builds=int(out[0]), partial_builds=int(out[1]), list_steps=int(out[2]),
                    since_full=int(out[3]))

    def list_entries(self):
        """Entries of the current neighbour lists (0 without current lists)."""
        v = int(N.lib().wcsph_sim_list_entries(self._h))
        if v < 0:
            raise N.WcsphError("wcsph_sim_list_entries", -1, "CUDA error")
        return v

    def invalidate_lists(self):
        """The next step rebuilds the neighbour lists (wcsph_sim_invalidate_lists)."""
        N.call("wcsph_sim_invalidate_lists", self._h)

    def profile_steps(self, nsteps):
        """Advance nsteps eagerly with CUDA events per phase; returns ms summed
        over the steps: [binning+sort+permute, density, hydro, total]."""
        ms = np.zeros(4, np.float64)
        N.call("wcsph_sim_profile_steps", self._h, int(nsteps), N.ptr(ms, C.c_double))
        return ms

    def profile_split(self, nsteps):
        """Like profile_steps, split by kind of step: returns a dict with the
        phase milliseconds summed over the steps that searched or built
        ("build"), over the steps that read the lists ("list"), the builds'
        scans alone ("scan_ms") and the step counts."""
        ms = np.zeros(9, np.float64)
        cnt = np.zeros(2, np.int32)
        N.call("wcsph_sim_profile_split", self._h, int(nsteps), N.ptr(ms, C.c_double), N.ptr(cnt, C.c_int32))
        return {"build": ms[0:4].copy(), "list": ms[4:8].copy(), "scan_ms": float(ms[8]),
                "build_steps": int(cnt[0]), "list_steps": int(cnt[1])}

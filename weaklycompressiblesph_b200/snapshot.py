"""Snapshots and restarts of a device-resident instance.

* ASCII snapshots in the reference's column layout (src/class.h:129-134,
  3-D branch; header of FileHeader::writeAscii, class.h:54-57):
      <time %e>\\n<N %d>\\n
      id  tag  mass  x  y  z  vx  vy  vz  dens  0.0  pres      (tab separated)
  one file per snapshot, named like FDPS's writeParticleAscii output
  ``<dir>/<snapshot:05d>_<nproc:05d>_<rank:05d>.dat`` (src/io.h:12-14).
* ``OutputSchedule``: a snapshot whenever the physical time passes the next
  output time, which advances by end_time / number_of_snapshots
  (src/io.h:6, :34; param.h:6 sets 1560 snapshots).
* Binary restarts: a portable little-endian file (magic, version, the
  instance description, time, step count, next dt, then FP32/int32 arrays)
  named ``<dir>/<snapshot % keep:05d>_<nproc:05d>_<rank:05d>.bin``.  The
  reference dumps raw C++ objects and writes ``step % 10`` but reads
  ``step % 100`` (src/io.h:21 vs :63); here writer and reader share one
  naming rule, the file also holds the device storage order, and the
  restored run continues bit for bit (``Solver.restore``).
* ``SnapshotWriter`` writes files on a background thread: the device state is
  copied to the host synchronously, the formatting and I/O overlap the next
  steps.
"""
from __future__ import annotations

import ctypes as C
import os
import queue
import struct
import threading

import numpy as np

from . import _native as N

MAGIC = b"WCSPHRS1"


def ascii_name(directory, index, nproc=1, rank=0):
    return os.path.join(directory, f"{index:05d}_{nproc:05d}_{rank:05d}.dat")


def restart_name(directory, index, keep=10, nproc=1, rank=0):
    return os.path.join(directory, f"{index % keep:05d}_{nproc:05d}_{rank:05d}.bin")


class OutputSchedule:
    """Snapshot times of OutputFileWithTimeInterval (src/io.h:2-37): ``due(t)``
    returns the snapshot index to write at physical time t, or None."""

    def __init__(self, end_time, count=1560, start_time=0.0, start_index=0):
        self.interval = end_time / count
        self.next_time = start_time
        self.index = start_index

    def due(self, time):
        if time < self.next_time:
            return None
        k = self.index
        self.next_time += self.interval
        self.index += 1
        return k


def write_ascii(path, time, ids, tags, mass, pos, vel, dens, pres):
    """The reference's 3-D RealPtcl::writeAscii rows under FileHeader::writeAscii."""
    n = len(ids)
    mass = np.broadcast_to(np.asarray(mass, np.float64), (n,))
    cols = np.column_stack([mass, pos, vel, dens, np.zeros(n), pres]).astype(np.float64)
    with open(path, "w") as f:
        f.write("%e\n%d\n" % (time, n))
        idt = np.column_stack([ids, tags]).astype(np.int64)
        lines = ["%d\t%d\t" % (a, b) + "\t".join("%.16f" % v for v in row) for (a, b), row in zip(idt, cols)]
        f.write("\n".join(lines))
        if n:
            f.write("\n")


def read_ascii(path):
    with open(path) as f:
        time = float(f.readline())
        n = int(f.readline())
        data = np.loadtxt(f, ndmin=2) if n else np.zeros((0, 12))
    return dict(time=time, n=n, id=data[:, 0].astype(np.int64), tag=data[:, 1].astype(np.int64), mass=data[:, 2],
                pos=data[:, 3:6], vel=data[:, 6:9], dens=data[:, 9], pres=data[:, 11])


def instance_state(solver, slot):
    """Host copy of everything an exact restart needs: the particle state,
    time, step count, next dt, and the device storage order (the binning sort
    is stable, so the order fixes the summation sequence of the next steps)."""
    st = solver.read(slot)
    s = solver.status(slot)
    n = len(st["dens"])
    perm, _ = solver.order(slot)
    rest = np.setdiff1d(np.arange(n, dtype=np.int32), perm, assume_unique=False)
    st.update(time=s["time"], steps=s["steps"], dt_next=solver.next_dt(slot),
              order=np.concatenate([np.asarray(perm, np.int32), rest.astype(np.int32)]),
              type=np.asarray(solver.slots[slot].type, np.int32))
    return st


_ARRAYS = (("pos", "<f4", 3), ("vel", "<f4", 3), ("dens", "<f4", 1), ("acc", "<f4", 3), ("div_v", "<f4", 1),
           ("alive", "<i4", 1), ("type", "<i4", 1), ("order", "<i4", 1))
_HEAD = "<iiqdqf"


def write_restart(path, desc, state):
    """Binary restart: magic, version, size of the instance description, n,
    time, steps, next dt, the description itself, then the arrays of _ARRAYS."""
    blob = bytes(desc)
    n = int(desc.n)
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack(_HEAD, 1, len(blob), n, float(state["time"]), int(state["steps"]),
                            float(state["dt_next"])))
        f.write(blob)
        for key, dt, w in _ARRAYS:
            a = np.asarray(state[key])
            if a.size != n * w:
                raise ValueError(f"restart: {key} has {a.size} values, expected {n * w}")
            f.write(np.ascontiguousarray(a.reshape(-1), dtype=dt).tobytes())
    os.replace(tmp, path)  # a crash mid-write leaves the previous restart intact


def read_restart(path):
    """Returns (InstanceDesc, state dict) for Solver.restore(None, state, desc)."""
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise ValueError(f"{path}: not a wcsph restart file")
        ver, nblob, n, time, steps, dt_next = struct.unpack(_HEAD, f.read(struct.calcsize(_HEAD)))
        if ver != 1 or nblob != C.sizeof(N.InstanceDesc):
            raise ValueError(f"{path}: unsupported restart version {ver} / description size {nblob}")
        desc = N.InstanceDesc.from_buffer_copy(f.read(nblob))
        st = dict(time=time, steps=steps, dt_next=dt_next)
        for key, dt, w in _ARRAYS:
            raw = f.read(4 * n * w)
            if len(raw) != 4 * n * w:
                raise ValueError(f"{path}: truncated at {key}")
            a = np.frombuffer(raw, dtype=dt).astype(np.float32 if dt.endswith("f4") else np.int32)
            st[key] = a.reshape(n, w) if w > 1 else a
    return desc, st


class SnapshotWriter:
    """Background writer: `snapshot` / `restart` copy the state now and queue the file I/O."""

    def __init__(self):
        self._q = queue.Queue()
        self._err = None
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        while True:
            job = self._q.get()
            if job is None:
                return
            try:
                job()
            except Exception as e:  # reported on wait()
                self._err = e
            finally:
                self._q.task_done()

    def snapshot(self, path, solver, slot, case):
        st = solver.read(slot)
        t = solver.status(slot)["time"]
        pres = pressure(case.phys, st["dens"])
        ids = np.arange(case.n)
        alive = st["alive"] == 1
        self._q.put(lambda: write_ascii(path, t, ids[alive], np.asarray(case.type)[alive], case.mass, st["pos"][alive],
                                        st["vel"][alive], st["dens"][alive], pres[alive]))

    def restart(self, path, solver, slot, desc):
        st = instance_state(solver, slot)
        self._q.put(lambda: write_restart(path, desc, st))

    def wait(self):
        self._q.join()
        if self._err is not None:
            e, self._err = self._err, None
            raise e

    def close(self):
        self.wait()
        self._q.put(None)
        self._t.join()


def pressure(phys, dens):
    """FP64 Tait pressure of the snapshot's pres column (src/EoS.h:80-82)."""
    x = np.asarray(dens, np.float64) / phys.rho0
    return np.maximum(phys.B * (x ** phys.gamma - 1.0), 0.0)

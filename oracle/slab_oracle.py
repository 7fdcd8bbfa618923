"""Host restatement of the slab exchange rules (test infrastructure only).

Restates what csrc/sim_slab.cuh does on the device, on host arrays, so that
the tests can (a) check the device's classification of a slab's particles
bit for bit (FP32 comparisons against the same bounds), and (b) run the
exchange protocol of weaklycompressiblesph_b200/slab.py over gloo on CPU
with a stand-in domain whose "physics" is a plain drift.  The reference's own
decomposition is FDPS's (src/main.cpp:61-62,109-110, FDPS itself not in the
reference tree): there is nothing of it to pin against; the parity of a
decomposed run is checked against the undecomposed run instead.
"""
from __future__ import annotations

import numpy as np

EMIG_L, GHOST_L, EMIG_R, GHOST_R, STAY = 0, 1, 2, 3, 4
RECORD = np.dtype([("pos", "<f4", 4), ("vel", "<f4", 4), ("acc", "<f4", 4), ("id", "<i4"), ("type", "<i4"),
                   ("pad", "<i4", 2)])


def classify(x, slab, W):
    """Class of each owned particle at x (FP32), as k_slab_classify assigns it."""
    x = np.asarray(x, np.float32)
    lo, hi, W = np.float32(slab.x_lo), np.float32(slab.x_hi), np.float32(W)
    c = np.full(len(x), STAY, np.int32)
    hl, hr = bool(slab.has_left), bool(slab.has_right)
    # the device tests in this order; the first match wins
    rules = [(hl, x < lo, EMIG_L), (hr, x >= hi, EMIG_R), (hl, x < np.float32(lo + W), GHOST_L),
             (hr, x >= np.float32(hi - W), GHOST_R)]
    done = np.zeros(len(x), bool)
    for on, m, k in rules:
        if on:
            sel = m & ~done
            c[sel] = k
            done |= sel
    return c


def counts(x, slab, W):
    c = classify(x, slab, W)
    return [int(np.sum(c == k)) for k in range(4)]


class DriftDomain:
    """Stand-in for SlabDomain on host memory: particles drift with constant
    velocity; the next dt is the minimum of a fixed per-particle value over
    the owned particles.  Same pack/unpack interface and record layout."""

    def __init__(self, pos, vel, slabs, rank, W, capacity=None):
        import torch
        self.slab, self.W = slabs[rank], np.float32(W)
        x = np.asarray(pos[:, 0], np.float32)
        m = np.ones(len(x), bool)
        if self.slab.has_left:
            m &= x >= np.float32(self.slab.x_lo)
        if self.slab.has_right:
            m &= x < np.float32(self.slab.x_hi)
        ids = np.nonzero(m)[0]
        self.n_total = len(pos)
        self.rec = np.zeros(len(ids), RECORD)
        self.rec["pos"][:, :3] = np.asarray(pos, np.float32)[ids]
        self.rec["vel"][:, :3] = np.asarray(vel, np.float32)[ids]
        self.rec["id"] = ids
        self.ghost = np.zeros(len(ids), bool)
        self.capacity = int(capacity or len(pos) + 16)
        self.device = torch.device("cpu")
        nbytes = self.capacity * RECORD.itemsize
        self.send = torch.zeros(nbytes, dtype=torch.uint8)
        self.recv = [torch.zeros(nbytes, dtype=torch.uint8) for _ in range(2)]
        self.dt_next = np.float32(np.inf)
        self.time = 0.0
        self.last_counts = None

    @staticmethod
    def dt_of(ids):
        return np.float32(1e-3) * (np.float32(1) + (np.asarray(ids) * 7919 % 1000).astype(np.float32) / 1000)

    def pack(self):
        own = ~self.ghost
        c = np.full(len(self.rec), STAY, np.int32)
        c[own] = classify(self.rec["pos"][own, 0], self.slab, self.W)
        parts = [self.rec[c == k] for k in range(4)]
        buf = np.concatenate(parts)
        self.send[:buf.nbytes] = __import__("torch").from_numpy(buf.view(np.uint8).copy())
        # retire the old ghosts; emigrants stay on as ghosts
        keep = ~self.ghost
        self.ghost = (c == EMIG_L) | (c == EMIG_R)
        self.rec, self.ghost = self.rec[keep], self.ghost[keep]
        self.last_counts = [len(p) for p in parts]
        return self.last_counts

    def unpack(self, buf, n_owned, n_ghost):
        n = n_owned + n_ghost
        r = buf[:n * RECORD.itemsize].numpy().view(RECORD).copy()
        self.rec = np.concatenate([self.rec, r])
        self.ghost = np.concatenate([self.ghost, np.arange(n) >= n_owned])

    def force_pass(self):
        own = ~self.ghost
        self.dt_next = np.float32(self.dt_of(self.rec["id"][own]).min()) if own.any() else np.float32(np.inf)

    def step(self):
        dt = np.float32(self.dt_next)
        self.rec["pos"][:, :3] += dt * self.rec["vel"][:, :3]
        self.time += float(dt)
        self.force_pass()

    def next_dt(self):
        return float(self.dt_next)

    def set_next_dt(self, dt):
        self.dt_next = np.float32(dt)

    def sync(self):
        pass

    def read(self):
        own = ~self.ghost
        out = dict(pos=np.zeros((self.n_total, 3), np.float32), alive=np.zeros(self.n_total, np.int32))
        ids = self.rec["id"][own]
        out["pos"][ids] = self.rec["pos"][own, :3]
        out["alive"][ids] = 1
        return out

    def ghost_ids(self):
        return np.sort(self.rec["id"][self.ghost])

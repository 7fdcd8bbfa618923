"""Slab decomposition of one simulation over several GPUs.

The reference decomposes the domain and exchanges particles through FDPS
every step (src/main.cpp:61-62,109-110).  Here the domain is cut along x into
one slab per rank; each rank's slab is an instance of its own device solver
(``SlabDomain``), which after every step packs its emigrants and a ghost layer
for each x-neighbour (``wcsph_sim_slab_pack``), receives theirs
(``wcsph_sim_slab_unpack``), and agrees with every other rank on the next dt
(minimum over the ranks).  The exchange is between steps: ghosts are kicked
and drifted by the receiver exactly as by their owner, and the layer
(4h + 2 margin wide) also holds the neighbours that the ghosts' own density
passes read.

Transports:

* ``DistRank`` — one slab per process, point-to-point over
  ``torch.distributed`` (NCCL with device buffers; gloo with host buffers for
  CPU tests of the protocol);
* ``LocalGroup`` — several slabs in one process, exchanged by device copies.

Per step and rank: step, pack, counts to both neighbours, records to both
neighbours, unpack what came from the left then what came from the right,
dt = min over ranks.
"""
from __future__ import annotations

import numpy as np

from . import _native as N
from .cases import Case

RECORD = np.dtype([("pos", "<f4", 4), ("vel", "<f4", 4), ("acc", "<f4", 4), ("id", "<i4"), ("type", "<i4"),
                   ("pad", "<i4", 2)])
assert RECORD.itemsize == N.SLAB_RECORD_BYTES


def layer_width(h, margin):
    """Ghost-layer width in FP32, as the library computes it."""
    return float(N.lib().wcsph_slab_layer_width(float(h), float(margin)))


def plan(case: Case, nranks: int, margin_h: float = 0.25):
    """Cut the domain along x into nranks slabs holding equal particle counts
    at the start.  margin (largest drift per step) = margin_h * h.  Returns a
    list of N.Slab."""
    margin = np.float32(margin_h * case.h)
    W = layer_width(case.h, margin)
    x = np.asarray(case.pos[:, 0], np.float32)
    cuts = [np.float32(np.quantile(x, k / nranks)) for k in range(1, nranks)]
    slabs = []
    for r in range(nranks):
        s = N.Slab()
        s.x_lo = cuts[r - 1] if r > 0 else np.float32(case.lo[0])
        s.x_hi = cuts[r] if r < nranks - 1 else np.float32(case.hi[0])
        s.margin = margin
        s.has_left = 1 if r > 0 else 0
        s.has_right = 1 if r < nranks - 1 else 0
        if nranks > 1 and s.x_hi - s.x_lo < 2 * W:
            raise ValueError(f"slab {r} is {s.x_hi - s.x_lo:.4g} wide, less than twice the ghost layer ({W:.4g}); "
                             "use fewer ranks")
        slabs.append(s)
    return slabs


def owned_ids(x, slab):
    """Particles a slab owns: x in [x_lo, x_hi), unbounded on a side without a neighbour."""
    x = np.asarray(x, np.float32)
    m = np.ones(len(x), bool)
    if slab.has_left:
        m &= x >= np.float32(slab.x_lo)
    if slab.has_right:
        m &= x < np.float32(slab.x_hi)
    return np.nonzero(m)[0].astype(np.int32)


class SlabDomain:
    """One rank's slab on one GPU: a solver holding the slab as its only instance."""

    def __init__(self, case: Case, slabs, rank, precision=N.PREC_TILED, device=0, capacity=None,
                 density_mode=None, t_end=None):
        import torch

        from .sim import Solver
        self.case, self.rank, self.slab = case, rank, slabs[rank]
        self.device = torch.device("cuda", device)
        cap = int(capacity or case.n + 1024)
        self.capacity = cap
        self.solver = Solver(cap, precision=precision, device=device, use_graph=False, autotune=False)
        ids = owned_ids(case.pos[:, 0], self.slab)
        self.slot = self.solver.add_slab(case, self.slab, ids, density_mode=density_mode, t_end=t_end)
        nbytes = cap * N.SLAB_RECORD_BYTES
        self.send = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        self.recv = [torch.empty(nbytes, dtype=torch.uint8, device=self.device) for _ in range(2)]

    # -- the interface the transports drive --------------------------------
    def pack(self):
        self.last_counts = self.solver.slab_pack(self.slot, self.send.data_ptr(), self.capacity)
        return self.last_counts

    def unpack(self, buf, n_owned, n_ghost):
        self.solver.slab_unpack(self.slot, buf.data_ptr(), n_owned, n_ghost)

    def step(self):
        self.solver.step(1)

    def force_pass(self):
        self.solver.force_pass(self.slot)

    def next_dt(self):
        return self.solver.next_dt(self.slot)

    def set_next_dt(self, dt):
        self.solver.set_next_dt(self.slot, dt)

    def sync(self):
        import torch
        torch.cuda.synchronize(self.device)

    # -- results -------------------------------------------------------------
    def read(self):
        """Owned particles, as arrays over the whole simulation's ids (alive = owned here)."""
        return self.solver.read(self.slot)

    def status(self):
        return self.solver.status(self.slot)

    def last_pairs(self):
        return self.solver.last_pairs()

    def close(self):
        self.solver.close()


def _route(counts):
    """Split pack counts into (left part: records, n_owned, n_ghost), (right part ...)."""
    el, gl, er, gr = counts
    return (0, el + gl, el, gl), (el + gl, er + gr, er, gr)


class LocalGroup:
    """All slabs in one process; records move by device copies."""

    def __init__(self, domains):
        self.d = list(domains)

    def exchange(self):
        import torch
        parts = []
        for dom in self.d:
            parts.append(_route(dom.pack()))
        inbox = [[None, None] for _ in self.d]  # [from left, from right] = (n_owned, n_ghost)
        for r, dom in enumerate(self.d):
            (ol, nl, eo_l, gh_l), (orr, nr, eo_r, gh_r) = parts[r]
            rec = N.SLAB_RECORD_BYTES
            if r > 0:  # my left part goes to r-1, arriving from its right
                self.d[r - 1].recv[1][:nl * rec].copy_(dom.send[ol * rec:(ol + nl) * rec])
                inbox[r - 1][1] = (eo_l, gh_l)
            if r + 1 < len(self.d):
                self.d[r + 1].recv[0][:nr * rec].copy_(dom.send[orr * rec:(orr + nr) * rec])
                inbox[r + 1][0] = (eo_r, gh_r)
        for dom in self.d:
            dom.sync()
        torch.cuda.synchronize()
        for r, dom in enumerate(self.d):
            for side in (0, 1):
                if inbox[r][side] is not None:
                    dom.unpack(dom.recv[side], *inbox[r][side])

    def reduce_dt(self):
        dt = min(dom.next_dt() for dom in self.d)
        for dom in self.d:
            dom.set_next_dt(dt)
        return dt

    def start(self):
        """First ghost layer, the initial force pass, the common dt, a fresh layer."""
        self.exchange()
        for dom in self.d:
            dom.force_pass()
        self.reduce_dt()
        self.exchange()

    def step(self, nsteps=1):
        for _ in range(nsteps):
            for dom in self.d:
                dom.step()
            self.exchange()
            self.reduce_dt()

    def gather(self):
        """Owned state of every slab merged into whole-simulation arrays."""
        return merge([dom.read() for dom in self.d])


class DistRank:
    """This process's slab, exchanged with its neighbours over torch.distributed."""

    def __init__(self, domain, rank, world, group=None):
        self.dom, self.rank, self.world, self.group = domain, rank, world, group

    def _p2p(self, sends, recvs):
        import torch.distributed as dist
        ops = [dist.P2POp(dist.isend, t, peer, self.group) for t, peer in sends]
        ops += [dist.P2POp(dist.irecv, t, peer, self.group) for t, peer in recvs]
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def exchange(self):
        import torch
        dev = self.dom.send.device
        left, right = _route(self.dom.pack())
        L, R = self.rank - 1, self.rank + 1
        has_l, has_r = L >= 0, R < self.world
        c_out_l = torch.tensor([left[2], left[3]], dtype=torch.int32, device=dev)
        c_out_r = torch.tensor([right[2], right[3]], dtype=torch.int32, device=dev)
        c_in_l = torch.zeros(2, dtype=torch.int32, device=dev)
        c_in_r = torch.zeros(2, dtype=torch.int32, device=dev)
        self._p2p([(c_out_l, L)] * has_l + [(c_out_r, R)] * has_r, [(c_in_l, L)] * has_l + [(c_in_r, R)] * has_r)
        il = [int(v) for v in c_in_l.tolist()] if has_l else [0, 0]
        ir = [int(v) for v in c_in_r.tolist()] if has_r else [0, 0]
        rec = N.SLAB_RECORD_BYTES
        sends, recvs = [], []
        if has_l and left[1]:
            sends.append((self.dom.send[left[0] * rec:(left[0] + left[1]) * rec], L))
        if has_r and right[1]:
            sends.append((self.dom.send[right[0] * rec:(right[0] + right[1]) * rec], R))
        if has_l and sum(il):
            recvs.append((self.dom.recv[0][:sum(il) * rec], L))
        if has_r and sum(ir):
            recvs.append((self.dom.recv[1][:sum(ir) * rec], R))
        self._p2p(sends, recvs)
        self.dom.sync()
        if sum(il):
            self.dom.unpack(self.dom.recv[0], il[0], il[1])
        if sum(ir):
            self.dom.unpack(self.dom.recv[1], ir[0], ir[1])

    def reduce_dt(self):
        import torch
        import torch.distributed as dist
        t = torch.tensor([self.dom.next_dt()], dtype=torch.float32, device=self.dom.send.device)
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
        dt = float(t.item())
        self.dom.set_next_dt(dt)
        return dt

    def start(self):
        self.exchange()
        self.dom.force_pass()
        self.reduce_dt()
        self.exchange()

    def step(self, nsteps=1):
        for _ in range(nsteps):
            self.dom.step()
            self.exchange()
            self.reduce_dt()


def merge(states):
    """Merge per-slab reads (whole-simulation arrays, alive = owned) into one."""
    out = {k: np.zeros_like(v) for k, v in states[0].items()}
    owner = np.zeros(len(states[0]["alive"]), np.int32)
    for st in states:
        m = st["alive"] == 1
        owner += m
        for k, v in st.items():
            out[k][m] = v[m]
    out["owners"] = owner
    return out

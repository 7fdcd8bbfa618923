"""Slab exchange protocol over gloo on CPU (world sizes 2 and 3), with the
host stand-in domain of oracle/slab_oracle.py (plain drift, no forces)."""
import datetime
import os
import socket

import numpy as np
import pytest

from oracle import slab_oracle as SO
from weaklycompressiblesph_b200 import _native as N

W = np.float32(0.06)
STEPS = 12


def particles(n=3000, seed=5):
    rng = np.random.default_rng(seed)
    pos = rng.random((n, 3)).astype(np.float32)
    vel = rng.normal(0.0, 2.0, size=(n, 3)).astype(np.float32)  # drifts 2-10 mm per step, layers are 60 mm
    return pos, vel


def slabs_for(world):
    cuts = [np.float32(k / world) for k in range(world + 1)]
    out = []
    for r in range(world):
        s = N.Slab()
        s.x_lo, s.x_hi, s.margin = cuts[r], cuts[r + 1], np.float32(0.01)
        s.has_left, s.has_right = int(r > 0), int(r < world - 1)
        out.append(s)
    return out


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from weaklycompressiblesph_b200.slab import DistRank
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        pos, vel = particles()
        dom = SO.DriftDomain(pos, vel, slabs_for(world), rank, W)
        r = DistRank(dom, rank, world)
        r.start()
        r.step(STEPS)
        mine = (dom.read(), dom.ghost_ids(), dom.time, dom.next_dt())
        everything = [None] * world
        dist.all_gather_object(everything, mine)
        if rank == 0:
            out.put(everything)
    finally:
        dist.destroy_process_group()


def run_world(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        res = q.get(timeout=120)
    finally:
        for p in procs:
            p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    return res


@pytest.mark.parametrize("world", [2, 3])
def test_slab_protocol_over_gloo(world):
    res = run_world(world)
    pos, vel = particles()
    # undecomposed stand-in over the same steps
    one = SO.DriftDomain(pos, vel, slabs_for(1), 0, W)
    one.force_pass()
    for _ in range(STEPS):
        one.step()
    ref = one.read()
    owners = sum(st["alive"] for st, _, _, _ in res)
    assert np.all(owners == 1), "every particle is owned by exactly one slab"
    got = np.zeros_like(ref["pos"])
    for st, _, _, _ in res:
        m = st["alive"] == 1
        got[m] = st["pos"][m]
    np.testing.assert_array_equal(got, ref["pos"])  # same dt sequence on every rank
    assert len({t for _, _, t, _ in res}) == 1 and abs(res[0][2] - one.time) == 0.0
    # ghosts: exactly the other slabs' particles within W beyond each face
    slabs = slabs_for(world)
    owner = np.zeros(len(pos), np.int32)
    for k, (st, _, _, _) in enumerate(res):
        owner[st["alive"] == 1] = k
    x = got[:, 0]
    for k, (_, ghosts, _, _) in enumerate(res):
        s = slabs[k]
        zone = np.zeros(len(x), bool)
        if s.has_left:
            zone |= (x >= np.float32(s.x_lo - W)) & (x < np.float32(s.x_lo))
        if s.has_right:
            zone |= (x >= np.float32(s.x_hi)) & (x < np.float32(s.x_hi + W))
        expect = np.nonzero(zone & (owner != k))[0]
        np.testing.assert_array_equal(ghosts, expect)

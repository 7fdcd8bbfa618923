"""bench.py's multi-rank plumbing (process group, max/sum over ranks) on CPU
over gloo, world size 2: the timing of an N-GPU run is the maximum over the
ranks and the throughput the sum of their work."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import argparse
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import bench
    w, r, local, pg = bench.dist_setup(argparse.Namespace(decomp="replicas"))
    try:
        bench.barrier(pg)
        ms = bench.max_over_ranks(pg, 1.0 + rank)
        pairs = bench.sum_over_ranks(pg, 10.0 * (rank + 1))
        q.put((r, w, ms, pairs))
    finally:
        bench.finish(pg)


@pytest.mark.parametrize("world", [2])
def test_max_and_sum_over_ranks(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in ps)
    assert [o[0] for o in out] == list(range(world))
    assert all(o[1] == world and o[2] == float(world) and o[3] == 10.0 * world * (world + 1) / 2 for o in out)


def test_clock_summary_keeps_the_timed_region():
    """The clock record summarises only the samples taken between mark_start()
    and mark_stop(), reports every active slowdown reason, and falls back to
    the nearest sample for a region shorter than one sampling period."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    c = bench.ClockSampler(0)
    c.samples = [(1.0, 1200.0, 1965.0, set()), (2.0, 1965.0, 1965.0, {"sw_power_cap"}),
                 (2.2, 1950.0, 1965.0, set()), (3.0, 1965.0, 1965.0, {"hw_slowdown"})]
    c.t0, c.t1 = 1.5, 2.5
    s = c.summary()
    assert s["samples"] == 2 and s["sm_mhz"] == 1957.5 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    c.t0, c.t1 = 2.12, 2.15
    s = c.summary()
    assert s["samples"] == 1 and s["sm_mhz"] == 1950.0

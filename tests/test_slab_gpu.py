"""Slab decomposition on the GPU: R slabs, each its own solver, exchanged by
device copies in one process (LocalGroup), against the undecomposed run."""
import numpy as np
import pytest

from oracle import slab_oracle as SO
from tests.helpers import rel_l2
from weaklycompressiblesph_b200 import _native as N
from weaklycompressiblesph_b200 import cases, slab
from weaklycompressiblesph_b200.sim import Solver

pytestmark = pytest.mark.gpu
STEPS = 40  # crosses the Shepard step 31


def dam(vel_sigma=0.0):
    c = cases.dam_break(dx=0.02)
    if vel_sigma:
        rng = np.random.default_rng(11)
        c.vel = rng.normal(0.0, vel_sigma, size=c.vel.shape)
        c.vel[c.type == N.FREEZE] = 0.0
    return c


def single(case, prec, steps):
    with Solver(case.n, precision=prec) as s:
        k = s.add(case)
        pairs0 = s.last_pairs()
        s.step(steps)
        return s.read(k), s.status(k), pairs0


@pytest.mark.parametrize("nranks", [2, 3])
@pytest.mark.parametrize("prec", [N.PREC_FP32, N.PREC_TILED], ids=["fp32", "tiled"])
def test_slabs_match_single_domain(nranks, prec, native):
    case = dam(vel_sigma=0.5)  # the flow crosses the faces from the first step
    ref, ref_status, ref_pairs0 = single(case, prec, STEPS)
    slabs = slab.plan(case, nranks)
    W = slab.layer_width(case.h, slabs[0].margin)
    doms = [slab.SlabDomain(case, slabs, r, precision=prec) for r in range(nranks)]
    try:
        g = slab.LocalGroup(doms)
        g.start()
        # the initial force pass sees exactly the undecomposed pair set
        assert sum(d.last_pairs() for d in doms) == ref_pairs0
        moved = 0
        for t in range(STEPS):
            for d in doms:
                d.step()
            owned_x = [d.read() for d in doms]
            g.exchange()
            g.reduce_dt()
            for d, st in zip(doms, owned_x):  # device classification == oracle rules, bit for bit
                m = st["alive"] == 1
                assert d.last_counts == SO.counts(st["pos"][m, 0], d.slab, W)
                moved += d.last_counts[0] + d.last_counts[2]
        got = g.gather()
        status = [d.status() for d in doms]
    finally:
        for d in doms:
            d.close()
    assert moved > 0, "no particle crossed a face: the test would not exercise migration"
    alive = ref["alive"] == 1
    np.testing.assert_array_equal(got["owners"], alive.astype(np.int32))
    assert len({s["steps"] for s in status}) == 1 and status[0]["steps"] == ref_status["steps"]
    assert len({s["time"] for s in status}) == 1
    assert abs(status[0]["time"] - ref_status["time"]) <= 1e-5 * ref_status["time"]
    # same physics up to FP32 summation order at the faces
    assert rel_l2(got["pos"][alive], ref["pos"][alive]) < 1e-6
    assert rel_l2(got["vel"][alive], ref["vel"][alive]) < 1e-4
    assert rel_l2(got["dens"][alive], ref["dens"][alive]) < 1e-6
    assert rel_l2(got["acc"][alive], ref["acc"][alive]) < 1e-4


def test_single_slab_is_the_plain_solver(native):
    """One slab with no neighbours is bit-identical to the ordinary solver."""
    case = dam()
    ref, ref_status, _ = single(case, N.PREC_TILED, 10)
    slabs = slab.plan(case, 1)
    d = slab.SlabDomain(case, slabs, 0, precision=N.PREC_TILED)
    try:
        g = slab.LocalGroup([d])
        g.start()
        g.step(10)
        got = g.gather()
        st = d.status()
    finally:
        d.close()
    assert st["steps"] == ref_status["steps"] and st["time"] == ref_status["time"]
    for key in ("pos", "vel", "dens", "acc"):
        np.testing.assert_array_equal(got[key], ref[key])


def test_drift_past_margin_is_reported(native):
    case = dam(vel_sigma=0.5)
    slabs = slab.plan(case, 2, margin_h=1e-6)
    doms = [slab.SlabDomain(case, slabs, r) for r in range(2)]
    try:
        g = slab.LocalGroup(doms)
        g.start()
        for d in doms:
            d.step()
        with pytest.raises(N.WcsphError, match="margin"):
            g.exchange()
    finally:
        for d in doms:
            d.close()


def test_invalid_slabs(native):
    case = dam()
    bad = slab.plan(case, 2)
    bad[0].x_hi = bad[0].x_lo + 0.05  # narrower than two ghost layers
    with Solver(case.n) as s:
        with pytest.raises(N.WcsphError, match="twice the ghost layer"):
            s.add_slab(case, bad[0], np.arange(10, dtype=np.int32))
        with pytest.raises(N.WcsphError, match="outside"):
            s.add_slab(case, slab.plan(case, 2)[0], np.array([-1], dtype=np.int32))
    with pytest.raises(ValueError):
        slab.plan(case, 8)

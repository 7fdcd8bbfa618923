"""Neighbour-list mode of the device solver (list_interval > 0) against the
per-step neighbour search, on the GPU."""
import numpy as np
import pytest

from tests.helpers import rel_l2, small_dam
from weaklycompressiblesph_b200 import _native as N
from weaklycompressiblesph_b200 import cases
from weaklycompressiblesph_b200.sim import Solver

pytestmark = pytest.mark.gpu


def run(case, prec, steps, **kw):
    with Solver(case.n, precision=prec, **kw) as s:
        k = s.add(case)
        s.step(steps)
        out = s.read(k), s.status(k), s.last_pairs()
        stats = s.list_stats() if kw.get("list_interval") else None
    return out + (stats,)


@pytest.mark.parametrize("prec", [N.PREC_TILED, N.PREC_HALF2], ids=["tiled", "half2"])
def test_lists_match_per_step_search(prec, native):
    """60 steps (Shepard steps 1, 31, from the lists when they fall on a list
    step) with lists rebuilt every 8 steps: the same trajectory as the
    per-step search up to FP32 summation order."""
    case = small_dam(dx=0.04, seed=5)
    ref, ref_st, ref_pairs, _ = run(case, prec, 60)
    got, st, pairs, stats = run(case, prec, 60, list_interval=8)
    assert stats["list_steps"] > 0 and stats["overflows"] == 0
    assert stats["builds"] + stats["list_steps"] == 60
    assert stats["builds"] >= 60 // 8 and stats["longest"] <= 192
    assert st["steps"] == ref_st["steps"] == 60
    assert abs(st["time"] - ref_st["time"]) <= 1e-5 * ref_st["time"]
    assert rel_l2(got["pos"], ref["pos"]) < 1e-6
    assert rel_l2(got["vel"], ref["vel"]) < 1e-4
    assert rel_l2(got["dens"], ref["dens"]) < 1e-6
    assert rel_l2(got["acc"], ref["acc"]) < 1e-3
    assert abs(pairs - ref_pairs) <= 1e-3 * ref_pairs


def test_list_step_sums_exactly_the_support(native, oracle_lib):
    """On a step that reads the lists, the pairs summed are exactly the
    in-support pairs of the current positions (the oracle's FP32 predicate)."""
    case = small_dam(dx=0.04, seed=6, vel_sigma=0.5)
    with Solver(case.n, precision=N.PREC_TILED, list_interval=6) as s:
        k = s.add(case)
        s.step(4)  # step 1 builds (the lists are new), steps 2-4 read them
        stats = s.list_stats()
        pairs = s.last_pairs()
        st = s.read(k)
    assert stats["builds"] == 1 and stats["list_steps"] == 3
    cfg = oracle_lib.config_from_case(case)
    alive = st["alive"] == 1
    assert alive.all()
    cnt, tot = oracle_lib.neighbors(oracle_lib.pos4(st["pos"]), cfg)
    assert pairs == tot


def test_lists_periodic_faces(native):
    """Particles cross the periodic faces between builds (wrapping waits for
    the next build); the flow matches the per-step search."""
    case = cases.periodic_lattice(n_side=20, dx=0.01, seed=3,
                                  phys=cases.Physics(g=0.0, density_mode=N.DENSITY_CONTINUITY))
    rng = np.random.default_rng(4)
    case.vel = rng.normal(0.0, 2.0, size=case.vel.shape)
    ref, ref_st, _, _ = run(case, N.PREC_TILED, 40)
    got, st, _, stats = run(case, N.PREC_TILED, 40, list_interval=10, list_skin=0.4)
    assert stats["list_steps"] > 0
    L = np.array(case.hi) - np.array(case.lo)
    d = got["pos"] - ref["pos"]
    d -= L * np.round(d / L)  # compare modulo the box (list steps leave wrapping to the builds)
    assert np.linalg.norm(d) / np.linalg.norm(ref["pos"]) < 1e-6
    assert rel_l2(got["vel"], ref["vel"]) < 1e-4
    assert rel_l2(got["dens"], ref["dens"]) < 1e-6


def test_lists_with_density_passes(native):
    """Summation density every step (the periodic micro-benchmark's mode) runs
    its density passes from the lists: list steps happen and the flow matches
    the per-step search."""
    case = cases.periodic_lattice(n_side=16, dx=0.01, seed=5)
    assert case.phys.density_mode == N.DENSITY_SUMMATION
    ref, ref_st, _, _ = run(case, N.PREC_TILED, 30)
    got, st, _, stats = run(case, N.PREC_TILED, 30, list_interval=10)
    assert stats["list_steps"] > 0 and st["steps"] == 30
    L = np.array(case.hi) - np.array(case.lo)
    d = got["pos"] - ref["pos"]
    d -= L * np.round(d / L)
    assert np.linalg.norm(d) / np.linalg.norm(ref["pos"]) < 1e-6
    assert rel_l2(got["dens"], ref["dens"]) < 1e-6
    assert rel_l2(got["vel"], ref["vel"]) < 1e-4


def test_tiny_skin_builds_every_step(native):
    case = small_dam(dx=0.05, seed=7, vel_sigma=0.5)
    _, st, _, stats = run(case, N.PREC_TILED, 12, list_interval=50, list_skin=1e-6)
    assert stats["builds"] == 12 and stats["list_steps"] == 0 and st["steps"] == 12


def test_lists_with_instance_changes(native):
    a = small_dam(dx=0.05, seed=1)
    b = small_dam(dx=0.04, seed=2, column=(0.3, 0.4, 0.6))
    with Solver(a.n + b.n, max_instances=2, precision=N.PREC_TILED) as s:
        ka = s.add(a)
        s.step(5)
        kb = s.add(b)
        s.step(20)
        ref_a, ref_b = s.read(ka), s.read(kb)
    with Solver(a.n + b.n, max_instances=2, precision=N.PREC_TILED, list_interval=5) as s:
        ka = s.add(a)
        s.step(5)
        kb = s.add(b)  # invalidates the lists: the next step builds
        s.step(20)
        got_a, got_b = s.read(ka), s.read(kb)
        assert s.status(kb)["steps"] == 20 and s.list_stats()["list_steps"] > 0
    for ref, got in ((ref_a, got_a), (ref_b, got_b)):
        assert rel_l2(got["pos"], ref["pos"]) < 1e-6
        assert rel_l2(got["vel"], ref["vel"]) < 1e-4


def test_list_options_rejected(native):
    with pytest.raises(N.WcsphError, match="tiled or half2"):
        Solver(1000, precision=N.PREC_FP32, list_interval=4)
    with pytest.raises(N.WcsphError):
        Solver(1000, precision=N.PREC_TILED, list_interval=-1)


def test_list_overflow_falls_back_to_search(native):
    """h = 2.5 dx gives about 500 neighbours, more than a list holds: every
    build overflows, the next step builds again, and the results are those of
    the per-step search."""
    case = small_dam(dx=0.05, seed=8, phys=cases.Physics(h_over_dx=2.5))
    ref, ref_st, _, _ = run(case, N.PREC_TILED, 6)
    got, st, _, stats = run(case, N.PREC_TILED, 6, list_interval=10)
    assert stats["overflows"] >= 1 and stats["list_steps"] == 0 and stats["builds"] == 6
    assert st["steps"] == ref_st["steps"] == 6
    assert rel_l2(got["pos"], ref["pos"]) < 1e-6
    assert rel_l2(got["vel"], ref["vel"]) < 1e-4

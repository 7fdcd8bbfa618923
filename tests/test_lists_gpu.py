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
    # the half2 list pass rebuilds displacements from 16-bit positions (about
    # 1e-4 relative per pair), the FP32 one only reorders the sums
    h16 = prec == N.PREC_HALF2
    assert abs(st["time"] - ref_st["time"]) <= (1e-4 if h16 else 1e-5) * ref_st["time"]
    assert rel_l2(got["pos"], ref["pos"]) < (1e-5 if h16 else 1e-6)
    assert rel_l2(got["vel"], ref["vel"]) < (1e-3 if h16 else 1e-4)
    assert rel_l2(got["dens"], ref["dens"]) < (1e-5 if h16 else 1e-6)
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


def f32(a):
    return np.asarray(a, np.float32)


def wrap_f32(pos, lo, hi):
    """The device's periodic wrap (one rounded FP32 operation per axis)."""
    p = f32(pos).copy()
    for k in range(3):
        L = np.float32(np.float32(hi[k]) - np.float32(lo[k]))
        top = np.float32(np.float32(lo[k]) + L)
        c = p[:, k]
        hi_m, lo_m = c >= top, c < np.float32(lo[k])
        c[hi_m] = (c[hi_m] - L).astype(np.float32)
        c[lo_m] = (c[lo_m] + L).astype(np.float32)
    return p


def oracle_list_check(oracle_lib, case, st, pr, density_pass, pos=None):
    """The probe's density pass and pair sums against the FP64 oracle on the
    state the probe saw; returns the relative L2 errors and the pair counts."""
    cfg = oracle_lib.config_from_case(case)
    p4 = oracle_lib.pos4(f32(st["pos"] if pos is None else pos))
    v4 = oracle_lib.pos4(f32(st["vel"]))
    out = {}
    if density_pass:
        ref = oracle_lib.density(p4, f32(st["dens"]), cfg, density_pass == 2)
        out["dens"] = rel_l2(pr["dens"], ref)
        dens = f32(pr["dens"])  # the hydro pass is checked on the densities it used
    else:
        dens = f32(st["dens"])
        np.testing.assert_array_equal(pr["dens"], dens)
    pres, snds = oracle_lib.eos(dens.astype(np.float64), case.phys.gamma, case.phys.rho0, case.phys.c0)
    acc, dv, dt = oracle_lib.hydro(p4, v4, dens, f32(pres), f32(snds), cfg)
    cnt, tot = oracle_lib.neighbors(p4, cfg)
    out.update(acc=rel_l2(pr["acc"], acc), div_v=rel_l2(pr["div_v"], dv), dt=rel_l2(pr["dt"], dt),
               cnt=cnt, tot=tot)
    return out


LIST_TOL = {N.PREC_TILED: 1e-5, N.PREC_HALF2: 1e-3}


@pytest.mark.parametrize("density_pass", [0, 1, 2], ids=["none", "summation", "shepard"])
@pytest.mark.parametrize("prec", [N.PREC_TILED, N.PREC_HALF2], ids=["tiled", "half2"])
def test_list_pass_vs_fp64(prec, density_pass, native, oracle_lib):
    """The passes a list step runs (k_density_list, k_hydro_list) on a list
    step after several steps of drift, against the FP64 oracle on the same
    state: force.h:31-60 pair sums and force.h:12-29 density sums, with the
    in-support test (0 < r^2 < (2h)^2 in FP32) giving the oracle's counts."""
    case = small_dam(dx=0.04, seed=11, vel_sigma=0.4)
    with Solver(case.n, precision=prec, list_interval=50, list_skin=0.6) as s:
        k = s.add(case)
        s.step(10)
        before = s.list_stats()
        st = s.read(k)
        pr = s.probe(k, density_pass=density_pass, lists=True)
        after = s.list_stats()
        s.step(2)  # the lists stay usable after a probe
        assert s.status(k)["steps"] == 12
    assert before["builds"] >= 1 and before["list_steps"] >= 5
    assert after["builds"] == before["builds"]  # the probe read the existing lists
    assert (st["alive"] == 1).all()
    r = oracle_list_check(oracle_lib, case, st, pr, density_pass)
    tol = LIST_TOL[prec]
    np.testing.assert_array_equal(pr["nbr"], r["cnt"])
    assert r["acc"] < tol and r["div_v"] < tol and r["dt"] < tol, r
    if density_pass:
        assert r["dens"] < 1e-5, r


@pytest.mark.parametrize("shape", range(N.LIST_SHAPES))
@pytest.mark.parametrize("prec", [N.PREC_TILED, N.PREC_HALF2], ids=["tiled", "half2"])
def test_list_pass_every_shape_vs_fp64(prec, shape, native, oracle_lib):
    """Every launch shape of the list pass (threads per particle, blocks per
    SM, lanes on consecutive or alternate entries), fixed instead of chosen
    by the autotuner: after a build and list steps, the list pass on the
    state read back against the FP64 oracle, with the oracle's neighbour
    counts; and the shape is the one the solver reports."""
    case = small_dam(dx=0.04, seed=31, vel_sigma=0.4)
    with Solver(case.n, precision=prec, list_interval=50, list_skin=0.6, list_shape=shape) as s:
        k = s.add(case)
        s.step(6)
        st = s.read(k)
        pr = s.probe(k, density_pass=2, lists=True)
        assert s.tuning()["list_shape"] == shape
        assert s.list_stats()["list_steps"] >= 3
    r = oracle_list_check(oracle_lib, case, st, pr, 2)
    tol = LIST_TOL[prec]
    np.testing.assert_array_equal(pr["nbr"], r["cnt"])
    assert r["acc"] < tol and r["div_v"] < tol and r["dt"] < tol and r["dens"] < 1e-5, r


@pytest.mark.parametrize("prec", [N.PREC_TILED, N.PREC_HALF2], ids=["tiled", "half2"])
def test_every_build_shape_builds_the_same_lists(prec, native, oracle_lib):
    """Every shape of the list build's scan (the tiled scan's block and tile
    shapes, and the lane-per-particle scan) writes the same entries in the
    same order: after builds and list steps the states are bit-identical,
    and the list pass on them matches the FP64 oracle."""
    case = small_dam(dx=0.04, seed=33, vel_sigma=0.4)
    states, probes, entries = [], [], []
    for b in range(N.BUILD_SHAPES):
        with Solver(case.n, precision=prec, list_interval=4, list_shape=0, build_shape=b) as s:
            k = s.add(case)
            s.step(9)  # builds at steps 1, 5, 9 at least
            assert s.tuning()["build_shape"] == b
            assert s.list_stats()["builds"] >= 3
            states.append(s.read(k))
            probes.append(s.probe(k, lists=True))
            entries.append(s.list_entries())
    for st, pr, ne in zip(states[1:], probes[1:], entries[1:]):
        assert ne == entries[0]
        for key in ("pos", "vel", "dens", "acc"):
            np.testing.assert_array_equal(st[key], states[0][key])
        for key in ("acc", "div_v", "nbr"):
            np.testing.assert_array_equal(pr[key], probes[0][key])
    r = oracle_list_check(oracle_lib, case, states[0], probes[0], 0)
    np.testing.assert_array_equal(probes[0]["nbr"], r["cnt"])
    assert r["acc"] < LIST_TOL[prec] and r["div_v"] < LIST_TOL[prec], r


@pytest.mark.parametrize("prec", [N.PREC_TILED, N.PREC_HALF2], ids=["tiled", "half2"])
def test_list_pass_periodic_vs_fp64(prec, native, oracle_lib):
    """Config-3 mode (periodic box, summation density every step) through the
    lists: particles run past the faces between builds (wrapping waits for the
    next build); the oracle sees the wrapped positions."""
    case = cases.periodic_lattice(n_side=20, dx=0.01, seed=21)
    rng = np.random.default_rng(22)
    case.vel = rng.normal(0.0, 0.1, size=case.vel.shape)
    # shift the lattice so that a layer sits just inside the +x face, and send
    # it outward: it crosses the face on the list steps after the first build
    side = case.hi[0] - case.lo[0]
    case.pos[:, 0] = np.mod(case.pos[:, 0] + 0.0048, side)
    case.vel[case.pos[:, 0] > side - 0.0006, 0] = 3.0
    # the default skin: 2.3 h holds about 110 lattice neighbours (a list holds 192)
    with Solver(case.n, precision=prec, list_interval=50) as s:
        k = s.add(case)
        s.step(3)
        st = s.read(k)
        pr = s.probe(k, density_pass=1, lists=True)
        stats = s.list_stats()
    assert stats["list_steps"] >= 2 and stats["overflows"] == 0
    wrapped = wrap_f32(st["pos"], case.lo, case.hi)
    assert np.any(wrapped != f32(st["pos"]))  # some particles crossed a face since the build
    r = oracle_list_check(oracle_lib, case, st, pr, 1, pos=wrapped)
    # unwrapped vs wrapped coordinates round differently in the last bit, which
    # can flip the support test of a pair at r = 2h exactly; none expected here
    assert abs(int(pr["nbr"].sum()) - int(r["tot"])) <= 2
    tol = LIST_TOL[prec]
    assert r["dens"] < 1e-5 and r["acc"] < tol and r["div_v"] < tol, r


def test_probe_lists_builds_when_stale(native, oracle_lib):
    """Without current lists (right after the instance was added) the probe
    builds them, and the steps that follow read them."""
    case = small_dam(dx=0.05, seed=12, vel_sigma=0.2)
    # autotune off: the tuner's probe pass re-sorts, which would drop the lists
    with Solver(case.n, precision=N.PREC_TILED, list_interval=20, autotune=False) as s:
        k = s.add(case)
        pr = s.probe(k, lists=True)
        st = s.read(k)
        s.step(3)
        stats = s.list_stats()
    assert stats["builds"] == 0 and stats["list_steps"] == 3
    r = oracle_list_check(oracle_lib, case, st, pr, 0)
    np.testing.assert_array_equal(pr["nbr"], r["cnt"])
    assert r["acc"] < 1e-5 and r["div_v"] < 1e-5


def test_probe_lists_needs_lists(native):
    case = small_dam(dx=0.05)
    with Solver(case.n, precision=N.PREC_TILED) as s:
        k = s.add(case)
        with pytest.raises(N.WcsphError, match="no neighbour lists"):
            s.probe(k, lists=True)


def test_half2_list_options(native):
    with pytest.raises(N.WcsphError, match="list_skin"):
        Solver(1000, precision=N.PREC_HALF2, list_interval=4, list_skin=2.0)


def test_half2_lists_far_particles(native, oracle_lib):
    """Particles thrown above the cell grid (whose top cells are clamped) are
    more than a cell edge from their build cell's centre: the half2 list pass
    reads them from the FP32 records, and the sums stay the oracle's."""
    case = small_dam(dx=0.05, seed=14, vel_sigma=0.1)
    fluid = np.nonzero(case.type == N.HYDRO)[0]
    top = fluid[np.argsort(-case.pos[fluid, 2], kind="stable")[:40]]
    case.pos[top, 2] += (case.hi[2] - case.pos[top, 2]) + 0.3  # two cells above the grid, inside the kill box
    with Solver(case.n, precision=N.PREC_HALF2, list_interval=20) as s:
        k = s.add(case, density_mode=N.DENSITY_CONTINUITY)
        s.step(3)
        st = s.read(k)
        pr = s.probe(k, lists=True)
    assert (st["alive"] == 1).all()
    assert (st["pos"][top, 2] > case.hi[2]).all()
    r = oracle_list_check(oracle_lib, case, st, pr, 0)
    np.testing.assert_array_equal(pr["nbr"], r["cnt"])
    assert r["acc"] < 1e-3 and r["div_v"] < 1e-3, r


def test_profile_split_follows_the_schedule(native):
    """wcsph_sim_profile_split: steps split into builds and list steps as the
    device decided them; a build's scan is part of its hydro phase; the
    steps advance the run like wcsph_sim_step."""
    case = small_dam(dx=0.04, seed=8)
    with Solver(case.n, precision=N.PREC_TILED, list_interval=5) as s:
        k = s.add(case)
        s.step(3)
        s.synchronize()
        s.invalidate_lists()
        l0 = s.list_stats()
        sp = s.profile_split(12)
        l1 = s.list_stats()
        assert s.status(k)["steps"] == 15
    assert sp["build_steps"] + sp["list_steps"] == 12
    assert sp["build_steps"] == l1["builds"] - l0["builds"] >= 3  # the invalidated step, then every 5 steps
    assert sp["list_steps"] == l1["list_steps"] - l0["list_steps"] > 0
    for kind in ("build", "list"):
        ph = sp[kind]
        assert (ph[:3] >= 0).all() and ph[2] > 0 and abs(ph[3] - ph[:3].sum()) < 1e-6 * max(1.0, ph[3])
    assert 0 < sp["scan_ms"] < sp["build"][2]
    with Solver(case.n, precision=N.PREC_TILED) as s:  # searching every step: all steps are of the first kind
        s.add(case)
        sp = s.profile_split(4)
    assert sp["build_steps"] == 4 and sp["list_steps"] == 0 and sp["scan_ms"] == 0.0


def calm_and_fast():
    """A dam break at rest beside a periodic lattice whose particles move at
    metres per second: the lattice needs new lists every few steps, the dam
    break none within the run, so most builds are partial."""
    calm = small_dam(dx=0.04, seed=9, vel_sigma=0.0)
    fast = cases.periodic_lattice(n_side=12, dx=0.01, seed=3,
                                  phys=cases.Physics(g=0.0, density_mode=N.DENSITY_CONTINUITY))
    fast.vel = np.random.default_rng(4).normal(0.0, 2.0, size=fast.vel.shape)
    return calm, fast


def run_pair(calm, fast, steps, list_interval, probe=False):
    with Solver(calm.n + fast.n, precision=N.PREC_TILED, list_interval=list_interval) as s:
        kc, kf = s.add(calm), s.add(fast)
        s.step(steps)
        states = [s.read(kc), s.read(kf)]
        sched = s.list_schedule() if list_interval else None
        probes = [s.probe(k, lists=True) for k in (kc, kf)] if probe else None
    return states, sched, probes


def periodic_rel(got, ref, case):
    L = np.array(case.hi) - np.array(case.lo)
    d = got - ref
    d -= L * np.round(d / L)
    return np.linalg.norm(d) / np.linalg.norm(ref)


def test_partial_builds_keep_calm_instances(native, oracle_lib):
    """Partial builds: only the instance whose particles could reach half the
    skin is re-sorted and gets new lists; the other keeps its lists, cells
    and slots.  The list passes of both match the FP64 oracle, and both
    trajectories match the per-step search."""
    calm, fast = calm_and_fast()
    ref, _, _ = run_pair(calm, fast, 40, 0)
    got, sched, probes = run_pair(calm, fast, 40, 30, probe=True)
    assert sched["partial_builds"] >= 5 and sched["builds"] >= sched["partial_builds"] + 1
    assert sched["builds"] + sched["list_steps"] == 40
    for case, st, pr in zip((calm, fast), got, probes):
        r = oracle_list_check(oracle_lib, case, st, pr, 0)
        np.testing.assert_array_equal(pr["nbr"], r["cnt"])
        assert r["acc"] < 1e-5 and r["div_v"] < 1e-5, r
    assert rel_l2(got[0]["pos"], ref[0]["pos"]) < 1e-6
    assert periodic_rel(got[1]["pos"], ref[1]["pos"], fast) < 1e-6
    for a, b in zip(got, ref):
        assert rel_l2(a["vel"], b["vel"]) < 1e-4
        assert rel_l2(a["dens"], b["dens"]) < 1e-6


def test_removal_during_partial_builds(native):
    """Particles leaving the kill box while the other instance forces partial
    builds stay in place, marked dead, until the next build compacts them in
    full; the survivors' trajectories match the per-step search."""
    calm, fast = calm_and_fast()
    fluid = np.nonzero(calm.type == N.HYDRO)[0]
    fluid = fluid[np.argsort(-calm.pos[fluid, 2], kind="stable")]  # top surface first
    calm.vel[fluid[:5]] = [0.0, 0.0, 200.0]
    calm.kill_hi = (calm.kill_hi[0], calm.kill_hi[1], 1.2)
    ref, _, _ = run_pair(calm, fast, 40, 0)
    got, sched, _ = run_pair(calm, fast, 40, 30)
    assert sched["partial_builds"] >= 5
    assert np.all(got[0]["alive"][fluid[:5]] == 0) and got[0]["alive"].sum() == calm.n - 5
    assert np.array_equal(got[0]["alive"], ref[0]["alive"])
    alive = got[0]["alive"] == 1
    assert rel_l2(got[0]["pos"][alive], ref[0]["pos"][alive]) < 1e-6
    assert rel_l2(got[0]["vel"][alive], ref[0]["vel"][alive]) < 1e-4
    assert periodic_rel(got[1]["pos"], ref[1]["pos"], fast) < 1e-6


def test_list_build_reaches_the_list_radius(native, oracle_lib):
    """A pair whose separation along one axis lies between 2h and the list
    radius 2h + skin must be in the lists: two particles 2.2h apart along x,
    placed so that they fall in cells two apart when cells are only 2h wide,
    close in head-on without a rebuild and must be summed once within 2h."""
    phys = cases.Physics(g=0.0, density_mode=N.DENSITY_CONTINUITY)
    dx = 0.01
    h = phys.h_over_dx * dx
    lo, hi = (0.0, 0.0, 0.0), (0.2605, 0.1, 0.1)  # 10 cells of 2.0038 h along x when cells are 2h
    x1 = 0.95 * 0.02605
    pos = np.array([[x1, 0.05, 0.05], [x1 + 2.2 * h, 0.05, 0.05]])
    vel = np.array([[0.5, 0.0, 0.0], [-0.5, 0.0, 0.0]])
    case = cases.Case(name="pair", pos=pos, vel=vel, dens=np.full(2, phys.rho0), type=np.zeros(2, np.int32),
                      dx=dx, h=h, mass=phys.rho0 * dx ** 3, phys=phys, lo=lo, hi=hi)
    cfg = oracle_lib.config_from_case(case)
    with Solver(64, precision=N.PREC_TILED, list_interval=1000) as s:
        k = s.add(case)
        met = False
        for _ in range(40):
            s.step(1)
            st = s.read(k)
            cnt, _ = oracle_lib.neighbors(oracle_lib.pos4(st["pos"].astype(np.float32)), cfg)
            if cnt.sum() == 2:
                met = True
                break
        sched = s.list_schedule()
        pr = s.probe(k, lists=True)
    assert met, "the particles never came within 2h"
    assert sched["builds"] == 1, sched  # the lists of the first step were read throughout
    np.testing.assert_array_equal(pr["nbr"], cnt)

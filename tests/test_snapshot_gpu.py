"""Exact restart of device-resident instances, and snapshot output, on the GPU."""
import numpy as np
import pytest

from tests.helpers import small_dam
from weaklycompressiblesph_b200 import cases, snapshot
from weaklycompressiblesph_b200 import _native as N
from weaklycompressiblesph_b200.sim import Solver

pytestmark = pytest.mark.gpu
STATE = ("pos", "vel", "dens", "acc", "div_v", "alive")


def escapee_dam():
    """Shepard density (filter every 30 steps) and five particles that leave
    the kill box before the save, so the restart carries dead particles."""
    case = small_dam(dx=0.05, seed=4)
    fluid = np.nonzero(case.type == N.HYDRO)[0]
    fluid = fluid[np.argsort(-case.pos[fluid, 2], kind="stable")]
    case.vel[fluid[:5]] = [0.0, 0.0, 200.0]
    case.kill_hi = (case.kill_hi[0], case.kill_hi[1], 1.2)
    return case


@pytest.mark.parametrize("prec", [N.PREC_FP32, N.PREC_TILED, N.PREC_HALF2], ids=["fp32", "tiled", "half2"])
def test_restart_continues_bit_identical(prec, native, tmp_path):
    case = escapee_dam()
    other = cases.periodic_lattice(n_side=14, dx=0.01, seed=9)
    n_save, n_more = 35, 30  # the Shepard filter runs at step 31 and again at 61
    with Solver(case.n, precision=prec) as s:
        k = s.add(case)
        s.step(n_save)
        saved = snapshot.instance_state(s, k)
        d = case.desc()
        path = snapshot.restart_name(str(tmp_path), 0)
        snapshot.write_restart(path, d, saved)
        s.step(n_more)
        ref = s.read(k)
        ref_status = s.status(k)
    assert saved["alive"].sum() == case.n - 5
    desc, st = snapshot.read_restart(path)
    # into a fresh solver that already holds another instance
    with Solver(case.n + other.n, max_instances=2, precision=prec) as s:
        ko = s.add(other)
        s.step(3)
        k = s.restore(None, st, desc)
        assert s.status(k)["steps"] == n_save and s.status(k)["n_alive"] == case.n - 5
        back = s.read(k)
        for key in STATE:
            np.testing.assert_array_equal(back[key], saved[key])
        s.step(n_more)
        got = s.read(k)
        got_status = s.status(k)
        assert s.status(ko)["steps"] == 3 + n_more
    assert got_status == ref_status
    for key in STATE:
        np.testing.assert_array_equal(got[key], ref[key], err_msg=key)


def test_restore_rejects_bad_order(native):
    case = small_dam(dx=0.05)
    with Solver(case.n) as s:
        k = s.add(case)
        s.step(2)
        st = snapshot.instance_state(s, k)
        st["order"] = st["order"].copy()
        st["order"][0] = st["order"][1]
        with pytest.raises(N.WcsphError, match="permutation"):
            s.restore(case, st)
        st["order"] = None
        st["dt_next"] = 0.0
        with pytest.raises(N.WcsphError):
            s.restore(case, st)


def test_snapshot_writer(native, tmp_path):
    case = escapee_dam()
    sched = snapshot.OutputSchedule(end_time=4e-3, count=4)
    w = snapshot.SnapshotWriter()
    written = []
    with Solver(case.n) as s:
        k = s.add(case)
        for _ in range(80):
            idx = sched.due(s.status(k)["time"])
            if idx is not None:
                p = snapshot.ascii_name(str(tmp_path), idx)
                w.snapshot(p, s, k, case)
                written.append((p, s.read(k), s.status(k)["time"]))
            s.step(1)
        w.close()
    assert len(written) >= 3
    for p, st, t in written:
        r = snapshot.read_ascii(p)
        alive = st["alive"] == 1
        assert r["n"] == alive.sum() and r["time"] == float("%e" % t)
        np.testing.assert_array_equal(r["id"], np.nonzero(alive)[0])
        np.testing.assert_array_equal(r["pos"].astype(np.float32), st["pos"][alive])
        np.testing.assert_array_equal(r["dens"].astype(np.float32), st["dens"][alive])

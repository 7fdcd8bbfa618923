"""Snapshot and restart formats on the host (no GPU)."""
import numpy as np
import pytest

from weaklycompressiblesph_b200 import cases, snapshot
from weaklycompressiblesph_b200 import _native as N


def fake_state(n, seed=0):
    rng = np.random.default_rng(seed)
    return dict(pos=rng.random((n, 3), dtype=np.float32), vel=rng.normal(size=(n, 3)).astype(np.float32),
                dens=(1000 + rng.random(n)).astype(np.float32), acc=rng.normal(size=(n, 3)).astype(np.float32),
                div_v=rng.normal(size=n).astype(np.float32), alive=(rng.random(n) > 0.1).astype(np.int32),
                type=(rng.random(n) > 0.7).astype(np.int32), order=rng.permutation(n).astype(np.int32),
                time=0.123456789, steps=4321, dt_next=np.float32(3.25e-5))


def test_ascii_columns_round_trip(tmp_path):
    c = cases.dam_break(dx=0.1)
    st = fake_state(c.n)
    pres = snapshot.pressure(c.phys, st["dens"])
    path = snapshot.ascii_name(str(tmp_path), 7)
    assert path.endswith("00007_00001_00000.dat")
    ids = np.arange(c.n)
    snapshot.write_ascii(path, 0.5, ids, c.type, c.mass, st["pos"], st["vel"], st["dens"], pres)
    lines = open(path).read().splitlines()
    assert lines[0] == "%e" % 0.5 and lines[1] == str(c.n)
    assert len(lines[2].split("\t")) == 12  # id tag mass x y z vx vy vz dens 0.0 pres
    r = snapshot.read_ascii(path)
    assert r["n"] == c.n and r["time"] == 0.5
    np.testing.assert_array_equal(r["id"], ids)
    np.testing.assert_array_equal(r["tag"], c.type)
    # %.16f of an FP32 value converts back to the same FP32 value
    np.testing.assert_array_equal(r["pos"].astype(np.float32), st["pos"])
    np.testing.assert_array_equal(r["vel"].astype(np.float32), st["vel"])
    np.testing.assert_array_equal(r["dens"].astype(np.float32), st["dens"])
    np.testing.assert_allclose(r["pres"], pres, rtol=1e-12)


def test_restart_round_trip(tmp_path):
    c = cases.dam_break(dx=0.1)
    d = c.desc(density_mode=N.DENSITY_SHEPARD, t_end=1.5)
    st = fake_state(c.n, seed=3)
    path = snapshot.restart_name(str(tmp_path), 23)
    assert path == snapshot.restart_name(str(tmp_path), 3)  # one naming rule for writer and reader
    snapshot.write_restart(path, d, st)
    d2, st2 = snapshot.read_restart(path)
    assert bytes(d2) == bytes(d)
    for k in ("time", "steps"):
        assert st2[k] == st[k]
    assert np.float32(st2["dt_next"]) == st["dt_next"]
    for k in ("pos", "vel", "dens", "acc", "div_v", "alive", "type", "order"):
        np.testing.assert_array_equal(st2[k], st[k])


def test_restart_rejects_bad_files(tmp_path):
    c = cases.dam_break(dx=0.1)
    st = fake_state(c.n)
    path = str(tmp_path / "r.bin")
    snapshot.write_restart(path, c.desc(), st)
    raw = open(path, "rb").read()
    open(path, "wb").write(raw[:-5])
    with pytest.raises(ValueError, match="truncated"):
        snapshot.read_restart(path)
    open(path, "wb").write(b"XXXXXXXX" + raw[8:])
    with pytest.raises(ValueError, match="not a wcsph restart"):
        snapshot.read_restart(path)
    st["dens"] = st["dens"][:-1]
    with pytest.raises(ValueError):
        snapshot.write_restart(path, c.desc(), st)


def test_output_schedule():
    """src/io.h:6,34: write when time >= next, next += end_time / count."""
    s = snapshot.OutputSchedule(end_time=1.0, count=10)
    got = [(t, s.due(t)) for t in (0.0, 0.05, 0.1, 0.12, 0.35, 0.36)]
    assert got == [(0.0, 0), (0.05, None), (0.1, 1), (0.12, None), (0.35, 2), (0.36, 3)]

"""Pin the oracle (oracle/wcsph_oracle.c) against the reference's own compiled
CPU functors (oracle/_ref, built from src/force.h, kernel.h, EoS.h, class.h,
integral.h) and against the committed golden vectors."""
import os

import numpy as np
import pytest

from tests.helpers import rel_l2, small_dam, walk_setup
from weaklycompressiblesph_b200 import fdps
from weaklycompressiblesph_b200 import _native as N

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def need_ref(oracle_lib):
    if not oracle_lib.ref_available():
        pytest.skip("oracle/_ref not built (reference sources absent)")


def test_layouts_match_reference(oracle_lib, native):
    need_ref(oracle_lib)
    import ctypes as C
    buf = (C.c_long * 64)()
    n = oracle_lib.ref().ref_layout(buf, 64)
    v = list(buf[:n])
    epi, epj, res = fdps.EPI_HYDRO, fdps.EPJ_HYDRO, fdps.RESULT_HYDRO
    want = [epi.itemsize] + [epi.fields[f][1] for f in ("pos", "vel", "smth", "dens", "pres", "snds", "visc", "tag")]
    want += [epj.itemsize] + [epj.fields[f][1] for f in ("pos", "vel", "dens", "mass", "smth", "pres", "snds", "visc",
                                                         "tag", "type")]
    want += [res.itemsize] + [res.fields[f][1] for f in ("acc", "dt", "div_v")]
    want += [fdps.EPI_FILTER.itemsize, 0, 24, fdps.EPJ_FILTER.itemsize, 0, 24, 32, fdps.RESULT_FILTER.itemsize, 0]
    assert v == want
    lay = fdps.default_layout()
    c_abi = [lay.epi_size, lay.epi_pos, lay.epi_vel, lay.epi_smth, lay.epi_dens, lay.epi_pres, lay.epi_snds,
             lay.epi_visc, lay.epj_size, lay.epj_pos, lay.epj_vel, lay.epj_dens, lay.epj_mass, lay.epj_smth,
             lay.epj_pres, lay.epj_snds, lay.epj_visc, lay.res_size, lay.res_acc, lay.res_dt, lay.res_div_v]
    ref_no_tag = v[0:8] + v[9:18] + v[20:24]
    assert c_abi == ref_no_tag


def test_kernel_function(oracle_lib):
    need_ref(oracle_lib)
    import ctypes as C
    rng = np.random.default_rng(1)
    R = oracle_lib.ref()
    O = oracle_lib.orc()
    for _ in range(200):
        h = rng.uniform(0.005, 0.05)
        d = rng.normal(size=3)
        d *= rng.uniform(0.01, 2.2) * h / np.linalg.norm(d)
        r = np.linalg.norm(d)
        assert O.orc_W(r, h) == pytest.approx(R.ref_W(*d, h), rel=1e-12, abs=1e-300)
        g = (C.c_double * 3)()
        R.ref_gradW(*d, h, g)
        gs = O.orc_gradW_scalar(r, h)
        np.testing.assert_allclose(gs * d, np.array(g[:]), rtol=1e-11, atol=1e-300)


def test_eos(oracle_lib):
    need_ref(oracle_lib)
    import ctypes as C
    rng = np.random.default_rng(2)
    dens = rng.uniform(900.0, 1100.0, 1000)
    p1, c1 = oracle_lib.eos(dens, 7.0, 1000.0, 28.01)
    p2 = np.zeros_like(dens)
    c2 = np.zeros_like(dens)
    f = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    oracle_lib.ref().ref_pressure(len(dens), f(dens), f(p2), f(c2), 7.0, 1000.0, 28.01)
    np.testing.assert_allclose(p1, p2, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(c1, c2, rtol=1e-12)
    assert np.all(p1[dens < 1000.0] == 0.0)  # no tension (EoS.h:82)


@pytest.mark.parametrize("periodic", [False, True])
def test_hydro_walks_cpu_semantics(oracle_lib, periodic):
    """orc_hydro_walks with the force.h parameters == CalcHydroForce over the same walks."""
    need_ref(oracle_lib)
    if periodic:
        from weaklycompressiblesph_b200 import cases
        case = cases.periodic_lattice(n_side=14, dx=0.01, seed=5)
    else:
        case = small_dam(dx=0.05)
    w, epi, epj = walk_setup(case, group_size=64)
    ref = oracle_lib.ref_hydro_walks(w.i_off, epi, w.j_off, epj)
    pp = oracle_lib.PairParams(0.01, 0.0, 0.3, 0.01, oracle_lib.VSIG_REF_CPU, oracle_lib.GRAD_HBAR)
    got = oracle_lib.hydro_walks(w.i_off, epi, w.j_off, epj, pp)
    assert rel_l2(got["acc"], ref["acc"]) < 1e-10
    assert rel_l2(got["div_v"], ref["div_v"]) < 1e-10
    np.testing.assert_allclose(got["dt"], ref["dt"], rtol=1e-12)


def test_filter_walks(oracle_lib):
    need_ref(oracle_lib)
    case = small_dam(dx=0.05)
    pres_w, epi, epj = walk_setup(case, group_size=64)
    w = pres_w
    epi_f = np.zeros(len(epi), fdps.EPI_FILTER)
    epi_f["pos"], epi_f["smth"] = epi["pos"], epi["smth"]
    epj_f = np.zeros(len(epj), fdps.EPJ_FILTER)
    epj_f["pos"], epj_f["dens"], epj_f["mass"] = epj["pos"], epj["dens"], epj["mass"]
    ref = oracle_lib.ref_filter_walks(w.i_off, epi_f, w.j_off, epj_f)
    got = oracle_lib.filter_walks(w.i_off, epi_f, w.j_off, epj_f)
    np.testing.assert_allclose(got, ref, rtol=1e-12)


def test_timestep(oracle_lib):
    need_ref(oracle_lib)
    import ctypes as C
    rng = np.random.default_rng(3)
    n = 500
    smth = np.full(n, 0.026)
    acc = rng.normal(0, 20, size=(n, 3))
    dt = rng.uniform(1e-4, 1e-3, n)
    typ = (rng.uniform(size=n) < 0.3).astype(np.int32)
    f = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    ref = oracle_lib.ref().ref_timestep(n, f(smth), f(acc), f(dt), typ.ctypes.data_as(C.POINTER(C.c_int32)), 1e-6)
    got = oracle_lib.orc().orc_dt_global(n, f(acc), f(dt), typ.ctypes.data_as(C.POINTER(C.c_int32)), 0.026, 1e-6)
    assert got == pytest.approx(ref, rel=1e-14)


def _ref_step(oracle_lib, case, st, step_index, filter_every):
    """One loop iteration of src/main.cpp:89-133 composed from the reference's
    own pieces (all-pairs walks, i.e. an exact superset j-list)."""
    import ctypes as C
    R = oracle_lib.ref()
    n = case.n
    f = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    typ = np.ascontiguousarray(case.type, np.int32)
    ti = typ.ctypes.data_as(C.POINTER(C.c_int32))
    smth = np.full(n, case.h)
    dt = R.ref_timestep(n, f(smth), f(st["acc"]), f(st["dt_i"]), ti, case.phys.nu)
    R.ref_kdk_first(n, f(st["pos"]), f(st["vel"]), f(st["vel_half"]), f(st["acc"]), f(st["dens"]), f(st["div_v"]), ti, dt)
    one = np.array([0, n], np.int32)
    if filter_every and step_index % filter_every == 0:
        epi_f = np.zeros(n, fdps.EPI_FILTER)
        epi_f["pos"], epi_f["smth"] = st["pos"], case.h
        epj_f = np.zeros(n, fdps.EPJ_FILTER)
        epj_f["pos"], epj_f["dens"], epj_f["mass"] = st["pos"], st["dens"], case.mass
        st["dens"][:] = oracle_lib.ref_filter_walks(one, epi_f, one, epj_f)
    pres = np.zeros(n)
    snds = np.zeros(n)
    p = case.phys
    R.ref_pressure(n, f(st["dens"]), f(pres), f(snds), p.gamma, p.rho0, p.c0)
    epi = np.zeros(n, fdps.EPI_HYDRO)
    epj = np.zeros(n, fdps.EPJ_HYDRO)
    for e in (epi, epj):
        e["pos"], e["vel"], e["smth"], e["dens"] = st["pos"], st["vel"], case.h, st["dens"]
        e["pres"], e["snds"], e["visc"] = pres, snds, p.nu
    epj["mass"] = case.mass
    out = oracle_lib.ref_hydro_walks(one, epi, one, epj)
    st["acc"][:] = out["acc"]
    st["acc"][:, 2] -= p.g
    st["div_v"][:] = out["div_v"]
    st["dt_i"][:] = out["dt"]
    R.ref_kdk_final(n, f(st["vel"]), f(st["vel_half"]), f(st["acc"]), ti, dt)
    st["dens"][:] = np.maximum(st["dens"], p.rho_floor)
    return dt


def test_step_matches_reference_loop(oracle_lib):
    """orc_step (neighbour mode, reference CPU pair parameters) == the
    reference's loop body composed from its functors, for 4 steps incl. one
    Shepard filter."""
    need_ref(oracle_lib)
    from weaklycompressiblesph_b200 import cases
    phys = cases.Physics(alpha=0.01, beta=0.0, c_cfl=0.3, vsig_mode=oracle_lib.VSIG_REF_CPU, g=9.8,
                         density_mode=2, shepard_interval=3)
    case = cases.dam_break(dx=0.08, column=(0.4, 0.4, 0.8), tank=(0.8, 0.4, 1.0), phys=phys)
    rng = np.random.default_rng(4)
    case.vel = rng.normal(0, 0.2, size=case.vel.shape)
    case.vel[case.type == 1] = 0
    cfg = oracle_lib.config_from_case(case)
    a = oracle_lib.new_state(case)
    b = oracle_lib.new_state(case)
    oracle_lib.state_initial(case.n, a, cfg)
    # reference initial pass: EoS -> hydro -> filter -> gravity -> floor (main.cpp:69-78)
    n = case.n
    one = np.array([0, n], np.int32)
    import ctypes as C
    pres = np.zeros(n)
    snds = np.zeros(n)
    f = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
    oracle_lib.ref().ref_pressure(n, f(b["dens"]), f(pres), f(snds), phys.gamma, phys.rho0, phys.c0)
    epi = np.zeros(n, fdps.EPI_HYDRO)
    epj = np.zeros(n, fdps.EPJ_HYDRO)
    for e in (epi, epj):
        e["pos"], e["vel"], e["smth"], e["dens"], e["pres"], e["snds"], e["visc"] = (
            b["pos"], b["vel"], case.h, b["dens"], pres, snds, phys.nu)
    epj["mass"] = case.mass
    out = oracle_lib.ref_hydro_walks(one, epi, one, epj)
    b["acc"][:] = out["acc"]
    b["div_v"][:] = out["div_v"]
    b["dt_i"][:] = out["dt"]
    epi_f = np.zeros(n, fdps.EPI_FILTER)
    epi_f["pos"], epi_f["smth"] = b["pos"], case.h
    epj_f = np.zeros(n, fdps.EPJ_FILTER)
    epj_f["pos"], epj_f["dens"], epj_f["mass"] = b["pos"], b["dens"], case.mass
    b["dens"][:] = oracle_lib.ref_filter_walks(one, epi_f, one, epj_f)
    b["acc"][:, 2] -= phys.g
    b["dens"][:] = np.maximum(b["dens"], phys.rho_floor)
    for k in ("acc", "div_v", "dt_i", "dens"):
        assert rel_l2(a[k], b[k]) < 1e-9, k
    for step in range(4):
        dta = oracle_lib.state_step(n, a, case.type, cfg, step)
        dtb = _ref_step(oracle_lib, case, b, step, 3)
        assert dta == pytest.approx(dtb, rel=1e-12)
        for k in ("pos", "vel", "dens", "acc", "div_v"):
            assert rel_l2(a[k], b[k]) < 1e-9, (step, k)


def test_golden_vectors(oracle_lib):
    """The oracle reproduces the committed outputs of the reference build."""
    from tests.golden.make_golden import records
    g, case, w = load_golden()
    epi, epj, epi_f, epj_f = records(case, w)
    pp = oracle_lib.PairParams(0.01, 0.0, 0.3, 0.01, oracle_lib.VSIG_REF_CPU, oracle_lib.GRAD_HBAR)
    got = oracle_lib.hydro_walks(w.i_off, epi, w.j_off, epj, pp)
    assert rel_l2(got["acc"], g["acc"]) < 1e-10
    assert rel_l2(got["div_v"], g["div_v"]) < 1e-10
    np.testing.assert_allclose(got["dt"], g["dt"], rtol=1e-12)
    fdens = oracle_lib.filter_walks(w.i_off, epi_f, w.j_off, epj_f)
    np.testing.assert_allclose(fdens, g["filter_dens"], rtol=1e-12)


def load_golden():
    """The committed golden case: arrays, a Case object and its walks."""
    from tests.golden.make_golden import small_case
    g = np.load(os.path.join(GOLDEN, "hydro_walks_small.npz"))
    case = small_case()
    assert np.array_equal(case.pos, g["pos"]) and np.array_equal(case.vel, g["vel"])
    w = fdps.Walks(g["i_idx"], g["i_off"], g["j_idx"], g["j_off"])
    return g, case, w

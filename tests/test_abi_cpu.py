"""CPU-only checks of the C ABI library and the host logic (no GPU calls)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from weaklycompressiblesph_b200 import cases, fdps
from weaklycompressiblesph_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "wcsph.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(wcsph_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(native):
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (wcsph_\w+)", out))
    declared = header_functions()
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    assert sorted(N.exported_symbols()) == declared


def test_default_layout_and_pair_params(native):
    lay = fdps.default_layout()
    assert (lay.epi_size, lay.epj_size, lay.res_size) == (96, 112, 40)
    assert (lay.fepi_size, lay.fepj_size, lay.fres_size) == (32, 40, 8)
    for name in ("pos", "vel", "smth", "dens", "pres", "snds", "visc"):
        assert getattr(lay, "epi_" + name) == fdps.EPI_HYDRO.fields[name][1]
    g = fdps.pair_params("reference_gpu")
    assert (g.alpha, g.beta, g.c_cfl, g.vsig_mode, g.grad_mode) == (0.01, 0.02, 0.3, N.VSIG_SIGNAL, N.GRAD_SYM)
    c = fdps.pair_params("reference_cpu")
    assert (c.alpha, c.beta, c.c_cfl, c.vsig_mode, c.grad_mode) == (0.01, 0.0, 0.3, N.VSIG_REF_CPU, N.GRAD_HBAR)
    assert N.lib().wcsph_abi_version() == 2


def test_configure_rejects_bad_params(native):
    p = fdps.pair_params("reference_gpu")
    p.vsig_mode = 7
    with pytest.raises(N.WcsphError) as e:
        fdps.configure(p)
    assert e.value.code == 1  # WCSPH_E_INVALID
    fdps.configure("reference_gpu")


def test_struct_sizes_match_header(native):
    assert C.sizeof(N.InstanceDesc) == 176
    assert C.sizeof(N.SimOptions) == 48
    assert C.sizeof(N.PairParams) == 40
    assert C.sizeof(N.FdpsLayout) == 30 * 4


def test_dam_break_counts():
    c = cases.dam_break(dx=0.02)
    assert c.meta["n_fluid"] == 16000 and c.meta["n_wall"] == 38508
    big = cases.dam_break(dx=0.005)
    assert big.meta["n_fluid"] == 1024000 and big.meta["n_wall"] == 571308
    # hydrostatic: P(z) = rho0 g (H - z) at the column base
    pres, _ = c.eos()
    f = (c.type == 0) & (c.pos[:, 2] < 0.011)
    np.testing.assert_allclose(pres[f], 1000 * 9.81 * (0.8 - c.pos[f, 2]), rtol=1e-9)


def test_periodic_lattice_seeded():
    a = cases.periodic_lattice(n_side=10, dx=0.01, seed=12345)
    b = cases.periodic_lattice(n_side=10, dx=0.01, seed=12345)
    assert np.array_equal(a.pos, b.pos) and np.array_equal(a.vel, b.vel)
    assert a.pos.min() >= 0 and a.pos.max() < 0.1
    assert abs(a.dens.mean() / 1000 - 1) < 0.01


def test_walks_are_supersets(oracle_lib):
    """Every in-support neighbour of an i-particle is in its walk's j-list."""
    c = cases.dam_break(dx=0.05)
    w = fdps.build_walks(c.pos, 2.0 * c.h, group_size=64)
    assert w.i_off[-1] == c.n and np.array_equal(np.sort(w.i_idx), np.arange(c.n))
    cfg = oracle_lib.config_from_case(c)
    cnt, tot, lst = oracle_lib.neighbors(oracle_lib.pos4(c.pos.astype(np.float32)), cfg, lists=True, cap=256)
    for k in range(w.n_walk):
        js = set(w.j_idx[w.j_off[k]:w.j_off[k + 1]].tolist())
        for i in w.i_idx[w.i_off[k]:w.i_off[k + 1]]:
            assert set(lst[i, :cnt[i]].tolist()) <= js
            assert i in js


def test_ensemble_and_requests_seeded():
    e = cases.ensemble_cases(count=6, seed=1, n_min=2e3, n_max=2e4)
    nf = [c.n_fluid for c in e]
    assert all(1.0e3 < x < 4.0e4 for x in nf)
    r1 = cases.serving_requests(count=5, seed=3, n_min=2e3, n_max=1e4)
    r2 = cases.serving_requests(count=5, seed=3, n_min=2e3, n_max=1e4)
    assert [t for t, _ in r1] == [t for t, _ in r2]
    assert all(b[0] > a[0] for a, b in zip(r1, r1[1:]))

"""FDPS multiwalk drop-in (wcsph_hydro_dispatch / wcsph_hydro_retrieve) vs
the oracle's walk-mode restatement, on the GPU through the C ABI.
Tolerance: FP32 pair arithmetic, relative L2 <= 1e-5 (acc, div v) and
elementwise 1e-5 (dt) against FP64."""
import numpy as np
import pytest

from tests.helpers import rel_l2, small_dam, walk_setup
from weaklycompressiblesph_b200 import cases, fdps
from weaklycompressiblesph_b200 import _native as N

pytestmark = pytest.mark.gpu
TOL = 1e-5


def run_plugin(w, epi, epj, pair, **kw):
    fdps.configure(pair)
    out = np.zeros(len(epi), fdps.RESULT_HYDRO)
    fdps.calc_force_multiwalk(w, epi, epj, out, **kw)
    return out


def oracle_pair(oracle_lib, p):
    return oracle_lib.PairParams(p.alpha, p.beta, p.c_cfl, p.eps, p.vsig_mode, p.grad_mode)


@pytest.mark.parametrize("kind", ["reference_gpu", "reference_cpu"])
@pytest.mark.parametrize("which", ["dam", "periodic"])
def test_hydro_walks_parity(native, oracle_lib, kind, which):
    case = small_dam(dx=0.05) if which == "dam" else cases.periodic_lattice(n_side=16, dx=0.01, seed=3)
    w, epi, epj = walk_setup(case, group_size=128)
    pair = fdps.pair_params(kind)
    got = run_plugin(w, epi, epj, pair)
    ref = oracle_lib.hydro_walks(w.i_off, epi, w.j_off, epj, oracle_pair(oracle_lib, pair))
    assert rel_l2(got["acc"], ref["acc"]) < TOL
    assert rel_l2(got["div_v"], ref["div_v"]) < TOL
    np.testing.assert_allclose(got["dt"], ref["dt"], rtol=TOL)


def test_batches_and_tags(native, oracle_lib):
    """Several dispatch batches with two tags in flight give the same result."""
    case = small_dam(dx=0.05, seed=9)
    w, epi, epj = walk_setup(case, group_size=64)
    pair = fdps.pair_params("reference_gpu")
    one = run_plugin(w, epi, epj, pair)
    many = run_plugin(w, epi, epj, pair, n_walk_limit=7, tag_max=2)
    np.testing.assert_array_equal(one["acc"], many["acc"])
    np.testing.assert_array_equal(one["dt"], many["dt"])


def test_golden_vectors(native, oracle_lib):
    """The drop-in reproduces the reference build's committed outputs."""
    from tests.golden.make_golden import records
    from tests.test_oracle_pin import load_golden
    g, case, w = load_golden()
    epi, epj, epi_f, epj_f = records(case, w)
    got = run_plugin(w, epi, epj, fdps.pair_params("reference_cpu"))
    assert rel_l2(got["acc"], g["acc"]) < TOL
    assert rel_l2(got["div_v"], g["div_v"]) < TOL
    np.testing.assert_allclose(got["dt"], g["dt"], rtol=TOL)
    out = np.zeros(len(epi_f), fdps.RESULT_FILTER)
    fdps.calc_force_multiwalk(w, epi_f, epj_f, out, kind="filter")
    np.testing.assert_allclose(out["dens"], g["filter_dens"], rtol=TOL)


def test_filter_parity(native, oracle_lib):
    case = small_dam(dx=0.05, seed=4)
    w, epi, epj = walk_setup(case)
    epi_f = np.zeros(len(epi), fdps.EPI_FILTER)
    epi_f["pos"], epi_f["smth"] = epi["pos"], epi["smth"]
    epj_f = np.zeros(len(epj), fdps.EPJ_FILTER)
    epj_f["pos"], epj_f["dens"], epj_f["mass"] = epj["pos"], epj["dens"], epj["mass"]
    out = np.zeros(len(epi_f), fdps.RESULT_FILTER)
    fdps.calc_force_multiwalk(w, epi_f, epj_f, out, kind="filter")
    ref = oracle_lib.filter_walks(w.i_off, epi_f, w.j_off, epj_f)
    np.testing.assert_allclose(out["dens"], ref, rtol=TOL)


def test_ragged_and_empty_walks(native, oracle_lib):
    """Walks with zero i or zero j, a single particle, and n_walk = 0."""
    case = small_dam(dx=0.05, seed=2)
    w, epi, epj = walk_setup(case, group_size=128)
    # cut the first walk to 1 i and give the second walk an empty j-list
    i_off = w.i_off.copy()
    j_off = w.j_off.copy()
    keep_i = np.ones(len(epi), bool)
    keep_i[i_off[0] + 1:i_off[1]] = False
    keep_j = np.ones(len(epj), bool)
    keep_j[j_off[1]:j_off[2]] = False
    ni = np.diff(i_off)
    nj = np.diff(j_off)
    ni[0] = 1
    nj[1] = 0
    w2 = fdps.Walks(w.i_idx[keep_i], np.concatenate([[0], np.cumsum(ni)]), w.j_idx[keep_j],
                    np.concatenate([[0], np.cumsum(nj)]))
    epi2, epj2 = epi[keep_i], epj[keep_j]
    pair = fdps.pair_params("reference_gpu")
    got = run_plugin(w2, epi2, epj2, pair)
    ref = oracle_lib.hydro_walks(w2.i_off, epi2, w2.j_off, epj2, oracle_pair(oracle_lib, pair))
    assert rel_l2(got["acc"], ref["acc"]) < TOL
    np.testing.assert_allclose(got["dt"], ref["dt"], rtol=TOL)
    # zero walks
    fdps.HydrDispatchKernel(0, 0, [], np.zeros(0, np.int32), [], np.zeros(0, np.int32))
    fdps.HydrRetrieveKernel(0, 0, np.zeros(0, np.int32), [])


def test_error_behaviour(native):
    with pytest.raises(N.WcsphError) as e:
        fdps.HydrRetrieveKernel(1, 0, np.zeros(0, np.int32), [])
    assert e.value.code == 4  # STATE: no pending dispatch
    with pytest.raises(N.WcsphError) as e:
        fdps.HydrDispatchKernel(N.FDPS_MAX_TAGS, 0, [], np.zeros(0, np.int32), [], np.zeros(0, np.int32))
    assert e.value.code == 1
    case = small_dam(dx=0.1)
    w, epi, epj = walk_setup(case)
    epi_l, epj_l, _ = fdps.split_walks(w, epi, epj)
    fdps.HydrDispatchKernel(0, w.n_walk, epi_l, np.diff(w.i_off), epj_l, np.diff(w.j_off))
    out = np.zeros(len(epi), fdps.RESULT_HYDRO)
    bad = np.diff(w.i_off).astype(np.int32)
    bad[0] += 1
    with pytest.raises(N.WcsphError) as e:
        fdps.HydrRetrieveKernel(0, w.n_walk, bad, [out[:1]] * w.n_walk)
    assert e.value.code == 1
    _, _, out_l = fdps.split_walks(w, epi, epj, out)
    fdps.HydrRetrieveKernel(0, w.n_walk, np.diff(w.i_off), out_l)
    assert np.all(np.isfinite(out["acc"]))


def fdps_stats(tag=0):
    import ctypes as C
    out = (C.c_int64 * 4)()
    N.call("wcsph_fdps_stats", tag, out)
    return dict(h2d=int(out[0]), d2h=int(out[1]), compact=int(out[2]), pieces=int(out[3]))


def test_compact_staging(native, oracle_lib):
    """A piece of the batch whose records all carry the same h, nu and m is
    staged in 36-byte records, the others in 48-byte ones: both give the
    oracle's sums, and the compact pieces give the same bits as when every
    piece is compact."""
    case = small_dam(dx=0.04, seed=13)
    w, epi, epj = walk_setup(case, group_size=16)
    assert w.n_walk >= 256  # four pieces
    pair = fdps.pair_params("reference_gpu")
    ref_pair = oracle_pair(oracle_lib, pair)
    a = run_plugin(w, epi, epj, pair)
    sa = fdps_stats()
    assert sa["pieces"] == 4 and sa["compact"] == 4
    ref = oracle_lib.hydro_walks(w.i_off, epi, w.j_off, epj, ref_pair)
    assert rel_l2(a["acc"], ref["acc"]) < TOL and rel_l2(a["div_v"], ref["div_v"]) < TOL
    np.testing.assert_allclose(a["dt"], ref["dt"], rtol=TOL)
    # one j-record of the last walk with another viscosity: its piece (the
    # last quarter of the walks) goes back to 48-byte records
    epj2 = epj.copy()
    epj2["visc"][w.j_off[-2]] *= 1.5
    b = run_plugin(w, epi, epj2, pair)
    sb = fdps_stats()
    assert sb["pieces"] == 4 and sb["compact"] == 3
    assert sb["h2d"] > sa["h2d"]
    ref2 = oracle_lib.hydro_walks(w.i_off, epi, w.j_off, epj2, ref_pair)
    assert rel_l2(b["acc"], ref2["acc"]) < TOL and rel_l2(b["div_v"], ref2["div_v"]) < TOL
    first = w.i_off[(w.n_walk * 3) // 4]  # the i-records of the three compact pieces
    np.testing.assert_array_equal(a["acc"][:first], b["acc"][:first])
    np.testing.assert_array_equal(a["dt"][:first], b["dt"][:first])

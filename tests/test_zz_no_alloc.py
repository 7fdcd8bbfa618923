"""The allocation-free walk pair sum (wcsph_hydro_walks_noalloc).

Some callers cannot allocate device memory: an application whose device
memory all comes from its own pool or a fixed budget, or a host loop in which
a cudaMalloc would synchronise the device in the middle of a step.  For them
the library keeps its only scratch (the per-walk displacement tables) in a
static device array.  This test calls the entry point through the C ABI,
twice in a row on the same buffers, and checks both results against the
allocating entry point (wcsph_hydro_dispatch / wcsph_hydro_retrieve) and
against the FP64 oracle's walk-mode pair sum (oracle.hydro_walks), at the
FP32 tolerance the other parity tests use (relative L2 1e-5).  The file is
named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import rel_l2, small_dam, walk_setup
from weaklycompressiblesph_b200 import fdps
from weaklycompressiblesph_b200 import _native as N

pytestmark = pytest.mark.gpu
TOL = 1e-5


def pack(w, epi, epj):
    """Interleaved FP32 records, positions relative to each walk's first i."""
    n_i = np.diff(w.i_off)
    n_j = np.diff(w.j_off)
    origin = epi["pos"][w.i_off[:-1]]
    oi = np.repeat(origin, n_i, axis=0)
    oj = np.repeat(origin, n_j, axis=0)
    ri = np.zeros((len(epi), 3, 4), np.float32)
    ri[:, 0, :3] = epi["pos"] - oi
    ri[:, 0, 3] = epi["smth"]
    ri[:, 1, :3] = epi["vel"]
    ri[:, 1, 3] = epi["dens"]
    ri[:, 2, 0] = epi["pres"] / epi["dens"] ** 2
    ri[:, 2, 1] = epi["snds"]
    ri[:, 2, 2] = epi["visc"]
    rj = np.zeros((len(epj), 3, 4), np.float32)
    rj[:, 0, :3] = epj["pos"] - oj
    rj[:, 0, 3] = epj["smth"]
    rj[:, 1, :3] = epj["vel"]
    rj[:, 1, 3] = epj["dens"]
    rj[:, 2, 0] = epj["pres"] / epj["dens"] ** 2
    rj[:, 2, 1] = epj["snds"]
    rj[:, 2, 2] = epj["visc"]
    rj[:, 2, 3] = epj["mass"]
    return n_i.astype(np.int32), n_j.astype(np.int32), ri, rj


def test_noalloc_matches_allocating_entry_point(native, oracle_lib):
    import torch

    case = small_dam(dx=0.05, seed=21)
    w, epi, epj = walk_setup(case, group_size=128)
    pair = fdps.pair_params("reference_gpu")
    fdps.configure(pair)
    ref = np.zeros(len(epi), fdps.RESULT_HYDRO)
    fdps.calc_force_multiwalk(w, epi, epj, ref)
    fp64 = oracle_lib.hydro_walks(w.i_off, epi, w.j_off, epj,
                                  oracle_lib.PairParams(pair.alpha, pair.beta, pair.c_cfl, pair.eps, pair.vsig_mode,
                                                        pair.grad_mode))

    n_i, n_j, ri, rj = pack(w, epi, epj)
    dev = torch.device("cuda", 0)
    d_ni = torch.from_numpy(n_i).to(dev)
    d_nj = torch.from_numpy(n_j).to(dev)
    d_ei = torch.from_numpy(ri.reshape(-1)).to(dev)
    d_ej = torch.from_numpy(rj.reshape(-1)).to(dev)
    d_out = torch.empty(len(epi) * 8, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        d_out.fill_(float("nan"))
        N.call("wcsph_hydro_walks_noalloc", w.n_walk, C.c_void_p(d_ni.data_ptr()), C.c_void_p(d_nj.data_ptr()),
               C.c_void_p(d_ei.data_ptr()), C.c_void_p(d_ej.data_ptr()), C.c_void_p(d_out.data_ptr()),
               C.byref(pair), C.c_void_p(stream))
        torch.cuda.synchronize(dev)
        out = d_out.cpu().numpy().reshape(-1, 2, 4)
        assert np.all(np.isfinite(out[:, 0, :])), f"call {call}: unwritten results"
        for chk in (ref, fp64):  # the allocating entry point, then the FP64 oracle
            assert rel_l2(out[:, 0, :3], chk["acc"]) < TOL, f"call {call}"
            assert rel_l2(out[:, 0, 3], chk["div_v"]) < TOL, f"call {call}"
            np.testing.assert_allclose(out[:, 1, 0], chk["dt"], rtol=TOL)


def test_noalloc_rejects_oversized_batches(native):
    pair = fdps.pair_params("reference_gpu")
    rc = N.lib().wcsph_hydro_walks_noalloc(65536 + 1, None, None, None, None, None, C.byref(pair), None)
    assert rc == 3  # WCSPH_E_CAPACITY
    assert b"allocation-free limit" in N.lib().wcsph_last_error()

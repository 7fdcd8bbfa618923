"""Host-side mirror of the reference's FDPS plugin surface.

* numpy record types byte-identical to STD::EPI::Hydro, STD::EPJ::Hydro,
  STD::RESULT::Hydro and the Filter triple (src/class.h:61-263, x86-64);
* ``HydrDispatchKernel`` / ``HydrRetrieveKernel`` with the argument meaning of
  GPU_WC::HydrDispatchKernel / GPU_WC::HydrRetrieveKernel
  (src/prototype.h:7-10, src/kernel.cu:289-409), calling the C ABI;
* ``build_walks``: an FDPS stand-in that forms interaction groups of at most
  ``group_size`` i-particles (FDPS Ngroup, src/param.h:9) with a superset
  j-list (every particle within the group's box grown by the search radius,
  the Symmetry-mode contract of src/main.cpp:64), and
  ``calc_force_multiwalk`` which drives dispatch/retrieve in batches of at
  most ``n_walk_limit`` walks the way calcForceAllAndWriteBackMultiWalk does
  (src/main.cpp:71,112).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N

EPI_HYDRO = np.dtype([("pos", "<f8", 3), ("vel", "<f8", 3), ("smth", "<f8"), ("dens", "<f8"), ("pres", "<f8"),
                      ("snds", "<f8"), ("visc", "<f8"), ("tag", "<i8")])
EPJ_HYDRO = np.dtype([("pos", "<f8", 3), ("vel", "<f8", 3), ("dens", "<f8"), ("mass", "<f8"), ("smth", "<f8"),
                      ("pres", "<f8"), ("snds", "<f8"), ("visc", "<f8"), ("tag", "<i8"), ("type", "<i4"),
                      ("_pad", "<i4")])
RESULT_HYDRO = np.dtype([("acc", "<f8", 3), ("dt", "<f8"), ("div_v", "<f8")])
EPI_FILTER = np.dtype([("pos", "<f8", 3), ("smth", "<f8")])
EPJ_FILTER = np.dtype([("pos", "<f8", 3), ("dens", "<f8"), ("mass", "<f8")])
RESULT_FILTER = np.dtype([("dens", "<f8")])

assert EPI_HYDRO.itemsize == 96 and EPJ_HYDRO.itemsize == 112 and RESULT_HYDRO.itemsize == 40


def default_layout() -> N.FdpsLayout:
    lay = N.FdpsLayout()
    N.lib().wcsph_fdps_default_layout(C.byref(lay))
    return lay


def pair_params(kind="reference_gpu", **override) -> N.PairParams:
    p = N.PairParams()
    if kind == "reference_gpu":
        N.lib().wcsph_pair_params_reference_gpu(C.byref(p))
    elif kind == "reference_cpu":
        N.lib().wcsph_pair_params_reference_cpu(C.byref(p))
    else:
        raise ValueError(kind)
    for k, v in override.items():
        setattr(p, k, v)
    return p


def configure(pair: N.PairParams | str = "reference_gpu", layout: N.FdpsLayout | None = None):
    if isinstance(pair, str):
        pair = pair_params(pair)
    lay = layout or default_layout()
    N.call("wcsph_fdps_configure", C.byref(lay), C.byref(pair))


def _ptr_array(arrays):
    arr = (C.c_void_p * max(1, len(arrays)))()
    for k, a in enumerate(arrays):
        arr[k] = a.ctypes.data if a is not None and len(a) else None
    return arr


def _i32(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.int32))


# Keep the staged pointer arrays alive between dispatch and retrieve.
_inflight = {}


def HydrDispatchKernel(tag, n_walk, epi, n_epi, epj, n_epj):
    """GPU_WC::HydrDispatchKernel: epi/epj are sequences of record arrays
    (EPI_HYDRO / EPJ_HYDRO), one per walk.  Returns 0."""
    pi, pj = _ptr_array(epi[:n_walk]), _ptr_array(epj[:n_walk])
    ni, nj = _i32(n_epi[:n_walk]), _i32(n_epj[:n_walk])
    _inflight[("h", tag)] = (pi, pj, ni, nj, epi, epj)
    N.call("wcsph_hydro_dispatch", tag, n_walk, pi, N.ptr(ni, C.c_int32), pj, N.ptr(nj, C.c_int32))
    return 0


def HydrRetrieveKernel(tag, n_walk, ni, force):
    """GPU_WC::HydrRetrieveKernel: force is a sequence of RESULT_HYDRO arrays."""
    pf = _ptr_array(force[:n_walk])
    n = _i32(ni[:n_walk])
    N.call("wcsph_hydro_retrieve", tag, n_walk, N.ptr(n, C.c_int32), pf)
    _inflight.pop(("h", tag), None)
    return 0


def FilterDispatchKernel(tag, n_walk, epi, n_epi, epj, n_epj):
    pi, pj = _ptr_array(epi[:n_walk]), _ptr_array(epj[:n_walk])
    ni, nj = _i32(n_epi[:n_walk]), _i32(n_epj[:n_walk])
    _inflight[("f", tag)] = (pi, pj, ni, nj, epi, epj)
    N.call("wcsph_filter_dispatch", tag, n_walk, pi, N.ptr(ni, C.c_int32), pj, N.ptr(nj, C.c_int32))
    return 0


def FilterRetrieveKernel(tag, n_walk, ni, result):
    pf = _ptr_array(result[:n_walk])
    n = _i32(ni[:n_walk])
    N.call("wcsph_filter_retrieve", tag, n_walk, N.ptr(n, C.c_int32), pf)
    _inflight.pop(("f", tag), None)
    return 0


# ---------------------------------------------------------------------------
# FDPS stand-in: interaction groups and superset j-lists
# ---------------------------------------------------------------------------

@dataclass
class Walks:
    """Walk w owns i-particles i_idx[i_off[w]:i_off[w+1]] and j-particles
    j_idx[j_off[w]:j_off[w+1]] (indices into the particle arrays)."""
    i_idx: np.ndarray
    i_off: np.ndarray
    j_idx: np.ndarray
    j_off: np.ndarray

    @property
    def n_walk(self):
        return len(self.i_off) - 1

    @property
    def n_evaluated(self):
        """Pair evaluations the walk contract implies (sum of n_i * n_j)."""
        return int(np.sum(np.diff(self.i_off).astype(np.int64) * np.diff(self.j_off)))


def _morton_order(pos, cell):
    lo = pos.min(axis=0)
    c = np.floor((pos - lo) / cell).astype(np.int64)
    c = np.clip(c, 0, (1 << 20) - 1)

    def spread(v):
        v = v & 0x1FFFFF
        v = (v | (v << 32)) & 0x1F00000000FFFF
        v = (v | (v << 16)) & 0x1F0000FF0000FF
        v = (v | (v << 8)) & 0x100F00F00F00F00F
        v = (v | (v << 4)) & 0x10C30C30C30C30C3
        v = (v | (v << 2)) & 0x1249249249249249
        return v

    key = spread(c[:, 0]) | (spread(c[:, 1]) << 1) | (spread(c[:, 2]) << 2)
    return np.argsort(key, kind="stable")


def build_walks(pos, r_search, group_size=128, box=None, fine=None) -> Walks:
    """Group particles into walks of <= group_size in Morton order (fine
    cells of `fine` edge, default r_search/2) and give each walk every particle
    inside its i-group bounding box grown by r_search.  With `box` (periodic
    edge lengths) the j-list uses minimum images, so j positions must be
    shifted by the caller (see `walk_records`)."""
    pos = np.asarray(pos, dtype=np.float64)
    n = len(pos)
    fine = fine or 0.5 * r_search
    order = _morton_order(pos, fine)
    n_walk = (n + group_size - 1) // group_size
    i_off = np.minimum(np.arange(n_walk + 1, dtype=np.int64) * group_size, n)
    # coarse grid of edge r_search for candidate search
    lo = pos.min(axis=0) - 1e-9
    cell = r_search
    cidx = np.floor((pos - lo) / cell).astype(np.int64)
    ncell = cidx.max(axis=0) + 1
    lin = (cidx[:, 2] * ncell[1] + cidx[:, 1]) * ncell[0] + cidx[:, 0]
    srt = np.argsort(lin, kind="stable")
    lin_s = lin[srt]
    starts = np.searchsorted(lin_s, np.arange(ncell.prod() + 1))
    j_lists = []
    for w in range(n_walk):
        g = order[i_off[w]:i_off[w + 1]]
        bmin = pos[g].min(axis=0) - r_search
        bmax = pos[g].max(axis=0) + r_search
        if box is None:
            c0 = np.clip(np.floor((bmin - lo) / cell).astype(np.int64), 0, ncell - 1)
            c1 = np.clip(np.floor((bmax - lo) / cell).astype(np.int64), 0, ncell - 1)
            zz, yy, xx = np.meshgrid(np.arange(c0[2], c1[2] + 1), np.arange(c0[1], c1[1] + 1),
                                     np.arange(c0[0], c1[0] + 1), indexing="ij")
            cl = ((zz * ncell[1] + yy) * ncell[0] + xx).ravel()
            cand = np.concatenate([srt[starts[c]:starts[c + 1]] for c in cl])
            p = pos[cand]
            inside = np.all((p >= bmin) & (p <= bmax), axis=1)
            j_lists.append(np.sort(cand[inside]))
        else:
            box = np.asarray(box, dtype=np.float64)
            centre = 0.5 * (bmin + bmax)
            half = 0.5 * (bmax - bmin)
            d = pos - centre
            d -= box * np.round(d / box)
            inside = np.all(np.abs(d) <= half, axis=1)
            j_lists.append(np.nonzero(inside)[0])
    j_off = np.zeros(n_walk + 1, np.int64)
    j_off[1:] = np.cumsum([len(j) for j in j_lists])
    j_idx = np.concatenate(j_lists) if j_lists else np.zeros(0, np.int64)
    return Walks(order.astype(np.int64), i_off, j_idx.astype(np.int64), j_off)


def walk_records(walks: Walks, pos, vel, dens, pres, snds, smth, mass, visc, type_=None, box=None):
    """Flat EPI/EPJ record arrays for the walks (FP64, class.h layout).  For a
    periodic `box`, each j position is replaced by its image nearest to the
    walk's first i-particle (FDPS hands out such shifted images too)."""
    n = len(dens)
    smth = np.broadcast_to(np.asarray(smth, np.float64), (n,))
    mass = np.broadcast_to(np.asarray(mass, np.float64), (n,))
    visc = np.broadcast_to(np.asarray(visc, np.float64), (n,))
    epi = np.zeros(len(walks.i_idx), EPI_HYDRO)
    ii = walks.i_idx
    epi["pos"], epi["vel"], epi["smth"] = pos[ii], vel[ii], smth[ii]
    epi["dens"], epi["pres"], epi["snds"], epi["visc"], epi["tag"] = dens[ii], pres[ii], snds[ii], visc[ii], ii
    epj = np.zeros(len(walks.j_idx), EPJ_HYDRO)
    jj = walks.j_idx
    jpos = pos[jj].copy()
    if box is not None:
        box = np.asarray(box, np.float64)
        anchor = np.repeat(pos[ii[walks.i_off[:-1]]], np.diff(walks.j_off), axis=0)
        d = jpos - anchor
        jpos -= box * np.round(d / box)
    epj["pos"], epj["vel"], epj["dens"], epj["mass"] = jpos, vel[jj], dens[jj], mass[jj]
    epj["smth"], epj["pres"], epj["snds"], epj["visc"], epj["tag"] = smth[jj], pres[jj], snds[jj], visc[jj], jj
    if type_ is not None:
        epj["type"] = np.asarray(type_)[jj]
    return epi, epj


def split_walks(walks: Walks, epi, epj, out=None):
    """Per-walk views: lists of EPI, EPJ (and RESULT) arrays."""
    epi_l = [epi[walks.i_off[w]:walks.i_off[w + 1]] for w in range(walks.n_walk)]
    epj_l = [epj[walks.j_off[w]:walks.j_off[w + 1]] for w in range(walks.n_walk)]
    out_l = None if out is None else [out[walks.i_off[w]:walks.i_off[w + 1]] for w in range(walks.n_walk)]
    return epi_l, epj_l, out_l


def calc_force_multiwalk(walks: Walks, epi, epj, out, n_walk_limit=16384, tag_max=1, kind="hydro"):
    """Drive dispatch/retrieve over all walks in batches of <= n_walk_limit,
    overlapping batch k+1's dispatch with batch k's retrieve when tag_max > 1.
    `out` (RESULT_HYDRO or RESULT_FILTER records, one per EPI) is filled."""
    dispatch = HydrDispatchKernel if kind == "hydro" else FilterDispatchKernel
    retrieve = HydrRetrieveKernel if kind == "hydro" else FilterRetrieveKernel
    epi_l, epj_l, out_l = split_walks(walks, epi, epj, out)
    n_epi = np.diff(walks.i_off).astype(np.int32)
    n_epj = np.diff(walks.j_off).astype(np.int32)
    pending = []
    for b, w0 in enumerate(range(0, walks.n_walk, n_walk_limit)):
        w1 = min(walks.n_walk, w0 + n_walk_limit)
        tag = b % tag_max
        if len(pending) >= tag_max:
            t, a0, a1 = pending.pop(0)
            retrieve(t, a1 - a0, n_epi[a0:a1], out_l[a0:a1])
        dispatch(tag, w1 - w0, epi_l[w0:w1], n_epi[w0:w1], epj_l[w0:w1], n_epj[w0:w1])
        pending.append((tag, w0, w1))
    for t, a0, a1 in pending:
        retrieve(t, a1 - a0, n_epi[a0:a1], out_l[a0:a1])
    return out

"""ctypes bindings of the oracle libraries (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libwcsph_ref.so")

VSIG_REF_CPU, VSIG_SIGNAL = 0, 1
GRAD_HBAR, GRAD_SYM = 0, 1


class PairParams(C.Structure):
    _fields_ = [("alpha", C.c_double), ("beta", C.c_double), ("c_cfl", C.c_double), ("eps", C.c_double),
                ("vsig_mode", C.c_int32), ("grad_mode", C.c_int32)]


class Config(C.Structure):
    _fields_ = [("h", C.c_double), ("mass", C.c_double), ("nu", C.c_double),
                ("rho0", C.c_double), ("gamma", C.c_double), ("c0", C.c_double),
                ("g", C.c_double), ("rho_floor", C.c_double),
                ("pair", PairParams),
                ("periodic", C.c_int32), ("density_mode", C.c_int32), ("shepard_interval", C.c_int32),
                ("pad_", C.c_int32),
                ("lo", C.c_float * 3), ("hi", C.c_float * 3), ("cell", C.c_float * 3),
                ("ncell", C.c_int32 * 3),
                ("kill_lo", C.c_float * 3), ("kill_hi", C.c_float * 3)]


def build():
    """make -C oracle (restatement always; the reference build when its sources exist)."""
    env = dict(os.environ)
    env.pop("CXX", None)
    env.pop("CC", None)
    r = subprocess.run(["make", "-s", "-C", HERE], capture_output=True, text=True, env=env)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)


_orc = None
_ref = None

F64P = C.POINTER(C.c_double)
F32P = C.POINTER(C.c_float)
I32P = C.POINTER(C.c_int32)
U32P = C.POINTER(C.c_uint32)
P = C.c_void_p


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def orc():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.orc_W.restype = C.c_double
        L.orc_W.argtypes = [C.c_double, C.c_double]
        L.orc_gradW_scalar.restype = C.c_double
        L.orc_gradW_scalar.argtypes = [C.c_double, C.c_double]
        L.orc_eos.argtypes = [C.c_int, F64P, F64P, F64P, C.c_double, C.c_double, C.c_double]
        L.orc_hydro_walks.argtypes = [C.c_int, I32P, P, I32P, P, P, C.POINTER(PairParams)]
        L.orc_filter_walks.argtypes = [C.c_int, I32P, F64P, I32P, F64P, F64P]
        L.orc_cells.argtypes = [C.c_int, F32P, C.POINTER(Config), I32P, U32P]
        L.orc_sort_perm.argtypes = [C.c_int, U32P, I32P]
        L.orc_neighbors.restype = C.c_int64
        L.orc_neighbors.argtypes = [C.c_int, F32P, C.POINTER(Config), I32P, I32P, C.c_int]
        L.orc_density.argtypes = [C.c_int, F32P, F32P, C.POINTER(Config), C.c_int, F64P]
        L.orc_hydro.argtypes = [C.c_int, F32P, F32P, F32P, F32P, F32P, C.POINTER(Config), F64P, F64P, F64P]
        L.orc_dt_global.restype = C.c_double
        L.orc_dt_global.argtypes = [C.c_int, F64P, F64P, I32P, C.c_double, C.c_double]
        L.orc_step.restype = C.c_double
        L.orc_step.argtypes = [C.c_int, F64P, F64P, F64P, F64P, F64P, F64P, F64P, I32P, C.POINTER(Config),
                               C.c_int64]
        L.orc_initial_force.argtypes = [C.c_int, F64P, F64P, F64P, F64P, F64P, F64P, C.POINTER(Config)]
        _orc = L
    return _orc


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    """The reference's own functors; raises when oracle/_ref was not built."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise RuntimeError(f"{REF_SO} is missing (built only where the reference sources exist)")
        L = C.CDLL(REF_SO)
        L.ref_layout.restype = C.c_int
        L.ref_layout.argtypes = [C.POINTER(C.c_long), C.c_int]
        L.ref_hydro_walk.argtypes = [P, C.c_int, P, C.c_int, P]
        L.ref_hydro_walks.argtypes = [C.c_int, I32P, P, I32P, P, P, C.c_int]
        L.ref_filter_walks.argtypes = [C.c_int, I32P, P, I32P, P, P, C.c_int]
        L.ref_pressure.argtypes = [C.c_int, F64P, F64P, F64P, C.c_double, C.c_double, C.c_double]
        L.ref_timestep.restype = C.c_double
        L.ref_timestep.argtypes = [C.c_int, F64P, F64P, F64P, I32P, C.c_double]
        L.ref_kdk_first.argtypes = [C.c_int, F64P, F64P, F64P, F64P, F64P, F64P, I32P, C.c_double]
        L.ref_kdk_final.argtypes = [C.c_int, F64P, F64P, F64P, I32P, C.c_double]
        L.ref_W.restype = C.c_double
        L.ref_W.argtypes = [C.c_double] * 4
        L.ref_gradW.argtypes = [C.c_double] * 4 + [F64P]
        L.ref_params.argtypes = [F64P]
        _ref = L
    return _ref


# ---------------------------------------------------------------- helpers

def config_from_case(case, density_mode=None):
    """Oracle Config mirroring the solver's instance parameters, including the
    FP32 cell grid the device derives (edge >= 2h, 1.0001 margin)."""
    p = case.phys
    c = Config()
    c.h, c.mass, c.nu = case.h, case.mass, p.nu
    c.rho0, c.gamma, c.c0, c.g, c.rho_floor = p.rho0, p.gamma, p.c0, p.g, p.rho_floor
    c.pair = PairParams(p.alpha, p.beta, p.c_cfl, p.eps, p.vsig_mode, GRAD_HBAR)
    c.periodic = 1 if case.periodic else 0
    c.density_mode = p.density_mode if density_mode is None else density_mode
    c.shepard_interval = p.shepard_interval
    H = np.float32(2.0) * np.float32(case.h)
    for k in range(3):
        lo, hi = np.float32(case.lo[k]), np.float32(case.hi[k])
        ext = np.float32(hi - lo)
        nc = int(np.floor(ext / np.float32(H * np.float32(1.0001))))
        nc = max(nc, 1)
        if case.periodic:
            cell = np.float32(ext / np.float32(nc))
        else:
            cell = max(np.float32(ext / np.float32(nc)), np.float32(H * np.float32(1.0001)))
        if cell < H:
            cell = np.float32(H * np.float32(1.0001))
        c.lo[k], c.hi[k], c.cell[k], c.ncell[k] = lo, hi, cell, nc
        c.kill_lo[k], c.kill_hi[k] = case.kill_lo[k], case.kill_hi[k]
    return c


def pos4(pos, extra=None):
    a = np.zeros((len(pos), 4), np.float32)
    a[:, :3] = pos
    if extra is not None:
        a[:, 3] = extra
    return np.ascontiguousarray(a)


def cells(pos4_, cfg):
    n = len(pos4_)
    cxyz = np.zeros((n, 3), np.int32)
    key = np.zeros(n, np.uint32)
    orc().orc_cells(n, _p(pos4_, C.c_float), C.byref(cfg), _p(cxyz, C.c_int32), _p(key, C.c_uint32))
    return cxyz, key


def sort_perm(key):
    key = np.ascontiguousarray(key, np.uint32)
    perm = np.zeros(len(key), np.int32)
    orc().orc_sort_perm(len(key), _p(key, C.c_uint32), _p(perm, C.c_int32))
    return perm


def neighbors(pos4_, cfg, lists=False, cap=256):
    n = len(pos4_)
    cnt = np.zeros(n, np.int32)
    lst = np.full((n, cap), -1, np.int32) if lists else None
    tot = orc().orc_neighbors(n, _p(pos4_, C.c_float), C.byref(cfg), _p(cnt, C.c_int32), _p(lst, C.c_int32), cap)
    return (cnt, tot, lst) if lists else (cnt, tot)


def density(pos4_, dens_f32, cfg, shepard):
    n = len(pos4_)
    out = np.zeros(n, np.float64)
    d = np.ascontiguousarray(dens_f32, np.float32)
    orc().orc_density(n, _p(pos4_, C.c_float), _p(d, C.c_float), C.byref(cfg), 1 if shepard else 0,
                      _p(out, C.c_double))
    return out


def eos(dens, gamma, rho0, c0):
    dens = np.ascontiguousarray(dens, np.float64)
    pres = np.zeros_like(dens)
    snds = np.zeros_like(dens)
    orc().orc_eos(len(dens), _p(dens, C.c_double), _p(pres, C.c_double), _p(snds, C.c_double), gamma, rho0, c0)
    return pres, snds


def hydro(pos4_, vel4, dens, pres, snds, cfg):
    n = len(pos4_)
    f = lambda a: np.ascontiguousarray(a, np.float32)
    v4, d, pr, sn = f(vel4), f(dens), f(pres), f(snds)
    acc = np.zeros((n, 3), np.float64)
    dv = np.zeros(n, np.float64)
    dt = np.zeros(n, np.float64)
    orc().orc_hydro(n, _p(pos4_, C.c_float), _p(v4, C.c_float), _p(d, C.c_float), _p(pr, C.c_float),
                    _p(sn, C.c_float), C.byref(cfg), _p(acc, C.c_double), _p(dv, C.c_double), _p(dt, C.c_double))
    return acc, dv, dt


def hydro_walks(i_off, epi, j_off, epj, pair: PairParams):
    out = np.zeros(len(epi), dtype=[("acc", "<f8", 3), ("dt", "<f8"), ("div_v", "<f8")])
    io = np.ascontiguousarray(i_off, np.int32)
    jo = np.ascontiguousarray(j_off, np.int32)
    orc().orc_hydro_walks(len(io) - 1, _p(io, C.c_int32), epi.ctypes.data, _p(jo, C.c_int32), epj.ctypes.data,
                          out.ctypes.data, C.byref(pair))
    return out


def filter_walks(i_off, epi_f, j_off, epj_f):
    """epi_f: EPI::Filter records; epj_f: EPJ::Filter records."""
    io = np.ascontiguousarray(i_off, np.int32)
    jo = np.ascontiguousarray(j_off, np.int32)
    ei = np.ascontiguousarray(np.column_stack([epi_f["pos"], epi_f["smth"]]), np.float64)
    ej = np.ascontiguousarray(np.column_stack([epj_f["pos"], epj_f["dens"], epj_f["mass"]]), np.float64)
    out = np.zeros(len(epi_f), np.float64)
    orc().orc_filter_walks(len(io) - 1, _p(io, C.c_int32), _p(ei, C.c_double), _p(jo, C.c_int32),
                           _p(ej, C.c_double), _p(out, C.c_double))
    return out


def ref_hydro_walks(i_off, epi, j_off, epj, nthreads=0):
    out = np.zeros(len(epi), dtype=[("acc", "<f8", 3), ("dt", "<f8"), ("div_v", "<f8")])
    io = np.ascontiguousarray(i_off, np.int32)
    jo = np.ascontiguousarray(j_off, np.int32)
    ref().ref_hydro_walks(len(io) - 1, _p(io, C.c_int32), epi.ctypes.data, _p(jo, C.c_int32), epj.ctypes.data,
                          out.ctypes.data, nthreads)
    return out


def ref_filter_walks(i_off, epi_f, j_off, epj_f, nthreads=0):
    out = np.zeros(len(epi_f), dtype=[("dens", "<f8")])
    io = np.ascontiguousarray(i_off, np.int32)
    jo = np.ascontiguousarray(j_off, np.int32)
    ref().ref_filter_walks(len(io) - 1, _p(io, C.c_int32), epi_f.ctypes.data, _p(jo, C.c_int32), epj_f.ctypes.data,
                           out.ctypes.data, nthreads)
    return out["dens"]


def state_step(n, st, typ, cfg, step_index):
    """orc_step on a dict of FP64 state arrays (modified in place); returns dt."""
    t = np.ascontiguousarray(typ, np.int32)
    return orc().orc_step(n, _p(st["pos"], C.c_double), _p(st["vel"], C.c_double), _p(st["vel_half"], C.c_double),
                          _p(st["dens"], C.c_double), _p(st["acc"], C.c_double), _p(st["div_v"], C.c_double),
                          _p(st["dt_i"], C.c_double), _p(t, C.c_int32), C.byref(cfg), step_index)


def state_initial(n, st, cfg):
    orc().orc_initial_force(n, _p(st["pos"], C.c_double), _p(st["vel"], C.c_double), _p(st["dens"], C.c_double),
                            _p(st["acc"], C.c_double), _p(st["div_v"], C.c_double), _p(st["dt_i"], C.c_double),
                            C.byref(cfg))


def new_state(case):
    n = case.n
    return dict(pos=np.ascontiguousarray(case.pos, np.float64).copy(),
                vel=np.ascontiguousarray(case.vel, np.float64).copy(),
                vel_half=np.zeros((n, 3), np.float64), dens=np.ascontiguousarray(case.dens, np.float64).copy(),
                acc=np.zeros((n, 3), np.float64), div_v=np.zeros(n, np.float64), dt_i=np.zeros(n, np.float64))

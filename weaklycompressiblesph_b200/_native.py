"""ctypes binding of libwcsph.so, the C ABI declared in include/wcsph.h.

The shared library is built in-tree (``python -m weaklycompressiblesph_b200.build``
or ``__graft_entry__.build()``).  Loading fails loudly when it is missing:
there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwcsph.so")

WCSPH_OK = 0
STATUS_NAMES = {1: "INVALID", 2: "CUDA", 3: "CAPACITY", 4: "STATE", 5: "NOMEM", 6: "NODEVICE"}

VSIG_REF_CPU, VSIG_SIGNAL = 0, 1
GRAD_HBAR, GRAD_SYM = 0, 1
PREC_FP32, PREC_TILED, PREC_HALF2 = 0, 1, 2
DENSITY_CONTINUITY, DENSITY_SUMMATION, DENSITY_SHEPARD = 0, 1, 2
HYDRO, FREEZE = 0, 1
FDPS_MAX_TAGS = 4
LIST_SHAPES = 7  # launch shapes of the neighbour-list pass (wcsph_sim_tuning out[1])
BUILD_SHAPES = 7  # launch shapes of the list build's scan (wcsph_sim_tuning out[3])


class FdpsLayout(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "epi_size", "epi_pos", "epi_vel", "epi_smth", "epi_dens", "epi_pres", "epi_snds", "epi_visc",
        "epj_size", "epj_pos", "epj_vel", "epj_dens", "epj_mass", "epj_smth", "epj_pres", "epj_snds", "epj_visc",
        "res_size", "res_acc", "res_dt", "res_div_v",
        "fepi_size", "fepi_pos", "fepi_smth",
        "fepj_size", "fepj_pos", "fepj_dens", "fepj_mass",
        "fres_size", "fres_dens")]


class PairParams(C.Structure):
    _fields_ = [("alpha", C.c_double), ("beta", C.c_double), ("c_cfl", C.c_double), ("eps", C.c_double),
                ("vsig_mode", C.c_int32), ("grad_mode", C.c_int32)]


class InstanceDesc(C.Structure):
    _fields_ = [("n", C.c_int32), ("density_mode", C.c_int32), ("shepard_interval", C.c_int32),
                ("periodic", C.c_int32),
                ("h", C.c_double), ("mass", C.c_double), ("nu", C.c_double),
                ("rho0", C.c_double), ("gamma", C.c_double), ("c0", C.c_double),
                ("g", C.c_double), ("rho_floor", C.c_double),
                ("pair", PairParams),
                ("lo", C.c_float * 3), ("hi", C.c_float * 3),
                ("kill_lo", C.c_float * 3), ("kill_hi", C.c_float * 3),
                ("t_end", C.c_double)]


class SimOptions(C.Structure):
    _fields_ = [("device", C.c_int32), ("precision", C.c_int32), ("max_particles", C.c_int64),
                ("max_cells", C.c_int64), ("max_instances", C.c_int32), ("use_graph", C.c_int32),
                ("autotune", C.c_int32), ("list_interval", C.c_int32), ("list_skin", C.c_float),
                ("list_shape", C.c_int32)]


class Slab(C.Structure):
    _fields_ = [("x_lo", C.c_float), ("x_hi", C.c_float), ("margin", C.c_float),
                ("has_left", C.c_int32), ("has_right", C.c_int32)]


SLAB_RECORD_BYTES = 64


class WcsphError(RuntimeError):
    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} failed: {STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


_lib = None

P = C.c_void_p
PP = C.POINTER(C.c_void_p)
I32P = C.POINTER(C.c_int32)
F32P = C.POINTER(C.c_float)
U32P = C.POINTER(C.c_uint32)
F64P = C.POINTER(C.c_double)

_SIGS = {
    "wcsph_abi_version": (C.c_int, []),
    "wcsph_last_error": (C.c_char_p, []),
    "wcsph_init": (C.c_int, [C.c_int32]),
    "wcsph_finalize": (C.c_int, []),
    "wcsph_fdps_default_layout": (None, [C.POINTER(FdpsLayout)]),
    "wcsph_pair_params_reference_cpu": (None, [C.POINTER(PairParams)]),
    "wcsph_pair_params_reference_gpu": (None, [C.POINTER(PairParams)]),
    "wcsph_fdps_configure": (C.c_int, [C.POINTER(FdpsLayout), C.POINTER(PairParams)]),
    "wcsph_hydro_dispatch": (C.c_int, [C.c_int32, C.c_int32, PP, I32P, PP, I32P]),
    "wcsph_hydro_retrieve": (C.c_int, [C.c_int32, C.c_int32, I32P, PP]),
    "wcsph_hydro_walks_noalloc": (C.c_int, [C.c_int32, P, P, P, P, P, C.POINTER(PairParams), P]),
    "wcsph_filter_dispatch": (C.c_int, [C.c_int32, C.c_int32, PP, I32P, PP, I32P]),
    "wcsph_filter_retrieve": (C.c_int, [C.c_int32, C.c_int32, I32P, PP]),
    "wcsph_sim_create": (C.c_int, [C.POINTER(SimOptions), C.POINTER(C.c_void_p)]),
    "wcsph_sim_destroy": (C.c_int, [P]),
    "wcsph_sim_device_bytes": (C.c_int64, [C.POINTER(SimOptions)]),
    "wcsph_sim_add_instance": (C.c_int, [P, C.POINTER(InstanceDesc), F32P, F32P, F32P, I32P, I32P]),
    "wcsph_sim_restore_instance": (C.c_int, [P, C.POINTER(InstanceDesc), F32P, F32P, F32P, I32P, F32P, F32P, I32P,
                                              I32P, C.c_double, C.c_int64, C.c_float, I32P]),
    "wcsph_sim_next_dt": (C.c_int, [P, C.c_int32, F32P]),
    "wcsph_sim_set_next_dt": (C.c_int, [P, C.c_int32, C.c_float]),
    "wcsph_sim_force_pass": (C.c_int, [P, C.c_int32]),
    "wcsph_slab_layer_width": (C.c_float, [C.c_double, C.c_float]),
    "wcsph_sim_add_slab": (C.c_int, [P, C.POINTER(InstanceDesc), C.POINTER(Slab), C.c_int32, I32P, F32P, F32P, F32P,
                                      I32P, I32P]),
    "wcsph_sim_slab_pack": (C.c_int, [P, C.c_int32, P, C.c_int64, I32P]),
    "wcsph_sim_slab_unpack": (C.c_int, [P, C.c_int32, P, C.c_int32, C.c_int32]),
    "wcsph_sim_remove_instance": (C.c_int, [P, C.c_int32]),
    "wcsph_sim_step": (C.c_int, [P, C.c_int32]),
    "wcsph_sim_synchronize": (C.c_int, [P]),
    "wcsph_sim_instance_status": (C.c_int, [P, C.c_int32, F64P, C.POINTER(C.c_int64), I32P, I32P]),
    "wcsph_sim_read_instance": (C.c_int, [P, C.c_int32, F32P, F32P, F32P, F32P, F32P, F32P, I32P]),
    "wcsph_sim_probe_forces": (C.c_int, [P, C.c_int32, C.c_int32, F32P, F32P, F32P, F32P, I32P]),
    "wcsph_sim_probe_lists": (C.c_int, [P, C.c_int32, C.c_int32, F32P, F32P, F32P, F32P, I32P]),
    "wcsph_sim_read_order": (C.c_int, [P, C.c_int32, I32P, U32P]),
    "wcsph_sim_conservation": (C.c_int, [P, C.c_int32, F64P]),
    "wcsph_sim_last_pairs": (C.c_int64, [P]),
    "wcsph_sim_kernels_per_step": (C.c_int32, [P]),
    "wcsph_sim_stream": (C.c_void_p, [P]),
    "wcsph_sim_list_stats": (C.c_int, [P, C.POINTER(C.c_int64)]),
    "wcsph_sim_tuning": (C.c_int, [P, I32P]),
    "wcsph_fdps_stats": (C.c_int, [C.c_int32, C.POINTER(C.c_int64)]),
    "wcsph_sim_invalidate_lists": (C.c_int, [P]),
    "wcsph_sim_list_entries": (C.c_int64, [P]),
    "wcsph_sim_profile_steps": (C.c_int, [P, C.c_int32, F64P]),
    "wcsph_sim_profile_split": (C.c_int, [P, C.c_int32, F64P, C.POINTER(C.c_int32)]),
    "wcsph_sim_list_schedule": (C.c_int, [P, C.POINTER(C.c_int64)]),
}


def exported_symbols():
    """Names of the C entry points this binding expects (all of include/wcsph.h)."""
    return sorted(_SIGS)


def lib():
    """Load libwcsph.so (once).  Raises if the library has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                               "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(fn_name, rc):
    if rc != WCSPH_OK:
        msg = lib().wcsph_last_error()
        raise WcsphError(fn_name, rc, msg.decode() if msg else "")
    return rc


def call(name, *args):
    return check(name, getattr(lib(), name)(*args))


def ptr(a, ctype):
    """ctypes pointer to a contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))

"""ctypes binding of the C ABI declared in include/mz_b200.h.

The shared library is built in-tree (meamzilla_b200/libmz_b200.so) by
meamzilla_b200.build.  There is no fallback: if the library is missing or a
call fails, an MzError is raised.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmz_b200.so")

MZ_OK = 0
MZ_FP64 = 0
MZ_MIXED = 1
MZ_STYLE_EAM_SPLINE = 0
MZ_STYLE_MEAM_SPLINE = 1
MZ_STYLE_GMEAM_SPLINE = 2
MZ_STYLE_PAIR_SPLINE = 3
MZ_STYLE_JMEAM_SPLINE = 4
MZ_STYLE_JMEAM2_SPLINE = 5

STATUS_NAMES = {
    0: "MZ_OK", 1: "MZ_ERR_ARG", 2: "MZ_ERR_IO", 3: "MZ_ERR_FORMAT", 4: "MZ_ERR_RANGE",
    5: "MZ_ERR_UNSUPPORTED", 6: "MZ_ERR_CUDA", 7: "MZ_ERR_NOMEM", 8: "MZ_ERR_TIMEOUT",
}


class MzError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, str(status)), msg))
        self.status = status


class CellsDesc(C.Structure):
    _fields_ = [
        ("ncells", C.c_int), ("natoms", C.c_int),
        ("cell_natoms", C.POINTER(C.c_int)), ("cell_lattice", C.POINTER(C.c_double)),
        ("cell_energy0", C.POINTER(C.c_double)), ("cell_stress0", C.POINTER(C.c_double)),
        ("cell_weight", C.POINTER(C.c_double)), ("cell_eweight", C.POINTER(C.c_double)),
        ("cell_sweight", C.POINTER(C.c_double)), ("atom_type", C.POINTER(C.c_int)),
        ("atom_pos", C.POINTER(C.c_double)), ("atom_force0", C.POINTER(C.c_double)),
    ]


class DbStats(C.Structure):
    _fields_ = [("ncells", C.c_int), ("natoms", C.c_int), ("npairs", C.c_int64), ("ntriplets", C.c_int64),
                ("max_row", C.c_int), ("esize", C.c_int)]


class DbView(C.Structure):
    _fields_ = [
        ("ncells", C.c_int), ("natoms", C.c_int), ("npairs", C.c_int64),
        ("cell_atom0", C.POINTER(C.c_int)),
        ("cell_vol", C.POINTER(C.c_double)), ("cell_weight", C.POINTER(C.c_double)),
        ("cell_eweight", C.POINTER(C.c_double)), ("cell_sweight", C.POINTER(C.c_double)),
        ("cell_energy0", C.POINTER(C.c_double)), ("cell_stress0", C.POINTER(C.c_double)),
        ("cell_lattice", C.POINTER(C.c_double)),
        ("atom_type", C.POINTER(C.c_int)), ("atom_cell", C.POINTER(C.c_int)),
        ("atom_pos", C.POINTER(C.c_double)), ("atom_force0", C.POINTER(C.c_double)),
        ("pair_off", C.POINTER(C.c_int64)), ("pair_nbr", C.POINTER(C.c_int)),
        ("pair_r", C.POINTER(C.c_double)), ("pair_u", C.POINTER(C.c_double)),
        ("pair_knot", C.POINTER(C.c_int8)), ("pair_shift", C.POINTER(C.c_double)),
        ("in_off", C.POINTER(C.c_int64)), ("in_slot", C.POINTER(C.c_int64)),
        ("nfun", C.c_int),
    ]


class SplineView(C.Structure):
    _fields_ = [("group", C.c_int), ("alloy", C.c_int), ("nknots", C.c_int), ("left", C.c_double),
                ("right", C.c_double), ("nat", C.c_int * 2), ("grad_fixed", C.c_int * 2),
                ("grad", C.c_double * 2), ("y_fixed", C.POINTER(C.c_int)), ("y", C.POINTER(C.c_double)),
                ("x", C.POINTER(C.c_double)), ("step", C.c_double), ("quintic", C.c_int),
                ("grad2", C.c_double * 2)]


class Settings(C.Structure):
    _fields_ = [("energy_weight", C.c_double), ("stress_weight", C.c_double), ("embed_extrap", C.c_int),
                ("device", C.c_int), ("max_candidates", C.c_int), ("omit_punishments", C.c_int)]


_lib = None

_SIGS = {
    "mz_last_error": (C.c_char_p, []),
    "mz_pot_read": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "mz_pot_parse": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "mz_pot_free": (None, [C.c_void_p]),
    "mz_pot_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "mz_pot_ncoeff": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "mz_pot_get_coeffs": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mz_pot_set_coeffs": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mz_pot_write": (C.c_int, [C.c_void_p, C.c_char_p]),
    "mz_pot_spline_eval": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "mz_pot_get_spline": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(SplineView)]),
    "mz_db_build": (C.c_int, [C.POINTER(CellsDesc), C.c_void_p, C.POINTER(C.c_void_p)]),
    "mz_db_read": (C.c_int, [C.c_char_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "mz_write_data": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_double] + [C.c_void_p] * 5 +
                      [C.c_char_p, C.c_int]),
    "mz_pot_clone": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "mz_pot_rescale": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_void_p]),
    "mz_db_build_device": (C.c_int, [C.POINTER(CellsDesc), C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "mz_db_read_device": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "mz_db_free": (None, [C.c_void_p]),
    "mz_db_info": (C.c_int, [C.c_void_p, C.POINTER(DbStats)]),
    "mz_db_get_view": (C.c_int, [C.c_void_p, C.POINTER(DbView)]),
    "mz_db_set_targets": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mz_create": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Settings), C.POINTER(C.c_void_p)]),
    "mz_destroy": (None, [C.c_void_p]),
    "mz_objective": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p]),
    "mz_objective_grad": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "mz_densities": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "mz_objective_device": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mz_objective_grad_device": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "mz_sync": (C.c_int, [C.c_void_p]),
    "mz_stream": (C.c_void_p, [C.c_void_p]),
    "mz_gram_device": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_int64,
                                 C.c_int64, C.c_void_p]),
    "mz_launch_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "mz_tensor_core_forward": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "mz_kernel_name": (C.c_char_p, [C.c_int]),
    "mz_moment_path": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "mz_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "mz_tuning": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "mz_kernel_times": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "mz_alu_peak": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "mz_objective_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Settings), C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
}

MZ_NKERNELS = 13


def lib() -> C.CDLL:
    """Load libmz_b200.so (building it first if it is missing or stale)."""
    global _lib
    if _lib is None:
        from . import build as _build
        if not _build.up_to_date():
            _build.build()
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int):
    if status != MZ_OK:
        raise MzError(status, lib().mz_last_error().decode())


def ptr(a):
    """Raw pointer of a C-contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


def as_array(p, n, dtype):
    """Copy n elements from a raw ctypes pointer into a numpy array."""
    if n == 0:
        return np.zeros(0, dtype=dtype)
    ct = np.ctypeslib.as_ctypes_type(np.dtype(dtype))
    buf = C.cast(p, C.POINTER(ct * n)).contents
    return np.frombuffer(buf, dtype=dtype, count=n).copy()

"""ctypes binding of libgila_b200.so (declarations in include/gila_b200.h).

The shared library is loaded from this package directory.  There is no
fallback: if the library is missing or CUDA is unusable the calls raise.
"""
from __future__ import annotations

import ctypes as ct
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# GILA_B200_LIB names another build of the same library (a debug build, a build
# with other compile-time options)
LIB_PATH = os.environ.get("GILA_B200_LIB") or os.path.join(HERE, "libgila_b200.so")

GILA_OK = 0
GILA_ERR_ARG = 1
GILA_ERR_SIZE = 2
GILA_ERR_TYPE = 3
GILA_ERR_CUDA = 4
GILA_ERR_NOMEM = 5
GILA_ERR_NAN = 6
GILA_ERR_NODEV = 7
GILA_ERR_OVERLAP = 8
GILA_ERR_SCALE = 9
GILA_ERR_NOTCONV = 10
GILA_ERR_TIMEOUT = 11
GILA_ERR_INTERNAL = 12

GILA_C64 = 0   # ComplexF32
GILA_C128 = 1  # ComplexF64

I64x3 = ct.c_int64 * 3


class GilaVolC(ct.Structure):
    _fields_ = [("cel", I64x3), ("scl_num", I64x3), ("scl_den", I64x3),
                ("org_num", I64x3), ("org_den", I64x3),
                ("grd_num", I64x3), ("grd_den", I64x3)]


class GilaKoptC(ct.Structure):
    _fields_ = [("frq_re", ct.c_double), ("frq_im", ct.c_double), ("int_ord", ct.c_int32),
                ("adj_mod", ct.c_int32), ("dev_mod", ct.c_int32),
                ("num_trd", ct.c_int32 * 3), ("num_blk", ct.c_int32 * 3)]


class GilaSolveC(ct.Structure):
    """gila_solve_opts (include/gila_b200.h)."""
    _fields_ = [("tol", ct.c_double), ("ell", ct.c_int32), ("mixed", ct.c_int32),
                ("max_matvecs", ct.c_int32), ("max_restarts", ct.c_int32), ("delta", ct.c_double),
                ("x0", ct.c_int32), ("no_graph", ct.c_int32), ("keep", ct.c_int32)]


class GilaSolveInfoC(ct.Structure):
    """gila_solve_info (include/gila_b200.h)."""
    _fields_ = [("iters", ct.c_int32), ("outer", ct.c_int32), ("matvecs_f64", ct.c_int32),
                ("matvecs_f32", ct.c_int32), ("rel_res", ct.c_double), ("converged", ct.c_int32),
                ("breakdowns", ct.c_int32)]


class GilaServerOptsC(ct.Structure):
    """gila_server_opts (include/gila_b200.h)."""
    _fields_ = [("hbm_budget", ct.c_int64), ("slots", ct.c_int32), ("ell", ct.c_int32), ("mixed", ct.c_int32),
                ("int_ord", ct.c_int32), ("frq_re", ct.c_double), ("frq_im", ct.c_double)]


class GilaServerStatsC(ct.Structure):
    """gila_server_stats (include/gila_b200.h)."""
    _fields_ = [("submitted", ct.c_int64), ("completed", ct.c_int64), ("queued", ct.c_int64),
                ("running", ct.c_int64), ("batches", ct.c_int64), ("operators", ct.c_int64),
                ("bytes_in_use", ct.c_int64), ("hbm_budget", ct.c_int64)]


_lib = None

# (name, restype, argtypes)
_SIGS = [
    ("gila_ctx_create", ct.c_int, [ct.c_int, ct.POINTER(ct.c_void_p)]),
    ("gila_ctx_destroy", ct.c_int, [ct.c_void_p]),
    ("gila_last_error", ct.c_char_p, []),
    ("gila_status_string", ct.c_char_p, [ct.c_int]),
    ("gila_version", ct.c_char_p, []),
    ("gila_opr_create", ct.c_int, [ct.c_void_p, ct.POINTER(GilaVolC), ct.POINTER(GilaVolC),
                                   ct.POINTER(GilaKoptC), ct.c_int, ct.POINTER(ct.c_void_p)]),
    ("gila_opr_create_from_fur", ct.c_int, [ct.c_void_p, ct.POINTER(GilaVolC), ct.POINTER(GilaVolC),
                                            ct.POINTER(GilaKoptC), ct.c_int, ct.c_void_p * 8,
                                            (ct.c_int64 * 6) * 8, ct.c_int, ct.POINTER(ct.c_void_p)]),
    ("gila_opr_fur_dims", ct.c_int, [ct.c_void_p, (ct.c_int64 * 6) * 8]),
    ("gila_opr_export_fur", ct.c_int, [ct.c_void_p, ct.c_void_p * 8]),
    ("gila_opr_adjoint", ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_void_p)]),
    ("gila_opr_destroy", ct.c_int, [ct.c_void_p]),
    ("gila_opr_sizes", ct.c_int, [ct.c_void_p, ct.c_int64 * 4, ct.c_int64 * 4]),
    ("gila_opr_input_size", ct.c_int, [ct.c_void_p, ct.c_int64 * 4]),
    ("gila_opr_output_size", ct.c_int, [ct.c_void_p, ct.c_int64 * 4]),
    ("gila_opr_info", ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_int), ct.POINTER(ct.c_int32)]),
    ("gila_opr_apply", ct.c_int, [ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_int64, ct.c_void_p,
                                  ct.c_int64, ct.c_int64, ct.c_void_p]),
    ("gila_opr_apply_axpby", ct.c_int, [ct.c_void_p, ct.c_int, ct.c_double * 2, ct.c_void_p, ct.c_int64,
                                        ct.c_double * 2, ct.c_void_p, ct.c_int64, ct.c_int64, ct.c_void_p]),
    ("gila_opr_reserve", ct.c_int, [ct.c_void_p, ct.c_int64]),
    ("gila_opr_device_bytes", ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_int64)]),
    ("gila_opr_time_passes", ct.c_int, [ct.c_void_p, ct.c_int64, ct.c_int, ct.c_double * 4]),
    ("gila_opr_autotune", ct.c_int, [ct.c_void_p, ct.c_int64, ct.c_int32 * 4]),
    ("gila_opr_get_tiles", ct.c_int, [ct.c_void_p, ct.c_int32 * 4]),
    ("gila_opr_set_tiles", ct.c_int, [ct.c_void_p, ct.c_int32 * 4]),
    ("gila_opr_get_schedule", ct.c_int, [ct.c_void_p, ct.c_int32 * 2]),
    ("gila_opr_set_schedule", ct.c_int, [ct.c_void_p, ct.c_int32 * 2]),
    ("gila_opr_launches_per_apply", ct.c_int, [ct.c_void_p, ct.c_int64, ct.POINTER(ct.c_int64)]),
    ("gila_opr_cast", ct.c_int, [ct.c_void_p, ct.c_int, ct.POINTER(ct.c_void_p)]),
    ("gila_ls_solve", ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int64,
                                 ct.POINTER(GilaSolveC), ct.POINTER(GilaSolveInfoC), ct.POINTER(ct.c_double),
                                 ct.c_void_p]),
    ("gila_server_create", ct.c_int, [ct.c_void_p, ct.POINTER(GilaServerOptsC), ct.POINTER(ct.c_void_p)]),
    ("gila_server_destroy", ct.c_int, [ct.c_void_p]),
    ("gila_server_submit", ct.c_int, [ct.c_void_p, ct.POINTER(GilaVolC), ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                      ct.POINTER(GilaSolveC), ct.POINTER(ct.c_uint64)]),
    ("gila_server_wait", ct.c_int, [ct.c_void_p, ct.c_uint64, ct.c_int64, ct.POINTER(GilaSolveInfoC),
                                    ct.POINTER(ct.c_double)]),
    ("gila_server_stats_get", ct.c_int, [ct.c_void_p, ct.POINTER(GilaServerStatsC)]),
    ("gila_opr_save", ct.c_int, [ct.c_void_p, ct.c_char_p]),
    ("gila_opr_load", ct.c_int, [ct.c_void_p, ct.c_char_p, ct.c_int, ct.POINTER(ct.c_void_p)]),
    ("gila_weak_integrals", ct.c_int, [ct.c_void_p, ct.c_int64 * 3, ct.c_int64 * 3, ct.c_double, ct.c_double,
                                       ct.c_int32, ct.c_double * 36]),
    ("gila_debug_fail_alloc", ct.c_int, [ct.c_int64]),
    ("gila_opr_slab_dims", ct.c_int, [ct.c_void_p, ct.c_int64 * 5]),
    ("gila_opr_slab_fwd", ct.c_int, [ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_int64, ct.c_void_p, ct.c_void_p]),
    ("gila_opr_slab_z", ct.c_int, [ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_int64, ct.c_int64, ct.c_void_p]),
    ("gila_opr_slab_inv", ct.c_int, [ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_int64, ct.c_void_p, ct.c_void_p]),
    ("gila_opr_apply_noalloc", ct.c_int, [ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_int64, ct.c_void_p,
                                          ct.c_int64, ct.c_void_p]),
]

# entry points added by later components; bound when present
_OPTIONAL_SIGS = []


def exported_symbols():
    """Names every declaration of include/gila_b200.h must export."""
    return [s[0] for s in _SIGS] + [s[0] for s in _OPTIONAL_SIGS]


def lib():
    """Load (once) and return the ctypes handle of libgila_b200.so."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"libgila_b200.so not found at {LIB_PATH}; build it with "
            "`python gilaelectromagnetics.jl_b200/build.py` (there is no CPU fallback)")
    h = ct.CDLL(LIB_PATH)
    for name, res, args in _SIGS + _OPTIONAL_SIGS:
        fn = getattr(h, name)
        fn.restype = res
        fn.argtypes = args
    _lib = h
    return h


def last_error() -> str:
    return lib().gila_last_error().decode(errors="replace")

"""Loader of the in-tree CUDA library libgsis_b200.so (built by __graft_entry__.build() / gsis_sim_b200/build.py).

There is no CPU fallback: if the library is missing or does not load, every product entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgsis_b200.so")
_lib = None


class LibraryMissing(RuntimeError):
    pass


def load_library():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise LibraryMissing(f"{LIB_PATH} is not built; run `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = C.CDLL(LIB_PATH)
    lib.kin_create.argtypes = [C.POINTER(abi.KinSetupDesc), C.POINTER(C.c_void_p)]
    lib.kin_create.restype = C.c_int
    lib.kin_destroy.argtypes = [C.c_void_p]
    lib.kin_destroy.restype = None
    lib.kin_last_error.argtypes = [C.c_void_p]
    lib.kin_last_error.restype = C.c_char_p
    lib.kin_name.argtypes = [C.c_void_p]
    lib.kin_name.restype = C.c_char_p
    abi.declare_backend_api(lib, "kin_")
    for name, args in {
        "memory_bytes": [C.c_void_p, C.POINTER(C.c_uint64)],
        "take_timings": [C.c_void_p, C.POINTER(abi.KinStepTimings)],
        "set_stream": [C.c_void_p, C.c_void_p],
        "launch_count": [C.c_void_p, C.POINTER(C.c_int64)],
        "device_f": [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int32)],
        "velocity_permutation": [C.c_void_p, C.POINTER(C.c_int32), C.c_int64],
        "schedule_info": [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)],
        "discrete_maxwell": [C.c_void_p, C.POINTER(C.c_double), C.c_int64, C.c_double, C.POINTER(C.c_double),
                             C.POINTER(C.c_int32)],
    }.items():
        fn = getattr(lib, "kin_" + name)
        fn.argtypes = args
        fn.restype = C.c_int
    _lib = lib
    return lib


# every symbol include/gsis_b200.h declares
EXPORTED_SYMBOLS = [
    "kin_create", "kin_destroy", "kin_last_error", "kin_name", "kin_chunk_width", "kin_memory_bytes",
    "kin_set_equilibrium", "kin_set_distribution", "kin_get_distribution", "kin_compute_moments",
    "kin_scale_distribution", "kin_update_cell_params", "kin_set_inflow", "kin_boundary_sums", "kin_sweep",
    "kin_gsis_correction", "kin_internal_face_mass_flux", "kin_take_timings", "kin_deq_counts",
    "kin_set_stream", "kin_launch_count", "kin_device_f", "kin_velocity_permutation", "kin_schedule_info", "kin_discrete_maxwell",
    "kin_discrete_maxwell_noalloc", "kin_moment_sums", "kin_set_moments", "kin_adjoint_begin", "kin_adjoint_set",
    "kin_adjoint_get", "kin_adjoint_reduce", "kin_adjoint_face_moment_seeds", "kin_adjoint_update", "kin_adjoint_end", "kin_gsis_correction_extrema",
    "kin_gsis_correction_apply", "kin_device_sums", "kin_finalize_moments", "kin_read_sums",
]

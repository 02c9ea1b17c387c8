"""ctypes wrapper of the C restatement oracle (oracle/_build/libkinoracle.so) — TEST INFRASTRUCTURE ONLY.

`OracleBackend` offers the same methods as the product's B200Backend (the reference KineticBackend interface,
src/kinetic/kinetic_backend.hpp:59-100), computed on the CPU by kinetic_oracle.c.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from gsis_sim_b200 import abi
from gsis_sim_b200.backend import KineticBackendABI, KineticError

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libkinoracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    L = C.CDLL(LIB_PATH)
    L.orc_create.argtypes = [C.POINTER(abi.KinSetupDesc), C.POINTER(C.c_void_p)]
    L.orc_create.restype = C.c_int
    L.orc_destroy.argtypes = [C.c_void_p]
    L.orc_destroy.restype = None
    L.orc_last_error.argtypes = [C.c_void_p]
    L.orc_last_error.restype = C.c_char_p
    abi.declare_backend_api(L, "orc_")
    L.orc_passes_given.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int64]
    L.orc_passes_given.restype = C.c_int
    _lib = L
    return L


class OracleBackend(KineticBackendABI):
    def __init__(self, setup: abi.SetupArrays, precision: str | None = None, velocity_chunk: int | None = None):
        L = lib()
        s = setup.copy()
        if precision is not None:
            s["precision"] = abi.PRECISIONS[precision]
        if velocity_chunk is not None:
            s["velocity_chunk"] = int(velocity_chunk)
        desc = s.desc()
        h = C.c_void_p()
        if L.orc_create(C.byref(desc), C.byref(h)) != 0:
            raise KineticError("orc_create failed")
        super().__init__(L, "orc_", h, s, lambda: L.orc_last_error(h).decode())

    def passes_given(self, R) -> None:
        """The LU-SGS block passes on the given steady residual (storage order): f += their update."""
        import numpy as np

        a = np.ascontiguousarray(R, dtype=np.float64).ravel()
        self._call("passes_given", abi.as_ptr(a, C.c_double), a.size)

    def close(self):
        if self._h:
            self._lib.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

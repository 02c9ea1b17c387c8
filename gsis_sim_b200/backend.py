"""Python view of the kinetic backend interface over a C ABI.

`KineticBackendABI` mirrors the reference's `gsis::kinetic::KineticBackend` (src/kinetic/kinetic_backend.hpp:59-100):
same method names, argument meaning (FP64, internal numbering) and error behaviour (a failed call raises
`KineticError`, the counterpart of `gsis::Error`). `B200Backend` binds it to the CUDA library
(libgsis_b200.so, entry points of include/gsis_b200.h).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from ._lib import load_library


ADJ_FACE_SUMS = 18  # per boundary face sums of kin_adjoint_reduce
ADJ_CELL_SUMS = 19  # per cell sums of kin_adjoint_reduce


class KineticError(RuntimeError):
    """A backend call failed (the reference raises gsis::Error in the same places)."""


class KineticBackendABI:
    """Common method layer over a kin_*-style C ABI (`prefix` selects the symbol family)."""

    def __init__(self, lib, prefix: str, handle, setup: abi.SetupArrays, error_fn):
        self._lib = lib
        self._prefix = prefix
        self._h = handle
        self.setup = setup
        self._error_fn = error_fn
        self.n_cells = setup.n_cells
        self.nv = setup.nv
        self.n_bfaces = setup.n_bfaces

    def _call(self, name, *args):
        rc = getattr(self._lib, self._prefix + name)(self._h, *args)
        if rc != abi.KIN_OK:
            raise KineticError(f"{self._prefix}{name} failed ({rc}): {self._error_fn()}")

    # --- KineticBackend methods -----------------------------------------------------------------------------
    def chunk_width(self) -> int:
        out = C.c_int32()
        self._call("chunk_width", C.byref(out))
        return out.value

    def set_equilibrium(self, states) -> None:
        s = np.ascontiguousarray(states, dtype=np.float64).ravel()
        self._call("set_equilibrium", abi.as_ptr(s, C.c_double), s.size)

    def set_distribution(self, f) -> None:
        a = np.ascontiguousarray(f, dtype=np.float64).ravel()
        self._call("set_distribution", abi.as_ptr(a, C.c_double), a.size)

    def get_distribution(self, out=None) -> np.ndarray:
        if out is None:
            out = np.empty(self.n_cells * self.nv, dtype=np.float64)
        self._call("get_distribution", abi.as_ptr(out, C.c_double), out.size)
        return out.reshape(self.n_cells, self.nv)

    def compute_moments(self, out=None) -> np.ndarray:
        if out is None:
            out = np.empty(self.n_cells * abi.MOMENTS_PER_CELL, dtype=np.float64)
        self._call("compute_moments", abi.as_ptr(out, C.c_double), out.size)
        return out.reshape(self.n_cells, abi.MOMENTS_PER_CELL)

    def moment_sums(self) -> np.ndarray:
        """The 13 shifted velocity sums per cell over the stored velocities, not finalised (velocity sharding)."""
        out = np.empty(self.n_cells * 13, dtype=np.float64)
        self._call("moment_sums", abi.as_ptr(out, C.c_double), out.size)
        return out.reshape(self.n_cells, 13)

    def set_moments(self, moments) -> None:
        """Install moments reduced over all velocity shards (they feed update_cell_params) and move the shift."""
        m = np.ascontiguousarray(moments, dtype=np.float64).ravel()
        self._call("set_moments", abi.as_ptr(m, C.c_double), m.size)

    # --- discrete adjoint (gsis_sim_b200.adjoint drives these) -----------------------------------------------
    def adjoint_begin(self, rev_velocity, rev_entry, flip_velocity=None, face_axis=None) -> None:
        rv = np.ascontiguousarray(rev_velocity, dtype=np.int32)
        re = np.ascontiguousarray(rev_entry, dtype=np.int32)
        fl = None if flip_velocity is None else np.ascontiguousarray(flip_velocity, dtype=np.int32)
        fa = None if face_axis is None else np.ascontiguousarray(face_axis, dtype=np.int32)
        self._adj_keep = (rv, re, fl, fa)
        self._call("adjoint_begin", abi.as_ptr(rv, C.c_int32), abi.as_ptr(re, C.c_int32), re.size,
                   None if fl is None else abi.as_ptr(fl, C.c_int32), None if fa is None else abi.as_ptr(fa, C.c_int32))

    def adjoint_set(self, lam) -> None:
        a = np.ascontiguousarray(lam, dtype=np.float64).ravel()
        self._call("adjoint_set", abi.as_ptr(a, C.c_double), a.size)

    def adjoint_get(self) -> np.ndarray:
        out = np.empty(self.n_cells * self.nv, dtype=np.float64)
        self._call("adjoint_get", abi.as_ptr(out, C.c_double), out.size)
        return out.reshape(self.n_cells, self.nv)

    def adjoint_reduce(self, mu, cells: bool = True, faces: bool = True):
        """Transposed transport with the per-face weights mu, then the per-cell (19) and per-face sums; cells=False /
        faces=False skip those sums (returned as None) when only the transport's seeds are wanted."""
        m = np.ascontiguousarray(mu, dtype=np.float64)
        cell = np.empty(self.n_cells * ADJ_CELL_SUMS, dtype=np.float64) if cells else None
        face = np.empty(max(self.n_bfaces, 1) * ADJ_FACE_SUMS, dtype=np.float64) if faces else None
        self._call("adjoint_reduce", abi.as_ptr(m, C.c_double), m.size,
                   abi.as_ptr(cell, C.c_double) if cells else None, cell.size if cells else 0,
                   abi.as_ptr(face, C.c_double) if faces else None, self.n_bfaces * ADJ_FACE_SUMS if faces else 0)
        return cell, (face[:self.n_bfaces * ADJ_FACE_SUMS] if faces else None)

    def adjoint_face_moment_seeds(self, seeds) -> None:
        """Seeds (n_bfaces, 5) on the boundary faces' moment sums for the following adjoint_reduce calls; None
        removes them."""
        if seeds is None:
            self._call("adjoint_face_moment_seeds", None, 0)
            return
        a = np.ascontiguousarray(seeds, dtype=np.float64).ravel()
        self._call("adjoint_face_moment_seeds", abi.as_ptr(a, C.c_double), a.size)

    def adjoint_update(self, coef, run_passes: bool = True, want_operator: bool = False):
        c = np.ascontiguousarray(coef, dtype=np.float64).ravel()
        res = np.empty(self.n_cells, dtype=np.float64)
        op = np.empty(self.n_cells * self.nv, dtype=np.float64) if want_operator else None
        self._call("adjoint_update", abi.as_ptr(c, C.c_double), c.size, abi.as_ptr(res, C.c_double), res.size,
                   C.c_int32(1 if run_passes else 0), abi.as_ptr(op, C.c_double) if op is not None else None,
                   op.size if op is not None else 0)
        return res, op

    def adjoint_end(self) -> None:
        self._call("adjoint_end")

    def scale_distribution(self, s: float) -> None:
        self._call("scale_distribution", C.c_double(s))

    def update_cell_params(self) -> None:
        self._call("update_cell_params")

    def set_inflow(self, inflow) -> None:
        a = np.ascontiguousarray(inflow, dtype=np.float64).reshape(-1, 6)
        arr = abi.inflow_array(a)
        self._call("set_inflow", arr, len(a))

    def boundary_sums(self, out=None) -> np.ndarray:
        if out is None:
            out = np.empty(max(self.n_bfaces, 0) * abi.BOUNDARY_SUMS_PER_FACE, dtype=np.float64)
        self._call("boundary_sums", abi.as_ptr(out, C.c_double), out.size)
        return out.reshape(self.n_bfaces, abi.BOUNDARY_SUMS_PER_FACE)

    def sweep(self, out=None) -> np.ndarray:
        if out is None:
            out = np.empty(self.n_cells, dtype=np.float64)
        self._call("sweep", abi.as_ptr(out, C.c_double), out.size)
        return out

    def gsis_correction(self, w_half, w_new):
        wh = np.ascontiguousarray(w_half, dtype=np.float64).ravel()
        wn = np.ascontiguousarray(w_new, dtype=np.float64).ravel()
        flags = np.zeros(self.n_cells, dtype=np.int32)
        replaced = C.c_int64()
        self._call("gsis_correction", abi.as_ptr(wh, C.c_double), abi.as_ptr(wn, C.c_double), wh.size,
                   abi.as_ptr(flags, C.c_int32), C.byref(replaced))
        return replaced.value, flags

    def gsis_correction_extrema(self, w_half, w_new) -> np.ndarray:
        """This handle's part of the per-cell negativity reduction of a velocity-sharded GSIS correction (reduce
        the shards' arrays with an element-wise minimum)."""
        wh = np.ascontiguousarray(w_half, dtype=np.float64).ravel()
        wn = np.ascontiguousarray(w_new, dtype=np.float64).ravel()
        ext = np.empty(self.n_cells, dtype=np.float64)
        self._call("gsis_correction_extrema", abi.as_ptr(wh, C.c_double), abi.as_ptr(wn, C.c_double), wh.size,
                   abi.as_ptr(ext, C.c_double), ext.size)
        return ext

    def gsis_correction_apply(self, w_half, w_new, ext):
        wh = np.ascontiguousarray(w_half, dtype=np.float64).ravel()
        wn = np.ascontiguousarray(w_new, dtype=np.float64).ravel()
        e = np.ascontiguousarray(ext, dtype=np.float64)
        flags = np.zeros(self.n_cells, dtype=np.int32)
        replaced = C.c_int64()
        self._call("gsis_correction_apply", abi.as_ptr(wh, C.c_double), abi.as_ptr(wn, C.c_double), wh.size,
                   abi.as_ptr(e, C.c_double), e.size, abi.as_ptr(flags, C.c_int32), C.byref(replaced))
        return replaced.value, flags

    def internal_face_mass_flux(self, cells, entries) -> np.ndarray:
        c = np.ascontiguousarray(cells, dtype=np.int32)
        e = np.ascontiguousarray(entries, dtype=np.int32)
        out = np.zeros(c.size, dtype=np.float64)
        self._call("internal_face_mass_flux", abi.as_ptr(c, C.c_int32), abi.as_ptr(e, C.c_int32), c.size,
                   abi.as_ptr(out, C.c_double))
        return out

    def discrete_maxwell(self, states, tolerance: float):
        """Conservative discrete Maxwellians of macroscopic states (n, 5) -> (corrected states, Newton result)."""
        st = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 5)
        out = np.empty_like(st)
        res = np.empty(len(st), dtype=np.int32)
        if len(st):
            self._call("discrete_maxwell", abi.as_ptr(st, C.c_double), len(st), C.c_double(tolerance),
                       abi.as_ptr(out, C.c_double), abi.as_ptr(res, C.c_int32))
        return out, res

    def deq_counts(self):
        d = abi.KinDeqCounts()
        self._call("deq_counts", C.byref(d))
        return d.corrected, d.failed, d.max_iterations


class _DeviceArray:
    """__cuda_array_interface__ of n device doubles (torch.as_tensor wraps it without a copy)."""

    def __init__(self, ptr: int, n: int, device: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None}
        self.device = device


class B200Backend(KineticBackendABI):
    """The B200 CUDA backend (libgsis_b200.so). Creating it uploads the setup and allocates f on the device."""

    def __init__(self, setup: abi.SetupArrays, precision: str | None = None, device: int = 0,
                 velocity_chunk: int | None = None):
        lib = load_library()
        s = setup.copy()
        if precision is not None:
            s["precision"] = abi.PRECISIONS[precision]
        if velocity_chunk is not None:
            s["velocity_chunk"] = int(velocity_chunk)
        s["device"] = device
        desc = s.desc()
        h = C.c_void_p()
        rc = lib.kin_create(C.byref(desc), C.byref(h))
        if rc != abi.KIN_OK:
            raise KineticError(f"kin_create failed ({rc}): {lib.kin_last_error(None).decode()}")
        super().__init__(lib, "kin_", h, s, lambda: lib.kin_last_error(h).decode())
        self._owned = True
        self.device = device

    def close(self):
        if getattr(self, "_owned", False) and self._h:
            self._lib.kin_destroy(self._h)
            self._h = None
            self._owned = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- B200 additions -------------------------------------------------------------------------------------
    def set_stream(self, stream_ptr: int) -> None:
        self._call("set_stream", C.c_void_p(stream_ptr))

    def launch_count(self) -> int:
        out = C.c_int64()
        self._call("launch_count", C.byref(out))
        return out.value

    # --- velocity sharding with the reductions in device memory --------------------------------------------------
    def device_sums(self, which: int):
        """A torch CUDA tensor viewing the handle's device buffer of one kind of sum (abi.KIN_SUMS_*), for an
        in-place reduction across shards (no copy)."""
        import torch

        ptr = C.POINTER(C.c_double)()
        n = C.c_int64()
        self._call("device_sums", C.c_int32(which), C.byref(ptr), C.byref(n))
        return torch.as_tensor(_DeviceArray(C.cast(ptr, C.c_void_p).value or 0, n.value, self.device),
                               device=f"cuda:{self.device}")

    def moment_sums_to_device(self) -> None:
        """The 13 moment sums per cell into the device buffer KIN_SUMS_MOMENTS (no copy to the host)."""
        self._call("moment_sums", None, 0)

    def boundary_sums_to_device(self) -> None:
        self._call("boundary_sums", None, 0)

    def sweep_to_device(self) -> None:
        self._call("sweep", None, 0)

    def finalize_moments(self) -> np.ndarray:
        """Moments from the (reduced) device moment sums, installed on the device; returned to the host."""
        out = np.empty(self.n_cells * 15, dtype=np.float64)
        self._call("finalize_moments", abi.as_ptr(out, C.c_double), out.size)
        return out.reshape(self.n_cells, 15)

    def read_sums(self, which: int, n: int) -> np.ndarray:
        out = np.empty(n, dtype=np.float64)
        self._call("read_sums", C.c_int32(which), abi.as_ptr(out, C.c_double), out.size)
        return out

    def device_f(self):
        p = C.c_void_p()
        es = C.c_int32()
        self._call("device_f", C.byref(p), C.byref(es))
        return p.value, es.value

    def velocity_permutation(self) -> np.ndarray:
        out = np.empty(self.nv, dtype=np.int32)
        self._call("velocity_permutation", abi.as_ptr(out, C.c_int32), out.size)
        return out

    def schedule_info(self):
        a, b = C.c_int32(), C.c_int32()
        self._call("schedule_info", C.byref(a), C.byref(b))
        return a.value, b.value

    def take_timings(self) -> dict:
        t = abi.KinStepTimings()
        self._call("take_timings", C.byref(t))
        return {k: getattr(t, k) for k, _ in abi.KinStepTimings._fields_}

    def memory_bytes(self) -> int:
        out = C.c_uint64()
        self._call("memory_bytes", C.byref(out))
        return out.value

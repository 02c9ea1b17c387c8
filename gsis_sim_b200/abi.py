"""ctypes mirror of the C ABI in include/gsis_b200.h.

`SetupArrays` is the host-side form of a `KinSetupDesc`: every array the backend needs from the reference's
`KineticSetup` (src/kinetic/kinetic_setup.hpp:56-115), kept alive in numpy so that a descriptor can point into
it. The same descriptor feeds the CUDA library and (in tests) the CPU checkers.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

KIN_ABI_VERSION = 2
KIN_OK = 0
KIN_E_ARG, KIN_E_CUDA, KIN_E_MEMORY, KIN_E_STATE, KIN_E_TIMEOUT = -1, -2, -3, -4, -5
KIN_NOALLOC_MAX_STATES = 4096
KIN_SUMS_MOMENTS, KIN_SUMS_BOUNDARY, KIN_SUMS_RESIDUAL = 0, 1, 2
KIN_PREC_FP32, KIN_PREC_FP64, KIN_PREC_MIXED = 0, 1, 2
PRECISIONS = {"fp32": KIN_PREC_FP32, "fp64": KIN_PREC_FP64, "mixed": KIN_PREC_MIXED}

# BoundaryKind (src/kinetic/kinetic_types.hpp:19-26)
BC_DIFFUSE_WALL, BC_PRESSURE, BC_VACUUM, BC_SYMMETRY, BC_PERIODIC, BC_MAXWELL_WALL = 0, 1, 2, 3, 4, 5
# LimiterMode (src/kinetic/kinetic_types.hpp:101-105)
LIMITER_NONE, LIMITER_VENKAT_ABSOLUTE, LIMITER_VENKAT_RELATIVE = 0, 1, 2
# gsis_negative_check (src/kinetic/kinetic_kernels.hpp:584-587)
NEGATIVE_MODES = {"all": 0, "created": 1, "limit": 2, "blend": 3}

MOMENTS_PER_CELL = 15
BOUNDARY_SUMS_PER_FACE = 20

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)
_up = C.POINTER(C.c_uint8)


class KinSetupDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("precision", C.c_int32), ("device", C.c_int32),
        ("n_cells", C.c_int32), ("nv", C.c_int32), ("n_bfaces", C.c_int32), ("n_blocks", C.c_int32),
        ("xi_x", _dp), ("xi_y", _dp), ("xi_z", _dp), ("weights", _dp), ("weight", C.c_double),
        ("csr_offsets", _ip), ("csr_other", _ip), ("csr_bface", _ip), ("csr_geom", _dp), ("eps2", _dp),
        ("bface_owner", _ip), ("bface_kind", _ip), ("bface_mirror_xor", _ip), ("bface_patch", _ip),
        ("bface_geom", _dp),
        ("volume", _dp), ("vdt", _dp),
        ("block_offsets", _ip), ("n_sweep_dirs", C.c_int32), ("sweep_order", _ip), ("sweep_pos", _ip),
        ("sweep_dir_of", _up),
        ("limiter_mode", C.c_int32), ("positivity", C.c_int32), ("diag_scale", C.c_double),
        ("interface_damping", C.c_double), ("block_passes", C.c_int32), ("negative_check_mode", C.c_int32),
        ("velocity_chunk", C.c_int64),
        ("mu0", C.c_double), ("omega", C.c_double), ("Pr", C.c_double), ("cold_bgk_temperature", C.c_double),
        ("discrete_eq", C.c_int32), ("deq_fallback_collisionless", C.c_int32),
        ("deq_lo", C.c_double * 3), ("deq_hi", C.c_double * 3), ("deq_d", C.c_double * 3),
        ("deq_criterion", C.c_double), ("deq_tolerance", C.c_double), ("deq_max_iterations", C.c_int32),
        ("n_maxwell_faces", C.c_int32), ("maxwell_offset", _lp), ("maxwell_specular_fraction", _dp),
        ("grid_to_storage", _ip), ("grid_n", C.c_int32 * 3),
        ("deq_nv", C.c_int32), ("deq_xi_x", _dp), ("deq_xi_y", _dp), ("deq_xi_z", _dp), ("deq_weights", _dp),
    ]


class KinInflowState(C.Structure):
    _fields_ = [("scale", C.c_double), ("rho", C.c_double), ("ux", C.c_double), ("uy", C.c_double),
                ("uz", C.c_double), ("T", C.c_double)]


class KinStepTimings(C.Structure):
    _fields_ = [("moments", C.c_double), ("boundary", C.c_double), ("gradient", C.c_double),
                ("residual", C.c_double), ("sweep_forward", C.c_double), ("sweep_backward", C.c_double),
                ("other", C.c_double)]


class KinDeqCounts(C.Structure):
    _fields_ = [("corrected", C.c_int64), ("failed", C.c_int64), ("max_iterations", C.c_int32)]


_ARRAY_DTYPES = {
    "xi_x": np.float64, "xi_y": np.float64, "xi_z": np.float64, "weights": np.float64,
    "csr_offsets": np.int32, "csr_other": np.int32, "csr_bface": np.int32, "csr_geom": np.float64,
    "eps2": np.float64, "bface_owner": np.int32, "bface_kind": np.int32, "bface_mirror_xor": np.int32,
    "bface_patch": np.int32, "bface_geom": np.float64, "volume": np.float64, "vdt": np.float64,
    "block_offsets": np.int32, "sweep_order": np.int32, "sweep_pos": np.int32, "sweep_dir_of": np.uint8,
    "maxwell_offset": np.int64, "maxwell_specular_fraction": np.float64, "grid_to_storage": np.int32,
    "deq_xi_x": np.float64, "deq_xi_y": np.float64, "deq_xi_z": np.float64, "deq_weights": np.float64,
}
_SCALARS = [
    "precision", "device", "n_cells", "nv", "n_bfaces", "n_blocks", "weight", "n_sweep_dirs", "limiter_mode",
    "positivity", "diag_scale", "interface_damping", "block_passes", "negative_check_mode", "velocity_chunk",
    "mu0", "omega", "Pr", "cold_bgk_temperature", "discrete_eq", "deq_fallback_collisionless", "deq_criterion",
    "deq_tolerance", "deq_max_iterations", "n_maxwell_faces", "deq_nv",
]
_VEC3 = ["deq_lo", "deq_hi", "deq_d", "grid_n"]


@dataclass
class SetupArrays:
    """Flat arrays + scalars of one kinetic setup (internal numbering, reference storage order)."""
    arrays: dict = field(default_factory=dict)
    scalars: dict = field(default_factory=dict)

    def __getitem__(self, k):
        if k in self.arrays:
            return self.arrays[k]
        return self.scalars[k]

    def __setitem__(self, k, v):
        if k in _ARRAY_DTYPES:
            self.arrays[k] = None if v is None else np.ascontiguousarray(v, dtype=_ARRAY_DTYPES[k])
        else:
            self.scalars[k] = v

    def get(self, k, default=None):
        try:
            return self[k]
        except KeyError:
            return default

    @property
    def n_cells(self) -> int:
        return int(self.scalars["n_cells"])

    @property
    def nv(self) -> int:
        return int(self.scalars["nv"])

    @property
    def n_bfaces(self) -> int:
        return int(self.scalars["n_bfaces"])

    def copy(self) -> "SetupArrays":
        return SetupArrays({k: (None if v is None else v.copy()) for k, v in self.arrays.items()},
                           {k: (list(v) if isinstance(v, (list, tuple)) else v) for k, v in self.scalars.items()})

    def desc(self) -> KinSetupDesc:
        """A KinSetupDesc pointing into these arrays (keep this object alive while the descriptor is used)."""
        d = KinSetupDesc()
        d.abi_version = KIN_ABI_VERSION
        for k in _SCALARS:
            setattr(d, k, self.scalars.get(k, 0))
        for k in _VEC3:
            v = self.scalars.get(k, (0, 0, 0))
            arr = getattr(d, k)
            for a in range(3):
                arr[a] = v[a]
        for k, dt in _ARRAY_DTYPES.items():
            a = self.arrays.get(k)
            if a is None:
                continue
            ctype = {np.float64: C.c_double, np.int32: C.c_int32, np.int64: C.c_int64, np.uint8: C.c_uint8}[dt]
            setattr(d, k, a.ctypes.data_as(C.POINTER(ctype)))
        return d

    @classmethod
    def from_desc(cls, d: KinSetupDesc) -> "SetupArrays":
        """Copy the arrays a descriptor points to (sizes derived from its scalars)."""
        s = cls()
        for k in _SCALARS:
            s.scalars[k] = getattr(d, k)
        for k in _VEC3:
            s.scalars[k] = tuple(getattr(d, k)[a] for a in range(3))
        nc, nv, nb = d.n_cells, d.nv, d.n_bfaces
        n_csr = d.csr_offsets[nc]
        nd = d.n_sweep_dirs
        sizes = {
            "xi_x": nv, "xi_y": nv, "xi_z": nv, "weights": nv, "csr_offsets": nc + 1, "csr_other": n_csr,
            "csr_bface": n_csr, "csr_geom": 12 * n_csr, "eps2": nc, "bface_owner": nb, "bface_kind": nb,
            "bface_mirror_xor": nb, "bface_patch": nb, "bface_geom": 7 * nb, "volume": nc, "vdt": nc,
            "block_offsets": d.n_blocks + 1, "sweep_order": nd * nc, "sweep_pos": nd * nc,
            "sweep_dir_of": nv if nd > 0 else 0, "maxwell_offset": nb, "maxwell_specular_fraction": nb,
            "grid_to_storage": nv, "deq_xi_x": d.deq_nv, "deq_xi_y": d.deq_nv, "deq_xi_z": d.deq_nv,
            "deq_weights": d.deq_nv,
        }
        for k, n in sizes.items():
            p = getattr(d, k)
            if not p or n == 0:
                s.arrays[k] = None
                continue
            s.arrays[k] = np.ctypeslib.as_array(p, shape=(n,)).astype(_ARRAY_DTYPES[k], copy=True)
        return s

    def to_npz_dict(self, prefix: str = "setup.") -> dict:
        out = {}
        for k, v in self.arrays.items():
            if v is not None:
                out[prefix + k] = v
        for k, v in self.scalars.items():
            out[prefix + "scalar." + k] = np.asarray(v)
        return out

    @classmethod
    def from_npz(cls, z, prefix: str = "setup.") -> "SetupArrays":
        s = cls()
        for name in z.files:
            if not name.startswith(prefix):
                continue
            k = name[len(prefix):]
            if k.startswith("scalar."):
                v = z[name]
                k = k[len("scalar."):]
                s.scalars[k] = tuple(v.tolist()) if v.ndim else v.item()
            else:
                s.arrays[k] = np.ascontiguousarray(z[name])
        return s


def as_ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def inflow_array(states: np.ndarray):
    """(n, 6) float64 array of (scale, rho, ux, uy, uz, T) -> ctypes array of KinInflowState."""
    states = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 6)
    arr = (KinInflowState * max(len(states), 1))()
    C.memmove(arr, states.ctypes.data, states.nbytes)
    return arr


def declare_backend_api(lib, prefix: str, handle_type=C.c_void_p):
    """Set argtypes/restype of the kin_* style entry points of `lib` (prefix "kin_" or "ref_kin_")."""
    h = handle_type
    sig = {
        "set_equilibrium": [h, _dp, C.c_int64],
        "set_distribution": [h, _dp, C.c_int64],
        "get_distribution": [h, _dp, C.c_int64],
        "compute_moments": [h, _dp, C.c_int64],
        "scale_distribution": [h, C.c_double],
        "update_cell_params": [h],
        "set_inflow": [h, C.POINTER(KinInflowState), C.c_int64],
        "boundary_sums": [h, _dp, C.c_int64],
        "sweep": [h, _dp, C.c_int64],
        "gsis_correction": [h, _dp, _dp, C.c_int64, _ip, _lp],
        "gsis_correction_extrema": [h, _dp, _dp, C.c_int64, _dp, C.c_int64],
        "device_sums": [h, C.c_int32, C.POINTER(_dp), _lp],
        "finalize_moments": [h, _dp, C.c_int64],
        "read_sums": [h, C.c_int32, _dp, C.c_int64],
        "gsis_correction_apply": [h, _dp, _dp, C.c_int64, _dp, C.c_int64, _ip, _lp],
        "internal_face_mass_flux": [h, _ip, _ip, C.c_int64, _dp],
        "deq_counts": [h, C.POINTER(KinDeqCounts)],
        "chunk_width": [h, _ip],
        "discrete_maxwell": [h, _dp, C.c_int64, C.c_double, _dp, _ip],
        "discrete_maxwell_noalloc": [h, _dp, C.c_int64, C.c_double, _dp, _ip],
        "moment_sums": [h, _dp, C.c_int64],
        "set_moments": [h, _dp, C.c_int64],
        "adjoint_begin": [h, _ip, _ip, C.c_int64, _ip, _ip],
        "adjoint_set": [h, _dp, C.c_int64],
        "adjoint_get": [h, _dp, C.c_int64],
        "adjoint_reduce": [h, _dp, C.c_int64, _dp, C.c_int64, _dp, C.c_int64],
        "adjoint_face_moment_seeds": [h, _dp, C.c_int64],
        "adjoint_update": [h, _dp, C.c_int64, _dp, C.c_int64, C.c_int32, _dp, C.c_int64],
        "adjoint_end": [h],
    }
    for name, args in sig.items():
        if not hasattr(lib, prefix + name):
            continue
        fn = getattr(lib, prefix + name)
        fn.argtypes = args
        fn.restype = C.c_int

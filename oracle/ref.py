"""ctypes wrapper of oracle/_ref/libgsisref.so — the reference's own CPU kinetic path (TEST INFRASTRUCTURE).

Only tests/, tests/golden/make_golden.py and bench.py's CPU-baseline leg use this module. It builds cases of the
reference (box meshes of tests/support/box_mesh.cpp or meshes given as arrays), exports the reference
`KineticSetup` as `SetupArrays`, and runs the reference `KineticSolver` (src/kinetic/kinetic_solver.cpp) and
`CpuBackend` (src/kinetic/kinetic_backend_cpu.cpp).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from gsis_sim_b200 import abi
from gsis_sim_b200.backend import KineticBackendABI, KineticError

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libgsisref.so")
# the reference KineticSolver linked with the B200 KineticBackend shim (gsis_sim_b200/integration/b200_backend.cpp)
DROPIN_PATH = os.path.join(HERE, "_ref", "libgsisdropin.so")
# the reference KineticSolver on the reference's own CudaBackend, rebuilt for sm_100a (bench.py's GPU baseline)
REFCUDA_PATH = os.path.join(HERE, "_ref", "libgsisrefcuda.so")
_libs = {}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)


def _path(dropin: bool, refcuda: bool) -> str:
    return REFCUDA_PATH if refcuda else (DROPIN_PATH if dropin else LIB_PATH)


def available(dropin: bool = False, refcuda: bool = False) -> bool:
    return os.path.exists(_path(dropin, refcuda))


def lib(dropin: bool = False, refcuda: bool = False):
    path = _path(dropin, refcuda)
    if path in _libs:
        return _libs[path]
    L = C.CDLL(path)
    L.ref_error.restype = C.c_char_p
    L.ref_mesh_box.argtypes = [C.c_char_p]
    L.ref_mesh_box.restype = C.c_void_p
    L.ref_mesh_arrays.argtypes = [C.c_int32, _dp, C.c_int32, _lp, _ip, _ip, C.c_int32, _ip, C.c_int32, C.c_int32,
                                  C.c_char_p, _ip, _ip]
    L.ref_mesh_arrays.restype = C.c_void_p
    L.ref_mesh_free.argtypes = [C.c_void_p]
    L.ref_mesh_sizes.argtypes = [C.c_void_p, _lp]
    L.ref_mesh_export.argtypes = [C.c_void_p, _dp, _lp, _ip, _ip, _ip, _ip, _ip, C.c_char_p, C.c_int32, _dp, _dp,
                                  _dp, _dp]
    L.ref_case_create.argtypes = [C.c_void_p, C.c_char_p]
    L.ref_case_create.restype = C.c_void_p
    L.ref_case_free.argtypes = [C.c_void_p]
    L.ref_case_desc.argtypes = [C.c_void_p, C.POINTER(abi.KinSetupDesc)]
    L.ref_case_info.argtypes = [C.c_void_p, _lp, _dp]
    L.ref_case_maps.argtypes = [C.c_void_p, _ip, _ip, _ip, _ip, _dp]
    L.ref_case_geometry.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _ip, _dp, _ip]
    L.ref_solver_init_uniform.argtypes = [C.c_void_p] + [C.c_double] * 5
    L.ref_solver_init_states.argtypes = [C.c_void_p, _dp]
    L.ref_solver_prepare.argtypes = [C.c_void_p, _dp]
    L.ref_solver_sweep.argtypes = [C.c_void_p, C.c_int, _dp]
    L.ref_solver_patch_mass_flow.argtypes = [C.c_void_p, _dp]
    L.ref_solver_last_timings.argtypes = [C.c_void_p, _dp]
    L.ref_solver_moments.argtypes = [C.c_void_p, _dp]
    L.ref_solver_boundary_fluxes.argtypes = [C.c_void_p, _dp, _dp, _dp]
    L.ref_solver_distribution.argtypes = [C.c_void_p, _dp]
    L.ref_solver_set_distribution.argtypes = [C.c_void_p, _dp, C.c_int64]
    L.ref_solver_gsis_correction.argtypes = [C.c_void_p, _dp, _dp, _lp]
    L.ref_solver_section_mass_flow.argtypes = [C.c_void_p, C.c_int32, _dp, C.c_int32, _dp]
    abi.declare_backend_api(L, "ref_kin_")
    _libs[path] = L
    return L


def _check(rc, L=None):
    if rc != 0:
        raise KineticError((L or lib()).ref_error().decode())


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


class RefMesh:
    """A reference PolyMesh + geometry (LoadedMesh)."""

    def __init__(self, handle):
        if not handle:
            raise KineticError(lib().ref_error().decode())
        self.h = handle

    @classmethod
    def box(cls, n, lo, hi, patches, distortion=0.0, tetrahedra=False, seed=1):
        spec = (f"mesh.n = {n[0]} {n[1]} {n[2]}\nmesh.lo = {lo[0]!r} {lo[1]!r} {lo[2]!r}\n"
                f"mesh.hi = {hi[0]!r} {hi[1]!r} {hi[2]!r}\nmesh.patches = {' '.join(patches)}\n"
                f"mesh.distortion = {distortion!r}\nmesh.tetrahedra = {int(tetrahedra)}\nmesh.seed = {seed}\n")
        return cls(lib().ref_mesh_box(spec.encode()))

    @classmethod
    def from_arrays(cls, m: dict):
        pts = np.ascontiguousarray(m["points"], dtype=np.float64)
        fo = np.ascontiguousarray(m["face_offsets"], dtype=np.int64)
        fn = np.ascontiguousarray(m["face_nodes"], dtype=np.int32)
        ow = np.ascontiguousarray(m["owner"], dtype=np.int32)
        nb = np.ascontiguousarray(m["neighbour"], dtype=np.int32)
        ps = np.ascontiguousarray(m["patch_start"], dtype=np.int32)
        pc = np.ascontiguousarray(m["patch_count"], dtype=np.int32)
        names = "".join(n + "\n" for n in m["patch_names"]).encode()
        h = lib().ref_mesh_arrays(len(pts) // 3 if pts.ndim == 1 else len(pts), _p(pts), len(ow), _p(fo, C.c_int64),
                                  _p(fn, C.c_int32), _p(ow, C.c_int32), len(nb), _p(nb, C.c_int32),
                                  int(m["n_cells"]), len(ps), names, _p(ps, C.c_int32), _p(pc, C.c_int32))
        return cls(h)

    def export(self) -> dict:
        s = np.zeros(6, dtype=np.int64)
        lib().ref_mesh_sizes(self.h, _p(s, C.c_int64))
        n_points, n_faces, n_int, n_fn, n_cells, n_patches = (int(x) for x in s)
        out = dict(points=np.zeros((n_points, 3)), face_offsets=np.zeros(n_faces + 1, np.int64),
                   face_nodes=np.zeros(n_fn, np.int32), owner=np.zeros(n_faces, np.int32),
                   neighbour=np.zeros(n_int, np.int32), patch_start=np.zeros(n_patches, np.int32),
                   patch_count=np.zeros(n_patches, np.int32), cell_volume=np.zeros(n_cells),
                   cell_center=np.zeros((n_cells, 3)), face_area_vector=np.zeros((n_faces, 3)),
                   face_center=np.zeros((n_faces, 3)))
        names = C.create_string_buffer(64 * n_patches + 64)
        _check(lib().ref_mesh_export(self.h, _p(out["points"]), _p(out["face_offsets"], C.c_int64),
                                     _p(out["face_nodes"], C.c_int32), _p(out["owner"], C.c_int32),
                                     _p(out["neighbour"], C.c_int32), _p(out["patch_start"], C.c_int32),
                                     _p(out["patch_count"], C.c_int32), names, len(names),
                                     _p(out["cell_volume"]), _p(out["cell_center"]), _p(out["face_area_vector"]),
                                     _p(out["face_center"])))
        out["patch_names"] = names.value.decode().split("\n")[:n_patches]
        out["n_cells"] = n_cells
        return out

    def __del__(self):
        if getattr(self, "h", None) and LIB_PATH in _libs:
            _libs[LIB_PATH].ref_mesh_free(self.h)
            self.h = None


def case_spec(bcs, Kn=None, delta_rp=None, nv=(10, 10, 10), vmax=5.0, vlo=None, vhi=None, kinetic=None,
              omega=0.66, molecular_mass=6.65e-27, mu_ref=1.916e-5, T_ref=273.15, T0=273.15, L_ref=1.0) -> str:
    """Config text for ref_case_create (same gas and conditions as tests/kinetic/kinetic_test_cases.cpp:9-32).

    bcs: list of (patch, type, dict(T=, p=, u=(x,y,z), alpha=)) with nondimensional values."""
    lo = vlo if vlo is not None else (-vmax,) * 3
    hi = vhi if vhi is not None else (vmax,) * 3
    lines = [f"gas.molecular_mass = {molecular_mass!r}", f"gas.mu_ref = {mu_ref!r}", f"gas.T_ref = {T_ref!r}",
             f"gas.omega = {omega!r}", f"conditions.L_ref = {L_ref!r}", f"conditions.T0 = {T0!r}",
             f"velocity_grid.n = {nv[0]} {nv[1]} {nv[2]}", f"velocity_grid.lo = {lo[0]!r} {lo[1]!r} {lo[2]!r}",
             f"velocity_grid.hi = {hi[0]!r} {hi[1]!r} {hi[2]!r}"]
    if Kn is not None:
        lines.append(f"conditions.Kn = {Kn!r}")
    if delta_rp is not None:
        lines.append(f"conditions.delta_rp = {delta_rp!r}")
    for patch, typ, o in bcs:
        parts = [patch, typ]
        if "T" in o:
            parts.append(f"T={o['T']!r}")
        if "p" in o:
            parts.append(f"p={o['p']!r}")
        if "u" in o:
            u = o["u"]
            parts.append(f"u={u[0]!r},{u[1]!r},{u[2]!r}")
        if "alpha" in o:
            parts.append(f"alpha={o['alpha']!r}")
        if "mdot" in o:  # mass_flow_inlet: nondimensional target mass flow, inflow positive
            parts.append(f"mdot={o['mdot']!r}")
        lines.append("boundary = " + " ".join(parts))
    for k, v in (kinetic or {}).items():
        if isinstance(v, bool):
            v = "true" if v else "false"
        elif isinstance(v, str):
            v = f'"{v}"'
        elif isinstance(v, float):
            v = repr(v) if ("." in repr(v) or "e" in repr(v)) else repr(v) + ".0"
        lines.append(f"kinetic.{k} = {v}")
    return "\n".join(lines) + "\n"


class RefCase:
    """The reference KineticSolver (backend = "cpu") on one mesh + config, and a separate CpuBackend."""

    def __init__(self, mesh: RefMesh, spec: str, dropin: bool = False, refcuda: bool = False):
        self.mesh = mesh
        self.L = lib(dropin, refcuda)
        if dropin or refcuda:
            # the drop-in / reference-CUDA library has its own copy of the mesh types: rebuild the mesh there
            self._mesh_arrays = mesh.export()
            m = self._mesh_arrays
            pts = np.ascontiguousarray(m["points"], dtype=np.float64)
            names = "".join(n + "\n" for n in m["patch_names"]).encode()
            self._dmesh = self.L.ref_mesh_arrays(len(pts), _p(pts), len(m["owner"]), _p(m["face_offsets"], C.c_int64),
                                                 _p(m["face_nodes"], C.c_int32), _p(m["owner"], C.c_int32),
                                                 len(m["neighbour"]), _p(m["neighbour"], C.c_int32), int(m["n_cells"]),
                                                 len(m["patch_start"]), names, _p(m["patch_start"], C.c_int32),
                                                 _p(m["patch_count"], C.c_int32))
            if not self._dmesh:
                raise KineticError(self.L.ref_error().decode())
            self.h = self.L.ref_case_create(self._dmesh, spec.encode())
        else:
            self.h = self.L.ref_case_create(mesh.h, spec.encode())
        if not self.h:
            raise KineticError(self.L.ref_error().decode())
        d = abi.KinSetupDesc()
        self._chk(self.L.ref_case_desc(self.h, C.byref(d)))
        self.setup = abi.SetupArrays.from_desc(d)
        iout = np.zeros(8, np.int64)
        dout = np.zeros(8)
        self._chk(self.L.ref_case_info(self.h, _p(iout, C.c_int64), _p(dout)))
        self.n_csr, closed, self.n_patches, self.n_internal_faces = (int(x) for x in iout[:4])
        self.inner_sweeps, self.inner_wall_update, self.boundary_iterations, self.orbit_size = \
            int(iout[4]), bool(iout[5]), int(iout[6]), int(iout[7])
        self.closed_domain = bool(closed)
        (self.length_scale, self.gamma, self.limiter_k, self.wall_relaxation, self.convergence_u_floor,
         self.mass_flow_scale, self.mu_hat0, self.xi_max) = (float(x) for x in dout)
        nc, nb, nv = self.setup.n_cells, self.setup.n_bfaces, self.setup.nv
        self.cell_new_to_old = np.zeros(nc, np.int32)
        self.bface_new_to_old = np.zeros(nb, np.int32)
        self.storage_to_grid = np.zeros(nv, np.int32)
        self.patch_int = np.zeros((self.n_patches, 4), np.int32)
        self.patch_dbl = np.zeros((self.n_patches, 7))
        self._chk(self.L.ref_case_maps(self.h, _p(self.cell_new_to_old, C.c_int32), _p(self.bface_new_to_old, C.c_int32),
                                   _p(self.storage_to_grid, C.c_int32), _p(self.patch_int, C.c_int32),
                                   _p(self.patch_dbl)))
        n_faces = self.n_internal_faces + nb
        self.geom = dict(cell_center=np.zeros((nc, 3)), face_center=np.zeros((n_faces, 3)),
                         face_normal=np.zeros((n_faces, 3)), face_area=np.zeros(n_faces),
                         owner=np.zeros(n_faces, np.int32), lsq=np.zeros((self.n_csr, 3)),
                         csr_faces=np.zeros(self.n_csr, np.int32))
        g = self.geom
        self._chk(self.L.ref_case_geometry(self.h, _p(g["cell_center"]), _p(g["face_center"]), _p(g["face_normal"]),
                                       _p(g["face_area"]), _p(g["owner"], C.c_int32), _p(g["lsq"]),
                                       _p(g["csr_faces"], C.c_int32)))
        self.backend = RefBackend(self)

    def _chk(self, rc):
        if rc != 0:
            raise KineticError(self.L.ref_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_case_free(self.h)
            self.h = None

    # --- reference KineticSolver ------------------------------------------------------------------------------
    def init_uniform(self, rho, u, T):
        self._chk(self.L.ref_solver_init_uniform(self.h, rho, u[0], u[1], u[2], T))

    def init_states(self, states_orig):
        s = np.ascontiguousarray(states_orig, dtype=np.float64)
        self._chk(self.L.ref_solver_init_states(self.h, _p(s)))

    def prepare(self):
        info = np.zeros(12)
        self._chk(self.L.ref_solver_prepare(self.h, _p(info)))
        return info

    def sweep(self, update_pressure=True):
        info = np.zeros(12)
        self._chk(self.L.ref_solver_sweep(self.h, int(update_pressure), _p(info)))
        return info

    def last_timings(self) -> dict:
        """Backend times of the last CIS iteration (StepTimings, src/kinetic/kinetic_backend.hpp:18-40), seconds."""
        out = np.zeros(7)
        self._chk(self.L.ref_solver_last_timings(self.h, _p(out)))
        return dict(zip(["moments", "boundary", "gradient", "residual", "sweep_forward", "sweep_backward", "other"],
                        (float(x) for x in out)))

    def patch_mass_flow(self):
        out = np.zeros(self.n_patches)
        self._chk(self.L.ref_solver_patch_mass_flow(self.h, _p(out)))
        return out

    def moments(self):
        out = np.zeros((self.setup.n_cells, 15))
        self._chk(self.L.ref_solver_moments(self.h, _p(out)))
        return out

    def boundary_fluxes(self):
        nb = self.setup.n_bfaces
        fp, fm, fs = np.zeros((nb, 5)), np.zeros((nb, 5)), np.zeros((nb, 5))
        self._chk(self.L.ref_solver_boundary_fluxes(self.h, _p(fp), _p(fm), _p(fs)))
        return fp, fm, fs

    def distribution(self):
        out = np.zeros((self.setup.n_cells, self.setup.nv))
        self._chk(self.L.ref_solver_distribution(self.h, _p(out)))
        return out

    def set_distribution(self, f):
        a = np.ascontiguousarray(f, dtype=np.float64).ravel()
        self._chk(self.L.ref_solver_set_distribution(self.h, _p(a), a.size))

    def gsis_correction(self, w_half_orig, w_new_orig):
        a = np.ascontiguousarray(w_half_orig, dtype=np.float64)
        b = np.ascontiguousarray(w_new_orig, dtype=np.float64)
        r = C.c_int64()
        self._chk(self.L.ref_solver_gsis_correction(self.h, _p(a), _p(b), C.byref(r)))
        return r.value

    def section_mass_flow(self, positions, axis=0):
        p = np.ascontiguousarray(positions, dtype=np.float64)
        out = np.zeros(len(p))
        self._chk(self.L.ref_solver_section_mass_flow(self.h, axis, _p(p), len(p), _p(out)))
        return out


class RefBackend(KineticBackendABI):
    """The backend of a RefCase (the reference CpuBackend<F>; in the drop-in build the B200 shim), called operation
    by operation."""

    def __init__(self, case: RefCase):
        super().__init__(case.L, "ref_kin_", C.c_void_p(case.h), case.setup, lambda: case.L.ref_error().decode())
        self._case = case


def tube_spec(nv: int, precision: str = "fp64", delta: float = 10.0, p_out: float = 0.01, vmax: float = 5.0,
              **kinetic) -> str:
    """Config text of the tube case (gsis_sim_b200.tube.tube_case) for the reference solver: inlet p 1, T 1,
    outlet p_out, diffuse walls T 1, omega 0.81, uniform nv^3 velocities on [-vmax, vmax]^3."""
    kin = {"precision": precision}
    kin.update(kinetic)
    return case_spec([("inlet", "pressure_inlet", dict(T=1.0, p=1.0)), ("wall", "diffuse_wall", dict(T=1.0)),
                      ("back", "diffuse_wall", dict(T=1.0)), ("outlet", "pressure_outlet", dict(p=p_out))],
                     delta_rp=delta, nv=(nv,) * 3, vmax=vmax, omega=0.81, kinetic=kin)


class HostArrays(dict):
    """Host-side data of a RefCase in the key layout of the golden fixtures (HostSetup.from_npz reads it)."""

    @property
    def files(self):
        return list(self.keys())


def host_arrays(case: RefCase) -> HostArrays:
    """Host-side data of the kinetic host loop (kinetic_solver.cpp) of a RefCase, internal numbering."""
    g = case.geom
    return HostArrays({
        "host.cell_new_to_old": case.cell_new_to_old, "host.bface_new_to_old": case.bface_new_to_old,
        "host.storage_to_grid": case.storage_to_grid, "host.patch_int": case.patch_int,
        "host.patch_dbl": case.patch_dbl, "host.cell_center": g["cell_center"], "host.face_center": g["face_center"],
        "host.face_normal": g["face_normal"], "host.face_area": g["face_area"], "host.owner": g["owner"],
        "host.lsq": g["lsq"], "host.csr_faces": g["csr_faces"],
        "host.scalars": np.array([case.length_scale, case.gamma, case.limiter_k, case.wall_relaxation,
                                  case.convergence_u_floor, case.mass_flow_scale, case.mu_hat0, case.xi_max]),
        "host.iscalars": np.array([case.n_internal_faces, int(case.closed_domain), case.inner_sweeps,
                                   int(case.inner_wall_update), case.boundary_iterations, case.orbit_size]),
    })

"""Host loop of the kinetic solver (CIS) over a backend.

Mirrors the reference's `KineticSolver` (src/kinetic/kinetic_solver.hpp:61-115, kinetic_solver.cpp): moments,
positivity check and closed-domain mass scaling, convergence measure eps (eq. 59), cell parameters, pressure-boundary
inflow states by limited reconstruction (App. A.2), boundary sums -> rho_Gamma, F+/-, face states and patch mass
flows, inner sweeps with wall refresh, residual norm, GSIS correction and numbering maps. Inputs and outputs of the
public methods use the ORIGINAL mesh numbering (as the reference); the backend works in the internal numbering.
The per-face loops of the reference are vectorised over faces; the discrete-Maxwellian correction of inflow
states runs on the backend (batched kin_discrete_maxwell) instead of a host loop over faces x velocities.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .kinetic_setup import BOUNDARY_TYPES, HostSetup

T_PRESSURE_INLET = BOUNDARY_TYPES.index("pressure_inlet")
T_MASS_FLOW_INLET = BOUNDARY_TYPES.index("mass_flow_inlet")
T_PRESSURE_OUTLET = BOUNDARY_TYPES.index("pressure_outlet")
T_VACUUM = BOUNDARY_TYPES.index("vacuum")


class KineticSolverError(RuntimeError):
    pass


def summarize_patches(names, types, patch_faces, area, normal, F_plus, F_minus, face_state, patch_dbl=None,
                      patch_target=None, length=1.0, ref_pressure=0.0, ref_velocity=0.0) -> list:
    """Per-patch boundary flows (summarize_kinetic_patches, src/kinetic/kinetic_output.cpp:198-268).

    names, types: patch names and BoundaryType names; patch_faces: per patch the boundary-face indices of the arrays
    below; area (nondimensional, per face), normal (outward unit normals), F_plus / F_minus (mass, momentum (3),
    energy fluxes through the face, outward positive) and face_state (rho, u (3), T) per face. Returns one dict per
    patch: the net nondimensional fluxes (outward positive), the area-averaged face state and, when the reference
    scales are given (length L_ref, p_ref, sqrt(R T0)), SI flows with flow INTO the domain positive: mass (kg/s),
    heat (W; the third central moment in the face's local rest frame), total energy (W), and the force (N)."""
    si = ref_pressure > 0.0 and ref_velocity > 0.0
    L2 = length * length
    mass_flux, heat_flux = ref_pressure / ref_velocity if si else 0.0, ref_pressure * ref_velocity
    out = []
    for pi, faces in enumerate(patch_faces):
        faces = np.asarray(faces, np.int64)
        A = area[faces]
        Fs = F_plus[faces] + F_minus[faces]
        F = Fs.sum(axis=0) if len(faces) else np.zeros(5)
        w = face_state[faces]
        u = w[:, 1:4]
        un = np.sum(u * normal[faces], axis=1)
        heat = float(np.sum(Fs[:, 4] - np.sum(u * Fs[:, 1:4], axis=1) + 0.5 * np.sum(u * u, axis=1) * Fs[:, 0]
                            - 1.5 * w[:, 0] * w[:, 4] * un * A))
        a = float(A.sum())
        p = {"name": names[pi], "type": types[pi], "faces": int(len(faces)), "area_nd": a, "mdot_nd": float(F[0]),
             "momentum_flux_nd": [float(x) for x in F[1:4]], "energy_flux_nd": float(F[4])}
        if types[pi] == "maxwell_wall" and patch_dbl is not None:
            p["accommodation"] = float(patch_dbl[pi, 5])
        if types[pi] == "mass_flow_inlet" and patch_target is not None:
            # nondimensional: written with or without the SI scales (kinetic_output.cpp:233-237)
            p["mass_flow_relative_error"] = abs(float(F[0]) + patch_target[pi]) / patch_target[pi]
        if si:
            p["mdot_kg_s"] = float(F[0]) * mass_flux * L2
            if types[pi] == "mass_flow_inlet" and patch_dbl is not None and patch_target is not None:
                p["pressure_Pa"] = float(patch_dbl[pi, 1]) * ref_pressure
                p["target_mass_flow_kg_s"] = float(patch_target[pi]) * mass_flux * L2
            p["area_m2"] = a * L2
            p["mass_flow_kg_s"] = -float(F[0]) * mass_flux * L2
            p["heat_flow_W"] = -heat * heat_flux * L2
            p["energy_flow_W"] = -float(F[4]) * heat_flux * L2
            p["force_N"] = [float(x) * ref_pressure * L2 for x in F[1:4]]
        if a > 0.0:
            p["face_rho_nd"] = float(np.sum(A * w[:, 0]) / a)
            p["face_u_nd"] = [float(np.sum(A * w[:, k]) / a) for k in (1, 2, 3)]
            p["face_T_nd"] = float(np.sum(A * w[:, 4]) / a)
        out.append(p)
    return out


@dataclass
class IterationInfo:
    """KineticIterationInfo (src/kinetic/kinetic_solver.hpp:37-59)."""
    iteration: int = 0
    epsilon: float = 0.0
    eps_rho: float = 0.0
    eps_u: float = 0.0
    eps_T: float = 0.0
    has_epsilon: bool = False
    residual: float = 0.0
    has_residual: bool = False
    total_mass: float = 0.0
    mass_scale: float = 1.0
    patch_mass_flow: np.ndarray = field(default_factory=lambda: np.zeros(0))
    seconds: float = 0.0
    deq_corrected: int = 0
    deq_failed: int = 0


class KineticSolver:
    def __init__(self, setup: abi.SetupArrays, host: HostSetup, backend):
        self.s = setup
        self.h = host
        self.backend = backend
        nc, nb = setup.n_cells, setup.n_bfaces
        self.nc, self.nb, self.nv = nc, nb, setup.nv
        self.iteration = 0
        self.version = 0
        self.prepared_version = -1
        self.info = IterationInfo()
        self.moments_ = np.zeros((nc, 15))
        self.prev_moments = np.zeros((nc, 15))
        self.has_prev = False
        self.bsums = np.zeros((nb, 20))
        self.inflow = np.zeros((nb, 6))
        self.inflow[:, 5] = 1.0
        self.F_plus = np.zeros((nb, 5))
        self.F_minus = np.zeros((nb, 5))
        self.face_state = np.zeros((nb, 5))
        self.has_face_state = False
        self.residual_cell = np.zeros(nc)
        self.mass_target = 0.0
        self.has_mass_target = False
        self.replaced = np.zeros(nc, np.int8)
        self.volume = np.asarray(setup["volume"])
        self.bpatch = np.asarray(setup["bface_patch"])
        self.pk = host.patch_int[:, 0]
        self.ptype = host.patch_int[:, 3]
        self.bkind = self.pk[self.bpatch] if nb else np.zeros(0, np.int32)
        ni = host.n_internal_faces
        self.ni = ni
        self.bf_global = np.arange(ni, ni + nb)
        L = host.length_scale
        self.barea = host.face_area[self.bf_global] / (L * L)
        self.bowner = np.asarray(setup["bface_owner"])
        self.discrete_eq = bool(setup["discrete_eq"])
        self.deq_grid = (np.asarray(setup["deq_lo"], float), np.asarray(setup["deq_hi"], float),
                         np.asarray(setup["deq_d"], float), float(setup["deq_criterion"]))
        self.wall_T = None  # per-face wall temperatures (set_wall_temperature), else the patch values
        self._build_pressure_stencils()
        self.init_static_inflow()

    # ---- numbering maps ----------------------------------------------------------------------------------------
    def _to_internal_cells(self, a):
        return np.asarray(a)[self.h.cell_new_to_old]

    # ---- inflow states -------------------------------------------------------------------------------------------
    def _deq_resolved(self, st):
        """deq_resolved (src/kinetic/discrete_equilibrium.hpp:35-48), vectorised; st (n, 5)."""
        lo, hi, d, crit = self.deq_grid
        T = st[:, 4]
        ok = T > 0
        for a in range(3):
            u = st[:, 1 + a]
            ok &= ~(2.0 * math.pi ** 2 * T / (d[a] * d[a]) < crit)
            m1, m2 = hi[a] - u, u - lo[a]
            ok &= (m1 > 0) & (m2 > 0)
            ok &= ~((m1 * m1 < 2.0 * T * crit) | (m2 * m2 < 2.0 * T * crit))
        return ok

    def correct_inflow(self, idx):
        """correct_inflow (src/kinetic/kinetic_solver.cpp:103-114) for the faces idx (discrete Maxwellian with the
        same discrete moments), batched on the backend."""
        if not self.discrete_eq or len(idx) == 0:
            return
        st = self.inflow[idx][:, 1:6]
        need = (st[:, 0] > 0) & (st[:, 4] > 0) & ~self._deq_resolved(st)
        sel = idx[need]
        if len(sel) == 0:
            return
        out, res = self.backend.discrete_maxwell(self.inflow[sel][:, 1:6], 1e-10)
        good = res > 0
        self.inflow[sel[good], 1:6] = out[good]

    def init_static_inflow(self):
        """init_static_inflow (src/kinetic/kinetic_solver.cpp:117-142)."""
        h = self.h
        self.inflow[:] = 0.0
        self.inflow[:, 5] = 1.0
        T = h.patch_dbl[self.bpatch, 0]
        p = h.patch_dbl[self.bpatch, 1]
        wall = (self.bkind == abi.BC_DIFFUSE_WALL) | (self.bkind == abi.BC_MAXWELL_WALL)
        self.inflow[wall, 0] = 1.0
        self.inflow[wall, 1] = 1.0
        self.inflow[wall, 2:5] = h.patch_dbl[self.bpatch[wall], 2:5]
        self.inflow[wall, 5] = T[wall] if self.wall_T is None else self.wall_T[wall]
        self.correct_inflow(np.flatnonzero(wall))
        pres = self.bkind == abi.BC_PRESSURE
        self.inflow[pres, 0] = 1.0
        self.inflow[pres, 1] = p[pres] / T[pres]
        self.inflow[pres, 5] = T[pres]
        mw = np.flatnonzero(self.bkind == abi.BC_MAXWELL_WALL)
        self.wall_unit = np.zeros((self.nb, 10))
        if len(mw):
            self.wall_unit[mw] = self._wall_unit_sums(mw)

    def set_wall_temperature(self, T_faces):
        """Temperature of every wall face (internal boundary-face numbering, one value per boundary face; the values of
        other faces are ignored) in place of the wall patch's temperature; None restores the patch temperatures.

        The reference sets wall temperatures per patch. A per-face field is the parameter whose derivative the adjoint
        gives (dM_dot / dT_w per face); the wall inflow state (rho = 1, patch velocity, T) is rebuilt at once, the
        wall density rho_Gamma is kept, and the field stays in force through re-initialisation."""
        if T_faces is None:
            self.wall_T = None
        else:
            T = np.asarray(T_faces, float).reshape(-1)
            if T.shape != (self.nb,):
                raise KineticSolverError(f"wall temperatures: {T.shape[0]} values for {self.nb} boundary faces")
            wall = (self.bkind == abi.BC_DIFFUSE_WALL) | (self.bkind == abi.BC_MAXWELL_WALL)
            if not np.all(T[wall] > 0):
                raise KineticSolverError("wall temperatures must be positive")
            self.wall_T = T.copy()
        wall = np.flatnonzero((self.bkind == abi.BC_DIFFUSE_WALL) | (self.bkind == abi.BC_MAXWELL_WALL))
        h = self.h
        self.inflow[wall, 1] = 1.0
        self.inflow[wall, 2:5] = h.patch_dbl[self.bpatch[wall], 2:5]
        self.inflow[wall, 5] = h.patch_dbl[self.bpatch[wall], 0] if self.wall_T is None else self.wall_T[wall]
        self.correct_inflow(wall)
        mw = np.flatnonzero(self.bkind == abi.BC_MAXWELL_WALL)
        if len(mw):
            self.wall_unit[mw] = self._wall_unit_sums(mw)
        self.version += 1

    def _wall_unit_sums(self, faces):
        """compute_wall_unit_sums (src/kinetic/kinetic_solver.cpp:263-277): discrete half-space moments of the unit
        wall Maxwellian (continuous form of the state), FP64 on the host."""
        xi = np.stack([self.s["xi_x"], self.s["xi_y"], self.s["xi_z"]], 1)
        w = self.s["weights"] if self.s.get("weights") is not None else np.full(self.nv, self.s["weight"])
        out = np.zeros((len(faces), 10))
        for i, b in enumerate(faces):
            n = self.h.face_normal[self.ni + b]
            st = self.inflow[b]
            rho, u, T = st[1], st[2:5], st[5]
            A = rho / (2 * math.pi * T) ** 1.5
            c = xi - u
            wf = w * A * np.exp(-(c * c).sum(1) / (2 * T))
            un = xi @ n
            m = un < 0
            psi = np.stack([np.ones(self.nv), xi[:, 0], xi[:, 1], xi[:, 2], 0.5 * (xi * xi).sum(1)], 1)
            out[i, :5] = (wf[m] * un[m]) @ psi[m]
            out[i, 5:] = wf[m] @ psi[m]
        return out

    def init_wall_scale_from_cells(self):
        """init_wall_scale_from_cells (src/kinetic/kinetic_solver.cpp:156-164)."""
        wall = np.flatnonzero((self.bkind == abi.BC_DIFFUSE_WALL) | (self.bkind == abi.BC_MAXWELL_WALL))
        c = self.bowner[wall]
        Tw = self.h.patch_dbl[self.bpatch[wall], 0]
        acc = self.h.patch_dbl[self.bpatch[wall], 5]
        self.inflow[wall, 0] = acc * self.moments_[c, 0] * np.sqrt(self.moments_[c, 4] / Tw)

    def _build_pressure_stencils(self):
        """Padded CSR stencils of the owner cells of pressure faces (for update_pressure_inflow)."""
        pres = np.flatnonzero(self.bkind == abi.BC_PRESSURE)
        self.pres_faces = pres
        off = np.asarray(self.s["csr_offsets"])
        other = np.asarray(self.s["csr_other"])
        bface = np.asarray(self.s["csr_bface"])
        own = self.bowner[pres]
        counts = off[own + 1] - off[own]
        E = int(counts.max()) if len(pres) else 0
        ent = off[own][:, None] + np.arange(E)[None, :]
        mask = np.arange(E)[None, :] < counts[:, None]
        ent = np.where(mask, ent, 0)
        self.ps_mask = mask
        self.ps_other = np.where(mask, other[ent], -1)
        self.ps_bface = np.where(mask, bface[ent], -1)
        self.ps_lsq = self.h.lsq[ent] if len(pres) else np.zeros((0, E, 3))
        fk = self.h.csr_faces[ent]
        self.ps_dx = self.h.face_center[fk] - self.h.cell_center[own][:, None, :]
        periodic = np.zeros_like(mask)
        bmask = mask & (self.ps_bface >= 0)
        periodic[bmask] = self.pk[self.bpatch[self.ps_bface[bmask]]] == abi.BC_PERIODIC
        self.ps_periodic = periodic
        # gathers of update_pressure_inflow, fixed for the set-up
        self.ps_owner = own
        self.ps_internal = mask & (self.ps_other >= 0)
        self.ps_int_cells = self.ps_other[self.ps_internal]
        self.ps_fs_entries = bmask & ~periodic  # entries that may carry a face state
        self.ps_fs_faces = self.ps_bface[self.ps_fs_entries]
        fb = self.bf_global[pres]
        self.ps_dxb = self.h.face_center[fb] - self.h.cell_center[own] if len(pres) else np.zeros((0, 3))
        self.ps_eps2 = self.h.limiter_k ** 3 * self.volume[own]
        self.ps_normal = self.h.face_normal[fb]
        ptype = self.ptype[self.bpatch[pres]]
        self.ps_inlet = (ptype == T_PRESSURE_INLET) | (ptype == T_MASS_FLOW_INLET)

    def update_pressure_inflow(self):
        """update_pressure_inflow (src/kinetic/kinetic_solver.cpp:172-260): W_b from the limited reconstruction of
        the owner cell's (p, u, T) and the acoustic correction of App. A.2."""
        pres = self.pres_faces
        if len(pres) == 0:
            return
        h = self.h
        limit = int(self.s["limiter_mode"]) != abi.LIMITER_NONE
        cols = [5, 1, 2, 3, 4]  # (p, u, T) of the moments
        m = self.moments_
        wi = m[self.ps_owner][:, cols]
        wk = np.repeat(wi[:, None, :], self.ps_mask.shape[1], axis=1)  # padding and other entries: the cell's value
        wk[self.ps_internal] = m[self.ps_int_cells][:, cols]
        if self.has_face_state:
            fs = self.face_state[self.ps_fs_faces]
            ok = (fs[:, 0] > 0) & (fs[:, 4] > 0)
            fs = fs[ok]
            use = self.ps_fs_entries.copy()
            use[use] = ok
            wk[use] = np.stack([fs[:, 0] * fs[:, 4], fs[:, 1], fs[:, 2], fs[:, 3], fs[:, 4]], -1)
        d = wk - wi[:, None, :]  # zero on the padding
        grad = np.matmul(d.transpose(0, 2, 1), self.ps_lsq)  # (faces, 5, 3): sum_e d_e c_e
        # the bounds start from the cell's own value (wmax = wmin = wi before the stencil loop)
        wmax = np.maximum(wi, wk.max(axis=1))
        wmin = np.minimum(wi, wk.min(axis=1))
        dxb = self.ps_dxb
        eps2 = self.ps_eps2
        phi = np.ones((len(pres), 5))
        if limit:
            proj = np.matmul(grad, self.ps_dx.transpose(0, 2, 1))  # (faces, 5, E): grad . dx_e
            dmax = (wmax - wi)[..., None]
            dmin = (wmin - wi)[..., None]
            d1 = np.where(proj > 0, dmax, np.where(proj < 0, dmin, 0.0))
            e2 = eps2[:, None, None]
            num = (d1 * d1 + e2) + 2.0 * d1 * proj
            den = d1 * d1 + 2.0 * proj * proj + d1 * proj + e2
            with np.errstate(divide="ignore", invalid="ignore"):
                v = np.clip(num / den, 0.0, 1.0)
            v = np.where(den > 0, v, 0.0)
            v = np.where(proj == 0, 1.0, v)
            active = (self.ps_mask & ~self.ps_periodic)[:, None, :]
            v = np.where(active, v, 1.0)
            phi = np.minimum(1.0, v.min(axis=2))
        wib = wi + phi * np.matmul(grad, dxb[:, :, None])[..., 0]
        bad = ~((wib[:, 0] > 0) & (wib[:, 4] > 0))
        wib[bad] = wi[bad]
        if h.pressure_boundary_reconstruction == "cell":
            wib = wi.copy()
        p_ib, u_ib, T_ib = wib[:, 0], wib[:, 1:4], wib[:, 4]
        rho_ib = p_ib / T_ib
        cs = np.sqrt(h.gamma * T_ib)
        n = self.ps_normal
        inlet = self.ps_inlet
        p_b = h.patch_dbl[self.bpatch[pres], 1]
        T_b = np.where(inlet, h.patch_dbl[self.bpatch[pres], 0], T_ib)
        du = (p_ib - p_b) / (rho_ib * cs)
        zt = h.patch_dbl[self.bpatch[pres], 6] > 0.5
        un = np.sum(u_ib * n, axis=1)
        u = np.where(zt[:, None], (un + du)[:, None] * n, u_ib + du[:, None] * n)
        self.inflow[pres, 0] = 1.0
        self.inflow[pres, 1] = p_b / T_b
        self.inflow[pres, 2:5] = u
        self.inflow[pres, 5] = T_b
        self.correct_inflow(pres)

    # ---- boundary sums ---------------------------------------------------------------------------------------------
    def process_boundary_sums(self):
        """process_boundary_sums (src/kinetic/kinetic_solver.cpp:280-335)."""
        sm = self.bsums
        kind = self.bkind
        in_scale = np.ones(self.nb)
        wall = kind == abi.BC_DIFFUSE_WALL
        jp, jm = sm[:, 0], sm[:, 5]
        with np.errstate(divide="ignore", invalid="ignore"):
            rho_g = np.where(jm < 0, np.maximum(0.0, -jp / np.where(jm < 0, jm, -1.0)), 0.0)
        w = self.h.wall_relaxation
        self.inflow[wall, 0] = rho_g[wall] if w == 1.0 else w * rho_g[wall] + (1 - w) * self.inflow[wall, 0]
        in_scale[wall] = rho_g[wall]
        in_scale[kind == abi.BC_VACUUM] = 0.0
        mw = kind == abi.BC_MAXWELL_WALL
        delta = np.zeros(self.nb)
        if np.any(mw):
            unit = self.wall_unit
            if np.any(unit[mw, 0] >= 0.0):
                raise KineticSolverError("Maxwell wall without inflowing velocities")
            delta[mw] = -(sm[mw, 0] + sm[mw, 5]) / unit[mw, 0]
            nxt = self.inflow[mw, 0] + delta[mw]
            if np.any(nxt < -1e-8):
                raise KineticSolverError("negative diffuse density on a Maxwell wall; refine the velocity grid")
            self.inflow[mw, 0] = np.maximum(0.0, nxt)
        area = self.barea[:, None]
        self.F_plus = area * sm[:, 0:5]
        Fm = area * in_scale[:, None] * sm[:, 5:10]
        mom = sm[:, 10:15] + in_scale[:, None] * sm[:, 15:20]
        if np.any(mw):
            Fm[mw] = area[mw] * (sm[mw, 5:10] + delta[mw, None] * self.wall_unit[mw, 0:5])
            mom[mw] = sm[mw, 10:15] + sm[mw, 15:20] + delta[mw, None] * self.wall_unit[mw, 5:10]
        self.F_minus = Fm
        fs = np.zeros((self.nb, 5))
        pos = mom[:, 0] > 0
        u = mom[pos, 1:4] / mom[pos, 0:1]
        fs[pos, 0] = mom[pos, 0]
        fs[pos, 1:4] = u
        fs[pos, 4] = (2.0 * mom[pos, 4] / mom[pos, 0] - np.sum(u * u, 1)) / 3.0
        self.face_state = fs
        n_patches = len(self.h.patch_int)
        self.info.patch_mass_flow = np.bincount(self.bpatch, weights=self.F_plus[:, 0] + self.F_minus[:, 0],
                                                minlength=n_patches) if self.nb else np.zeros(n_patches)
        self.has_face_state = True

    def compute_epsilon(self):
        """eq. (59) with the u floor (compute_epsilon, src/kinetic/kinetic_solver.cpp:338-363)."""
        V = self.volume
        a, b = self.moments_[:, :5], self.prev_moments[:, :5]
        d = a - b
        n5 = (d * d).T @ V  # per moment: sum_c (a - b)^2 V
        d5 = (b * b).T @ V
        num = [n5[0], n5[1] + n5[2] + n5[3], n5[4]]
        den = [d5[0], d5[1] + d5[2] + d5[3], d5[4]]
        fl = self.h.convergence_u_floor
        den[1] = max(den[1], fl * fl * np.sum(V))
        ratio = lambda n, d: math.sqrt(n / d) if d > 0 else (1.0 if n > 0 else 0.0)  # noqa: E731
        i = self.info
        i.eps_rho, i.eps_u, i.eps_T = ratio(num[0], den[0]), ratio(num[1], den[1]), ratio(num[2], den[2])
        i.epsilon = max(i.eps_rho, i.eps_u, i.eps_T)
        i.has_epsilon = True

    # ---- iteration ----------------------------------------------------------------------------------------------
    def prepare(self) -> IterationInfo:
        """KineticSolver::prepare (src/kinetic/kinetic_solver.cpp:365-452)."""
        if self.prepared_version == self.version:
            return self.info
        t0 = time.perf_counter()
        self.info = IterationInfo(iteration=self.iteration)
        self.moments_ = self.backend.compute_moments().copy()
        m = self.moments_
        bad = ~((m[:, 0] > 0) & (m[:, 4] > 0) & np.isfinite(m[:, 0]) & np.isfinite(m[:, 4]))
        if np.any(bad):
            c = int(np.flatnonzero(bad)[0])
            raise KineticSolverError(f"iteration {self.iteration}: {int(bad.sum())} cells with non-positive density or "
                                     f"temperature (e.g. original cell {int(self.h.cell_new_to_old[c])})")
        mass = float(np.sum(m[:, 0] * self.volume))
        self.info.total_mass = mass
        if self.h.closed_domain:
            if not self.has_mass_target:
                self.mass_target = mass
                self.has_mass_target = True
            scale = self.mass_target / mass
            if scale != 1.0:
                self.backend.scale_distribution(scale)
                m[:, 0] *= scale
                m[:, 5:] *= scale
            self.info.mass_scale = scale
        if self.has_prev:
            self.compute_epsilon()
        self.backend.update_cell_params()
        if self.discrete_eq:
            corrected, failed, _ = self.backend.deq_counts()
            self.info.deq_corrected, self.info.deq_failed = corrected, failed
        if not self.has_face_state:
            self.init_wall_scale_from_cells()
        self.update_pressure_inflow()
        self.backend.set_inflow(self.inflow)
        self.bsums = self.backend.boundary_sums().copy()
        self.process_boundary_sums()
        self.backend.set_inflow(self.inflow)
        for _ in range(1, self.h.boundary_iterations):
            self.update_pressure_inflow()
            self.backend.set_inflow(self.inflow)
            self.bsums = self.backend.boundary_sums().copy()
            self.process_boundary_sums()
            self.backend.set_inflow(self.inflow)
        self.prepared_version = self.version
        self.info.seconds = time.perf_counter() - t0
        return self.info

    def refresh_wall_inflow(self):
        """refresh_wall_inflow (src/kinetic/kinetic_solver.cpp:456-480)."""
        self.bsums = self.backend.boundary_sums().copy()
        sm = self.bsums
        kind = self.bkind
        any_ = False
        mw = kind == abi.BC_MAXWELL_WALL
        if np.any(mw):
            nxt = self.inflow[mw, 0] - (sm[mw, 0] + sm[mw, 5]) / self.wall_unit[mw, 0]
            if np.any(nxt < -1e-8):
                raise KineticSolverError("negative diffuse density on a Maxwell wall; refine the velocity grid")
            self.inflow[mw, 0] = np.maximum(0.0, nxt)
            any_ = True
        wall = kind == abi.BC_DIFFUSE_WALL
        if np.any(wall):
            jp, jm = sm[wall, 0], sm[wall, 5]
            with np.errstate(divide="ignore", invalid="ignore"):
                rho_g = np.where(jm < 0, np.maximum(0.0, -jp / np.where(jm < 0, jm, -1.0)), 0.0)
            w = self.h.wall_relaxation
            self.inflow[wall, 0] = rho_g if w == 1.0 else w * rho_g + (1 - w) * self.inflow[wall, 0]
            any_ = True
        if any_:
            self.backend.set_inflow(self.inflow)

    def update_mass_flow_pressure(self):
        """update_mass_flow_pressure (src/kinetic/kinetic_solver.cpp:482-501)."""
        self.prepare()
        changed = False
        h = self.h
        for pi in range(len(h.patch_int)):
            if h.patch_int[pi, 3] != T_MASS_FLOW_INLET:
                continue
            fb, nf = h.patch_int[pi, 1], h.patch_int[pi, 2]
            faces = np.arange(fb, fb + nf)
            T = self.moments_[self.bowner[faces], 4]
            D = float(np.sum(self.barea[faces] * (1.0 / math.sqrt(2 * math.pi * h.patch_dbl[pi, 0]) +
                                                  0.5 / np.sqrt(h.gamma * T))))
            if not D > 0:
                raise KineticSolverError("mass-flow inlet with zero area")
            p = h.patch_dbl[pi, 1]
            dp = 0.2 * (h.patch_target[pi] + self.info.patch_mass_flow[pi]) / D
            h.patch_dbl[pi, 1] = max(1e-12, p + min(max(dp, -0.1 * p), 0.1 * p))
            changed = True
        if changed:
            self.version += 1
            self.prepare()

    def sweep(self, update_pressure: bool = True) -> IterationInfo:
        """KineticSolver::sweep (src/kinetic/kinetic_solver.cpp:503-531)."""
        self.prepare()
        if update_pressure:
            self.update_mass_flow_pressure()
        t0 = time.perf_counter()
        self.residual_cell = self.backend.sweep().copy()
        for _ in range(1, self.h.inner_sweeps):
            if self.h.inner_wall_update:
                self.refresh_wall_inflow()
            self.backend.sweep()
        V = self.volume
        self.info.residual = math.sqrt(float(np.sum(self.residual_cell / V)) * self._weight_scale() / float(np.sum(V)))
        self.info.has_residual = True
        # prepare() replaces moments_ by a new array (and scales only that one), so the reference is enough
        self.prev_moments = self.moments_
        self.has_prev = True
        self.version += 1
        self.iteration += 1
        self.info.seconds += time.perf_counter() - t0
        return self.info

    def _weight_scale(self) -> float:
        return float(self.s["weight"])

    # ---- initialisation and results (original numbering) ---------------------------------------------------------
    def _reset_after_initialization(self):
        self.version += 1
        self.iteration = 0
        self.has_prev = False
        self.has_face_state = False
        self.has_mass_target = False
        self.init_static_inflow()

    def initialize_uniform(self, rho, u, T):
        if not (rho > 0 and T > 0):
            raise KineticSolverError("initial density and temperature must be positive")
        self.backend.set_equilibrium(np.tile([rho, u[0], u[1], u[2], T], self.nc))
        self._reset_after_initialization()

    def initialize_equilibrium(self, states_orig):
        st = np.asarray(states_orig, float).reshape(self.nc, 5)[self.h.cell_new_to_old]
        if not np.all((st[:, 0] > 0) & (st[:, 4] > 0)):
            raise KineticSolverError("initial density and temperature must be positive")
        self.backend.set_equilibrium(st)
        self._reset_after_initialization()

    def moments(self) -> np.ndarray:
        """15 moments per cell in the original numbering (KineticSolver::moments)."""
        self.prepare()
        out = np.empty_like(self.moments_)
        out[self.h.cell_new_to_old] = self.moments_
        return out

    def boundary_fluxes(self):
        """(F_plus, F_minus, face_state) per boundary face in the original numbering."""
        self.prepare()
        o = self.h.bface_new_to_old
        fp, fm, fs = (np.empty_like(a) for a in (self.F_plus, self.F_minus, self.face_state))
        fp[o], fm[o], fs[o] = self.F_plus, self.F_minus, self.face_state
        return fp, fm, fs

    def distribution(self) -> np.ndarray:
        """f in the original cell numbering x velocity-grid order."""
        internal = self.backend.get_distribution()
        out = np.empty_like(internal)
        out[np.ix_(self.h.cell_new_to_old, self.h.storage_to_grid)] = internal
        return out

    def set_distribution(self, f_orig):
        f = np.asarray(f_orig, float).reshape(self.nc, self.nv)
        self.backend.set_distribution(f[np.ix_(self.h.cell_new_to_old, self.h.storage_to_grid)])
        self._reset_after_initialization()

    def apply_gsis_correction(self, w_half_orig, w_new_orig) -> int:
        """apply_gsis_correction (src/kinetic/kinetic_solver.cpp:624-654); W: (n_cells, 5) original numbering."""
        wh = np.asarray(w_half_orig, float).reshape(self.nc, 5)[self.h.cell_new_to_old]
        wn = np.asarray(w_new_orig, float).reshape(self.nc, 5)[self.h.cell_new_to_old]
        if not np.all((wn[:, 0] > 0) & (wn[:, 4] > 0) & (wh[:, 0] > 0) & (wh[:, 4] > 0)):
            raise KineticSolverError("non-positive density or temperature in the GSIS correction")
        replaced, flags = self.backend.gsis_correction(wh, wn)
        self.replaced = np.zeros(self.nc, np.int8)
        self.replaced[self.h.cell_new_to_old] = flags != 0
        self.version += 1
        return replaced

    def residual_per_cell(self) -> np.ndarray:
        out = np.empty(self.nc)
        out[self.h.cell_new_to_old] = np.sqrt(self._weight_scale() * self.residual_cell) / self.volume
        return out

    def mass_flow(self):
        """Nondimensional tube mass flow M_dot = 1/2 (mdot_in + mdot_out) sqrt(2/pi) of the last prepare
        (tube_mass_flow_json, src/kinetic/kinetic_output.cpp:273-284; mass_flow_scale, case_config.cpp:663).
        Returns (M_dot_in, M_dot_out, M_dot)."""
        pm = self.prepare().patch_mass_flow
        f = math.sqrt(2.0 / math.pi)
        mdot_in = -sum(pm[p] for p in range(len(pm)) if self.ptype[p] in (T_PRESSURE_INLET, T_MASS_FLOW_INLET))
        mdot_out = sum(pm[p] for p in range(len(pm)) if self.ptype[p] in (T_PRESSURE_OUTLET, T_VACUUM))
        return mdot_in * f, mdot_out * f, 0.5 * (mdot_in + mdot_out) * f

    def patch_summary(self) -> list:
        """Per-patch flows of the last prepare (summarize_patches; SI values when the set-up carries its reference
        scales, as the builder's do)."""
        self.prepare()
        h = self.h
        names = h.patch_names or [f"patch{i}" for i in range(len(h.patch_int))]
        types = [BOUNDARY_TYPES[t] for t in h.patch_int[:, 3]]
        faces = [np.flatnonzero(self.bpatch == pi) for pi in range(len(h.patch_int))]
        return summarize_patches(names, types, faces, self.barea, h.face_normal[self.bf_global], self.F_plus,
                                 self.F_minus, self.face_state, h.patch_dbl, h.patch_target, h.length_scale,
                                 h.ref_pressure, h.ref_velocity)

    # ---- section cuts ------------------------------------------------------------------------------------------
    def section_cuts(self, spec):
        """section_cuts (src/kinetic/kinetic_solver.cpp:687-690): the cuts of `spec` on the internal (renumbered)
        mesh, with the (cell, CSR entry) pairs the backend reads (build_sections, kinetic_solver.cpp:56-79).
        Cached until the spec changes."""
        from . import section as sec

        if getattr(self, "_section_spec", None) == spec:
            return self._section_cuts
        h = self.h
        if getattr(self, "_face_entry", None) is None:
            self._face_neighbour, self._face_entry = sec.owner_entries(
                self.s["csr_offsets"], self.s["csr_other"], h.csr_faces, h.owner, self.ni)
        cuts = sec.build_section_cuts(h.owner, self._face_neighbour, h.cell_center, h.face_center, h.face_normal,
                                      h.face_area, h.length_scale, spec)
        faces = np.concatenate([c.faces for c in cuts]) if cuts else np.zeros(0, np.int64)
        self._section_cells = np.asarray(h.owner)[faces].astype(np.int32)
        self._section_entries = self._face_entry[faces].astype(np.int32)
        self._section_spec = sec.SectionSpec(spec.axis, list(spec.positions))
        self._section_cuts = cuts
        return cuts

    def section_mass_flow(self, spec) -> np.ndarray:
        """section_mass_flow (src/kinetic/kinetic_solver.cpp:669-685): nondimensional mass flow through each cut of
        `spec` (+axis direction) from the current f: prepare, the backend's discrete internal-face flux on the cut
        faces, summed with the cut signs."""
        if spec.empty():
            return np.zeros(0)
        self.prepare()
        cuts = self.section_cuts(spec)
        flux = self.backend.internal_face_mass_flux(self._section_cells, self._section_entries)
        out = np.zeros(len(cuts))
        k = 0
        for i, c in enumerate(cuts):
            s = 0.0
            for j in range(len(c.faces)):
                s += float(c.sign[j]) * flux[k]
                k += 1
            out[i] = s
        return out

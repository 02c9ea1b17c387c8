"""Discrete adjoint of the converged CIS fixed point: dM_dot / d(mu_hat0, delta, T_w per wall face, accommodation per
wall face at alpha = 1) on the B200 backend.

There is no reference counterpart; the steady problem differentiated is the one the reference's CIS iteration
converges to (src/kinetic/kinetic_solver.cpp prepare + sweep, src/kinetic/kinetic_kernels.hpp):

  F(x; p) = ( R(f, rho_Gamma, fs)             residual_value with the limited LSQ gradient, Shakhov target of the
                                              cell moments, inflow of walls / pressure faces
              rho_Gamma - Phi(f, rho_Gamma)   zero net mass flux of every diffuse wall face
              fs - FS(f, fs) )                the face states of the boundary sums (process_boundary_sums,
                                              src/kinetic/kinetic_solver.cpp:280-335), which the "limited" pressure-
                                              boundary reconstruction (the reference default) reads: W_b is the owner's
                                              (p, u, T) reconstructed at the face from its stencil, whose boundary
                                              entries carry those face states (:172-260); absent with the "cell"
                                              reconstruction (W_b = the owner's state)
  J = M_dot = 1/2 (mdot_in + mdot_out) sqrt(2/pi)   (tube_mass_flow_json, src/kinetic/kinetic_output.cpp:273-284)

The adjoint y = (lambda, nu, kappa) solves O(y) = y^T dF/dx - dJ/dx = 0 by the preconditioned fixed-point iteration
  lambda <- lambda - P^-T O_f(y),   nu <- nu - O_nu(y),   kappa <- kappa - O_kappa(y)
where P^-T is the forward LU-SGS block passes run on velocity-reversed storage (the transposed sweep; the device does
it, kin_adjoint_update). Then dJ/dp = dJ/dp|_x - y^T dF/dp. The transposed transport, the per-cell sums against the
Shakhov target and the per-face sums against the inflow Maxwellians run on the device (csrc/kin_adjoint.cu); this
module finishes the per-cell / per-face algebra: the moments -> cell parameter chain, the pressure-face chain
(App. A.2 acoustic correction), the wall-density equations and the parameter gradients.

Equilibrium: continuous, or discrete (the reference default). Where the grid does not resolve a cell's state the
Shakhov target is built on the discrete Maxwellian of a Newton solve with the conservative correction gamma; the
derivative goes through both solves by the implicit function theorem (gsis_sim_b200.deq_adjoint: the device gives
the lambda sums at fixed (beta, gamma), the host the 5 x 5 chain). Inflow states of walls and pressure faces that
the reference corrects to their discrete Maxwellian are differentiated through that correction the same way.

Precision: FP64, or mixed (f of the converged mixed-precision solve stored in FP32). In mixed precision lambda and
the transport seeds are stored in FP32 and the transposed block passes run in FP32, while O(y) is evaluated in FP64
arithmetic from the stored values and every sum the host reads is FP64: the adjoint counterpart of the forward's
FP64 residual with FP32 sweeps. Its fixed point holds to the FP32 storage of lambda (relative residual floor about
1e-6 instead of 1e-12).

Scope (`check_scope`): FP64 or mixed-precision backend with one velocity chunk; a tensor velocity grid when the equilibrium is discrete
(every grid of the reference is one) and no failed Newton solve; diffuse walls, pressure inlets / outlets with
the "limited" (default) or "cell" pressure-boundary reconstruction, vacuum, symmetry, periodic faces; no Maxwell
walls, mass-flow inlets, positivity limiter or closed-domain scaling.

Face states (limited reconstruction): the device adds the seeds -kappa^T dFS/df on the outgoing reconstructed face
values (kin_adjoint_face_moment_seeds: weights of w psi, psi = (1, xi, |xi|^2 / 2); at symmetry faces also the
mirrored incoming half); the host carries the rest: the wall density rho_Gamma = -sm0 / sm5 in the walls' face
moments (an extra weight in mu), the pressure faces' own incoming halves (a loop back through W_b), the vector-
Jacobian product of the reconstruction (PressureReconstruction) and the wall-temperature and accommodation terms of
the gradients.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import abi
from .deq_adjoint import CellDerivatives, InflowDerivatives, TensorGrid
from .kinetic_setup import BOUNDARY_TYPES

C_J = 0.5 * math.sqrt(2.0 / math.pi)
_INLETS = (BOUNDARY_TYPES.index("pressure_inlet"), BOUNDARY_TYPES.index("mass_flow_inlet"))
_OUTLETS = (BOUNDARY_TYPES.index("pressure_outlet"), BOUNDARY_TYPES.index("vacuum"))


class AdjointScopeError(ValueError):
    pass


def reversed_velocities(xi: np.ndarray) -> np.ndarray:
    """rev[p] = index of -xi_p in the same list (a velocity grid symmetric about 0). Raises AdjointScopeError."""
    xi = np.asarray(xi, float)
    scale = max(float(np.abs(xi).max()), 1e-300)
    key = np.round(xi / scale * 2.0 ** 40).astype(np.int64)
    index = {tuple(k): i for i, k in enumerate(key.tolist())}
    rev = np.array([index.get(tuple((-k).tolist()), -1) for k in key], np.int32)
    if np.any(rev < 0):
        raise AdjointScopeError("the velocity grid is not symmetric about 0 (no reversed velocity)")
    return rev


def flipped_velocities(xi: np.ndarray) -> np.ndarray:
    """(3, nv): for each axis a, the index of xi with component a negated. Raises AdjointScopeError."""
    xi = np.asarray(xi, float)
    scale = max(float(np.abs(xi).max()), 1e-300)
    key = np.round(xi / scale * 2.0 ** 40).astype(np.int64)
    index = {tuple(k): i for i, k in enumerate(key.tolist())}
    out = np.empty((3, len(xi)), np.int32)
    for a in range(3):
        sgn = np.ones(3, np.int64)
        sgn[a] = -1
        out[a] = [index.get(tuple((k * sgn).tolist()), -1) for k in key]
    if np.any(out < 0):
        raise AdjointScopeError("the velocity grid is not symmetric in every axis")
    return out


def face_axes(normals: np.ndarray, tol: float = 1e-10) -> np.ndarray:
    """The axis each unit normal is aligned with, -1 if none."""
    n = np.abs(np.asarray(normals, float))
    ax = np.argmax(n, axis=1).astype(np.int32)
    return np.where(np.abs(n[np.arange(len(n)), ax] - 1.0) < tol, ax, -1).astype(np.int32)


def reverse_entries(csr_offsets, csr_other, csr_faces) -> np.ndarray:
    """For every internal CSR entry (cell j -> i through face f) the entry of cell i that points back to j through f;
    -1 for boundary entries."""
    offs = np.asarray(csr_offsets, np.int64)
    other = np.asarray(csr_other, np.int64)
    faces = np.asarray(csr_faces, np.int64)
    row = np.repeat(np.arange(len(offs) - 1), np.diff(offs))
    out = np.full(len(other), -1, np.int32)
    internal = np.flatnonzero(other >= 0)
    # key (face, cell of the row) -> entry
    key = {(int(faces[e]), int(row[e])): int(e) for e in internal}
    for e in internal.tolist():
        back = key.get((int(faces[e]), int(other[e])))
        if back is None:
            raise AdjointScopeError(f"CSR entry {e} has no reverse entry")
        out[e] = back
    return out


def moment_expansion_coefficients(m: np.ndarray, rho_b, u_b, T_b, q_b) -> np.ndarray:
    """Per cell the coefficients (a0, a (3), a2, b (3)) of d(rho_b rho + u_b.u + T_b T + q_b.q)/d f_q
    = w_q (a0 + a.c + a2 c^2 + b.c c^2), c = xi_q - u, for the moments of finalize_moments
    (rho = sum w f, u = sum w xi f / rho, T = sum w c^2 f / (3 rho), q = 1/2 sum w c c^2 f); m: (n, 15) moments."""
    rho, T, p = m[:, 0], m[:, 4], m[:, 5]
    s = m[:, 6:12]
    P = np.empty((len(m), 3, 3))
    P[:, 0, 0], P[:, 1, 1], P[:, 2, 2] = s[:, 0] + p, s[:, 1] + p, s[:, 2] + p
    P[:, 0, 1] = P[:, 1, 0] = s[:, 3]
    P[:, 1, 2] = P[:, 2, 1] = s[:, 4]
    P[:, 0, 2] = P[:, 2, 0] = s[:, 5]
    Pq = np.einsum("nab,na->nb", P, q_b)
    out = np.empty((len(m), 8))
    out[:, 0] = rho_b - T_b * T / rho
    out[:, 1:4] = (u_b - 1.5 * p[:, None] * q_b - Pq) / rho[:, None]
    out[:, 4] = T_b / (3.0 * rho)
    out[:, 5:8] = 0.5 * q_b
    return out


def pressure_face_adjoint(p_o, u_o, T_o, n, p_patch, inlet, zero_tan, gamma, rho_bar, u_bar, T_bar):
    """Adjoint of the pressure-face state W_b = (rho_b, u_b, T_b) of the "cell" reconstruction (update_pressure_inflow,
    src/kinetic/kinetic_solver.cpp:172-260) with respect to the owner cell's (p, u, T): returns (p_bar, u_bar, T_bar)
    of the owners. u_b = u_o + du n (or (u_o.n + du) n with zero tangential velocity), du = (p_o - p_b) / (rho_o c_s),
    rho_o = p_o / T_o, c_s = sqrt(gamma T_o); T_b = T_patch at inlets, T_o at outlets; rho_b = p_b / T_b."""
    sg = math.sqrt(gamma)
    sT = np.sqrt(T_o)
    dbar = np.einsum("na,na->n", u_bar, n)
    uo_bar = np.where(zero_tan[:, None], dbar[:, None] * n, u_bar)
    p_bar = dbar * sT / sg * p_patch / (p_o * p_o)
    T_out = dbar * (p_o - p_patch) / (p_o * sg) * 0.5 / sT
    T_b = np.where(inlet, 0.0, 1.0)  # outlet: T_b = T_o
    T_out = T_out + T_b * (T_bar - rho_bar * p_patch / (T_o * T_o))
    return p_bar, uo_bar, T_out


def collision_moment_adjoint(m, volume, mu0, omega, cell_sums):
    """Adjoints of the cell moments (rho, u, T, q) from the collision term -coll (f^S - f) of the residual
    (make_cell_params, src/kinetic/kinetic_kernels.hpp:451-471: coll = V p / (mu0 T^omega), p = rho T), given the
    per-cell sums of k_adj_cell: Lambda0 = sum lambda (f^S - f), Lambda_theta = sum lambda d f^S / d theta.
    Returns (rho_bar, u_bar, T_bar, q_bar, coll)."""
    rho, T, p = m[:, 0], m[:, 4], m[:, 5]
    coll = volume * p / (mu0 * T ** omega)
    L0, Lr, Lu, LT, Lq = cell_sums[:, 0], cell_sums[:, 1], cell_sums[:, 2:5], cell_sums[:, 5], cell_sums[:, 6:9]
    rho_b = -(coll / rho) * L0 - coll * Lr
    T_b = -((1.0 - omega) * coll / T) * L0 - coll * LT
    u_b = -coll[:, None] * Lu
    q_b = -coll[:, None] * Lq
    return rho_b, u_b, T_b, q_b, coll


class PressureReconstruction:
    """W_ib = (p, u, T) of every pressure face by the "limited" reconstruction of update_pressure_inflow
    (src/kinetic/kinetic_solver.cpp:172-260) as a function of the cell states and the face states of the boundary
    sums, with its vector-Jacobian product. The owner's (p, u, T) plus phi * (grad . dx_b): grad the LSQ gradient over
    the owner's stencil, whose internal entries carry the neighbour's state, whose boundary entries carry the face
    state (rho T, u, T) where it is positive (periodic entries and the others the owner's own value); phi the
    Venkatakrishnan limiter with epsilon^2 = K^3 V over the non-periodic entries; the owner's own state where the
    result is not positive. The stencil arrays are the solver's (KineticSolver._build_pressure_stencils)."""

    def __init__(self, sol):
        h = sol.h
        self.nc, self.nb = sol.nc, sol.nb
        self.faces = sol.pres_faces
        self.own = sol.bowner[self.faces]
        self.mask, self.other, self.bface = sol.ps_mask, sol.ps_other, sol.ps_bface
        self.lsq, self.dx, self.periodic = sol.ps_lsq, sol.ps_dx, sol.ps_periodic
        fb = sol.bf_global[self.faces]
        self.dxb = h.face_center[fb] - h.cell_center[self.own]
        self.eps2 = h.limiter_k ** 3 * sol.volume[self.own]
        self.limit = int(sol.s["limiter_mode"]) != abi.LIMITER_NONE

    def forward(self, m, fs):
        """W_ib (n_pressure, 5) from the cell moments m (nc, 15) and the face states fs (nb, 5: rho, u, T)."""
        state = np.stack([m[:, 5], m[:, 1], m[:, 2], m[:, 3], m[:, 4]], -1)
        self.state, self.fs = state, fs
        wi = state[self.own]
        internal = self.mask & (self.other >= 0)
        bmask = self.mask & (self.bface >= 0)
        f = fs[np.where(bmask, self.bface, 0)]
        use = bmask & ~self.periodic & (f[..., 0] > 0) & (f[..., 4] > 0)
        wk = np.broadcast_to(wi[:, None, :], self.mask.shape + (5,)).copy()
        wk[internal] = state[self.other[internal]]
        wk[use] = np.stack([f[use][:, 0] * f[use][:, 4], f[use][:, 1], f[use][:, 2], f[use][:, 3], f[use][:, 4]], -1)
        grad = np.einsum("fek,fea->fka", np.where(self.mask[..., None], wk - wi[:, None, :], 0.0), self.lsq)
        wm = np.where(self.mask[..., None], wk, np.nan)
        # the bounds start from the owner's value; a stencil entry takes over only when strictly beyond it (the
        # reference's std::max / std::min keep the earlier value on a tie)
        xmax, xmin = np.nanmax(wm, axis=1), np.nanmin(wm, axis=1)
        self.amax = np.where(xmax > wi, np.nanargmax(np.where(np.isnan(wm), -np.inf, wm), axis=1), -1)
        self.amin = np.where(xmin < wi, np.nanargmin(np.where(np.isnan(wm), np.inf, wm), axis=1), -1)
        wmax, wmin = np.maximum(wi, xmax), np.minimum(wi, xmin)
        phi = np.ones_like(wi)
        self.estar = np.full(wi.shape, -1)
        if self.limit:
            proj = np.einsum("fka,fea->fke", grad, self.dx)
            dmax, dmin = (wmax - wi)[..., None], (wmin - wi)[..., None]
            d1 = np.where(proj > 0, dmax, np.where(proj < 0, dmin, 0.0))
            e2 = self.eps2[:, None, None]
            num = (d1 * d1 + e2) + 2.0 * d1 * proj
            den = d1 * d1 + 2.0 * proj * proj + d1 * proj + e2
            with np.errstate(divide="ignore", invalid="ignore"):
                v = np.clip(num / den, 0.0, 1.0)
            v = np.where(den > 0, v, 0.0)
            v = np.where(proj == 0, 1.0, v)
            v = np.where((self.mask & ~self.periodic)[:, None, :], v, 1.0)
            vmin = v.min(axis=2)
            phi = np.minimum(1.0, vmin)
            e = np.argmin(v, axis=2)
            self.estar = np.where(vmin < 1.0, e, -1)
            self.proj, self.d1, self.num, self.den = proj, d1, num, den
        wib = wi + phi * np.einsum("fka,fa->fk", grad, self.dxb)
        self.good = (wib[:, 0] > 0) & (wib[:, 4] > 0)
        self.wi, self.wk, self.use, self.internal, self.grad, self.phi = wi, wk, use, internal, grad, phi
        return np.where(self.good[:, None], wib, wi)

    def vjp(self, wb):
        """Seeds wb (n_pressure, 5) on W_ib -> (seeds (nc, 5) on the cells' (p, u, T), seeds (nb, 5) on the face
        states (rho, u, T)) at the point of the last forward."""
        npf, E = self.mask.shape
        wi_bar = np.where(self.good[:, None], 0.0, wb)
        wg = np.where(self.good[:, None], wb, 0.0)
        wi_bar = wi_bar + wg
        wk_bar = np.zeros((npf, E, 5))
        grad_bar = (wg * self.phi)[:, :, None] * self.dxb[:, None, :]
        if self.limit:
            phi_bar = wg * np.einsum("fka,fa->fk", self.grad, self.dxb)
            f_i, k_i = np.nonzero(self.estar >= 0)
            e = self.estar[f_i, k_i]
            p = self.proj[f_i, k_i, e]
            d1 = self.d1[f_i, k_i, e]
            num, den = self.num[f_i, k_i, e], self.den[f_i, k_i, e]
            with np.errstate(divide="ignore", invalid="ignore"):
                ok = (p != 0) & (den > 0) & (num < den) & (num / den > 0)
            den2 = np.where(ok, den * den, 1.0)
            dv_dp = np.where(ok, (2.0 * d1 * den - num * (4.0 * p + d1)) / den2, 0.0)
            dv_dd1 = np.where(ok, ((2.0 * d1 + 2.0 * p) * den - num * (2.0 * d1 + p)) / den2, 0.0)
            pb = phi_bar[f_i, k_i] * dv_dp
            np.add.at(grad_bar, (f_i, k_i), pb[:, None] * self.dx[f_i, e])
            d1b = phi_bar[f_i, k_i] * dv_dd1
            # d1 = wmax - wi (proj > 0) or wmin - wi (proj < 0); wmax / wmin is the owner's value or one entry
            for sel, arg in ((p > 0, self.amax), (p < 0, self.amin)):
                fi_, ki_, db = f_i[sel], k_i[sel], d1b[sel]
                a = arg[fi_, ki_]
                np.add.at(wi_bar, (fi_, ki_), -db)
                on = a >= 0
                np.add.at(wi_bar, (fi_[~on], ki_[~on]), db[~on])
                np.add.at(wk_bar, (fi_[on], a[on], ki_[on]), db[on])
        # grad = sum_e lsq_e (wk_e - wi) over the stencil
        g_e = np.einsum("fka,fea->fek", grad_bar, self.lsq) * self.mask[..., None]
        wk_bar += g_e
        wi_bar -= g_e.sum(axis=1)
        cell_bar = np.zeros((self.nc, 5))
        fs_bar = np.zeros((self.nb, 5))
        np.add.at(cell_bar, self.own, wi_bar)
        np.add.at(cell_bar, self.other[self.internal], wk_bar[self.internal])
        # entries that carry the owner's own value (periodic, no face state, padding)
        own_val = ~self.internal & ~self.use
        np.add.at(cell_bar, np.broadcast_to(self.own[:, None], self.mask.shape)[own_val], wk_bar[own_val])
        # face states: wk = (rho T, u, T)
        b = self.bface[self.use]
        fsv = self.fs[b]
        wu = wk_bar[self.use]
        fsb = np.column_stack([wu[:, 0] * fsv[:, 4], wu[:, 1:4], wu[:, 4] + wu[:, 0] * fsv[:, 0]])
        np.add.at(fs_bar, b, fsb)
        return cell_bar, fs_bar


def face_moment_state_adjoint(mom, fs_bar):
    """Seeds on the face moments mom = (m0, m1, m2, m3, m4) (sums of w psi f, psi = (1, xi, |xi|^2 / 2)) of the seeds
    fs_bar on the face state (rho, u, T) = (m0, m_a / m0, (2 m4 / m0 - |u|^2) / 3) of process_boundary_sums
    (src/kinetic/kinetic_solver.cpp:280-335); zero where m0 <= 0 (face state 0)."""
    pos = mom[:, 0] > 0
    m0 = np.where(pos, mom[:, 0], 1.0)
    u = mom[:, 1:4] / m0[:, None]
    kr, ku, kT = fs_bar[:, 0], fs_bar[:, 1:4], fs_bar[:, 4]
    out = np.empty_like(mom)
    out[:, 0] = kr - np.sum(ku * u, 1) / m0 + kT * (-2.0 * mom[:, 4] / (3.0 * m0 * m0) + (2.0 / 3.0) * np.sum(u * u, 1) / m0)
    out[:, 1:4] = ku / m0[:, None] - (2.0 / 3.0) * kT[:, None] * u / m0[:, None]
    out[:, 4] = 2.0 * kT / (3.0 * m0)
    return np.where(pos[:, None], out, 0.0)


def inflow_moment_derivatives(xi, w, normals, states):
    """Per face: D[k, j] = sum_{xi.n < 0} w psi_k(xi) dM/dtheta_j and d5[j] = sum_{xi.n < 0} w (xi.n) dM/dtheta_j for
    the Maxwellian M of theta = (rho, u (3), T), psi = (1, xi, |xi|^2 / 2): the derivatives of the incoming halves of
    a face's moment and flux sums (k_boundary_sums) with respect to its inflow state."""
    n = len(states)
    D = np.zeros((n, 5, 5))
    d5 = np.zeros((n, 5))
    psi = np.column_stack([np.ones(len(xi)), xi, 0.5 * np.sum(xi * xi, 1)])
    for i in range(n):
        rho, u, T = states[i, 0], states[i, 1:4], states[i, 4]
        an = xi @ normals[i]
        m = an < 0
        c = xi[m] - u
        c2 = np.sum(c * c, 1)
        M = w[m] * rho / (2.0 * math.pi * T) ** 1.5 * np.exp(-c2 / (2.0 * T))
        dM = np.column_stack([M / rho, M[:, None] * c / T, M * (c2 / (2.0 * T * T) - 1.5 / T)])  # (nin, 5)
        D[i] = psi[m].T @ dM
        d5[i] = an[m] @ dM
    return D, d5


@dataclass
class AdjointResult:
    J: float
    dJ_dmu0: float
    dJ_dTw: np.ndarray       # per boundary face (internal numbering), zero off the diffuse walls
    dJ_dalpha: np.ndarray    # per boundary face: the accommodation derivative at alpha = 1 (from below) of the
    #                          axis-aligned diffuse walls, NaN for other wall faces, zero off the walls
    iterations: int
    residual: float
    history: list

    def dJ_ddelta(self, mu0: float, delta: float) -> float:
        """dJ/d delta when mu_hat0 = 1 / (sqrt(2) delta)."""
        return -self.dJ_dmu0 * mu0 / delta


class KineticAdjoint:
    """Adjoint of M_dot at the converged state of a KineticSolver whose backend is a B200Backend (FP64 or mixed)."""

    def __init__(self, solver):
        self.sol = solver
        s, h = solver.s, solver.h
        self.check_scope()
        solver.prepare()
        self.nc, self.nb, self.nv = solver.nc, solver.nb, solver.nv
        xi = np.stack([np.asarray(s["xi_x"]), np.asarray(s["xi_y"]), np.asarray(s["xi_z"])], 1)
        self.rev_v = reversed_velocities(xi)
        self.rev_e = reverse_entries(s["csr_offsets"], s["csr_other"], h.csr_faces)
        self.flip = flipped_velocities(xi)
        self.axis = face_axes(np.asarray(s["bface_geom"], float).reshape(-1, 7)[:, 0:3]) if solver.nb else \
            np.zeros(0, np.int32)
        solver.backend.adjoint_begin(self.rev_v, self.rev_e, self.flip.ravel(), self.axis)
        bk = solver.bkind
        self.wall = np.flatnonzero(bk == abi.BC_DIFFUSE_WALL)
        self.pres = np.flatnonzero(bk == abi.BC_PRESSURE)
        ptype = solver.ptype[solver.bpatch] if self.nb else np.zeros(0, int)
        self.sgn = np.where(np.isin(ptype, _INLETS), -1.0, np.where(np.isin(ptype, _OUTLETS), 1.0, 0.0))
        self.sgn[(bk != abi.BC_PRESSURE) & (bk != abi.BC_VACUUM)] = 0.0
        self.nu = np.zeros(len(self.wall))
        self.history = []
        # the "limited" pressure-boundary reconstruction (the reference default): W_b also reads the neighbours'
        # states and the face states of the boundary sums, whose adjoint kappa (nb, 5) is iterated like nu
        self.limited = h.pressure_boundary_reconstruction != "cell" and len(self.pres) > 0
        self.kappa = np.zeros((self.nb, 5))
        self.fs_seed = np.zeros((self.nb, 5))
        if self.limited:
            self.recon = PressureReconstruction(solver)
            self.wib = self.recon.forward(solver.moments_, solver.face_state)
            self._face_state_constants()
        self._discrete_chains()

    # ---- derivatives through the discrete equilibrium ---------------------------------------------------------
    def _discrete_chains(self):
        """The cells whose Shakhov target is built on the discrete Maxwellian and the inflow faces corrected to it,
        with the per-state constants of their derivative chains (gsis_sim_b200.deq_adjoint)."""
        sol = self.sol
        s = sol.s
        self.deq_cells = np.zeros(0, np.int64)
        self.deq_pres = np.zeros(0, np.int64)
        self.deq_wall = np.zeros(0, np.int64)
        if not sol.discrete_eq:
            return
        grid = TensorGrid.from_setup(s)
        m = sol.moments_
        st = m[:, [0, 1, 2, 3, 4]]
        self.deq_cells = np.flatnonzero(~sol._deq_resolved(st))
        if len(self.deq_cells):
            self.cell_deq = CellDerivatives(grid, m[self.deq_cells], float(s["Pr"]), float(s["cold_bgk_temperature"]),
                                            float(s["deq_tolerance"]), int(s["deq_max_iterations"]))
            if not self.cell_deq.ok.all():
                raise AdjointScopeError("a cell's discrete-equilibrium Newton solve did not converge")
        # pressure faces: W_b of the owner ("cell" reconstruction) before the correction
        if len(self.pres):
            wb = self._pressure_states()
            need = (wb[:, 0] > 0) & (wb[:, 4] > 0) & ~sol._deq_resolved(wb)
            self.deq_pres = self.pres[need]
            if len(self.deq_pres):
                self.pres_deq = InflowDerivatives(grid, wb[need])
                keep = self.pres_deq.ok
                self.deq_pres = self.deq_pres[keep]
                self.pres_deq = InflowDerivatives(grid, wb[need][keep])
        if len(self.wall):
            h = sol.h
            T = h.patch_dbl[sol.bpatch[self.wall], 0] if sol.wall_T is None else sol.wall_T[self.wall]
            ws = np.column_stack([np.ones(len(self.wall)), h.patch_dbl[sol.bpatch[self.wall], 2:5], T])
            need = ~sol._deq_resolved(ws)
            if need.any():
                idv = InflowDerivatives(grid, ws[need])
                sel = np.flatnonzero(need)[idv.ok]
                self.deq_wall = sel  # indices into self.wall
                self.wall_deq = InflowDerivatives(grid, ws[sel])

    def _face_state_constants(self):
        """The face moments mom = sm[10:15] + s_in sm[15:20] of the last boundary sums (process_boundary_sums:
        s_in = rho_Gamma = -sm0 / sm5 on diffuse walls, 0 on vacuum faces, 1 elsewhere) and the derivatives of the
        incoming halves with respect to the inflow state of the pressure faces and of the walls whose face state a
        pressure face reads."""
        sol = self.sol
        sm = sol.bsums
        sm0, sm5 = sm[:, 0], sm[:, 5]
        with np.errstate(divide="ignore", invalid="ignore"):
            self.wall_pos = (sm5 < 0) & (-sm0 / sm5 > 0)
            rg = np.where(self.wall_pos, -sm0 / sm5, 0.0)
        s_in = np.ones(self.nb)
        bk = sol.bkind
        s_in[bk == abi.BC_DIFFUSE_WALL] = rg[bk == abi.BC_DIFFUSE_WALL]
        s_in[bk == abi.BC_VACUUM] = 0.0
        self.fs_mom = sm[:, 10:15] + s_in[:, None] * sm[:, 15:20]
        r = self.recon
        read = np.unique(r.bface[r.use]) if r.use.any() else np.zeros(0, np.int64)
        self.fs_read = read  # the boundary faces whose face state a pressure face reads
        self.fs_walls = read[bk[read] == abi.BC_DIFFUSE_WALL]
        s = sol.s
        xi = np.stack([np.asarray(s["xi_x"]), np.asarray(s["xi_y"]), np.asarray(s["xi_z"])], 1)
        w = np.asarray(s["weights"]) if s.get("weights") is not None else np.full(sol.nv, float(s["weight"]))
        nrm = sol.h.face_normal[sol.bf_global]
        # the inflow states as the device holds them (after the discrete-Maxwellian correction)
        self.Dp, _ = inflow_moment_derivatives(xi, w, nrm[self.pres], sol.inflow[self.pres][:, 1:6])
        self.Dw, self.d5w = inflow_moment_derivatives(xi, w, nrm[self.fs_walls], sol.inflow[self.fs_walls][:, 1:6])

    def _mom_bar(self):
        """Seeds on the face moments from kappa (zero on faces no pressure face reads)."""
        return face_moment_state_adjoint(self.fs_mom, self.kappa)

    def _face_moment_seeds(self):
        """The seeds of -kappa^T dFS/df (F_fs = fs - FS(f, ...)): per face the weights of w psi on the outgoing
        reconstructed values (and the mirrored incoming half of symmetry faces) for the device, and for diffuse walls
        the extra weight of w a on the outgoing values through rho_Gamma = -sm0 / sm5 (added to mu)."""
        mb = self._mom_bar()
        mu_extra = np.zeros(self.nb)
        sol = self.sol
        w = sol.bkind == abi.BC_DIFFUSE_WALL
        with np.errstate(divide="ignore", invalid="ignore"):
            c0 = np.where(w & self.wall_pos, np.sum(mb * sol.bsums[:, 15:20], 1) / sol.bsums[:, 5], 0.0)
        mu_extra[w] = c0[w] / sol.barea[w]
        return -mb, mu_extra

    def _pressure_states(self):
        """(rho_b, u_b, T_b) of the pressure faces from W_ib (update_pressure_inflow, src/kinetic/kinetic_solver.cpp:
        172-260): the owner cell's state ("cell" reconstruction) or its limited reconstruction at the face."""
        sol = self.sol
        h = sol.h
        b = self.pres
        m = sol.moments_
        o = sol.bowner[b]
        p_o, u_o, T_o = m[o, 5], m[o, 1:4], m[o, 4]
        if self.limited:
            p_o, u_o, T_o = self.wib[:, 0], self.wib[:, 1:4], self.wib[:, 4]
        patch = sol.bpatch[b]
        p_b = h.patch_dbl[patch, 1]
        inlet = np.isin(sol.ptype[patch], _INLETS)
        T_b = np.where(inlet, h.patch_dbl[patch, 0], T_o)
        cs = np.sqrt(h.gamma * T_o)
        du = (p_o - p_b) / ((p_o / T_o) * cs)
        n = h.face_normal[sol.bf_global[b]]
        un = np.einsum("na,na->n", u_o, n)
        zero_tan = h.patch_dbl[patch, 6] > 0.5
        u_b = np.where(zero_tan[:, None], (un + du)[:, None] * n, u_o + du[:, None] * n)
        return np.column_stack([p_b / T_b, u_b, T_b])

    # ---- scope ---------------------------------------------------------------------------------------------------
    def check_scope(self):
        sol = self.sol
        s, h = sol.s, sol.h
        if int(s["precision"]) not in (abi.KIN_PREC_FP64, abi.KIN_PREC_MIXED):
            raise AdjointScopeError("the adjoint needs precision = fp64 or mixed")
        if int(s["positivity"]) != 0:
            raise AdjointScopeError("positivity limiter")
        if h.closed_domain:
            raise AdjointScopeError("closed-domain mass scaling")
        if np.any(sol.bkind == abi.BC_MAXWELL_WALL):
            raise AdjointScopeError("Maxwell walls (accommodation < 1)")
        if np.any(sol.ptype == BOUNDARY_TYPES.index("mass_flow_inlet")):
            raise AdjointScopeError("mass-flow inlets")
        if float(s["cold_bgk_temperature"]) > 0.0:
            raise AdjointScopeError("cold-BGK switch")
        if sol.discrete_eq:
            if TensorGrid.from_setup(s) is None:
                raise AdjointScopeError("the discrete equilibrium's derivative needs a tensor velocity grid")
            sol.prepare()
            if sol.backend.deq_counts()[1] > 0:
                raise AdjointScopeError("a cell's discrete-equilibrium Newton solve failed")

    # ---- one evaluation of O(y) ----------------------------------------------------------------------------------
    def _mu(self):
        sol = self.sol
        mu = np.zeros(self.nb)
        sm0, sm5 = sol.bsums[:, 0], sol.bsums[:, 5]
        w = self.wall
        with np.errstate(divide="ignore", invalid="ignore"):
            pos = (sm5[w] < 0) & (-sm0[w] / sm5[w] > 0)
            mu[w] = np.where(pos, self.nu / (sol.barea[w] * sm5[w]), 0.0)
        j = self.sgn != 0
        mu[j] = -C_J * self.sgn[j]
        if self.limited:
            mu = mu + self._mu_extra
        return mu

    def _reduce(self, cells: bool = True, faces: bool = True):
        if self.limited:
            mom_seeds, self._mu_extra = self._face_moment_seeds()
            self.sol.backend.adjoint_face_moment_seeds(mom_seeds)
        cell, face = self.sol.backend.adjoint_reduce(self._mu(), cells=cells, faces=faces)
        from .backend import ADJ_CELL_SUMS, ADJ_FACE_SUMS

        if cells:
            cell = cell.reshape(self.nc, ADJ_CELL_SUMS)
            out = cell[:, :9].copy()
            d = self.deq_cells
            if len(d):
                out[d, 1:9] = self.cell_deq.lambda_sums(cell[d, 1:9], cell[d, 9:14], cell[d, 14:19])
            cell = out
        return (cell if cells else None), (face.reshape(max(self.nb, 0), ADJ_FACE_SUMS) if faces else None)

    def _pressure_chain(self, face):
        """Seeds on the cells' (p, u, T) (nc, 5) of the pressure faces' inflow: from the device's sums of the seeds
        on the incoming values (face), through the correction to the discrete Maxwellian, the acoustic correction
        (App. A.2) and W_ib; with the limited reconstruction also the seeds on the face states (self.fs_seed), which
        include the pressure faces' own incoming halves read by their face states (-kappa^T dFS/dW_b)."""
        sol = self.sol
        m = sol.moments_
        cell_bar = np.zeros((self.nc, 5))
        self.fs_seed = np.zeros((self.nb, 5))
        b = self.pres
        if len(b) == 0:
            return cell_bar
        inf = sol.inflow[b]
        rb, Tb = inf[:, 1], inf[:, 5]
        S = face[b]
        rho_bar = S[:, 0] / rb
        u_bar = S[:, 1:4] / Tb[:, None]
        T_bar = S[:, 4] / (2.0 * Tb * Tb) - 1.5 * S[:, 0] / Tb
        if self.limited:
            th = -np.einsum("fk,fkj->fj", self._mom_bar()[b], self.Dp)
            rho_bar, u_bar, T_bar = rho_bar + th[:, 0], u_bar + th[:, 1:4], T_bar + th[:, 4]
        if len(self.deq_pres):
            # through the correction of W_b to its discrete Maxwellian
            k = np.searchsorted(b, self.deq_pres)
            tb = self.pres_deq.pullback(np.column_stack([rho_bar[k], u_bar[k], T_bar[k]]))
            rho_bar, u_bar, T_bar = rho_bar.copy(), u_bar.copy(), T_bar.copy()
            rho_bar[k], u_bar[k], T_bar[k] = tb[:, 0], tb[:, 1:4], tb[:, 4]
        o = sol.bowner[b]
        h = sol.h
        n = h.face_normal[sol.bf_global[b]]
        patch = sol.bpatch[b]
        inlet = np.isin(sol.ptype[patch], _INLETS)
        if self.limited:
            p_i, u_i, T_i = self.wib[:, 0], self.wib[:, 1:4], self.wib[:, 4]
        else:
            p_i, u_i, T_i = m[o, 5], m[o, 1:4], m[o, 4]
        p_bar, ui_bar, Ti_bar = pressure_face_adjoint(p_i, u_i, T_i, n, h.patch_dbl[patch, 1], inlet,
                                                      h.patch_dbl[patch, 6] > 0.5, h.gamma, rho_bar, u_bar, T_bar)
        wb = np.column_stack([p_bar, ui_bar, Ti_bar])
        if self.limited:
            cell_bar, self.fs_seed = self.recon.vjp(wb)
        else:
            np.add.at(cell_bar, o, wb)
        return cell_bar

    def _coefficients(self, cell, face):
        sol = self.sol
        m = sol.moments_
        rho, T = m[:, 0], m[:, 4]
        rho_b, u_b, T_b, q_b, coll = collision_moment_adjoint(m, sol.volume, float(sol.s["mu0"]),
                                                              float(sol.s["omega"]), cell)
        if len(self.pres):
            cb = self._pressure_chain(face)
            # p = rho T
            rho_b = rho_b + cb[:, 0] * T
            T_b = T_b + cb[:, 0] * rho + cb[:, 4]
            u_b = u_b + cb[:, 1:4]
        return moment_expansion_coefficients(m, rho_b, u_b, T_b, q_b), coll

    def _refresh_kappa(self, face):
        """kappa <- -(the face-state rows of y^T dF/dx - dJ/dx without kappa) (Jacobi on the face-state equations)."""
        if self.limited:
            self._pressure_chain(face)
            k_old = self.kappa
            self.kappa = -self.fs_seed
            return float(np.sqrt(np.sum((self.kappa - k_old) ** 2))), float(np.sqrt(np.sum(self.kappa ** 2)))
        return 0.0, 0.0

    def operator(self, lam=None, nu=None, with_objective=True):
        """O(y) (or y^T dF/dx without the objective term) for the given lambda (storage order) and auxiliary adjoint
        nu: the wall densities' (n_wall), followed with the limited pressure reconstruction by the face states'
        kappa (n_bfaces x 5). Returns (O_f (nc, nv), O_aux in the layout of nu)."""
        be = self.sol.backend
        nw = len(self.wall)
        if lam is not None:
            be.adjoint_set(np.asarray(lam, float))
        if nu is not None:
            nu = np.asarray(nu, float).ravel()
            self.nu = nu[:nw].copy()
            if self.limited and len(nu) > nw:
                self.kappa = nu[nw:].reshape(self.nb, 5).copy()
        sgn = self.sgn
        if not with_objective:
            self.sgn = np.zeros_like(sgn)
        try:
            cell, face = self._reduce()
            coef, _ = self._coefficients(cell, face)
            _, op = be.adjoint_update(coef, run_passes=False, want_operator=True)
        finally:
            self.sgn = sgn
        o_aux = face[self.wall, 0] + self.nu
        if self.limited:
            o_aux = np.concatenate([o_aux, (self.kappa + self.fs_seed).ravel()])
        return op.reshape(self.nc, self.nv), o_aux

    # ---- the solve -----------------------------------------------------------------------------------------------
    def solve(self, tol: float = 1e-10, max_iterations: int = 5000, inner: int | None = None,
              callback=None, stall_iterations: int | None = None) -> AdjointResult:
        """Iterate to ||O_f||_2 / ||O_f(0)||_2 < tol (and the wall densities settled to tol); return the gradients.

        stall_iterations: also stop once the residual has not fallen below 0.99 of its best value for that many outer
        iterations (the storage floor of a mixed-precision handle, where lambda is FP32); the result's residual says
        where it stopped.

        Mirrors the forward CIS iteration: per outer iteration the coupling terms (moment expansion of the cell
        parameters, pressure-face chain) are evaluated once and frozen for `inner` transposed transport sweeps
        (default: the set-up's inner_sweeps); before every sweep the wall adjoint is recomputed from the current
        lambda, as the forward recomputes rho_Gamma from the current f. The outer iteration then has the spectrum of the forward's. `max_iterations` counts
        outer iterations; the residual is that of the first sweep of each outer iteration (fresh coupling)."""
        be = self.sol.backend
        inner = max(1, int(self.sol.h.inner_sweeps if inner is None else inner))
        walls = len(self.wall) > 0
        ref = None
        it = 0
        res = math.inf
        best, since_best = math.inf, 0
        for it in range(1, max_iterations + 1):
            # wall adjoint first, from the current lambda (the transpose of the forward's rho_Gamma = Phi(f) before
            # each sweep; a one-sweep lag on these strongly coupled unknowns can make the iteration unstable)
            nu_old = self.nu
            dk = (0.0, 0.0)
            if walls or self.limited:
                _, face = self._reduce(cells=False)
                self.nu = -face[self.wall, 0]
                dk = self._refresh_kappa(face)
            cell, face = self._reduce()
            coef, _ = self._coefficients(cell, face)
            res_cell, _ = be.adjoint_update(coef, run_passes=True)
            nu_new = self.nu
            dnu = float(np.sqrt(np.sum((nu_new - nu_old) ** 2)))
            r = math.sqrt(float(np.sum(res_cell)))
            if ref is None:
                ref = max(r, 1e-300)
            res = max(r / ref, dnu / max(float(np.sqrt(np.sum(nu_new ** 2))), 1e-300) if len(nu_new) else 0.0,
                      dk[0] / max(dk[1], 1e-300) if self.limited else 0.0)
            self.history.append(r)
            if callback is not None:
                callback(it, r)
            if not math.isfinite(r):
                raise FloatingPointError(f"adjoint iteration diverged at outer iteration {it}")
            if r / ref < tol and (len(nu_new) == 0 or dnu <= tol * max(float(np.abs(nu_new).max()), 1e-300)) and \
                    (not self.limited or dk[0] <= tol * max(dk[1], 1e-300)):
                break
            if r < 0.99 * best:
                best, since_best = r, 0
            else:
                since_best += 1
            if stall_iterations is not None and since_best >= stall_iterations:
                break
            for _ in range(1, inner):
                if walls or self.limited:
                    _, face = self._reduce(cells=False)
                    self.nu = -face[self.wall, 0]
                    self._refresh_kappa(face)
                # the transport's seeds with the new nu (the coupling sums stay frozen over the inner sweeps)
                self._reduce(cells=False, faces=False)
                be.adjoint_update(coef, run_passes=True)
        return self.gradients(it, res)

    def gradients(self, iterations: int = 0, residual: float = 0.0) -> AdjointResult:
        sol = self.sol
        cell, face = self._reduce()
        _, coll = self._coefficients(cell, face)
        mu0 = float(sol.s["mu0"])
        dmu = -float(np.sum(coll / mu0 * cell[:, 0]))
        dTw = np.zeros(self.nb)
        w = self.wall
        if len(w):
            # adjoint of the wall inflow Maxwellian's parameters (rho', u', T'): through the wall term rho_Gamma M of
            # the residual and through sm5 of the wall-density equation
            rp, T = sol.inflow[w, 1], sol.inflow[w, 5]
            S = face[w]
            rg = sol.inflow[w, 0]
            sm0, sm5 = sol.bsums[w, 0], sol.bsums[w, 5]
            dR = np.column_stack([rg * S[:, 0] / rp, rg[:, None] * S[:, 1:4] / T[:, None],
                                  rg * (S[:, 4] / (2.0 * T * T) - 1.5 * S[:, 0] / T)])
            D5 = np.column_stack([S[:, 6] / rp, S[:, 10:13] / T[:, None], S[:, 5] / (2.0 * T * T) - 1.5 * S[:, 6] / T])
            with np.errstate(divide="ignore", invalid="ignore"):
                pos = (sm5 < 0) & (-sm0 / sm5 > 0)
                dPhi = np.where(pos[:, None], (sm0 / (sm5 * sm5))[:, None] * D5, 0.0)
            th = -(dR - self.nu[:, None] * dPhi)
            if self.limited and len(self.fs_walls):
                # + kappa^T dFS/dtheta: the face states of walls a pressure face reads, through the incoming half
                # rho_Gamma sm[15:20] (rho_Gamma = -sm0 / sm5)
                fw = self.fs_walls
                k = np.searchsorted(w, fw)
                mb = self._mom_bar()[fw]
                sm0f, sm5f = sol.bsums[fw, 0], sol.bsums[fw, 5]
                pos_f = self.wall_pos[fw]
                rgf = np.where(pos_f, -sm0f / np.where(pos_f, sm5f, -1.0), 0.0)
                drg = np.where(pos_f, sm0f / np.where(pos_f, sm5f * sm5f, 1.0), 0.0)
                smi = sol.bsums[fw, 15:20]
                th[k] += rgf[:, None] * np.einsum("fk,fkj->fj", mb, self.Dw) + \
                    (drg * np.sum(mb * smi, 1))[:, None] * self.d5w
            if len(self.deq_wall):
                # through the correction of (1, u_w, T_w) to its discrete Maxwellian
                th[self.deq_wall] = self.wall_deq.pullback(th[self.deq_wall])
            dTw[w] = th[:, 4]
        # accommodation at alpha = 1: the inflow rho M + (1 - alpha) f_spec of a Maxwell wall and its zero-net-flux
        # density rho = -(sm0 + (1 - alpha) S_spec) / sm5; dJ/dalpha = A1 + A2 + nu S_spec / sm5
        dA = np.zeros(self.nb)
        if len(w):
            S = face[w]
            with np.errstate(divide="ignore", invalid="ignore"):
                nu_t = np.where(pos, self.nu * S[:, 9] / sm5, 0.0)
            dA[w] = np.where(self.axis[w] >= 0, S[:, 7] + S[:, 8] + nu_t, np.nan)
            if self.limited and len(self.fs_walls):
                # + kappa^T dFS/dalpha: rho_Gamma = -(sm0 + (1 - alpha) S_spec) / sm5 and the specular part
                # (1 - alpha) sum_in w psi f_spec of the wall's face moments
                fw = self.fs_walls
                mb = self._mom_bar()[fw]
                Sf = face[fw]
                pos_f = self.wall_pos[fw]
                ratio = np.where(pos_f, Sf[:, 9] / np.where(pos_f, sol.bsums[fw, 5], -1.0), 0.0)
                dA[fw] += np.sum(mb * (ratio[:, None] * sol.bsums[fw, 15:20] - Sf[:, 13:18]), 1)
        J = sol.mass_flow()[2]
        return AdjointResult(J=J, dJ_dmu0=dmu, dJ_dTw=dTw, dJ_dalpha=dA, iterations=iterations, residual=residual,
                             history=list(self.history))

    def close(self):
        self.sol.backend.adjoint_end()


# ---- torch.autograd: M_dot as a differentiable function of (delta, T_w per wall face, alpha per wall face) -----

class MassFlowProblem:
    """M_dot of one kinetic case as a function of the rarefaction parameter delta, the temperature of every diffuse
    wall face and the accommodation of every diffuse wall face. The forward is a CIS solve on a B200Backend converged
    to `tol`; the derivative is the discrete adjoint of that fixed point (KineticAdjoint). `mass_flow` makes it a
    torch.autograd.Function.

    setup, host: a set-up in the adjoint's scope (see KineticAdjoint.check_scope). Its mu_hat0 is 1 / (sqrt(2) delta)
    (derive_quantities), so delta defaults to 1 / (sqrt(2) mu_hat0) and mu_hat0 scales as 1 / delta for other
    values. `wall_faces` (internal boundary-face indices of the diffuse walls) is the order of the T_wall and alpha
    vectors."""

    def __init__(self, setup: abi.SetupArrays, host, delta: float | None = None, tol: float = 1e-12,
                 max_iterations: int = 20000,
                 adjoint_tol: float = 1e-12, adjoint_max_iterations: int = 20000,
                 initial=(1.0, (0.0, 0.0, 0.0), 1.0), device: int = 0, stall_iterations: int | None = None,
                 polish_iterations: int = 20):
        self.setup, self.host = setup, host
        self.mu0_0 = float(setup["mu0"])
        self.delta0 = 1.0 / (math.sqrt(2.0) * self.mu0_0) if delta is None else float(delta)
        bpatch = np.asarray(setup["bface_patch"]) if setup.n_bfaces else np.zeros(0, np.int32)
        bkind = host.patch_int[:, 0][bpatch] if setup.n_bfaces else np.zeros(0, np.int32)
        self.wall_faces = np.flatnonzero(bkind == abi.BC_DIFFUSE_WALL)
        self.T_patch = np.asarray(host.patch_dbl[bpatch[self.wall_faces], 0], float)
        self.tol, self.max_iterations = float(tol), int(max_iterations)
        self.adjoint_tol, self.adjoint_max_iterations = float(adjoint_tol), int(adjoint_max_iterations)
        self.initial = initial
        self.device = device
        # mixed precision: accept the storage floor (the residual no longer falls below 0.99 of its best value for
        # this many iterations) as convergence of the forward and adjoint solves
        self.stall_iterations = stall_iterations
        # mixed precision: FP64 CIS iterations from the converged mixed state before the adjoint (polish_state)
        self.polish_iterations = int(polish_iterations)
        self.last_polish = None

    def solve(self, delta: float, T_wall=None, alpha=None):
        """Converged forward solve at (delta, T_wall, alpha) -> (solver, M_dot). T_wall: one temperature per wall
        face (None: the patch temperatures). alpha: one accommodation per wall face, which must be 1: the adjoint
        gives the derivative at alpha = 1 from below (alpha <= 1), and walls with alpha < 1 are Maxwell walls, outside
        its scope."""
        if not delta > 0:
            raise ValueError(f"delta must be positive, got {delta}")
        if alpha is not None and np.any(np.asarray(alpha, float).reshape(-1) != 1.0):
            raise AdjointScopeError("the accommodation derivative is taken at alpha = 1 (from below); alpha < 1 makes "
                                    "the walls Maxwell walls, outside the adjoint's scope")
        sol = self._solver(delta, T_wall)
        be = sol.backend
        try:
            r = math.inf
            best, since_best, stalled = math.inf, 0, False
            for _ in range(self.max_iterations):
                r = sol.sweep().residual
                if r < self.tol:
                    break
                if r < 0.99 * best:
                    best, since_best = r, 0
                else:
                    since_best += 1
                if self.stall_iterations is not None and since_best >= self.stall_iterations:
                    stalled = True
                    break
            self.last_residual = r
            if not (r < self.tol or stalled):
                raise FloatingPointError(f"forward CIS stopped at residual {r:.3e} after {self.max_iterations} "
                                         f"iterations (tolerance {self.tol:g})")
        except BaseException:
            be.close()
            raise
        return sol, sol.mass_flow()[2]

    def _solver(self, delta: float, T_wall=None, precision: int | None = None):
        """A KineticSolver on a new B200Backend at (delta, T_wall), initialised to the problem's uniform state."""
        from .backend import B200Backend
        from .solver import KineticSolver

        s = abi.SetupArrays(dict(self.setup.arrays), dict(self.setup.scalars))  # arrays shared, scalars own
        s["mu0"] = self.mu0_0 if float(delta) == self.delta0 else self.mu0_0 * (self.delta0 / float(delta))
        if precision is not None:
            s["precision"] = precision
        be = B200Backend(s, device=self.device)
        try:
            sol = KineticSolver(s, self.host, be)
            if T_wall is not None:
                Tw = np.asarray(T_wall, float).reshape(-1)
                if Tw.shape != self.wall_faces.shape:
                    raise ValueError(f"T_wall: {Tw.shape[0]} values for {len(self.wall_faces)} wall faces")
                T = np.ones(s.n_bfaces)
                T[self.wall_faces] = Tw
                sol.set_wall_temperature(T)
            rho, u, T0 = self.initial
            sol.initialize_uniform(rho, u, T0)
        except BaseException:
            be.close()
            raise
        return sol

    def polish_state(self, sol, delta: float):
        """FP64 defect correction of a converged mixed-precision state before its adjoint: `polish_iterations` CIS
        iterations of the FP64 solver from the mixed solver's f, whose result (rounded to FP32) replaces it in a new
        mixed-precision solver; `sol` is released (the two handles are not held at the same time: at full size
        they do not fit one device together). Returns the new solver.

        Why: the mixed solve stops at its storage floor, where every value of f sits within an ulp of FP32 but the
        pattern of roundings is not monotone between neighbours. In flat regions that creates stencil extrema that
        the FP64 state does not have, and the limiter's derivative there (of order 1 / (g . ds)) makes the
        linearised iteration unstable: on the 134,528-cell tube the FP64 adjoint at the mixed state diverges, while
        the mixed adjoint at the FP64 state rounded to FP32 converges like the FP64 one. Twenty FP64 iterations
        (residual 7.5e-8 -> 4e-10) remove the pattern; five do not."""
        if int(sol.s["precision"]) != abi.KIN_PREC_MIXED or self.polish_iterations <= 0:
            return sol
        f = sol.distribution()
        Tw = None if sol.wall_T is None else np.asarray(sol.wall_T, float)[self.wall_faces].copy()
        self.release(sol)
        s64 = self._solver(delta, Tw, precision=abi.KIN_PREC_FP64)
        history = []
        try:
            s64.set_distribution(f)
            for _ in range(self.polish_iterations):
                history.append(s64.sweep().residual)
            f = s64.distribution()
        finally:
            self.release(s64)
        out = self._solver(delta, Tw)
        out.set_distribution(f)
        self.last_polish = history
        return out

    def gradients(self, sol, delta: float):
        """(dM_dot/d delta, dM_dot/dT_w per wall face, dM_dot/d alpha per wall face at alpha = 1) at a converged
        solve; the alpha derivative is NaN on wall faces not aligned with a coordinate axis. A mixed-precision state
        is first polished in FP64 (polish_state; `sol` is then released here and the caller's release is a no-op)."""
        polished = int(sol.s["precision"]) == abi.KIN_PREC_MIXED and self.polish_iterations > 0
        sol = self.polish_state(sol, delta)
        try:
            ka = KineticAdjoint(sol)
            try:
                res = ka.solve(tol=self.adjoint_tol, max_iterations=self.adjoint_max_iterations,
                               stall_iterations=self.stall_iterations)
            finally:
                ka.close()
        finally:
            if polished:
                self.release(sol)
        if not (res.residual < self.adjoint_tol or
                (self.stall_iterations is not None and res.iterations < self.adjoint_max_iterations)):
            raise FloatingPointError(f"adjoint stopped at residual {res.residual:.3e} after {res.iterations} "
                                     f"iterations (tolerance {self.adjoint_tol:g})")
        w = self.wall_faces
        return res.dJ_ddelta(float(sol.s["mu0"]), float(delta)), res.dJ_dTw[w].copy(), res.dJ_dalpha[w].copy()

    def release(self, sol):
        sol.backend.close()


_FUNCTION = None


def _mass_flow_function():
    """The torch.autograd.Function of mass_flow (built on first use, so that importing this module needs no torch)."""
    global _FUNCTION
    if _FUNCTION is not None:
        return _FUNCTION
    import torch

    class MassFlowFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, delta, T_wall, alpha, problem):
            Tw = None if T_wall is None else T_wall.detach().to("cpu", torch.float64).numpy()
            al = None if alpha is None else alpha.detach().to("cpu", torch.float64).numpy()
            state, J = problem.solve(float(delta), Tw, al)
            ctx.problem, ctx.state, ctx.delta = problem, state, float(delta)
            ctx.given = (T_wall is not None, alpha is not None)
            return torch.tensor(J, dtype=torch.float64, device=delta.device)

        @staticmethod
        def backward(ctx, grad):
            # one adjoint solve per forward; its gradients serve every later backward through the same graph
            if getattr(ctx, "grads", None) is None:
                try:
                    ctx.grads = ctx.problem.gradients(ctx.state, ctx.delta)
                finally:
                    ctx.problem.release(ctx.state)
                    ctx.state = None
            g_delta, g_T, g_alpha = ctx.grads
            g = grad.to(torch.float64)
            dev = g.device
            out_delta = g * torch.tensor(g_delta, dtype=torch.float64, device=dev)
            out_T = g * torch.as_tensor(g_T, dtype=torch.float64, device=dev) if ctx.given[0] else None
            out_alpha = g * torch.as_tensor(g_alpha, dtype=torch.float64, device=dev) if ctx.given[1] else None
            return out_delta, out_T, out_alpha, None

    _FUNCTION = MassFlowFunction
    return _FUNCTION


def mass_flow(problem, delta, T_wall=None, alpha=None):
    """M_dot as a differentiable torch scalar (float64): the forward solves the kinetic case to convergence, the
    backward runs the discrete adjoint once and returns dM_dot/d delta, dM_dot/dT_w and dM_dot/d alpha (per wall
    face, in problem.wall_faces order; alpha at 1 from below). `problem` is a MassFlowProblem, or any object with the
    same solve / gradients / release methods. T_wall and alpha may be None (patch temperatures, alpha = 1; no
    gradient). The converged solver is kept for the backward, which releases it after the adjoint solve."""
    import torch

    if not isinstance(delta, torch.Tensor):
        delta = torch.tensor(float(delta), dtype=torch.float64)
    return _mass_flow_function().apply(delta, T_wall, alpha, problem)

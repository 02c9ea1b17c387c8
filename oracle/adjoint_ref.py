"""CPU reference of the discrete adjoint of the converged CIS fixed point (TEST INFRASTRUCTURE: used only by tests/
as the checker of the B200 adjoint; never by the product).

The steady discrete problem that the CIS iteration of the reference converges to (src/kinetic/kinetic_solver.cpp
prepare + sweep, src/kinetic/kinetic_kernels.hpp) is written here as one differentiable map in torch (float64, CPU),
and its transposed Jacobian is taken by autograd:

  unknowns   x = (f [cell][velocity], rho_Gamma [diffuse wall face], with the "limited" pressure-boundary
             reconstruction also fs [boundary face][rho, u, T])
  equations  R(f, rho_Gamma, fs; p) = 0   the residual of residual_value (kinetic_kernels.hpp:238-278) with the
                                          limited LSQ gradient (:161-201), the Shakhov target of the cell moments
                                          (make_cell_params :451-471) and the inflow of the boundary faces
             rho_Gamma - Phi(f, rho_Gamma) = 0   zero net mass flux of each diffuse wall face
                                          (process_boundary_sums, kinetic_solver.cpp:280-335)
             fs - FS(f, fs) = 0           the face states of the boundary sums (the same function), which the limited
                                          reconstruction of the pressure faces' W_b reads (update_pressure_inflow,
                                          kinetic_solver.cpp:172-260); FS of a pressure face depends on fs through
                                          its own inflow
  objective  J = M_dot = 1/2 (mdot_in + mdot_out) sqrt(2/pi) from the patch flows of the boundary sums
  parameters p = (mu_hat0, T_w per boundary face, accommodation alpha per wall face at 1: the partially specular
             inflow rho M + (1 - alpha) f_spec of axis-aligned walls, maxwell_inflow / reflected_value,
             kinetic_kernels.hpp:86-133); delta enters only through mu_hat0 = 1 / (sqrt(2) delta)

The adjoint y solves (dF/dx)^T y = dJ/dx (GMRES over autograd vector-Jacobian products) and
dJ/dp = dJ/dp|_x - y^T dF/dp.

Scope (the same as the B200 adjoint; `check_scope` raises outside it): diffuse walls, pressure inlets / outlets with
the "limited" or the "cell" boundary reconstruction (W_b reconstructed at the face, or the owner cell's state; App.
A.2 acoustic correction), vacuum, symmetry and periodic faces; Venkatakrishnan limiter (absolute or relative epsilon) or none; no positivity limiter, no closed-domain
scaling, no mass-flow inlets, no Maxwell walls.

Equilibrium: the continuous Maxwellian, or the discrete one (kinetic.equilibrium = "discrete", the reference default):
for every cell and inflow state the velocity grid does not resolve (deq_resolved, src/kinetic/
discrete_equilibrium.hpp:35-48) the Maxwellian is E = exp(beta . psi(c)), psi = (1, c, |c|^2 / 2), c = xi - u, with
beta solving sum_q w E psi = (rho, 0, 0, 0, 3/2 rho T) (deq_* :56-188), and the cells' Shakhov target carries the
correction gamma . psi that makes its polynomial part conservative (deq_shakhov_correction :183-188). The Newton
iteration runs without gradients to convergence; one Newton step from the converged beta then carries the
derivative (dbeta = -J^-1 dG, the implicit function theorem), and gamma = -J^-1 sum w E P psi is differentiated as it
is.
"""
from __future__ import annotations

import math

import numpy as np
import torch

BC_DIFFUSE_WALL, BC_PRESSURE, BC_VACUUM, BC_SYMMETRY, BC_PERIODIC, BC_MAXWELL_WALL = 0, 1, 2, 3, 4, 5
LIMITER_NONE, LIMITER_ABS, LIMITER_REL = 0, 1, 2
# BoundaryType indices (gsis_sim_b200.kinetic_setup.BOUNDARY_TYPES)
T_INLETS = ("pressure_inlet", "mass_flow_inlet")
T_OUTLETS = ("pressure_outlet", "vacuum")


class ScopeError(ValueError):
    pass


def _t(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype)


class SteadyMap:
    """The steady map F(x; p) and objective J(x; p) of one kinetic set-up (internal numbering, storage order)."""

    def __init__(self, setup, host):
        from gsis_sim_b200.kinetic_setup import BOUNDARY_TYPES

        s = setup
        self.nc, self.nv, self.nb = s.n_cells, s.nv, s.n_bfaces
        nc, nv = self.nc, self.nv
        self.xi = torch.stack([_t(s["xi_x"]), _t(s["xi_y"]), _t(s["xi_z"])], 1)  # (nv, 3)
        w = s.arrays.get("weights") if hasattr(s, "arrays") else None
        self.w = _t(w) if w is not None else torch.full((nv,), float(s["weight"]), dtype=torch.float64)
        off = np.asarray(s["csr_offsets"], np.int64)
        cnt = np.diff(off)
        E = int(cnt.max())
        self.E = E
        ent = off[:-1, None] + np.arange(E)[None, :]
        mask = np.arange(E)[None, :] < cnt[:, None]
        ent = np.where(mask, ent, 0)
        geom = np.asarray(s["csr_geom"], float).reshape(-1, 12)[ent]  # (nc, E, 12)
        other = np.where(mask, np.asarray(s["csr_other"])[ent], -1)
        bface = np.where(mask, np.asarray(s["csr_bface"])[ent], -1)
        bkind = np.asarray(s["bface_kind"])
        kind = np.where(bface >= 0, bkind[np.maximum(bface, 0)], -1)
        self.mask = torch.as_tensor(mask)
        self.internal = torch.as_tensor(mask & (other >= 0))
        self.other = torch.as_tensor(np.maximum(other, 0))
        self.bface = torch.as_tensor(np.maximum(bface, 0))
        self.kind = torch.as_tensor(np.where(mask, kind, -2))
        self.S, self.ds, self.dn, self.c = (_t(geom[..., 3 * k:3 * k + 3]) for k in range(4))
        self.eps2 = _t(s["eps2"])
        self.limiter = int(s["limiter_mode"])
        mx = np.asarray(s["bface_mirror_xor"])
        q = np.arange(nv)
        self.mirror = torch.as_tensor(np.where((kind == BC_SYMMETRY)[..., None], q[None, None, :] ^
                                               mx[np.maximum(bface, 0)][..., None], q[None, None, :]))
        bg = np.asarray(s["bface_geom"], float).reshape(-1, 7)
        self.bn, self.barea, self.bd = _t(bg[:, 0:3]), _t(bg[:, 3]), _t(bg[:, 4:7])
        self.bowner = torch.as_tensor(np.asarray(s["bface_owner"], np.int64))
        self.bkind = torch.as_tensor(bkind)
        self.bpatch = np.asarray(s["bface_patch"])
        self.volume = _t(s["volume"])
        self.discrete = bool(int(s["discrete_eq"]))
        self.deq_lo, self.deq_hi = np.asarray(s["deq_lo"], float), np.asarray(s["deq_hi"], float)
        self.deq_d, self.deq_crit = np.asarray(s["deq_d"], float), float(s["deq_criterion"])
        self.deq_tol, self.deq_maxit = float(s["deq_tolerance"]), int(s["deq_max_iterations"])
        self.omega, self.Pr = float(s["omega"]), float(s["Pr"])
        self.mu0 = float(s["mu0"])
        self.cold = float(s["cold_bgk_temperature"])
        self.gamma = host.gamma
        pd = np.asarray(host.patch_dbl, float)
        ptype = np.asarray(host.patch_int)[:, 3]
        self.ptype_names = [BOUNDARY_TYPES[t] for t in ptype]
        bp = self.bpatch
        self.T_patch = _t(pd[bp, 0])
        self.p_patch = _t(pd[bp, 1])
        self.u_patch = _t(pd[bp, 2:5])
        self.zero_tan = torch.as_tensor(pd[bp, 6] > 0.5)
        self.inlet_face = torch.as_tensor(np.array([self.ptype_names[p] in T_INLETS for p in bp], bool))
        self.outlet_face = torch.as_tensor(np.array([self.ptype_names[p] in T_OUTLETS for p in bp], bool))
        self.wall = self.bkind == BC_DIFFUSE_WALL
        self.wall_idx = torch.nonzero(self.wall).ravel()
        # specular reflection of axis-aligned walls (the accommodation derivative at alpha = 1): the velocity with the
        # normal component negated, per boundary face and per stencil entry
        xi = np.stack([np.asarray(s["xi_x"]), np.asarray(s["xi_y"]), np.asarray(s["xi_z"])], 1)
        key = {tuple(np.round(x * 2.0 ** 30).astype(np.int64).tolist()): i for i, x in enumerate(xi)}
        flips = []
        for a in range(3):
            sg = np.ones(3)
            sg[a] = -1.0
            flips.append([key.get(tuple(np.round(x * sg * 2.0 ** 30).astype(np.int64).tolist()), -1) for x in xi])
        flips = np.array(flips)
        an = np.abs(bg[:, 0:3])
        axis = np.argmax(an, 1)
        aligned = np.abs(an[np.arange(len(an)), axis] - 1.0) < 1e-10
        self.bflip = torch.as_tensor(np.where(aligned[:, None], flips[axis], q[None, :]))  # (nb, nv)
        self.baligned = torch.as_tensor(aligned)
        self.eflip = self.bflip[self.bface]  # (nc, E, nv)
        self.setup, self.host = setup, host
        self.n_wall = len(self.wall_idx)
        # per boundary face: the storage position of the mirrored velocity (symmetry faces), q elsewhere
        self.bmirror = torch.as_tensor(np.where((bkind == BC_SYMMETRY)[:, None], q[None, :] ^ mx[:, None],
                                                q[None, :]))
        # the "limited" pressure-boundary reconstruction (the reference default): the face states of the boundary
        # sums become auxiliary unknowns
        self.limited = (host.pressure_boundary_reconstruction != "cell" and bool(torch.any(self.bkind == BC_PRESSURE)))
        if self.limited:
            self._pressure_stencils(s, host)
        self.n_aux = self.n_wall + (5 * self.nb if self.limited else 0)

    def _pressure_stencils(self, s, host):
        """Padded CSR stencils of the owners of the pressure faces (update_pressure_inflow, kinetic_solver.cpp:172-260)
        with the host geometry the solver uses."""
        pres = np.flatnonzero(self.bkind.numpy() == BC_PRESSURE)
        off = np.asarray(s["csr_offsets"], np.int64)
        own = np.asarray(s["bface_owner"], np.int64)[pres]
        cnt = off[own + 1] - off[own]
        E = int(cnt.max())
        ent = off[own][:, None] + np.arange(E)[None, :]
        mask = np.arange(E)[None, :] < cnt[:, None]
        ent = np.where(mask, ent, 0)
        other = np.where(mask, np.asarray(s["csr_other"])[ent], -1)
        bface = np.where(mask, np.asarray(s["csr_bface"])[ent], -1)
        bkind = np.asarray(s["bface_kind"])
        periodic = mask & (bface >= 0) & (bkind[np.maximum(bface, 0)] == BC_PERIODIC)
        fk = np.asarray(host.csr_faces)[ent]
        cc = np.asarray(host.cell_center, float)
        fg = host.n_internal_faces + pres
        self.p_idx = torch.as_tensor(pres)
        self.p_own = torch.as_tensor(own)
        self.p_mask = torch.as_tensor(mask)
        self.p_internal = torch.as_tensor(mask & (other >= 0))
        self.p_other = torch.as_tensor(np.maximum(other, 0))
        self.p_bmask = torch.as_tensor(mask & (bface >= 0) & ~periodic)
        self.p_bface = torch.as_tensor(np.maximum(bface, 0))
        self.p_periodic = torch.as_tensor(periodic)
        self.p_lsq = _t(np.asarray(host.lsq, float)[ent])                                   # (np, E, 3)
        self.p_dx = _t(np.asarray(host.face_center, float)[fk] - cc[own][:, None, :])       # (np, E, 3)
        self.p_dxb = _t(np.asarray(host.face_center, float)[fg] - cc[own])                  # (np, 3)
        self.p_eps2 = _t(host.limiter_k ** 3 * np.asarray(s["volume"], float)[own])
        self.p_limit = int(s["limiter_mode"]) != LIMITER_NONE

    def split_aux(self, z):
        """The auxiliary unknowns (rho_Gamma of the walls, then the face states (nb, 5) with the limited
        reconstruction) of one vector."""
        rg = z[:self.n_wall]
        fs = z[self.n_wall:].view(self.nb, 5) if self.limited else None
        return rg, fs

    # ---- scope ---------------------------------------------------------------------------------------------------
    def check_scope(self, solver=None):
        s, h = self.setup, self.host
        if int(s["positivity"]) != 0:
            raise ScopeError("positivity limiter")
        if h.closed_domain:
            raise ScopeError("closed-domain mass scaling")
        if torch.any(self.bkind == BC_MAXWELL_WALL):
            raise ScopeError("Maxwell walls (alpha < 1)")
        if "mass_flow_inlet" in self.ptype_names:
            raise ScopeError("mass-flow inlets")
        if int(s["deq_fallback_collisionless"]) and solver is not None and solver.discrete_eq:
            if solver.backend.deq_counts()[1] > 0:
                raise ScopeError("a cell's discrete equilibrium failed (collisionless fallback)")

    # ---- pieces --------------------------------------------------------------------------------------------------
    def moments(self, f):
        w = self.w
        rho = f @ w
        u = (f * w) @ self.xi / rho[:, None]
        c = self.xi[None, :, :] - u[:, None, :]
        c2 = (c * c).sum(-1)
        p = ((f * w) * c2).sum(1) / 3.0
        T = p / rho
        q = 0.5 * ((f * w * c2)[..., None] * c).sum(1)
        return rho, u, T, p, q

    def resolved(self, rho, u, T):
        """deq_resolved (src/kinetic/discrete_equilibrium.hpp:35-48) of n states (no gradient)."""
        u = u.detach().numpy()
        T = T.detach().numpy()
        ok = T > 0
        for a in range(3):
            ok &= ~(2.0 * math.pi ** 2 * T / (self.deq_d[a] * self.deq_d[a]) < self.deq_crit)
            m1, m2 = self.deq_hi[a] - u[:, a], u[:, a] - self.deq_lo[a]
            ok &= (m1 > 0) & (m2 > 0)
            ok &= ~((m1 * m1 < 2.0 * T * self.deq_crit) | (m2 * m2 < 2.0 * T * self.deq_crit))
        return torch.as_tensor(ok)

    def discrete_maxwell(self, rho, u, T, poly=None, tol=None, max_iterations=None):
        """The discrete Maxwellian E (n, nv) of n states and, with the Shakhov polynomial P (n, nv), the correction
        gamma . psi (n, nv) (deq_* and deq_shakhov_correction, src/kinetic/discrete_equilibrium.hpp:56-188). The
        Newton iteration is the solver's (initial beta, damped step, stopping rule: deq_newton_step :159-180,
        deq_accept, kinetic_kernels.hpp:489-493), so beta is the one the forward solve used."""
        tol = self.deq_tol if tol is None else tol
        max_iterations = self.deq_maxit if max_iterations is None else max_iterations
        c = self.xi[None, :, :] - u[:, None, :]
        psi = torch.cat([torch.ones_like(c[..., :1]), c, 0.5 * (c * c).sum(-1, keepdim=True)], -1)  # (n, nv, 5)
        w = self.w[None, :, None]
        W = torch.stack([rho, torch.zeros_like(rho), torch.zeros_like(rho), torch.zeros_like(rho), 1.5 * rho * T], 1)
        with torch.no_grad():
            p0 = psi.detach()
            Td, rd = T.detach(), rho.detach()
            beta = torch.stack([torch.log(rd / (2.0 * math.pi * Td) ** 1.5), torch.zeros_like(Td),
                                torch.zeros_like(Td), torch.zeros_like(Td), -1.0 / Td], 1)
            Wd = W.detach()
            prev = torch.full_like(Td, 1e300)
            done = torch.zeros(len(Td), dtype=torch.bool)
            for it in range(max_iterations):
                E = torch.exp((p0 * beta[:, None, :]).sum(-1))
                G = (w * E[..., None] * p0).sum(1) - Wd
                su = rd * torch.sqrt(Td)
                rel = torch.maximum(G[:, 0].abs() / rd, torch.maximum(G[:, 1:4].abs().amax(1) / su,
                                                                      G[:, 4].abs() / (rd * Td)))
                last = it + 1 == max_iterations
                accept = ~done & ((rel < tol) | ((rel < 1e-4) & ((rel > 0.5 * prev) | last)))
                done = done | accept
                if bool(done.all()):
                    break
                J = torch.einsum("nq,nqa,nqb->nab", self.w[None, :] * E, p0, p0)
                d = torch.linalg.solve(J, -G)
                scale = torch.ones_like(Td)
                big = d[:, 4].abs() > 0.5 * beta[:, 4].abs()
                scale = torch.where(big, 0.5 * beta[:, 4].abs() / d[:, 4].abs(), scale)
                scale = torch.where(d[:, 0].abs() * scale > 1.0, 1.0 / d[:, 0].abs(), scale)
                step = ~done
                beta = torch.where(step[:, None], beta + scale[:, None] * d, beta)
                prev = torch.where(step, rel, prev)
            if not bool(done.all()):
                raise ScopeError("the discrete-equilibrium Newton iteration did not converge for a state")
            E = torch.exp((p0 * beta[:, None, :]).sum(-1))
            J = torch.einsum("nq,nqa,nqb->nab", self.w[None, :] * E, p0, p0)
        # beta as a function of the state: the value of the accepted iterate, the derivative of the implicit
        # function, dbeta = -J^-1 dG (G - G.detach() is zero in value and carries dG)
        E0 = torch.exp((psi * beta[:, None, :]).sum(-1))
        G = (w * E0[..., None] * psi).sum(1) - W
        beta_g = beta - torch.linalg.solve(J, G - G.detach())
        E = torch.exp((psi * beta_g[:, None, :]).sum(-1))
        if poly is None:
            return E, None
        Jg = torch.einsum("nq,nqa,nqb->nab", self.w[None, :] * E, psi, psi)
        r = (w * (E * poly)[..., None] * psi).sum(1)
        gamma = -torch.linalg.solve(Jg, r)
        return E, (psi * gamma[:, None, :]).sum(-1)

    def equilibrium(self, rho, u, T, poly=None, tol=None):
        """The equilibrium of n states: continuous where the grid resolves the state (or the continuous equilibrium is
        chosen), discrete elsewhere; with poly, the Shakhov factor (1 + P + gamma . psi)."""
        M = self.maxwell(rho, u, T)
        fac = None if poly is None else 1.0 + poly
        if not self.discrete:
            return M if poly is None else M * fac
        res = self.resolved(rho, u, T)
        if bool(res.all()):
            return M if poly is None else M * fac
        idx = torch.nonzero(~res).ravel()
        E, gp = self.discrete_maxwell(rho[idx], u[idx], T[idx], None if poly is None else poly[idx], tol=tol)
        M = M.index_put((idx,), E)
        if poly is None:
            return M
        fac = fac.index_put((idx,), fac[idx] + gp)
        return M * fac

    def maxwell(self, rho, u, T):
        """rho, T: (n,), u: (n, 3) -> (n, nv)."""
        c = self.xi[None, :, :] - u[:, None, :]
        tp = 2.0 * math.pi * T
        return (rho / (tp * torch.sqrt(tp)))[:, None] * torch.exp(-(c * c).sum(-1) / (2.0 * T)[:, None])

    def target(self, f, mu0):
        rho, u, T, p, q = self.moments(f)
        c = self.xi[None, :, :] - u[:, None, :]
        c2 = (c * c).sum(-1)
        coef = torch.where(T < self.cold, torch.zeros_like(T), (1.0 - self.Pr) / (5.0 * (rho * T) * T))
        poly = coef[:, None] * (c * q[:, None, :]).sum(-1) * (c2 / T[:, None] - 5.0)
        fS = self.equilibrium(rho, u, T, poly)
        coll = self.volume * p / (mu0 * T ** self.omega)
        return coll, fS, (rho, u, T, p, q)

    def limited_state(self, mom, fs):
        """W_ib = (p, u, T) of the pressure faces' owners reconstructed at the face (update_pressure_inflow,
        kinetic_solver.cpp:172-260): LSQ gradient over the owner's stencil, whose boundary entries carry the face
        state (rho, u, T) of the last boundary sums where it is positive (periodic entries and the others the owner's
        own value); Venkatakrishnan limiter with the absolute epsilon^2 = K^3 V; the owner's value where the
        reconstruction is not positive. (np, 5)"""
        rho, u, T, p, q = mom
        st = torch.cat([p[:, None], u, T[:, None]], 1)  # (nc, 5): p, u, T
        wi = st[self.p_own]
        fsw = torch.stack([fs[:, 0] * fs[:, 4], fs[:, 1], fs[:, 2], fs[:, 3], fs[:, 4]], 1)[self.p_bface]
        fsd = fs.detach()[self.p_bface]
        use = self.p_bmask & (fsd[..., 0] > 0) & (fsd[..., 4] > 0)
        wiE = wi[:, None, :].expand(-1, self.p_mask.shape[1], -1)
        wk = torch.where(self.p_internal[..., None], st[self.p_other], torch.where(use[..., None], fsw, wiE))
        wk = torch.where(self.p_mask[..., None], wk, wiE)
        grad = torch.einsum("fek,fea->fka", wk - wi[:, None, :], self.p_lsq)  # (np, 5, 3)
        wmax = torch.maximum(wi, wk.amax(1))
        wmin = torch.minimum(wi, wk.amin(1))
        phi = torch.ones_like(wi)
        if self.p_limit:
            proj = torch.einsum("fka,fea->fke", grad, self.p_dx)  # (np, 5, E)
            dmax = (wmax - wi)[..., None]
            dmin = (wmin - wi)[..., None]
            d1 = torch.where(proj > 0, dmax.expand_as(proj), torch.where(proj < 0, dmin.expand_as(proj),
                                                                          torch.zeros_like(proj)))
            e2 = self.p_eps2[:, None, None]
            num = (d1 * d1 + e2) + 2.0 * d1 * proj
            den = d1 * d1 + 2.0 * proj * proj + d1 * proj + e2
            ok = den > 0
            v = torch.clamp(num / torch.where(ok, den, torch.ones_like(den)), 0.0, 1.0)
            v = torch.where(ok, v, torch.zeros_like(v))
            v = torch.where(proj == 0, torch.ones_like(v), v)
            active = (self.p_mask & ~self.p_periodic)[:, None, :]
            v = torch.where(active, v, torch.ones_like(v))
            phi = torch.clamp(v.amin(2), max=1.0)
        wib = wi + phi * torch.einsum("fka,fa->fk", grad, self.p_dxb)
        good = (wib.detach()[:, 0] > 0) & (wib.detach()[:, 4] > 0)
        return torch.where(good[:, None], wib, wi)

    def inflow(self, mom, rho_gamma, Tw, fs=None):
        """(scale (nb,), Maxwellian values (nb, nv)) of every boundary face; walls at rest-frame density 1 with the
        wall velocity and temperature Tw, pressure faces W_b (App. A.2, kinetic_solver.cpp:172-260) from the owner
        cell ("cell" reconstruction) or from its limited reconstruction at the face with the face states fs."""
        rho, u, T, p, q = mom
        nb = self.nb
        own = self.bowner
        # pressure: (p_ib, u_ib, T_ib) = owner state, or its reconstruction at the face
        p_ib, u_ib, T_ib = p[own], u[own], T[own]
        if self.limited:
            wib = self.limited_state(mom, fs)
            pi = self.p_idx
            p_ib = p_ib.index_put((pi,), wib[:, 0])
            u_ib = u_ib.index_put((pi,), wib[:, 1:4])
            T_ib = T_ib.index_put((pi,), wib[:, 4])
        rho_ib = p_ib / T_ib
        cs = torch.sqrt(self.gamma * T_ib)
        T_b = torch.where(self.inlet_face, self.T_patch, T_ib)
        du = (p_ib - self.p_patch) / (rho_ib * cs)
        un = (u_ib * self.bn).sum(1)
        u_p = torch.where(self.zero_tan[:, None], (un + du)[:, None] * self.bn, u_ib + du[:, None] * self.bn)
        rho_p = self.p_patch / T_b
        wall = self.wall
        rho_s = torch.where(wall, torch.ones(nb, dtype=torch.float64), rho_p)
        u_s = torch.where(wall[:, None], self.u_patch, u_p)
        T_s = torch.where(wall, Tw, T_b)
        pres = self.bkind == BC_PRESSURE
        use = wall | pres
        safe_T = torch.where(use, T_s, torch.ones_like(T_s))
        safe_rho = torch.where(use, rho_s, torch.ones_like(rho_s))
        # the inflow states corrected to their discrete Maxwellian (correct_inflow, kinetic_solver.cpp:103-114)
        M = self.equilibrium(safe_rho, u_s, safe_T, tol=1e-10)
        rg = torch.zeros(nb, dtype=torch.float64)
        if len(self.wall_idx):
            rg = rg.index_put((self.wall_idx,), rho_gamma)
        scale = torch.where(wall, rg, torch.where(pres, torch.ones(nb, dtype=torch.float64),
                                                  torch.zeros(nb, dtype=torch.float64)))
        return scale, M

    def _entry_f(self, f, scale, M, alpha):
        """f at the stencil entries (nc, E, nv) and the inflow values of boundary entries (first order: the specular
        part of a wall with alpha < 1 is the cell's own value at the reflected velocity)."""
        fi = f[:, None, :].expand(-1, self.E, -1)
        fo = f[self.other]  # (nc, E, nv)
        b = self.bface
        a = (self.S @ self.xi.T)  # (nc, E, nv)
        infl = scale[b][..., None] * M[b]
        wall_e = (self.kind == BC_DIFFUSE_WALL)[..., None]
        infl = infl + torch.where(wall_e, (1.0 - alpha[b])[..., None] * torch.gather(fi, 2, self.eflip),
                                  torch.zeros_like(infl))
        fm = torch.gather(fi, 2, self.mirror)
        k = self.kind[..., None]
        bval = torch.where(k == BC_PERIODIC, fi,
                           torch.where(k == BC_SYMMETRY, 0.5 * (fi + fm),
                                       torch.where(a >= 0, fi, torch.where(k == BC_VACUUM, torch.zeros_like(fi), infl))))
        fk = torch.where(self.internal[..., None], fo, bval)
        fk = torch.where(self.mask[..., None], fk, fi)
        return fk, a, infl

    def gradient(self, f, fk):
        """limited_gradient (kinetic_kernels.hpp:161-201) at every (cell, velocity): (nc, nv, 3)."""
        fi = f[:, None, :]
        d = torch.where(self.mask[..., None], fk - fi, torch.zeros_like(fk))
        G = torch.einsum("cek,cev->cvk", self.c, d)
        if self.limiter == LIMITER_NONE:
            return G
        fmax = torch.maximum(f, fk.amax(1))
        fmin = torch.minimum(f, fk.amin(1))
        eps2 = self.eps2[:, None].expand(-1, self.nv)
        if self.limiter == LIMITER_REL:
            sc = torch.maximum(fmax.abs(), fmin.abs())
            eps2 = eps2 * sc * sc
        proj = torch.einsum("cvk,cek->cev", G, self.ds)
        dmax = (fmax - f)[:, None, :]
        dmin = (fmin - f)[:, None, :]
        d1 = torch.where(proj > 0, dmax, dmin)
        e2 = eps2[:, None, :]
        num = (d1 * d1 + e2) + 2.0 * d1 * proj
        den = d1 * d1 + 2.0 * proj * proj + d1 * proj + e2
        ok = (proj != 0) & (den > 0)
        v = torch.clamp(num / torch.where(ok, den, torch.ones_like(den)), 0.0, 1.0)
        v = torch.where(proj == 0, torch.ones_like(v), torch.where(den > 0, v, torch.zeros_like(v)))
        active = (self.mask & (self.kind != BC_PERIODIC))[..., None]
        v = torch.where(active, v, torch.ones_like(v))
        phi = torch.clamp(v.amin(1), max=1.0)
        return phi[..., None] * G

    def residual(self, f, g, fk, a, infl, coll, fS, alpha=None, scale=None, M=None):
        """residual_value (kinetic_kernels.hpp:238-278) at every (cell, velocity). The incoming value of a wall is
        rho M + (1 - alpha) f_spec with f_spec the cell's reconstructed face value at the reflected velocity."""
        if alpha is not None:
            b = self.bface
            gi4 = g[:, None, :, :].expand(-1, self.E, -1, -1)
            gr = torch.gather(gi4, 2, self.eflip[..., None].expand(-1, -1, -1, 3))
            fr = torch.gather(f[:, None, :].expand(-1, self.E, -1), 2, self.eflip)
            spec = fr + (gr * self.ds[:, :, None, :]).sum(-1)
            wall_e = (self.kind == BC_DIFFUSE_WALL)[..., None]
            infl = torch.where(wall_e, scale[b][..., None] * M[b] + (1.0 - alpha[b])[..., None] * spec, infl)
        gi = g[:, None, :, :]  # (nc, 1, nv, 3)
        own_face = f[:, None, :] + (gi * self.ds[:, :, None, :]).sum(-1)
        go = g[self.other]  # (nc, E, nv, 3)
        nb_face = f[self.other] + (go * self.dn[:, :, None, :]).sum(-1)
        gm = torch.gather(g[:, None, :, :].expand(-1, self.E, -1, -1), 2,
                          self.mirror[..., None].expand(-1, -1, -1, 3))
        fmr = torch.gather(f[:, None, :].expand(-1, self.E, -1), 2, self.mirror)
        sym_face = fmr + (gm * self.ds[:, :, None, :]).sum(-1)
        k = self.kind[..., None]
        ff = torch.where(a >= 0, own_face,
                         torch.where(self.internal[..., None], nb_face,
                                     torch.where(k == BC_SYMMETRY, sym_face,
                                                 torch.where(k == BC_VACUUM, torch.zeros_like(infl), infl))))
        use = (self.mask & (self.kind != BC_PERIODIC))[..., None]
        R = torch.where(use, a * ff, torch.zeros_like(ff)).sum(1)
        return R - coll[:, None] * (fS - f)

    def boundary_sums(self, f, g, M):
        """sm0 = sum_{an >= 0} w an f_b (reconstructed) and sm5 = sum_{an < 0} w an M_b per face
        (k_boundary_sums, kinetic_cuda_kernels.cu:275-323; the other 18 sums are not needed here), and
        S_spec = sum_{an < 0} w an f_spec (reconstructed at the reflected velocity)."""
        own = self.bowner
        an = self.bn @ self.xi.T  # (nb, nv)
        fb = f[own] + (g[own] * self.bd[:, None, :]).sum(-1)
        out = an >= 0
        sm0 = torch.where(out, self.w * an * fb, torch.zeros_like(fb)).sum(1)
        sm5 = torch.where(out, torch.zeros_like(fb), self.w * an * M).sum(1)
        fr = torch.gather(f[own], 1, self.bflip)
        gr = torch.gather(g[own], 1, self.bflip[..., None].expand(-1, -1, 3))
        spec = fr + (gr * self.bd[:, None, :]).sum(-1)
        sspec = torch.where(out, torch.zeros_like(fb), self.w * an * spec).sum(1)
        return sm0, sm5, sspec

    def face_states(self, f, g, M, sm0, sm5, sspec, alpha):
        """face_state (rho, u, T) of every boundary face from the moment sums of the face distribution
        (k_boundary_sums, kinetic_cuda_kernels.cu:275-323, and process_boundary_sums, kinetic_solver.cpp:280-335):
        the outgoing half the reconstructed face values, the incoming half the mirrored face values (symmetry), the
        inflow Maxwellian (pressure), rho_Gamma times the unit wall Maxwellian (walls; rho_Gamma = -sm0 / sm5 of
        these sums, plus the specular part (1 - alpha) f_spec of a Maxwell wall) or nothing (vacuum). (nb, 5)"""
        own = self.bowner
        an = self.bn @ self.xi.T  # (nb, nv)
        fb = f[own] + (g[own] * self.bd[:, None, :]).sum(-1)
        out = (an >= 0) | (self.bkind == BC_PERIODIC)[:, None]
        psi = torch.cat([torch.ones(self.nv, 1, dtype=torch.float64), self.xi,
                         0.5 * (self.xi * self.xi).sum(-1, keepdim=True)], 1)  # (nv, 5)
        zero = torch.zeros_like(fb)
        smo = torch.where(out, self.w * fb, zero) @ psi
        fin = torch.where((self.bkind == BC_SYMMETRY)[:, None], torch.gather(fb, 1, self.bmirror), M)
        smi = torch.where(out, zero, self.w * fin) @ psi
        wall = self.wall
        rg = torch.where(sm5 < 0, torch.clamp(-(sm0 + (1.0 - alpha) * sspec) / torch.where(sm5 < 0, sm5,
                                                                                            -torch.ones_like(sm5)),
                                               min=0.0), torch.zeros_like(sm5))
        in_scale = torch.where(wall, rg, torch.where(self.bkind == BC_VACUUM, torch.zeros_like(rg),
                                                     torch.ones_like(rg)))
        mom = smo + in_scale[:, None] * smi
        # the specular part of a wall with alpha < 1: (1 - alpha) sum_in w psi f_spec
        fr = torch.gather(f[own], 1, self.bflip)
        gr = torch.gather(g[own], 1, self.bflip[..., None].expand(-1, -1, 3))
        spec = fr + (gr * self.bd[:, None, :]).sum(-1)
        spec_mom = torch.where(out, zero, self.w * spec) @ psi
        mom = mom + torch.where(wall[:, None], (1.0 - alpha)[:, None] * spec_mom, torch.zeros_like(mom))
        pos = mom.detach()[:, 0] > 0
        m0 = torch.where(pos, mom[:, 0], torch.ones_like(mom[:, 0]))
        u = mom[:, 1:4] / m0[:, None]
        T = (2.0 * mom[:, 4] / m0 - (u * u).sum(1)) / 3.0
        fs = torch.cat([mom[:, :1], u, T[:, None]], 1)
        return torch.where(pos[:, None], fs, torch.zeros_like(fs))

    # ---- the map -------------------------------------------------------------------------------------------------
    def evaluate(self, f, aux, mu0, Tw, alpha=None):
        """(R (nc, nv), auxiliary equations (n_aux,), J = M_dot). aux: the auxiliary unknowns (split_aux): rho_Gamma
        of the walls with their zero-net-flux equations rho_Gamma - Phi, and with the limited reconstruction the face
        states with fs - FS(f, fs). alpha (per boundary face, walls only; default 1): the accommodation, with the
        specular part of axis-aligned walls (a Maxwell wall)."""
        if alpha is None:
            alpha = torch.ones(self.nb, dtype=torch.float64)
        rho_gamma, fs = self.split_aux(aux)
        coll, fS, mom = self.target(f, mu0)
        scale, M = self.inflow(mom, rho_gamma, Tw, fs)
        fk, a, infl = self._entry_f(f, scale, M, alpha)
        g = self.gradient(f, fk)
        R = self.residual(f, g, fk, a, infl, coll, fS, alpha, scale, M)
        sm0, sm5, sspec = self.boundary_sums(f, g, M)
        wi = self.wall_idx
        phi = torch.clamp(-(sm0[wi] + (1.0 - alpha[wi]) * sspec[wi]) / sm5[wi], min=0.0)
        Fw = rho_gamma - phi
        if self.limited:
            Fw = torch.cat([Fw, (fs - self.face_states(f, g, M, sm0, sm5, sspec, alpha)).ravel()])
        in_scale = scale  # pressure 1, vacuum 0, walls rho_Gamma
        flow = self.barea * (sm0 + in_scale * sm5)
        mdot_in = -flow[self.inlet_face].sum()
        mdot_out = flow[self.outlet_face].sum()
        J = 0.5 * (mdot_in + mdot_out) * math.sqrt(2.0 / math.pi)
        return R, Fw, J

    def params_of(self, solver=None):
        Tw = self.T_patch.clone()
        return torch.tensor(self.mu0, dtype=torch.float64), Tw


def state_of(solver, limited=None):
    """(f, auxiliary unknowns) of a KineticSolver (internal numbering, storage order): rho_Gamma of the wall faces,
    followed by the face states (nb, 5) of the last boundary sums when the pressure faces use the limited
    reconstruction (limited=None: decided from the solver's set-up)."""
    f = torch.as_tensor(np.asarray(solver.backend.get_distribution(), float))
    wall = np.flatnonzero(solver.bkind == BC_DIFFUSE_WALL)
    aux = [np.asarray(solver.inflow[wall, 0], float)]
    if limited is None:
        limited = solver.h.pressure_boundary_reconstruction != "cell" and bool(np.any(solver.bkind == BC_PRESSURE))
    if limited:
        aux.append(np.asarray(solver.face_state, float).ravel())
    return f, torch.as_tensor(np.concatenate(aux))


def adjoint_gradient(sm: SteadyMap, f, rho_gamma, tol=1e-12, maxiter=4000):
    """dJ/d(mu_hat0), dJ/dT_w and dJ/dalpha (per boundary face; alpha at 1, the derivative from below) at the fixed
    point (f, auxiliary unknowns of state_of: rho_Gamma, and the face states with the limited reconstruction), with
    the adjoint solved by GMRES. Returns (dJ_dmu0, dJ_dTw (nb,), info) with
    info = (J, ||F||, gmres iterations, y, dJ_dalpha (nb,))."""
    from scipy.sparse.linalg import LinearOperator, gmres

    mu0, Tw = sm.params_of()
    f = f.clone().requires_grad_(True)
    rg = rho_gamma.clone().requires_grad_(True)
    mu0 = mu0.clone().requires_grad_(True)
    Tw = Tw.clone().requires_grad_(True)
    alpha = torch.ones(sm.nb, dtype=torch.float64, requires_grad=True)
    R, Fw, J = sm.evaluate(f, rg, mu0, Tw, alpha)
    nf, nw = f.numel(), rg.numel()
    # J depends on alpha explicitly too: the limited gradient of an inlet / outlet owner that also has a wall face
    gJ = torch.autograd.grad(J, (f, rg, mu0, Tw, alpha), allow_unused=True, retain_graph=True)
    gJ = [torch.zeros_like(t) if g is None else g for g, t in zip(gJ, (f, rg, mu0, Tw, alpha))]
    rhs = torch.cat([gJ[0].ravel(), gJ[1].ravel()]).numpy()

    def vjp(y):
        yt = torch.as_tensor(y)
        yR, yW = yt[:nf].view_as(R), yt[nf:]
        gf, gr = torch.autograd.grad((R, Fw), (f, rg), grad_outputs=(yR, yW), retain_graph=True, allow_unused=True)
        gr = torch.zeros_like(rg) if gr is None else gr
        return torch.cat([gf.ravel(), gr.ravel()]).numpy()

    n = nf + nw
    it = [0]

    def cb(_):
        it[0] += 1

    op = LinearOperator((n, n), matvec=vjp, dtype=np.float64)
    y, code = gmres(op, rhs, rtol=tol, atol=0.0, restart=400, maxiter=maxiter, callback=cb, callback_type="pr_norm")
    if code != 0:
        raise RuntimeError(f"adjoint GMRES did not converge (code {code})")
    yt = torch.as_tensor(y)
    gp = torch.autograd.grad((R, Fw), (mu0, Tw, alpha), grad_outputs=(yt[:nf].view_as(R), yt[nf:]),
                             allow_unused=True)
    gp = [torch.zeros_like(t) if g is None else g for g, t in zip(gp, (mu0, Tw, alpha))]
    dmu = float(gJ[2] - gp[0])
    dTw = (gJ[3] - gp[1]).detach().numpy()
    dal = (gJ[4] - gp[2]).detach().numpy()
    fres = float(torch.sqrt((R.detach() ** 2).sum() + (Fw.detach() ** 2).sum()))
    return dmu, dTw, (float(J.detach()), fres, it[0], y, dal)


def transposed_jacobian_product(sm: SteadyMap, f, rho_gamma, y_f, y_w):
    """(dF/dx)^T y at (f, auxiliary unknowns): the adjoint residual operator the B200 kernels compute; y_w in the
    layout of the auxiliary unknowns. Returns (x_f, x_w)."""
    mu0, Tw = sm.params_of()
    f = f.clone().requires_grad_(True)
    rg = rho_gamma.clone().requires_grad_(True)
    R, Fw, J = sm.evaluate(f, rg, mu0, Tw)
    gf, gr = torch.autograd.grad((R, Fw), (f, rg), grad_outputs=(torch.as_tensor(y_f), torch.as_tensor(y_w)),
                                 allow_unused=True)
    return gf.numpy(), (torch.zeros_like(rg) if gr is None else gr).numpy()

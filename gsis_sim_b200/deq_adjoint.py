"""Derivatives through the discrete equilibrium for the adjoint (no reference counterpart).

Where the velocity grid does not resolve a state (deq_resolved, src/kinetic/discrete_equilibrium.hpp:35-48) the
reference replaces the Maxwellian of that state by the discrete one,

    E(xi) = exp(beta . psi(c)),   psi(c) = (1, c_x, c_y, c_z, |c|^2 / 2),   c = xi - u,

with beta solving G(beta; rho, u, T) = sum_q w_q E psi - (rho, 0, 0, 0, 3/2 rho T) = 0 by Newton (deq_*, :56-188).
A cell's Shakhov target becomes f^S = E (1 + P + gamma . psi) with P = coef (c . q)(|c|^2 / T - 5) and gamma solving
Phi = J gamma + sum_q w E P psi = 0, J = sum_q w E psi psi^T (deq_shakhov_correction :183-188). Inflow states are
corrected to E (correct_inflow, src/kinetic/kinetic_solver.cpp:103-114).

For the adjoint, the lambda-weighted derivative of f^S with respect to the cell moments theta = (rho, u, T, q) is

    Lambda = D - Phi_theta^T mu_g - G_theta^T mu_b,   mu_g = J^-1 a_g,   mu_b = J^-1 (a_b - Phi_beta mu_g),

where D = sum lambda df^S/dtheta at fixed (beta, gamma), a_b = sum lambda E (1 + P + gamma . psi) psi and
a_g = sum lambda E psi come from the device (k_adj_cell), and J, Phi_beta = sum w E psi psi^T (gamma . psi + P),
Phi_theta and G_theta are sums of E times polynomials in c over the grid. On a tensor velocity grid every such sum is
a combination of the moments sum_q w E c_x^i c_y^j c_z^k, and E factors per axis, so they come from per-axis sums
X_a[k] = sum_i w_a[i] exp(beta_a c + beta_4 c^2 / 2) c^k (this module, NumPy, vectorised over cells).
"""
from __future__ import annotations

import math
from itertools import product

import numpy as np


class TensorGrid:
    """A velocity set as a tensor grid: per-axis nodes and weights, w(q) = w0 w_x[i] w_y[j] w_z[k]."""

    def __init__(self, nodes, weights, w0):
        self.nodes = [np.asarray(n, float) for n in nodes]
        self.weights = [np.asarray(w, float) for w in weights]
        self.w0 = float(w0)

    @classmethod
    def from_setup(cls, setup):
        xi = [np.asarray(setup[k], float) for k in ("xi_x", "xi_y", "xi_z")]
        w = setup.arrays.get("weights") if hasattr(setup, "arrays") else None
        nv = len(xi[0])
        nodes, idx = [], []
        for a in range(3):
            n, inv = np.unique(xi[a], return_inverse=True)
            nodes.append(n)
            idx.append(inv)
        if len(nodes[0]) * len(nodes[1]) * len(nodes[2]) != nv:
            return None
        flat = (idx[0] * len(nodes[1]) + idx[1]) * len(nodes[2]) + idx[2]
        if len(np.unique(flat)) != nv:
            return None
        if w is None:
            return cls(nodes, [np.ones(len(n)) for n in nodes], float(setup["weight"]))
        w = np.asarray(w, float)
        full = np.zeros(len(nodes[0]) * len(nodes[1]) * len(nodes[2]))
        full[flat] = w
        full = full.reshape(len(nodes[0]), len(nodes[1]), len(nodes[2]))
        w0 = full[0, 0, 0]
        wx, wy, wz = full[:, 0, 0] / w0, full[0, :, 0] / w0, full[0, 0, :] / w0
        if not np.allclose(np.einsum("i,j,k->ijk", wx, wy, wz) * w0, full, rtol=1e-12, atol=0.0):
            return None
        return cls(nodes, [wx, wy, wz], w0)

    def axis_sums(self, beta, u, deg):
        """X (n, 3, deg + 1): X[:, a, k] = sum_i w_a[i] exp(beta_a c + beta_4 c^2 / 2) c^k, c = node_a[i] - u_a."""
        n = len(beta)
        X = np.empty((n, 3, deg + 1))
        for a in range(3):
            c = self.nodes[a][None, :] - u[:, a:a + 1]
            e = self.weights[a][None, :] * np.exp(beta[:, 1 + a:2 + a] * c + 0.5 * beta[:, 4:5] * c * c)
            p = e
            for k in range(deg + 1):
                X[:, a, k] = p.sum(1)
                p = p * c
        return X

    def moments(self, beta, u, deg):
        """m[(i, j, k)] (n,) = sum_q w E c_x^i c_y^j c_z^k for i + j + k <= deg."""
        X = self.axis_sums(beta, u, deg)
        pre = self.w0 * np.exp(beta[:, 0])
        return {(i, j, k): pre * X[:, 0, i] * X[:, 1, j] * X[:, 2, k]
                for i, j, k in product(range(deg + 1), repeat=3) if i + j + k <= deg}


# ---- polynomials in c = (c_x, c_y, c_z) with per-state coefficients: {(i, j, k): coefficient (n,) or scalar} --------

def _padd(a, b, s=1.0):
    out = dict(a)
    for k, v in b.items():
        out[k] = out.get(k, 0.0) + s * v
    return out


def _pmul(a, b):
    out = {}
    for (ka, va), (kb, vb) in product(a.items(), b.items()):
        k = (ka[0] + kb[0], ka[1] + kb[1], ka[2] + kb[2])
        out[k] = out.get(k, 0.0) + va * vb
    return out


def _pscale(a, s):
    return {k: v * s for k, v in a.items()}


def _integrate(p, m):
    out = 0.0
    for k, v in p.items():
        out = out + v * m[k]
    return out


_ONE = {(0, 0, 0): 1.0}
_C = [{(1, 0, 0): 1.0}, {(0, 1, 0): 1.0}, {(0, 0, 1): 1.0}]
_C2 = {(2, 0, 0): 1.0, (0, 2, 0): 1.0, (0, 0, 2): 1.0}
PSI = [_ONE, _C[0], _C[1], _C[2], _pscale(_C2, 0.5)]
# d psi / d u_a = (0, -e_a, -c_a)
DPSI = [[{}, _pscale(_ONE, -1.0) if a == 0 else {}, _pscale(_ONE, -1.0) if a == 1 else {},
         _pscale(_ONE, -1.0) if a == 2 else {}, _pscale(_C[a], -1.0)] for a in range(3)]


def _dot(coeffs, polys):
    out = {}
    for cf, p in zip(coeffs, polys):
        out = _padd(out, _pscale(p, cf))
    return out


# ---- the Newton iteration of the solver, on the tensor grid ---------------------------------------------------------

def newton(grid: TensorGrid, rho, u, T, tol, max_iterations):
    """beta of the discrete Maxwellian of n states, by the solver's iteration (initial beta, damped step, stopping
    rule: deq_newton_step, src/kinetic/discrete_equilibrium.hpp:159-180; deq_accept, kinetic_kernels.hpp:489-493).
    Returns (beta (n, 5), ok (n,))."""
    n = len(rho)
    beta = np.stack([np.log(rho / (2.0 * math.pi * T) ** 1.5), np.zeros(n), np.zeros(n), np.zeros(n), -1.0 / T], 1)
    W = np.stack([rho, np.zeros(n), np.zeros(n), np.zeros(n), 1.5 * rho * T], 1)
    prev = np.full(n, 1e300)
    done = np.zeros(n, bool)
    for it in range(max_iterations):
        m = grid.moments(beta, u, 4)
        G = np.stack([_integrate(p, m) for p in PSI], 1) - W
        su = rho * np.sqrt(T)
        rel = np.maximum(np.abs(G[:, 0]) / rho, np.maximum(np.abs(G[:, 1:4]).max(1) / su, np.abs(G[:, 4]) / (rho * T)))
        last = it + 1 == max_iterations
        done |= (rel < tol) | ((rel < 1e-4) & ((rel > 0.5 * prev) | last))
        if done.all():
            break
        J = jacobian(m)
        d = np.linalg.solve(J, -G[..., None])[..., 0]
        scale = np.ones(n)
        big = np.abs(d[:, 4]) > 0.5 * np.abs(beta[:, 4])
        scale = np.where(big, 0.5 * np.abs(beta[:, 4]) / np.where(big, np.abs(d[:, 4]), 1.0), scale)
        scale = np.where(np.abs(d[:, 0]) * scale > 1.0, 1.0 / np.abs(d[:, 0]), scale)
        step = ~done
        beta = np.where(step[:, None], beta + scale[:, None] * d, beta)
        prev = np.where(step, rel, prev)
    return beta, done


def jacobian(m):
    """J (n, 5, 5) = sum w E psi psi^T from the moments."""
    n = len(next(iter(m.values())))
    J = np.empty((n, 5, 5))
    for a in range(5):
        for b in range(a, 5):
            J[:, a, b] = J[:, b, a] = _integrate(_pmul(PSI[a], PSI[b]), m)
    return J


def g_theta(beta, m, rho, T, n_params):
    """dG/dtheta (n, 5, n_params) for theta = (rho, u_x, u_y, u_z, T[, q_x, q_y, q_z])."""
    n = len(rho)
    out = np.zeros((n, 5, n_params))
    out[:, 0, 0] = -1.0
    out[:, 4, 0] = -1.5 * T
    out[:, 4, 4] = -1.5 * rho
    for a in range(3):
        bdp = _dot([beta[:, 1 + a], beta[:, 4]], [_ONE, _C[a]])  # -(beta . dpsi/du_a)
        for r in range(5):
            p = _padd(_pscale(_pmul(bdp, PSI[r]), -1.0), DPSI[a][r])
            out[:, r, 1 + a] = _integrate(p, m)
    return out


class CellDerivatives:
    """J, Phi_beta, Phi_theta and G_theta of the discrete-equilibrium cells, theta = (rho, u, T, q)."""

    def __init__(self, grid: TensorGrid, moments15, Pr, cold_T, tol, max_iterations):
        mo = np.asarray(moments15, float)
        rho, u, T, q = mo[:, 0], mo[:, 1:4], mo[:, 4], mo[:, 12:15]
        beta, ok = newton(grid, rho, u, T, tol, max_iterations)
        self.ok = ok
        m = grid.moments(beta, u, 7)
        kap = np.where(T < cold_T, 0.0, (1.0 - Pr) / (5.0 * rho * T * T))
        cq = _dot([q[:, 0], q[:, 1], q[:, 2]], _C)
        h = _padd(_pscale(_C2, 1.0 / T), _ONE, -5.0)
        P = _pscale(_pmul(cq, h), kap)
        J = jacobian(m)
        r = np.stack([_integrate(_pmul(P, PSI[a]), m) for a in range(5)], 1)
        gamma = -np.linalg.solve(J, r[..., None])[..., 0]
        gpsi = _dot([gamma[:, k] for k in range(5)], PSI)
        F = _padd(gpsi, P)  # gamma . psi + P
        n = len(rho)
        Phb = np.empty((n, 5, 5))
        for a in range(5):
            for b in range(a, 5):
                Phb[:, a, b] = Phb[:, b, a] = _integrate(_pmul(_pmul(PSI[a], PSI[b]), F), m)
        Pht = np.zeros((n, 5, 8))
        dP_drho = _pscale(P, -1.0 / rho)
        dP_dT = _pscale(_pmul(cq, _padd(_pscale(_C2, -3.0 / (T * T)), _pscale(_ONE, 10.0 / T))), kap)
        for r_ in range(5):
            Pht[:, r_, 0] = _integrate(_pmul(PSI[r_], dP_drho), m)
            Pht[:, r_, 4] = _integrate(_pmul(PSI[r_], dP_dT), m)
            for a in range(3):
                Pht[:, r_, 5 + a] = _integrate(_pmul(PSI[r_], _pscale(_pmul(_C[a], h), kap)), m)
        for a in range(3):
            bdp = _dot([-beta[:, 1 + a], -beta[:, 4]], [_ONE, _C[a]])  # beta . dpsi/du_a
            gdp = _dot([-gamma[:, 1 + a], -gamma[:, 4]], [_ONE, _C[a]])  # gamma . dpsi/du_a
            dPu = _pscale(_padd(_pscale(h, -q[:, a]), _pscale(_pmul(cq, _C[a]), -2.0 / T)), kap)
            for r_ in range(5):
                p = _pmul(_pmul(bdp, PSI[r_]), F)
                p = _padd(p, _pmul(DPSI[a][r_], F))
                p = _padd(p, _pmul(PSI[r_], _padd(gdp, dPu)))
                Pht[:, r_, 1 + a] = _integrate(p, m)
        self.J, self.Phi_beta, self.Phi_theta = J, Phb, Pht
        self.G_theta = g_theta(beta, m, rho, T, 8)
        self.beta, self.gamma = beta, gamma

    def lambda_sums(self, D, a_b, a_g):
        """Lambda (n, 8) from the device sums: D (n, 8) at fixed (beta, gamma), a_b, a_g (n, 5)."""
        mu_g = np.linalg.solve(self.J, a_g[..., None])[..., 0]
        rhs = a_b - np.einsum("nab,nb->na", self.Phi_beta, mu_g)
        mu_b = np.linalg.solve(self.J, rhs[..., None])[..., 0]
        return D - np.einsum("nrt,nr->nt", self.Phi_theta, mu_g) - np.einsum("nrt,nr->nt", self.G_theta, mu_b)


class InflowDerivatives:
    """The correction of inflow states theta_s = (rho, u, T) to their discrete Maxwellian theta' = (rho', u', T')
    (the continuous form with the discrete Maxwellian's parameters): theta_s_bar = (dtheta'/dtheta_s)^T theta'_bar."""

    def __init__(self, grid: TensorGrid, states, tol=1e-10, max_iterations=20):
        st = np.asarray(states, float)
        rho, u, T = st[:, 0], st[:, 1:4], st[:, 4]
        beta, ok = newton(grid, rho, u, T, tol, max_iterations)
        self.ok = ok
        m = grid.moments(beta, u, 4)
        self.J = jacobian(m)
        self.G_theta = g_theta(beta, m, rho, T, 5)
        self.beta = beta
        b, b4 = beta[:, 1:4], beta[:, 4]
        Tp = -1.0 / b4
        rho_p = np.exp(beta[:, 0] - (b * b).sum(1) / (2.0 * b4)) * (2.0 * math.pi * Tp) ** 1.5
        n = len(rho)
        dth = np.zeros((n, 5, 5))  # d theta' / d beta, theta' = (rho', u'_x, u'_y, u'_z, T')
        dth[:, 0, 0] = rho_p
        dth[:, 0, 1:4] = rho_p[:, None] * (-b / b4[:, None])
        dth[:, 0, 4] = rho_p * ((b * b).sum(1) / (2.0 * b4 * b4) - 1.5 / b4)
        for a in range(3):
            dth[:, 1 + a, 1 + a] = -1.0 / b4
            dth[:, 1 + a, 4] = b[:, a] / (b4 * b4)
        dth[:, 4, 4] = 1.0 / (b4 * b4)
        self.dtheta_dbeta = dth
        self.corrected = np.stack([rho_p, u[:, 0] - b[:, 0] / b4, u[:, 1] - b[:, 1] / b4, u[:, 2] - b[:, 2] / b4, Tp], 1)

    def pullback(self, theta_bar):
        """theta_s_bar (n, 5) from theta'_bar (n, 5) = (rho', u', T') adjoints."""
        beta_bar = np.einsum("nrb,nr->nb", self.dtheta_dbeta, theta_bar)
        mu = np.linalg.solve(self.J, beta_bar[..., None])[..., 0]
        out = -np.einsum("nrt,nr->nt", self.G_theta, mu)
        out[:, 1:4] += theta_bar[:, 1:4]  # u' = u_s + d at fixed beta
        return out

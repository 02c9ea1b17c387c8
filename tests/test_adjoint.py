"""Discrete adjoint of the converged CIS fixed point (CPU part).

* The reference adjoint (oracle/adjoint_ref.py: the steady map in torch, transposed by autograd) is pinned against
  finite differences of the converged CPU-oracle forward solver: dM_dot/d mu_hat0 and dM_dot/dT_w (central) and
  dM_dot/d alpha at alpha = 1 (one-sided from below, through Maxwell-wall solves).
* The host algebra of gsis_sim_b200/adjoint.py (moments -> Shakhov target -> collision term chain, pressure-face
  chain, index maps) against torch autograd of the same forward formulas.
The device kernels are checked against the reference adjoint in tests/test_gpu_adjoint.py."""
import math

import numpy as np
import pytest
import torch

from gsis_sim_b200 import adjoint as adj
from gsis_sim_b200 import kinetic_setup as ks
from gsis_sim_b200.mesh import box_mesh
from gsis_sim_b200.solver import KineticSolver


def channel_case(mu_scale=1.0, Tw=1.0, n=(5, 3, 1), nv=(10, 10, 10), side="periodic_slab", limiter="venkatakrishnan",
                 eps="relative", half=False, quarter=False, alpha=1.0, equilibrium="continuous", precision="fp64",
                 reconstruction="cell"):
    """Pressure-driven channel (inlet p 1, outlet p 0.5, diffuse walls) in the adjoint's scope; `half`: symmetry
    plane at y = 0 instead of the lower wall; `quarter`: a duct quarter, symmetry planes at y = 0 and z = 0, walls at
    y = 1 and z = 0.7 (a flow that varies in y and z)."""
    lower = "sym" if (half or quarter) else "wall"
    sides = ("symz", "wall") if quarter else ("side", "side")
    hz = 0.7 if quarter else 1.0 / 3  # quarter: not square, so no y <-> z mirror symmetry (no limiter ties)
    m = box_mesh(n, (0, 0, 0), (2.0, 1.0, hz), ("inlet", "outlet", lower, "wall", *sides))
    bcs = [ks.BC("inlet", "pressure_inlet", T=1.0, p=1.0), ks.BC("outlet", "pressure_outlet", p=0.5),
           ks.BC("wall", "diffuse_wall", T=Tw, alpha=alpha)]
    if not quarter:
        bcs.append(ks.BC("side", side))
    if half or quarter:
        bcs.append(ks.BC("sym", "symmetry"))
    if quarter:
        bcs.append(ks.BC("symz", "symmetry"))
    kp = ks.KineticParams(precision=precision, pressure_boundary_reconstruction=reconstruction, limiter=limiter,
                          limiter_eps=eps, sweep_blocks=1, equilibrium=equilibrium)
    setup, host = ks.build_kinetic_setup(m, ks.Gas(omega=0.81), ks.Conditions(L_ref=1.0, T0=273.15, Kn=0.3), bcs,
                                         ks.VelocityGrid(n=nv), kp)
    if mu_scale != 1.0:
        setup["mu0"] = setup["mu0"] * mu_scale
    return setup, host


def converge(backend, setup, host, tol=1e-13, iters=3000):
    sol = KineticSolver(setup, host, backend)
    sol.initialize_uniform(0.75, (0.0, 0.0, 0.0), 1.0)
    r = 1.0
    for _ in range(iters):
        r = sol.sweep().residual
        if r < tol:
            break
    assert r < 1e-12
    return sol


def _oracle_solution(**kw):
    from oracle.kinetic_oracle import OracleBackend

    setup, host = channel_case(**kw)
    return converge(OracleBackend(setup), setup, host), setup, host


@pytest.mark.timeout(600)
@pytest.mark.parametrize("equilibrium,reconstruction", [("continuous", "cell"), ("discrete", "cell"),
                                                        ("discrete", "limited")])
def test_reference_adjoint_matches_finite_differences(equilibrium, reconstruction):
    """discrete: the reference default; on this 10^3 grid the Newton solve of the discrete Maxwellian is active in
    every cell and for every wall and pressure-face inflow state. limited: the reference's default pressure-boundary
    reconstruction (W_b reconstructed at the face from the owner's stencil, with the face states of the boundary sums
    as auxiliary unknowns)."""
    from oracle import adjoint_ref as ar

    eq = dict(equilibrium=equilibrium, reconstruction=reconstruction)
    sol, setup, host = _oracle_solution(**eq)
    if equilibrium == "discrete":
        assert sol.backend.deq_counts()[0] == sol.nc
    sm = ar.SteadyMap(setup, host)
    assert sm.limited == (reconstruction == "limited")
    sm.check_scope(sol)
    f, rg = ar.state_of(sol)
    assert rg.numel() == sm.n_aux
    mu0, Tw = sm.params_of()
    R, Fw, J = sm.evaluate(f, rg, mu0, Tw)
    # the torch map is the fixed point the oracle converged to
    assert float(R.abs().max()) < 1e-13 and float(Fw.abs().max()) < 1e-12
    assert abs(float(J) - sol.mass_flow()[2]) < 1e-14
    dmu, dTw, info = ar.adjoint_gradient(sm, f, rg)
    h = 1e-5
    Jp = _oracle_solution(mu_scale=1 + h, **eq)[0].mass_flow()[2]
    Jm = _oracle_solution(mu_scale=1 - h, **eq)[0].mass_flow()[2]
    fd_mu = (Jp - Jm) / (2 * h * sm.mu0)
    assert abs(dmu - fd_mu) <= 1e-6 * abs(fd_mu)
    Jp = _oracle_solution(Tw=1 + h, **eq)[0].mass_flow()[2]
    Jm = _oracle_solution(Tw=1 - h, **eq)[0].mass_flow()[2]
    fd_T = (Jp - Jm) / (2 * h)
    assert abs(dTw.sum() - fd_T) <= 1e-6 * abs(fd_T)
    assert np.all(dTw[sm.bkind.numpy() != ar.BC_DIFFUSE_WALL] == 0.0)
    # accommodation at alpha = 1, from below (alpha <= 1): second-order one-sided difference of Maxwell-wall solves
    ha = 1e-4
    J1 = _oracle_solution(alpha=1 - ha, **eq)[0].mass_flow()[2]
    J2 = _oracle_solution(alpha=1 - 2 * ha, **eq)[0].mass_flow()[2]
    fd_a = (3 * sol.mass_flow()[2] - 4 * J1 + J2) / (2 * ha)
    dal = info[4]
    assert abs(dal.sum() - fd_a) <= 1e-6 * abs(fd_a)


def _maxwellian_f(rng, nc, xi, w):
    rho = 0.5 + rng.random(nc)
    u = 0.3 * rng.standard_normal((nc, 3))
    T = 0.8 + 0.4 * rng.random(nc)
    c = xi[None] - u[:, None]
    f = rho[:, None] / (2 * np.pi * T[:, None]) ** 1.5 * np.exp(-(c * c).sum(-1) / (2 * T[:, None]))
    return f * (1 + 0.1 * rng.standard_normal(f.shape) * np.exp(-0.1 * (c * c).sum(-1)))


def _moments(f, xi, w):
    rho = f @ w
    u = (f * w) @ xi / rho[:, None]
    c = xi[None] - u[:, None]
    c2 = (c * c).sum(-1)
    p = (f * w * c2).sum(1) / 3
    P = np.einsum("nq,nqa,nqb->nab", f * w, c, c)
    q = 0.5 * np.einsum("nq,nqa->na", f * w * c2, c)
    m = np.zeros((len(f), 15))
    m[:, 0], m[:, 1:4], m[:, 4], m[:, 5] = rho, u, p / rho, p
    m[:, 6], m[:, 7], m[:, 8] = P[:, 0, 0] - p, P[:, 1, 1] - p, P[:, 2, 2] - p
    m[:, 9], m[:, 10], m[:, 11] = P[:, 0, 1], P[:, 1, 2], P[:, 0, 2]
    m[:, 12:15] = q
    return m


def test_collision_chain_matches_autograd():
    """lambda^T d[-coll (f^S(f) - f)]/df through the k_adj_cell sums, collision_moment_adjoint and the moment
    expansion equals torch autograd of the same forward formulas."""
    rng = np.random.default_rng(7)
    g = np.linspace(-4.5, 4.5, 8)
    xi = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    w = np.full(len(xi), (g[1] - g[0]) ** 3)
    nc = 5
    f = _maxwellian_f(rng, nc, xi, w)
    lam = rng.standard_normal(f.shape)
    vol, mu0, omega, Pr = 0.3 + rng.random(nc), 0.07, 0.81, 2.0 / 3.0
    # forward in torch
    ft = torch.tensor(f, requires_grad=True)
    xt, wt = torch.tensor(xi), torch.tensor(w)
    rho = ft @ wt
    u = (ft * wt) @ xt / rho[:, None]
    c = xt[None] - u[:, None]
    c2 = (c * c).sum(-1)
    p = (ft * wt * c2).sum(1) / 3
    T = p / rho
    q = 0.5 * ((ft * wt * c2)[..., None] * c).sum(1)
    kap = (1 - Pr) / (5 * rho * T * T)
    M = rho[:, None] / (2 * np.pi * T[:, None]) ** 1.5 * torch.exp(-c2 / (2 * T[:, None]))
    fS = M * (1 + kap[:, None] * (c * q[:, None]).sum(-1) * (c2 / T[:, None] - 5))
    coll = torch.tensor(vol) * p / (mu0 * T ** omega)
    R = -coll[:, None] * (fS - ft)
    (g_ref,) = torch.autograd.grad(R, ft, grad_outputs=torch.tensor(lam))
    # the same through the adjoint pieces (k_adj_cell sums restated in numpy)
    m = _moments(f, xi, w)
    rho_n, u_n, T_n = m[:, 0], m[:, 1:4], m[:, 4]
    q_n = m[:, 12:15]
    cc = xi[None] - u_n[:, None]
    c2n = (cc * cc).sum(-1)
    kn = (1 - Pr) / (5 * rho_n * T_n * T_n)
    Mn = rho_n[:, None] / (2 * np.pi * T_n[:, None]) ** 1.5 * np.exp(-c2n / (2 * T_n[:, None]))
    cq = (cc * q_n[:, None]).sum(-1)
    h = c2n / T_n[:, None] - 5
    P = kn[:, None] * cq * h
    lm = lam * Mn
    Tt, kk = T_n[:, None], kn[:, None]
    sums = np.zeros((nc, 9))
    sums[:, 0] = (lam * (Mn * (1 + P) - f)).sum(1)
    sums[:, 1] = (lm / rho_n[:, None]).sum(1)
    for a in range(3):
        sums[:, 2 + a] = (lm * (cc[..., a] / Tt * (1 + P) + kk * (-q_n[:, a:a + 1] * h - 2 * cq * cc[..., a] / Tt))).sum(1)
        sums[:, 6 + a] = (lm * kk * cc[..., a] * h).sum(1)
    sums[:, 5] = (lm * ((c2n / (2 * Tt * Tt) - 1.5 / Tt) * (1 + P) + cq * (-2 * kk / Tt * h - kk * c2n / (Tt * Tt)))).sum(1)
    rb, ub, Tb, qb, colln = adj.collision_moment_adjoint(m, vol, mu0, omega, sums)
    coef = adj.moment_expansion_coefficients(m, rb, ub, Tb, qb)
    fb = colln[:, None] * lam + w * (coef[:, 0:1] + (cc * coef[:, None, 1:4]).sum(-1) + coef[:, 4:5] * c2n +
                                    (cc * coef[:, None, 5:8]).sum(-1) * c2n)
    assert np.max(np.abs(fb - g_ref.numpy())) <= 1e-11 * np.max(np.abs(g_ref.numpy()))


def test_pressure_face_adjoint_matches_autograd():
    rng = np.random.default_rng(3)
    n_f = 6
    p_o = torch.tensor(0.5 + rng.random(n_f), requires_grad=True)
    u_o = torch.tensor(0.2 * rng.standard_normal((n_f, 3)), requires_grad=True)
    T_o = torch.tensor(0.8 + 0.4 * rng.random(n_f), requires_grad=True)
    nrm = rng.standard_normal((n_f, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    p_pat = 0.3 + rng.random(n_f)
    T_pat = 0.9 + 0.2 * rng.random(n_f)
    inlet = np.array([True, False, True, False, True, False])
    zt = np.array([False, False, True, True, False, True])
    gamma = 5.0 / 3.0
    nt = torch.tensor(nrm)
    rho_ib = p_o / T_o
    du = (p_o - torch.tensor(p_pat)) / (rho_ib * torch.sqrt(gamma * T_o))
    un = (u_o * nt).sum(1)
    u_b = torch.where(torch.tensor(zt)[:, None], (un + du)[:, None] * nt, u_o + du[:, None] * nt)
    T_b = torch.where(torch.tensor(inlet), torch.tensor(T_pat), T_o)
    rho_b = torch.tensor(p_pat) / T_b
    rbar, ubar, Tbar = rng.standard_normal(n_f), rng.standard_normal((n_f, 3)), rng.standard_normal(n_f)
    L = (rho_b * torch.tensor(rbar)).sum() + (u_b * torch.tensor(ubar)).sum() + (T_b * torch.tensor(Tbar)).sum()
    gp, gu, gT = torch.autograd.grad(L, (p_o, u_o, T_o))
    pb, ub, Tb = adj.pressure_face_adjoint(p_o.detach().numpy(), u_o.detach().numpy(), T_o.detach().numpy(), nrm,
                                           p_pat, inlet, zt, gamma, rbar, ubar, Tbar)
    assert np.allclose(pb, gp.numpy(), rtol=1e-12, atol=1e-14)
    assert np.allclose(ub, gu.numpy(), rtol=1e-12, atol=1e-14)
    assert np.allclose(Tb, gT.numpy(), rtol=1e-12, atol=1e-14)


@pytest.mark.timeout(600)
def test_limited_pressure_reconstruction_matches_autograd():
    """PressureReconstruction (the "limited" W_b of update_pressure_inflow) equals the reference adjoint's torch form
    in value at the oracle's converged state of the half channel (limiter active on some pressure faces), and its
    vector-Jacobian product equals torch autograd with respect to the cell states and the face states."""
    from oracle import adjoint_ref as ar

    sol, setup, host = _oracle_solution(half=True, reconstruction="limited", equilibrium="discrete")
    r = adj.PressureReconstruction(sol)
    wib = r.forward(sol.moments_, sol.face_state)
    assert np.any(r.estar >= 0) and np.all(r.good)
    sm = ar.SteadyMap(setup, host)
    m = sol.moments_
    p = torch.tensor(m[:, 5], requires_grad=True)
    u = torch.tensor(m[:, 1:4], requires_grad=True)
    T = torch.tensor(m[:, 4], requires_grad=True)
    fs = torch.tensor(sol.face_state, requires_grad=True)
    wt = sm.limited_state((torch.tensor(m[:, 0]), u, T, p, None), fs)
    assert np.max(np.abs(wt.detach().numpy() - wib)) <= 1e-14 * np.max(np.abs(wib))
    wb = np.random.default_rng(3).standard_normal(wib.shape)
    gp, gu, gT, gfs = torch.autograd.grad(wt, (p, u, T, fs), grad_outputs=torch.as_tensor(wb))
    cell_bar, fs_bar = r.vjp(wb)
    ref_cell = np.column_stack([gp.numpy(), gu.numpy(), gT.numpy()])
    assert np.max(np.abs(cell_bar - ref_cell)) <= 1e-12 * np.max(np.abs(ref_cell))
    assert np.max(np.abs(fs_bar - gfs.numpy())) <= 1e-12 * np.max(np.abs(gfs.numpy()))
    assert np.max(np.abs(fs_bar)) > 0


def test_face_state_and_inflow_derivatives():
    """face_moment_state_adjoint against torch autograd of (rho, u, T) of the face moments; inflow_moment_derivatives
    against central differences of the incoming-half sums of the Maxwellian."""
    rng = np.random.default_rng(5)
    mom = np.column_stack([0.5 + rng.random(6), 0.2 * rng.standard_normal((6, 3)), 2.0 + rng.random(6)])
    mom[2, 0] = -1.0  # no face state
    kap = rng.standard_normal((6, 5))
    mt = torch.tensor(mom, requires_grad=True)
    m0 = mt[:, 0]
    ut = mt[:, 1:4] / m0[:, None]
    Tt = (2.0 * mt[:, 4] / m0 - (ut * ut).sum(1)) / 3.0
    fs = torch.cat([m0[:, None], ut, Tt[:, None]], 1)
    (g,) = torch.autograd.grad(fs, mt, grad_outputs=torch.as_tensor(kap))
    ref = g.numpy()
    ref[2] = 0.0
    out = adj.face_moment_state_adjoint(mom, kap)
    assert np.max(np.abs(out - ref)) <= 1e-13 * np.max(np.abs(ref))
    gr = np.linspace(-4.5, 4.5, 10)
    xi = np.stack(np.meshgrid(gr, gr, gr, indexing="ij"), -1).reshape(-1, 3)
    w = np.full(len(xi), (gr[1] - gr[0]) ** 3)
    nrm = np.array([[1.0, 0.0, 0.0], [0.0, -0.6, 0.8]])
    st = np.array([[1.0, 0.1, -0.2, 0.05, 1.1], [0.8, 0.0, 0.3, -0.1, 0.9]])
    D, d5 = adj.inflow_moment_derivatives(xi, w, nrm, st)
    psi = np.column_stack([np.ones(len(xi)), xi, 0.5 * np.sum(xi * xi, 1)])

    def sums(n, s):
        an = xi @ n
        c = xi - s[1:4]
        M = w * s[0] / (2 * np.pi * s[4]) ** 1.5 * np.exp(-np.sum(c * c, 1) / (2 * s[4]))
        m = an < 0
        return np.concatenate([psi[m].T @ M[m], [an[m] @ M[m]]])

    h = 1e-6
    for i in range(2):
        for j in range(5):
            e = np.zeros(5)
            e[j] = h
            fd = (sums(nrm[i], st[i] + e) - sums(nrm[i], st[i] - e)) / (2 * h)
            assert np.max(np.abs(fd[:5] - D[i, :, j])) <= 1e-7 * max(np.max(np.abs(D[i])), 1.0)
            assert abs(fd[5] - d5[i, j]) <= 1e-7 * max(np.max(np.abs(d5[i])), 1.0)


def test_index_maps():
    setup, host = channel_case()
    xi = np.stack([setup["xi_x"], setup["xi_y"], setup["xi_z"]], 1)
    rev = adj.reversed_velocities(xi)
    assert np.array_equal(xi[rev], -xi) and np.array_equal(rev[rev], np.arange(len(xi)))
    re = adj.reverse_entries(setup["csr_offsets"], setup["csr_other"], host.csr_faces)
    offs, other = np.asarray(setup["csr_offsets"]), np.asarray(setup["csr_other"])
    row = np.repeat(np.arange(len(offs) - 1), np.diff(offs))
    internal = other >= 0
    assert np.all(re[~internal] == -1)
    e = np.flatnonzero(internal)
    assert np.array_equal(row[re[e]], other[e]) and np.array_equal(other[re[e]], row[e])
    assert np.array_equal(re[re[e]], e)
    with pytest.raises(adj.AdjointScopeError):
        adj.reversed_velocities(xi + 0.1)


@pytest.mark.timeout(600)
@pytest.mark.parametrize("reconstruction", ["cell", "limited"])
def test_reversed_velocity_sweeps_solve_the_adjoint(reconstruction):
    """The iteration scheme of gsis_sim_b200.adjoint on the CPU: the exact operator O(y) of the reference adjoint,
    the wall adjoint (and, with the limited pressure reconstruction, the face-state adjoint) recomputed from the
    current lambda, and the forward LU-SGS block passes (the oracle's) run on velocity-reversed storage as the
    transposed preconditioner. It converges, and to the GMRES adjoint's gradients."""
    from oracle import adjoint_ref as ar
    from oracle.kinetic_oracle import OracleBackend

    sol, setup, host = _oracle_solution(reconstruction=reconstruction)
    sm = ar.SteadyMap(setup, host)
    f, rg = ar.state_of(sol)
    mu0, Tw = sm.params_of()
    ft, rt = f.clone().requires_grad_(True), rg.clone().requires_grad_(True)
    mut = mu0.clone().requires_grad_(True)
    R, Fw, J = sm.evaluate(ft, rt, mut, Tw)
    gJ = torch.autograd.grad(J, (ft, rt), retain_graph=True)
    Jf, Jw = gJ[0].numpy(), gJ[1].numpy()

    def op(lam, nu):
        gf, gr = torch.autograd.grad((R, Fw), (ft, rt), grad_outputs=(torch.as_tensor(lam), torch.as_tensor(nu)),
                                     retain_graph=True)
        return gf.numpy() - Jf, gr.numpy() - Jw

    xi = np.stack([setup["xi_x"], setup["xi_y"], setup["xi_z"]], 1)
    rev = adj.reversed_velocities(xi)
    pre = OracleBackend(setup)  # its f holds lambda at the reversed positions; cell parameters of the forward state
    pre.set_distribution(np.zeros((sol.nc, sol.nv)))
    pre.set_moments(sol.moments_)
    pre.update_cell_params()
    lam, nu = np.zeros((sol.nc, sol.nv)), np.zeros(len(rg))
    r0 = None
    for _ in range(400):
        nu = nu - op(lam, nu)[1]
        Of, _ = op(lam, nu)
        r = np.linalg.norm(Of)
        r0 = r0 or r
        if r < 1e-11 * r0:
            break
        pre.passes_given(Of[:, rev])
        lam = pre.get_distribution()[:, rev]
    assert r < 1e-11 * r0
    (gmu,) = torch.autograd.grad((R, Fw), (mut,), grad_outputs=(torch.as_tensor(lam), torch.as_tensor(nu)))
    dmu_ref, _, _ = ar.adjoint_gradient(sm, f, rg)
    assert abs(-float(gmu) - dmu_ref) <= 1e-8 * abs(dmu_ref)


def _wall_field_solution(T_faces):
    """The channel on the CPU oracle with a per-face wall temperature field (internal boundary-face numbering)."""
    from oracle.kinetic_oracle import OracleBackend

    setup, host = channel_case()
    sol = KineticSolver(setup, host, OracleBackend(setup))
    sol.set_wall_temperature(T_faces)
    sol.initialize_uniform(0.75, (0.0, 0.0, 0.0), 1.0)
    r = 1.0
    for _ in range(3000):
        r = sol.sweep().residual
        if r < 1e-13:
            break
    assert r < 1e-12
    return sol


@pytest.mark.timeout(600)
def test_wall_temperature_field_matches_reference_adjoint():
    """KineticSolver.set_wall_temperature on the CPU oracle: the patch values leave the inflow table unchanged, and
    the central difference of M_dot along a random per-face wall-temperature direction equals the reference
    adjoint's per-face dM_dot/dT_w projected on that direction."""
    from oracle import adjoint_ref as ar

    sol, setup, host = _oracle_solution()
    before = sol.inflow.copy()
    T_patch = host.patch_dbl[np.asarray(setup["bface_patch"]), 0]
    sol.set_wall_temperature(T_patch)
    assert np.array_equal(sol.inflow, before)
    sm = ar.SteadyMap(setup, host)
    f, rg = ar.state_of(sol)
    _, dTw, _ = ar.adjoint_gradient(sm, f, rg)
    walls = np.flatnonzero(sol.bkind == ar.BC_DIFFUSE_WALL)
    rng = np.random.default_rng(2026)
    v = np.zeros(sol.nb)
    v[walls] = rng.standard_normal(len(walls))
    v /= np.linalg.norm(v)
    h = 1e-5
    Jp = _wall_field_solution(T_patch + h * v).mass_flow()[2]
    Jm = _wall_field_solution(T_patch - h * v).mass_flow()[2]
    fd = (Jp - Jm) / (2 * h)
    assert abs(float(dTw @ v) - fd) <= 1e-6 * abs(fd)


class _ClosedFormProblem:
    """Stand-in for MassFlowProblem with a closed-form M_dot(delta, T, alpha) and its exact gradients."""

    def __init__(self, n):
        self.n = n
        self.solves = self.adjoints = self.released = 0

    @staticmethod
    def J(d, T, a):
        return d * d * np.sum(T ** 1.5) + np.sum(np.sin(T) * a) + math.log(d)

    def solve(self, d, T, a):
        T = np.linspace(0.9, 1.1, self.n) if T is None else T
        a = np.ones(self.n) if a is None else a
        self.solves += 1
        return (d, T.copy(), a.copy()), self.J(d, T, a)

    def gradients(self, state, d):
        self.adjoints += 1
        _, T, a = state
        return 2 * d * np.sum(T ** 1.5) + 1 / d, 1.5 * d * d * np.sqrt(T) + np.cos(T) * a, np.sin(T)

    def release(self, state):
        self.released += 1


def test_mass_flow_function_chain_rule():
    """mass_flow, the torch.autograd.Function over a forward solve and one adjoint solve, on a closed-form stand-in:
    gradcheck of all three inputs, the upstream gradient scales the result, one adjoint solve per forward even
    through repeated backward passes, and inputs given as None get no gradient."""
    prob = _ClosedFormProblem(4)
    d = torch.tensor(0.7, dtype=torch.float64, requires_grad=True)
    T = torch.tensor([1.0, 1.2, 0.8, 1.1], dtype=torch.float64, requires_grad=True)
    a = torch.tensor([0.5, 0.9, 1.3, 1.0], dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda d, T, a: adj.mass_flow(prob, d, T, a), (d, T, a))
    prob.solves = prob.adjoints = prob.released = 0
    J = adj.mass_flow(prob, d, T, a)
    assert abs(float(J.detach()) - prob.J(0.7, T.detach().numpy(), a.detach().numpy())) < 1e-15
    gd, gT, ga = torch.autograd.grad(3.0 * J, (d, T, a), retain_graph=True)
    rd, rT, ra = _ClosedFormProblem(4).gradients((0.7, T.detach().numpy(), a.detach().numpy()), 0.7)
    assert abs(float(gd) - 3 * rd) < 1e-12 and np.allclose(gT.numpy(), 3 * rT, rtol=1e-14, atol=0)
    assert np.allclose(ga.numpy(), 3 * ra, rtol=1e-14, atol=0)
    torch.autograd.grad(J, (d,))
    assert (prob.solves, prob.adjoints, prob.released) == (1, 1, 1)
    J2 = adj.mass_flow(prob, d)
    (g2,) = torch.autograd.grad(J2, (d,))
    T0 = np.linspace(0.9, 1.1, 4)
    assert abs(float(g2) - (2 * 0.7 * np.sum(T0 ** 1.5) + 1 / 0.7)) < 1e-12

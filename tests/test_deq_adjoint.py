"""The discrete equilibrium's derivative chain of the adjoint (gsis_sim_b200.deq_adjoint) against torch autograd.

For random cell states on a 10^3 tensor grid, where the Newton solve of the discrete Maxwellian is active:
* CellDerivatives.lambda_sums, fed with the lambda sums the device computes at fixed (beta, gamma), equals the
  lambda-weighted derivative of the Shakhov target E (1 + P + gamma . psi) with respect to (rho, u, T, q) taken by
  autograd through one implicit Newton step and the gamma solve;
* InflowDerivatives reproduces the corrected state (rho', u', T') of a Newton solve and pulls adjoints of it back to
  the uncorrected inflow state as autograd does;
* the Newton replica stops at the same iterate as the solver's discrete_maxwell (the corrected states agree)."""
import math

import numpy as np
import torch

from gsis_sim_b200 import deq_adjoint as da
from gsis_sim_b200 import kinetic_setup as ks
from gsis_sim_b200.mesh import box_mesh


def _setup():
    m = box_mesh((2, 1, 1), (0, 0, 0), (1, 1, 1), ("a", "b", "w", "w", "w", "w"))
    bcs = [ks.BC("a", "pressure_inlet", T=1.0, p=1.0), ks.BC("b", "pressure_outlet", p=0.5),
           ks.BC("w", "diffuse_wall", T=1.0)]
    return ks.build_kinetic_setup(m, ks.Gas(omega=0.81), ks.Conditions(L_ref=1.0, T0=273.15, Kn=0.3), bcs,
                                  ks.VelocityGrid(n=(10, 10, 10)), ks.KineticParams(precision="fp64"))[0]


def _states(n, seed):
    rng = np.random.default_rng(seed)
    return (0.5 + rng.random(n), 0.3 * rng.standard_normal((n, 3)), 0.7 + 0.5 * rng.random(n),
            0.05 * rng.standard_normal((n, 3)), rng)


def test_cell_chain_matches_autograd():
    setup = _setup()
    grid = da.TensorGrid.from_setup(setup)
    assert grid is not None
    xi = torch.stack([torch.as_tensor(np.asarray(setup[k], float)) for k in ("xi_x", "xi_y", "xi_z")], 1)
    w, Pr = float(setup["weight"]), float(setup["Pr"])
    rho, u, T, q, rng = _states(6, 3)
    n = len(rho)
    mo = np.zeros((n, 15))
    mo[:, 0], mo[:, 1:4], mo[:, 4], mo[:, 12:15] = rho, u, T, q
    cd = da.CellDerivatives(grid, mo, Pr, 0.0, float(setup["deq_tolerance"]), int(setup["deq_max_iterations"]))
    assert cd.ok.all()
    th = torch.tensor(np.concatenate([rho[:, None], u, T[:, None], q], 1), requires_grad=True)
    r, uu, TT, qq = th[:, 0], th[:, 1:4], th[:, 4], th[:, 5:8]
    c = xi[None] - uu[:, None]
    c2 = (c * c).sum(-1)
    psi = torch.cat([torch.ones_like(c[..., :1]), c, 0.5 * c2[..., None]], -1)
    beta = torch.as_tensor(cd.beta)
    W = torch.stack([r, 0 * r, 0 * r, 0 * r, 1.5 * r * TT], 1)
    G = (w * torch.exp((psi * beta[:, None, :]).sum(-1))[..., None] * psi).sum(1) - W
    bg = beta - torch.linalg.solve(torch.as_tensor(cd.J), G - G.detach())
    E = torch.exp((psi * bg[:, None, :]).sum(-1))
    P = ((1 - Pr) / (5 * r * TT * TT))[:, None] * (c * qq[:, None, :]).sum(-1) * (c2 / TT[:, None] - 5)
    Jg = torch.einsum("nq,nqa,nqb->nab", w * E, psi, psi)
    gam = -torch.linalg.solve(Jg, (w * (E * P)[..., None] * psi).sum(1))
    fS = E * (1 + P + (psi * gam[:, None, :]).sum(-1))
    lam = torch.as_tensor(rng.standard_normal((n, xi.shape[0])))
    (g,) = torch.autograd.grad((lam * fS).sum(), th)
    # the device's sums at fixed (beta, gamma) (k_adj_cell, discrete branch)
    E, P, psi, gam, L = (t.detach().numpy() for t in (E, P, psi, gam, lam))
    c = xi.numpy()[None] - u[:, None]
    c2 = (c * c).sum(-1)
    kap = (1 - Pr) / (5 * rho * T * T)
    cq = (c * q[:, None, :]).sum(-1)
    h = c2 / T[:, None] - 5
    F = 1 + P + (psi * gam[:, None, :]).sum(-1)
    D = np.zeros((n, 8))
    D[:, 0] = (L * E * (-P / rho[:, None])).sum(1)
    for a in range(3):
        dE = -E * (cd.beta[:, 1 + a, None] + cd.beta[:, 4, None] * c[..., a])
        dF = kap[:, None] * (-q[:, a, None] * h - 2 * cq * c[..., a] / T[:, None]) - (gam[:, 1 + a, None] +
                                                                                     gam[:, 4, None] * c[..., a])
        D[:, 1 + a] = (L * (dE * F + E * dF)).sum(1)
        D[:, 5 + a] = (L * E * kap[:, None] * c[..., a] * h).sum(1)
    D[:, 4] = (L * E * cq * (-2 * kap[:, None] * h / T[:, None] - kap[:, None] * c2 / T[:, None] ** 2)).sum(1)
    lam_sums = cd.lambda_sums(D, np.einsum("nq,nqk->nk", L * E * F, psi), np.einsum("nq,nqk->nk", L * E, psi))
    assert np.max(np.abs(lam_sums - g.numpy())) <= 1e-12 * np.max(np.abs(g.numpy()))


def test_inflow_chain_matches_autograd_and_the_solver_correction():
    setup = _setup()
    grid = da.TensorGrid.from_setup(setup)
    xi = torch.stack([torch.as_tensor(np.asarray(setup[k], float)) for k in ("xi_x", "xi_y", "xi_z")], 1)
    w = float(setup["weight"])
    rho, u, T, _, rng = _states(5, 7)
    st = np.column_stack([rho, u, T])
    idv = da.InflowDerivatives(grid, st)
    assert idv.ok.all()
    ths = torch.tensor(st, requires_grad=True)
    r, uu, TT = ths[:, 0], ths[:, 1:4], ths[:, 4]
    c = xi[None] - uu[:, None]
    psi = torch.cat([torch.ones_like(c[..., :1]), c, 0.5 * (c * c).sum(-1, keepdim=True)], -1)
    beta = torch.as_tensor(idv.beta)
    W = torch.stack([r, 0 * r, 0 * r, 0 * r, 1.5 * r * TT], 1)
    G = (w * torch.exp((psi * beta[:, None, :]).sum(-1))[..., None] * psi).sum(1) - W
    bg = beta - torch.linalg.solve(torch.as_tensor(idv.J), G - G.detach())
    b, b4 = bg[:, 1:4], bg[:, 4]
    Tp = -1 / b4
    rp = torch.exp(bg[:, 0] - (b * b).sum(1) / (2 * b4)) * (2 * math.pi * Tp) ** 1.5
    out = torch.stack([rp, uu[:, 0] - b[:, 0] / b4, uu[:, 1] - b[:, 1] / b4, uu[:, 2] - b[:, 2] / b4, Tp], 1)
    tb = torch.as_tensor(rng.standard_normal((len(rho), 5)))
    (g,) = torch.autograd.grad((out * tb).sum(), ths)
    assert np.max(np.abs(out.detach().numpy() - idv.corrected)) <= 1e-14
    assert np.max(np.abs(idv.pullback(tb.numpy()) - g.numpy())) <= 1e-12 * np.max(np.abs(g.numpy()))
    # the same corrected states as the solver's discrete_maxwell (the C oracle's Newton, tolerance 1e-10)
    from oracle.kinetic_oracle import OracleBackend

    corr, res = OracleBackend(setup).discrete_maxwell(st, 1e-10)
    assert (res > 0).all()
    assert np.max(np.abs(corr - idv.corrected) / np.maximum(np.abs(corr), 1.0)) <= 1e-13

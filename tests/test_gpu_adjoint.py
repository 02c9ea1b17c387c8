"""Discrete adjoint on the B200 (csrc/kin_adjoint.cu + gsis_sim_b200/adjoint.py) against the reference adjoint of
oracle/adjoint_ref.py (the steady map transposed by torch autograd, itself pinned against finite differences in
tests/test_adjoint.py), at the fixed point the B200 forward solver converged to:
* the operator y^T dF/dx (and the objective term dJ/dx) for random adjoint states, to 1e-10, with the continuous
  and with the discrete equilibrium (the Newton solve active in every cell and inflow state), and with the "cell"
  and the "limited" pressure-boundary reconstruction (the reference default: W_b reconstructed at the face from the
  owner's stencil and the face states of the boundary sums);
* the converged adjoint's dM_dot/d mu_hat0, dM_dot/dT_w and dM_dot/d alpha (at alpha = 1), to 1e-8 against the
  reference adjoint and to 1e-5 against finite differences of the B200 forward solver (alpha: one-sided, through
  Maxwell-wall solves)."""
import numpy as np
import pytest
import torch

from tests.test_adjoint import channel_case, converge

pytestmark = pytest.mark.gpu


def _gpu_solution(**kw):
    from gsis_sim_b200.backend import B200Backend

    setup, host = channel_case(**kw)
    be = B200Backend(setup)
    return converge(be, setup, host), setup, host


# States with exact ties in the limiter's stencil extrema are left out of the operator comparison: a channel between
# two symmetry planes z = const does not vary in z and is mirror-symmetric in xi_z to the last bit, so neighbour and
# symmetry-face values equal the cell's own. There the max / min has no derivative, the kernels take the first
# extremum (the cell's own value) and autograd splits the seed; both agree on every mirror-symmetric direction, which
# the gradient test covers (side="symmetry").
@pytest.mark.parametrize("kw", [dict(), dict(half=True), dict(limiter="none"), dict(eps="absolute"),
                                dict(n=(5, 3, 3), quarter=True), dict(n=(5, 3, 3), quarter=True, limiter="none"),
                                dict(equilibrium="discrete"), dict(n=(5, 3, 3), quarter=True, equilibrium="discrete"),
                                dict(half=True, equilibrium="discrete", reconstruction="limited"),
                                dict(n=(5, 3, 3), quarter=True, reconstruction="limited")])
def test_gpu_adjoint_operator_matches_reference(kw):
    """With the limited pressure reconstruction the auxiliary adjoint also carries the face states' kappa (5 per
    boundary face; random on the faces a pressure face reads, zero on the others, whose face states nothing reads)."""
    from gsis_sim_b200.adjoint import KineticAdjoint
    from oracle import adjoint_ref as ar

    assert torch.cuda.is_available()
    sol, setup, host = _gpu_solution(**kw)
    try:
        ka = KineticAdjoint(sol)
        sm = ar.SteadyMap(setup, host)
        f, rg = ar.state_of(sol)
        assert len(rg) == sm.n_aux and ka.limited == sm.limited
        rng = np.random.default_rng(11)
        lam = rng.standard_normal((sol.nc, sol.nv))
        nu = rng.standard_normal(sm.n_aux)
        if ka.limited:
            kap = np.zeros((sol.nb, 5))
            kap[ka.fs_read] = nu[len(ka.wall):].reshape(sol.nb, 5)[ka.fs_read]
            nu[len(ka.wall):] = kap.ravel()
            assert len(ka.fs_read) > 0
        op_f, op_w = ka.operator(lam, nu, with_objective=False)
        ref_f, ref_w = ar.transposed_jacobian_product(sm, f, rg, lam, nu)
        scale = np.max(np.abs(ref_f))
        assert np.max(np.abs(op_f - ref_f)) <= 1e-10 * scale
        assert np.max(np.abs(op_w - ref_w)) <= 1e-10 * max(np.max(np.abs(ref_w)), 1e-300)
        # the objective term: O(y) - y^T dF/dx = -dJ/dx
        mu0, Tw = sm.params_of()
        ft = f.clone().requires_grad_(True)
        rt = rg.clone().requires_grad_(True)
        _, _, J = sm.evaluate(ft, rt, mu0, Tw)
        gJ = torch.autograd.grad(J, (ft, rt), allow_unused=True)
        gJf = gJ[0].numpy()
        gJw = np.zeros(len(nu)) if gJ[1] is None else gJ[1].numpy()
        opJ_f, opJ_w = ka.operator(lam, nu, with_objective=True)
        assert np.max(np.abs((opJ_f - op_f) + gJf)) <= 1e-10 * max(np.max(np.abs(gJf)), scale)
        assert np.max(np.abs((opJ_w - op_w) + gJw)) <= 1e-10 * max(np.max(np.abs(ref_w)), 1e-300)
        ka.close()
    finally:
        sol.backend.close()


def test_gpu_adjoint_operator_on_tube_mesh():
    """The operator on a small O-grid tube + reservoir (curved walls, reservoir back walls, near-vacuum outlet,
    4 LU-SGS blocks): y^T dF/dx equals the reference's for random y. The O-grid is mirror-symmetric in y and z and
    symmetric under y <-> z, so on a cubic velocity grid the converged state has exact limiter ties at velocities with
    |xi_y| = |xi_z| (two neighbours with the same value); 12 x 12 x 10 velocities have no such velocity, and the
    CPU oracle's converged state on this grid has no tie in any stencil extremum or limiter minimum."""
    from gsis_sim_b200 import kinetic_setup as ks
    from gsis_sim_b200 import tube
    from gsis_sim_b200.adjoint import KineticAdjoint
    from gsis_sim_b200.backend import B200Backend
    from oracle import adjoint_ref as ar

    setup, host = tube.tube_case(delta=10.0, grid=ks.VelocityGrid(n=(12, 12, 10)), precision="fp64",
                                 equilibrium="continuous",
                                 pressure_boundary_reconstruction="cell", sweep_blocks=4,
                                 mesh_kw=dict(n_x=6, n_c=2, n_r=2, n_o=2, n_xr=3))
    be = B200Backend(setup)
    try:
        sol = converge(be, setup, host)
        ka = KineticAdjoint(sol)
        sm = ar.SteadyMap(setup, host)
        f, rg = ar.state_of(sol)
        rng = np.random.default_rng(5)
        lam = rng.standard_normal((sol.nc, sol.nv))
        nu = rng.standard_normal(len(ka.wall))
        op_f, op_w = ka.operator(lam, nu, with_objective=False)
        ref_f, ref_w = ar.transposed_jacobian_product(sm, f, rg, lam, nu)
        assert np.max(np.abs(op_f - ref_f)) <= 1e-10 * np.max(np.abs(ref_f))
        assert np.max(np.abs(op_w - ref_w)) <= 1e-10 * np.max(np.abs(ref_w))
        res = ka.solve(tol=1e-8, max_iterations=2000)
        assert res.residual < 1e-7
        ka.close()
    finally:
        be.close()


@pytest.mark.timeout(900)
@pytest.mark.parametrize("kw", [dict(), dict(side="symmetry"), dict(equilibrium="discrete"),
                                dict(half=True, equilibrium="discrete", reconstruction="limited")])
def test_gpu_adjoint_gradients_match_reference_and_finite_differences(kw):
    from gsis_sim_b200.adjoint import KineticAdjoint
    from oracle import adjoint_ref as ar

    sol, setup, host = _gpu_solution(**kw)
    try:
        ka = KineticAdjoint(sol)
        res = ka.solve(tol=1e-12, max_iterations=4000)
        assert res.residual < 1e-10
        sm = ar.SteadyMap(setup, host)
        f, rg = ar.state_of(sol)
        dmu, dTw, info = ar.adjoint_gradient(sm, f, rg)
        assert abs(res.dJ_dmu0 - dmu) <= 1e-8 * abs(dmu)
        assert np.max(np.abs(res.dJ_dTw - dTw)) <= 1e-8 * np.max(np.abs(dTw))
        walls = np.flatnonzero(sol.bkind == 0)
        assert np.max(np.abs(res.dJ_dalpha[walls] - info[4][walls])) <= 1e-8 * np.max(np.abs(info[4]))
        ka.close()
    finally:
        sol.backend.close()
    h = 1e-5
    Jp = _gpu_solution(mu_scale=1 + h, **kw)
    Jm = _gpu_solution(mu_scale=1 - h, **kw)
    fd_mu = (Jp[0].mass_flow()[2] - Jm[0].mass_flow()[2]) / (2 * h * float(setup["mu0"]))
    for s in (Jp, Jm):
        s[0].backend.close()
    assert abs(res.dJ_dmu0 - fd_mu) <= 1e-5 * abs(fd_mu)
    Tp = _gpu_solution(Tw=1 + h, **kw)
    Tm = _gpu_solution(Tw=1 - h, **kw)
    fd_T = (Tp[0].mass_flow()[2] - Tm[0].mass_flow()[2]) / (2 * h)
    for s in (Tp, Tm):
        s[0].backend.close()
    assert abs(res.dJ_dTw.sum() - fd_T) <= 1e-5 * abs(fd_T)
    # accommodation at alpha = 1 from below: Maxwell-wall solves on the B200
    ha = 1e-4
    A1 = _gpu_solution(alpha=1 - ha, **kw)
    A2 = _gpu_solution(alpha=1 - 2 * ha, **kw)
    J0 = res.J
    fd_a = (3 * J0 - 4 * A1[0].mass_flow()[2] + A2[0].mass_flow()[2]) / (2 * ha)
    for s in (A1, A2):
        s[0].backend.close()
    assert abs(np.nansum(res.dJ_dalpha) - fd_a) <= 1e-5 * abs(fd_a)


@pytest.mark.timeout(900)
def test_gpu_mass_flow_autograd_matches_reference_and_finite_differences():
    """mass_flow through torch.autograd on the B200 (MassFlowProblem: converged CIS solve forward, discrete adjoint in
    the backward): the delta, per-face T_w and per-face alpha gradients equal the reference adjoint's at the same
    fixed point to 1e-8, and the T_w gradient projected on a random per-face direction equals a central difference
    of two forward solves with that wall-temperature field to 1e-5."""
    from gsis_sim_b200.adjoint import MassFlowProblem, mass_flow
    from oracle import adjoint_ref as ar

    setup, host = channel_case()
    prob = MassFlowProblem(setup, host, tol=1e-13, adjoint_tol=1e-12, initial=(0.75, (0.0, 0.0, 0.0), 1.0))
    delta = torch.tensor(prob.delta0, dtype=torch.float64, requires_grad=True)
    T = torch.tensor(prob.T_patch, dtype=torch.float64, requires_grad=True)
    alpha = torch.ones(len(prob.wall_faces), dtype=torch.float64, requires_grad=True)
    J = mass_flow(prob, delta, T, alpha)
    gd, gT, ga = torch.autograd.grad(J, (delta, T, alpha))
    sol, J0 = prob.solve(prob.delta0)
    try:
        assert abs(J0 - float(J.detach())) <= 1e-12 * abs(J0)
        sm = ar.SteadyMap(setup, host)
        f, rg = ar.state_of(sol)
        dmu, dTw, info = ar.adjoint_gradient(sm, f, rg)
    finally:
        prob.release(sol)
    ref_d = -dmu * float(setup["mu0"]) / prob.delta0
    assert abs(float(gd) - ref_d) <= 1e-8 * abs(ref_d)
    w = prob.wall_faces
    assert np.max(np.abs(gT.numpy() - dTw[w])) <= 1e-8 * np.max(np.abs(dTw))
    assert np.max(np.abs(ga.numpy() - info[4][w])) <= 1e-8 * np.max(np.abs(info[4]))
    rng = np.random.default_rng(2026)
    v = rng.standard_normal(len(w))
    v /= np.linalg.norm(v)
    h = 1e-5
    Js = []
    for sgn in (1.0, -1.0):
        s, Jv = prob.solve(prob.delta0, prob.T_patch + sgn * h * v)
        prob.release(s)
        Js.append(Jv)
    fd = (Js[0] - Js[1]) / (2 * h)
    assert abs(float(gT.numpy() @ v) - fd) <= 1e-5 * abs(fd)

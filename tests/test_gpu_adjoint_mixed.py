"""The discrete adjoint on a mixed-precision handle (f of the converged mixed solve, lambda and the transport seeds
stored in FP32, FP32 transposed block passes, the operator O(y) in FP64 arithmetic; csrc/kin_adjoint.cu with S =
float):
* the operator y^T dF/dx for random y (rounded to FP32, the storage of lambda) at the mixed solver's own state
  equals the reference adjoint's (oracle/adjoint_ref.py, FP64 torch) at that state to 2e-6 of its largest entry (the
  FP32 storage of the seeds and of O_f), with the continuous and with the discrete equilibrium;
* the converged mixed adjoint's dM_dot/d mu_hat0, dM_dot/dT_w per wall face and dM_dot/d alpha equal the FP64 B200
  adjoint's at the FP64 fixed point to 1e-4, and its T_w gradient projected on seeded random per-face directions
  equals central differences of two FP64 forward solves to 1e-4."""
import numpy as np
import pytest
import torch

from tests.test_adjoint import channel_case

pytestmark = pytest.mark.gpu

MIXED_FLOOR = 3e-7  # residual floor of the mixed forward solve (FP32 storage of f)


def _solution(precision, tol, **kw):
    from gsis_sim_b200.backend import B200Backend
    from gsis_sim_b200.solver import KineticSolver

    setup, host = channel_case(precision=precision, **kw)
    be = B200Backend(setup)
    sol = KineticSolver(setup, host, be)
    sol.initialize_uniform(0.75, (0.0, 0.0, 0.0), 1.0)
    r = 1.0
    for _ in range(4000):
        r = sol.sweep().residual
        if r < tol:
            break
    assert r < 10 * tol, r
    return sol, setup, host


@pytest.mark.parametrize("kw", [dict(), dict(equilibrium="discrete"), dict(n=(5, 3, 3), quarter=True),
                                dict(half=True, equilibrium="discrete", reconstruction="limited")])
def test_gpu_mixed_adjoint_operator_matches_reference(kw):
    """With the limited pressure reconstruction the auxiliary adjoint also carries the face states' kappa (random on
    the faces a pressure face reads)."""
    from gsis_sim_b200.adjoint import KineticAdjoint
    from oracle import adjoint_ref as ar

    assert torch.cuda.is_available()
    sol, setup, host = _solution("mixed", MIXED_FLOOR, **kw)
    try:
        ka = KineticAdjoint(sol)
        sm = ar.SteadyMap(setup, host)
        f, rg = ar.state_of(sol)
        rng = np.random.default_rng(17)
        lam = rng.standard_normal((sol.nc, sol.nv)).astype(np.float32).astype(np.float64)
        nu = rng.standard_normal(sm.n_aux)
        if ka.limited:
            kap = np.zeros((sol.nb, 5))
            kap[ka.fs_read] = nu[len(ka.wall):].reshape(sol.nb, 5)[ka.fs_read]
            nu[len(ka.wall):] = kap.ravel()
        op_f, op_w = ka.operator(lam, nu, with_objective=False)
        ref_f, ref_w = ar.transposed_jacobian_product(sm, f, rg, lam, nu)
        err_f = np.max(np.abs(op_f - ref_f)) / np.max(np.abs(ref_f))
        err_w = np.max(np.abs(op_w - ref_w)) / max(np.max(np.abs(ref_w)), 1e-300)
        print(f"mixed operator {kw}: O_f {err_f:.2e}, O_nu {err_w:.2e}")
        assert err_f <= 2e-6 and err_w <= 2e-6
        ka.close()
    finally:
        sol.backend.close()


@pytest.mark.timeout(900)
@pytest.mark.parametrize("kw", [dict(), dict(equilibrium="discrete")])
def test_gpu_mixed_adjoint_gradients_match_fp64(kw):
    from gsis_sim_b200.adjoint import KineticAdjoint, MassFlowProblem

    sol64, setup64, host64 = _solution("fp64", 1e-13, **kw)
    try:
        ka = KineticAdjoint(sol64)
        r64 = ka.solve(tol=1e-12, max_iterations=4000)
        ka.close()
    finally:
        sol64.backend.close()
    solmx, _, _ = _solution("mixed", MIXED_FLOOR, **kw)
    try:
        ka = KineticAdjoint(solmx)
        rmx = ka.solve(tol=1e-6, max_iterations=4000)
        ka.close()
    finally:
        solmx.backend.close()
    assert rmx.residual < 1e-5, rmx.residual
    e_mu = abs(rmx.dJ_dmu0 - r64.dJ_dmu0) / abs(r64.dJ_dmu0)
    e_T = np.max(np.abs(rmx.dJ_dTw - r64.dJ_dTw)) / np.max(np.abs(r64.dJ_dTw))
    walls = np.flatnonzero(np.isfinite(r64.dJ_dalpha) & (r64.dJ_dalpha != 0))
    e_a = np.max(np.abs(rmx.dJ_dalpha[walls] - r64.dJ_dalpha[walls])) / np.max(np.abs(r64.dJ_dalpha[walls]))
    print(f"mixed vs FP64 adjoint {kw}: mu0 {e_mu:.2e}, T_w {e_T:.2e}, alpha {e_a:.2e}, "
          f"{rmx.iterations} vs {r64.iterations} outer iterations, residual {rmx.residual:.2e}")
    assert e_mu <= 1e-4 and e_T <= 1e-4 and e_a <= 1e-4
    # directional differences of the FP64 forward solver along seeded random per-face temperature directions
    prob = MassFlowProblem(setup64, host64, tol=1e-13, initial=(0.75, (0.0, 0.0, 0.0), 1.0))
    w = prob.wall_faces
    rng = np.random.default_rng(2027)
    h = 1e-5
    for _ in range(2):
        v = rng.standard_normal(len(w))
        v /= np.linalg.norm(v)
        Js = []
        for sgn in (1.0, -1.0):
            s, Jv = prob.solve(prob.delta0, prob.T_patch + sgn * h * v)
            prob.release(s)
            Js.append(Jv)
        fd = (Js[0] - Js[1]) / (2 * h)
        g = float(rmx.dJ_dTw[w] @ v)
        print(f"direction: adjoint {g:.10e}, FP64 difference {fd:.10e}, relative {abs(g - fd) / abs(fd):.2e}")
        assert abs(g - fd) <= 1e-4 * abs(fd)


@pytest.mark.timeout(900)
def test_gpu_mixed_mass_flow_autograd_with_fp64_polish():
    """mass_flow through torch.autograd on a mixed-precision problem: the forward stops at the mixed solve's storage
    floor, the backward polishes that state with FP64 iterations (MassFlowProblem.polish_state) and runs the mixed
    adjoint; the delta and per-face T_w gradients equal the FP64 adjoint's at the FP64 fixed point to 1e-4."""
    from gsis_sim_b200.adjoint import KineticAdjoint, MassFlowProblem, mass_flow

    sol64, setup64, host64 = _solution("fp64", 1e-13)
    try:
        ka = KineticAdjoint(sol64)
        r64 = ka.solve(tol=1e-12, max_iterations=4000)
        ka.close()
    finally:
        sol64.backend.close()
    setup, host = channel_case(precision="mixed")
    prob = MassFlowProblem(setup, host, tol=1e-12, adjoint_tol=1e-8, initial=(0.75, (0.0, 0.0, 0.0), 1.0),
                           stall_iterations=40, polish_iterations=20)
    delta = torch.tensor(prob.delta0, dtype=torch.float64, requires_grad=True)
    T = torch.tensor(prob.T_patch, dtype=torch.float64, requires_grad=True)
    J = mass_flow(prob, delta, T)
    gd, gT = torch.autograd.grad(J, (delta, T))
    assert prob.last_polish is not None and len(prob.last_polish) == 20
    ref_d = r64.dJ_ddelta(float(setup64["mu0"]), prob.delta0)
    w = prob.wall_faces
    e_d = abs(float(gd) - ref_d) / abs(ref_d)
    e_T = np.max(np.abs(gT.numpy() - r64.dJ_dTw[w])) / np.max(np.abs(r64.dJ_dTw[w]))
    print(f"mixed autograd with polish: delta {e_d:.2e}, T_w {e_T:.2e}, polish residuals "
          f"{prob.last_polish[0]:.2e} -> {prob.last_polish[-1]:.2e}")
    assert e_d <= 1e-4 and e_T <= 1e-4

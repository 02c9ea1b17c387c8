"""The host loop (gsis_sim_b200.solver.KineticSolver) reproduces the reference KineticSolver.

Driven here by the CPU oracle backend; the same host loop drives the B200 backend in tests/test_gpu_solver.py.
Golden values: the reference KineticSolver (src/kinetic/kinetic_solver.cpp) after a few CIS iterations
(tests/golden/make_golden.py)."""
import numpy as np
import pytest

from tests import common
from gsis_sim_b200.kinetic_setup import HostSetup
from gsis_sim_b200.section import SectionSpec
from gsis_sim_b200.solver import KineticSolver


def run_solver(backend, setup, z):
    host = HostSetup.from_npz(z)
    sol = KineticSolver(setup, host, backend)
    init = z["solver.init"]
    sol.initialize_uniform(init[0], init[1:4], init[4])
    infos = []
    for _ in range(len(z["solver.infos"])):
        i = sol.sweep()
        infos.append([i.iteration, i.epsilon, i.residual, i.total_mass, i.mass_scale])
    return sol, np.array(infos)


def check_solver(sol, infos, z, tol):
    ref = z["solver.infos"]
    # residual history (the reference compares it at 100x the field tolerance) and total mass
    assert common.max_rel(infos[:, 2], ref[:, 6]) < 100 * tol
    assert common.max_rel(infos[:, 3], ref[:, 8]) < tol
    assert common.max_rel(infos[:, 1], ref[:, 1]) < 1e3 * tol + 1e-12
    assert common.max_rel(sol.moments(), z["solver.moments"]) < 10 * tol
    fp, fm, fs = sol.boundary_fluxes()
    assert common.max_rel(fp, z["solver.F_plus"]) < 10 * tol
    assert common.max_rel(fm, z["solver.F_minus"]) < 10 * tol
    assert common.max_rel(sol.prepare().patch_mass_flow, z["solver.patch_mass_flow"]) < 100 * tol
    assert common.max_rel(sol.distribution(), z["solver.f"]) < tol
    # section mass flows (KineticSolver::section_mass_flow); the empty cuts (x = 0 before every cell centre,
    # x = 3 behind them) must give exactly 0
    for ax, key in ((0, "x"), (1, "y")):
        spec = SectionSpec(ax, list(z[f"solver.section_{key}"]))
        flows = sol.section_mass_flow(spec)
        assert common.max_rel(flows, z[f"solver.section_flow_{key}"]) < 100 * tol
        for c, q in zip(sol.section_cuts(spec), flows):
            if len(c.faces) == 0:
                assert q == 0.0 and c.face_position == c.position


@pytest.mark.parametrize("name", common.golden_names())
def test_host_loop_matches_reference_solver(name):
    from oracle.kinetic_oracle import OracleBackend

    z, setup = common.load(name)
    prec = common.precision_of(setup)
    sol, infos = run_solver(OracleBackend(setup), setup, z)
    check_solver(sol, infos, z, common.TOL[prec])

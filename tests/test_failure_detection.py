"""Failure detection of the host loop, with the faults injected on the host (no GPU is faulted): a distribution whose
moments give a non-positive or non-finite density or temperature stops the iteration with an error naming the cell
(KineticSolver::prepare, src/kinetic/kinetic_solver.cpp:371-386); non-positive initial or GSIS states are rejected
before they reach the backend. The C oracle stands in for the device."""
import numpy as np
import pytest

from gsis_sim_b200 import kinetic_setup as ks
from gsis_sim_b200.mesh import box_mesh
from gsis_sim_b200.solver import KineticSolver, KineticSolverError


def _solver():
    from oracle.kinetic_oracle import OracleBackend

    mesh = box_mesh((3, 1, 1), (0.0, 0.0, 0.0), (1.0, 1 / 3, 1 / 3), ("inlet", "outlet", "wall", "wall", "wall", "wall"))
    bcs = [ks.BC("inlet", "pressure_inlet"), ks.BC("outlet", "vacuum"), ks.BC("wall", "diffuse_wall")]
    setup, host = ks.build_kinetic_setup(mesh, ks.Gas(omega=0.81), ks.Conditions(Kn=0.5), bcs,
                                         ks.VelocityGrid(n=(6, 6, 6)), ks.KineticParams(precision="fp64"))
    return KineticSolver(setup, host, OracleBackend(setup))


@pytest.mark.parametrize("fault", ["negative", "nan"])
def test_bad_moments_stop_the_iteration_and_name_the_cell(fault):
    s = _solver()
    s.initialize_uniform(1.0, (0.0, 0.0, 0.0), 1.0)
    f = s.distribution()
    f[1] = -f[1] if fault == "negative" else np.nan
    s.set_distribution(f)
    with pytest.raises(KineticSolverError, match="original cell 1"):
        s.sweep()


def test_non_positive_states_are_rejected():
    s = _solver()
    with pytest.raises(KineticSolverError):
        s.initialize_uniform(0.0, (0.0, 0.0, 0.0), 1.0)
    with pytest.raises(KineticSolverError):
        s.initialize_uniform(1.0, (0.0, 0.0, 0.0), -1.0)
    w = np.tile([1.0, 0.0, 0.0, 0.0, 1.0], (3, 1))
    bad = w.copy()
    bad[2, 4] = 0.0
    with pytest.raises(KineticSolverError):
        s.initialize_equilibrium(bad)
    s.initialize_equilibrium(w)
    s.sweep()
    with pytest.raises(KineticSolverError):
        s.apply_gsis_correction(w, bad)
    # the rejected calls left the state usable
    assert np.isfinite(s.sweep().residual)

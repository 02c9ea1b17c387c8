"""Nonuniform (sinh-clustered) velocity grid with per-velocity quadrature weights, an extension of the reference's
uniform grids: three CIS iterations of a pressure-driven channel with symmetry sides, B200 backend against the CPU
oracle on the same set-up (FP64 and mixed precision)."""
import numpy as np
import pytest

from tests import common

pytestmark = pytest.mark.gpu


def _case(precision):
    from gsis_sim_b200 import kinetic_setup as ks
    from gsis_sim_b200.mesh import box_mesh

    mesh = box_mesh((6, 4, 2), (0.0, 0.0, 0.0), (3.0, 1.0, 0.5), ("inlet", "outlet", "wall", "wall", "sym", "sym"))
    bcs = [ks.BC("inlet", "pressure_inlet", T=1.0, p=1.0), ks.BC("outlet", "pressure_outlet", p=0.5),
           ks.BC("wall", "diffuse_wall", T=1.0), ks.BC("sym", "symmetry")]
    grid = ks.VelocityGrid.clustered((12, 12, 8), 6.0, 2.0)
    return ks.build_kinetic_setup(mesh, ks.Gas(omega=0.81), ks.Conditions(L_ref=1.0, T0=273.15, delta_rp=5.0), bcs,
                                  grid, ks.KineticParams(precision=precision))


def _run(backend, setup, host, iters=3):
    from gsis_sim_b200.solver import KineticSolver

    sol = KineticSolver(setup, host, backend)
    sol.initialize_uniform(1.0, (0.0, 0.0, 0.0), 1.0)
    res = [sol.sweep().residual for _ in range(iters)]
    return sol.moments(), np.array(res), sol.mass_flow()[2]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 2e-5)])
def test_clustered_grid_gpu_matches_oracle(precision, tol):
    import torch

    if not torch.cuda.is_available():
        pytest.fail("no CUDA device")
    from gsis_sim_b200.backend import B200Backend
    from oracle.kinetic_oracle import OracleBackend

    setup, host = _case(precision)
    assert setup["weights"] is not None  # per-velocity weights reach the device
    with B200Backend(setup) as be:
        g = _run(be, setup, host)
    o = _run(OracleBackend(setup, precision=precision), setup, host)
    assert common.max_rel(g[0], o[0]) < tol
    assert common.max_rel(g[1], o[1]) < tol
    assert abs(g[2] - o[2]) <= tol * abs(o[2]) and g[2] > 0

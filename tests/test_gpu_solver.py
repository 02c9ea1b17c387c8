"""The host loop on the B200 backend reproduces the reference KineticSolver (golden histories)."""
import pytest

from tests import common
from tests.test_solver_host import check_solver, run_solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", common.golden_names())
def test_gpu_host_loop_matches_reference_solver(name):
    import torch

    assert torch.cuda.is_available()
    from gsis_sim_b200.backend import B200Backend

    z, setup = common.load(name)
    prec = common.precision_of(setup)
    with B200Backend(setup) as be:
        sol, infos = run_solver(be, setup, z)
        check_solver(sol, infos, z, common.TOL[prec])

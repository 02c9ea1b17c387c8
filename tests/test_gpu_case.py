"""A case given as files (TOML + .pmesh, tests/golden/case_channel) run on the B200 backend through the host loop,
against the CPU oracle on the same set-up: three CIS iterations of a pressure-driven channel."""
import os

import numpy as np
import pytest

from tests import common

pytestmark = pytest.mark.gpu
CHANNEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "case_channel", "channel.toml")


def _run(backend, setup, host, iters=3):
    from gsis_sim_b200.solver import KineticSolver

    sol = KineticSolver(setup, host, backend)
    sol.initialize_uniform(1.0, (0.0, 0.0, 0.0), 1.0)
    res = [sol.sweep().residual for _ in range(iters)]
    return sol.moments(), np.array(res), sol.mass_flow()


def test_channel_case_files_gpu_matches_oracle():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("no CUDA device")
    from gsis_sim_b200 import case
    from gsis_sim_b200.backend import B200Backend
    from oracle.kinetic_oracle import OracleBackend

    cfg = case.load_case(CHANNEL)
    setup, host = case.case_setup(cfg)
    with B200Backend(setup) as be:
        g = _run(be, setup, host)
    o = _run(OracleBackend(setup), setup, host)
    assert common.max_rel(g[0], o[0]) < common.TOL["fp64"]
    assert common.max_rel(g[1], o[1]) < common.TOL["fp64"]
    assert abs(g[2][2] - o[2][2]) <= common.TOL["fp64"] * abs(o[2][2])
    assert g[2][2] > 0.0  # flow from the high-pressure inlet to the outlet

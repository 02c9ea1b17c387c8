"""The planar Couette slab at full size solved on the B200 backend from rest to residual 1e-8, against the reference
KineticSolver's converged run (tests/golden/converged/couette_slab_200.npz; case in tests/test_couette_slab.py).

FP64 moment fields must agree to 1e-6 relative; the residual history, the iteration count and the
wall fluxes are compared too, and the converged fields against the reference's independent 1-D solver ref1d."""
import time

import numpy as np
import pytest

from gsis_sim_b200.solver import KineticSolver
from tests import common
from tests.test_couette_slab import SXY, check_against_ref1d, load, x_order

pytestmark = pytest.mark.gpu

MOMENT_TOL = 1e-6


def test_gpu_couette_slab_converges_to_the_reference_state():
    import torch

    assert torch.cuda.is_available()
    from gsis_sim_b200.backend import B200Backend

    z, setup, host = load()
    ref = z["solver.infos"]
    tol = float(z["solver.tol"])
    with B200Backend(setup) as be:
        sol = KineticSolver(setup, host, be)
        init = z["solver.init"]
        sol.initialize_uniform(init[0], init[1:4], init[4])
        res = []
        t0 = time.perf_counter()
        while len(res) < len(ref) + 10:
            res.append(sol.sweep().residual)
            if len(res) > 1 and res[-1] < tol:
                break
        wall = time.perf_counter() - t0
        moments = sol.moments()
        fp, fm, _ = sol.boundary_fluxes()
        flows = sol.prepare().patch_mass_flow
    res = np.array(res)
    n = min(len(res), len(ref))
    print(f"B200: {len(res)} CIS iterations to residual {res[-1]:.3e} in {wall:.2f} s "
          f"(reference: {len(ref)} iterations)")
    # same iteration (the histories agree closely; the stop test may flip by one iteration at the threshold)
    assert abs(len(res) - len(ref)) <= 1
    assert res[-1] < tol
    assert common.max_rel(res[:n] / ref[:n, 6], np.ones(n)) < 1e-6
    assert common.max_rel(moments, z["solver.moments"]) < MOMENT_TOL
    for k in range(15):
        col = z["solver.moments"][:, k]
        if np.max(np.abs(col)) > 1e-3:
            assert common.max_rel(moments[:, k], col) < MOMENT_TOL, k
    order = x_order(z)
    assert common.max_rel(moments[order, SXY], z["solver.moments"][order, SXY]) < MOMENT_TOL
    assert common.max_rel(fp, z["solver.F_plus"]) < MOMENT_TOL
    assert common.max_rel(fm, z["solver.F_minus"]) < MOMENT_TOL
    assert np.max(np.abs(flows)) < 1e-8
    # and the independent 1-D solver of the same problem
    check_against_ref1d(z, moments)

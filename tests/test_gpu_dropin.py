"""Drop-in check: the reference's own KineticSolver, linked with the B200 KineticBackend shim
(gsis_sim_b200/integration/b200_backend.cpp) instead of its CUDA backend, reproduces the reference CPU results.

Needs oracle/_ref/libgsisref.so and libgsisdropin.so, which are built from the reference sources (oracle/Makefile,
targets ref and dropin); where they were not built the test is skipped."""
import numpy as np
import pytest

from tests import common

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", common.golden_names())
def test_reference_solver_on_b200_backend(name):
    from oracle import ref

    if not (ref.available() and ref.available(dropin=True)):
        pytest.skip("reference drop-in libraries not built here")
    from tests.golden.make_golden import CASES

    mesh_kw, bcs, Kn, nv, kin, init, iterations = CASES[name]
    z, setup = common.load(name)
    tol = common.TOL[common.precision_of(setup)]
    mesh = ref.RefMesh.box(**mesh_kw)
    case = ref.RefCase(mesh, ref.case_spec(bcs, Kn=Kn, nv=nv, kinetic=kin), dropin=True)
    case.init_uniform(init[0], init[1], init[2])
    infos = np.array([case.sweep() for _ in range(iterations)])
    ref_infos = z["solver.infos"]
    assert common.max_rel(infos[:, 6], ref_infos[:, 6]) < 100 * tol
    assert common.max_rel(case.moments(), z["solver.moments"]) < 10 * tol
    fp, fm, _ = case.boundary_fluxes()
    assert common.max_rel(fp, z["solver.F_plus"]) < 10 * tol
    assert common.max_rel(case.distribution(), z["solver.f"]) < tol

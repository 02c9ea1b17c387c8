"""The GPU baseline of bench.py is sound: the reference's own CUDA backend (CudaBackend, src/kinetic/
kinetic_backend_cuda.cpp + kinetic_cuda_kernels.cu, rebuilt unchanged for sm_100a by oracle/Makefile target refcuda)
under the reference KineticSolver reproduces the reference's CPU results on a B200, to the reference's own GPU-vs-CPU
tolerances (tests/kinetic/test_kinetic_gpu.cpp:133-158). Skipped where the reference sources were not present at
build time."""
import numpy as np
import pytest

from tests import common

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["mixed_strong_fp64", "vacuum_tube_fp64", "mixed_strong_fp32"])
def test_reference_cuda_backend_on_b200(name):
    from oracle import ref

    if not (ref.available() and ref.available(refcuda=True)):
        pytest.skip("reference CUDA library not built here")
    from tests.golden.make_golden import CASES

    mesh_kw, bcs, Kn, nv, kin, init, iterations = CASES[name]
    z, setup = common.load(name)
    tol = common.TOL[common.precision_of(setup)]
    mesh = ref.RefMesh.box(**mesh_kw)
    case = ref.RefCase(mesh, ref.case_spec(bcs, Kn=Kn, nv=nv, kinetic=kin), refcuda=True)
    case.init_uniform(init[0], init[1], init[2])
    infos = np.array([case.sweep() for _ in range(iterations)])
    assert common.max_rel(infos[:, 6], z["solver.infos"][:, 6]) < 100 * tol
    assert common.max_rel(case.moments(), z["solver.moments"]) < 10 * tol
    assert common.max_rel(case.distribution(), z["solver.f"]) < tol
    t = case.last_timings()
    assert t["gradient"] > 0.0 and t["sweep_forward"] > 0.0

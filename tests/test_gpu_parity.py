"""Parity of the B200 CUDA backend (through the C ABI) with the reference and with the oracle.

Reference values are the golden vectors of the reference's own CPU backend (tests/golden/*.npz); the tolerances
are those of the reference's GPU-vs-CPU tests (tests/kinetic/test_kinetic_gpu.cpp:133-158).
"""
import numpy as np
import pytest

from tests import common

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def B200Backend():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("no CUDA device")
    from gsis_sim_b200.backend import B200Backend as cls

    return cls


@pytest.mark.parametrize("name", common.golden_names())
def test_gpu_matches_reference_ops(B200Backend, name):
    z, setup = common.load(name)
    prec = common.precision_of(setup)
    with B200Backend(setup) as be:
        out = common.run_op_sequence(be, z)
        assert be.launch_count() > 0
    common.check_op_sequence(out, z, common.TOL[prec])


@pytest.mark.parametrize("name", ["mixed_strong_fp64", "mixed_strong_fp32", "dir13_fp32"])
def test_gpu_deterministic_and_chunk_independent(B200Backend, name):
    """Bitwise determinism and independence of the launch splitting (test_kinetic_gpu.cpp:175-186)."""
    z, setup = common.load(name)
    with B200Backend(setup) as be:
        a = common.run_op_sequence(be, z)
    with B200Backend(setup) as be:
        b = common.run_op_sequence(be, z)
    with B200Backend(setup, velocity_chunk=100) as be:
        c = common.run_op_sequence(be, z)
        assert be.chunk_width() == 100
    for k in ["f1", "f3", "res1", "bsums0", "moments2", "face_flux"]:
        assert np.array_equal(a[k], b[k]), k
    # With mirror orbits (symmetry planes) the backend orders velocities by (chunk, sweep direction), so a
    # different chunk width only changes the summation order of the velocity sums: agreement to rounding.
    tol = 1e-13 if common.precision_of(setup) == "fp64" else 1e-6
    for k in ["f1", "f3", "bsums0", "moments2", "res1"]:
        assert common.max_rel(a[k], c[k]) < tol, k


@pytest.mark.parametrize("name", ["mixed_strong_fp64", "maxwell_wall_fp64", "couette_fp64"])
@pytest.mark.parametrize("scheme", ["fp64", "defect"])
def test_gpu_mixed_precision_matches_oracle(B200Backend, name, scheme, monkeypatch):
    """Mixed precision (f, gradients and LU-SGS passes in FP32; residual, moments and sums in FP64) against the
    same scheme on the CPU oracle. Quantities computed in FP64 from the same FP32 f agree to 1e-6; the FP32
    arithmetic of the sweeps gets the reference's FP32 tolerance (FMA contraction differs between the two)."""
    from oracle.kinetic_oracle import OracleBackend

    monkeypatch.setenv("KIN_MIXED_RESIDUAL", scheme)  # both the B200 backend and the oracle read it
    z, setup = common.load(name)
    with B200Backend(setup, precision="mixed") as be:
        g = common.run_op_sequence(be, z)
    o = common.run_op_sequence(OracleBackend(setup, precision="mixed"), z)
    for k in ["moments0", "bsums0"]:
        assert common.max_rel(g[k], o[k]) < 1e-6, k
    for k in ["f1", "moments2", "f3", "face_flux", "res1"]:
        assert common.max_rel(g[k], o[k]) < common.TOL["fp32"], k
    # and it stays within the FP32 tolerance of the FP64 reference
    for k in ["f1", "f3", "res1"]:
        assert common.max_rel(g[k], z["op." + k]) < common.TOL["fp32"], k


@pytest.mark.parametrize("name", ["mixed_strong_fp64", "couette_fp64", "tet_positivity_fp32", "dir13_fp32", "vacuum_tube_fp64"])
def test_gpu_sweep_kernels_agree(B200Backend, name, monkeypatch):
    """Every LU-SGS block-pass kernel gives the same sweep: the staged tile kernel (default; 6- and 8-entry bounds,
    and another compiled tile shape), the resident kernel (6 and 8) and the plain level kernel."""
    z, setup = common.load(name)
    runs = {}
    kernels = ["auto", "staged8", "shape", "resident", "resident8", "legacy"]
    for kernel in kernels:
        monkeypatch.setenv("KIN_SWEEP_KERNEL", kernel)
        if kernel == "shape":  # the other compiled tile shape of the arithmetic type (velocities per thread x CTAs)
            monkeypatch.setenv("KIN_SWEEP_KERNEL", "auto")
            monkeypatch.setenv("KIN_SHAPE", "tile=4x4" if common.precision_of(setup) == "fp64" else "tile=2x8")
        with B200Backend(setup) as be:
            runs[kernel] = common.run_op_sequence(be, z)
    tol = 1e-14 if common.precision_of(setup) == "fp64" else 1e-6
    for kernel in kernels[1:]:
        for k in ["f1", "f3", "res1"]:
            assert common.max_rel(runs["auto"][k], runs[kernel][k]) < tol, (kernel, k)


@pytest.mark.parametrize("name", ["mixed_strong_fp64", "couette_fp64", "tet_positivity_fp32", "maxwell_wall_fp64"])
def test_gpu_tensor_grid_sums_agree(B200Backend, name, monkeypatch):
    """On a tensor velocity grid the discrete-equilibrium Newton sums are formed from per-axis sums; the per-velocity
    sums (KIN_VELOCITY_SUMS=pointwise) give the same operation sequence to rounding."""
    z, setup = common.load(name)
    runs = {}
    for mode in ["auto", "pointwise"]:
        monkeypatch.setenv("KIN_VELOCITY_SUMS", mode)
        with B200Backend(setup) as be:
            runs[mode] = common.run_op_sequence(be, z)
    # both stop the Newton iteration at its tolerance (1e-11 FP64, 1e-6 FP32), possibly one step apart
    tol = common.TOL[common.precision_of(setup)]
    for k in ["moments0", "bsums0", "f1", "f3", "moments2"]:
        assert common.max_rel(runs["auto"][k], runs["pointwise"][k]) < tol, k
    assert common.max_rel(runs["auto"]["res1"], runs["pointwise"]["res1"]) < 100 * tol
    assert np.array_equal(runs["auto"]["flags"], runs["pointwise"]["flags"])

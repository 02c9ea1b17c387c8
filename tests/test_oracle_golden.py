"""The CPU oracle (oracle/kinetic_oracle.c) against the golden vectors of the reference CPU backend.

This pins the oracle: every operation of the golden sequence must agree with the reference's own CpuBackend
(src/kinetic/kinetic_backend_cpu.cpp) within the reference's GPU-vs-CPU tolerances.
"""
import pytest

from tests import common
from oracle.kinetic_oracle import OracleBackend


@pytest.mark.parametrize("name", common.golden_names())
def test_oracle_matches_reference_ops(name):
    z, setup = common.load(name)
    prec = common.precision_of(setup)
    out = common.run_op_sequence(OracleBackend(setup), z)
    errs = common.check_op_sequence(out, z, common.TOL[prec])
    if prec == "fp64":
        # same arithmetic in the same order up to FMA contraction: far inside the tolerance
        assert max(errs.values()) < 1e-12, errs


@pytest.mark.parametrize("name", ["mixed_strong_fp64", "vacuum_tube_fp64"])
def test_oracle_chunk_independence(name):
    """Results do not depend on the velocity chunk width (tests/kinetic/test_kinetic_cpu.cpp:308-328)."""
    z, setup = common.load(name)
    a = common.run_op_sequence(OracleBackend(setup, velocity_chunk=0), z)
    b = common.run_op_sequence(OracleBackend(setup, velocity_chunk=96), z)
    for k in ["f1", "f3", "res1", "res2", "bsums0"]:
        assert common.max_rel(a[k], b[k]) < 1e-13, k


@pytest.mark.parametrize("name", ["mixed_strong_fp64", "vacuum_tube_fp64"])
@pytest.mark.parametrize("scheme", ["fp64", "defect"])
def test_oracle_mixed_precision_within_fp32_of_fp64(name, scheme, monkeypatch):
    """Mixed precision (f in FP32, FP32 gradient and sweeps) stays within the FP32 tolerance of the FP64 reference
    through the golden operation sequence, with the FP64 residual at every sweep (default) and with the defect scheme
    (KIN_MIXED_RESIDUAL=defect: FP64 residual at the first sweep after the cell parameters change, FP32 residual plus
    the stored defect at the sweeps after it; the sequence's second sweep runs on the defect)."""
    monkeypatch.setenv("KIN_MIXED_RESIDUAL", scheme)
    z, setup = common.load(name)
    out = common.run_op_sequence(OracleBackend(setup, precision="mixed"), z)
    tol = common.TOL["fp32"]
    for k in ["f1", "f3", "moments2", "face_flux"]:
        assert common.max_rel(out[k], z["op." + k]) < tol, k
    for k in ["res1", "res2"]:
        assert common.max_rel(out[k], z["op." + k]) < 100 * tol, k

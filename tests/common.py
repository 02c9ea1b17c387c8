"""Shared helpers of the tests: golden fixtures, comparisons, tolerances."""
from __future__ import annotations

import glob
import os

import numpy as np

from gsis_sim_b200 import abi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Tolerances of the reference's own GPU-vs-CPU parity tests (tests/kinetic/test_kinetic_gpu.cpp:133-158):
# FP32 2e-5, FP64 1e-11 (old CIS settings) / 1e-10 (default strong CIS).
TOL = {"fp32": 2e-5, "fp64": 1e-10, "mixed": 2e-5}


def golden_names():
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load(name: str):
    z = np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False)
    return z, abi.SetupArrays.from_npz(z)


def precision_of(setup: abi.SetupArrays) -> str:
    return {abi.KIN_PREC_FP32: "fp32", abi.KIN_PREC_FP64: "fp64", abi.KIN_PREC_MIXED: "mixed"}[int(setup["precision"])]


def max_rel(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.max(np.abs(a - b)) if a.size else 0.0
    s = np.max(np.abs(b)) if b.size else 0.0
    return float(d / s) if s > 0 else float(d)


def run_op_sequence(backend, z) -> dict:
    """The golden operation sequence (tests/golden/make_golden.py, run_case) on any backend."""
    out = {}
    backend.set_equilibrium(z["op.states"])
    out["moments0"] = backend.compute_moments().copy()
    backend.update_cell_params()
    out["deq0"] = np.array(backend.deq_counts())
    backend.set_inflow(z["op.inflow"])
    out["bsums0"] = backend.boundary_sums().copy()
    out["res1"] = backend.sweep().copy()
    out["f1"] = backend.get_distribution().copy()
    out["res2"] = backend.sweep().copy()
    out["moments2"] = backend.compute_moments().copy()
    replaced, flags = backend.gsis_correction(z["op.w_half"], z["op.w_new"])
    out["replaced"] = np.array([replaced])
    out["flags"] = flags
    out["f3"] = backend.get_distribution().copy()
    out["face_flux"] = backend.internal_face_mass_flux(z["op.face_cells"], z["op.face_entries"])
    return out


def check_op_sequence(out: dict, z, tol: float):
    """Compare an operation sequence against the golden reference outputs."""
    errors = {}
    for k in ["moments0", "bsums0", "res1", "f1", "res2", "moments2", "f3", "face_flux"]:
        errors[k] = max_rel(out[k], z["op." + k])
    for k, e in errors.items():
        # residual sums of squares: relative 100x the field tolerance, as the reference compares the history
        lim = 100 * tol if k.startswith("res") else tol
        assert e < lim, f"{k}: max relative difference {e:.3e} >= {lim:.1e} ({errors})"
    assert int(out["replaced"][0]) == int(z["op.replaced"][0])
    assert np.array_equal(out["flags"], z["op.flags"])
    assert np.array_equal(out["deq0"][:2], z["op.deq0"][:2])
    return errors

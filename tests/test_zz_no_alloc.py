"""kin_discrete_maxwell_noalloc (the allocation-free discrete Maxwellian) against kin_discrete_maxwell.

Both are called through the C ABI on the same states. The file name makes pytest collect it last, so it runs after
every other GPU test has used the device, and it also passes on its own.
"""
import ctypes as C

import numpy as np
import pytest

from tests import common

pytestmark = pytest.mark.gpu


def _states(n, seed):
    """Inflow-like macroscopic states (rho, ux, uy, uz, T), many of them poorly resolved by the velocity grid."""
    rng = np.random.default_rng(seed)
    st = np.empty((n, 5))
    st[:, 0] = rng.uniform(0.2, 3.0, n)
    st[:, 1:4] = rng.uniform(-1.0, 1.0, (n, 3))
    st[:, 4] = rng.uniform(0.4, 2.0, n)
    return st


def _noalloc(be, fn, st, tol):
    from gsis_sim_b200 import abi

    st = np.ascontiguousarray(st)
    out = np.full_like(st, np.nan)
    res = np.full(len(st), -99, dtype=np.int32)
    rc = fn(be._h, abi.as_ptr(st, C.c_double), len(st), C.c_double(tol), abi.as_ptr(out, C.c_double),
            abi.as_ptr(res, C.c_int32))
    return rc, out, res


def test_noalloc_matches_discrete_maxwell():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("no CUDA device")
    from gsis_sim_b200 import abi
    from gsis_sim_b200.backend import B200Backend

    _, setup = common.load("mixed_strong_fp64")
    tol = 1e-10
    with B200Backend(setup) as be:
        fn = be._lib.kin_discrete_maxwell_noalloc
        # two calls in a row: a full scratch, then a shorter batch of other states
        for n, seed in [(abi.KIN_NOALLOC_MAX_STATES, 1), (1000, 2)]:
            st = _states(n, seed)
            ref_out, ref_res = be.discrete_maxwell(st, tol)
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            rc, out, res = _noalloc(be, fn, st, tol)
            assert rc == abi.KIN_OK, be._error_fn()
            # the point of the entry point: the call reserves no device memory
            assert torch.cuda.mem_get_info()[0] == free_before
            np.testing.assert_array_equal(res, ref_res)
            assert (res > 0).any(), "no state was corrected: the case does not exercise the Newton solve"
            assert common.max_rel(out, ref_out) < common.TOL["fp64"]


def test_noalloc_rejects_oversize_and_accepts_empty():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("no CUDA device")
    from gsis_sim_b200 import abi
    from gsis_sim_b200.backend import B200Backend

    _, setup = common.load("mixed_strong_fp64")
    with B200Backend(setup) as be:
        fn = be._lib.kin_discrete_maxwell_noalloc
        st = _states(abi.KIN_NOALLOC_MAX_STATES + 1, 3)
        rc, out, res = _noalloc(be, fn, st, 1e-10)
        assert rc == abi.KIN_E_ARG
        assert "split the batch" in be._error_fn()
        assert np.isnan(out).all() and (res == -99).all()
        rc, _, _ = _noalloc(be, fn, st[:0], 1e-10)
        assert rc == abi.KIN_OK

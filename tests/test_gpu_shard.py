"""Velocity sharding on the B200 backend: two shards of one case on the same GPU in one process (host-side
reductions; no kernel waits on another), against the unsharded backend, FP64 and mixed precision. Exercises
kin_moment_sums, kin_set_moments and the full-grid discrete equilibrium of a shard."""
import numpy as np
import pytest

from tests import common

pytestmark = pytest.mark.gpu


def _run(backend, setup, name, iters=2):
    from gsis_sim_b200.kinetic_setup import HostSetup
    from gsis_sim_b200.solver import KineticSolver

    z, _ = common.load(name)
    sol = KineticSolver(setup, HostSetup.from_npz(z), backend)
    sol.initialize_uniform(1.0, (0.0, 0.0, 0.0), 1.0)
    res = [sol.sweep().residual for _ in range(iters)]
    return sol.moments(), np.array(res), sol.mass_flow()[2]


@pytest.mark.parametrize("name", ["mixed_strong_fp64", "couette_fp64"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
@pytest.mark.parametrize("device", [False, True])
def test_two_shards_on_one_gpu_match_unsharded(name, precision, tol, device):
    """device=True: the sums are added in device memory (kin_device_sums) and the moments finalised on the device
    (kin_finalize_moments), the path a multi-GPU run takes with NCCL between the ranks."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("no CUDA device")
    from gsis_sim_b200 import shard
    from gsis_sim_b200.backend import B200Backend

    _, setup = common.load(name)
    with B200Backend(setup, precision=precision) as be:
        ref = _run(be, setup, name)
    ranges = shard.shard_ranges(setup, 2)
    bes = [B200Backend(shard.shard_setup(setup, lo, hi), precision=precision) for lo, hi in ranges]
    try:
        got = _run(shard.ShardedBackend(setup, bes, ranges, device=device), setup, name)
    finally:
        for be in bes:
            be.close()
    assert common.max_rel(got[0], ref[0]) < tol
    assert common.max_rel(got[1], ref[1]) < tol
    assert abs(got[2] - ref[2]) <= tol * abs(ref[2])


@pytest.mark.parametrize("mode", ["all", "limit", "blend"])
def test_two_shards_gsis_correction_on_one_gpu(mode):
    """The two-phase GSIS correction (kin_gsis_correction_extrema / _apply) over two B200 shards makes the same
    decisions and the same f as kin_gsis_correction on the whole grid."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("no CUDA device")
    from gsis_sim_b200 import abi, shard
    from gsis_sim_b200.backend import B200Backend

    z, setup = common.load("mixed_strong_fp64")
    setup = setup.copy()
    setup.scalars["negative_check_mode"] = abi.NEGATIVE_MODES[mode]

    def run(be):
        be.set_equilibrium(z["op.states"])
        be.compute_moments()
        be.update_cell_params()
        r, fl = be.gsis_correction(z["op.w_half"], z["op.w_new"])
        return r, fl, be.compute_moments()

    with B200Backend(setup) as be:
        ref = run(be)
    ranges = shard.shard_ranges(setup, 2)
    bes = [B200Backend(shard.shard_setup(setup, lo, hi)) for lo, hi in ranges]
    try:
        got = run(shard.ShardedBackend(setup, bes, ranges))
    finally:
        for be in bes:
            be.close()
    assert got[0] == ref[0] and np.array_equal(got[1], ref[1])
    assert common.max_rel(got[2], ref[2]) < 1e-12

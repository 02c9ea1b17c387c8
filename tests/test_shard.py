"""Velocity sharding (gsis_sim_b200.shard) on the CPU oracle: the host loop over 2 or 3 shards, in one process and as
two gloo ranks, reproduces the unsharded run (sums in another order: agreement to rounding)."""
import os
import socket

import numpy as np
import pytest

from tests import common

CASES = ["couette_fp64", "mixed_strong_fp64", "vacuum_tube_fp64"]


def _run(backend, setup, iters=2):
    from gsis_sim_b200.kinetic_setup import HostSetup
    from gsis_sim_b200.solver import KineticSolver

    z, _ = common.load(setup[1])
    host = HostSetup.from_npz(z)
    sol = KineticSolver(setup[0], host, backend)
    sol.initialize_uniform(1.0, (0.0, 0.0, 0.0), 1.0)
    res = [sol.sweep().residual for _ in range(iters)]
    return sol.moments(), np.array(res), sol.mass_flow()[2]


def _sharded(setup, n, allreduce=None, ranks=None):
    from gsis_sim_b200 import shard
    from oracle.kinetic_oracle import OracleBackend

    ranges = shard.shard_ranges(setup, n)
    keep = range(n) if ranks is None else ranks
    bes = [OracleBackend(shard.shard_setup(setup, *ranges[k])) for k in keep]
    return shard.ShardedBackend(setup, bes, [ranges[k] for k in keep], allreduce)


def _check(a, b):
    assert common.max_rel(a[0], b[0]) < 1e-12
    assert common.max_rel(a[1], b[1]) < 1e-12
    assert abs(a[2] - b[2]) <= 1e-12 * max(abs(b[2]), 1e-300)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("n", [2, 3])
def test_sharded_host_loop_matches_unsharded(name, n):
    from oracle.kinetic_oracle import OracleBackend

    _, setup = common.load(name)
    ref = _run(OracleBackend(setup), (setup, name))
    got = _run(_sharded(setup, n), (setup, name))
    _check(got, ref)


def test_shard_ranges_follow_mirror_orbits():
    from gsis_sim_b200 import shard

    _, setup = common.load("couette_fp64")  # symmetry plane: orbits of two velocities
    orb = shard.orbit_size(setup)
    assert orb > 1
    for lo, hi in shard.shard_ranges(setup, 3):
        assert lo % orb == 0 and hi % orb == 0
    with pytest.raises(ValueError):
        shard.shard_setup(common.load("maxwell_wall_fp64")[1], 0, 256)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, name, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=120))
    from gsis_sim_b200 import shard

    _, setup = common.load(name)
    be = _sharded(setup, 2, shard.torch_allreduce(), ranks=[rank])
    m, res, mdot = _run(be, (setup, name))
    dist.barrier()
    out.put((rank, m, res, mdot))
    dist.destroy_process_group()


def test_sharded_over_two_gloo_ranks():
    import torch.multiprocessing as mp

    from oracle.kinetic_oracle import OracleBackend

    name = "mixed_strong_fp64"
    _, setup = common.load(name)
    ref = _run(OracleBackend(setup), (setup, name))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, name, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, m, res, mdot in got:
        _check((m, res, mdot), ref)


def _correction(backend, setup, z):
    """An equilibrium state, then the golden GSIS correction (w_half, w_new) with its negativity rule."""
    backend.set_equilibrium(z["op.states"])
    backend.compute_moments()
    backend.update_cell_params()
    replaced, flags = backend.gsis_correction(z["op.w_half"], z["op.w_new"])
    backend.compute_moments()
    f = backend.get_distribution()
    return replaced, flags, f


@pytest.mark.parametrize("mode", ["all", "created", "limit", "blend"])
@pytest.mark.parametrize("n", [2, 3])
def test_sharded_gsis_correction_matches_unsharded(mode, n):
    """The two-phase GSIS correction over velocity shards (per-cell extrema reduced with a minimum) makes the same
    per-cell decisions and the same f as the correction on the whole grid, for every negativity rule."""
    from gsis_sim_b200 import abi
    from oracle.kinetic_oracle import OracleBackend

    z, setup = common.load("mixed_strong_fp64")
    setup = setup.copy()
    setup.scalars["negative_check_mode"] = abi.NEGATIVE_MODES[mode]
    r0, fl0, f0 = _correction(OracleBackend(setup), setup, z)
    r1, fl1, f1 = _correction(_sharded(setup, n), setup, z)
    assert r0 == r1 and np.array_equal(fl0, fl1)
    assert (fl0 != 0).any() and (fl0 == 0).any(), "the case must exercise both outcomes of the rule"
    assert common.max_rel(f1, f0) < 1e-14


def _rank_correction(rank, port, mode, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=120))
    from gsis_sim_b200 import abi, shard

    z, setup = common.load("mixed_strong_fp64")
    setup = setup.copy()
    setup.scalars["negative_check_mode"] = abi.NEGATIVE_MODES[mode]
    be = _sharded(setup, 2, shard.torch_allreduce(), ranks=[rank])
    be.set_equilibrium(z["op.states"])
    be.compute_moments()
    be.update_cell_params()
    replaced, flags = be.gsis_correction(z["op.w_half"], z["op.w_new"])
    m = be.compute_moments()
    dist.barrier()
    out.put((rank, replaced, flags, m))
    dist.destroy_process_group()


@pytest.mark.parametrize("mode", ["limit", "blend"])
def test_sharded_gsis_correction_over_two_gloo_ranks(mode):
    """The same over two gloo ranks: the per-cell extrema are all-reduced with a minimum between the phases."""
    import torch.multiprocessing as mp

    from gsis_sim_b200 import abi
    from oracle.kinetic_oracle import OracleBackend

    z, setup = common.load("mixed_strong_fp64")
    setup = setup.copy()
    setup.scalars["negative_check_mode"] = abi.NEGATIVE_MODES[mode]
    be = OracleBackend(setup)
    r0, fl0, _ = _correction(be, setup, z)
    m0 = be.compute_moments()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_correction, args=(r, port, mode, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, r, fl, m in got:
        assert r == r0 and np.array_equal(fl, fl0)
        assert common.max_rel(m, m0) < 1e-12

"""The multi-rank timing path of bench.py (replicas, one per GPU) with two gloo ranks on the CPU: every rank
reports the element-wise maximum of the ranks' timings."""
import os
import socket


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    import bench

    vals = bench.max_over_ranks([1.0 + rank, 5.0 - rank, 0.25 * rank], ws, device="cpu")
    dist.barrier()
    out.put((rank, vals))
    dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == res[1] == [2.0, 5.0, 0.25]


def test_max_over_ranks_single_rank_is_identity():
    import bench

    assert bench.max_over_ranks([3, 1.5], 1) == [3.0, 1.5]

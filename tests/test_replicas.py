"""The multi-process path (one process per GPU, replicated joins) on CPU:
two gloo ranks reduce their step numbers to the slowest rank's time and the
sum of the pairs, as bench.py reports them."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import torch.distributed as dist

    from gpu_self_join_b200.replicas import reduce_step

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms, pairs = reduce_step(10.0 + 5.0 * rank, 1000.0 * (rank + 1))
        out.put((rank, ms, pairs))
    finally:
        dist.destroy_process_group()


def test_reduce_step_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, ms, pairs in res:
        assert ms == pytest.approx(15.0) and pairs == pytest.approx(3000.0)


def test_reduce_step_single_process():
    from gpu_self_join_b200.replicas import reduce_step

    assert reduce_step(3.5, 42.0) == (3.5, 42.0)

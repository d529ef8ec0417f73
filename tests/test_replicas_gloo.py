"""Multi-GPU path of bench.py on CPU: replicas with no data-path collective, timed
as the maximum over ranks. Two gloo ranks (127.0.0.1) stand in for two GPUs."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r "took" 100 + 10 r ms for the refined arm and 300 - r ms for the plain arm
        mx = bench.max_over_ranks(dist, [100.0 + 10 * rank, 300.0 - rank])
        q.put((rank, mx, bench.replica_value(64 * 8, world, mx[0])))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_take_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, value in out:
        assert mx == [110.0, 300.0]
        assert value == pytest.approx(2 * 64 * 8 / 0.110)

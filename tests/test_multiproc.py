"""The N>1 path of bench.py on CPU: independent replicas, one process per
rank, timing taken as the maximum over ranks (gloo, world size 2)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = bench.max_over_ranks(10.0 + 5.0 * rank, "cpu", world)
        r, w, _ = bench.dist_env()
        q.put((rank, got, r, w))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [r[1] for r in res] == [15.0, 15.0]
    assert [(r[2], r[3]) for r in res] == [(0, 2), (1, 2)]


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(3.5, "cpu", 1) == 3.5


@pytest.mark.parametrize("n", [1, 2])
def test_reference_arm_other_ranks_do_no_work(monkeypatch, n):
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        pass
    assert bench.run_reference(A()) is None

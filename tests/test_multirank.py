"""Host logic of the multi-GPU bench path on CPU: two gloo ranks agree on the max of
their step times and use distinct seeded replicas (no data-path collective)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(1.5 + rank, dist, "cpu")
        q.put((rank, t, bench.shard_seeds(rank), bench.dist_env()))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(world))
    assert [o[1] for o in out] == [2.5, 2.5]
    assert out[0][2] != out[1][2]
    assert out[1][3] == (1, 2, 1)

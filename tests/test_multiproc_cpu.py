"""The N>1 host path on CPU: two gloo ranks. Roots are independent, so ranks
that take disjoint root shards (oracle root sampling, stride = world size)
sum to the full count, and device times are combined as the max over ranks
(bench.py's helpers)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import beep_b200 as B
        from beep_b200 import patterns as P
        from oracle import pyoracle as O

        rp, col = B.gen_rmat(11, 8, 0.57, 0.19, 0.19, 5)
        part = O.count(rp, col, P.DIAMOND, apply_root_cap=False, root_stride=world, root_offset=rank, threads=1)
        total = bench.sum_over_ranks(int(part["count"]), world)
        slowest = bench.max_over_ranks(float(rank + 1), world)
        bench.barrier(world)
        q.put((rank, total, slowest, part["roots_processed"]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_roots(built):
    from beep_b200 import gen_rmat
    from beep_b200 import patterns as P
    from oracle import pyoracle as O

    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    rp, col = gen_rmat(11, 8, 0.57, 0.19, 0.19, 5)
    full = O.count(rp, col, P.DIAMOND, apply_root_cap=False)
    for rank, total, slowest, processed in res:
        assert total == full["count"]
        assert slowest == float(world)
    assert sum(r[3] for r in res) == full["roots"]

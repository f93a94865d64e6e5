"""The N>1 host path on CPU: two gloo ranks through bench.py's own sharding
helper (sharded_counts), with the oracle standing in for beep_count_shard:
each rank counts the roots whose input id % world == rank, one all-reduce
sums the per-pattern counts, and device times are combined as the max over
ranks."""
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
        processed = []

        def count_shard(name, shard, nshards):
            r = O.count(rp, col, P.NAMED[name], apply_root_cap=False, root_mod=nshards, root_rem=shard, threads=1)
            processed.append(r["roots_processed"])
            return r["count"]

        totals = bench.sharded_counts(count_shard, ["diamond", "k4"], world, rank)
        slowest = bench.max_over_ranks(float(rank + 1), world)
        bench.barrier(world)
        q.put((rank, totals, slowest, processed[0]))
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
    full = [O.count(rp, col, P.NAMED[name], apply_root_cap=False) for name in ("diamond", "k4")]
    for rank, totals, slowest, processed in res:
        assert totals == [f["count"] for f in full]
        assert slowest == float(world)
    # the shards partition the roots
    assert sum(r[3] for r in res) == full[0]["roots_processed"]

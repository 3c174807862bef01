"""The multi-GPU path of bench.py on CPU ranks (gloo, world size 2): every
rank joins the same build table against its own probe shard, the partial
SUM/COUNT are summed over ranks and the step time is the slowest rank's.
The combined result must equal the join over all shards at once."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

BUILD, PROBE, DOMAIN = 20_000, 50_000, 25_000


def shard(rank):
    import qumirdb_b200 as q
    b = [np.empty(BUILD, np.int64), np.empty(BUILD, np.int64), np.empty(BUILD, np.int32)]
    q.lib().qdb_gen_join(1, BUILD, 0, DOMAIN, *[x.ctypes.data for x in b], None, None)
    p = [np.empty(PROBE, np.int64), np.empty(PROBE, np.int64)]
    tmp = [np.empty(1, np.int64), np.empty(1, np.int64), np.empty(1, np.int32)]
    q.lib().qdb_gen_join(1000 + rank, 1, PROBE, DOMAIN, *[t.ctypes.data for t in tmp], *[x.ctypes.data for x in p])
    return b, p


def oracle_join_sum(b, p):
    import qumirdb_b200 as q
    from oracle import oracle as O
    from qumirdb_b200 import queries
    jspec, aspec = queries.join_sum(20)
    rows = O.join_aggregate(jspec, aspec, [q.HostRowSet(b)], [q.HostRowSet(p)])
    return int(rows[0][0]), int(rows[0][1])


def worker(rank, world, port, out):
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b, p = shard(rank)
        s, c = oracle_join_sum(b, p)
        total = bench.combine_partials(dist, s, c, device="cpu")
        slowest = bench.max_over_ranks(dist, 10.0 + rank, device="cpu")
        if rank == 0:
            ps = [shard(r)[1] for r in range(world)]
            whole = oracle_join_sum(b, [np.concatenate([x[j] for x in ps]) for j in range(2)])
            out.put((total, whole, slowest))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_join_partials_combine_over_two_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port, out)) for r in range(2)]
    for pr in procs:
        pr.start()
    total, whole, slowest = out.get(timeout=240)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    assert total == whole
    assert total[1] > 0
    assert slowest == 11.0

"""Multi-GPU batch / serve split: every rank derives its share of a process map or request stream
from the same seeded inputs (greedy bin-packing by HBM footprint, no exchange), so the shares
cover every domain exactly once and balance the footprint. Checked with two gloo ranks on CPU."""
import os
import socket

import torch.distributed as dist
import torch.multiprocessing as mp

from exaca_b200 import batch, serve


def test_partition_balances_and_covers():
    w = [batch.footprint(p) for p in batch.process_map(256, seed=3)]
    for n in (1, 2, 3, 8):
        parts = batch.partition(w, n)
        assert sorted(i for p in parts for i in p) == list(range(len(w)))
        loads = [sum(w[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(w)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    params = batch.process_map(64, seed=3)
    mine = batch.partition([batch.footprint(p) for p in params], world)[rank]
    reqs = serve.request_stream(40, rate=200.0, seed=4)
    mine_r = batch.partition([batch.footprint(p) for _, p in reqs], world)[rank]
    got = [None] * world
    dist.all_gather_object(got, (mine, mine_r))
    if rank == 0:
        out.put(got)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_cover_the_map_and_the_stream():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    domains = sorted(i for part, _ in got for i in part)
    requests = sorted(i for _, part in got for i in part)
    assert domains == list(range(64)) and requests == list(range(40))
    assert set(got[0][0]).isdisjoint(got[1][0]) and set(got[0][1]).isdisjoint(got[1][1])

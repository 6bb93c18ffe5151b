"""The multi-rank plumbing of bench.py and of sharded runs
(polystring_b200/dist.py) on two gloo ranks on the CPU: barriers,
max / sum over ranks, the whole-job throughput, and the partition of units
(batch solves, string images) over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from polystring_b200.dist import shard


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from polystring_b200.dist import Ranks, shard, throughput
    r = Ranks("gloo", timeout_s=30)
    r.barrier()
    t = 1.0 + rank                       # this rank's "time"
    units = 100 * (rank + 1)             # and its work
    out = {"rank": r.rank, "max": r.allmax(t), "sum": r.allsum(units), "thr": throughput(units, t, r),
           "mine": list(shard(11, r.rank, r.world))}
    r.close()
    q.put(out)


def test_two_gloo_ranks_reduce_and_partition():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_worker, args=(k, world, port, q)) for k in range(world)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda d: d["rank"])
    for d in res:
        assert d["max"] == 2.0
        assert d["sum"] == 300.0
        assert d["thr"] == 150.0         # all units / slowest rank's time
    assert res[0]["mine"] + res[1]["mine"] == list(range(11))


@pytest.mark.parametrize("n,world", [(40, 1), (40, 3), (7, 8), (0, 2), (256, 8)])
def test_shard_covers_every_unit_once_and_balances(n, world):
    parts = [list(shard(n, r, world)) for r in range(world)]
    assert sum(parts, []) == list(range(n))
    sizes = [len(p) for p in parts]
    assert max(sizes) - min(sizes) <= 1


def test_single_process_needs_no_group():
    from polystring_b200.dist import Ranks
    for k in ("RANK", "WORLD_SIZE"):
        os.environ.pop(k, None)
    r = Ranks()
    assert r.world == 1 and r.dist is None
    assert r.allmax(3.5) == 3.5 and r.allsum(2) == 2.0
    r.close()

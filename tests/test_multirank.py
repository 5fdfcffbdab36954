"""CPU, world_size 2 over gloo: the multi-GPU path (shard the range at
== 2 (mod 30) boundaries, count each shard, all_reduce the six totals) gives
exactly the single-range counts. Each rank's shard is counted by the oracle
here (the CPU stand-in for that rank's GPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import REPO


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def worker(rank, world, port, cases, q):
    import sys
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import torch.distributed as dist
    from conftest import Oracle, load_package
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    psg = load_package()
    orc = Oracle()
    res = []
    for a, b in cases:
        res.append(psg.count_sharded(lambda x, y, k: orc.plain(x, y, k), a, b, 0x3F, rank, world))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, res))


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_counts_match(world, oracle, ref_counts):
    cases = [(0, 10 ** 6), (999999900, 1000000331), (10 ** 12, 10 ** 12 + 3 * 10 ** 5), (0, 40), (7, 7)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, cases, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = {}
    for _ in range(world):
        r, res = q.get(timeout=300)
        results[r] = res
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for i, (a, b) in enumerate(cases):
        want = oracle.plain(a, b)
        for r in range(world):
            assert results[r][i] == want, (a, b, r)


def test_balance_ranges_partitions_the_batch_evenly(psg):
    """The multi-GPU batch split: every range goes to exactly one rank, each
    rank's estimated work is within 2% of the mean on the 4096-range
    workload, and the split is the same whichever process computes it."""
    import json
    from conftest import GOLDEN
    with open(os.path.join(GOLDEN, "batch4096.json")) as f:
        rows = [(a, b) for a, b, _, _ in json.load(f)["ranges"]]
    for world in (1, 2, 3, 4, 8):
        parts = psg.balance_ranges(rows, world)
        assert len(parts) == world
        assert sorted(i for p in parts for i in p) == list(range(len(rows)))
        loads = [sum(psg.range_cost(*rows[i]) for i in p) for p in parts]
        assert max(loads) <= 1.02 * sum(loads) / world, (world, loads)
        assert parts == psg.balance_ranges(list(rows), world)
    # by index (i mod N) the same workload is far from even
    loads = [sum(psg.range_cost(*rows[i]) for i in range(r, len(rows), 8)) for r in range(8)]
    assert max(loads) > 1.05 * sum(loads) / 8


def batch_worker(rank, world, port, ranges, q):
    import sys
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import torch
    import torch.distributed as dist
    from conftest import Oracle, load_package
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    psg = load_package()
    orc = Oracle()
    mine = psg.balance_ranges([(a, b) for a, b, _ in ranges], world)[rank]
    rows = torch.zeros(len(ranges), 6, dtype=torch.int64)
    for i in mine:
        a, b, k = ranges[i]
        rows[i] = torch.tensor(orc.plain(a, b, k), dtype=torch.int64)
    dist.all_reduce(rows, op=dist.ReduceOp.SUM)     # every row comes from exactly one rank
    dist.destroy_process_group()
    q.put((rank, rows.tolist()))


def test_balanced_batch_over_ranks_matches(oracle):
    """A batch split over 3 gloo ranks by balance_ranges, each rank counting
    its share (the oracle stands in for its GPU), gives every range's counts
    once: summing the rows over ranks equals counting all ranges in one place."""
    import random
    rng = random.Random(3)
    ranges = [(x, x + rng.randrange(1, 2 * 10 ** 5), rng.choice([1, 2, 4, 63]))
              for x in (rng.randrange(10 ** 12) for _ in range(40))]
    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=batch_worker, args=(r, world, port, ranges, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = [oracle.plain(a, b, k) for a, b, k in ranges]
    for _, rows in got:
        assert rows == want

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

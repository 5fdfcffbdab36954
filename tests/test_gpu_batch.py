"""GPU: the batched path (psg_count_batch -> persistent batch kernel plus the
windowed bucket path for long high ranges). Every row must equal the
per-range count bit for bit: the 4096-range fixture whose counts were made
by the reference's CPU library, edge cases against psg_count, seeded random
ranges against the oracle, and each range alone against the same range in
a mixed batch."""
import json
import os
import random

import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

BATCH = os.path.join(REPO, "tests", "golden", "batch4096.json")


def _load():
    with open(BATCH) as f:
        return json.load(f)["ranges"]


def _rows(ranges):
    return [(a, b, 1 << k) for a, b, k, _ in ranges]


def test_batch_fixture_4096(ctx):
    data = _load()
    got = ctx.count_batch(_rows(data))
    bad = [(a, b, k, want, g) for (a, b, k, want), g in zip(data, got)
           if g[k] != want or any(g[j] for j in range(6) if j != k)]
    assert not bad, bad[:5]
    stats = ctx.kernel_stats()
    assert stats["batch_sieve_kernel"][0] >= 1       # the persistent kernel ran


def test_batch_uses_both_paths(ctx):
    ctx.reset_kernel_stats()
    ranges = [(10 ** 15, 10 ** 15 + 10 ** 10, 1),     # long, many big primes: bucket path
              (10 ** 15, 10 ** 15 + 10 ** 6, 1),      # short: batch kernel (direct tier)
              (10 ** 9, 10 ** 9 + 10 ** 9, 63)]       # no big primes: batch kernel
    got = ctx.count_batch(ranges)
    stats = ctx.kernel_stats()
    assert stats["batch_sieve_kernel"][0] == 1
    assert stats["bucket_fill_kernel"][0] >= 1
    for (a, b, k), g in zip(ranges, got):
        assert g == ctx.count(a, b, k)


EDGES = [
    (0, 0, 63), (0, 1, 63), (0, 2, 63), (2, 2, 1), (3, 5, 63), (4, 4, 63), (5, 17, 63),
    (0, 6, 63), (6, 6, 63), (7, 7, 63), (0, 30, 63), (0, 100, 0), (10, 5, 63),
    (2 ** 64 - 1, 2 ** 64 - 1, 63), (2 ** 64 - 59, 2 ** 64 - 59, 1),
    (2 ** 64 - 10 ** 6, 2 ** 64 - 1, 63), (2 ** 63 - 10 ** 6, 2 ** 63 + 10 ** 6, 63),
    (2 ** 32 - 1000, 2 ** 32 + 1000, 63), (999999999989, 1000000200000, 63),
    (10 ** 12, 10 ** 12 + 10 ** 9, 63), (10 ** 13, 10 ** 13 + 2 ** 34, 7),
    (10 ** 18, 10 ** 18 + 10 ** 8, 63), (0, 10 ** 9, 63), (10 ** 6, 10 ** 6 + 2 ** 16, 2),
]


def test_batch_edges_match_single(ctx):
    got = ctx.count_batch(EDGES)
    for (a, b, k), g in zip(EDGES, got):
        assert g == ctx.count(a, b, k), (a, b, k)


def test_batch_empty(ctx):
    assert ctx.count_batch([]) == []


def test_batch_random_vs_oracle(ctx, oracle):
    rnd = random.Random(7)
    ranges = []
    for _ in range(300):
        a = rnd.choice([rnd.randrange(0, 10 ** 4), rnd.randrange(0, 10 ** 9), rnd.randrange(0, 10 ** 13)])
        b = a + rnd.choice([0, 1, 29, 31, 1000, rnd.randrange(0, 3 * 10 ** 6)])
        ranges.append((a, b, 63))
    got = ctx.count_batch(ranges)
    for (a, b, k), g in zip(ranges, got):
        assert g == oracle.plain(a, b), (a, b)


def test_batch_alone_equals_in_mix(ctx):
    data = _load()
    rnd = random.Random(3)
    picks = rnd.sample(range(len(data)), 12)
    mix = _rows(data[:600])
    for i in picks:
        a, b, k, want = data[i]
        alone = ctx.count_batch([(a, b, 1 << k)])[0]
        assert alone[k] == want
        in_mix = ctx.count_batch(mix + [(a, b, 1 << k)] + mix[:50])[600]
        assert in_mix == alone


def test_autotune_then_exact(psg):
    """The autotuner changes only how ranges are scheduled: after tuning on a
    sample every row of the fixture is still bit-exact."""
    data = _load()
    with psg.Context() as c:
        rep = c.autotune_batch(_rows(data[:1500]), budget_seconds=20.0)
        assert rep and all(r["best_seconds"] <= r["default_seconds"] + 1e-9 or r["default_seconds"] == 0 for r in rep)
        got = c.count_batch(_rows(data))
    bad = [(a, b, k, want, g) for (a, b, k, want), g in zip(data, got) if g[k] != want]
    assert not bad, bad[:5]

"""GPU parity: every count from the CUDA path (through the C ABI, the
primesieve C API, the C++ API and the CLI) equals the reference's counts
bit for bit: the reference's own golden vectors, counts computed by the
reference's CPU library, and the oracle on the same seeded inputs."""
import ctypes
import os
import random
import subprocess

import pytest

from conftest import REPO, PKG_DIR

pytestmark = pytest.mark.gpu


def test_reference_computed_cases(ctx, ref_counts):
    """test/gpu_count.cpp case list (every kind at 18 small stops, every start
    residue mod 30, segment boundaries near 1e9, five larger ranges), edges
    near 2^32, 2^63 and 2^64, and seeded random ranges."""
    by_range = {}
    for c in ref_counts["cases"]:
        by_range.setdefault((c["start"], c["stop"]), []).append(c)
    for (a, b), cs in by_range.items():
        got = ctx.count(a, b)
        for c in cs:
            assert got[c["kind"]] == c["count"], (a, b, c, got)


def test_reference_vectors(ctx, ref_vectors):
    """Known answers from the reference's tests, including the stress-test
    tables (99 windows of 1e11 at 1e13 and at 1e19)."""
    by_range = {}
    for v in ref_vectors:
        by_range.setdefault((v["start"], v["stop"]), []).append(v)
    for (a, b), vs in sorted(by_range.items()):
        kinds = 0
        for v in vs:
            kinds |= 1 << v["kind"]
        got = ctx.count(a, b, kinds)
        for v in vs:
            assert got[v["kind"]] == v["count"], (v, got)


def test_benchmark_workloads(ctx, ref_counts):
    """pi(1e9); [1e15, 1e15+1e11]; [0, 1e11]; [2^64-2^34, 2^64-1] ... all six
    counts each, against the reference CPU library."""
    for row in ref_counts["bench"]:
        assert ctx.count(row["start"], row["stop"]) == row["counts"], row


def test_oracle_random_ranges(ctx, oracle):
    rng = random.Random(7)
    for base in [0, 10 ** 5, 10 ** 8, 10 ** 10, 10 ** 12, 2 ** 40]:
        for _ in range(10):
            a = base + rng.randrange(10 ** 6)
            b = a + rng.randrange(2 * 10 ** 6)
            assert ctx.count(a, b) == oracle.plain(a, b), (a, b)


CONFIGS = [
    dict(seg_bytes=4096, block=256),                        # many tiny segments
    dict(seg_bytes=8192, block=512, presieve=2),            # no pre-sieve
    dict(seg_bytes=16384, block=256, small_limit=64),       # no warp-cooperative tier
    dict(seg_bytes=16384, block=256, small_limit=100000),   # only warp-cooperative
    dict(seg_bytes=4096, block=256, big_limit=200, window_segments=3, bucket_lists=5),
    dict(seg_bytes=65536, block=1024, big_limit=1000, window_segments=7),
    dict(seg_bytes=4096, block=256, big_limit=300, window_segments=5),                     # many short windows
    dict(seg_bytes=16384, block=512, big_limit=500, bucket_lists=3),                       # few lists
    dict(seg_bytes=32768, block=512, ctas_per_sm=2),
    # segment size not a power of two: the fill's segment index by reciprocal
    dict(seg_bytes=12288, block=256, big_limit=300, window_segments=9),
    # thread walk with many wheel rotations per window: staggered starts,
    # wraps, rounds and flushes between rounds
    dict(seg_bytes=16384, block=1024, big_limit=2000, window_segments=64),
]


@pytest.mark.parametrize("cfg", CONFIGS, ids=[str(c) for c in CONFIGS])
def test_engine_configs(psg, oracle, ref_counts, cfg):
    """Segment sizes, block sizes, tier limits, bucket windows and list
    counts change the work split, never the result."""
    c = psg.Context(**cfg)
    try:
        rng = random.Random(11)
        ranges = [(0, 10 ** 6), (0, 1000), (999999900, 1000000231), (10 ** 12, 10 ** 12 + 10 ** 6)]
        ranges += [(x, x + rng.randrange(3 * 10 ** 5)) for x in
                   (rng.randrange(10 ** 13) for _ in range(6))]
        for a, b in ranges:
            assert c.count(a, b) == oracle.plain(a, b), (cfg, a, b)
        top = 2 ** 64 - 1
        row = [r for r in ref_counts["cases"] if r["start"] == top - 10 ** 6 and r["stop"] == top]
        got = c.count(top - 10 ** 6, top)
        for r in row:
            assert got[r["kind"]] == r["count"]
    finally:
        c.close()


def test_small_limit_per_range(psg, oracle, ctx):
    """By default the warp-cooperative tier ends at 4096, 2048 or 1024 as
    sqrt(stop) passes 2e6 and 8e6; ranges on both sides of each switch
    count the same as the oracle and as contexts with each limit fixed."""
    ranges = [(4 * 10 ** 12 - 10 ** 7, 4 * 10 ** 12 - 1), (4 * 10 ** 12, 4 * 10 ** 12 + 10 ** 7),
              (64 * 10 ** 12 - 10 ** 7, 64 * 10 ** 12 - 1), (64 * 10 ** 12, 64 * 10 ** 12 + 10 ** 7)]
    fixed = [psg.Context(small_limit=s) for s in (4096, 2048, 1024)]
    try:
        for a, b in ranges:
            want = oracle.plain(a, b)
            assert ctx.count(a, b) == want, (a, b)
            for c in fixed:
                assert c.count(a, b) == want, (a, b)
    finally:
        for c in fixed:
            c.close()


def test_contexts_with_different_layouts_coexist(psg, ctx):
    """Kernel shared-memory limits are per process, not per context: a
    context with small segments and windows, created and used after the
    default one, must not shrink them under the default context's launches
    (232 KB sieve, 204 KB bucket fill)."""
    a, b = 10 ** 15, 10 ** 15 + 10 ** 10
    before = ctx.count(a, b)
    with psg.Context(seg_bytes=16384, block=1024, big_limit=2000, window_segments=3) as small:
        assert small.count(10 ** 12, 10 ** 12 + 10 ** 8) == ctx.count(10 ** 12, 10 ** 12 + 10 ** 8)
        assert ctx.count(a, b) == before
        assert ctx.count_batch([(a, b, 63), (0, 10 ** 9, 63)]) == [before, ctx.count(0, 10 ** 9, 63)]


def test_additivity_full_size(ctx, ref_counts, psg):
    """Size-independent property at the benchmark size: the six counts of
    [1e15, 1e15+1e11] equal the sum over 5 shards cut at == 2 (mod 30)."""
    row = [r for r in ref_counts["bench"] if r["start"] == 10 ** 15 and r["stop"] == 10 ** 15 + 10 ** 11][0]
    total = [0] * 6
    for a, b in psg.split_range(row["start"], row["stop"], 5):
        total = [t + c for t, c in zip(total, ctx.count(a, b))]
    assert total == row["counts"]


def test_random_chunks_sum(psg):
    """The reference's chunked-count test (test/count_primes3.cpp:31-57):
    [1e12, 1e12+1e9] cut into seeded random chunks (any cut, not only at
    == 2 (mod 30), so primes only), each counted by a context with a
    different segment size and bucket window, sums to 36190991."""
    rng = random.Random(1234)
    a, b = 10 ** 12, 10 ** 12 + 10 ** 9
    cuts = sorted(rng.sample(range(a + 1, b), 40))
    bounds = [a] + cuts + [b + 1]
    configs = [dict(), dict(seg_bytes=16384, block=512, window_segments=7),
               dict(seg_bytes=65536, block=1024, big_limit=100000, window_segments=3)]
    ctxs = [psg.Context(**c) for c in configs]
    try:
        total = 0
        for i, (x, y) in enumerate(zip(bounds, bounds[1:])):
            total += ctxs[i % len(ctxs)].count(x, y - 1, 1)[0]
    finally:
        for c in ctxs:
            c.close()
    assert total == 36190991


def test_empty_and_single(ctx):
    assert ctx.count(10, 5) == [0] * 6
    assert ctx.count(0, 0) == [0] * 6
    assert ctx.count(2, 2) == [1, 0, 0, 0, 0, 0]
    assert ctx.count(7, 7) == [1, 0, 0, 0, 0, 0]
    assert ctx.count(2 ** 64 - 1, 2 ** 64 - 1) == [0] * 6
    assert ctx.count(2 ** 64 - 59, 2 ** 64 - 59)[0] == 1      # largest 64-bit prime
    assert ctx.count(0, 100, 0) == [0] * 6                    # no kinds requested
    assert ctx.count(0, 100, 1 << 2) == [0, 0, 8, 0, 0, 0]    # one kind only


def test_batch_matches_single(ctx):
    ranges = [(0, 10 ** 7, 63), (10 ** 12, 10 ** 12 + 10 ** 7, 1), (5, 4, 63), (2 ** 64 - 10 ** 5, 2 ** 64 - 1, 6)]
    got = ctx.count_batch(ranges)
    for (a, b, k), g in zip(ranges, got):
        assert g == ctx.count(a, b, k)


def test_count_async_accumulates(ctx, psg):
    import torch
    dev = torch.zeros(6, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    ctx.count_async(0, 10 ** 8, 63, dev.data_ptr(), stream.cuda_stream)
    ctx.count_async(0, 10 ** 8, 63, dev.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    assert [x // 2 for x in dev.tolist()] == ctx.count(0, 10 ** 8)


@pytest.mark.parametrize("a,b,k", [
    (10 ** 15, 10 ** 15 + 10 ** 11, 1),            # bench workload: group-walk fill
    (2 ** 64 - 2 ** 34, 2 ** 64 - 1, 63),          # thread-walk fill, all six kinds
    (10 ** 18, 10 ** 18 + 10 ** 10, 1),
    (10 ** 13, 10 ** 13 + 3 * 10 ** 10, 63),
])
def test_count_async_first_call_exact(psg, a, b, k):
    """The asynchronous path has no overflow recount: on a fresh context (list
    capacities at their defaults) its first count over bucket windows must
    already be exact, i.e. no bucket list may overflow."""
    import torch
    with psg.Context() as c:
        dev = torch.zeros(6, dtype=torch.int64, device="cuda")
        c.count_async(a, b, k, dev.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        got = dev.tolist()
        want = c.count(a, b, k)
    assert got == want
    if (a, k) == (10 ** 15, 1):
        assert got[0] == 2895317534               # reference CPU library


def test_count_async_overflow_is_reported(psg):
    """With lists at a quarter of their estimated capacity the bucket fill
    drops entries. psg_count_async cannot recount, so psg_count_async_status
    must report PSG_ERR_OVERFLOW (9) -- also after a synchronous count on the
    same context, which resets only its own flag -- and, once the lists have
    grown, an asynchronous count is exact again and reports PSG_OK."""
    import torch
    a, b = 10 ** 15, 10 ** 15 + 10 ** 10
    stream = torch.cuda.current_stream().cuda_stream
    with psg.Context(list_capacity_pct=25) as c:
        dev = torch.zeros(6, dtype=torch.int64, device="cuda")
        c.count_async(a, b, 1, dev.data_ptr(), stream)
        want = c.count(a, b, 1)                  # recounts internally: exact
        with pytest.raises(psg.PsgError) as e:
            c.count_async_status()
        assert e.value.status == 9 and "overflow" in str(e.value)
        c.count_async_status()                   # the record was cleared
        for attempt in range(4):
            dev.zero_()
            c.count_async(a, b, 1, dev.data_ptr(), stream)
            try:
                c.count_async_status()
                break
            except psg.PsgError as err:
                assert err.status == 9
        else:
            pytest.fail("lists did not grow")
        torch.cuda.synchronize()
        assert dev.tolist() == want
    assert want[0] == 289531946                  # oracle: pi[1e15, 1e15+1e10]


def test_count_recounts_on_overflow(psg, ctx):
    """The synchronous path detects the overflow and recounts with grown
    lists: exact however small the lists start."""
    cases = [(10 ** 15, 10 ** 15 + 10 ** 10, 1), (2 ** 64 - 2 ** 33, 2 ** 64 - 1, 63)]
    with psg.Context(list_capacity_pct=20) as c:
        for a, b, k in cases:
            assert c.count(a, b, k) == ctx.count(a, b, k), (a, b, k)
        assert c.count_batch([(a, b, k) for a, b, k in cases]) == [ctx.count(a, b, k) for a, b, k in cases]


def test_device_prime_table(psg, oracle):
    """The sieving-prime table generated on the device up to 2^32: its
    length (the primes 59 < p < 2^32: pi(2^32) = 203280221 less the 17 primes
    <= 59), its first and last entries, its index at 1e9 (pi(1e9) =
    50847534) and seeded windows, against the oracle's primes."""
    with psg.Context() as c:
        top = 2 ** 64 - 1
        total, lo, hi, head = c.sieving_primes(top, 0, 2000)
        assert (lo, hi) == (59, 2 ** 32 - 1)
        assert total == 203280221 - 17
        assert head == oracle.primes(60, head[-1]) and len(head) == 2000
        _, _, _, tail = c.sieving_primes(top, total - 500, 1000)
        assert len(tail) == 500 and tail[-1] == 4294967291
        assert tail == oracle.primes(tail[0], 2 ** 32 - 1)
        _, _, _, at = c.sieving_primes(top, 50847534 - 17 - 1, 2)
        assert at == [999999937, 1000000007]
        rng = random.Random(7)
        for _ in range(12):
            i = rng.randrange(total - 20000)
            _, _, _, win = c.sieving_primes(top, i, 20000)
            assert win == oracle.primes(win[0], win[-1]), i


def test_c_api(psg, ctx):
    lib = psg.load()
    a, b = 10 ** 12, 10 ** 12 + 10 ** 8
    want = ctx.count(a, b)
    for k, name in enumerate(psg.KIND_NAMES):
        assert getattr(lib, "primesieve_count_" + name)(a, b) == want[k]
    out = (ctypes.c_uint64 * 6)()
    assert lib.primesieve_count_all(ctypes.c_uint64(a), ctypes.c_uint64(b), out) == 0
    assert list(out) == want
    lib.primesieve_get_max_stop.restype = ctypes.c_uint64
    assert lib.primesieve_get_max_stop() == 2 ** 64 - 1


def test_cpp_api(tmp_path, ctx):
    exe = tmp_path / "api_check"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(REPO, "include"),
                    os.path.join(REPO, "tests", "cpp", "api_check.cpp"), "-o", str(exe),
                    "-L", os.path.join(PKG_DIR, "lib"), "-lprimesieve_gpu",
                    "-Wl,-rpath," + os.path.join(PKG_DIR, "lib")], check=True)
    a, b = 10 ** 9, 10 ** 9 + 10 ** 7
    out = subprocess.run([str(exe), str(a), str(b)], capture_output=True, text=True, check=True).stdout
    lines = dict(l.split(" ", 1) for l in out.strip().split("\n"))
    want = " ".join(str(x) for x in ctx.count(a, b))
    assert lines["count"] == want and lines["gpu"] == want and lines["all"] == want
    assert lines["knobs"] == f"1 {ctx.count(a, b)[0]}"
    assert lines["worthwhile"] == "1 0"


def cli(*args):
    return subprocess.run([os.path.join(PKG_DIR, "bin", "primesieve"), *args], capture_output=True, text=True)


def test_cli(ref_counts):
    r = cli("1e12", "1e12+1e9", "-c123456", "--gpu")
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().split("\n")
    assert lines[0].startswith("GPU = ") and lines[1].startswith("Seconds: ")
    assert lines[2:] == ["Primes: 36190991", "Twin primes: 1730012", "Prime triplets: 271316",
                         "Prime quadruplets: 7171", "Prime quintuplets: 1259", "Prime sextuplets: 42"]
    r = cli("1e9", "--count", "--gpu", "-q")
    assert r.returncode == 0 and r.stdout == "50847534\n"
    r = cli("1e10", "--dist=1e3", "-c12", "-q")
    assert r.stdout == "Primes: 44\nTwin primes: 2\n"
    r = cli("100", "10", "-q")
    assert r.stdout == "0\n"
    r = cli("18446744056529682432", "18446744073709551615", "-c6", "-q", "--time")
    assert r.returncode == 0 and r.stdout.split("\n")[1] == "39"

"""CPU: pin the oracle (C restatement of the reference's counting path)
against the reference's own golden vectors and against counts computed by
the reference's CPU library, and check its two counters against each other."""
import random

import pytest

KINDS = 6


def small_enough(v, max_len=10 ** 9 + 1, max_stop=2 * 10 ** 12):
    return v["stop"] - v["start"] <= max_len and v["stop"] <= max_stop


def test_reference_vectors_plain(oracle, ref_vectors):
    """Known-answer values from the reference's tests (count_primes1.cpp,
    count_<kind>.cpp, src/app/test.cpp, test/gpu_count.cpp) that the plain
    byte-array sieve finishes in seconds."""
    # group by range so that all kinds come from one pass
    by_range = {}
    for v in ref_vectors:
        if small_enough(v):
            by_range.setdefault((v["start"], v["stop"]), []).append(v)
    assert len(by_range) >= 10
    for (a, b), vs in sorted(by_range.items()):
        got = oracle.plain(a, b)
        for v in vs:
            assert got[v["kind"]] == v["count"], (v, got)


def test_reference_computed_cases(oracle, ref_counts):
    """Every case of the reference-computed table (test/gpu_count.cpp case
    list, 2^64 edges, seeded random ranges) on both oracle counters."""
    cases = ref_counts["cases"]
    by_range = {}
    for c in cases:
        by_range.setdefault((c["start"], c["stop"]), []).append(c)
    checked = 0
    for (a, b), cs in by_range.items():
        # plain sieve up to 3.1e6 long ranges; one wide wheel segment beyond
        got = oracle.plain(a, b) if b - a <= 31 * 10 ** 5 else oracle.wheel(a, b, 400000)
        for c in cs:
            assert got[c["kind"]] == c["count"], (c, got)
            checked += 1
        if b - a <= 10 ** 5 and b < 2 ** 40:
            w = oracle.wheel(a, b, 977)
            for c in cs:
                assert w[c["kind"]] == c["count"], (c, w)
    assert checked == len(cases)


@pytest.mark.parametrize("sieve_bytes", [32, 977, 4096])
def test_wheel_vs_plain_random(oracle, sieve_bytes):
    """The wheel-30 restatement with tiny segments (forcing many segment and
    byte boundaries) agrees with the plain sieve (reference
    tools/ref_sieve.cpp:118-142 does the same with xorshift ranges)."""
    rng = random.Random(0x9E3779B97F4A7C15)
    for base in [0, 1000, 10 ** 6, 10 ** 9, 10 ** 11, 10 ** 13]:
        for _ in range(12):
            a = base + rng.randrange(100000)
            b = a + rng.randrange(60000)
            assert oracle.wheel(a, b, sieve_bytes) == oracle.plain(a, b), (a, b, sieve_bytes)


def test_ktuplet_tables(oracle):
    """Byte LUTs derived from the tuplet definitions equal the reference's
    bitmask tables (src/CountPrintPrimes.cpp:33-41)."""
    masks = {1: [0x06, 0x18, 0xc0], 2: [0x07, 0x0e, 0x1c, 0x38], 3: [0x1e],
             4: [0x1f, 0x3e], 5: [0x3f]}
    for k, ms in masks.items():
        t = oracle.ktable(k)
        for x in range(256):
            assert t[x] == sum(1 for m in ms if x & m == m)
    assert oracle.ktable(0) == [bin(x).count("1") for x in range(256)]


def test_empty_and_tiny(oracle):
    assert oracle.plain(10, 5) == [0] * 6
    assert oracle.wheel(10, 5) == [0] * 6
    assert oracle.plain(0, 1) == [0] * 6
    assert oracle.plain(2, 2)[0] == 1
    assert oracle.plain(0, 17) == [7, 3, 3, 1, 1, 0]      # incl. (5,7,11,13,17)
    top = 2 ** 64 - 1
    assert oracle.plain(top, top) == [0] * 6               # 2^64-1 is composite


def test_batch_fixture_pinned(oracle):
    """The 4096-range fixture: its ranges regenerate from the documented RNG
    recipe, and its shortest rows (counts from the reference library) agree
    with the oracle."""
    import importlib.util
    import json
    import os
    from conftest import REPO
    golden = os.path.join(REPO, "tests", "golden")
    spec = importlib.util.spec_from_file_location("make_batch", os.path.join(golden, "make_batch.py"))
    mb = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mb)
    with open(os.path.join(golden, "batch4096.json")) as f:
        rows = json.load(f)["ranges"]
    assert [tuple(r[:3]) for r in rows] == mb.make_ranges(4096, 0)
    short = sorted(rows, key=lambda r: r[1] - r[0])[:40]
    for a, b, k, want in short:
        assert oracle.plain(a, b, 1 << k)[k] == want, (a, b, k)


def test_nth_prime_fixture_pinned(oracle):
    """nth_prime.json (made by the reference library): every case whose
    answer the plain oracle reaches quickly is a prime with exactly |n|
    primes between start and it (n = 0 counts as 1)."""
    import json
    import os
    from conftest import REPO
    with open(os.path.join(REPO, "tests", "golden", "nth_prime.json")) as f:
        data = json.load(f)
    checked = 0
    for n, start, p in data["nth"]:
        k = max(1, abs(n))
        lo, hi = (start + 1, p) if n >= 0 else (p, start - 1)
        if hi - lo > 3 * 10 ** 7 or p > 10 ** 13:
            continue
        assert oracle.plain(p, p, 1)[0] == 1, (n, start, p)
        assert oracle.plain(lo, hi, 1)[0] == k, (n, start, p)
        checked += 1
    assert checked >= 30

"""GPU: prime extraction (psg_generate_primes, primesieve_generate_primes,
the C++ templates, the CLI --print) and nth_prime (psg_nth_prime,
primesieve_nth_prime, the CLI --nth-prime) against the reference library's
answers (tests/golden/nth_prime.json), the oracle, and properties that hold
at any size (every value prime, count = the GPU count)."""
import ctypes
import json
import os
import subprocess

import pytest

from conftest import REPO, PKG_DIR

pytestmark = pytest.mark.gpu
M64 = (1 << 64) - 1

with open(os.path.join(REPO, "tests", "golden", "nth_prime.json")) as _f:
    GOLD = json.load(_f)


def is_prime(n):
    """Deterministic Miller-Rabin for n < 3.3e24."""
    if n < 2:
        return False
    small = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)
    for q in small:
        if n % q == 0:
            return n == q
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in small:
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def test_generate_vs_oracle(ctx, oracle):
    for a, b in [(0, 0), (0, 2), (0, 100), (5, 5), (7, 7), (100, 10), (0, 10 ** 6),
                 (999_000, 2_000_000), (10 ** 8, 10 ** 8 + 10 ** 6)]:
        got = ctx.generate_primes(a, b)
        want = oracle.primes(a, b)
        assert got == want, (a, b)


@pytest.mark.parametrize("row", GOLD["gen"], ids=[f"{r[0]}-{r[1]}" for r in GOLD["gen"]])
def test_generate_vs_reference(ctx, row):
    a, b, n, s, x = row
    got = ctx.generate_primes(a, b)
    assert len(got) == n
    assert sum(got) % (1 << 64) == s
    acc = 0
    for v in got:
        acc ^= v
    assert acc == x


def test_generate_properties_large(ctx):
    for a, b in [(10 ** 15, 10 ** 15 + 3 * 10 ** 7), (M64 - 3 * 10 ** 7, M64), (10 ** 12, 10 ** 12 + 10 ** 9)]:
        got = ctx.generate_primes(a, b)
        assert len(got) == ctx.count(a, b, 1)[0]
        assert all(x < y for x, y in zip(got, got[1:]))
        assert got[0] >= a and got[-1] <= b
        step = max(1, len(got) // 2000)
        assert all(is_prime(v) for v in got[::step])


@pytest.mark.parametrize("row", GOLD["nth"], ids=[f"{r[0]}@{r[1]}" for r in GOLD["nth"]])
def test_nth_prime_vs_reference(ctx, row):
    n, start, p = row
    assert ctx.nth_prime(n, start) == p


def test_nth_prime_errors(ctx, psg):
    for n, start in GOLD["errors"]:
        with pytest.raises(psg.PsgError):
            ctx.nth_prime(n, start)
    with pytest.raises(psg.PsgError) as e:
        ctx.nth_prime(-4, 3)
    assert "abs(n) must be < start" in str(e.value)
    with pytest.raises(psg.PsgError) as e:
        ctx.nth_prime(-1, 2)
    assert "nth prime < 2 is impossible" in str(e.value)
    with pytest.raises(psg.PsgError) as e:
        ctx.nth_prime(1, 18446744073709551557)
    assert "cannot generate primes > 2^64" in str(e.value)


def test_nth_prime_walk(ctx):
    # consecutive nth_prime calls walk the primes of a window both ways
    primes = ctx.generate_primes(10 ** 14, 10 ** 14 + 20000)
    for i, p in enumerate(primes[:50]):
        assert ctx.nth_prime(i + 1, 10 ** 14 - 1) == p
    for i, p in enumerate(reversed(primes[-50:])):
        assert ctx.nth_prime(-(i + 1), 10 ** 14 + 20001) == p


def test_c_api_generate_and_nth(psg, ctx):
    lib = psg.load()
    f = lib.primesieve_nth_prime
    f.argtypes, f.restype = [ctypes.c_int64, ctypes.c_uint64], ctypes.c_uint64
    assert f(10 ** 6, 0) == 15485863
    assert f(-1, 2) == M64                                  # error convention
    g = lib.primesieve_generate_primes
    g.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_size_t), ctypes.c_int]
    g.restype = ctypes.c_void_p
    lib.primesieve_free.argtypes = [ctypes.c_void_p]
    size = ctypes.c_size_t(0)
    ptr = g(100, 200, ctypes.byref(size), 13)               # UINT64_PRIMES
    vals = list((ctypes.c_uint64 * size.value).from_address(ptr))
    lib.primesieve_free(ptr)
    assert vals == [p for p in range(100, 201) if is_prime(p)]
    ptr = g(0, 100, ctypes.byref(size), 8)                  # INT16_PRIMES
    assert size.value == 25 and list((ctypes.c_int16 * 25).from_address(ptr))[-1] == 97
    lib.primesieve_free(ptr)
    ptr = g(0, 70000, ctypes.byref(size), 8)                # too narrow for int16_t
    assert not ptr and size.value == 0
    gn = lib.primesieve_generate_n_primes
    gn.argtypes, gn.restype = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int], ctypes.c_void_p
    ptr = gn(5, 1000, 13)
    assert list((ctypes.c_uint64 * 5).from_address(ptr)) == [1009, 1013, 1019, 1021, 1031]
    lib.primesieve_free(ptr)


def cli(*args):
    return subprocess.run([os.path.join(PKG_DIR, "bin", "primesieve"), *args], capture_output=True, text=True)


def test_cli_nth_prime_and_print():
    r = cli("1000000", "--nth-prime", "-q")
    assert r.returncode == 0 and r.stdout.strip() == "15485863"
    r = cli("10", "1000000000000", "-n")
    assert r.returncode == 0 and "Nth prime: 1000000000193" in r.stdout     # reference CLI
    r = cli("90", "120", "--print", "-q")
    assert r.returncode == 0 and r.stdout.split() == ["97", "101", "103", "107", "109", "113"]

"""CPU: the C-ABI library loads, exports every function that include/*.h
declares, and fails loudly (no silent CPU fallback) when there is no GPU."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import REPO, PKG_DIR

HEADERS = ["include/psgpu.h", "include/primesieve.h"]


def declared_functions(path):
    text = open(os.path.join(REPO, path)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n.startswith(("psg_", "primesieve_"))))


def gpu_count(psg):
    return psg.device_count()


def test_symbols_exported(psg):
    lib = psg.load()
    names = []
    for h in HEADERS:
        names += declared_functions(h)
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/ but not exported"
    for n in psg.PSG_SYMBOLS:
        assert n in names


def test_cpp_symbols_exported():
    out = subprocess.run(["nm", "-D", "-C", os.path.join(PKG_DIR, "lib", "libprimesieve_gpu.so")],
                         capture_output=True, text=True, check=True).stdout
    for fn in ["primesieve::count_primes", "primesieve::count_sextuplets", "primesieve::count_all",
               "primesieve::gpu_count_primes", "primesieve::gpu_try_count", "primesieve::set_gpu_sieve_size",
               "primesieve::gpu_devices", "primesieve::gpu_worthwhile", "primesieve::set_gpu_presieve"]:
        assert re.search(re.escape(fn) + r"(\[abi:cxx11\])?\(", out), fn


def test_status_strings(psg):
    lib = psg.load()
    for s in range(0, 9):
        assert lib.psg_status_string(s)
    assert lib.psg_version().startswith(b"primesieve-b200")


def test_no_device_fails_loudly(psg):
    if gpu_count(psg) > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(psg.PsgError) as e:
        psg.Context()
    assert e.value.status == 2
    lib = ctypes.CDLL(psg.LIB_PATH, use_errno=True)
    lib.primesieve_count_primes.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
    lib.primesieve_count_primes.restype = ctypes.c_uint64
    ctypes.set_errno(0)
    assert lib.primesieve_count_primes(0, 100) == psg.PRIMESIEVE_ERROR
    assert ctypes.get_errno() == 33          # EDOM


def test_null_handles_are_argument_errors(psg):
    """Every psg_* entry point that takes a context or server turns a NULL
    handle into PSG_ERR_ARG (1) with a message; none crashes or throws
    (no GPU needed: the check comes before any device work)."""
    lib = psg.load()
    u64 = ctypes.c_uint64
    out6 = (u64 * 6)()
    rid = u64(0)
    d = ctypes.c_double(0)
    n = ctypes.c_size_t(0)
    calls = {
        "psg_count": lambda: lib.psg_count(None, 0, 100, 63, out6),
        "psg_count_async": lambda: lib.psg_count_async(None, 0, 100, 63, out6, None),
        "psg_count_batch": lambda: lib.psg_count_batch(None, None, 0, None),
        "psg_nth_prime": lambda: lib.psg_nth_prime(None, 1, 0, ctypes.byref(rid)),
        "psg_generate_primes": lambda: lib.psg_generate_primes(None, 0, 100, None, 0, ctypes.byref(n)),
        "psg_prepare": lambda: lib.psg_prepare(None, 100),
        "psg_set_profiling": lambda: lib.psg_set_profiling(None, 1),
        "psg_reset_kernel_stats": lambda: lib.psg_reset_kernel_stats(None),
        "psg_bucket_entries": lambda: lib.psg_bucket_entries(None, ctypes.byref(rid), 0),
        "psg_server_start": lambda: lib.psg_server_start(None, None, ctypes.byref(ctypes.c_void_p())),
        "psg_server_submit": lambda: lib.psg_server_submit(None, 0, 100, 1, ctypes.byref(rid)),
        "psg_server_wait": lambda: lib.psg_server_wait(None, 1, out6, ctypes.byref(d)),
        "psg_server_replay": lambda: lib.psg_server_replay(None, None, None, 0, None, None),
    }
    for name, call in calls.items():
        assert call() == 1, name
        assert lib.psg_last_error(), name
    lib.psg_server_stop(None)          # no-ops
    lib.psg_destroy(None)


def cli(*args):
    return subprocess.run([os.path.join(PKG_DIR, "bin", "primesieve"), *args], capture_output=True, text=True)


def test_cli_options_cpu(psg):
    r = cli("--help")
    assert r.returncode == 0 and "Usage: primesieve" in r.stdout
    r = cli("100", "-c7")
    assert r.returncode == 1 and "invalid option '-c7'" in r.stderr
    r = cli("2^64")
    assert r.returncode == 1 and "overflow" in r.stderr
    r = cli("10", "--print=2")
    assert r.returncode == 1 and "not supported" in r.stderr
    r = cli("100", "--stress-test")
    assert r.returncode == 1 and "not supported" in r.stderr
    r = cli("--bogus")
    assert r.returncode == 1 and "unrecognized option" in r.stderr
    r = cli("--version")
    assert r.returncode == 0 and "12.16" in r.stdout
    if gpu_count(psg) == 0:
        r = cli("1e9", "--count", "--gpu")
        assert r.returncode == 1 and "GPU" in r.stderr


def test_split_range(psg, oracle):
    """Shard boundaries are == 2 (mod 30): no k-tuplet is split, so shard
    counts add up exactly (reference src/ParallelSieve.cpp:122-133)."""
    for a, b, n in [(0, 10 ** 6, 3), (12345, 987654, 7), (5, 1000, 4), (10 ** 12, 10 ** 12 + 10 ** 6, 5), (0, 40, 8)]:
        parts = psg.split_range(a, b, n)
        assert parts[0][0] == a and parts[-1][1] == b
        for (x0, x1), (y0, y1) in zip(parts, parts[1:]):
            assert y0 == x1 + 1 and y0 % 30 == 2
        total = [0] * 6
        for x0, x1 in parts:
            total = [t + c for t, c in zip(total, oracle.plain(x0, x1))]
        assert total == oracle.plain(a, b)


def test_shard_of_covers_range(psg):
    """One process per GPU: the ranks' shards are disjoint, consecutive, cut
    at == 2 (mod 30), and together cover [start, stop] exactly; ranks past
    the last non-empty shard get None."""
    import random
    rnd = random.Random(3)
    cases = [(0, 10, 4), (5, 5, 3), (0, 89, 8), (2 ** 64 - 1000, 2 ** 64 - 1, 5)]
    cases += [(a, a + rnd.randrange(10 ** 7), rnd.randrange(1, 9)) for a in (rnd.randrange(10 ** 15) for _ in range(50))]
    for a, b, world in cases:
        shards = [psg.shard_of(a, b, r, world) for r in range(world)]
        got = [s for s in shards if s is not None]
        assert shards[:len(got)] == got                     # None only at the end
        assert got[0][0] == a and got[-1][1] == b
        for (x0, x1), (y0, y1) in zip(got, got[1:]):
            assert x0 <= x1 and y0 == x1 + 1 and y0 % 30 == 2


def test_serving_workload_stream(psg):
    """The seed-1 serving stream is reproducible and has the stated shape:
    Poisson arrivals at the rate, log-uniform starts and lengths, one kind per
    request, stops clamped to 2^64 - 1."""
    reqs, arr = psg.serving_workload(3000, 500.0)
    assert (reqs, arr) == psg.serving_workload(3000, 500.0)
    assert psg.serving_workload(50, 500.0, seed=2)[0] != reqs[:50]
    assert all(t1 > t0 for t0, t1 in zip(arr, arr[1:]))
    assert abs(arr[-1] / len(arr) - 1.0 / 500.0) < 0.1 / 500.0     # mean gap within 10%
    for a, b, k in reqs:
        assert 10 ** 6 <= a <= 1.8e19 and a <= b <= 2 ** 64 - 1
        assert b - a + 1 <= 2 ** 36 and (b - a + 1 >= 2 ** 12 or b == 2 ** 64 - 1)
        assert k in (1, 2, 4, 8, 16, 32)
    assert len({k for _, _, k in reqs}) == 6

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

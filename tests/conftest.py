"""Shared fixtures: the engine binding (C ABI via ctypes), the oracle (the
C restatement of the reference's counting path, test-only) and the golden
fixtures."""
import ctypes
import importlib.util
import json
import os
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(REPO, "primesieve-gpu_b200")
GOLDEN = os.path.join(REPO, "tests", "golden")
ORACLE_DIR = os.path.join(REPO, "oracle")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu)")


def load_package():
    spec = importlib.util.spec_from_file_location("primesieve_gpu_b200", os.path.join(PKG_DIR, "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def ensure_built():
    """Build the engine and the oracle if their shared objects are missing."""
    if not os.path.exists(os.path.join(PKG_DIR, "lib", "libprimesieve_gpu.so")) or \
            not os.path.exists(os.path.join(PKG_DIR, "bin", "primesieve")):
        subprocess.run(["make", "-C", PKG_DIR, "-j8"], check=True, capture_output=True)
    if not os.path.exists(os.path.join(ORACLE_DIR, "liboracle.so")):
        subprocess.run(["make", "-C", ORACLE_DIR], check=True, capture_output=True)


class Oracle:
    """ctypes wrapper of oracle/liboracle.so (the checker, never the product)."""

    def __init__(self):
        self.lib = ctypes.CDLL(os.path.join(ORACLE_DIR, "liboracle.so"))
        self.lib.oracle_count_plain.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32,
                                                ctypes.POINTER(ctypes.c_uint64)]
        self.lib.oracle_count_wheel.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32,
                                                ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64)]
        self.lib.oracle_ktuplet_table.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_uint8)]
        self.lib.oracle_primes_u32.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32),
                                               ctypes.c_size_t]
        self.lib.oracle_primes_u32.restype = ctypes.c_int64

    def plain(self, a, b, kinds=0x3F):
        out = (ctypes.c_uint64 * 6)()
        assert self.lib.oracle_count_plain(a, b, kinds, out) == 0
        return list(out)

    def primes(self, lo, hi):
        """The primes in [lo, hi], hi < 2^32."""
        if hi < lo:
            return []
        cap = int((hi - lo) / 2) + 16
        out = (ctypes.c_uint32 * cap)()
        n = self.lib.oracle_primes_u32(lo, hi, out, cap)
        assert n >= 0
        return list(out[:n])

    def wheel(self, a, b, sieve_bytes=4096, kinds=0x3F):
        out = (ctypes.c_uint64 * 6)()
        assert self.lib.oracle_count_wheel(a, b, sieve_bytes, kinds, out) == 0
        return list(out)

    def ktable(self, kind):
        t = (ctypes.c_uint8 * 256)()
        self.lib.oracle_ktuplet_table(kind, t)
        return list(t)


@pytest.fixture(scope="session")
def psg():
    ensure_built()
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    ensure_built()
    return Oracle()


@pytest.fixture(scope="session")
def ctx(psg):
    c = psg.Context()
    yield c
    c.close()


@pytest.fixture(scope="session")
def ref_vectors():
    with open(os.path.join(GOLDEN, "reference_vectors.json")) as f:
        return json.load(f)["vectors"]


@pytest.fixture(scope="session")
def ref_counts():
    with open(os.path.join(GOLDEN, "ref_counts.json")) as f:
        return json.load(f)

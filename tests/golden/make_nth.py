#!/usr/bin/env python3
"""nth_prime and prime-generation golden data from the reference's CPU
library (oracle/_ref/libprimesieve_ref.so, built by `make -C oracle ref`).

  nth   : [n, start, prime] for a spread of n (both signs) and starts up to
          near 2^64, plus the edge cases of test/nth_prime2.cpp
  errors: [n, start] the reference rejects (PRIMESIEVE_ERROR, errno EDOM)
  gen   : [start, stop, count, sum mod 2^64, xor] of primesieve_generate_primes
          (UINT64_PRIMES) for ranges up to 2e6 integers

Usage: python tests/golden/make_nth.py   (writes tests/golden/nth_prime.json)
"""
import ctypes
import json
import os
import random

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
UINT64_PRIMES = 13
M64 = (1 << 64) - 1


def main():
    lib = ctypes.CDLL(os.path.join(REPO, "oracle", "_ref", "libprimesieve_ref.so"), use_errno=True)
    nth = lib.primesieve_nth_prime
    nth.argtypes, nth.restype = [ctypes.c_int64, ctypes.c_uint64], ctypes.c_uint64
    gen = lib.primesieve_generate_primes
    gen.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_size_t), ctypes.c_int]
    gen.restype = ctypes.c_void_p
    free = lib.primesieve_free
    free.argtypes = [ctypes.c_void_p]

    rnd = random.Random(2)
    cases = [(1, 1), (1, 2), (-1, 102), (-1, 101), (-9592, 100000), (-9591, 100000),   # test/nth_prime2.cpp
             (0, 0), (0, 7), (0, 8), (1, 0), (-1, 3), (10 ** 6, 0), (10 ** 8, 0), (10 ** 9, 0),
             (-1, M64), (1, M64 - 59), (-10 ** 6, 10 ** 12), (-(10 ** 8), 10 ** 12)]
    for e in (9, 12, 15, 18):
        for n in (1, 2, 100, 10 ** 5, 10 ** 7, -1, -1000, -(10 ** 6)):
            cases.append((n, 10 ** e + rnd.randrange(10 ** (e - 3))))
    for _ in range(16):
        cases.append((rnd.choice([1, -1]) * rnd.randrange(1, 10 ** 6), rnd.randrange(10 ** 7, 10 ** 13)))
    for n in (1, 5, -1, -5, -1000):
        cases.append((n, M64 - rnd.randrange(10 ** 6)))
    nth_rows, err_rows = [], []
    for n, s in cases:
        ctypes.set_errno(0)
        p = nth(n, s)
        if p == M64 and ctypes.get_errno() != 0:
            err_rows.append([n, s])
        else:
            nth_rows.append([n, s, p])
    for n, s in [(-1, 2), (1, 18446744073709551557), (-4, 3), (0, 18446744073709551557), (2, M64 - 60)]:
        ctypes.set_errno(0)
        p = nth(n, s)
        assert p == M64 and ctypes.get_errno() != 0, (n, s)
        err_rows.append([n, s])

    gen_rows = []
    for a, b in [(0, 10 ** 6), (10 ** 9, 10 ** 9 + 10 ** 6), (2 ** 32 - 10 ** 6, 2 ** 32 + 10 ** 6),
                 (10 ** 15, 10 ** 15 + 2 * 10 ** 6), (10 ** 18, 10 ** 18 + 10 ** 6), (M64 - 10 ** 6, M64),
                 (0, 100), (5, 5), (100, 10)]:
        size = ctypes.c_size_t(0)
        ptr = gen(a, b, ctypes.byref(size), UINT64_PRIMES)
        arr = (ctypes.c_uint64 * size.value).from_address(ptr) if size.value else []
        s, x = 0, 0
        for v in arr:
            s = (s + v) & M64
            x ^= v
        gen_rows.append([a, b, size.value, s, x])
        if ptr:
            free(ptr)
    with open(os.path.join(HERE, "nth_prime.json"), "w") as f:
        json.dump({"note": "computed with the reference CPU library (oracle/_ref)",
                   "nth": nth_rows, "errors": err_rows, "gen": gen_rows}, f, indent=0)
    print(len(nth_rows), "nth", len(err_rows), "errors", len(gen_rows), "gen")


if __name__ == "__main__":
    main()

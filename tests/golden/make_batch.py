#!/usr/bin/env python3
"""The batched workload: 4096 ranges, seed 0, and their counts from the
reference's CPU library (oracle/_ref/libprimesieve_ref.so).

RNG: numpy.random.default_rng(0) (PCG64), drawn in this order per range:
  start  = floor(10 ** U(6, 16))            (log-uniform in [1e6, 1e16])
  length = floor(2 ** U(16, 34))            (log-uniform in [2^16, 2^34])
  kind   = integers(0, 3)                   (0 primes, 1 twins, 2 triplets)
The range is [start, start + length - 1] (length integers, inclusive).

Usage: python tests/golden/make_batch.py [--n 4096] [--seed 0]
Writes tests/golden/batch4096.json.
"""
import argparse
import ctypes
import json
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
KINDS = ["primes", "twins", "triplets"]


def make_ranges(n=4096, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        start = int(np.floor(10.0 ** rng.uniform(6.0, 16.0)))
        length = int(np.floor(2.0 ** rng.uniform(16.0, 34.0)))
        kind = int(rng.integers(0, 3))
        out.append((start, start + length - 1, kind))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--lib", default=os.path.join(REPO, "oracle", "_ref", "libprimesieve_ref.so"))
    args = ap.parse_args()
    ranges = make_ranges(args.n, args.seed)
    lib = ctypes.CDLL(args.lib)
    fns = []
    for k in KINDS:
        f = getattr(lib, "primesieve_count_" + k)
        f.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        f.restype = ctypes.c_uint64
        fns.append(f)
    t = time.time()
    rows = []
    for i, (a, b, k) in enumerate(ranges):
        rows.append([a, b, k, int(fns[k](a, b))])
        if i % 256 == 0:
            print(i, time.time() - t, flush=True)
    total = sum(b - a + 1 for a, b, _ in ranges)
    with open(os.path.join(HERE, f"batch{args.n}.json"), "w") as f:
        json.dump({"note": "seeded batched workload; counts from the reference CPU library",
                   "rng": "numpy default_rng(%d): start=floor(10**U(6,16)), length=floor(2**U(16,34)), "
                          "kind=integers(0,3); range [start, start+length-1]" % args.seed,
                   "integers": total, "ranges": rows}, f)
    print("done", total, time.time() - t)


if __name__ == "__main__":
    main()

#!/usr/bin/env python3
"""Generate the golden fixtures under tests/golden/ (run in the build
container, where the reference sources exist; the GPU box only reads the
committed JSON).

1. reference_vectors.json -- every known-answer value the reference's own
   tests hold for the counting path, parsed from the reference sources:
     test/count_primes1.cpp, test/count_primes2.cpp, test/count_primes3.cpp,
     test/count_{twins,triplets,quadruplets,quintuplets,sextuplets}.cpp,
     src/app/test.cpp (countSmallPrimes, countPrimeKTuplets,
     countLargePrimes, countPrimesRandom), src/app/stressTest.cpp
     (primeCounts_1e13 / primeCounts_1e19 windows), test/gpu_count.cpp
     (known pi values).
2. ref_counts.json -- counts computed by the reference's own CPU library
   (oracle/_ref/libprimesieve_ref.so, built from the reference sources by
   oracle/Makefile.ref) for the case list of test/gpu_count.cpp:86-113, the
   sizes the benchmark runs, edge ranges near 2^64 and seeded random ranges.

Usage: python tests/golden/make_golden.py --ref <reference source tree>
"""
import argparse
import ctypes
import json
import os
import random
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
KINDS = ["primes", "twins", "triplets", "quadruplets", "quintuplets", "sextuplets"]


def src_lines(ref, rel):
    with open(os.path.join(ref, rel)) as f:
        return f.read().split("\n")


def vec(start, stop, kind, count, rel, line):
    return {"start": start, "stop": stop, "kind": kind, "count": count,
            "source": f"{rel}:{line}"}


def parse_reference(ref):
    out = []
    # count_primes1.cpp: pi(10^k), k = 1..9
    rel = "test/count_primes1.cpp"
    for i, l in enumerate(src_lines(ref, rel), 1):
        m = re.match(r"\s*(\d+),?\s*//\s*pi\(10\^(\d+)\)", l)
        if m:
            out.append(vec(0, 10 ** int(m.group(2)), 0, int(m.group(1)), rel, i))
    # count_primes2.cpp: pi[10^k, 10^k+10^8]
    rel = "test/count_primes2.cpp"
    for i, l in enumerate(src_lines(ref, rel), 1):
        m = re.match(r"\s*(\d+),?\s*//\s*pi\[10\^(\d+), 10\^\d+\+10\^8\]", l)
        if m:
            k = int(m.group(2))
            out.append(vec(10 ** k, 10 ** k + 10 ** 8, 0, int(m.group(1)), rel, i))
    # count_primes3.cpp: [1e12, 1e12+1e9] counted in random chunks
    rel = "test/count_primes3.cpp"
    for i, l in enumerate(src_lines(ref, rel), 1):
        m = re.search(r"check\(count == (\d+)\)", l)
        if m:
            out.append(vec(10 ** 12, 10 ** 12 + 10 ** 9, 0, int(m.group(1)), rel, i))
    # count_<kind>.cpp: [1e12, 1e12+1e9]
    for k in range(1, 6):
        rel = f"test/count_{KINDS[k]}.cpp"
        for i, l in enumerate(src_lines(ref, rel), 1):
            m = re.search(r"check\(count == (\d+)\)", l)
            if m:
                out.append(vec(10 ** 12, 10 ** 12 + 10 ** 9, k, int(m.group(1)), rel, i))
    # src/app/test.cpp
    rel = "src/app/test.cpp"
    for i, l in enumerate(src_lines(ref, rel), 1):
        m = re.match(r"\s*(\d+),?\s*//\s*PrimePi\(10\^(\d+)\)\s*$", l)
        if m:
            out.append(vec(0, 10 ** int(m.group(2)), 0, int(m.group(1)), rel, i))
        m = re.match(r"\s*(\d+),?\s*//\s*PrimePi(\d)\(10\^(\d+), 10\^\d+\+10\^10\)", l)
        if m:
            k = int(m.group(3))
            out.append(vec(10 ** k, 10 ** k + 10 ** 10, int(m.group(2)) - 1, int(m.group(1)), rel, i))
        m = re.match(r"\s*(\d+),?\s*//\s*PrimePi\(10\^(\d+), 10\^\d+\+10\^10\)", l)
        if m:
            k = int(m.group(2))
            out.append(vec(10 ** k, 10 ** k + 10 ** 10, 0, int(m.group(1)), rel, i))
        m = re.search(r"check\(count == (\d+)\)", l)
        if m:   # countPrimesRandom: [1e13, 1e13+1e10] in random chunks
            out.append(vec(10 ** 13, 10 ** 13 + 10 ** 10, 0, int(m.group(1)), rel, i))
    # src/app/stressTest.cpp: primeCounts_1e13 / _1e19, window i covers
    # [start + (i-1)*1e11, start + i*1e11]
    rel = "src/app/stressTest.cpp"
    lines = src_lines(ref, rel)
    cur = None
    idx = 0
    for i, l in enumerate(lines, 1):
        m = re.search(r"primeCounts_(1e\d+)\s*=", l)
        if m:
            cur, idx = m.group(1), 0
            continue
        if cur is None:
            continue
        m = re.search(r"Start number = \*/\s*(\d+)", l)
        if m:
            start0 = int(m.group(1))
            continue
        if "};" in l:
            cur = None
            continue
        for num in re.findall(r"(\d+)ull|(\d+)", l):
            v = int(num[0] or num[1])
            idx += 1
            a = start0 + (idx - 1) * 10 ** 11
            out.append(vec(a, a + 10 ** 11, 0, v, rel, i))
    # test/gpu_count.cpp: known pi values
    rel = "test/gpu_count.cpp"
    in_known = False
    for i, l in enumerate(src_lines(ref, rel), 1):
        if "known[]" in l:
            in_known = True
        m = re.match(r"\s*\{\s*(\d+)ull,\s*(\d+)ull\s*\}", l)
        if m and in_known:
            out.append(vec(0, int(m.group(1)), 0, int(m.group(2)), rel, i))
    return out


class RefLib:
    def __init__(self, path):
        self.lib = ctypes.CDLL(path)
        for k in KINDS:
            f = getattr(self.lib, "primesieve_count_" + k)
            f.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
            f.restype = ctypes.c_uint64

    def count(self, a, b, k):
        return getattr(self.lib, "primesieve_count_" + KINDS[k])(a, b)


def ref_cases():
    """Case list: test/gpu_count.cpp:86-113 plus benchmark sizes, 2^64 edges
    and seeded random ranges (seed 20261203, random.Random)."""
    cases = []
    small_stops = [0, 1, 2, 3, 5, 6, 7, 8, 30, 31, 49, 100, 163, 164, 241, 1000, 65537, 1000000]
    for k in range(6):
        for s in small_stops:
            cases.append((0, s, k, "test/gpu_count.cpp:88-92"))
    for base in range(0, 121):
        for ln in range(0, 71, 7):
            cases.append((base, base + ln, 0, "test/gpu_count.cpp:95-97"))
    for st in range(999999900, 1000000001):
        cases.append((st, st + 331, 0, "test/gpu_count.cpp:100-101"))
    for a, b in [(0, 10000000), (0, 100000000), (1000000000, 1100000000),
                 (999999999989, 1000000200000), (10000000000000, 10000010000000)]:
        for k in range(6):
            cases.append((a, b, k, "test/gpu_count.cpp:104-113"))
    top = 2 ** 64 - 1
    for a, b in [(top - 10 ** 6, top), (top - 2 ** 20, top - 2 ** 19), (top, top),
                 (top - 30, top), (2 ** 63 - 10 ** 6, 2 ** 63 + 10 ** 6),
                 (2 ** 32 - 10 ** 5, 2 ** 32 + 10 ** 5), (10 ** 19, 10 ** 19 + 10 ** 7)]:
        for k in range(6):
            cases.append((a, b, k, "edge"))
    rng = random.Random(20261203)
    for base in [0, 10 ** 3, 10 ** 6, 10 ** 9, 10 ** 11, 10 ** 13, 10 ** 15, 10 ** 17, 10 ** 18]:
        for _ in range(12):
            a = base + rng.randrange(0, 10 ** 6)
            b = a + rng.randrange(0, 3 * 10 ** 6)
            cases.append((a, b, rng.randrange(6), "random"))
    return cases


BENCH_CASES = [
    # (start, stop, kinds) -- the benchmark workloads, all six counts
    (0, 10 ** 9),
    (10 ** 15, 10 ** 15 + 10 ** 11),
    (0, 10 ** 11),
    (2 ** 64 - 2 ** 34, 2 ** 64 - 1),
    (10 ** 15, 10 ** 15 + 10 ** 10),
    (10 ** 12, 10 ** 12 + 10 ** 10),
]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference source tree")
    ap.add_argument("--lib", default=os.path.join(REPO, "oracle", "_ref", "libprimesieve_ref.so"))
    ap.add_argument("--skip-bench", action="store_true")
    args = ap.parse_args()

    vectors = parse_reference(args.ref)
    with open(os.path.join(HERE, "reference_vectors.json"), "w") as f:
        json.dump({"note": "known-answer values parsed from the reference's own tests",
                   "vectors": vectors}, f, indent=0)
    print(f"{len(vectors)} reference vectors")

    lib = RefLib(args.lib)
    rows = [{"start": a, "stop": b, "kind": k, "count": lib.count(a, b, k), "source": src}
            for a, b, k, src in ref_cases()]
    bench = []
    if not args.skip_bench:
        for a, b in BENCH_CASES:
            counts = [lib.count(a, b, k) for k in range(6)]
            bench.append({"start": a, "stop": b, "counts": counts})
            print("bench", a, b, counts, flush=True)
    with open(os.path.join(HERE, "ref_counts.json"), "w") as f:
        json.dump({"note": "counts from the reference CPU library (oracle/_ref)",
                   "cases": rows, "bench": bench}, f, indent=0)
    print(f"{len(rows)} reference-computed cases")


if __name__ == "__main__":
    sys.exit(main())

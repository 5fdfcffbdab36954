"""Python binding of the B200 prime / k-tuplet counting engine (ctypes).

The engine itself is C++/CUDA in ``lib/libprimesieve_gpu.so``; this module
only loads it and mirrors its C ABI (``include/psgpu.h``) and the
primesieve-compatible count API (``include/primesieve.h``). There is no
Python or CPU fallback: if the shared library or a CUDA device is missing,
every counting call raises.
"""
from __future__ import annotations

import ctypes
import os
import weakref
from typing import Iterable, List, Optional, Sequence, Tuple

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libprimesieve_gpu.so")
CLI_PATH = os.path.join(HERE, "bin", "primesieve")

PRIMES, TWINS, TRIPLETS, QUADRUPLETS, QUINTUPLETS, SEXTUPLETS = (1 << i for i in range(6))
ALL_KINDS = 0x3F
KIND_NAMES = ("primes", "twins", "triplets", "quadruplets", "quintuplets", "sextuplets")
PRIMESIEVE_ERROR = (1 << 64) - 1

# Exported symbols of the C ABI and of the primesieve-compatible C API.
PSG_SYMBOLS = (
    "psg_device_count", "psg_device_describe", "psg_init", "psg_destroy",
    "psg_get_config", "psg_describe", "psg_count", "psg_count_async",
    "psg_count_batch", "psg_prepare", "psg_last_error", "psg_status_string",
    "psg_set_profiling", "psg_kernel_stats", "psg_reset_kernel_stats", "psg_version",
    "psg_bucket_entries", "psg_measure_smem_atomic_rate", "psg_count_noalloc",
    "psg_server_start", "psg_server_submit", "psg_server_wait", "psg_server_replay",
    "psg_server_get_stats", "psg_server_stop", "psg_generate_primes", "psg_nth_prime",
    "psg_autotune_batch", "psg_count_async_status", "psg_server_inject_failure",
    "psg_sieving_primes",
)


class PsgError(RuntimeError):
    """A psg_* call returned a non-zero status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"psg status {status}: {message}")
        self.status = status


class PsgConfig(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in (
        "seg_bytes", "block", "ctas_per_sm", "small_limit", "big_limit",
        "window_segments", "bucket_lists", "presieve", "segments_per_launch", "list_capacity_pct")]


class PsgRange(ctypes.Structure):
    _fields_ = [("start", ctypes.c_uint64), ("stop", ctypes.c_uint64),
                ("kinds", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class PsgTuneClass(ctypes.Structure):
    _fields_ = [("range_class", ctypes.c_int32), ("sample_ranges", ctypes.c_uint32),
                ("sample_integers", ctypes.c_double), ("direct_budget", ctypes.c_double),
                ("big_limit", ctypes.c_uint32), ("stripe", ctypes.c_uint32),
                ("best_seconds", ctypes.c_double), ("default_seconds", ctypes.c_double),
                ("small_limit", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class PsgServerConfig(ctypes.Structure):
    _fields_ = [("max_slots", ctypes.c_uint32), ("step_segments", ctypes.c_uint32),
                ("prime_limit", ctypes.c_uint64), ("hbm_budget", ctypes.c_uint64)]


class PsgServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("refused", ctypes.c_uint64), ("steps", ctypes.c_uint64),
                ("bucket_requests", ctypes.c_uint64), ("batch_requests", ctypes.c_uint64),
                ("integers", ctypes.c_double), ("gpu_busy_seconds", ctypes.c_double)]


_lib: Optional[ctypes.CDLL] = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the engine library and declare the C signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: build it with `make -C primesieve-gpu_b200`")
    lib = ctypes.CDLL(path)
    u64, u32, i32, vp, sz = (ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int,
                             ctypes.c_void_p, ctypes.c_size_t)
    U64P = ctypes.POINTER(ctypes.c_uint64)
    lib.psg_device_count.argtypes = [ctypes.POINTER(ctypes.c_int)]
    lib.psg_device_describe.argtypes = [i32, ctypes.c_char_p, sz]
    lib.psg_init.argtypes = [i32, ctypes.POINTER(PsgConfig), ctypes.POINTER(vp)]
    lib.psg_destroy.argtypes = [vp]
    lib.psg_destroy.restype = None
    lib.psg_get_config.argtypes = [vp, ctypes.POINTER(PsgConfig)]
    lib.psg_describe.argtypes = [vp, ctypes.c_char_p, sz]
    lib.psg_count.argtypes = [vp, u64, u64, u32, U64P]
    lib.psg_count_async.argtypes = [vp, u64, u64, u32, vp, vp]
    lib.psg_count_async_status.argtypes = [vp]
    lib.psg_count_batch.argtypes = [vp, ctypes.POINTER(PsgRange), sz, U64P]
    lib.psg_prepare.argtypes = [vp, u64]
    lib.psg_sieving_primes.argtypes = [vp, u64, sz, ctypes.POINTER(ctypes.c_uint32), sz,
                                       ctypes.POINTER(sz), U64P, U64P]
    lib.psg_last_error.restype = ctypes.c_char_p
    lib.psg_status_string.restype = ctypes.c_char_p
    lib.psg_status_string.argtypes = [i32]
    lib.psg_set_profiling.argtypes = [vp, i32]
    lib.psg_kernel_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_char_p), U64P,
                                     ctypes.POINTER(ctypes.c_double), sz, ctypes.POINTER(sz)]
    lib.psg_reset_kernel_stats.argtypes = [vp]
    lib.psg_bucket_entries.argtypes = [vp, U64P, i32]
    lib.psg_measure_smem_atomic_rate.argtypes = [vp, ctypes.POINTER(ctypes.c_double),
                                                 ctypes.POINTER(ctypes.c_double)]
    lib.psg_count_noalloc.argtypes = [u64, u64, u32, vp, vp]
    lib.psg_version.restype = ctypes.c_char_p
    DP = ctypes.POINTER(ctypes.c_double)
    lib.psg_server_start.argtypes = [vp, ctypes.POINTER(PsgServerConfig), ctypes.POINTER(vp)]
    lib.psg_server_submit.argtypes = [vp, u64, u64, u32, U64P]
    lib.psg_server_wait.argtypes = [vp, u64, U64P, DP]
    lib.psg_server_replay.argtypes = [vp, ctypes.POINTER(PsgRange), DP, sz, U64P, DP]
    lib.psg_server_get_stats.argtypes = [vp, ctypes.POINTER(PsgServerStats)]
    lib.psg_server_inject_failure.argtypes = [vp, u32, i32]
    lib.psg_server_stop.argtypes = [vp]
    lib.psg_server_stop.restype = None
    lib.psg_generate_primes.argtypes = [vp, u64, u64, U64P, sz, ctypes.POINTER(sz)]
    lib.psg_nth_prime.argtypes = [vp, ctypes.c_int64, u64, U64P]
    lib.psg_autotune_batch.argtypes = [vp, ctypes.POINTER(PsgRange), sz, ctypes.c_double,
                                       ctypes.POINTER(PsgTuneClass), sz, ctypes.POINTER(sz)]
    for name in ("primes", "twins", "triplets", "quadruplets", "quintuplets", "sextuplets"):
        fn = getattr(lib, "primesieve_count_" + name, None)
        if fn is not None:
            fn.argtypes = [u64, u64]
            fn.restype = u64
    _lib = lib
    return lib


def _check(status: int) -> None:
    if status != 0:
        lib = load()
        raise PsgError(status, (lib.psg_last_error() or b"").decode(errors="replace"))


def device_count() -> int:
    n = ctypes.c_int(0)
    _check(load().psg_device_count(ctypes.byref(n)))
    return n.value


class Context:
    """One engine context on one CUDA device (``psg_init``)."""

    def __init__(self, device: int = -1, **config: int):
        lib = load()
        cfg = PsgConfig()
        for k, v in config.items():
            setattr(cfg, k, int(v))
        h = ctypes.c_void_p()
        _check(lib.psg_init(device, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._lib = lib
        self._servers = weakref.WeakSet()     # servers running on this context

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def close(self) -> None:
        """Stops the context's servers (their worker threads use the
        engine), then destroys the context."""
        for srv in list(getattr(self, "_servers", ())):
            srv.close()
        if self._h:
            self._lib.psg_destroy(self._h)
            self._h = None

    def __enter__(self) -> "Context":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self) -> None:  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def config(self) -> dict:
        c = PsgConfig()
        _check(self._lib.psg_get_config(self._h, ctypes.byref(c)))
        return {n: getattr(c, n) for n, _ in PsgConfig._fields_}

    def describe(self) -> str:
        buf = ctypes.create_string_buffer(512)
        _check(self._lib.psg_describe(self._h, buf, 512))
        return buf.value.decode()

    def count(self, start: int, stop: int, kinds: int = ALL_KINDS) -> List[int]:
        out = (ctypes.c_uint64 * 6)()
        _check(self._lib.psg_count(self._h, start, stop, kinds, out))
        return list(out)

    def count_async(self, start: int, stop: int, kinds: int, dev_counts_ptr: int,
                    stream_ptr: int = 0) -> None:
        _check(self._lib.psg_count_async(self._h, start, stop, kinds,
                                         ctypes.c_void_p(dev_counts_ptr),
                                         ctypes.c_void_p(stream_ptr or None)))

    def count_async_status(self) -> None:
        """Waits for the counts enqueued so far; raises PsgError (status 9,
        PSG_ERR_OVERFLOW) if an asynchronous count since the last call
        dropped bucket entries, so that its counts are too high."""
        _check(self._lib.psg_count_async_status(self._h))

    def count_batch(self, ranges: Sequence[Tuple[int, int, int]]) -> List[List[int]]:
        n = len(ranges)
        arr = (PsgRange * max(n, 1))()
        for i, (a, b, k) in enumerate(ranges):
            arr[i].start, arr[i].stop, arr[i].kinds = a, b, k
        out = (ctypes.c_uint64 * (6 * max(n, 1)))()
        _check(self._lib.psg_count_batch(self._h, arr, n, out))
        return [list(out[6 * i:6 * i + 6]) for i in range(n)]

    def generate_primes(self, start: int, stop: int) -> List[int]:
        """The primes in [start, stop] (psg_generate_primes)."""
        n = ctypes.c_size_t(0)
        cap = 0
        for _ in range(2):
            out = (ctypes.c_uint64 * max(cap, 1))()
            st = self._lib.psg_generate_primes(self._h, start, stop, out, cap, ctypes.byref(n))
            if st == 0:
                return list(out[:n.value])
            if st != 5:                        # PSG_ERR_LIMIT: capacity too small
                _check(st)
            cap = n.value
        _check(st)
        return []

    def nth_prime(self, n: int, start: int = 0) -> int:
        """primesieve's nth_prime(n, start) (psg_nth_prime)."""
        p = ctypes.c_uint64(0)
        _check(self._lib.psg_nth_prime(self._h, n, start, ctypes.byref(p)))
        return p.value

    def autotune_batch(self, ranges: Sequence[Tuple[int, int, int]], budget_seconds: float = 30.0) -> List[dict]:
        """Tune the batch parameters per range class on samples of `ranges`."""
        n = len(ranges)
        arr = (PsgRange * max(n, 1))()
        for i, (a, b, k) in enumerate(ranges):
            arr[i].start, arr[i].stop, arr[i].kinds = a, b, k
        cap = 32
        rep = (PsgTuneClass * cap)()
        cnt = ctypes.c_size_t(0)
        _check(self._lib.psg_autotune_batch(self._h, arr, n, budget_seconds, rep, cap, ctypes.byref(cnt)))
        return [{f: getattr(rep[i], f) for f, _ in PsgTuneClass._fields_} for i in range(min(cnt.value, cap))]

    def prepare(self, stop: int) -> None:
        _check(self._lib.psg_prepare(self._h, stop))

    def sieving_primes(self, stop: int, first: int = 0, n: int = 0):
        """The device sieving-prime table after prepare(stop): returns
        (length, lo_excl, hi_incl, entries [first, first + n))."""
        out = (ctypes.c_uint32 * max(n, 1))()
        total, lo, hi = ctypes.c_size_t(0), ctypes.c_uint64(0), ctypes.c_uint64(0)
        _check(self._lib.psg_sieving_primes(self._h, stop, first, out, n, ctypes.byref(total),
                                            ctypes.byref(lo), ctypes.byref(hi)))
        m = max(0, min(n, total.value - first))
        return total.value, lo.value, hi.value, list(out[:m])

    def set_profiling(self, on: bool) -> None:
        _check(self._lib.psg_set_profiling(self._h, 1 if on else 0))

    def kernel_stats(self) -> dict:
        cap = 16
        names = (ctypes.c_char_p * cap)()
        launches = (ctypes.c_uint64 * cap)()
        ms = (ctypes.c_double * cap)()
        n = ctypes.c_size_t(0)
        _check(self._lib.psg_kernel_stats(self._h, names, launches, ms, cap, ctypes.byref(n)))
        return {names[i].decode(): (launches[i], ms[i]) for i in range(min(n.value, cap))}

    def reset_kernel_stats(self) -> None:
        _check(self._lib.psg_reset_kernel_stats(self._h))

    def smem_atomic_rates(self) -> Tuple[float, float]:
        """(random-address, conflict-free) shared atomicAnd rates, atomics/s."""
        r, c = ctypes.c_double(0), ctypes.c_double(0)
        _check(self._lib.psg_measure_smem_atomic_rate(self._h, ctypes.byref(r), ctypes.byref(c)))
        return r.value, c.value

    def bucket_entries(self, reset: bool = False) -> int:
        v = ctypes.c_uint64(0)
        _check(self._lib.psg_bucket_entries(self._h, ctypes.byref(v), 1 if reset else 0))
        return v.value


class Server:
    """Request server with continuous batching on a context (psg_server_*).
    The server keeps its context alive; closing the context stops it."""

    def __init__(self, ctx: "Context", **config: int):
        lib = load()
        cfg = PsgServerConfig()
        for k, v in config.items():
            setattr(cfg, k, int(v))
        h = ctypes.c_void_p()
        _check(lib.psg_server_start(ctx.handle, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._lib = lib
        self._ctx = ctx                       # the context outlives the server
        ctx._servers.add(self)

    def submit(self, start: int, stop: int, kinds: int = 0x3F) -> int:
        rid = ctypes.c_uint64(0)
        _check(self._lib.psg_server_submit(self._h, start, stop, kinds, ctypes.byref(rid)))
        return rid.value

    def wait(self, rid: int) -> Tuple[List[int], float]:
        out = (ctypes.c_uint64 * 6)()
        lat = ctypes.c_double(0)
        _check(self._lib.psg_server_wait(self._h, rid, out, ctypes.byref(lat)))
        return list(out), lat.value

    def replay(self, requests: Sequence[Tuple[int, int, int]], arrivals: Sequence[float]):
        """Submit requests[i] at arrivals[i] seconds; returns (counts, latencies)."""
        n = len(requests)
        arr = (PsgRange * max(n, 1))()
        for i, (a, b, k) in enumerate(requests):
            arr[i].start, arr[i].stop, arr[i].kinds = a, b, k
        t = (ctypes.c_double * max(n, 1))(*arrivals)
        out = (ctypes.c_uint64 * (6 * max(n, 1)))()
        lat = (ctypes.c_double * max(n, 1))()
        _check(self._lib.psg_server_replay(self._h, arr, t, n, out, lat))
        return [list(out[6 * i:6 * i + 6]) for i in range(n)], list(lat[:n])

    def inject_failure(self, nth: int, status: int) -> None:
        """Tests: the nth request planned from now on fails its step with
        `status` (psg_server_inject_failure)."""
        _check(self._lib.psg_server_inject_failure(self._h, nth, status))

    def stats(self) -> dict:
        st = PsgServerStats()
        _check(self._lib.psg_server_get_stats(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in PsgServerStats._fields_}

    def close(self) -> None:
        if self._h:
            self._lib.psg_server_stop(self._h)
            self._h = None

    def __enter__(self) -> "Server":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self) -> None:  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


def serving_workload(n: int, rate: float, seed: int = 1, len_log2: Tuple[float, float] = (12.0, 36.0),
                     start_range: Tuple[float, float] = (1e6, 1.8e19)):
    """The serving request stream: Poisson arrivals at `rate` requests/s,
    start log-uniform in start_range, length log-uniform in 2^len_log2,
    kind uniform over 1..6 (primes .. sextuplets), stop clamped to 2^64 - 1.
    numpy.random.default_rng(seed), drawn per request in the order
    gap, start, length, kind. Returns (requests [(start, stop, kinds)],
    arrival seconds)."""
    import math
    import numpy as np
    rng = np.random.default_rng(seed)
    lo, hi = math.log10(start_range[0]), math.log10(start_range[1])
    reqs, arrivals, t = [], [], 0.0
    for _ in range(n):
        t += float(rng.exponential(1.0 / rate))
        start = int(10.0 ** rng.uniform(lo, hi))
        length = int(2.0 ** rng.uniform(len_log2[0], len_log2[1]))
        kind = int(rng.integers(1, 7))
        stop = min(start + length - 1, (1 << 64) - 1)
        reqs.append((start, stop, 1 << (kind - 1)))
        arrivals.append(t)
    return reqs, arrivals


def split_range(start: int, stop: int, parts: int) -> List[Tuple[int, int]]:
    """Split [start, stop] into `parts` consecutive sub-ranges whose inner
    boundaries are == 2 (mod 30), so that no k-tuplet straddles two parts
    (reference src/ParallelSieve.cpp:122-133). Empty parts are dropped."""
    if start > stop:
        return []
    parts = max(1, parts)
    n = stop - start + 1
    bounds = [start]
    for i in range(1, parts):
        b = start + n * i // parts
        b += (2 - b) % 30          # next value == 2 (mod 30)
        b = min(b, stop + 1)
        bounds.append(max(b, bounds[-1]))
    bounds.append(stop + 1)
    return [(a, b - 1) for a, b in zip(bounds, bounds[1:]) if a <= b - 1]


def shard_of(start: int, stop: int, rank: int, world: int) -> Optional[Tuple[int, int]]:
    """This rank's part of [start, stop] for a one-process-per-GPU run: the
    range is cut into `world` consecutive parts at == 2 (mod 30) boundaries
    (no collective is needed to count them; only the six totals are summed)."""
    parts = split_range(start, stop, world)
    # split_range drops empty parts; re-split so that rank indices line up
    if len(parts) < world:
        parts = parts + [None] * (world - len(parts))
    return parts[rank]


def range_cost(start: int, stop: int) -> float:
    """Estimated GPU work of counting [start, stop]: its crossings,
    (8/30) * length * sum(1/p) over the sieving primes 59 < p <= sqrt(stop)
    (~ ln ln sqrt(stop) - ln ln 59), plus a fixed per-range cost worth
    1e7 integers (planning, launches, the last partial segment)."""
    import math
    if start > stop:
        return 0.0
    r = max(math.isqrt(stop), 61)
    density = (8.0 / 30.0) * max(math.log(math.log(r)) - math.log(math.log(59.0)), 0.0)
    return (stop - start + 1) * (density + 0.01) + 1e7 * 0.3


def balance_ranges(ranges: Sequence[Tuple[int, int]], world: int) -> List[List[int]]:
    """Indices of `ranges` ([(start, stop), ...]) per rank for a
    one-process-per-GPU batch: longest-processing-time greedy on range_cost,
    so that ranks get equal estimated work (lengths in a batch differ by
    orders of magnitude; a split by index would not balance). Deterministic:
    every rank computes the same split. Within a rank indices ascend."""
    world = max(1, world)
    order = sorted(range(len(ranges)), key=lambda i: (-range_cost(*ranges[i]), i))
    load = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += range_cost(*ranges[i])
    return [sorted(p) for p in parts]


def count_sharded(count_fn, start: int, stop: int, kinds: int, rank: int, world: int,
                  group=None) -> List[int]:
    """Count [start, stop] across `world` ranks: each rank counts its shard
    with count_fn(a, b, kinds) -> [6 counts], then the six totals are summed
    with one all_reduce over torch.distributed (NCCL on GPUs, gloo on CPU)."""
    import torch
    import torch.distributed as dist
    part = shard_of(start, stop, rank, world)
    local = count_fn(part[0], part[1], kinds) if part else [0] * 6
    if world == 1 or not dist.is_initialized():
        return list(local)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([int(x) for x in local], dtype=torch.int64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return [int(x) for x in t.cpu().tolist()]

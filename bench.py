#!/usr/bin/env python3
"""Benchmark: integers sieved per second, exact prime counts, on B200.

Workload (one step = one full pass): count the primes in
[1e15, 1e15 + 1e11] -- 1,951,957 sieving primes up to ~3.16e7, so the bucket
sieve (big primes) and the shared-memory cross-off (small and medium primes)
both run. With N GPUs (one process per GPU under torchrun) rank r counts
[1e15 + r*1e11, 1e15 + (r+1)*1e11] (weak scaling) and the totals are summed
with one NCCL all_reduce.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value : device-timed throughput (CUDA events on the launch stream around K
        passes of psg_count_async; the sieving-prime table is prepared in the
        warm-up, so the timed region is pure GPU work), max over ranks.
e2e   : the same metric through the C ABI call psg_count() with host
        arguments and a host result (launches, accumulator reset and the
        device->host copy inside the timed region), wall clock, max over ranks.
--impl reference : the reference's own CPU sieve (oracle/_ref/primesieve,
        built from the reference sources) on all host cores, one full pass of
        the same workload per step (a bounded sample if the host is too slow
        for the run to end within a few minutes); the C restatement in
        oracle/ stands in if that binary is missing.

Besides the headline line's own workload, one GPU (N=1) also reports:
configs  : pi(1e9), the six counts of [0, 1e11] and of [2^64-2^34, 2^64-1],
           each device-timed, end to end through psg_count, and with the
           reference CLI's time on the full range in the same run;
serving  : the seed-1 request stream (lengths 2^12..2^36, starts up to
           1.8e19, kinds 1..6) replayed through psg_server_replay at
           100, 300, 1k, 3k, 10k and 50k requests/s: p50/p99 latency and integers/s per rate,
           beside the reference library replaying a seeded sample of it;
batched  : the 4096-range workload through psg_count_batch vs one psg_count
           per range, beside the reference library on a sample of it.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
START = 10 ** 15
LENGTH = 10 ** 11
METRIC = "integers sieved/s, exact pi/k-tuplet counts: batched vs per-range; p50/p99 latency"
UNIT = "integers/s"
WORKLOAD = "count primes in [1e15, 1e15+1e11] (sieving primes <= 3.16e7, bucket sieve)"
GOLDEN_1E15 = 2895317534          # pi[1e15, 1e15+1e11], reference CPU library
# ncu, [1e15, 1e15+4e9] (one 1018-segment window of the default engine,
# 312,728,441 bucket entries: the multiples of the primes 393,216..3.16e7
# with cofactors prime to 30, counted exactly on the host): fill kernel
# 1332.425 MB written + 166.158 MB read, sieve kernel 1358.508 MB read +
# 5.942 MB written
FILL_DRAM_BYTES_PER_ENTRY = (1332.425e6 + 166.157824e6) / 312728441
SIEVE_DRAM_BYTES_PER_ENTRY = (1358.508e6 + 5.942016e6) / 312728441


CONFIGS = [
    # (name, start, stop, kinds mask, reference CLI count flags)
    ("pi(1e9)", 0, 10 ** 9, 0x01, "-c1"),
    ("counts 1-6 of [0, 1e11]", 0, 10 ** 11, 0x3F, "-c123456"),
    ("counts 1-6 of [2^64-2^34, 2^64-1]", 2 ** 64 - 2 ** 34, 2 ** 64 - 1, 0x3F, "-c123456"),
]
GOLDEN_COUNTS = os.path.join(REPO, "tests", "golden", "ref_counts.json")


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def load_pkg():
    import importlib.util
    spec = importlib.util.spec_from_file_location("primesieve_gpu_b200",
                                                  os.path.join(REPO, "primesieve-gpu_b200", "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"psg_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # nvidia-smi takes a few hundred ms to start: begin the timed region
        # only once it has written its first sample (at most 5 s)
        t = time.perf_counter()
        while time.perf_counter() - t < 5.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.01)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        try:
            os.remove(self.path)
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def cpu_reference_rate(budget_s, threads=None):
    """The reference's CPU sieve on this host: largest sample of the workload
    [1e15, 1e15+S] that takes about `budget_s` seconds. Returns
    (integers/s, sample length, seconds, kind, cores)."""
    exe = os.path.join(REPO, "oracle", "_ref", "primesieve")
    cores = threads or os.cpu_count() or 1
    if os.path.exists(exe):
        def run(n):
            t = time.perf_counter()
            out = subprocess.run([exe, str(START), str(START + n), "-c1", "-q", "-t", str(cores)],
                                 capture_output=True, text=True, check=True).stdout
            return time.perf_counter() - t, int(out.split()[0])
        kind = "reference"
    else:
        sys.path.insert(0, os.path.join(REPO, "tests"))
        from conftest import Oracle  # the C restatement (single-threaded), checker only
        orc = Oracle()
        cores = 1

        def run(n):
            t = time.perf_counter()
            c = orc.plain(START, START + n, 1)[0]
            return time.perf_counter() - t, c
        kind = "port"
    n = 10 ** 9
    el, _ = run(n)
    while el < budget_s / 4 and n < LENGTH:
        n = min(LENGTH, int(n * max(2.0, min(8.0, budget_s / max(el, 1e-3) / 2))))
        el, _ = run(n)
    return n / el, n, el, kind, cores


def reference_arm(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    exe = os.path.join(REPO, "oracle", "_ref", "primesieve")
    cores = os.cpu_count() or 1
    steps = args.warmup + args.steps
    if os.path.exists(exe):
        kind = "reference"

        def run(n):
            subprocess.run([exe, str(START), str(START + n), "-c1", "-q", "-t", str(cores)],
                           capture_output=True, check=True)
        # one full pass of the workload per step when the whole run fits in
        # about three minutes on this host, else the largest sample that does
        t = time.perf_counter()
        run(LENGTH)
        full_s = time.perf_counter() - t
        n = LENGTH if full_s * steps <= 180.0 else max(10 ** 9, int(LENGTH * 180.0 / (full_s * steps)))
    else:
        kind, cores = "port", 1
        sys.path.insert(0, os.path.join(REPO, "tests"))
        from conftest import Oracle     # the C restatement, single-threaded
        orc = Oracle()

        def run(n):
            orc.plain(START, START + n, 1)
        n = 10 ** 9
    times = []
    for i in range(steps):
        t = time.perf_counter()
        run(n)
        if i >= args.warmup:
            times.append(time.perf_counter() - t)
    total = sum(times)
    value = n * len(times) / total
    sample = f"[1e15, 1e15+{n:.3g}] per step, -t {cores}"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic", "config": {"workload": WORKLOAD, "sample": sample, "full_range": n == LENGTH},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "cpu": cpu_model(), "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="own", choices=["own", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-vs-per-range section")
    ap.add_argument("--no-configs", action="store_true", help="skip the per-config section")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving section")
    ap.add_argument("--serving-requests", type=int, default=1000, help="requests per serving rate")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.warmup < 3:
        args.warmup = 3

    import torch
    import torch.distributed as dist
    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    psg = load_pkg()
    ctx = psg.Context(device=local)
    a = START + rank * LENGTH
    b = a + LENGTH
    # a dedicated (non-default) stream: the kernels, the accumulator reset and
    # the CUDA events all go on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    counts = torch.zeros(6, dtype=torch.int64, device="cuda")
    ctx.prepare(b)

    def step():
        counts.zero_()
        ctx.count_async(a, b, psg.PRIMES, counts.data_ptr(), stream.cuda_stream)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    got0 = int(counts[0].item())

    # ---- device-timed region ------------------------------------------------
    ctx.reset_kernel_stats()
    ctx.bucket_entries(reset=True)
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    # the asynchronous passes cannot recount: every one of them must have
    # kept all of its bucket entries
    try:
        ctx.count_async_status()
        async_exact = True
    except psg.PsgError:
        async_exact = False
    stats = ctx.kernel_stats()
    launches = sum(v[0] for v in stats.values())
    entries = ctx.bucket_entries(reset=True)
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * LENGTH * args.steps / (ms_max * 1e-3)

    # ---- per-kernel roofline (CUDA events per launch, separate pass; the
    # engine runs the windows of a profiled pass one after another, so each
    # kernel's time is its own -- the timed passes overlap consecutive
    # windows on two streams) ------------------------------------------------
    ctx.set_profiling(True)
    ctx.reset_kernel_stats()
    step()
    torch.cuda.synchronize()
    kst = ctx.kernel_stats()
    ctx.set_profiling(False)
    smem_rand, smem_cf = ctx.smem_atomic_rates()
    hbm_peak, peak_src = load_peaks()
    entries_per_pass = entries / args.steps
    sieve_l, sieve_ms = kst.get("sieve_count_kernel", (0, 0.0))
    fill_l, fill_ms = kst.get("bucket_fill_kernel", (0, 0.0))
    # algorithmic bytes of the bucket kernel: 4 B per entry written
    fill_bytes = 4.0 * entries_per_pass
    fill_gbs = fill_bytes / max(fill_ms, 1e-9) / 1e6
    # cross-off phase: crossings = (8/30) * N * sum(1/p) over sieving primes
    # p > 59 (pre-sieved below); the sieve kernel does these with shared atomics
    crossings = crossing_count(b)
    sieve_rate = crossings / max(sieve_ms * 1e-3, 1e-12)
    dominant = "bucket_fill_kernel" if fill_ms > sieve_ms else "sieve_count_kernel"
    # DRAM traffic per launch: bytes per bucket entry from one ncu capture of
    # each kernel on [1e15, 1e15+4e9] (one 1018-segment window, 312,728,441
    # entries), scaled by this launch's entries
    entries_per_launch = entries_per_pass / max(fill_l, 1)
    fill_traffic = FILL_DRAM_BYTES_PER_ENTRY * entries_per_launch
    sieve_traffic = SIEVE_DRAM_BYTES_PER_ENTRY * entries_per_launch
    roof_fill = {"kernel": "bucket_fill_kernel", "bound": "hbm", "achieved": fill_gbs, "peak": hbm_peak,
                 "unit": "GB/s", "frac": fill_gbs / hbm_peak, "traffic": fill_traffic,
                 "traffic_source": "ncu dram__bytes_read+write per entry on a one-window case, scaled",
                 "algorithmic_bytes_per_launch": fill_bytes / max(fill_l, 1),
                 "avg_launch_ms": fill_ms / max(fill_l, 1), "peak_source": peak_src}
    # the sieve kernel's DRAM work is reading the window's bucket lists once
    # (4 B per entry); what bounds it is the shared-memory atomics of the
    # cross-off, reported beside the HBM figure against the in-run probe
    sieve_bytes = 4.0 * entries_per_pass
    sieve_gbs = sieve_bytes / max(sieve_ms, 1e-9) / 1e6
    roof_sieve = {"kernel": "sieve_count_kernel", "bound": "hbm", "achieved": sieve_gbs, "peak": hbm_peak,
                  "unit": "GB/s", "frac": sieve_gbs / hbm_peak, "traffic": sieve_traffic,
                  "traffic_source": "ncu dram__bytes_read+write per entry on a one-window case, scaled",
                  "algorithmic_bytes_per_launch": sieve_bytes / max(sieve_l, 1),
                  "avg_launch_ms": sieve_ms / max(sieve_l, 1), "peak_source": peak_src,
                  "limit": {"bound": "smem_atomic", "achieved": sieve_rate / 1e9, "unit": "Gatomic/s",
                            "peak": smem_cf / 1e9, "frac": sieve_rate / max(smem_cf, 1),
                            "peak_source": "measured in-run: conflict-free smem atomicAnd probe (lane l on bank l)",
                            "peak_random": smem_rand / 1e9, "frac_random": sieve_rate / max(smem_rand, 1),
                            "peak_random_source": "measured in-run: random-address smem atomicAnd probe",
                            "crossings_per_pass": crossings, "bucket_entries_applied_per_pass": entries_per_pass}}

    # ---- end to end through the C ABI with host buffers ----------------------
    # psg_count: host arguments in, host counts out (launches, the device
    # accumulator reset and the device->host copy all inside the timed region)
    ctx.count(a, b, psg.PRIMES)
    barrier()
    te = time.perf_counter()
    for _ in range(max(1, args.steps // 2)):
        e2e_count = ctx.count(a, b, psg.PRIMES)[0]
    te = time.perf_counter() - te
    te_t = torch.tensor([te], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(te_t, op=dist.ReduceOp.MAX)
    e2e_value = world * LENGTH * max(1, args.steps // 2) / float(te_t.item())

    tot = torch.tensor([got0], dtype=torch.int64, device="cuda")
    if world > 1:
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    ok0 = async_exact and ((rank != 0) or (got0 == GOLDEN_1E15 and e2e_count == GOLDEN_1E15))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, n, el, kind, cores = cpu_reference_rate(12.0)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "cpu": cpu_model(), "kind": kind,
               "sample": f"[1e15, 1e15+{n:.3g}] in {el:.1f} s, -t {cores}"}

    configs = None
    if world == 1 and not args.no_configs:
        configs = config_section(psg, ctx, stream, args, torch)
    serving = None
    if world == 1 and not args.no_serving:
        serving = serving_section(psg, ctx, args)
    batched = None
    if not args.no_batch:
        batched = batch_section(psg, ctx, rank, world, args, torch, dist)

    if rank == 0:
        cfg = ctx.config()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "range_per_gpu": [a, b], "kinds": "primes",
                       "segment_bytes": cfg["seg_bytes"], "block": cfg["block"],
                       "l2": "inputs larger than L2: each pass streams %.1f GB of bucket lists" % (8 * entries_per_pass / 1e9),
                       "count_ok": bool(ok0), "async_passes_exact": async_exact,
                       "total_count": int(tot.item())},
            "roofline": roof_fill if dominant == "bucket_fill_kernel" else roof_sieve,
            "rooflines": [roof_sieve, roof_fill],
            "kernel_ms_per_pass": {k: v[1] for k, v in kst.items()},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 16, "d2h_bytes_per_step": 52,
                    "api": "psg_count (C ABI, host result)"},
            "gpu_launches": launches,
            "clocks": clk,
            "configs": configs,
            "serving": serving,
            "batched": batched,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    ok_all = ok0 and all(c["count_ok"] for c in (configs or [])) and (serving is None or serving["count_ok"]) \
        and (batched is None or batched["count_ok"])
    return 0 if ok_all else 1


def cli_seconds(start, stop, flag):
    """The reference CLI (oracle/_ref/primesieve) on [start, stop] with all
    host threads: (seconds, counts in -c order) or None without the binary."""
    exe = os.path.join(REPO, "oracle", "_ref", "primesieve")
    if not os.path.exists(exe):
        return None
    cores = os.cpu_count() or 1
    t = time.perf_counter()
    out = subprocess.run([exe, str(start), str(stop), flag, "-t", str(cores)], capture_output=True, text=True,
                         check=True).stdout
    el = time.perf_counter() - t
    counts = [int(x.rsplit(":", 1)[1]) for x in out.strip().split("\n") if ":" in x and not x.startswith("Sec")]
    return el, counts, cores


def config_section(psg, ctx, stream, args, torch):
    """The other single-range configurations: device-timed passes of
    psg_count_async (CUDA events on the launch stream), the same count end to
    end through psg_count, and the reference CLI on the full range."""
    with open(GOLDEN_COUNTS) as f:
        golden = {(r["start"], r["stop"]): r["counts"] for r in json.load(f)["bench"]}
    hbm_peak, _ = load_peaks()
    out = []
    counts = torch.zeros(6, dtype=torch.int64, device="cuda")
    for name, a, b, kinds, flag in CONFIGS:
        ints = b - a + 1
        ctx.prepare(b)

        def step():
            counts.zero_()
            ctx.count_async(a, b, kinds, counts.data_ptr(), stream.cuda_stream)
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        # about half a second of timed passes, at least 3
        t = time.perf_counter()
        step()
        torch.cuda.synchronize()
        one = time.perf_counter() - t
        k = max(3, min(200, int(0.5 / max(one, 1e-4))))
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(k):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / k
        try:
            ctx.count_async_status()
            exact_async = True
        except psg.PsgError:
            exact_async = False
        dev_counts = [int(x) for x in counts.tolist()]
        # end to end: host arguments in, host counts out
        ctx.count(a, b, kinds)
        ke = max(3, k // 2)
        t = time.perf_counter()
        for _ in range(ke):
            host = ctx.count(a, b, kinds)
        te = (time.perf_counter() - t) / ke
        want = [c if (kinds >> i) & 1 else 0 for i, c in enumerate(golden[(a, b)])]
        ok = exact_async and dev_counts == want and host == want
        line = {"workload": f"{name}: [{a}, {b}]", "kinds": kinds, "value": ints / (ms * 1e-3), "unit": UNIT,
                "ms_per_pass": ms, "passes": k, "counts": host, "count_ok": ok,
                "e2e": {"value": ints / te, "unit": UNIT, "ms_per_call": te * 1e3,
                        "h2d_bytes_per_step": 16, "d2h_bytes_per_step": 52, "api": "psg_count (C ABI, host result)"}}
        if not args.no_cpu_baseline:
            r = cli_seconds(a, b, flag)
            if r:
                el, cc, cores = r
                line["cpu_baseline"] = {"value": ints / el, "unit": UNIT, "cores": cores, "cpu": cpu_model(),
                                        "kind": "reference", "seconds": el,
                                        "sample": f"full range, reference CLI {flag} -t {cores}"}
                line["cpu_counts_match"] = cc == [want[i] for i in range(6) if (kinds >> i) & 1]
                line["vs_cpu"] = line["e2e"]["value"] / line["cpu_baseline"]["value"]
        out.append(line)
    return out


def serving_section(psg, ctx, args):
    """The seed-1 serving stream replayed through one request server
    (psg_server_replay paces the arrivals from C++; latency from each
    request's scheduled arrival to its completion) at each rate, the same
    requests at every rate. Throughput = integers of all requests / (last
    completion - first arrival). A seeded sample of the results is checked
    against psg_count."""
    import random
    import numpy as np
    n = args.serving_requests
    rates = [100.0, 300.0, 1000.0, 3000.0, 10000.0, 50000.0]
    rows = []
    ok = True
    with psg.Server(ctx) as srv:
        for rate in rates:
            reqs, arr = psg.serving_workload(n, rate, seed=1)
            ints = float(sum(b - a + 1 for a, b, _ in reqs))
            t = time.perf_counter()
            res, lats = srv.replay(reqs, arr)
            wall = time.perf_counter() - t
            lat = np.array(lats)
            span = max(wall, 1e-9)
            rows.append({"rate": rate, "requests": n, "p50_ms": float(np.percentile(lat, 50) * 1e3),
                         "p99_ms": float(np.percentile(lat, 99) * 1e3), "max_ms": float(lat.max() * 1e3),
                         "integers": ints, "value": ints / span, "unit": UNIT,
                         "offered": ints / max(arr[-1], 1e-9), "seconds": wall})
            for i in random.Random(int(rate)).sample(range(n), 8):
                a, b, k = reqs[i]
                ok = ok and res[i] == ctx.count(a, b, k)
        st = srv.stats()
    out = {"workload": "serving stream seed 1: Poisson arrivals, start log-uniform [1e6, 1.8e19], length "
                       "log-uniform [2^12, 2^36], kind uniform over 1..6",
           "api": "psg_server_replay (C ABI)", "rates": rows, "count_ok": ok,
           "sustained": max(rows, key=lambda r: r["value"]),
           "server": {k: st[k] for k in ("steps", "bucket_requests", "batch_requests", "refused")}}
    if not args.no_cpu_baseline:
        reqs, _ = psg.serving_workload(n, 1000.0, seed=1)
        out["cpu_baseline"] = cpu_trace_rate(reqs, 10.0)
    return out


def cpu_trace_rate(reqs, budget_s):
    """The reference library replaying a seeded sample of a request trace, one
    count call per request with all host threads; stops after budget_s."""
    import ctypes
    import random
    lib_path = os.path.join(REPO, "oracle", "_ref", "libprimesieve_ref.so")
    if not os.path.exists(lib_path):
        return None
    lib = ctypes.CDLL(lib_path)
    cores = os.cpu_count() or 1
    lib.primesieve_set_num_threads.argtypes = [ctypes.c_int]
    lib.primesieve_set_num_threads(cores)
    fns = []
    for name in ("primes", "twins", "triplets", "quadruplets", "quintuplets", "sextuplets"):
        f = getattr(lib, "primesieve_count_" + name)
        f.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        f.restype = ctypes.c_uint64
        fns.append(f)
    order = list(range(len(reqs)))
    random.Random(0).shuffle(order)
    done, ints, t0 = 0, 0, time.perf_counter()
    for i in order:
        a, b, k = reqs[i]
        fns[k.bit_length() - 1](a, b)
        done += 1
        ints += b - a + 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return {"value": ints / el, "unit": UNIT, "cores": cores, "cpu": cpu_model(), "kind": "reference",
            "sample": f"{done} of {len(reqs)} requests (seeded shuffle), {ints:.3g} integers in {el:.1f} s"}


BATCH_FIXTURE = os.path.join(REPO, "tests", "golden", "batch4096.json")
BATCH_WORKLOAD = ("4096 ranges, seed 0: start log-uniform [1e6, 1e16], length log-uniform "
                  "[2^16, 2^34], kind uniform over primes/twins/triplets")


def batch_section(psg, ctx, rank, world, args, torch, dist):
    """Batched vs per-range on the 4096-range workload (each rank takes an
    equal share of the estimated work, psg.balance_ranges). Both arms go through the C ABI with host arguments and host
    results: per-range = one psg_count() per range, batched = one
    psg_count_batch() for all of them. Wall clock, max over ranks."""
    with open(BATCH_FIXTURE) as f:
        rows = json.load(f)["ranges"]
    mine = [rows[i] for i in psg.balance_ranges([(a, b) for a, b, _, _ in rows], world)[rank]]
    q = [(a, b, 1 << k) for a, b, k, _ in mine]
    ints = sum(b - a + 1 for a, b, _, _ in rows)
    ctx.prepare(max(b for _, b, _, _ in rows))

    def check(res):
        return all(r[k] == want and not any(r[j] for j in range(6) if j != k)
                   for (a, b, k, want), r in zip(mine, res))

    def tmax(x):
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    ctx.count_batch(q[:64])                      # warm-up
    # per-class batch parameters, tuned on samples of these ranges (outside
    # the timed region, like the sieving-prime table)
    t = time.perf_counter()
    tuned = ctx.autotune_batch(q, budget_seconds=25.0)
    t_tune = time.perf_counter() - t
    ok = True
    times = []
    for _ in range(2):
        if world > 1:
            dist.barrier()
        t = time.perf_counter()
        res = ctx.count_batch(q)
        times.append(tmax(time.perf_counter() - t))
        ok = ok and check(res)
    ctx.set_profiling(True)
    ctx.reset_kernel_stats()
    ctx.count_batch(q)
    kst = ctx.kernel_stats()
    ctx.set_profiling(False)
    if world > 1:
        dist.barrier()
    t = time.perf_counter()
    res = [ctx.count(a, b, k) for a, b, k in q]
    t_single = tmax(time.perf_counter() - t)
    ok = ok and check(res)
    ok_t = torch.tensor([1 if ok else 0], dtype=torch.int64, device="cuda")
    if world > 1:
        dist.all_reduce(ok_t, op=dist.ReduceOp.MIN)
    t_batch = min(times)
    out = {
        "workload": BATCH_WORKLOAD, "ranges": len(rows), "integers": ints,
        "value": ints / t_batch, "unit": UNIT, "seconds": t_batch,
        "per_range_value": ints / t_single, "per_range_seconds": t_single,
        "speedup_vs_per_range": t_single / t_batch,
        "count_ok": bool(ok_t.item()),
        "kernel_ms": {k: round(v[1], 2) for k, v in kst.items() if v[0]},
        "kernel_launches": {k: v[0] for k, v in kst.items() if v[0]},
        "api": "psg_count_batch vs psg_count per range (C ABI, host results)",
        "autotune": {"seconds": round(t_tune, 2),
                     "classes": [{"digits": r["range_class"] + 1, "direct_budget": r["direct_budget"],
                                  "big_limit": r["big_limit"], "stripe": r["stripe"],
                                  "small_limit": r["small_limit"],
                                  "sample_s": round(r["best_seconds"], 4), "default_s": round(r["default_seconds"], 4)}
                                 for r in tuned]},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_batch_rate(rows, 10.0)
        out["vs_cpu"] = out["value"] / out["cpu_baseline"]["value"]
    return out


def cpu_batch_rate(rows, budget_s):
    """The reference library (oracle/_ref/libprimesieve_ref.so) counting a
    seeded random sample of the batch ranges one call at a time with all
    host threads, as the reference's callers would; stops after budget_s."""
    import ctypes
    import random
    lib_path = os.path.join(REPO, "oracle", "_ref", "libprimesieve_ref.so")
    if not os.path.exists(lib_path):
        return None
    lib = ctypes.CDLL(lib_path)
    cores = os.cpu_count() or 1
    lib.primesieve_set_num_threads.argtypes = [ctypes.c_int]
    lib.primesieve_set_num_threads(cores)
    fns = []
    for name in ("primes", "twins", "triplets"):
        f = getattr(lib, "primesieve_count_" + name)
        f.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        f.restype = ctypes.c_uint64
        fns.append(f)
    order = list(range(len(rows)))
    random.Random(0).shuffle(order)
    done, ints, t0 = 0, 0, time.perf_counter()
    for i in order:
        a, b, k, want = rows[i]
        if fns[k](a, b) != want:
            raise RuntimeError("reference library disagrees with the fixture")
        done += 1
        ints += b - a + 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return {"value": ints / el, "unit": UNIT, "cores": cores, "cpu": cpu_model(), "kind": "reference",
            "sample": f"{done} of {len(rows)} ranges (seeded shuffle), {ints:.3g} integers in {el:.1f} s"}


def crossing_count(stop):
    """Crossings of one pass: sum over sieving primes 59 < p <= sqrt(stop) of
    the multiples p*q (q coprime to 30) in the range, (8/30) * LENGTH / p."""
    import math
    import numpy as np
    lim = math.isqrt(stop)
    sieve = np.ones(lim + 1, dtype=bool)
    sieve[:2] = False
    for i in range(2, math.isqrt(lim) + 1):
        if sieve[i]:
            sieve[i * i::i] = False
    p = np.nonzero(sieve)[0]
    p = p[p > 59].astype(np.float64)
    return float(LENGTH * 8.0 / 30.0 * np.sum(1.0 / p))


if __name__ == "__main__":
    sys.exit(main())

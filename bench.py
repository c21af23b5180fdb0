#!/usr/bin/env python
"""Benchmark: microseconds per Lucas-Lehmer iteration at the 8M-point NTT.

Workload: the Lucas-Lehmer test of q = 139000003 (the first prime above 1.39e8)
at the reference's length n = 2^23 (ntt_lengths.cu:88-98 picks it), from
s0 = 4.  One step = ITERATIONS_PER_STEP squarings (-2 each) of that residue.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value`: device time of the K steps (CUDA events on the test's stream, residue
resident in HBM, L2 flushed between steps) per squaring.  `e2e`: the same
through the C ABI with host buffers -- every step uploads the residue from
pinned memory (lnt_set_digits), squares, and reads the canonical residue back
(lnt_get_digits).  With N > 1 every rank runs an independent replica (one LL
test does not shard); the time is the max over ranks.

--impl reference times the reference's algorithm on the host cores: the
reference has no CPU implementation, so this is the CPU oracle
(oracle/lnt_oracle.c, a port of its per-iteration arithmetic) on all threads.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

EXPONENT = 139000003
LOG2N = 23
N = 1 << LOG2N
ITERATIONS_PER_STEP = 1000
METRIC = "µs/iteration at 8M-pt NTT"
UNIT = "us/iteration"
FLUSH_BYTES = 256 << 20  # larger than the 126 MB L2
ALGO_BYTES_PER_WORD_PER_SWEEP = 16  # one read + one write of a uint64 word


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--iterations-per-step", type=int, default=ITERATIONS_PER_STEP)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["c1", "c2", "c3", "c4", "c5", "lengths"], default="c2",
                    help="c2: one 8M-point LL test (default); c3/c4: batched tests/hour; c5: serving; "
                         "lengths: one LL test at each of 2^24, 2^25, 2^26")
    ap.add_argument("--seconds", type=float, default=30.0, help="timed window of c3/c4/c5")
    ap.add_argument("--rates", default="0.5,1,2", help="c5: arrival rates as multiples of plain capacity")
    ap.add_argument("--c5-range", default="10000,200000",
                    help="c5: exponent range (full tests must finish inside the timed window)")
    return ap.parse_args()


def rank_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, or None."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    v = d.get("kernels", {}).get(kernel)
    return None if v is None else float(v)


def cpu_port_sample(threads: int, iterations: int):
    """Time the CPU oracle on `iterations` LL squarings of the workload."""
    from oracle import oracle as O

    O.set_threads(threads)
    with O.OracleTest(EXPONENT, N, prp=False) as T:
        T.iterate(1)  # warm caches and the thread pool
        t0 = time.perf_counter()
        T.iterate(iterations)
        dt = time.perf_counter() - t0
    return dt * 1e6 / iterations


def run_reference(args, rank, world):
    """CPU reference arm: the oracle port on all host threads."""
    if rank != 0:
        return
    from oracle import oracle as O

    threads = O.max_threads()
    per_step = 3
    O.set_threads(threads)
    with O.OracleTest(EXPONENT, N, prp=False) as T:
        for _ in range(args.warmup):
            T.iterate(per_step)
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            T.iterate(per_step)
            times.append(time.perf_counter() - t0)
    us = sum(times) * 1e6 / (args.steps * per_step)
    sample = f"{per_step} LL squarings of q={EXPONENT} at n=2^{LOG2N} per step"
    line = {
        "impl": "reference", "metric": METRIC, "value": us, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sum(times) * 1e3 / args.steps,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic: LL residue sequence from s0 = 4",
        "config": {"workload": f"LL q={EXPONENT} n=2^{LOG2N} (8M-pt NTT)", "exponent": EXPONENT,
                   "n": N, "iterations_per_step": per_step,
                   "implementation": "CPU oracle port of the reference arithmetic (reference has no CPU path)"},
        "cpu_baseline": {"value": us, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": us, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- batches ----

def primes_between(lo: int, hi: int) -> list[int]:
    import numpy as np

    sieve = np.ones(hi + 1, dtype=bool)
    sieve[:2] = False
    for k in range(2, int(hi ** 0.5) + 1):
        if sieve[k]:
            sieve[k * k::k] = False
    return [int(x) for x in np.nonzero(sieve)[0] if x >= lo]


def plain_us_per_iteration(cuda_b200, exponent: int, prp: bool, iters: int = 200, device: int = 0) -> float:
    """One test alone through the single-test path (the reference's way)."""
    with cuda_b200.LucasTest(exponent, 0, prp, device=device) as t:
        t.iterate(20)
        t.synchronize()
        t0 = time.perf_counter()
        t.iterate(iters)
        t.synchronize()
        return (time.perf_counter() - t0) * 1e6 / iters


def reference_us_per_iteration() -> dict:
    """The reference CUDA build's own per-iteration time at each length, measured
    on a B200 (tests/golden/ref_timings.json); its autotune keeps the fastest
    pool, so the best run per length is its plain path."""
    p = ROOT / "tests" / "golden" / "ref_timings.json"
    if not p.exists():
        return {}
    d = json.loads(p.read_text())["by_n"]
    return {int(n): min(r["per_iteration_us"] for r in runs) for n, runs in d.items()}


LENGTH_EXPONENTS = [300000007, 600000001, 1100000009]  # policy lengths 2^24, 2^25, 2^26


def run_lengths(args):
    """One LL test alone at each larger policy length: µs per squaring from
    CUDA events on the test's stream around `--iterations-per-step` squarings
    (after `--warmup` untimed calls of the same size), the kernel split of one
    more call, and the reference build's time at that length."""
    import torch

    import cuda_b200

    ref = reference_us_per_iteration()
    ips = min(args.iterations_per_step, 200)
    for q in LENGTH_EXPONENTS:
        stream = torch.cuda.Stream()
        with cuda_b200.LucasTest(q) as t:
            t.set_stream(stream.cuda_stream)
            for _ in range(max(args.warmup, 1)):
                t.iterate(ips)
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t.iterate(ips)
            e1.record(stream)
            stream.synchronize()
            us = e0.elapsed_time(e1) * 1e3 / ips
            prof = t.profile_iterations(ips)
            n = 1 << cuda_b200.secured_log2_length(q)
            line = {"metric": f"us/iteration, LL q={q} at n=2^{n.bit_length() - 1}", "value": us,
                    "unit": "us/iteration", "higher_is_better": False, "n_gpus": 1, "dtype": "u64",
                    "data": "LL residue sequence from s0 = 4",
                    "config": {"workload": f"LL q={q} n=2^{n.bit_length() - 1}", "plan": t.plan,
                               "iterations": ips, "res64": f"{t.res64():016x}"},
                    "kernels": {k: {"launches": v[0], "avg_us": v[1] * 1e3 / max(v[0], 1)}
                                for k, v in prof.items()},
                    "reference_build_us_per_iteration": ref.get(n)}
        print(json.dumps(line), flush=True)


def reference_plain_tests_per_hour(cuda_b200, exps, target_of):
    ref = reference_us_per_iteration()
    try:
        t = [target_of(q) * ref[1 << cuda_b200.secured_log2_length(q)] * 1e-6 for q in exps]
    except KeyError:
        return None
    return 3600 / (sum(t) / len(t))


def run_batch_workload(args, exps, prp, target_of, label, config, rank=0, world=1, local_rank=0):
    """tests/hour of the batch engine against one-test-at-a-time, on a bounded
    window.  With N ranks (one process per GPU) each rank runs its own batch over
    a cost-balanced share of the work list (cuda_b200/shard.py) and rank 0
    reports the whole job: the tests all ranks advanced over the slowest rank's
    window.  No collective touches the data path."""
    import cuda_b200
    from cuda_b200 import shard

    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    mine = shard.partition_by_cost(exps, world, lambda q: shard.test_cost(q, target_of(q), prp))[rank]
    step = 50
    with cuda_b200.Batch(device=local_rank) as b:
        for q in mine:
            b.submit(q, 0, prp, target_of(q))
        for _ in range(3):
            b.run(step)
        if dist is not None:
            dist.barrier()
        steps = 0
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < args.seconds:
            b.run(step)
            steps += 1
        elapsed = time.perf_counter() - t0
        finished = b.poll()
    done_local = sum(min(1.0, steps * step / target_of(q)) for q in mine)
    done = sum(shard.gather_results([done_local], dist))
    elapsed = shard.max_over_ranks(elapsed, dist)
    n_finished = sum(shard.gather_results([len(finished)], dist))
    tests_per_hour = done / elapsed * 3600
    plain_tests_per_hour = ref_plain = None
    if rank == 0:
        # plain path: a sample spread over the exponents, each test alone on one GPU
        sample = sorted(exps)[:: max(1, len(exps) // 12)]
        times = [target_of(q) * plain_us_per_iteration(cuda_b200, q, prp, device=local_rank) * 1e-6
                 for q in sample]
        plain_tests_per_hour = 3600 / (sum(times) / len(times))
        ref_plain = reference_plain_tests_per_hour(cuda_b200, exps, target_of)
        line = {"metric": f"tests/hour, {label}", "value": tests_per_hour, "unit": "tests/hour",
                "higher_is_better": True, "n_gpus": world, "data": "synthetic (seeded exponents)",
                "dtype": "u64", "config": config,
                "scaling": "strong" if world > 1 else "weak",
                "plain_tests_per_hour": plain_tests_per_hour,
                "speedup_vs_plain": tests_per_hour / plain_tests_per_hour,
                "reference_plain_tests_per_hour": ref_plain,
                "speedup_vs_reference_plain": tests_per_hour / ref_plain if ref_plain else None,
                "window_s": elapsed, "squarings_per_test_in_window": steps * step,
                "plain_sample": len(sample), "finished_in_window": n_finished}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


C1_EXPONENTS = [44497, 44501, 44507, 44519, 44531, 44533, 44537, 44543, 44549]


def run_c1(args):
    """Full LL of M_44497 and the next 8 prime exponents at the policy length
    (2048 words): each test alone through the single-test path, then all nine
    in one batch (one SMEM-resident launch).  Res64 checked against the
    committed fixture of the reference build's residues."""
    import cuda_b200

    golden = json.loads((ROOT / "tests" / "golden" / "ref_residues.json").read_text())["cases"]
    want = {c["q"]: c["res64"] for c in golden if c["n"] == 2048}
    per_it, ok = [], True
    with cuda_b200.LucasTest(C1_EXPONENTS[0]) as t:  # warm-up: module load, first launch
        t.iterate(100)
        t.synchronize()
    t_alone = 0.0
    for q in C1_EXPONENTS:
        with cuda_b200.LucasTest(q) as t:
            t0 = time.perf_counter()
            t.iterate(q - 2)
            r = t.res64()
            dt = time.perf_counter() - t0
        t_alone += dt
        per_it.append(dt * 1e6 / (q - 2))
        ok &= f"{r:016x}" == want.get(q, f"{r:016x}")
    with cuda_b200.Batch(device=0) as b:  # warm-up of the batch path: 1000 squarings each, untimed
        for q in C1_EXPONENTS:
            b.submit(q, 0, False, 1000)
        left = len(C1_EXPONENTS)
        while left:
            b.run(1000)
            left -= len(b.poll())
    t0 = time.perf_counter()
    with cuda_b200.Batch(device=0) as b:
        for q in C1_EXPONENTS:
            b.submit(q, 0, False)
        done = []
        while len(done) < len(C1_EXPONENTS):
            b.run(100000)
            done += b.poll()
    t_batch = time.perf_counter() - t0
    ok &= all(f"{r['res64']:016x}" == want.get(r["exponent"], f"{r['res64']:016x}") for r in done)
    line = {"metric": "us/iteration, full LL at n=2048 (M_44497 and the next 8 primes)",
            "value": sum(per_it) / len(per_it), "unit": "us/iteration", "higher_is_better": False,
            "n_gpus": 1, "dtype": "u64", "data": "LL from s0 = 4 (no synthetic inputs)",
            "config": {"workload": "C1: q = " + ",".join(map(str, C1_EXPONENTS)), "n": 2048,
                       "plan": "RESIDENT_2048"},
            "tests_per_hour_alone": len(C1_EXPONENTS) / t_alone * 3600,
            "tests_per_hour_batch": len(C1_EXPONENTS) / t_batch * 3600,
            "res64_equal_reference_build": bool(ok),
            "reference_build_us_per_iteration": reference_us_per_iteration().get(2048)}
    print(json.dumps(line), flush=True)


def run_serving(args, rank=0, world=1, local_rank=0):
    """Poisson stream of LL/PRP requests against the continuous-batching engine,
    beside the plain sequential path (a FIFO queue over measured service times).
    With N ranks the stream's rate is N times higher and request i goes to rank
    i mod N (round-robin dispatch to one engine per GPU); rank 0 reports the
    percentiles over all ranks' latencies."""
    import math
    import random

    import numpy as np

    import cuda_b200
    from cuda_b200 import shard

    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    lo, hi = (int(x) for x in args.c5_range.split(","))
    primes = primes_between(lo, min(hi * 2, hi + 100000))
    rng = random.Random(2)

    def draw():
        x = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        import bisect
        return primes[min(bisect.bisect_left(primes, int(x)), len(primes) - 1)], rng.random() < 0.5

    pool = [draw() for _ in range(64)]
    service = [(q if prp else q - 2) * plain_us_per_iteration(cuda_b200, q, prp, 100, local_rank) * 1e-6
               for q, prp in pool[:16]]
    mean_service = sum(service) / len(service)
    plain_capacity = 1.0 / mean_service  # tests per second, one at a time
    budget = 150 << 30
    for mult in (float(r) for r in args.rates.split(",")):
        rate = mult * plain_capacity * world
        t = 0.0
        arrivals = []
        while t < args.seconds:
            t += rng.expovariate(rate)
            q, prp = pool[rng.randrange(len(pool))]
            arrivals.append((t, q, prp))
        arrivals = [a for a in arrivals if a[0] < args.seconds]
        all_arrivals = arrivals
        arrivals = arrivals[rank::world]
        lat, done = [], 0
        if dist is not None:
            dist.barrier()
        with cuda_b200.Batch(device=local_rank, hbm_budget_bytes=budget) as b:
            t0 = time.perf_counter()
            k, enq = 0, {}
            while (k < len(arrivals) or done < len(arrivals)) and time.perf_counter() - t0 < 4 * args.seconds:
                now = time.perf_counter() - t0
                while k < len(arrivals) and arrivals[k][0] <= now:
                    i = b.enqueue(arrivals[k][1], 0, arrivals[k][2])
                    enq[i] = now - arrivals[k][0]  # wait before enqueue
                    k += 1
                b.run(200)
                for r in b.poll():
                    lat.append(r["seconds"] + enq.pop(r["id"], 0.0))
                    done += 1
            wall = time.perf_counter() - t0
        lat = shard.gather_results(lat, dist)
        done = sum(shard.gather_results([done], dist))
        wall = shard.max_over_ranks(wall, dist)
        if rank != 0:
            continue
        # plain sequential path: one GPU, FIFO over the same arrivals, service =
        # measured per-test time
        serv = {}
        free_at, plain_lat = 0.0, []
        for (ta, q, prp) in all_arrivals:
            if (q, prp) not in serv:
                serv[(q, prp)] = (q if prp else q - 2) * plain_us_per_iteration(cuda_b200, q, prp, 100, local_rank) * 1e-6
            start = max(free_at, ta)
            free_at = start + serv[(q, prp)]
            plain_lat.append(free_at - ta)
        line = {"metric": "serving p50/p99 latency and tests/hour", "rate_multiple_of_plain_capacity": mult,
                "requests": len(all_arrivals), "completed": done, "wall_s": wall, "n_gpus": world,
                "p50_s": float(np.percentile(lat, 50)) if lat else None,
                "p99_s": float(np.percentile(lat, 99)) if lat else None,
                "tests_per_hour": done / wall * 3600,
                "plain_p50_s": float(np.percentile(plain_lat, 50)), "plain_p99_s": float(np.percentile(plain_lat, 99)),
                "plain_tests_per_hour": len(all_arrivals) / free_at * 3600 if free_at else None,
                "config": {"exponents": f"primes log-uniform in [{lo}, {hi}], LL/PRP by a seeded coin (seed 2)",
                           "hbm_budget_gb": 150, "arrival": "Poisson",
                           "dispatch": "round-robin over ranks" if world > 1 else "one engine"}}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse_args()
    rank, local_rank, world = rank_info()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "c1":
        if rank == 0:
            run_c1(args)
        return
    if args.workload == "lengths":
        if rank == 0:
            run_lengths(args)
        return
    if args.workload in ("c3", "c4", "c5"):
        import random

        if args.workload == "c3":
            exps = random.Random(0).sample(primes_between(100000, 2000000), 256)
            run_batch_workload(args, exps, False, lambda q: q - 2, "256 full LL tests, q in [1e5, 2e6] (seed 0)",
                               {"workload": "C3 batch", "count": 256, "lengths": "4K-128K"},
                               rank, world, local_rank)
        elif args.workload == "c4":
            exps = random.Random(1).sample(primes_between(5000000, 20000000), 64)
            run_batch_workload(args, exps, True, lambda q: 20000, "64 PRP tests x 20000 squarings, q in [5e6, 2e7] (seed 1)",
                               {"workload": "C4 batch", "count": 64, "lengths": "512K-1M"},
                               rank, world, local_rank)
        else:
            run_serving(args, rank, world, local_rank)
        return

    import torch

    import cuda_b200

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ips = args.iterations_per_step

    stream = torch.cuda.Stream(device=dev)
    test = cuda_b200.LucasTest(EXPONENT, N, prp=False, device=local_rank)
    test.set_stream(stream.cuda_stream)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def flush_l2():
        with torch.cuda.stream(stream):
            flush.random_(0, 255)

    # warm-up steps (untimed)
    for _ in range(args.warmup):
        flush_l2()
        test.iterate(ips)
    stream.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # ---- device-resident timed region -------------------------------------
    barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    # headline: the production path (lnt_iterate, captured-graph replay), CUDA
    # events on the test's stream around each step
    step_ms, kernels = [], {}
    ev_a = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev_b = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for k in range(args.steps):
        flush_l2()
        ev_a[k].record(stream)
        test.iterate(ips)
        ev_b[k].record(stream)
    stream.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in zip(ev_a, ev_b)]
    # per-kernel breakdown (roofline): one more step of the same work with CUDA
    # events between the launches, inside the same sampled region
    flush_l2()
    prof = test.profile_iterations(ips)
    for name, (launches, ms) in prof.items():
        kernels[name] = [launches, ms]
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    barrier()
    total_ms = sum(step_ms)
    if dist is not None:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = total_ms * 1e3 / (world * args.steps * ips)

    # ---- end to end through the C ABI with host buffers --------------------
    host = torch.empty(N, dtype=torch.int64, pin_memory=True)
    test.digits(host.numpy().view("uint64"))
    stream.synchronize()
    barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    wall0 = time.perf_counter()
    ev0.record(stream)
    for _ in range(args.steps):
        test.set_digits(host.numpy().view("uint64"))
        test.iterate(ips)
        test.digits(host.numpy().view("uint64"))
    ev1.record(stream)
    ev1.synchronize()
    wall = time.perf_counter() - wall0
    e2e_ms = ev0.elapsed_time(ev1)
    barrier()
    if dist is not None:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = e2e_ms * 1e3 / (world * args.steps * ips)
    res64 = test.res64()

    # ---- roofline of the dominant kernel -----------------------------------
    dom = max(kernels.items(), key=lambda kv: kv[1][1])
    dom_name, (dom_launches, dom_ms) = dom
    avg_s = dom_ms / dom_launches / 1e3
    if test.plan.startswith("TWOPASS"):
        algo_bytes = ALGO_BYTES_PER_WORD_PER_SWEEP * N  # each pass reads and writes the residue once
    else:
        algo_bytes = ALGO_BYTES_PER_WORD_PER_SWEEP * N * ips
    achieved = algo_bytes / avg_s / 1e9
    peak, peak_kind = measured_peak_hbm()
    traffic = ncu_traffic(dom_name)
    # every timed step launches the same kernels as the profiled one
    launches_in_timed = sum(a[0] for a in kernels.values()) * (args.steps + 1)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sample_iters = 4
        cpu_us = cpu_port_sample(1, sample_iters)
        cpu = {"value": cpu_us, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{sample_iters} LL squarings of q={EXPONENT} at n=2^{LOG2N}, one thread"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic: LL residue sequence from s0 = 4",
            "config": {"workload": f"LL q={EXPONENT} n=2^{LOG2N} (8M-pt NTT), {ips} squarings per step",
                       "exponent": EXPONENT, "n": N, "iterations_per_step": ips, "plan": test.plan,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "flushed between steps (256 MiB write)", "res64_after_run": f"{res64:016x}",
                       "timing": "value: CUDA events around lnt_iterate per step (graph replay); kernels: "
                                 "one more step with events between launches",
                       "reference_build_us_per_iteration": reference_us_per_iteration().get(N)},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": N * 8, "d2h_bytes_per_step": N * 8,
                    "wall_s": wall},
            "gpu_launches": launches_in_timed,
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "algo_bytes_per_launch": algo_bytes,
                         "avg_launch_us": avg_s * 1e6},
            "kernels": {k: {"launches": v[0], "avg_us": v[1] * 1e3 / v[0]} for k, v in kernels.items()},
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    test.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

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
                         "lengths: one LL test at each of 2^24, 2^25, 2^26, 5*2^20, 5*2^21")
    ap.add_argument("--seconds", type=float, default=120.0, help="c5: arrival window")
    ap.add_argument("--autotune-loops", type=int, default=20, help="c3/c4: autotuner squarings per candidate (0: policy plans)")
    ap.add_argument("--plan-cache", default="", help="c3/c4: JSON plan cache file")
    ap.add_argument("--autotune-group", type=int, default=1,
                    help="c3/c4: tests timed together per candidate plan (1: one test alone)")
    ap.add_argument("--checkpoint-every", type=int, default=20000, help="c3/c4: Res64 checkpoint interval")
    ap.add_argument("--batch-step", type=int, default=2000, help="c3/c4/c5: squarings per engine call")
    ap.add_argument("--c3-count", type=int, default=256, help="c3: tests of the seeded sample to run")
    ap.add_argument("--short-lengths", action="store_true",
                    help="c3/c4: the batch runs each test at its smallest length (5*2^k where that "
                         "meets the bound) instead of the reference's power of two")
    ap.add_argument("--plain", choices=["real", "per-length"], default="per-length",
                    help="c3/c4: plain path run test by test, or summed from per-length times")
    ap.add_argument("--rates", default="0.25,1", help="c5: arrival rates, requests per second")
    ap.add_argument("--drain", type=float, default=60.0, help="c5: seconds the engine runs on after the window")
    ap.add_argument("--step-seconds", type=float, default=0.25,
                    help="c5: time budget of one engine call (iteration-level scheduling; 0: lockstep)")
    ap.add_argument("--c5-range", default="10000,30000000", help="c5: exponent range")
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


def ncu_counters() -> dict:
    """Per-launch ncu counters of the C2 kernels (profiles/ncu_traffic.json)."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    return json.loads(p.read_text()) if p.exists() else {}


def ncu_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, or None."""
    v = ncu_counters().get("kernels", {}).get(kernel)
    return None if v is None else float(v)


def issue_roofline(kernel: str, avg_launch_s: float, sms: int, sm_mhz):
    """The binding roofline of the integer-bound kernels: warp instructions
    issued per launch (ncu's count, committed) over the launch's CUDA-event
    duration, against the SMs' issue rate (4 schedulers per SM, one warp
    instruction per clock each) at the SM clock sampled during the timed region.
    The ALU and FMA pipe fractions are ncu's, from the same capture."""
    d = ncu_counters()
    inst = d.get("warp_instructions", {}).get(kernel)
    if inst is None or not sm_mhz:
        return None
    peak = sms * 4 * sm_mhz * 1e6
    achieved = inst / avg_launch_s
    out = {"warp_instructions_per_launch": inst, "achieved": achieved, "peak": peak,
           "unit": "warp instructions/s", "frac": achieved / peak, "sm_mhz": sm_mhz, "sms": sms}
    out.update({f"ncu_{k}": v for k, v in d.get("pipes", {}).get(kernel, {}).items()})
    return out


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
# exponents whose smallest length is 5 * 2^k: 5 * 2^21 (reference 2^24), 5 * 2^20 (2^23)
FIVE_EXPONENTS = [170000009, 100000007]


def length_name(n: int) -> str:
    return f"2^{n.bit_length() - 1}" if n & (n - 1) == 0 else f"5*2^{(n // 5).bit_length() - 1}"


def run_lengths(args):
    """One LL test alone at each larger policy length, and at the 5 * 2^k
    lengths of two exponents whose reference length is a power of two 8/5 as
    long: µs per squaring from CUDA events on the test's stream around
    `--iterations-per-step` squarings (after `--warmup` untimed calls of the
    same size), the kernel split of one more call, and the reference build's
    time at the reference's length for that exponent."""
    import torch

    import cuda_b200

    ref = reference_us_per_iteration()
    ips = min(args.iterations_per_step, 200)
    cases = [(q, 1 << cuda_b200.secured_log2_length(q)) for q in LENGTH_EXPONENTS]
    cases += [(q, cuda_b200.smallest_length(q)) for q in FIVE_EXPONENTS]
    for q, n in cases:
        stream = torch.cuda.Stream()
        ref_n = 1 << cuda_b200.secured_log2_length(q)
        with cuda_b200.LucasTest(q, n) as t:
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
            line = {"metric": f"us/iteration, LL q={q} at n={length_name(n)}", "value": us,
                    "unit": "us/iteration", "higher_is_better": False, "n_gpus": 1, "dtype": "u64",
                    "data": "LL residue sequence from s0 = 4",
                    "config": {"workload": f"LL q={q} n={length_name(n)}", "plan": t.plan,
                               "iterations": ips, "res64": f"{t.res64():016x}"},
                    "kernels": {k: {"launches": v[0], "avg_us": v[1] * 1e3 / max(v[0], 1)}
                                for k, v in prof.items()},
                    "reference_length": length_name(ref_n),
                    "reference_build_us_per_iteration": ref.get(ref_n)}
        print(json.dumps(line), flush=True)


def reference_plain_tests_per_hour(cuda_b200, exps, target_of):
    ref = reference_us_per_iteration()
    try:
        t = [target_of(q) * ref[1 << cuda_b200.secured_log2_length(q)] * 1e-6 for q in exps]
    except KeyError:
        return None
    return 3600 / (sum(t) / len(t))


def c3_exponents() -> list[int]:
    """C3: 256 primes in [1e5, 2e6], random.Random(0).sample."""
    import random

    return random.Random(0).sample(primes_between(100000, 2000000), 256)


def c4_exponents() -> list[int]:
    """C4: 64 primes in [5e6, 2e7], random.Random(1).sample."""
    import random

    return random.Random(1).sample(primes_between(5000000, 20000000), 64)


def c5_pool(lo: int = 10000, hi: int = 30000000, count: int = 64) -> list[tuple[int, bool]]:
    """C5 requests: `count` draws of (q, prp), q the smallest prime >= exp(U(ln lo,
    ln hi)), prp by a fair coin, random.Random(2)."""
    import bisect
    import math
    import random

    primes = primes_between(lo, hi + 100000)
    rng = random.Random(2)
    out = []
    for _ in range(count):
        x = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        out.append((primes[min(bisect.bisect_left(primes, int(x)), len(primes) - 1)], rng.random() < 0.5))
    return out


def reference_pins() -> dict:
    """(q, prp, iterations) -> Res64 of the reference build (tests/golden/ref_residues.json)."""
    return {(c["q"], bool(c["prp"]), c["iterations"]): c["res64"] for c in reference_residues()}


def plans_used(path: str):
    """The tuned plans the batch kept in its JSON cache, or None."""
    try:
        return json.loads(Path(path).read_text())["plans"] if path else None
    except (OSError, ValueError, KeyError):
        return None


def single_test_us(cuda_b200, exponents, prp: bool, device: int, iters: int = 1000) -> dict:
    """This repository's single-test path (one test alone, lnt_iterate), µs per
    squaring at each policy length of `exponents`: CUDA events around `iters`
    squarings of the first exponent of each length, after a warm-up call."""
    import torch

    out = {}
    for q in exponents:
        n = 1 << cuda_b200.secured_log2_length(q)
        if n in out:
            continue
        stream = torch.cuda.Stream(device=device)
        with cuda_b200.LucasTest(q, 0, prp, device=device) as t:
            t.set_stream(stream.cuda_stream)
            t.iterate(min(iters, 200))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t.iterate(iters)
            e1.record(stream)
            e1.synchronize()
            out[n] = e0.elapsed_time(e1) * 1e3 / iters
    return out


def run_batch_workload(args, exps, prp, target_of, label, config, rank=0, world=1, local_rank=0):
    """tests/hour of the batch engine over the whole work list, timed from the
    first submission to the last completion (wall clock around the engine's
    calls, which synchronise the device), with the autotuner on (plans cached
    in --plan-cache) and Res64 checkpoints every --checkpoint-every squarings.
    Every final Res64 and checkpoint that the reference build has a residue for
    is compared with it; a mismatch fails the run.  With N ranks (one process
    per GPU) each rank runs its own batch over a cost-balanced share of the
    work list (cuda_b200/shard.py); no collective touches the data path.

    The plain one-at-a-time path: --plain real runs every test alone through
    the single-test path (lnt_iterate) back to back; --plain per-length sums
    (squarings x µs per squaring alone at the test's length), that time
    measured once per length.  The reference build's plain time is the same sum
    over its own per-length time (tests/golden/ref_timings.json)."""
    import cuda_b200
    from cuda_b200 import shard

    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=3600))
    pins = reference_pins()
    mine = shard.partition_by_cost(exps, world, lambda q: shard.test_cost(q, target_of(q), prp))[rank]
    results, marks = {}, {}
    # the autotuner's one-time cost, outside the timed run: a scratch batch
    # admits the tests once (each new length and carry-run class is tuned) and
    # writes the plans to the cache, which the timed batch then loads
    tune_s = 0.0
    cache = args.plan_cache
    if cache and world > 1:
        cache = f"{cache}.rank{rank}"  # one file per process: the ranks tune and write concurrently
    if args.autotune_loops:
        import tempfile

        if not cache:
            cache = str(Path(tempfile.mkdtemp()) / f"plans_rank{rank}.json")
        tt = time.perf_counter()
        with cuda_b200.Batch(device=local_rank, autotune_loops=args.autotune_loops, plan_cache=cache,
                             autotune_group=args.autotune_group, short_lengths=args.short_lengths) as tb:
            for q in mine:
                tb.submit(q, 0, prp, target_of(q))
        tune_s = time.perf_counter() - tt
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    with cuda_b200.Batch(device=local_rank, autotune_loops=args.autotune_loops,
                         plan_cache=cache or None, checkpoint_every=args.checkpoint_every,
                         autotune_group=args.autotune_group, short_lengths=args.short_lengths) as b:
        ids = {b.submit(q, 0, prp, target_of(q)): q for q in mine}
        t_admitted = time.perf_counter() - t0
        while len(results) < len(ids):
            b.run(args.batch_step)
            for r in b.poll():
                results[r["id"]] = r
            for c in b.poll_checkpoints():
                marks[(ids[c["id"]], c["iteration"])] = c
    elapsed = time.perf_counter() - t0
    # parity: every pinned final residue and checkpoint
    checked, bad = 0, []
    for i, r in results.items():
        key = (ids[i], prp, r["iterations"])
        if r["status"] != 0:
            bad.append(("status", ids[i], r["status"]))
        elif key in pins:
            checked += 1
            if f"{r['res64']:016x}" != pins[key]:
                bad.append(("final", ids[i], f"{r['res64']:016x}", pins[key]))
    for (q, it), c in marks.items():
        key = (q, prp, it)
        if key in pins:
            checked += 1
            if c["status"] != 0 or f"{c['res64']:016x}" != pins[key]:
                bad.append(("checkpoint", q, it, f"{c['res64']:016x}", pins[key]))
    checked = sum(shard.gather_results([checked], dist))
    bad = shard.gather_results(bad, dist)
    n_done = sum(shard.gather_results([len(results)], dist))
    elapsed = shard.max_over_ranks(elapsed, dist)
    if rank == 0:
        lengths = {}
        for q in exps:
            n = cuda_b200.smallest_length(q) if args.short_lengths else 1 << cuda_b200.secured_log2_length(q)
            lengths[n] = lengths.get(n, 0) + 1
        alone = single_test_us(cuda_b200, sorted(exps), prp, local_rank)
        plain_kind = args.plain
        if plain_kind == "real":
            pt0 = time.perf_counter()
            for q in exps:
                with cuda_b200.LucasTest(q, 0, prp, device=local_rank) as t:
                    t.iterate(target_of(q))
                    r = t.res64()
                key = (q, prp, target_of(q))
                if key in pins and f"{r:016x}" != pins[key]:
                    bad.append(("plain", q, f"{r:016x}", pins[key]))
            plain_s = time.perf_counter() - pt0
        else:
            plain_s = sum(target_of(q) * alone[1 << cuda_b200.secured_log2_length(q)] * 1e-6 for q in exps)
        ref = reference_us_per_iteration()
        try:
            ref_plain_s = sum(target_of(q) * ref[1 << cuda_b200.secured_log2_length(q)] * 1e-6 for q in exps)
        except KeyError:
            ref_plain_s = None
        tph = n_done / elapsed * 3600
        line = {"metric": f"tests/hour, {label}", "value": tph, "unit": "tests/hour",
                "higher_is_better": True, "n_gpus": world, "data": "seeded exponents (no synthetic data)",
                "dtype": "u64", "config": config, "scaling": "strong" if world > 1 else "weak",
                "tests": len(exps), "finished": n_done, "wall_s": elapsed, "admission_s": t_admitted,
                "timing": "wall clock from the first submission to the last completion, max over ranks",
                "autotune_loops": args.autotune_loops, "autotune_group": args.autotune_group,
                "tuning_s": tune_s, "tuning": "before the timed run (plans cached in a JSON file)",
                "plans": plans_used(cache), "lengths": {str(k): v for k, v in sorted(lengths.items())},
                "short_lengths": args.short_lengths,
                "plain": plain_kind, "plain_s": plain_s, "plain_tests_per_hour": len(exps) / plain_s * 3600,
                "speedup_vs_plain": tph / (len(exps) / plain_s * 3600),
                "alone_us_per_squaring": {str(k): v for k, v in sorted(alone.items())},
                "reference_plain_s": ref_plain_s,
                "reference_plain_tests_per_hour": len(exps) / ref_plain_s * 3600 if ref_plain_s else None,
                "speedup_vs_reference_plain": tph / (len(exps) / ref_plain_s * 3600) if ref_plain_s else None,
                "parity": {"res64_checked_against_reference_build": checked, "mismatches": bad[:10],
                           "equal_reference_build": not bad}}
        print(json.dumps(line), flush=True)
        if bad:
            raise SystemExit(f"bench: {len(bad)} residues differ from the reference build: {bad[:3]}")
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


C1_EXPONENTS = [44497, 44501, 44507, 44519, 44531, 44533, 44537, 44543, 44549]
C2_PARITY_MARKS = (1000, 10000)


def reference_residues() -> list[dict]:
    """The reference build's residues (tests/golden/ref_residues.json)."""
    return json.loads((ROOT / "tests" / "golden" / "ref_residues.json").read_text())["cases"]


def c2_parity(test) -> dict:
    """Square the freshly initialised C2 test to 1,000 and then 10,000
    iterations and compare its Res64 with the reference build's at those
    marks.  A mismatch ends the run with an error: a time for a path whose
    residues differ from the reference's is not a result."""
    want = {c["iterations"]: c["res64"] for c in reference_residues()
            if c["q"] == EXPONENT and c["n"] == N and not c["prp"]}
    out, done = {}, 0
    for mark in C2_PARITY_MARKS:
        test.iterate(mark - done)
        done = mark
        got = f"{test.res64():016x}"
        out[f"res64_{mark // 1000}k"] = got
        if mark not in want:
            raise SystemExit(f"bench: no reference-build Res64 for q={EXPONENT} after {mark} squarings")
        if got != want[mark]:
            raise SystemExit(f"bench: Res64 after {mark} squarings is {got}, the reference build's is "
                             f"{want[mark]}: the timed path is not bit-exact")
    out["reference_res64"] = {f"{m // 1000}k": want[m] for m in C2_PARITY_MARKS}
    out["equal_reference_build"] = True
    return out


def run_c1(args):
    """Full LL of M_44497 and the next 8 prime exponents at the policy length
    (2048 words): each test alone through the single-test path, then all nine
    in one batch (one SMEM-resident launch).  Res64 checked against the
    committed fixture of the reference build's residues."""
    import cuda_b200

    want = {c["q"]: c["res64"] for c in reference_residues() if c["n"] == 2048 and not c["prp"]}
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
    """Serving: LL/PRP requests (the seeded C5 pool: q log-uniform in
    [1e4, 3e7], LL or PRP by a fair coin) arrive as a Poisson stream at each
    rate of --rates (requests per second) for --seconds; the continuous-batching
    engine admits them under a 150 GB HBM budget as they arrive and keeps every
    residue on the device until its verdict.  After the window the engine runs
    on for --drain seconds, then stops.  Latency = completion - arrival for the
    requests that finished; the others are counted as unfinished with their
    age at the stop (a lower bound on their latency) and are left out of the
    percentiles, which the line says.  The plain path is the same arrivals
    served one at a time in arrival order (FIFO) with service times = squarings
    x this repository's single-test µs per squaring at the request's length
    (measured once per length): a simulation, labelled as one.  Each engine
    call has a time budget (--step-seconds, lnt_batch_step_seconds): every
    launch group and resident test runs as many squarings as fit in it at its
    own pace, so new requests are admitted and finished ones retired about that
    often, and small tests are not held to the pace of large ones.  Every finished
    request whose full-test Res64 the reference build has is compared with it.
    With N ranks the stream's rate is N times higher and request i goes to rank
    i mod N (round-robin dispatch to one engine per GPU)."""
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
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=3600))

    lo, hi = (int(x) for x in args.c5_range.split(","))
    pool = c5_pool(lo, hi)
    pins = reference_pins()
    alone = single_test_us(cuda_b200, sorted({q for q, _ in pool}), False, local_rank, iters=200) if rank == 0 else {}
    rng = random.Random(2)
    budget = 150 << 30
    for rate in (float(r) for r in args.rates.split(",")):
        t, arrivals = 0.0, []
        while True:
            t += rng.expovariate(rate * world)
            if t >= args.seconds:
                break
            q, prp = pool[rng.randrange(len(pool))]
            arrivals.append((t, q, prp))
        mine = arrivals[rank::world]
        lat, unfinished, bad, checked = [], [], [], 0
        work_done = 0.0
        if dist is not None:
            dist.barrier()
        with cuda_b200.Batch(device=local_rank, hbm_budget_bytes=budget, step_seconds=args.step_seconds) as b:
            t0 = time.perf_counter()
            k, info = 0, {}
            stop = args.seconds + args.drain
            while time.perf_counter() - t0 < stop:
                now = time.perf_counter() - t0
                while k < len(mine) and mine[k][0] <= now:
                    i = b.enqueue(mine[k][1], 0, mine[k][2])
                    info[i] = mine[k]
                    k += 1
                if k >= len(mine) and not info:
                    break
                if not info:  # nothing in flight: wait for the next arrival
                    time.sleep(max(0.0, min(mine[k][0] - now, 0.05)))
                    continue
                b.run(args.batch_step if args.step_seconds <= 0 else 1 << 40)
                now = time.perf_counter() - t0
                for r in b.poll():
                    ta, q, prp = info.pop(r["id"])
                    lat.append(now - ta)
                    work_done += r["iterations"] * r["n"]
                    key = (q, prp, q if prp else q - 2)
                    if r["status"] != 0:
                        bad.append(("status", q, prp, r["status"]))
                    elif key in pins:
                        checked += 1
                        if f"{r['res64']:016x}" != pins[key]:
                            bad.append((q, prp, f"{r['res64']:016x}", pins[key]))
            wall = time.perf_counter() - t0
            unfinished = [wall - ta for ta, _, _ in info.values()]
        lat = shard.gather_results(lat, dist)
        unfinished = shard.gather_results(unfinished, dist)
        bad = shard.gather_results(bad, dist)
        checked = sum(shard.gather_results([checked], dist))
        wall = shard.max_over_ranks(wall, dist)
        if rank != 0:
            continue
        # plain path: FIFO over the same arrivals, one test at a time, stopped at the same time
        free_at, plain_lat, plain_unfinished = 0.0, [], []
        for (ta, q, prp) in arrivals:
            n = 1 << cuda_b200.secured_log2_length(q)
            start_t = max(free_at, ta)
            end_t = start_t + (q if prp else q - 2) * alone[n] * 1e-6
            if end_t <= wall:
                plain_lat.append(end_t - ta)
                free_at = end_t
            else:
                plain_unfinished.append(wall - ta)
                free_at = max(free_at, end_t)
        pct = lambda v, p: float(np.percentile(v, p)) if v else None  # noqa: E731
        lens = sorted({1 << cuda_b200.secured_log2_length(q) for _, q, _ in arrivals})
        line = {"metric": "serving p50/p99 latency and tests/hour", "rate_requests_per_s": rate * world,
                "requests": len(arrivals), "completed": len(lat), "unfinished": len(unfinished),
                "wall_s": wall, "n_gpus": world,
                "p50_s": pct(lat, 50), "p99_s": pct(lat, 99), "tests_per_hour": len(lat) / wall * 3600,
                "unfinished_age_s": {"min": min(unfinished) if unfinished else None,
                                     "max": max(unfinished) if unfinished else None},
                "percentiles": "over completed requests; unfinished requests are excluded (their latency "
                               "is at least their age at the stop)",
                "plain": "simulated FIFO, one test at a time, service = squarings x measured single-test "
                         "µs per squaring at the request's length",
                "plain_completed": len(plain_lat), "plain_unfinished": len(plain_unfinished),
                "plain_p50_s": pct(plain_lat, 50), "plain_p99_s": pct(plain_lat, 99),
                "plain_tests_per_hour": len(plain_lat) / wall * 3600,
                "lengths_requested": lens,
                "parity": {"res64_checked_against_reference_build": checked, "mismatches": bad[:10],
                           "equal_reference_build": not bad},
                "config": {"exponents": f"seeded pool of 64: q log-uniform in [{lo}, {hi}], LL/PRP by a "
                                        "fair coin (random.Random(2))", "window_s": args.seconds,
                           "drain_s": args.drain, "hbm_budget_gb": 150, "arrival": "Poisson",
                           "engine_call_budget_s": args.step_seconds,
                           "dispatch": "round-robin over ranks" if world > 1 else "one engine"}}
        print(json.dumps(line), flush=True)
        if bad:
            raise SystemExit(f"bench: serving residues differ from the reference build: {bad[:3]}")
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
            exps = c3_exponents()[:args.c3_count]
            run_batch_workload(args, exps, False, lambda q: q - 2,
                               f"{len(exps)} full LL tests, q in [1e5, 2e6] (seed 0)",
                               {"workload": "C3 batch", "count": len(exps), "lengths": "4K-128K",
                                "subset": "the first tests of the seeded sample" if len(exps) < 256 else "all"},
                               rank, world, local_rank)
        elif args.workload == "c4":
            exps = c4_exponents()
            run_batch_workload(args, exps, True, lambda q: 20000,
                               "64 PRP tests x 20000 squarings, q in [5e6, 2e7] (seed 1)",
                               {"workload": "C4 batch", "count": 64, "lengths": "256K-1M"},
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

    # parity of the timed path before timing: Res64 after 1,000 and 10,000
    # squarings against the reference build's residues of this exact test
    parity = c2_parity(test)

    # warm-up steps (untimed), continuing the same test
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
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    issue = issue_roofline(dom_name, avg_s, sms, (clk or {}).get("sm_mhz"))
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
            "parity": parity,
            "gpu_launches": launches_in_timed,
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "algo_bytes_per_launch": algo_bytes,
                         "avg_launch_us": avg_s * 1e6, "issue": issue},
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

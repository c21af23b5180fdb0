"""ctypes binding of liblucasntt.so (C ABI in include/lucasntt.h).

Python face of the reference's LucasPRP / NttLengths interface
(lucas_prp.cu, ntt_lengths.cu): create a test for an exponent, iterate,
read the residue back in the reference's dump order.  There is no CPU
fallback: if the shared library is missing the import fails loudly.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
# LUCASNTT_LIBRARY selects another build of the library (a tuned variant)
LIB_PATH = Path(os.environ["LUCASNTT_LIBRARY"]) if os.environ.get("LUCASNTT_LIBRARY") else _HERE / "liblucasntt.so"
HEADER = _HERE.parent / "include" / "lucasntt.h"

LNT_OK = 0
LNT_ERR_INVALID_ARGUMENT = 1
LNT_ERR_UNSUPPORTED_LENGTH = 2
LNT_ERR_CUDA = 3
LNT_ERR_OUT_OF_MEMORY = 4
LNT_ERR_NUMERIC = 5
LNT_ERR_NO_DEVICE = 6
LNT_ERR_BUDGET = 7

_lib = None


class KernelTime(ctypes.Structure):
    """lnt_kernel_time: per-kernel-kind CUDA-event totals."""
    _fields_ = [("name", ctypes.c_char * 32), ("launches", ctypes.c_uint32),
                ("total_ms", ctypes.c_float)]


class BatchResult(ctypes.Structure):
    """lnt_batch_result."""
    _fields_ = [("id", ctypes.c_uint64), ("iterations", ctypes.c_uint64), ("res64", ctypes.c_uint64),
                ("seconds", ctypes.c_double), ("exponent", ctypes.c_uint32), ("n", ctypes.c_uint32),
                ("prp", ctypes.c_int), ("is_prime", ctypes.c_int), ("status", ctypes.c_int)]


class BatchCheckpoint(ctypes.Structure):
    """lnt_batch_checkpoint."""
    _fields_ = [("id", ctypes.c_uint64), ("iteration", ctypes.c_uint64), ("res64", ctypes.c_uint64),
                ("status", ctypes.c_int)]


class PlanOptions(ctypes.Structure):
    """lnt_plan_options: kernel family (1 resident, 2 register passes, 3 radix-2),
    log2 n2, tile, largest pass radix (8/16), fused (1) or two launches (2)."""
    _fields_ = [("kind", ctypes.c_uint32), ("log2_rows", ctypes.c_uint32), ("tile", ctypes.c_uint32),
                ("radix", ctypes.c_uint32), ("fused", ctypes.c_uint32)]

    def as_tuple(self) -> tuple[int, int, int, int, int]:
        return int(self.kind), int(self.log2_rows), int(self.tile), int(self.radix), int(self.fused)


class LucasNTTError(RuntimeError):
    def __init__(self, status: int, where: str):
        L = lib()
        msg = L.lnt_status_string(status).decode()
        detail = L.lnt_last_error().decode()
        super().__init__(f"{where}: {msg}" + (f" ({detail})" if detail else ""))
        self.status = status


def lib() -> ctypes.CDLL:
    """Load liblucasntt.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C cuda_b200`")
    L = ctypes.CDLL(str(LIB_PATH))
    u32, u64, i32, vp, sz = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t
    cp = ctypes.c_char_p
    sigs = {
        "lnt_status_string": ([i32], cp),
        "lnt_last_error": ([], cp),
        "lnt_secured_log2_length": ([u32], u32),
        "lnt_length_candidates": ([u32, cp, sz], i32),
        "lnt_parse_length": ([cp, ctypes.POINTER(u32)], i32),
        "lnt_check_provided_length": ([u32, cp, ctypes.POINTER(i32)], i32),
        "lnt_smallest_length": ([u32, ctypes.POINTER(u32)], i32),
        "lnt_shifted_words": ([u32, u32, ctypes.POINTER(u32), ctypes.POINTER(u32)], i32),
        "lnt_create": ([u32, u32, i32, i32, ctypes.POINTER(vp)], i32),
        "lnt_create_with_plan": ([u32, u32, i32, i32, ctypes.POINTER(PlanOptions), ctypes.POINTER(vp)], i32),
        "lnt_get_plan": ([vp, ctypes.POINTER(PlanOptions)], i32),
        "lnt_plan_candidates": ([u32, u32, ctypes.POINTER(PlanOptions), i32, ctypes.POINTER(i32)], i32),
        "lnt_plan_describe": ([ctypes.POINTER(PlanOptions), u32, u32, cp, sz], i32),
        "lnt_autotune": ([u32, u32, i32, i32, u32, ctypes.POINTER(PlanOptions), ctypes.POINTER(ctypes.c_float),
                          i32, ctypes.POINTER(i32), ctypes.POINTER(i32)], i32),
        "lnt_destroy": ([vp], i32),
        "lnt_init_test": ([vp], i32),
        "lnt_iterate": ([vp, u64], i32),
        "lnt_set_digits": ([vp, vp, sz], i32),
        "lnt_get_digits": ([vp, vp, sz], i32),
        "lnt_res64": ([vp, ctypes.POINTER(u64)], i32),
        "lnt_is_prime": ([vp, ctypes.POINTER(i32)], i32),
        "lnt_get_length": ([vp, ctypes.POINTER(u32)], i32),
        "lnt_get_raw_state": ([vp, vp, sz], i32),
        "lnt_get_widths": ([vp, vp, sz], i32),
        "lnt_plan_name": ([vp, cp, sz], i32),
        "lnt_set_stream": ([vp, vp], i32),
        "lnt_synchronize": ([vp], i32),
        "lnt_profile_iterations": ([vp, u64, ctypes.POINTER(KernelTime), i32, ctypes.POINTER(i32)], i32),
        "lnt_test_device_bytes": ([u32, u32], u64),
        "lnt_batch_create": ([i32, u64, ctypes.POINTER(vp)], i32),
        "lnt_batch_destroy": ([vp], i32),
        "lnt_batch_submit": ([vp, u32, u32, i32, u64, ctypes.POINTER(u64)], i32),
        "lnt_batch_run": ([vp, u64], i32),
        "lnt_batch_enqueue": ([vp, u32, u32, i32, u64, ctypes.POINTER(u64)], i32),
        "lnt_batch_pending": ([vp, ctypes.POINTER(u32)], i32),
        "lnt_batch_poll": ([vp, ctypes.POINTER(BatchResult), i32, ctypes.POINTER(i32)], i32),
        "lnt_batch_status": ([vp, ctypes.POINTER(u32), ctypes.POINTER(u64)], i32),
        "lnt_batch_autotune": ([vp, u32], i32),
        "lnt_gerbicz_enable": ([vp, u32], i32),
        "lnt_gerbicz_stats": ([vp, ctypes.POINTER(u64), ctypes.POINTER(u64), ctypes.POINTER(u64)], i32),
        "lnt_debug_corrupt": ([vp, u32], i32),
        "lnt_debug_corrupt_add": ([vp, u32, ctypes.c_int64], i32),
        "lnt_batch_use_graphs": ([vp, i32], i32),
        "lnt_batch_short_lengths": ([vp, i32], i32),
        "lnt_batch_checkpoint_every": ([vp, u64], i32),
        "lnt_batch_autotune_group": ([vp, u32], i32),
        "lnt_batch_step_seconds": ([vp, ctypes.c_double], i32),
        "lnt_batch_poll_checkpoints": ([vp, ctypes.POINTER(BatchCheckpoint), i32, ctypes.POINTER(i32)], i32),
        "lnt_batch_plan_cache": ([vp, cp], i32),
        "lnt_arith_selftest": ([i32, ctypes.POINTER(u64), ctypes.POINTER(u64)], i32),
    }
    for name, (args, res) in sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _check(status: int, where: str) -> None:
    if status != LNT_OK:
        raise LucasNTTError(status, where)


def secured_log2_length(exponent: int) -> int:
    """NttLengths::GetNttSecuredLength (ntt_lengths.cu:88-98)."""
    return int(lib().lnt_secured_log2_length(exponent))


def smallest_length(exponent: int) -> int:
    """lnt_smallest_length: the smallest 2^k or 5 * 2^k length meeting the
    reference's bound (ntt_lengths.cu:94) that has a plan here."""
    n = ctypes.c_uint32()
    _check(lib().lnt_smallest_length(exponent, ctypes.byref(n)), "lnt_smallest_length")
    return n.value


def shifted_words(exponent: int, n: int) -> tuple[int, int]:
    """(count, first j) of the words where the reference's widths
    (pre_calculation.cu:35, evaluated in double) start word j one bit below
    ceil(qj/n), the bit its weight assumes; there the reference's residues are
    not those of M_q.  This library's widths are the exact integers.  Host only."""
    count, first = ctypes.c_uint32(), ctypes.c_uint32()
    _check(lib().lnt_shifted_words(exponent, n, ctypes.byref(count), ctypes.byref(first)),
           "lnt_shifted_words")
    return count.value, first.value


def length_candidates(exponent: int) -> list[str]:
    """NttLengths::GetCandidates (ntt_lengths.cu:100-128)."""
    buf = ctypes.create_string_buffer(1024)
    lib().lnt_length_candidates(exponent, buf, 1024)
    return [s for s in buf.value.decode().split(";") if s]


def parse_length(description: str) -> int:
    """NttLengths::StringToLengths + GetTotalLength (ntt_lengths.cu:32-75, :130-142)."""
    n = ctypes.c_uint32()
    _check(lib().lnt_parse_length(description.encode(), ctypes.byref(n)), "parse_length")
    return int(n.value)


def check_provided_length(exponent: int, description: str) -> int:
    """NttLengths::CheckProvidedLength (ntt_lengths.cu:77-86)."""
    d = ctypes.c_int()
    _check(lib().lnt_check_provided_length(exponent, description.encode(), ctypes.byref(d)),
           "check_provided_length")
    return int(d.value)


def plan_candidates(exponent: int, n: int = 0) -> list[tuple[int, int, int, int, int]]:
    """Every valid plan (kind, log2 n2, tile, radix, fused) for (q, n): lnt_plan_candidates."""
    buf = (PlanOptions * 128)()
    c = ctypes.c_int()
    _check(lib().lnt_plan_candidates(exponent, n, buf, 128, ctypes.byref(c)), "lnt_plan_candidates")
    return [buf[i].as_tuple() for i in range(min(c.value, 128))]


def plan_describe(plan: tuple[int, ...], exponent: int, n: int = 0) -> str:
    buf = ctypes.create_string_buffer(128)
    o = PlanOptions(*plan)
    _check(lib().lnt_plan_describe(ctypes.byref(o), exponent, n, buf, 128), "lnt_plan_describe")
    return buf.value.decode()


def arith_selftest(device: int = 0) -> int:
    """lnt_arith_selftest: the device modular arithmetic against the host build
    on edge and seeded random operands; returns the number of results checked
    and raises LucasNTTError (LNT_ERR_NUMERIC) on any mismatch."""
    checked, bad = ctypes.c_uint64(), ctypes.c_uint64()
    _check(lib().lnt_arith_selftest(device, ctypes.byref(checked), ctypes.byref(bad)), "lnt_arith_selftest")
    return int(checked.value)


def autotune(exponent: int, n: int = 0, prp: bool = False, device: int = 0, loops: int = 100):
    """lnt_autotune: [(plan, ms for `loops` squarings or -1)], index of the fastest."""
    tried = (PlanOptions * 128)()
    ms = (ctypes.c_float * 128)()
    c, b = ctypes.c_int(), ctypes.c_int()
    _check(lib().lnt_autotune(exponent, n, int(bool(prp)), device, loops, tried, ms, 128, ctypes.byref(c),
                              ctypes.byref(b)), "lnt_autotune")
    return [(tried[i].as_tuple(), float(ms[i])) for i in range(min(c.value, 128))], int(b.value)


class LucasTest:
    """One Lucas-Lehmer (prp=False) or base-3 PRP test of M = 2^exponent - 1."""

    def __init__(self, exponent: int, n: int = 0, prp: bool = False, device: int = 0,
                 plan: tuple[int, ...] | None = None):
        h = ctypes.c_void_p()
        if plan is None:
            _check(lib().lnt_create(exponent, n, int(bool(prp)), device, ctypes.byref(h)), "lnt_create")
        else:
            o = PlanOptions(*plan)
            _check(lib().lnt_create_with_plan(exponent, n, int(bool(prp)), device, ctypes.byref(o),
                                              ctypes.byref(h)), "lnt_create_with_plan")
        self._h = h
        self.exponent = int(exponent)
        self.prp = bool(prp)
        nn = ctypes.c_uint32()
        _check(lib().lnt_get_length(self._h, ctypes.byref(nn)), "lnt_get_length")
        self.n = int(nn.value)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().lnt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def init_test(self) -> None:
        _check(lib().lnt_init_test(self._h), "lnt_init_test")

    def iterate(self, iterations: int) -> None:
        _check(lib().lnt_iterate(self._h, int(iterations)), "lnt_iterate")

    def set_digits(self, digits) -> None:
        d = np.ascontiguousarray(digits, dtype=np.uint64)
        _check(lib().lnt_set_digits(self._h, d.ctypes.data, d.size), "lnt_set_digits")

    def digits(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.n, np.uint64)
        _check(lib().lnt_get_digits(self._h, out.ctypes.data, out.size), "lnt_get_digits")
        return out

    def res64(self) -> int:
        r = ctypes.c_uint64()
        _check(lib().lnt_res64(self._h, ctypes.byref(r)), "lnt_res64")
        return int(r.value)

    def is_prime(self) -> bool:
        r = ctypes.c_int()
        _check(lib().lnt_is_prime(self._h, ctypes.byref(r)), "lnt_is_prime")
        return bool(r.value)

    def raw_state(self) -> np.ndarray:
        """Internal signed words (diagnostic; see lnt_get_raw_state)."""
        out = np.empty(self.n, np.int64)
        _check(lib().lnt_get_raw_state(self._h, out.ctypes.data, out.size), "lnt_get_raw_state")
        return out

    def widths(self) -> np.ndarray:
        w = np.empty(self.n, np.uint8)
        _check(lib().lnt_get_widths(self._h, w.ctypes.data, w.size), "lnt_get_widths")
        return w

    @property
    def plan(self) -> str:
        buf = ctypes.create_string_buffer(64)
        _check(lib().lnt_plan_name(self._h, buf, 64), "lnt_plan_name")
        return buf.value.decode()

    def plan_options(self) -> tuple[int, int, int, int, int]:
        o = PlanOptions()
        _check(lib().lnt_get_plan(self._h, ctypes.byref(o)), "lnt_get_plan")
        return o.as_tuple()

    def gerbicz_enable(self, block: int) -> None:
        """Gerbicz-Li check for PRP tests: verify every block^2 squarings (0: off)."""
        _check(lib().lnt_gerbicz_enable(self._h, int(block)), "lnt_gerbicz_enable")

    def gerbicz_stats(self) -> dict:
        v, c, e = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().lnt_gerbicz_stats(self._h, ctypes.byref(v), ctypes.byref(c), ctypes.byref(e)),
               "lnt_gerbicz_stats")
        return {"verified_iterations": int(v.value), "checks": int(c.value), "errors": int(e.value)}

    def debug_corrupt(self, word: int = 1, delta: int = 1) -> None:
        """Test hook: add `delta` to one word of the device state (a simulated
        hardware error; a large delta makes the kernels raise the carry flag)."""
        _check(lib().lnt_debug_corrupt_add(self._h, int(word), int(delta)), "lnt_debug_corrupt_add")

    def set_stream(self, stream_handle: int | None) -> None:
        _check(lib().lnt_set_stream(self._h, stream_handle), "lnt_set_stream")

    def synchronize(self) -> None:
        _check(lib().lnt_synchronize(self._h), "lnt_synchronize")

    def profile_iterations(self, iterations: int) -> dict[str, tuple[int, float]]:
        """Squarings with CUDA events between launches: {kernel: (launches, total_ms)}."""
        cap = 16
        arr = (KernelTime * cap)()
        count = ctypes.c_int()
        _check(lib().lnt_profile_iterations(self._h, int(iterations), arr, cap, ctypes.byref(count)),
               "lnt_profile_iterations")
        return {arr[i].name.decode(): (int(arr[i].launches), float(arr[i].total_ms))
                for i in range(min(cap, count.value))}


def test_device_bytes(exponent: int, n: int = 0) -> int:
    """Device bytes one test occupies (the batch engine's budget unit)."""
    return int(lib().lnt_test_device_bytes(exponent, n))


class Batch:
    """Many LL / PRP tests on one GPU, admitted under an HBM budget and retired
    as they finish (lnt_batch_*).

    autotune_loops > 0 tunes each length's plan (lnt_batch_autotune), timing
    each candidate on `autotune_group` tests together, and `plan_cache` keeps
    the plans in a JSON file; checkpoint_every > 0 records Res64 checkpoints
    (poll_checkpoints); step_seconds > 0 gives every run() call a time budget
    split among the launch groups by their pace (lnt_batch_step_seconds);
    graphs=False replaces the captured-graph replay by plain launches."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, autotune_loops: int = 0,
                 graphs: bool = True, checkpoint_every: int = 0, plan_cache: str | None = None,
                 autotune_group: int = 1, step_seconds: float = 0.0, short_lengths: bool = False):
        h = ctypes.c_void_p()
        _check(lib().lnt_batch_create(device, int(hbm_budget_bytes), ctypes.byref(h)), "lnt_batch_create")
        self._h = h
        if plan_cache:
            _check(lib().lnt_batch_plan_cache(self._h, str(plan_cache).encode()), "lnt_batch_plan_cache")
        if autotune_loops:
            _check(lib().lnt_batch_autotune(self._h, int(autotune_loops)), "lnt_batch_autotune")
        if autotune_group > 1:
            _check(lib().lnt_batch_autotune_group(self._h, int(autotune_group)), "lnt_batch_autotune_group")
        if checkpoint_every:
            _check(lib().lnt_batch_checkpoint_every(self._h, int(checkpoint_every)), "lnt_batch_checkpoint_every")
        if step_seconds:
            _check(lib().lnt_batch_step_seconds(self._h, float(step_seconds)), "lnt_batch_step_seconds")
        if not graphs:
            _check(lib().lnt_batch_use_graphs(self._h, 0), "lnt_batch_use_graphs")
        if short_lengths:
            _check(lib().lnt_batch_short_lengths(self._h, 1), "lnt_batch_short_lengths")

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().lnt_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, exponent: int, n: int = 0, prp: bool = False, iterations: int = 0):
        """Admit a test; returns its id, or None when it does not fit the budget."""
        i = ctypes.c_uint64()
        st = lib().lnt_batch_submit(self._h, exponent, n, int(bool(prp)), int(iterations), ctypes.byref(i))
        if st == LNT_ERR_BUDGET:
            return None
        _check(st, "lnt_batch_submit")
        return int(i.value)

    def enqueue(self, exponent: int, n: int = 0, prp: bool = False, iterations: int = 0) -> int:
        """Queue a test; it is admitted when the budget allows.  Returns its id."""
        i = ctypes.c_uint64()
        _check(lib().lnt_batch_enqueue(self._h, exponent, n, int(bool(prp)), int(iterations),
                                       ctypes.byref(i)), "lnt_batch_enqueue")
        return int(i.value)

    def pending(self) -> int:
        c = ctypes.c_uint32()
        _check(lib().lnt_batch_pending(self._h, ctypes.byref(c)), "lnt_batch_pending")
        return int(c.value)

    def run(self, iterations: int) -> None:
        _check(lib().lnt_batch_run(self._h, int(iterations)), "lnt_batch_run")

    def poll(self) -> list[dict]:
        out = []
        buf = (BatchResult * 64)()
        while True:
            c = ctypes.c_int()
            _check(lib().lnt_batch_poll(self._h, buf, 64, ctypes.byref(c)), "lnt_batch_poll")
            for k in range(c.value):
                r = buf[k]
                out.append({"id": r.id, "exponent": r.exponent, "n": r.n, "prp": bool(r.prp),
                            "iterations": r.iterations, "res64": r.res64, "is_prime": bool(r.is_prime),
                            "status": r.status, "seconds": r.seconds})
            if c.value < 64:
                return out

    def poll_checkpoints(self) -> list[dict]:
        """Res64 checkpoints recorded since the last call: {id, iteration, res64, status}."""
        out = []
        buf = (BatchCheckpoint * 256)()
        while True:
            c = ctypes.c_int()
            _check(lib().lnt_batch_poll_checkpoints(self._h, buf, 256, ctypes.byref(c)), "lnt_batch_poll_checkpoints")
            out += [{"id": buf[k].id, "iteration": buf[k].iteration, "res64": buf[k].res64,
                     "status": buf[k].status} for k in range(c.value)]
            if c.value < 256:
                return out

    def status(self) -> tuple[int, int]:
        a, b = ctypes.c_uint32(), ctypes.c_uint64()
        _check(lib().lnt_batch_status(self._h, ctypes.byref(a), ctypes.byref(b)), "lnt_batch_status")
        return int(a.value), int(b.value)

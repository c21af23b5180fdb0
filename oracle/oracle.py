"""ctypes front end of the CPU oracle (oracle/lnt_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
baseline.  Only tests/, __graft_entry__.smoke() and the CPU legs of bench.py
import this module; the product path never does.

The oracle restates the reference's per-iteration arithmetic
(common/pre_calculation.cu:23-36 weights and widths, a radix-2 NTT over
554^((p-1)/n) roots, kernels/r2b.cu:25-50 carry, kernels/m2.cu:23-41 minus two)
and its length policy (ntt_lengths.cu:88-128).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "liblntoracle.so"
_lib = None

P = 0xFFFFFFFF00000001


def build(force: bool = False) -> Path:
    """Compile the oracle shared library in place (gcc + OpenMP)."""
    src = _HERE / "lnt_oracle.c"
    if force or not _LIB_PATH.exists() or _LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(_HERE), "liblntoracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(_LIB_PATH))
        u32, u64, vp = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p
        L.oracle_secured_log2.argtypes = [u32]
        L.oracle_secured_log2.restype = u32
        L.oracle_candidates.argtypes = [u32, ctypes.c_char_p, ctypes.c_size_t]
        L.oracle_candidates.restype = ctypes.c_int
        L.oracle_weights_widths.argtypes = [u32, u32, vp, vp, vp]
        L.oracle_create.argtypes = [u32, u32, ctypes.c_int]
        L.oracle_create.restype = vp
        L.oracle_destroy.argtypes = [vp]
        L.oracle_set_digits.argtypes = [vp, vp]
        L.oracle_get_digits.argtypes = [vp, vp]
        L.oracle_get_widths.argtypes = [vp, vp]
        L.oracle_set_widths.argtypes = [vp, vp]
        L.oracle_get_weights.argtypes = [vp, vp, vp]
        L.oracle_iterate.argtypes = [vp, u64]
        L.oracle_iterate.restype = ctypes.c_int
        L.oracle_res64.argtypes = [vp]
        L.oracle_res64.restype = u64
        L.oracle_res64_of.argtypes = [vp, vp, u32]
        L.oracle_res64_of.restype = u64
        L.oracle_is_prime.argtypes = [vp]
        L.oracle_is_prime.restype = ctypes.c_int
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_max_threads.restype = ctypes.c_int
        for name in ("oracle_gl_mul", "oracle_gl_add", "oracle_gl_sub", "oracle_gl_pow"):
            f = getattr(L, name)
            f.argtypes = [u64, u64]
            f.restype = u64
        L.oracle_gl_inv.argtypes = [u64]
        L.oracle_gl_inv.restype = u64
        _lib = L
    return _lib


def secured_log2(exponent: int) -> int:
    """NttLengths::GetNttSecuredLength (ntt_lengths.cu:88-98)."""
    return int(lib().oracle_secured_log2(exponent))


def candidates(exponent: int) -> list[str]:
    """NttLengths::GetCandidates (ntt_lengths.cu:100-128), same strings."""
    buf = ctypes.create_string_buffer(1024)
    lib().oracle_candidates(exponent, buf, 1024)
    return [s for s in buf.value.decode().split(";") if s]


def weights_widths(n: int, exponent: int):
    """calc_weights_widths (common/pre_calculation.cu:23-36)."""
    w = np.empty(n, np.uint64)
    uw = np.empty(n, np.uint64)
    widths = np.empty(n, np.uint8)
    lib().oracle_weights_widths(n, exponent, w.ctypes.data, uw.ctypes.data, widths.ctypes.data)
    return w, uw, widths


def set_threads(t: int) -> None:
    lib().oracle_set_threads(int(t))


def max_threads() -> int:
    return int(lib().oracle_max_threads())


class OracleTest:
    """One LL or PRP test on the CPU, mirroring LucasPRP (lucas_prp.cu:24-229)."""

    def __init__(self, exponent: int, n: int | None = None, prp: bool = False):
        if n is None:
            n = 1 << secured_log2(exponent)
        self.exponent, self.n, self.prp = int(exponent), int(n), bool(prp)
        self._h = lib().oracle_create(self.exponent, self.n, int(self.prp))
        if not self._h:
            raise ValueError(f"unsupported length {n}")

    def close(self):
        if self._h:
            lib().oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_digits(self, digits) -> None:
        d = np.ascontiguousarray(digits, dtype=np.uint64)
        assert d.size == self.n
        lib().oracle_set_digits(self._h, d.ctypes.data)

    def digits(self) -> np.ndarray:
        d = np.empty(self.n, np.uint64)
        lib().oracle_get_digits(self._h, d.ctypes.data)
        return d

    def widths(self) -> np.ndarray:
        w = np.empty(self.n, np.uint8)
        lib().oracle_get_widths(self._h, w.ctypes.data)
        return w

    def set_widths(self, widths) -> None:
        """Run on other digit widths (the exact-integer table where the
        reference's double one differs); not the reference's behaviour."""
        w = np.ascontiguousarray(widths, dtype=np.uint8)
        assert w.size == self.n
        lib().oracle_set_widths(self._h, w.ctypes.data)

    def iterate(self, k: int) -> None:
        if lib().oracle_iterate(self._h, int(k)) != 0:
            raise OverflowError("carry overflowed 64 bits")

    def res64(self) -> int:
        return int(lib().oracle_res64(self._h))

    def is_prime(self) -> bool:
        return bool(lib().oracle_is_prime(self._h))


def res64_of(digits, widths) -> int:
    d = np.ascontiguousarray(digits, dtype=np.uint64)
    w = np.ascontiguousarray(widths, dtype=np.uint8)
    return int(lib().oracle_res64_of(d.ctypes.data, w.ctypes.data, d.size))

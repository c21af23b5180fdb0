"""CPU: the C ABI library loads, exports every symbol include/*.h declares,
and reports the absence of a device instead of falling back to the CPU."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(lnt_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("lnt_create", "lnt_iterate", "lnt_get_digits", "lnt_set_digits", "lnt_res64",
                 "lnt_secured_log2_length", "lnt_length_candidates", "lnt_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol(lnt):
    L = lnt.lib()
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(ROOT / "cuda_b200" / "liblucasntt.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (lnt_\w+)", out))
    assert set(declared_symbols()) <= exported


def test_no_device_is_an_error_not_a_fallback(lnt):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(lnt.LucasNTTError) as e:
        lnt.LucasTest(44497)
    assert e.value.status == 6


def test_status_strings(lnt):
    L = lnt.lib()
    for s in range(8):
        assert L.lnt_status_string(s)
    assert L.lnt_status_string(0) == b"ok"


def test_device_arithmetic_host_build(tmp_path):
    """goldilocks.cuh / carry.cuh compiled for the host, checked exhaustively."""
    exe = tmp_path / "gl_selftest"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe),
                    str(ROOT / "tests" / "native" / "gl_selftest.cpp")], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout


def test_canonical_readout_host_build(tmp_path):
    """canon_core.cuh (the readout's per-block steps) against an exact
    sequential cyclic carry, on balanced, zero, all-maximal and sparse states."""
    exe = tmp_path / "canon_selftest"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I/usr/local/cuda/include", "-o", str(exe),
                    str(ROOT / "tests" / "native" / "canon_selftest.cpp")], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout


def test_register_ntt_host_build(tmp_path):
    """ntt_core.cuh: register NTTs of 1..64 points against a naive DFT, and every
    power-of-two shift against a 128-bit remainder."""
    exe = tmp_path / "ntt_selftest"
    subprocess.run(["g++", "-O1", "-std=c++17", "-ftemplate-depth=2000", "-o", str(exe),
                    str(ROOT / "tests" / "native" / "ntt_selftest.cpp")], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout


def test_new_entry_points_reject_null_handles(lnt):
    """The batch, plan-cache and Jacobi entry points return LNT_ERR_INVALID_ARGUMENT
    (1) for a null handle instead of dereferencing it (no device needed)."""
    L = lnt.lib()
    assert L.lnt_batch_step_seconds(None, 0.25) == 1
    assert L.lnt_batch_checkpoint_every(None, 100) == 1
    assert L.lnt_batch_autotune_group(None, 8) == 1
    assert L.lnt_batch_plan_cache(None, b"plans.json") == 1
    assert L.lnt_batch_poll_checkpoints(None, None, 0, None) == 1
    assert L.lnt_jacobi_enable(None, 1000) == 1
    assert L.lnt_jacobi_check(None, None) == 1
    assert L.lnt_jacobi_stats(None, None, None, None) == 1
    assert L.lnt_jacobi_of_digits(None, None, 0, 0, None) == 1
    assert L.lnt_batch_short_lengths(None, 1) == 1


def test_length_queries_reject_bad_arguments(lnt):
    """lnt_smallest_length and lnt_shifted_words are host-only: bad pointers,
    exponents and lengths are LNT_ERR_INVALID_ARGUMENT, an exponent past the
    largest length LNT_ERR_UNSUPPORTED_LENGTH."""
    import ctypes

    L = lnt.lib()
    n, c = ctypes.c_uint32(), ctypes.c_uint32()
    assert L.lnt_smallest_length(100003, None) == 1
    assert L.lnt_smallest_length(2, ctypes.byref(n)) == 1
    assert L.lnt_smallest_length(2**31 - 1, ctypes.byref(n)) == 2
    assert L.lnt_shifted_words(100003, 1 << 12, None, None) == 1
    assert L.lnt_shifted_words(100003, 3 << 12, ctypes.byref(c), None) == 1  # not a power of two
    assert L.lnt_shifted_words(100003, 1 << 27, ctypes.byref(c), None) == 1
    assert L.lnt_shifted_words(100003, 1 << 12, ctypes.byref(c), None) == 0 and c.value == 0

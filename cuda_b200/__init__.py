"""B200-native Lucas-Lehmer / PRP squaring loop (LucasNTT drop-in for that path).

The product is liblucasntt.so (CUDA for sm_100a behind the C ABI in
include/lucasntt.h); this package is its Python binding.
"""
from .api import (  # noqa: F401
    Batch,
    LucasNTTError,
    LucasTest,
    PlanOptions,
    arith_selftest,
    autotune,
    check_provided_length,
    length_candidates,
    lib,
    parse_length,
    plan_candidates,
    plan_describe,
    secured_log2_length,
    shifted_words,
    smallest_length,
    test_device_bytes,
)

"""CPU: the library's length policy equals the reference's (ntt_lengths.cu:32-128)."""
import random

import numpy as np

import pytest

from oracle import oracle as O


def test_secured_length_matches_oracle(lnt):
    rng = random.Random(5)
    qs = [33, 64, 89, 1000, 44497, 53248, 53249, 65536, 100000, 2000000, 5000000,
          20000000, 30000000, 139000003, 1 << 30, 2**31 - 1]
    qs += [rng.randrange(40, 2**31) for _ in range(2000)]
    for q in qs:
        assert lnt.secured_log2_length(q) == O.secured_log2(q), q


@pytest.mark.parametrize("q,log2n", [(44497, 11), (139000003, 23), (100000, 12), (2000000, 17),
                                     (5000000, 18), (20000000, 20), (10000, 9), (30000000, 21)])
def test_config_lengths(lnt, q, log2n):
    assert lnt.secured_log2_length(q) == log2n


def test_candidate_strings(lnt):
    for q in (44497, 139000003, 300000000, 600000000, 1100000000, 1000):
        assert lnt.length_candidates(q) == O.candidates(q)
    assert lnt.length_candidates(139000003) == [
        "8388608.000000", "2048.000000:4096.000000", "4096.000000:2048.000000",
        "256:256:128", "512:256:64"]


def test_parse_length(lnt):
    assert lnt.parse_length("4096") == 4096
    assert lnt.parse_length("8M") == 1 << 23
    assert lnt.parse_length("4K") == 4096
    assert lnt.parse_length("2048:4096") == 1 << 23
    assert lnt.parse_length("2048.000000:4096.000000") == 1 << 23
    with pytest.raises(lnt.LucasNTTError) as e:
        lnt.parse_length("3072")  # 3 * 2^10: valid in the reference, no kernel for it
    assert e.value.status == 2
    for bad in ("7", "9", "", "abc", "25"):
        with pytest.raises(lnt.LucasNTTError) as e:
            lnt.parse_length(bad)
        assert e.value.status == 1


def test_check_provided_length(lnt):
    assert lnt.check_provided_length(44497, "2048") == 0
    assert lnt.check_provided_length(44497, "4096") == -1
    assert lnt.check_provided_length(44497, "1024") == 1
    assert lnt.check_provided_length(139000003, "2048:4096") == 0


def _shifted_by_definition(q, n):
    """Words j > 0 whose start bit (the prefix sum of the double-precision
    widths of pre_calculation.cu:35) differs from floor(qj/n) + 1, the bit the
    weight formula of pre_calculation.cu:30-31 assumes."""
    j = np.arange(n + 1, dtype=np.float64)
    start = np.ceil(np.float64(q) * j / n)  # = the prefix sums of the widths
    widths = np.diff(start)
    assert widths.min() >= q // n and widths.max() <= q // n + 1
    k = np.arange(1, n, dtype=np.int64)
    at = (np.int64(q) * k) // n + 1
    return np.nonzero(start[1:n].astype(np.int64) != at)[0] + 1


@pytest.mark.parametrize("q,log2n,count,first", [(600000001, 25, 1, 23116289),
                                                 (1000000007, 25, 1, 21529527),
                                                 (300000007, 24, 0, 0), (139000003, 23, 0, 0)])
def test_shifted_words(lnt, q, log2n, count, first):
    """Past q*j = 2^53 the double widths start a word one bit below its weight's
    bit; the library lists exactly the words the definition gives."""
    want = _shifted_by_definition(q, 1 << log2n)
    assert lnt.shifted_words(q, 1 << log2n) == (len(want), int(want[0]) if len(want) else 0)
    assert (len(want), int(want[0]) if len(want) else 0) == (count, first)


def test_no_shifted_words_below_2e25(lnt):
    """q*j < 2^53 for every exponent a length below 2^25 takes (at most 30 bits a
    word): the double widths are exact there."""
    for log2n in range(2, 25):
        n = 1 << log2n
        q = min(30 * n - 1, 2**31 - 1) | 1
        assert q * n < 2**53
        assert lnt.shifted_words(q, n) == (0, 0)


def test_five_lengths(lnt):
    """5 * 2^k totals parse and have plans (13 <= k <= 24); 3 * 2^k has none."""
    assert lnt.parse_length("5120") == 5120 and lnt.parse_length("5:2048") == 10240
    assert "x5x" in lnt.plan_describe(lnt.plan_candidates(300007, 5 << 13)[0], 300007, 5 << 13)
    for n in (5 << 12, 5 << 25, 3 << 13):
        with pytest.raises(lnt.LucasNTTError) as e:
            lnt.plan_candidates(300007 if n < 1e6 else 1000000007, n)
        assert e.value.status == 2
    assert all(p[3] == 8 for p in lnt.plan_candidates(1000003, 5 << 15))  # radix-8 passes only


def test_smallest_length(lnt):
    """The smallest 2^k or 5 * 2^k length meeting the reference's bound: never
    above the reference's power of two, and 5 * 2^k for about a quarter of the
    exponents (q = 170000009: 5 * 2^21 where the reference takes 2^24)."""
    rng = random.Random(11)
    five = 0
    qs = [rng.randrange(100000, 2**30) for _ in range(500)]
    for q in qs:
        n = lnt.smallest_length(q)
        ref = 1 << O.secured_log2(q)
        assert n <= ref
        if n % 5 == 0:
            five += 1
            assert n * 8 == ref * 5  # between the failing 2^(k+2) and the reference's 2^(k+3)
        else:
            assert n == ref
    assert 0.1 < five / len(qs) < 0.5
    assert lnt.smallest_length(170000009) == 5 << 21 and lnt.smallest_length(139000003) == 1 << 23


def test_five_length_plans_at_every_k(lnt):
    """Every 5 * 2^k length, 13 <= k <= 24, has register-pass plans only (radix
    8), rows of 5 L words with 2^7 <= L <= 2^12 and columns 2^6 ... 2^12; the
    policy takes L = 2^11 where the columns allow (2^(k-6) below k = 17, 2^12 at
    k = 24)."""
    for k in range(13, 25):
        n = 5 << k
        q = 15 * n + 1  # 15-16 bits a word: within the bound at every k here
        plans = lnt.plan_candidates(q, n)
        assert plans and all(p[0] == 2 and p[3] == 8 for p in plans), k
        for p in plans:
            name = lnt.plan_describe(p, q, n)
            n2, rest = name.split("_")[1].split("x", 1)
            L = int(rest.split("x")[1])
            assert rest.startswith("5x") and int(n2) * 5 * L == n
            assert 64 <= int(n2) <= 4096 and 128 <= L <= 4096
        policy_L = int(lnt.plan_describe(plans[0], q, n).split("_")[1].split("x")[2])
        assert policy_L == (1 << min(11, k - 6) if k < 24 else 1 << 12), k

"""CPU: pin the oracle (oracle/lnt_oracle.c) before trusting it.

Pins: field arithmetic against Python integers; the IBDWT tables against the
reference's per-element formulas (common/pre_calculation.cu:23-36); whole
residues against the independent big-integer model and its committed
fixture; known Mersenne primes (public facts) end with residue 0 (LL) and 9
(PRP), the reference's verdict (lucas_prp.cu:169-176).
"""
import json
import random
from pathlib import Path

import numpy as np
import pytest

from oracle import bigint_model as B

P = 0xFFFFFFFF00000001
GOLDEN = Path(__file__).resolve().parent / "golden"
# exponents of known Mersenne primes small enough for the CPU suite
MERSENNE = [89, 107, 127, 521, 607, 1279, 2203, 2281, 3217, 4253, 4423]


def test_field_arithmetic(oracle_mod):
    L = oracle_mod.lib()
    rng = random.Random(1)
    vals = [0, 1, 2, P - 1, P - 2, P // 2, 2**32, 2**32 - 1, 2**63] + [rng.randrange(P) for _ in range(300)]
    for i, a in enumerate(vals):
        b = vals[(7 * i + 3) % len(vals)]
        assert L.oracle_gl_mul(a, b) == a * b % P
        assert L.oracle_gl_add(a, b) == (a + b) % P
        assert L.oracle_gl_sub(a, b) == (a - b) % P
    assert L.oracle_gl_pow(554, (P - 1) // 64) == 8
    assert L.oracle_gl_pow(7, (P - 1) // 192 * 5) == 2


@pytest.mark.parametrize("q,n", [(44497, 2048), (1009, 64), (139000003, 1 << 23)])
def test_weights_match_reference_formula(oracle_mod, q, n):
    w, uw, widths = oracle_mod.weights_widths(n, q)
    rng = random.Random(q)
    js = [0, 1, 2, n - 1] + [rng.randrange(n) for _ in range(40)]
    for j in js:
        if j == 0:
            assert w[0] == 1 and uw[0] == pow(n, P - 2, P)
            continue
        r = (q * j) & 0xFFFFFFFF & (n - 1)
        e = ((P - 1) // 192 // n) * 5 * (n - r)
        wj = pow(7, e, P)
        assert int(w[j]) == wj
        assert int(uw[j]) == pow(wj * n % P, P - 2, P)
    pos = [-(-q * j // n) for j in range(n + 1)]
    assert np.array_equal(widths, np.diff(np.array(pos, dtype=np.int64)).astype(np.uint8))


@pytest.mark.parametrize("q", [101, 1009, 4099, 9973])
@pytest.mark.parametrize("prp", [False, True])
def test_oracle_matches_bigint_model(oracle_mod, q, prp):
    n0 = 1 << oracle_mod.secured_log2(q)
    for n in (n0, 2 * n0):
        with oracle_mod.OracleTest(q, n, prp) as T:
            T.iterate(150)
            v = B.run(q, 150, prp)
            assert T.digits().tolist() == B.to_digits(v, q, n)


def test_oracle_matches_committed_bigint_fixture(oracle_mod):
    cases = json.loads((GOLDEN / "small_bigint.json").read_text())["cases"]
    for c in cases:
        with oracle_mod.OracleTest(c["q"], c["n"], c["prp"]) as T:
            T.iterate(c["iterations"])
            assert f"{T.res64():016x}" == c["res64"], c
            assert T.digits()[:4].tolist() == c["digits_head"], c


@pytest.mark.parametrize("q", MERSENNE)
def test_known_mersenne_primes(oracle_mod, q):
    with oracle_mod.OracleTest(q, prp=False) as T:
        T.iterate(q - 2)
        assert T.is_prime() and T.res64() == 0
    with oracle_mod.OracleTest(q, prp=True) as T:
        T.iterate(q)
        assert T.is_prime() and T.res64() == 9


@pytest.mark.parametrize("q", [101, 1009, 2003, 4099])
def test_composites_are_not_prime(oracle_mod, q):
    with oracle_mod.OracleTest(q, prp=False) as T:
        T.iterate(q - 2)
        assert not T.is_prime()


def test_zero_and_full_residues(oracle_mod):
    """Edge states: all-zero digits and all-full digits (the value M = 0 mod M)."""
    q = 1009
    n = 1 << oracle_mod.secured_log2(q)
    widths = B.widths(q, n)
    full = [(1 << w) - 1 for w in widths]
    for prp in (False, True):
        for start in ([0] * n, full):
            with oracle_mod.OracleTest(q, n, prp) as T:
                T.set_digits(start)
                T.iterate(3)
                v = B.run(q, 3, prp, start=B.from_digits(start, q, n))
                assert T.digits().tolist() == B.to_digits(v, q, n)


def test_c1_fixture_consistency():
    """The committed C1 fixture says exactly one exponent, 44497, is prime."""
    path = GOLDEN / "c1_oracle.json"
    if not path.exists():
        pytest.skip("c1 fixture not generated")
    cases = json.loads(path.read_text())["cases"]
    for c in cases:
        assert c["is_prime"] == (c["q"] == 44497)
        assert (c["res64"] == "0" * 16) == (c["q"] == 44497)


def test_oracle_fixtures_match_reference_build():
    """The C1 and C2 oracle fixtures agree with residues the reference's own
    build produced on a B200 (tests/golden/ref_residues.json)."""
    ref = json.loads((GOLDEN / "ref_residues.json").read_text())["cases"]
    c1 = {(c["q"], c["n"]): c["res64"] for c in json.loads((GOLDEN / "c1_oracle.json").read_text())["cases"]}
    c2 = json.loads((GOLDEN / "c2_oracle.json").read_text())["res64_after"]
    checked = 0
    for c in ref:
        if (c["q"], c["n"]) in c1 and c["iterations"] == c["q"] - 2 and not c["prp"]:
            assert c1[(c["q"], c["n"])] == c["res64"], c
            checked += 1
        elif c["q"] == 139000003 and not c["prp"] and str(c["iterations"]) in c2:
            assert c2[str(c["iterations"])] == c["res64"], c
            checked += 1
    assert checked >= 11
    assert {c["conclusion"] for c in ref if c["q"] == 44497 and not c["prp"]} == {"Prime"}
    assert {c["conclusion"] for c in ref if c["q"] == 44497 and c["prp"]} == {"Probably Prime"}


def test_oracle_matches_reference_build_prp_and_batch_pins(oracle_mod):
    """The oracle's PRP mode (s0 = 3, no -2, residue 9 for primes) and a C3
    batch exponent after 20,000 LL squarings, against the reference build's
    residues: full PRP tests of four serving-stream exponents (n = 512, 1024)
    and q = 100267 at n = 4096."""
    ref = json.loads((GOLDEN / "ref_residues.json").read_text())["cases"]
    cases = [c for c in ref if c["prp"] and c["iterations"] == c["q"] and c["q"] in (11863, 12799, 13381, 15727)]
    cases += [c for c in ref if c["q"] == 100267 and c["iterations"] == 20000 and not c["prp"]]
    assert len(cases) == 5
    oracle_mod.set_threads(oracle_mod.max_threads())
    for c in cases:
        with oracle_mod.OracleTest(c["q"], c["n"], c["prp"]) as T:
            T.iterate(c["iterations"])
            assert f"{T.res64():016x}" == c["res64"], c



@pytest.mark.parametrize("q,n,prp", [(3001, 320, False), (3001, 320, True), (20011, 2560, False),
                                     (100005, 10240, True), (100003, 10240, False)])
def test_five_length_oracle_matches_bigint_model(oracle_mod, q, n, prp):
    """The oracle's n = 5 * 2^k path (no reference counterpart: exact widths, a
    5-point step and five power-of-two transforms) gives the big-integer model's
    digits from a random state, q = 100005 (divisible by 5: words on whole bits)
    included."""
    import random

    rng = random.Random(q + n)
    v = rng.randrange((1 << q) - 1)
    with oracle_mod.OracleTest(q, n, prp) as O:
        assert O.widths().tolist() == B.widths(q, n)
        O.set_digits(np.array(B.to_digits(v, q, n), dtype=np.uint64))
        for k in (1, 2, 3):
            O.iterate(k)
            for _ in range(k):
                v = B.step(v, q, prp)
            assert O.digits().tolist() == B.to_digits(v, q, n), k


def test_five_length_oracle_known_prime(oracle_mod):
    with oracle_mod.OracleTest(9941, 640, False) as O:
        O.iterate(9939)
        assert O.is_prime() and O.res64() == 0

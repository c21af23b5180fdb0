"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Bar: bit-exact digits.  Small sizes compare every digit with the CPU oracle
(oracle/lnt_oracle.c) or the big-integer fixture; full sizes compare Res64
with committed fixtures and use size-independent properties (split
iterations, set/get round trips, canonical digit ranges).
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import bigint_model as B

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
MERSENNE = [89, 107, 127, 521, 607, 1279, 2203, 2281, 3217, 4253, 4423, 9689, 9941, 11213]


def random_digits(q, n, seed):
    rng = np.random.default_rng(seed)
    w = np.array(B.widths(q, n), dtype=np.uint64)
    return (rng.integers(0, 2**62, size=n, dtype=np.uint64) % (np.uint64(1) << w)).astype(np.uint64)


def compare_with_oracle(lnt, oracle_mod, q, n, prp, iterations, start=None, steps=None):
    with lnt.LucasTest(q, n, prp) as G, oracle_mod.OracleTest(q, n, prp) as O:
        if start is not None:
            G.set_digits(start)
            O.set_digits(start)
        for k in (steps or [iterations]):
            G.iterate(k)
            O.iterate(k)
        g, o = G.digits(), O.digits()
        bad = np.nonzero(g != o)[0]
        assert bad.size == 0, f"q={q} n={n} prp={prp} first mismatch at {bad[:5]}: {g[bad[:5]]} vs {o[bad[:5]]}"
        assert G.res64() == O.res64()
        return G.plan


@pytest.mark.parametrize("q", MERSENNE)
def test_known_primes_resident(lnt, q):
    with lnt.LucasTest(q, prp=False) as T:
        T.iterate(q - 2)
        assert T.is_prime() and T.res64() == 0
    with lnt.LucasTest(q, prp=True) as T:
        T.iterate(q)
        assert T.is_prime() and T.res64() == 9


def test_bigint_fixture(lnt):
    cases = json.loads((GOLDEN / "small_bigint.json").read_text())["cases"]
    for c in cases:
        with lnt.LucasTest(c["q"], c["n"], c["prp"]) as T:
            T.iterate(c["iterations"])
            assert f"{T.res64():016x}" == c["res64"], c
            assert T.digits()[:4].tolist() == c["digits_head"], c


@pytest.mark.parametrize("q,n", [(89, 4), (127, 8), (1009, 64), (9973, 512), (44497, 2048),
                                 (44497, 4096), (53239, 2048), (100003, 4096)])
@pytest.mark.parametrize("prp", [False, True])
def test_resident_random_state(lnt, oracle_mod, q, n, prp):
    """Random canonical digits at the top of their range, several squarings."""
    plan = compare_with_oracle(lnt, oracle_mod, q, n, prp, 0, start=random_digits(q, n, q + n),
                               steps=[1, 4])
    assert plan.startswith("RESIDENT")


@pytest.mark.parametrize("q,n", [(160001, 8192), (300007, 16384), (1000003, 65536),
                                 (2000003, 131072), (5000011, 262144), (20000003, 1 << 20)])
def test_twopass_random_state(lnt, oracle_mod, q, n):
    plan = compare_with_oracle(lnt, oracle_mod, q, n, False, 0, start=random_digits(q, n, q),
                               steps=[1, 2])
    assert plan.startswith("TWOPASS")


@pytest.mark.parametrize("prp", [False, True])
def test_twopass_from_start_value(lnt, oracle_mod, prp):
    compare_with_oracle(lnt, oracle_mod, 160001, 8192, prp, 0, steps=[1, 1, 30])


def test_c2_first_iterations(lnt, oracle_mod):
    """q = 139000003 at the reference's length 2^23: bit-exact after 2 squarings."""
    compare_with_oracle(lnt, oracle_mod, 139000003, 1 << 23, False, 0, steps=[1, 1])


def test_c2_res64_fixture(lnt):
    path = GOLDEN / "c2_oracle.json"
    if not path.exists():
        pytest.skip("c2 fixture not generated")
    fx = json.loads(path.read_text())
    with lnt.LucasTest(fx["q"], fx["n"], False) as T:
        done = 0
        for mark in sorted(int(k) for k in fx["res64_after"]):
            T.iterate(mark - done)
            done = mark
            assert f"{T.res64():016x}" == fx["res64_after"][str(mark)], mark


def test_c1_full_tests(lnt):
    path = GOLDEN / "c1_oracle.json"
    if not path.exists():
        pytest.skip("c1 fixture not generated")
    for c in json.loads(path.read_text())["cases"]:
        with lnt.LucasTest(c["q"], c["n"], False) as T:
            T.iterate(c["iterations"])
            assert f"{T.res64():016x}" == c["res64"], c
            assert T.is_prime() == c["is_prime"], c


@pytest.mark.parametrize("q,n", [(1009, 64), (44497, 2048), (160001, 8192)])
def test_split_iterations_equal_one_call(lnt, q, n):
    with lnt.LucasTest(q, n) as A, lnt.LucasTest(q, n) as Bt:
        A.iterate(37)
        for k in (1, 5, 10, 21):
            Bt.iterate(k)
        assert np.array_equal(A.digits(), Bt.digits())


@pytest.mark.parametrize("q,n", [(1009, 64), (160001, 8192)])
def test_set_get_round_trip(lnt, q, n):
    d = random_digits(q, n, 7)
    with lnt.LucasTest(q, n) as T:
        T.set_digits(d)
        assert np.array_equal(T.digits(), d)
        T.iterate(3)
        out = T.digits()
        assert np.all(out < (np.uint64(1) << T.widths().astype(np.uint64)))


@pytest.mark.parametrize("q,n", [(1009, 64), (4099, 256), (160001, 8192)])
@pytest.mark.parametrize("prp", [False, True])
def test_zero_and_full_residues(lnt, oracle_mod, q, n, prp):
    """All-zero and all-full (= M) starts exercise the 0 / M choice and the
    long borrow chains of the canonical readout."""
    widths = B.widths(q, n)
    full = np.array([(1 << w) - 1 for w in widths], dtype=np.uint64)
    for start in (np.zeros(n, np.uint64), full):
        compare_with_oracle(lnt, oracle_mod, q, n, prp, 0, start=start, steps=[1, 2])


def test_two_pass_known_prime(lnt):
    """M_132049 is prime; its length 8192 runs on the two-pass plan."""
    with lnt.LucasTest(132049, prp=False) as T:
        assert T.plan.startswith("TWOPASS")
        T.iterate(132049 - 2)
        assert T.is_prime()


def _reference_cases():
    return json.loads((GOLDEN / "ref_residues.json").read_text())["cases"]


def test_reference_build_residues(lnt):
    """Res64 equal to the reference's own build (run on a B200), each test
    alone: C1 full LL tests at n = 2048 and 4096; q = 139000003 after 1,000 and
    10,000 LL squarings and 1,000 PRP squarings at n = 2^23; full PRP tests of
    Mersenne primes (residue 9) and composites on the resident and two-pass
    plans; one C4 exponent per length (PRP, 20,000 squarings); the C3 full LL
    tests up to 32K words; 1,000 squarings at 2^24 (LL and PRP) and 2^26.  The
    2^25 case (q = 600000001) has a shifted word: test_true_residues."""
    cases = _reference_cases()
    c2 = sorted((c for c in cases if c["q"] == 139000003 and not c["prp"]), key=lambda c: c["iterations"])
    c4_lengths = {}
    for c in cases:
        if c.get("set") == "c4":
            c4_lengths.setdefault(c["n"], c)
    alone_cases = [c for c in cases if c.get("set") in (None, "prp", "large") and c not in c2
                   and not c.get("shifted_words")]
    alone_cases += list(c4_lengths.values())
    alone_cases += [c for c in cases if c.get("set") == "c3_full" and c["n"] <= 32768]
    assert len(c4_lengths) == 3 and sum(c["prp"] for c in alone_cases) >= 9
    for c in alone_cases:
        with lnt.LucasTest(c["q"], c["n"], c["prp"]) as T:
            T.iterate(c["iterations"])
            assert f"{T.res64():016x}" == c["res64"], c
            assert T.is_prime() == (c["conclusion"] in ("Prime", "Probably Prime")), c
    with lnt.LucasTest(139000003, 1 << 23, False) as T:
        done = 0
        for c in c2:
            T.iterate(c["iterations"] - done)
            done = c["iterations"]
            assert f"{T.res64():016x}" == c["res64"], c


def test_true_residues(lnt):
    """Where the reference's double-precision widths start a word one bit below
    the bit its weight assumes (q = 600000001 at n = 2^25: j = 23116289), the
    reference squares another number and its Res64 is not that of M_q.  This
    library's widths are the exact integers: Res64 equals GMP's big-integer LL
    sequence (true_residues.json) and differs from the reference build's."""
    fx = json.loads((GOLDEN / "true_residues.json").read_text())["cases"]
    ref = {(c["q"], c["n"], c["prp"], c["iterations"]): c["res64"] for c in _reference_cases()}
    for c in fx:
        q, n = c["q"], c["n"]
        count, first = lnt.shifted_words(q, n)
        assert count > 0
        with lnt.LucasTest(q, n, c["prp"]) as T:
            # exact widths; the reference's double table differs at (first - 1, first)
            j = np.arange(n + 1, dtype=np.uint64)
            exact = np.diff((np.uint64(q) * j + np.uint64(n - 1)) // np.uint64(n))
            theirs = np.diff(np.ceil(np.float64(q) * j.astype(np.float64) / n))
            assert np.array_equal(T.widths(), exact.astype(np.uint8))
            assert exact[first - 1] != theirs[first - 1] and exact[first] != theirs[first]
            done = 0
            for mark in sorted(int(k) for k in c["res64_after"]):
                T.iterate(mark - done)
                done = mark
                got = f"{T.res64():016x}"
                assert got == c["res64_after"][str(mark)], (c["q"], mark, got)
                assert got != ref.get((c["q"], c["n"], c["prp"], mark)), "the reference's residue"


def test_reference_build_residues_in_one_batch(lnt):
    """Every pinned reference-build residue at once in one batch: resident,
    two-pass and carry-fused plans, LL and PRP mixed -- the nine C1 tests, the
    64 C4 PRP tests (20,000 squarings), the 256 C3 exponents (20,000 LL
    squarings) and one full C3 test per length, the serving stream's full tests
    up to q = 610,000, the PRP full tests, the C2 exponent (1,000 squarings LL
    and PRP) and 1,000 squarings at 2^24 and 2^26.  Each Res64 equals the
    reference build's."""
    cases = [c for c in _reference_cases() if not (c["q"] == 139000003 and c["iterations"] == 10000)
             and not c.get("shifted_words")]
    want = {}
    with lnt.Batch(device=0) as b:
        for c in cases:
            i = b.submit(c["q"], c["n"], c["prp"], c["iterations"])
            want[i] = c
        got = {}
        for _ in range(2000):
            b.run(4000)
            for r in b.poll():
                got[r["id"]] = r
            if len(got) == len(want):
                break
        assert b.status()[0] == 0
    assert set(got) == set(want)
    bad = [(want[i]["q"], want[i]["n"], want[i]["prp"], want[i]["iterations"])
           for i, r in got.items() if r["status"] != 0 or f"{r['res64']:016x}" != want[i]["res64"]]
    assert not bad, bad[:10]


def test_device_arithmetic_against_host(lnt):
    """The device reductions (multiplier-pipe sums, canonical step, shift
    twiddles, digit products) equal the host build on edge operands that reach
    their rare branches and on seeded random operands."""
    checked = lnt.arith_selftest(0)
    assert checked == (25 * 25 + 3 * 8192) * 16

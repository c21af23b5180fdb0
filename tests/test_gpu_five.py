"""GPU: lengths n = 5 * 2^k (rows of five stride-5 planes and a radix-5 step).

The reference has no kernel for any non-power-of-two length, so there is no
reference residue to pin; the checks are the big-integer model (digit for
digit), known Mersenne primes, and the length independence of the residue:
the same test at 5 * 2^k and at a power of two gives the same Res64.
"""
import numpy as np
import pytest

from oracle import bigint_model as B

pytestmark = pytest.mark.gpu


def to_digits(v, q, n):
    """bigint_model.to_digits, vectorised: digit j = bits [pos_j, pos_j + w_j)."""
    w = np.array(B.widths(q, n), dtype=np.uint64)
    pos = np.concatenate([[0], np.cumsum(w)[:-1]]).astype(np.uint64)
    raw = np.frombuffer(v.to_bytes((q + 7) // 8 + 8, "little"), dtype=np.uint8)
    idx = (pos // np.uint64(8)).astype(np.int64)[:, None] + np.arange(8)
    words = np.zeros(n, dtype=np.uint64)
    for b in range(8):
        words |= raw[idx[:, b]].astype(np.uint64) << np.uint64(8 * b)
    return (words >> (pos % np.uint64(8))) & ((np.uint64(1) << w) - np.uint64(1))


def random_value(q, seed):
    rng = np.random.default_rng(seed)
    return int.from_bytes(rng.bytes((q + 7) // 8), "little") % ((1 << q) - 1)


@pytest.mark.parametrize("q,n", [(300007, 5 << 13), (1000003, 5 << 15), (4000037, 5 << 17)])
@pytest.mark.parametrize("prp", [False, True])
def test_digits_equal_bigint_model(lnt, q, n, prp):
    """Random canonical state, then 1, 2 and 5 squarings: every digit equal to
    the model's (exact integer squaring mod M with the reference's carry)."""
    v = random_value(q, q + n)
    with lnt.LucasTest(q, n, prp) as T:
        assert "x5x" in T.plan
        T.set_digits(to_digits(v, q, n))
        for k in (1, 2, 5):
            T.iterate(k)
            for _ in range(k):
                v = B.step(v, q, prp)
            want = to_digits(v, q, n)
            got = T.digits()
            bad = np.nonzero(got != want)[0]
            assert bad.size == 0, (q, n, prp, k, bad[:5])
            assert T.res64() == B.res64(v)


@pytest.mark.parametrize("q,n,prp", [(216091, 5 << 13, False), (216091, 5 << 13, True)])
def test_known_primes(lnt, q, n, prp):
    with lnt.LucasTest(q, n, prp) as T:
        T.iterate(q if prp else q - 2)
        assert T.is_prime() and T.res64() == (9 if prp else 0)


def test_every_plan_of_a_length_agrees(lnt):
    q, n = 1000003, 5 << 15
    plans = lnt.plan_candidates(q, n)
    assert len(plans) > 2
    got = set()
    for p in plans:
        with lnt.LucasTest(q, n, False, plan=p) as T:
            T.iterate(50)
            got.add(T.res64())
    assert len(got) == 1


def test_same_residue_as_the_power_of_two_length(lnt):
    """q = 170000009: the smallest length is 5 * 2^21 (the reference takes 2^24);
    1,000 squarings give the Res64 of the 2^24 test."""
    q = 170000009
    assert lnt.smallest_length(q) == 5 << 21
    res = []
    for n in (5 << 21, 1 << 24):
        with lnt.LucasTest(q, n, False) as T:
            T.iterate(1000)
            res.append(T.res64())
    assert res[0] == res[1]


def test_in_a_batch_and_with_the_gerbicz_check(lnt):
    q, n = 1000003, 5 << 15
    with lnt.LucasTest(q, n, True) as T:
        T.iterate(3000)
        alone = T.res64()
    with lnt.LucasTest(q, n, True) as T:
        T.gerbicz_enable(20)  # a check every 400 squarings
        T.iterate(3000)
        assert T.res64() == alone
        st = T.gerbicz_stats()
        assert st["checks"] >= 7 and st["errors"] == 0
    with lnt.Batch(device=0) as b:
        ids = [b.submit(q, n, True, 3000), b.submit(q, 1 << 16, True, 3000), b.submit(300007, 5 << 13, False, 3000)]
        got = {}
        for _ in range(100):
            b.run(1000)
            for r in b.poll():
                got[r["id"]] = r
            if len(got) == len(ids):
                break
    assert got[ids[0]]["res64"] == alone and got[ids[1]]["res64"] == alone
    with lnt.LucasTest(300007, 5 << 13, False) as T:
        T.iterate(3000)
        assert got[ids[2]]["res64"] == T.res64()


def test_short_length_batch_matches_reference_pins(lnt):
    """A batch with short lengths on runs the C4 exponents whose smallest length is
    5 * 2^k (327,680 or 655,360 words instead of the reference's 2^19 / 2^20) and
    gives the reference build's Res64 after 20,000 PRP squarings."""
    import json
    from pathlib import Path

    cases = json.loads((Path(__file__).resolve().parent / "golden" / "ref_residues.json").read_text())["cases"]
    c4 = [c for c in cases if c.get("set") == "c4" and lnt.smallest_length(c["q"]) % 5 == 0][:8]
    assert len(c4) == 8
    with lnt.Batch(device=0, short_lengths=True) as b:
        want = {b.submit(c["q"], 0, True, c["iterations"]): c for c in c4}
        got = {}
        for _ in range(200):
            b.run(4000)
            for r in b.poll():
                got[r["id"]] = r
            if len(got) == len(want):
                break
    assert set(got) == set(want)
    for i, r in got.items():
        assert r["n"] == lnt.smallest_length(want[i]["q"]) < want[i]["n"]
        assert r["status"] == 0 and f"{r['res64']:016x}" == want[i]["res64"], want[i]


def test_batched_rows_per_cta(lnt, tmp_path):
    """Twelve tests of one 5 * 2^15 plan with rows of 640 words (forced through a
    plan cache) run as one launch group whose row kernel packs four rows per CTA;
    every residue equals the test alone (one row per CTA, the policy's plan)."""
    import json

    import torch

    n = 5 << 15
    cache = tmp_path / "plans.json"
    cache.write_text(json.dumps({"device": torch.cuda.get_device_name(0), "plans": [
        {"n": n, "run": 8, "kind": 2, "log2_rows": 8, "tile": 8, "radix": 8, "fused": 2, "ms": 1}]}))
    qs = [1000003 + 2 * i for i in range(12)]
    with lnt.Batch(device=0, autotune_loops=5, plan_cache=str(cache)) as b:
        ids = {b.submit(q, n, False, 30): q for q in qs}
        got = {}
        while len(got) < len(ids):
            b.run(30)
            got.update({r["id"]: r for r in b.poll()})
    for i, q in ids.items():
        with lnt.LucasTest(q, n, False) as T:
            T.iterate(30)
            assert got[i]["status"] == 0 and got[i]["res64"] == T.res64(), q


def test_every_row_length(lnt):
    """n = 5 * 2^18: every plan, rows of 5 L words for L = 256 ... 4096 (the
    largest, 174 KB of planes and 1024 threads a CTA), gives one Res64, which is
    the Res64 of the same test at 2^21."""
    q, n = 20000003, 5 << 18
    plans = lnt.plan_candidates(q, n)
    assert {p[1] for p in plans} >= {6, 10}  # n2 = 64 (L = 4096) ... 1024 (L = 256)
    got = set()
    for p in plans:
        with lnt.LucasTest(q, n, False, plan=p) as T:
            T.iterate(30)
            got.add(T.res64())
    with lnt.LucasTest(q, 1 << 21, False) as T:
        T.iterate(30)
        assert got == {T.res64()}


@pytest.mark.parametrize("q,n", [(1000005, 5 << 15), (1000006, 1 << 16)])
def test_exponents_sharing_a_factor_with_the_length(lnt, q, n):
    """q divisible by 5 at n = 5 * 2^k (and an even q at 2^k) puts some words
    j > 0 exactly on a whole bit (qj = 0 mod n); their weight is 1.  Digits equal
    the big-integer model after 1, 2 and 5 squarings (PRP: any exponent)."""
    v = random_value(q, q)
    with lnt.LucasTest(q, n, True) as T:
        T.set_digits(to_digits(v, q, n))
        for k in (1, 2, 5):
            T.iterate(k)
            for _ in range(k):
                v = B.step(v, q, True)
            assert np.array_equal(T.digits(), to_digits(v, q, n)), (q, n, k)


@pytest.mark.parametrize("q,n,prp", [(300007, 5 << 13, False), (1000005, 5 << 15, True),
                                     (2000003, 5 << 16, False)])
def test_digits_equal_oracle(lnt, oracle_mod, q, n, prp):
    """Digit for digit against the oracle's 5 * 2^k path after 1 and 3 squarings
    from a random canonical state."""
    start = to_digits(random_value(q, n), q, n)
    with lnt.LucasTest(q, n, prp) as T, oracle_mod.OracleTest(q, n, prp) as O:
        T.set_digits(start)
        O.set_digits(start)
        for k in (1, 3):
            T.iterate(k)
            O.iterate(k)
            assert np.array_equal(T.digits(), O.digits()), (q, n, prp, k)
        assert T.res64() == O.res64()

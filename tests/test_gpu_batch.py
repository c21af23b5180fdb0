"""GPU: the batch engine (lnt_batch_*) gives every test the residue it gets alone.

Tests of mixed lengths share batched launches (two-pass groups by length, one
SMEM-resident launch for all n <= 4096); results must equal the single-test
path bit for bit, and known Mersenne primes must come out prime.
"""
import pytest

pytestmark = pytest.mark.gpu

# (exponent, length (0 = policy), prp, iterations)
MIX = [(9973, 0, False, 300), (44497, 0, False, 250), (44501, 4096, True, 200),
       (100003, 0, False, 180), (160001, 0, True, 150), (160009, 0, False, 150),
       (300007, 0, False, 120), (1000003, 0, True, 90), (1000033, 0, False, 97),
       (5000011, 0, False, 40), (20000003, 0, True, 25)]


def alone(lnt, q, n, prp, k):
    with lnt.LucasTest(q, n, prp) as t:
        t.iterate(k)
        return t.res64()


@pytest.mark.parametrize("graphs,tune", [(True, 0), (False, 0), (True, 20)])
def test_batch_equals_alone(lnt, graphs, tune):
    """Captured-graph replay, plain launches and autotuned plans all give the
    single-test residues."""
    expected = {}
    with lnt.Batch(device=0, autotune_loops=tune, graphs=graphs) as b:
        for q, n, prp, k in MIX:
            i = b.submit(q, n, prp, k)
            expected[i] = alone(lnt, q, n, prp, k)
        got = {}
        for _ in range(400):
            b.run(37)
            for r in b.poll():
                assert r["status"] == 0, r
                got[r["id"]] = r
            if len(got) == len(MIX):
                break
        assert b.status()[0] == 0
    assert set(got) == set(expected)
    for i, r in got.items():
        assert r["res64"] == expected[i], r


def test_batch_full_known_primes(lnt):
    """Full LL and PRP tests of Mersenne primes across both plans, in one batch."""
    primes = [9689, 9941, 11213, 21701, 23209, 44497, 86243, 110503, 132049]
    with lnt.Batch(device=0) as b:
        for q in primes:
            b.submit(q, 0, False)
            b.submit(q, 0, True)
        done = []
        while len(done) < 2 * len(primes):
            b.run(5000)
            done += b.poll()
    for r in done:
        assert r["status"] == 0 and r["is_prime"], r
        assert r["res64"] == (9 if r["prp"] else 0), r
        assert r["iterations"] == (r["exponent"] if r["prp"] else r["exponent"] - 2)


def test_batch_budget_admission_and_refill(lnt):
    """A budget for two 1M-word tests admits two; a third waits until one retires."""
    q = 20000003
    per = lnt.test_device_bytes(q)
    with lnt.Batch(device=0, hbm_budget_bytes=2 * per + per // 2) as b:
        a1 = b.submit(q, 0, False, 5)
        a2 = b.submit(q + 30, 0, False, 9)
        assert a1 is not None and a2 is not None
        assert b.submit(q + 66, 0, False, 5) is None
        b.run(5)
        first = b.poll()
        assert [r["id"] for r in first] == [a1]
        a3 = b.submit(q + 66, 0, False, 5)
        assert a3 is not None
        b.run(10)
        rest = {r["id"]: r for r in b.poll()}
        assert set(rest) == {a2, a3}
        assert rest[a3]["res64"] == alone(lnt, q + 66, 0, False, 5)
        assert b.status() == (0, 0)

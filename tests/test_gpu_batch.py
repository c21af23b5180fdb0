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


def _primes_from(lo, count):
    out, k = [], lo
    while len(out) < count:
        if all(k % d for d in range(2, int(k ** 0.5) + 1)):
            out.append(k)
        k += 1
    return out


def test_fused_groups_beside_resident_tests(lnt):
    """Two carry-fused groups (2^19 and 2^20 words, 44 tests each, on their own
    streams) and 20 SMEM-resident tests running thousands of squarings in one
    launch beside them, graphs on.  A fused CTA waits only for CTAs that started
    before it, so however the other launches hold the GPU's CTA slots no wait
    runs out (that would fail the batch with a timeout status) and every test
    ends with the residue it gets alone."""
    resident = _primes_from(60000, 20)
    fused = _primes_from(8000000, 44) + _primes_from(12000000, 44)
    assert {lnt.secured_log2_length(q) for q in fused[:44]} == {19}
    assert {lnt.secured_log2_length(q) for q in fused[44:]} == {20}
    k_res, k_fused = 6000, 17  # the two-pass tests: one squaring alone, then 2 graph chunks of 8
    jobs = {}
    with lnt.Batch(device=0, graphs=True) as b:
        for i, q in enumerate(resident):
            jobs[b.submit(q, 0, bool(i & 1), k_res)] = (q, bool(i & 1), k_res)
        for i, q in enumerate(fused):
            jobs[b.submit(q, 0, bool(i & 1), k_fused)] = (q, bool(i & 1), k_fused)
        assert b.status()[0] == len(jobs)
        got = {}
        for _ in range(20):
            b.run(3000)
            for r in b.poll():
                assert r["status"] == 0, r
                got[r["id"]] = r
            if len(got) == len(jobs):
                break
        assert b.status()[0] == 0
    assert set(got) == set(jobs)
    for i, (q, prp, k) in jobs.items():
        assert got[i]["res64"] == alone(lnt, q, 0, prp, k), (q, prp, k)


def test_batch_checkpoints_equal_alone(lnt):
    """Res64 checkpoints every 100 squarings of a resident, a two-pass and a
    carry-fused test (LL and PRP) equal the same test alone after 100, 200 and
    300 squarings; the final result comes at 350."""
    tests = [(44497, 0, False), (160001, 0, True), (8000009, 0, False)]
    with lnt.Batch(device=0, checkpoint_every=100) as b:
        ids = {b.submit(q, n, prp, 350): (q, n, prp) for q, n, prp in tests}
        done, marks = {}, {}
        while len(done) < len(ids):
            b.run(64)
            for c in b.poll_checkpoints():
                assert c["status"] == 0, c
                marks.setdefault(c["id"], {})[c["iteration"]] = c["res64"]
            for r in b.poll():
                done[r["id"]] = r
    for i, (q, n, prp) in ids.items():
        assert sorted(marks[i]) == [100, 200, 300], (q, marks.get(i))
        with lnt.LucasTest(q, n, prp) as t:
            for k in (100, 200, 300):
                t.iterate(100)
                assert t.res64() == marks[i][k], (q, k)
            t.iterate(50)
            assert t.res64() == done[i]["res64"]


def test_batch_autotune_plan_cache(lnt, tmp_path):
    """A tuned plan is written to the JSON cache and a later batch uses it
    without timing again; the residues equal the policy plan's."""
    import json

    path = tmp_path / "plans.json"
    q = 1000003
    with lnt.Batch(device=0, autotune_loops=5, plan_cache=str(path)) as b:
        i = b.submit(q, 0, False, 40)
        b.run(40)
        r1 = {r["id"]: r for r in b.poll()}[i]
    cache = json.loads(path.read_text())
    assert cache["plans"] and cache["plans"][0]["n"] == 65536
    chosen = cache["plans"][0]
    before = path.read_text()
    with lnt.Batch(device=0, autotune_loops=5, plan_cache=str(path)) as b:
        i = b.submit(q + 30, 0, False, 40)  # same length and carry-run class: the cached plan
        b.run(40)
        r2 = {r["id"]: r for r in b.poll()}[i]
    assert path.read_text() == before
    assert r1["res64"] == alone(lnt, q, 0, False, 40)
    assert r2["res64"] == alone(lnt, q + 30, 0, False, 40)
    assert chosen["radix"] in (8, 16) and chosen["fused"] in (1, 2)


def test_serving_admits_requests_mid_flight(lnt):
    """Continuous batching: requests enqueued while others are running, across
    the resident (n <= 4096), two-pass and carry-fused (n >= 2^19) plans, LL and
    PRP, under a budget that holds only part of them at once, so later requests
    wait and are admitted as earlier ones retire.  Each result equals the same
    test alone."""
    first = [(44497, False, 3000), (160001, True, 400), (8000009, False, 60)]
    later = [(9941, True, 2500), (300007, False, 300), (12000017, True, 40), (59063, False, 2000),
             (1000003, True, 200)]
    # the 2^20-word request cannot join the 2^19-word one: it waits for it to retire
    budget = lnt.test_device_bytes(8000009) + lnt.test_device_bytes(12000017) - 1
    jobs, got = {}, {}
    with lnt.Batch(device=0, hbm_budget_bytes=budget) as b:
        for q, prp, k in first:
            jobs[b.enqueue(q, 0, prp, k)] = (q, prp, k)
        b.run(25)  # the first requests are mid-flight
        assert not b.poll()
        for q, prp, k in later:
            jobs[b.enqueue(q, 0, prp, k)] = (q, prp, k)
        waited = b.pending() > 0
        for _ in range(500):
            b.run(100)
            for r in b.poll():
                assert r["status"] == 0, r
                got[r["id"]] = r
            if len(got) == len(jobs):
                break
        assert b.status()[0] == 0 and b.pending() == 0
    assert waited, "the budget should have held some requests back"
    assert set(got) == set(jobs)
    for i, (q, prp, k) in jobs.items():
        assert got[i]["res64"] == alone(lnt, q, 0, prp, k), (q, prp, k)


def test_batch_keeps_plans_of_one_length_apart(lnt, tmp_path):
    """Tests of one length whose plans differ only in pass radix and column
    fusion (here from a plan cache: carry-run class 4 -> radix 16, fused;
    class 8 -> radix 8, two launches; both with 8-word tiles) run in separate
    launch groups, since their pass tables differ: every residue equals the
    test alone."""
    import json

    import torch

    cache = tmp_path / "plans.json"
    cache.write_text(json.dumps({"device": torch.cuda.get_device_name(0), "plans": [
        {"n": 524288, "run": 4, "kind": 2, "log2_rows": 9, "tile": 8, "radix": 16, "fused": 1, "ms": 1},
        {"n": 524288, "run": 8, "kind": 2, "log2_rows": 9, "tile": 8, "radix": 8, "fused": 2, "ms": 1}]}))
    tests = [(6291587, False), (6291599, True), (5767789, False), (5767841, True)]
    with lnt.Batch(device=0, autotune_loops=5, plan_cache=str(cache)) as b:
        ids = {b.submit(q, 0, prp, 30): (q, prp) for q, prp in tests}
        got = {}
        while len(got) < len(ids):
            b.run(30)
            got.update({r["id"]: r for r in b.poll()})
    for i, (q, prp) in ids.items():
        assert got[i]["status"] == 0 and got[i]["res64"] == alone(lnt, q, 0, prp, 30), (q, prp)


def test_time_budgeted_calls_equal_alone(lnt):
    """With a time budget per call (lnt_batch_step_seconds) each launch group and
    each resident test runs its own number of squarings per call: a small test
    is not held to the pace of a large one.  Residues equal the tests alone, and
    the small resident test finishes in fewer calls than the 2^20-word test."""
    tests = [(9941, 0, True, 2000), (160001, 0, False, 300), (12000017, 0, False, 400)]
    calls = {}
    with lnt.Batch(device=0, step_seconds=0.01) as b:
        ids = {b.submit(q, n, prp, k): (q, n, prp, k) for q, n, prp, k in tests}
        got, c = {}, 0
        while len(got) < len(ids):
            b.run(100000)
            c += 1
            for r in b.poll():
                got[r["id"]] = r
                calls[ids[r["id"]][0]] = c
    for i, (q, n, prp, k) in ids.items():
        assert got[i]["status"] == 0 and got[i]["res64"] == alone(lnt, q, n, prp, k), (q, prp)
    assert calls[9941] < calls[12000017], calls

"""GPU: every plan the autotuner may pick gives the oracle's digits.

The reference's autotune times several pools and kernels per length and keeps
the fastest (process.cu:45-127); any of them must produce the same residue.
Here each candidate plan (4-step split, column tile, pass radix 8 or 16,
carry-fused or plain column launches, or the radix-2 kernels) is run from the
same random state and compared digit for digit with the oracle, including the
largest lengths, 2^25 and 2^26 words.
"""
import numpy as np
import pytest

from oracle import bigint_model as B

pytestmark = pytest.mark.gpu


def random_digits(q, n, seed):
    rng = np.random.default_rng(seed)
    w = np.array(B.widths(q, n), dtype=np.uint64)
    return (rng.integers(0, 2**62, size=n, dtype=np.uint64) % (np.uint64(1) << w)).astype(np.uint64)


def oracle_digits(oracle_mod, q, n, prp, start, steps):
    """The oracle on the exact integer widths the library uses: they differ from
    the reference's double ones only where those break the squaring (q = 600000001
    at 2^25), and there the oracle then squares the number the digits hold."""
    with oracle_mod.OracleTest(q, n, prp) as O:
        j = np.arange(n + 1, dtype=np.uint64)
        O.set_widths(np.diff((np.uint64(q) * j + np.uint64(n - 1)) // np.uint64(n)).astype(np.uint8))
        O.set_digits(start)
        O.iterate(steps)
        return O.digits()


def run_plan(lnt, q, n, prp, plan, start, steps):
    with lnt.LucasTest(q, n, prp, plan=plan) as G:
        assert G.plan_options()[:len(plan)] == tuple(plan) or plan[0] == 0
        G.set_digits(start)
        G.iterate(steps)
        return G.digits(), G.plan


@pytest.mark.parametrize("q,n,prp", [(160001, 8192, False), (300007, 16384, True),
                                     (1000003, 65536, False), (5000011, 262144, True),
                                     (20000003, 1 << 20, False)])
def test_every_candidate_plan_matches_oracle(lnt, oracle_mod, q, n, prp):
    start = random_digits(q, n, q ^ n)
    want = oracle_digits(oracle_mod, q, n, prp, start, 3)
    plans = lnt.plan_candidates(q, n)
    assert len(plans) >= 2
    # the radix-2 kernels at the same lengths (reached by the policy only at 2^25, 2^26)
    l2 = (n.bit_length() - 1) // 2
    plans += [(3, l2, 8), (3, l2, 4)]
    for plan in plans:
        got, name = run_plan(lnt, q, n, prp, plan, start, 3)
        bad = np.nonzero(got != want)[0]
        assert bad.size == 0, f"{name}: first mismatch at {bad[:5]}"


@pytest.mark.parametrize("q", [600000001, 1100000009])
def test_largest_lengths(lnt, oracle_mod, q):
    """2^25 and 2^26 words: the policy's pass-kernel plan (rows of 8K / 16K words)
    and the radix-2 plan, one squaring from a random state, against the oracle."""
    n = 1 << lnt.secured_log2_length(q)
    start = random_digits(q, n, 11)
    want = oracle_digits(oracle_mod, q, n, False, start, 1)
    got, name = run_plan(lnt, q, n, False, (0, 0, 0), start, 1)
    assert name.startswith("TWOPASS_4096x") and "_R2" not in name
    assert np.array_equal(got, want)
    got, name = run_plan(lnt, q, n, False, (3, 12, 4), start, 1)
    assert "_R2" in name
    assert np.array_equal(got, want)


def test_invalid_plans_are_refused(lnt):
    with pytest.raises(lnt.LucasNTTError):
        lnt.LucasTest(139000003, 1 << 23, plan=(2, 13, 4))   # n2 > n1
    with pytest.raises(lnt.LucasNTTError):
        lnt.LucasTest(1000003, 1 << 16, plan=(2, 8, 16))     # no such tile
    with pytest.raises(lnt.LucasNTTError):
        lnt.LucasTest(9973, 512, plan=(2, 4, 4))             # two-pass below 8192 words


def test_autotune_picks_a_working_plan(lnt):
    q = 1000003
    results, best = lnt.autotune(q, 0, False, 0, loops=50)
    assert len(results) == len(lnt.plan_candidates(q)) and 0 <= best < len(results)
    assert all(ms > 0 for _, ms in results)
    assert results[best][1] == min(ms for _, ms in results)
    with lnt.LucasTest(q, plan=results[best][0]) as A, lnt.LucasTest(q) as Bt:
        A.iterate(200)
        Bt.iterate(200)
        assert A.res64() == Bt.res64()

"""GPU: the Gerbicz-Li check of PRP tests (lnt_gerbicz_enable).

The check multiplies residues (a product kernel path beside the squaring), so
it is exercised end to end: a checked PRP test of a Mersenne prime still ends
with residue 9; a checked test gives the same residue as an unchecked one; and
a residue word corrupted between calls (what a hardware error would do) is
detected at the next verification and the test recovers to the error-free
residue; a corruption large enough to make the kernels raise the carry flag is
recovered the same way instead of failing the call.
"""
import pytest

pytestmark = pytest.mark.gpu


def plain_res64(lnt, q, iterations):
    with lnt.LucasTest(q, prp=True) as t:
        t.iterate(iterations)
        return t.res64()


def test_checked_prp_of_a_mersenne_prime(lnt):
    q = 132049  # M_132049 is prime; n = 8192, a two-pass plan
    with lnt.LucasTest(q, prp=True) as t:
        t.gerbicz_enable(64)
        t.iterate(q)
        assert t.is_prime() and t.res64() == 9
        st = t.gerbicz_stats()
        assert st["errors"] == 0 and st["checks"] == q // (64 * 64)
        assert st["verified_iterations"] == st["checks"] * 64 * 64


@pytest.mark.parametrize("q,block,iterations", [(160001, 32, 20000), (1000003, 40, 9000)])
def test_checked_equals_unchecked(lnt, q, block, iterations):
    with lnt.LucasTest(q, prp=True) as t:
        t.gerbicz_enable(block)
        for k in (777, iterations - 777):  # calls not aligned to the blocks
            t.iterate(k)
        assert t.res64() == plain_res64(lnt, q, iterations)
        st = t.gerbicz_stats()
        assert st["errors"] == 0 and st["checks"] == iterations // (block * block)


def test_corrupted_word_is_caught_and_undone(lnt):
    q, block, iterations = 160001, 32, 12000
    with lnt.LucasTest(q, prp=True) as t:
        t.gerbicz_enable(block)
        t.iterate(5000)
        t.debug_corrupt(17)
        t.iterate(iterations - 5000)
        st = t.gerbicz_stats()
        assert st["errors"] >= 1
        assert t.res64() == plain_res64(lnt, q, iterations)


def test_checked_c2_length(lnt):
    q, block, iterations = 139000003, 50, 5000  # n = 2^23, two verifications
    with lnt.LucasTest(q, prp=True) as t:
        t.gerbicz_enable(block)
        t.iterate(iterations)
        assert t.gerbicz_stats()["checks"] == 2
        assert t.res64() == plain_res64(lnt, q, iterations)


def test_check_needs_prp_and_a_two_pass_plan(lnt):
    with lnt.LucasTest(160001, prp=False) as t:
        with pytest.raises(lnt.LucasNTTError):
            t.gerbicz_enable(64)
    with lnt.LucasTest(9941, prp=True) as t:  # n = 512: SMEM-resident plan
        with pytest.raises(lnt.LucasNTTError):
            t.gerbicz_enable(64)


@pytest.mark.parametrize("at", [4992, 5009])  # on a block boundary, inside a block
def test_carry_flag_from_a_corrupted_word_is_recovered(lnt, at):
    q, block, iterations = 160001, 32, 12000
    with lnt.LucasTest(q, prp=True) as t:
        t.gerbicz_enable(block)
        t.iterate(at)
        t.debug_corrupt(17, 1 << 40)  # far outside the balanced-digit range
        t.iterate(iterations - at)
        t.synchronize()
        st = t.gerbicz_stats()
        assert st["errors"] >= 1
        assert st["checks"] == iterations // (block * block)
        assert t.res64() == plain_res64(lnt, q, iterations)


def test_jacobi_check_ll(lnt):
    """LL error check: the symbol of an LL residue is -1 after every checked
    interval, a full test of M_132049 passes every check, and a word corrupted
    between calls is detected (now or, since an error leaves the symbol at -1
    half of the time, at a later check after more corruptions) and rolled
    back: the final residue equals the unchecked one."""
    import ctypes

    L = lnt.lib()
    L.lnt_jacobi_enable.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
    with lnt.LucasTest(9941, 0, False) as T:  # the SMEM-resident plan (no pending run carries)
        assert T.plan.startswith("RESIDENT")
        assert L.lnt_jacobi_enable(T._h, 1000) == 0, L.lnt_last_error()
        T.iterate(9941 - 2)
        assert T.is_prime()
    with lnt.LucasTest(132049, 0, False) as T:
        assert L.lnt_jacobi_enable(T._h, 5000) == 0, L.lnt_last_error()
        T.iterate(132049 - 2)
        assert T.is_prime()
        v, c, e = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        assert L.lnt_jacobi_stats(T._h, ctypes.byref(v), ctypes.byref(c), ctypes.byref(e)) == 0
        assert c.value == (132049 - 2) // 5000 and e.value == 0
    q = 1000003
    with lnt.LucasTest(q, 0, False) as ref:
        ref.iterate(400)
        want = ref.res64()
    caught = 0
    for k in range(20):  # a changed word leaves the symbol at -1 half of the time: try words until one is caught
        with lnt.LucasTest(q, 0, False) as T:
            assert L.lnt_jacobi_enable(T._h, 100) == 0
            T.iterate(100)
            s = ctypes.c_int()
            assert L.lnt_jacobi_check(T._h, ctypes.byref(s)) == 0 and s.value == -1
            T.debug_corrupt(word=17 + 31 * k, delta=1)
            T.iterate(300)
            v, c, e = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
            assert L.lnt_jacobi_stats(T._h, ctypes.byref(v), ctypes.byref(c), ctypes.byref(e)) == 0
            if e.value:
                assert e.value == 1 and v.value == 400
                assert T.res64() == want  # rolled back and redone
                caught += 1
                break
    assert caught == 1

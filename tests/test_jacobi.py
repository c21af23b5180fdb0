"""CPU: the Jacobi symbol of LL residues (lnt_jacobi_of_digits, host code of
the library that the LL error check calls), on residues from the oracle."""
import numpy as np

from oracle import bigint_model as B


def test_jacobi_symbol_of_ll_residues(oracle_mod, lnt):
    """lnt_jacobi_of_digits (host code, GMP's mpz_jacobi): every LL term u_k,
    k >= 1, has (u_k - 2 | M_q) = -1, for a prime and a composite M_q; the
    start value 4 has +1; a residue changed in one digit is caught about half
    of the time (here: some of 16 corruptions give +1)."""
    import ctypes

    L = lnt.lib()
    f = L.lnt_jacobi_of_digits
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_int)]
    f.restype = ctypes.c_int

    def symbol(digits, widths, q):
        s = ctypes.c_int(7)
        d = np.ascontiguousarray(digits, dtype=np.uint64)
        w = np.ascontiguousarray(widths, dtype=np.uint8)
        st = f(d.ctypes.data, w.ctypes.data, d.size, q, ctypes.byref(s))
        assert st == 0, L.lnt_last_error()
        return s.value

    for q, n in ((4423, 256), (4409, 256)):  # M_4423 prime, M_4409 composite
        w = np.array(B.widths(q, n), dtype=np.uint8)
        with oracle_mod.OracleTest(q, n, False) as T:
            assert symbol(T.digits(), w, q) == 1  # u_0 = 4: (2 | M_q) = +1
            prev = 0
            for k in (1, 2, 7, 50):
                T.iterate(1 if k == 1 else k - prev)
                prev = k
                assert symbol(T.digits(), w, q) == -1, (q, k)
            d = T.digits()
        rng = np.random.default_rng(q)
        flips = []
        for _ in range(16):
            e = d.copy()
            j = int(rng.integers(1, n))
            e[j] = (int(e[j]) + 1) % (1 << int(w[j]))
            flips.append(symbol(e, w, q))
        assert 1 in flips and -1 in flips, flips

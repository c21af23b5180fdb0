"""Generate tests/golden/true_residues.json: Res64 of the true LL / PRP
sequence of M_q, computed with GMP big integers (libgmp through ctypes).

These pin the cases where the reference's digit widths and weights disagree
(pre_calculation.cu:30-35: the double-precision width prefix starts some word
one bit below the bit its weight assumes, once q*j passes 2^53), so that its
own residues are not those of M_q.  Independent of this package and of the
oracle: s <- s^2 (- 2 for LL) mod 2^q - 1 with mpz_mul and a shift-and-add
reduction.

    python tests/golden/make_true_residues.py            # about an hour
"""
import ctypes
import ctypes.util
import json
import sys
import time
from pathlib import Path

OUT = Path(__file__).resolve().parent / "true_residues.json"
# (q, n, prp, iteration marks): q = 600000001 at n = 2^25 has one shifted word (j = 23116289)
CASES = [(600000001, 1 << 25, False, (100, 1000))]


class Mpz(ctypes.Structure):
    _fields_ = [("alloc", ctypes.c_int), ("size", ctypes.c_int), ("d", ctypes.POINTER(ctypes.c_uint64))]


def gmp():
    g = ctypes.CDLL(ctypes.util.find_library("gmp") or "libgmp.so.10")
    P, ul = ctypes.POINTER(Mpz), ctypes.c_ulong
    for name, args in (("init", [P]), ("set_ui", [P, ul]), ("mul", [P, P, P]), ("add", [P, P, P]),
                       ("sub", [P, P, P]), ("add_ui", [P, P, ul]), ("sub_ui", [P, P, ul]),
                       ("tdiv_q_2exp", [P, P, ul]), ("tdiv_r_2exp", [P, P, ul]),
                       ("ui_pow_ui", [P, ul, ul])):
        f = getattr(g, "__gmpz_" + name)
        f.argtypes, f.restype = args, None
    for name, args in (("cmp", [P, P]), ("cmp_ui", [P, ul])):
        f = getattr(g, "__gmpz_" + name)
        f.argtypes, f.restype = args, ctypes.c_int
    return g


def residues(g, q, prp, marks):
    s, t, h, m = Mpz(), Mpz(), Mpz(), Mpz()
    for z in (s, t, h, m):
        g.__gmpz_init(ctypes.byref(z))
    g.__gmpz_ui_pow_ui(m, 2, q)
    g.__gmpz_sub_ui(m, m, 1)
    g.__gmpz_set_ui(s, 3 if prp else 4)
    out, done, t0 = {}, 0, time.time()
    for mark in marks:
        for _ in range(mark - done):
            g.__gmpz_mul(t, s, s)
            g.__gmpz_tdiv_q_2exp(h, t, q)
            g.__gmpz_tdiv_r_2exp(t, t, q)
            g.__gmpz_add(s, t, h)
            if g.__gmpz_cmp(s, m) >= 0:
                g.__gmpz_sub(s, s, m)
            if not prp:
                if g.__gmpz_cmp_ui(s, 2) < 0:
                    g.__gmpz_add(s, s, m)
                g.__gmpz_sub_ui(s, s, 2)
        done = mark
        out[str(mark)] = f"{(s.d[0] if s.size else 0):016x}"
        print(q, mark, out[str(mark)], f"{time.time() - t0:.0f} s", file=sys.stderr, flush=True)
    return out


def main():
    g = gmp()
    # self-check on a known prime: the LL residue of M_9941 after q - 2 squarings is 0
    assert residues(g, 9941, False, (9939,)) == {"9939": "0000000000000000"}
    cases = [{"q": q, "n": n, "prp": prp, "res64_after": residues(g, q, prp, marks)}
             for q, n, prp, marks in CASES]
    OUT.write_text(json.dumps({"source": "GMP mpz, s <- s^2 (- 2) mod 2^q - 1", "cases": cases},
                              indent=1) + "\n")


if __name__ == "__main__":
    main()

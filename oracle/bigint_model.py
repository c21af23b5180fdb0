"""Independent big-integer model of the reference's residue sequence.

TEST INFRASTRUCTURE ONLY (pins the C oracle; never used by the product).

This model does not use an NTT at all.  It follows the value the reference's
digit vector represents, using only the algebra of its carry and borrow passes:

* kernels/r2b.cu:25-50 ripples carries cyclically until every word fits its
  width.  The represented value V is then in [0, M] (M = 2^q - 1).  A carry
  wraps past the top only while V >= 2^q, so a non-zero convolution never
  collapses to 0: after the carry V' = 0 when the digits were all zero, else
  V' = ((V^2 - 1) mod M) + 1  (so a multiple of M shows as M, all digits full).
* kernels/m2.cu:23-41 subtracts 2 with a cyclic borrow: for V' >= 2 it gives
  V' - 2, for V' in {0, 1} it gives V' + M - 2.
* lucas_prp.cu:129 starts LL at 4 and PRP at 3.

Digits are d_j = bits [pos_j, pos_j + w_j) of the value, pos_j = ceil(q j / n).
Fast only for small exponents (Python big-integer squaring).
"""
from __future__ import annotations


def widths(exponent: int, n: int) -> list[int]:
    """Exact integer form of pre_calculation.cu:35."""
    pos = [-(-exponent * j // n) for j in range(n + 1)]
    return [pos[j + 1] - pos[j] for j in range(n)]


def to_digits(value: int, exponent: int, n: int) -> list[int]:
    out, pos = [], 0
    for w in widths(exponent, n):
        out.append((value >> pos) & ((1 << w) - 1))
        pos += w
    return out


def from_digits(digits, exponent: int, n: int) -> int:
    v, pos = 0, 0
    for d, w in zip(digits, widths(exponent, n)):
        v += int(d) << pos
        pos += w
    return v


def mod_mersenne(x: int, exponent: int) -> int:
    """x mod 2^q - 1 for x >= 0 by folding (2^q == 1), no long division."""
    m = (1 << exponent) - 1
    while x > m:
        x = (x & m) + (x >> exponent)
    return 0 if x == m else x


def step(value: int, exponent: int, prp: bool) -> int:
    m = (1 << exponent) - 1
    if value == 0:
        f = 0
    else:
        f = mod_mersenne(value * value - 1, exponent) + 1
    if prp:
        return f
    return f - 2 if f >= 2 else f + m - 2


def run(exponent: int, iterations: int, prp: bool = False, start: int | None = None) -> int:
    v = (3 if prp else 4) if start is None else start
    for _ in range(iterations):
        v = step(v, exponent, prp)
    return v


def res64(value: int) -> int:
    return value & 0xFFFFFFFFFFFFFFFF

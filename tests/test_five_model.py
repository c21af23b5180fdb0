"""CPU: the algebra of the 5 * 2^k row transform, in exact integers mod p.

A model of one squaring's transform at n = 5 L n2 (L = 16, n2 = 8) built from
the same definitions as the kernels and tables (lnt_radix16.cu row5_r16,
lnt_tables.cu launch_five_twiddles / twiddle_kernel): column transforms in
bit-reversed row order, the 4-step twiddle omega_n^(c' brev(row)); in each row
(c' = c + L j5) the pair-form 5-point transform over j5 with constants
(w^k +- w^-k)/2, the twiddle omega_5L^(c k5), five L-point plane transforms
(bit-reversed output), the square, and the inverse steps in reverse order (the
inverse 5-point transform is the forward one with outputs 1/4 and 2/3
exchanged).  Forward, square and unscaled inverse must give n times the cyclic
self-convolution.
"""
import random

P = 2**64 - 2**32 + 1


def brev(x, bits):
    return int(format(x, f"0{bits}b")[::-1], 2) if bits else 0


def inv(a):
    return pow(a, P - 2, P)


def dft(v, w):
    m = len(v)
    return [sum(v[j] * pow(w, j * k, P) for j in range(m)) % P for k in range(m)]


def constants(w5):
    half = inv(2)
    w2, w3, w4 = pow(w5, 2, P), pow(w5, 3, P), pow(w5, 4, P)
    return [(w5 + w4) * half % P, (w2 + w3) * half % P, (w5 - w4) * half % P, (w2 - w3) * half % P]


def dft5(u, c):
    a1, b1 = (u[1] + u[4]) % P, (u[1] - u[4]) % P
    a2, b2 = (u[2] + u[3]) % P, (u[2] - u[3]) % P
    t1, t2 = (a1 * c[0] + a2 * c[1]) % P, (a1 * c[1] + a2 * c[0]) % P
    s1, s2 = (b1 * c[2] + b2 * c[3]) % P, (b1 * c[3] - b2 * c[2]) % P
    u0 = u[0]
    return [(u0 + a1 + a2) % P, (u0 + t1 + s1) % P, (u0 + t2 + s2) % P, (u0 + t2 - s2) % P,
            (u0 + t1 - s1) % P]


def test_pair_form_is_the_5_point_transform():
    rng = random.Random(1)
    w5 = pow(554, (P - 1) // 5, P)
    assert w5 != 1 and pow(w5, 5, P) == 1
    c = constants(w5)
    for _ in range(20):
        u = [rng.randrange(P) for _ in range(5)]
        want = dft(u, w5)
        assert dft5(u, c) == want
        inverse = dft5(want, c)
        assert [inverse[0], inverse[4], inverse[3], inverse[2], inverse[1]] == [5 * x % P for x in u]


def test_five_plane_squaring_is_the_cyclic_convolution():
    rng = random.Random(2)
    n2, L, lg2, lgL = 8, 16, 3, 4
    n1 = 5 * L
    n = n1 * n2
    wn = pow(554, (P - 1) // n, P)
    w_n2, w_L, w_5L = pow(wn, n1, P), pow(wn, 5 * n2, P), pow(wn, n2, P)
    assert w_5L == pow(554, (P - 1) // (5 * L), P)  # the root launch_five_twiddles takes
    c = constants(pow(w_5L, L, P))
    x = [rng.randrange(1 << 12) for _ in range(n)]
    rows = [[0] * n1 for _ in range(n2)]
    for col in range(n1):
        f = dft([x[r * n1 + col] for r in range(n2)], w_n2)
        for row in range(n2):
            rows[row][col] = f[brev(row, lg2)] * pow(wn, col * brev(row, lg2), P) % P
    for row in range(n2):
        planes = [[0] * L for _ in range(5)]
        for cc in range(L):
            u = dft5([rows[row][cc + L * j5] for j5 in range(5)], c)
            for k5 in range(5):
                planes[k5][cc] = u[k5] * pow(w_5L, cc * k5, P) % P
        for k5 in range(5):
            f = dft(planes[k5], w_L)
            sq = [f[brev(e, lgL)] ** 2 % P for e in range(L)]  # bit-reversed, squared
            nat = [0] * L
            for e in range(L):
                nat[brev(e, lgL)] = sq[e]
            planes[k5] = dft(nat, inv(w_L))
        for cc in range(L):
            y = [planes[k5][cc] * pow(inv(w_5L), cc * k5, P) % P for k5 in range(5)]
            z = dft5(y, c)
            for j5, k5 in enumerate((0, 4, 3, 2, 1)):
                rows[row][cc + L * j5] = z[k5]
    out = [0] * n
    for col in range(n1):
        freq = [0] * n2
        for row in range(n2):
            freq[brev(row, lg2)] = rows[row][col] * pow(inv(wn), col * brev(row, lg2), P) % P
        t = dft(freq, inv(w_n2))
        for r in range(n2):
            out[r * n1 + col] = t[r]
    conv = [0] * n
    for i in range(n):
        for j in range(n):
            conv[(i + j) % n] += x[i] * x[j]
    assert out == [v * n % P for v in conv]


def test_weights_exist_for_five_lengths():
    """g = 7^(((p-1)/192/n) 5) has g^n = 2 for n = 5 * 2^k (k <= 26): the
    reference's weight formula works unchanged; for n = 3 * 2^k no n-th root of
    2 exists (192 n does not divide p - 1)."""
    for k in (13, 20, 24):
        n = 5 << k
        assert (P - 1) % (192 * n) == 0
        g = pow(7, ((P - 1) // 192 // n) * 5, P)
        assert pow(g, n, P) == 2
    # 2 is an n-th power mod p iff 2^((p-1)/gcd(n, p-1)) = 1: not for n = 3 * 2^k
    for k in (13, 20):
        assert pow(2, (P - 1) // (3 << k), P) != 1
        assert pow(2, (P - 1) // (5 << k), P) == 1

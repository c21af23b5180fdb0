/*
 * lnt_oracle.c -- CPU restatement of LucasNTT's Lucas-Lehmer / PRP squaring loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path and the
 * timed CPU baseline.  The product library never links, loads or calls it.
 *
 * Every function restates one piece of the reference (LucasNTT/cuda); the
 * citation in front of each function is the reference file:line it follows.
 * One section has no reference counterpart and says so: lengths n = 5 * 2^k,
 * the checker of the library's own extension, pinned to the big-integer model.
 * The arithmetic is exact uint64 arithmetic modulo the Goldilocks prime
 * p = 2^64 - 2^32 + 1, written here from the algebra (2^64 = 2^32 - 1 and
 * 2^96 = -1 mod p), not transcribed.
 *
 * Parity pins: known Mersenne primes (LL residue 0, PRP residue 9), an
 * independent big-integer model (oracle/bigint_model.py), and residues the
 * reference's own build produced on a B200 (tests/golden/).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define GL_P   0xFFFFFFFF00000001ULL
#define GL_EPS 0x00000000FFFFFFFFULL /* 2^64 mod p */

typedef unsigned __int128 u128;

/* ---- field arithmetic (common/arithmetics.cuh:37-185) ------------------ */

static inline uint64_t gl_add(uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    int wrapped = s < a;
    if (wrapped || s >= GL_P) s -= GL_P; /* on wrap, s - p == s + 2^64 - p */
    return s;
}

static inline uint64_t gl_sub(uint64_t a, uint64_t b) {
    uint64_t d = a - b;
    if (a < b) d += GL_P;
    return d;
}

/* reduce a 128-bit value: v = lo + 2^64 (h0 + 2^32 h1) == lo + h0 (2^32-1) - h1 */
static inline uint64_t gl_reduce128(uint64_t lo, uint64_t hi) {
    uint64_t h1 = hi >> 32, h0 = hi & 0xFFFFFFFFULL;
    uint64_t t = lo - h1;
    if (lo < h1) t -= GL_EPS;
    uint64_t m = (h0 << 32) - h0;
    uint64_t r = t + m;
    if (r < m) r += GL_EPS;
    if (r >= GL_P) r -= GL_P;
    return r;
}

static inline uint64_t gl_mul(uint64_t a, uint64_t b) {
    u128 v = (u128)a * b;
    return gl_reduce128((uint64_t)v, (uint64_t)(v >> 64));
}

/* pow_Mod (arithmetics.cuh:161-171) */
uint64_t oracle_gl_pow(uint64_t a, uint64_t e) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = gl_mul(r, a);
        a = gl_mul(a, a);
        e >>= 1;
    }
    return r;
}

/* inv_Mod: a^(p-2) (arithmetics.cuh:182-185) */
uint64_t oracle_gl_inv(uint64_t a) { return oracle_gl_pow(a, GL_P - 2); }
uint64_t oracle_gl_mul(uint64_t a, uint64_t b) { return gl_mul(a, b); }
uint64_t oracle_gl_add(uint64_t a, uint64_t b) { return gl_add(a, b); }
uint64_t oracle_gl_sub(uint64_t a, uint64_t b) { return gl_sub(a, b); }

/* ---- length policy (ntt_lengths.cu:88-98, :100-128) -------------------- */

/* GetNttSecuredLength: smallest log2 n with q/n <= 32 bits per word, bumped
 * once when 2 n m^2 >= p for m = 2^ceil(q/n) - 1.  Same double arithmetic. */
uint32_t oracle_secured_log2(uint32_t exponent) {
    double log_n = ceil(log2(1.0 * exponent / 32));
    double m = exp2(ceil(1.0 * exponent / exp2(log_n))) - 1;
    if (m * m >= 1.0 * GL_P / (2 * exp2(log_n))) log_n++;
    return (uint32_t)log_n;
}

/* GetCandidates: writes the ';'-separated candidate strings the reference
 * builds with std::to_string(double) (printf "%f"). Returns the count. */
int oracle_candidates(uint32_t exponent, char* out, size_t outlen) {
    char buf[1024];
    size_t k = 0;
    int count = 0;
    uint32_t l = oracle_secured_log2(exponent);
#define ADD(...) do { int w_ = snprintf(buf + k, sizeof(buf) - k, __VA_ARGS__); k += (size_t)w_; count++; } while (0)
    ADD("%f;", exp2(l));
    if (l >= 10 && l <= 24) {
        uint32_t a = l / 2;
        ADD("%f:%f;", exp2(a), exp2(l - a));
        if (l - a != a) ADD("%f:%f;", exp2(l - a), exp2(a));
    }
    if (l == 23) { ADD("256:256:128;"); ADD("512:256:64;"); }
    if (l == 24) { ADD("512:256:128;"); ADD("512:512:64;"); }
    if (l == 25) { ADD("512:512:128;"); ADD("1024:256:128;"); ADD("1024:512:64;"); }
    if (l == 26) { ADD("512:512:256;"); ADD("1024:256:256;"); ADD("1024:512:128;"); }
#undef ADD
    if (out && outlen) {
        size_t n = k < outlen - 1 ? k : outlen - 1;
        memcpy(out, buf, n);
        out[n] = 0;
    }
    return count;
}

/* ---- IBDWT tables (common/pre_calculation.cu:23-36) -------------------- */

/* weights[j] = 7^(((p-1)/192/n) * 5 * (n - r)), r = q*j mod n (uint32 product,
 * low bits only); weights[0] = 1; unweights[j] = (weights[j]*n)^-1,
 * unweights[0] = n^-1; widths[j] = ceil(q(j+1)/n) - ceil(qj/n) in double.
 * Computed through a power table of g = 7^((p-1)/192/n*5) (g^n = 2), which
 * gives the same field elements as the per-element pow of the reference. */
void oracle_weights_widths(uint32_t n, uint32_t exponent, uint64_t* weights,
                           uint64_t* unweights, uint8_t* widths) {
    uint64_t c = ((GL_P - 1) / 192 / n) * 5ULL;
    uint64_t g = oracle_gl_pow(7, c);
    uint64_t* gp = (uint64_t*)malloc(sizeof(uint64_t) * ((size_t)n + 1));
    gp[0] = 1;
    for (uint32_t k = 1; k <= n; k++) gp[k] = gl_mul(gp[k - 1], g);
    uint64_t inv_n = oracle_gl_inv(n);
    uint64_t inv_2n = oracle_gl_inv(2ULL * n);
    /* unweight = (g^(n-r) n)^-1 = g^r / (g^n n) = g^r / (2n) */
    #pragma omp parallel for schedule(static) if (n >= (1u << 16))
    for (int64_t j = 0; j < (int64_t)n; j++) {
        if (j == 0) {
            weights[0] = 1;
            unweights[0] = inv_n;
        } else {
            uint32_t r = ((uint32_t)exponent * (uint32_t)j) & (n - 1);
            weights[j] = gp[n - r];
            unweights[j] = gl_mul(gp[r], inv_2n);
        }
        widths[j] = (uint8_t)(ceil(1.0 * exponent * (double)(j + 1) / n) - ceil(1.0 * exponent * (double)j / n));
    }
    free(gp);
}

/* ---- radix-2 NTT (roots as pre_calculation.cu:61-66: 554^((p-1)/n)) ---- */

static void make_roots(uint32_t n, uint64_t* rt, uint64_t* irt) {
    uint64_t w = oracle_gl_pow(554, (GL_P - 1) / n);
    uint64_t wi = oracle_gl_inv(w);
    uint32_t half = n / 2 ? n / 2 : 1;
    rt[0] = 1; irt[0] = 1;
    for (uint32_t k = 1; k < half; k++) {
        rt[k] = gl_mul(rt[k - 1], w);
        irt[k] = gl_mul(irt[k - 1], wi);
    }
}

/* decimation in frequency: natural order in, bit-reversed order out */
static void ntt_dif(uint64_t* a, uint32_t n, const uint64_t* rt) {
    for (uint32_t h = n / 2, step = 1; h >= 1; h >>= 1, step <<= 1) {
        uint32_t lg = 0;
        while ((1u << lg) < h) lg++;
        #pragma omp parallel for schedule(static) if (n >= (1u << 15))
        for (int64_t b = 0; b < (int64_t)(n / 2); b++) {
            uint32_t i = (uint32_t)b & (h - 1);
            uint32_t i0 = (((uint32_t)b >> lg) << (lg + 1)) + i;
            uint32_t i1 = i0 + h;
            uint64_t x = a[i0], y = a[i1];
            a[i0] = gl_add(x, y);
            a[i1] = gl_mul(gl_sub(x, y), rt[(size_t)i * step]);
        }
    }
}

/* decimation in time with inverse roots: bit-reversed in, natural out (unscaled) */
static void intt_dit(uint64_t* a, uint32_t n, const uint64_t* irt) {
    for (uint32_t h = 1, step = n / 2; h < n; h <<= 1, step >>= 1) {
        uint32_t lg = 0;
        while ((1u << lg) < h) lg++;
        #pragma omp parallel for schedule(static) if (n >= (1u << 15))
        for (int64_t b = 0; b < (int64_t)(n / 2); b++) {
            uint32_t i = (uint32_t)b & (h - 1);
            uint32_t i0 = (((uint32_t)b >> lg) << (lg + 1)) + i;
            uint32_t i1 = i0 + h;
            uint64_t x = a[i0], y = gl_mul(a[i1], irt[(size_t)i * step]);
            a[i0] = gl_add(x, y);
            a[i1] = gl_sub(x, y);
        }
    }
}

/* ---- carry and subtract-2 ---------------------------------------------- */

/* reduceToBase (kernels/r2b.cu:25-50): every word is masked to its width and
 * its high bits are carried to the next word, cyclically (2^q == 1 mod M),
 * until no carry is left.  The reference runs this as racing CAS loops; the
 * fixed point is unique, so a sequential sweep gives the same digits.
 * Returns -1 if an addition would overflow 64 bits (the reference's uint64
 * arithmetic would then be meaningless). */
static int reduce_to_base(uint64_t* x, const uint8_t* widths, uint32_t n) {
    uint64_t carry = 0;
    uint32_t j = 0;
    int wrapped = 0;
    for (;;) {
        uint64_t v = x[j] + carry;
        if (v < carry) return -1;
        uint8_t w = widths[j];
        x[j] = v & ((1ULL << w) - 1);
        carry = v >> w;
        j++;
        if (j == n) { j = 0; wrapped = 1; }
        if (wrapped && carry == 0) break;
    }
    return 0;
}

/* minus_two (kernels/m2.cu:23-41): x[0] -= 2 with a cyclic borrow ripple. */
static void minus_two(uint64_t* x, const uint8_t* widths, uint32_t n) {
    uint64_t a = x[0];
    x[0] = a - 2;
    if (a < 2) {
        x[0] &= (1ULL << widths[0]) - 1;
        uint32_t id = 0;
        int borrow = 1;
        while (borrow) {
            id = (id == n - 1) ? 0 : id + 1;
            uint64_t mask = (1ULL << widths[id]) - 1;
            uint64_t v = x[id];
            x[id] = (v - 1) & mask;
            borrow = (v == 0);
        }
    }
}

/* ---- test state --------------------------------------------------------- */

typedef struct {
    uint32_t q, n;
    int prp;
    uint64_t *w, *uw, *rt, *irt, *x;
    uint8_t* widths;
    /* n = 5 m (m = 2^k): no reference counterpart (its Length names factors of
     * 5 but no kernel runs them).  rt/irt are then the roots of the m-point
     * plane transforms, tw5[(k5 - 1) m + c] = omega_n^(c k5), c5 the pair-form
     * constants of the 5-point transform (omega_5 = omega_n^m). */
    uint32_t m;
    uint64_t *tw5, *itw5, c5[4];
} oracle_ctx;

/* ---- lengths n = 5 * 2^k (not a reference path) --------------------------
 *
 * Same arithmetic as the power-of-two path except the transform and two table
 * details, both written for this length only: the widths are exact integers
 * (ceil(q(j+1)/n) - ceil(qj/n); the double expression can be off once q*j
 * passes 2^53), and a word with qj = 0 mod n, j > 0, sits on a whole bit and
 * takes weight 1 (the power-of-two formula would give g^n = 2).  The transform
 * of x (c' = c + m j5) is X[5 km + k5] =
 *   sum_c omega_m^(c km) omega_n^(c k5) sum_j5 omega_5^(j5 k5) x[c + m j5]:
 * a 5-point transform per c, a twiddle, and five m-point transforms. */

static void dft5(uint64_t u[5], const uint64_t c[4]) {
    uint64_t a1 = gl_add(u[1], u[4]), b1 = gl_sub(u[1], u[4]);
    uint64_t a2 = gl_add(u[2], u[3]), b2 = gl_sub(u[2], u[3]);
    uint64_t t1 = gl_add(gl_mul(a1, c[0]), gl_mul(a2, c[1]));
    uint64_t t2 = gl_add(gl_mul(a1, c[1]), gl_mul(a2, c[0]));
    uint64_t s1 = gl_add(gl_mul(b1, c[2]), gl_mul(b2, c[3]));
    uint64_t s2 = gl_sub(gl_mul(b1, c[3]), gl_mul(b2, c[2]));
    uint64_t u0 = u[0];
    u[0] = gl_add(u0, gl_add(a1, a2));
    u[1] = gl_add(gl_add(u0, t1), s1);
    u[4] = gl_sub(gl_add(u0, t1), s1);
    u[2] = gl_add(gl_add(u0, t2), s2);
    u[3] = gl_sub(gl_add(u0, t2), s2);
}

static void* oracle_create_five(uint32_t exponent, uint32_t n, int prp) {
    uint32_t m = n / 5;
    oracle_ctx* c = (oracle_ctx*)calloc(1, sizeof(oracle_ctx));
    c->q = exponent; c->n = n; c->prp = prp; c->m = m;
    c->w = (uint64_t*)malloc(8ULL * n);
    c->uw = (uint64_t*)malloc(8ULL * n);
    c->x = (uint64_t*)calloc(n, 8);
    c->rt = (uint64_t*)malloc(8ULL * (m / 2 ? m / 2 : 1));
    c->irt = (uint64_t*)malloc(8ULL * (m / 2 ? m / 2 : 1));
    c->widths = (uint8_t*)malloc(n);
    c->tw5 = (uint64_t*)malloc(8ULL * 4 * m);
    c->itw5 = (uint64_t*)malloc(8ULL * 4 * m);
    uint64_t g = oracle_gl_pow(7, ((GL_P - 1) / 192 / n) * 5ULL);
    uint64_t inv_n = oracle_gl_inv(n), inv_2n = oracle_gl_inv(2ULL * n);
    uint64_t prev = 0;
    for (uint32_t j = 0; j < n; j++) {
        uint64_t next = ((uint64_t)exponent * (j + 1) + n - 1) / n;
        c->widths[j] = (uint8_t)(next - prev);
        prev = next;
        uint64_t r = ((uint64_t)exponent * j) % n;
        if (r == 0) {
            c->w[j] = 1;
            c->uw[j] = inv_n;
        } else {
            c->w[j] = oracle_gl_pow(g, n - r);
            c->uw[j] = gl_mul(oracle_gl_pow(g, r), inv_2n);
        }
    }
    make_roots(m, c->rt, c->irt);
    uint64_t wn = oracle_gl_pow(554, (GL_P - 1) / n), iwn = oracle_gl_inv(wn);
    for (uint32_t k5 = 1; k5 < 5; k5++)
        for (uint32_t cc = 0; cc < m; cc++) {
            c->tw5[(k5 - 1) * m + cc] = oracle_gl_pow(wn, (uint64_t)cc * k5);
            c->itw5[(k5 - 1) * m + cc] = oracle_gl_pow(iwn, (uint64_t)cc * k5);
        }
    uint64_t w5 = oracle_gl_pow(wn, m), half = oracle_gl_inv(2);
    uint64_t w2 = gl_mul(w5, w5), w3 = gl_mul(w2, w5), w4 = gl_mul(w3, w5);
    c->c5[0] = gl_mul(gl_add(w5, w4), half);
    c->c5[1] = gl_mul(gl_add(w2, w3), half);
    c->c5[2] = gl_mul(gl_sub(w5, w4), half);
    c->c5[3] = gl_mul(gl_sub(w2, w3), half);
    c->x[0] = prp ? 3 : 4;
    return c;
}

/* forward transform, pointwise square, unscaled inverse (factor n in uw) */
static void five_square(oracle_ctx* c) {
    uint32_t m = c->m;
    uint64_t* x = c->x;
    uint64_t* y = (uint64_t*)malloc(8ULL * c->n);
    #pragma omp parallel for schedule(static) if (m >= (1u << 12))
    for (int64_t cc = 0; cc < (int64_t)m; cc++) {
        uint64_t u[5];
        for (int j5 = 0; j5 < 5; j5++) u[j5] = x[cc + (uint64_t)m * j5];
        dft5(u, c->c5);
        y[cc] = u[0];
        for (int k5 = 1; k5 < 5; k5++) y[(uint64_t)k5 * m + cc] = gl_mul(u[k5], c->tw5[(k5 - 1) * m + cc]);
    }
    for (int k5 = 0; k5 < 5; k5++) {
        uint64_t* plane = y + (uint64_t)k5 * m;
        ntt_dif(plane, m, c->rt);
        for (uint32_t e = 0; e < m; e++) plane[e] = gl_mul(plane[e], plane[e]);
        intt_dit(plane, m, c->irt);
    }
    #pragma omp parallel for schedule(static) if (m >= (1u << 12))
    for (int64_t cc = 0; cc < (int64_t)m; cc++) {
        uint64_t u[5];
        u[0] = y[cc];
        for (int k5 = 1; k5 < 5; k5++) u[k5] = gl_mul(y[(uint64_t)k5 * m + cc], c->itw5[(k5 - 1) * m + cc]);
        dft5(u, c->c5);
        x[cc] = u[0];
        x[cc + m] = u[4];
        x[cc + 2ULL * m] = u[3];
        x[cc + 3ULL * m] = u[2];
        x[cc + 4ULL * m] = u[1];
    }
    free(y);
}

static int is_pow2(uint32_t n) { return n >= 2 && (n & (n - 1)) == 0; }

void* oracle_create(uint32_t exponent, uint32_t n, int prp) {
    if (n % 5 == 0 && is_pow2(n / 5) && n <= (5u << 24)) return oracle_create_five(exponent, n, prp);
    if (n < 2 || (n & (n - 1)) || n > (1u << 26)) return NULL;
    oracle_ctx* c = (oracle_ctx*)calloc(1, sizeof(oracle_ctx));
    c->q = exponent; c->n = n; c->prp = prp;
    c->w = (uint64_t*)malloc(8ULL * n);
    c->uw = (uint64_t*)malloc(8ULL * n);
    c->x = (uint64_t*)calloc(n, 8);
    c->rt = (uint64_t*)malloc(8ULL * (n / 2));
    c->irt = (uint64_t*)malloc(8ULL * (n / 2));
    c->widths = (uint8_t*)malloc(n);
    oracle_weights_widths(n, exponent, c->w, c->uw, c->widths);
    make_roots(n, c->rt, c->irt);
    /* InitializeTest (lucas_prp.cu:127-134): s0 = 4 (LL) or 3 (PRP) */
    c->x[0] = prp ? 3 : 4;
    return c;
}

void oracle_destroy(void* p) {
    oracle_ctx* c = (oracle_ctx*)p;
    if (!c) return;
    free(c->w); free(c->uw); free(c->x); free(c->rt); free(c->irt); free(c->widths);
    free(c->tw5); free(c->itw5);
    free(c);
}

void oracle_set_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void oracle_set_digits(void* p, const uint64_t* d) {
    oracle_ctx* c = (oracle_ctx*)p;
    memcpy(c->x, d, 8ULL * c->n);
}

void oracle_get_digits(void* p, uint64_t* d) {
    oracle_ctx* c = (oracle_ctx*)p;
    memcpy(d, c->x, 8ULL * c->n);
}

void oracle_get_widths(void* p, uint8_t* w) {
    oracle_ctx* c = (oracle_ctx*)p;
    memcpy(w, c->widths, c->n);
}

/* Replaces the digit widths (the reference's double-precision table) with the
 * caller's; used to run the same arithmetic on the exact-integer widths
 * ceil(q(j+1)/n) - ceil(qj/n), which differ from the double ones for some
 * (q, n) with q*n > 2^53.  Not part of the reference's behaviour. */
void oracle_set_widths(void* p, const uint8_t* w) {
    oracle_ctx* c = (oracle_ctx*)p;
    memcpy(c->widths, w, c->n);
}

void oracle_get_weights(void* p, uint64_t* w, uint64_t* uw) {
    oracle_ctx* c = (oracle_ctx*)p;
    memcpy(w, c->w, 8ULL * c->n);
    memcpy(uw, c->uw, 8ULL * c->n);
}

/* One squaring as the FFT_1SMEM / FFT_2SMEM pools order it
 * (kernel_pool.cu:31-48): weight, forward NTT, square, inverse NTT,
 * unweight (w_fft_sqr_ifft_uw__r2_8to4k.cu:20-55), r2b, then m2 for LL. */
int oracle_iterate(void* p, uint64_t iterations) {
    oracle_ctx* c = (oracle_ctx*)p;
    uint32_t n = c->n;
    uint64_t* x = c->x;
    for (uint64_t it = 0; it < iterations; it++) {
        #pragma omp parallel for schedule(static) if (n >= (1u << 15))
        for (int64_t j = 0; j < (int64_t)n; j++) x[j] = gl_mul(x[j], c->w[j]);
        if (c->m) {
            five_square(c);
        } else {
            ntt_dif(x, n, c->rt);
            #pragma omp parallel for schedule(static) if (n >= (1u << 15))
            for (int64_t j = 0; j < (int64_t)n; j++) x[j] = gl_mul(x[j], x[j]);
            intt_dit(x, n, c->irt);
        }
        #pragma omp parallel for schedule(static) if (n >= (1u << 15))
        for (int64_t j = 0; j < (int64_t)n; j++) x[j] = gl_mul(x[j], c->uw[j]);
        if (reduce_to_base(x, c->widths, n) != 0) return -1;
        if (!c->prp) minus_two(x, c->widths, n);
    }
    return 0;
}

/* Res64 of the residue: the low 64 bits of sum d_j 2^ceil(q j / n).  The
 * reference dumps the full digit vector (lucas_prp.cu:254-263); Res64 is
 * derived from it. */
uint64_t oracle_res64_of(const uint64_t* d, const uint8_t* widths, uint32_t n) {
    uint64_t r = 0;
    uint32_t pos = 0;
    for (uint32_t j = 0; j < n && pos < 64; j++) {
        r += d[j] << pos;
        pos += widths[j];
    }
    return r;
}

uint64_t oracle_res64(void* p) {
    oracle_ctx* c = (oracle_ctx*)p;
    return oracle_res64_of(c->x, c->widths, c->n);
}

/* Verdict of LucasPRP::Run (lucas_prp.cu:169-176): residue 0 for LL, 9 for PRP. */
int oracle_is_prime(void* p) {
    oracle_ctx* c = (oracle_ctx*)p;
    if (c->x[0] != (uint64_t)(c->prp ? 9 : 0)) return 0;
    for (uint32_t j = 1; j < c->n; j++)
        if (c->x[j]) return 0;
    return 1;
}

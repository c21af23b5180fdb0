// Host build of the device arithmetic (cuda_b200/csrc/goldilocks.cuh,
// carry.cuh) checked against plain 128-bit remainder arithmetic.
// Prints "ok <cases>" or the first mismatch; exit code 1 on failure.
#include <cstdio>
#include <cstdint>
#include <random>
#include <vector>
#include "../../cuda_b200/csrc/goldilocks.cuh"
#include "../../cuda_b200/csrc/carry.cuh"

typedef unsigned __int128 u128;
static const uint64_t P = 0xFFFFFFFF00000001ull;
static uint64_t rmul(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a * b) % P); }
static uint64_t radd(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a + b) % P); }
static uint64_t rsub(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a + P - b) % P); }
static uint64_t rpow2(unsigned s) { uint64_t r = 1; for (unsigned i = 0; i < s; ++i) r = radd(r, r); return r; }

static int fails = 0;
static long cases = 0;
#define CHECK(cond, ...) do { ++cases; if (!(cond)) { if (fails++ < 10) { std::printf(__VA_ARGS__); std::printf("\n"); } } } while (0)

int main() {
  std::mt19937_64 rng(12345);
  std::vector<uint64_t> vals = {0, 1, 2, P - 1, P - 2, P >> 1, (P >> 1) + 1, 1ull << 32,
                                (1ull << 32) - 1, (1ull << 32) + 1, 0xFFFFFFFF00000000ull,
                                1ull << 63, (1ull << 63) - 1, 0x8000000100000000ull};
  for (int i = 0; i < 4000; ++i) vals.push_back(rng() % P);
  for (size_t i = 0; i < vals.size(); ++i)
    for (size_t k = 0; k < 24; ++k) {
      uint64_t a = vals[i], b = vals[(i * 7 + k * 13 + 1) % vals.size()];
      CHECK(gl::mul(a, b) == rmul(a, b), "mul %llx %llx", (unsigned long long)a, (unsigned long long)b);
      CHECK(gl::add(a, b) == radd(a, b), "add %llx %llx", (unsigned long long)a, (unsigned long long)b);
      CHECK(gl::sub(a, b) == rsub(a, b), "sub %llx %llx", (unsigned long long)a, (unsigned long long)b);
    }
  for (unsigned s = 0; s < 192; ++s) {
    uint64_t t = rpow2(s);
    for (uint64_t a : vals) CHECK(gl::mul_pow2(a, s) == rmul(a, t), "mul_pow2 %llx s=%u", (unsigned long long)a, s);
  }
  // roots: 554^((p-1)/64) is 2^3, so small sub-transforms need only shifts
  CHECK(gl::pow(554, (P - 1) / 64) == 8, "omega_64 != 8");
  CHECK(gl::pow(gl::pow(7, (P - 1) / 192 * 5), 1) == 2, "7^(5(p-1)/192) != 2");
  for (uint64_t a : vals) if (a) CHECK(gl::mul(a, gl::inv(a)) == 1, "inv %llx", (unsigned long long)a);
  // digit x weight: |d| < 2^32 times a field element, against the general product
  {
    std::vector<int64_t> ds = {0, 1, -1, 2, -2, (1ll << 31) - 1, -(1ll << 31), (1ll << 32) - 1,
                               -((1ll << 32) - 1), 65535, -65536};
    for (int i = 0; i < 2000; ++i) ds.push_back((int64_t)(rng() >> 31) - (int64_t)(1ull << 32));
    for (int64_t d : ds)
      for (size_t k = 0; k < vals.size(); k += 7)
        CHECK(gl::mul_digit(d, vals[k]) == gl::mul(gl::from_signed(d), vals[k]), "mul_digit %lld %llx",
              (long long)d, (unsigned long long)vals[k]);
  }
  // signed views
  for (int64_t d : {0ll, 1ll, -1ll, 12345ll, -12345ll, (1ll << 40), -(1ll << 40)})
    CHECK(gl::to_signed(gl::from_signed(d)) == d, "signed round trip %lld", (long long)d);
  // balanced split: t = k 2^w + d with -2^(w-1) <= d < 2^(w-1)
  for (unsigned w = 1; w <= 30; ++w)
    for (int i = 0; i < 2000; ++i) {
      int64_t t = (int64_t)(rng() >> 12) - (int64_t)(1ull << 51);
      int64_t k, d = lnt::balance(t, w, k);
      CHECK(k * (int64_t(1) << w) + d == t && d >= -(int64_t(1) << (w - 1)) && d < (int64_t(1) << (w - 1)),
            "balance t=%lld w=%u", (long long)t, w);
    }
  // split_output: c = hi 2^w + lo, both readings
  for (unsigned w = 1; w <= 30; ++w)
    for (uint64_t c : vals) {
      int64_t hi, lo;
      lnt::split_output(c, true, w, hi, lo);
      CHECK((u128)(uint64_t)hi * ((u128)1 << w) + (u128)lo == (u128)c && lo >= 0 && lo < (int64_t(1) << w),
            "split unsigned %llx w=%u", (unsigned long long)c, w);
      lnt::split_output(c, false, w, hi, lo);
      __int128 s = (__int128)gl::to_signed(c);
      CHECK((__int128)hi * ((__int128)1 << w) + lo == s && lo >= 0 && lo < (int64_t(1) << w),
            "split signed %llx w=%u", (unsigned long long)c, w);
    }
  // carry_digit = split_output then balance(lo + carry), both readings; signed
  // outputs within the p/4 bound, carries of either sign
  for (unsigned w = 1; w <= 30; ++w)
    for (int i = 0; i < 4000; ++i) {
      const bool um = (i & 1) != 0;
      uint64_t c = rng() % gl::P;
      if (!um) c = gl::from_signed((int64_t)(rng() >> 3) - (int64_t)(1ull << 60));  // |s| < 2^61
      const int64_t carry = (int64_t)(rng() >> 28) - (int64_t)(1ull << 35);
      int64_t hi, lo, q, out;
      lnt::split_output(c, um, w, hi, lo);
      const int64_t d0 = lnt::balance(lo + carry, w, q);
      const int64_t d1 = lnt::carry_digit(c, um, carry, w, out);
      CHECK(d1 == d0 && out == hi + q, "carry_digit %llx carry=%lld w=%u um=%d", (unsigned long long)c,
            (long long)carry, w, (int)um);
    }
  if (fails) { std::printf("FAILED %d of %ld\n", fails, cases); return 1; }
  std::printf("ok %ld\n", cases);
  return 0;
}

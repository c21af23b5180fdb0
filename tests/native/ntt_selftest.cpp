// Host check of the register NTTs (cuda_b200/csrc/ntt_core.cuh): dif<R> equals
// the naive DFT with root 2^(192/R) in bit-reversed order, and dit_inv<R>
// inverts it up to the factor R.  Also checks shl_c for every shift.
#include <cstdio>
#include <cstdint>
#include <random>
#include "../../cuda_b200/csrc/ntt_core.cuh"

typedef unsigned __int128 u128;
static const uint64_t P = 0xFFFFFFFF00000001ull;
static uint64_t mulm(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a * b) % P); }
static uint64_t powm(uint64_t a, uint64_t e) { uint64_t r = 1; while (e) { if (e & 1) r = mulm(r, a); a = mulm(a, a); e >>= 1; } return r; }
static int fails = 0;

template <unsigned S> void check_shift(std::mt19937_64& rng) {
  for (int i = 0; i < 50; ++i) {
    uint64_t x = rng() % P;
    if (lnt::shl_c<S>(x) != mulm(x, powm(2, S))) { if (fails++ < 5) std::printf("shl_c<%u> %llx\n", S, (unsigned long long)x); }
  }
  if constexpr (S + 1 < 192) check_shift<S + 1>(rng);
}

template <int R> void check(std::mt19937_64& rng) {
  uint64_t w = powm(2, 192 / R);
  for (int rep = 0; rep < 40; ++rep) {
    uint64_t x[R], y[R];
    for (int i = 0; i < R; ++i) x[i] = y[i] = (rep == 0) ? P - 1 - i : rng() % P;
    lnt::dif<R>(y);
    for (int k = 0; k < R; ++k) {
      uint64_t s = 0;
      for (int i = 0; i < R; ++i) s = (uint64_t)(((u128)s + mulm(x[i], powm(w, (uint64_t)i * k))) % P);
      if (y[lnt::brev_c<R>(k)] != s) { if (fails++ < 5) std::printf("dif<%d> k=%d\n", R, k); }
    }
    lnt::dit_inv<R>(y);
    for (int i = 0; i < R; ++i)
      if (y[i] != mulm(x[i], R)) { if (fails++ < 5) std::printf("dit_inv<%d> i=%d\n", R, i); }
  }
}

int main() {
  std::mt19937_64 rng(3);
  check_shift<0>(rng);
  check<1>(rng); check<2>(rng); check<4>(rng); check<8>(rng); check<16>(rng); check<32>(rng); check<64>(rng);
  if (fails) { std::printf("FAILED %d\n", fails); return 1; }
  std::printf("ok\n");
  return 0;
}

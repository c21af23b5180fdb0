// Host run of the canonical-readout steps (cuda_b200/csrc/canon_core.cuh)
// against an exact sequential cyclic carry.  Prints "ok <cases>" or the first
// mismatch; exit code 1 on failure.
#include <cstdio>
#include <cstdint>
#include <random>
#include <vector>
#include "../../cuda_b200/csrc/canon_core.cuh"

using namespace lnt;

static std::vector<uint8_t> widths_of(uint32_t q, uint32_t n) {
  std::vector<uint8_t> w(n);
  for (uint32_t j = 0; j < n; ++j)
    w[j] = (uint8_t)(((uint64_t)q * (j + 1) + n - 1) / n - ((uint64_t)q * j + n - 1) / n);
  return w;
}

// exact reference: cyclic carry until stable, digits in [0, 2^w)
static std::vector<uint64_t> reference(std::vector<int64_t> v, const std::vector<uint8_t>& w) {
  const size_t n = v.size();
  int64_t carry = 0;
  size_t j = 0;
  bool wrapped = false;
  for (;;) {
    int64_t s = v[j] + carry;
    v[j] = s & ((int64_t(1) << w[j]) - 1);
    carry = s >> w[j];
    if (++j == n) { j = 0; wrapped = true; }
    if (wrapped && carry == 0) break;
  }
  return std::vector<uint64_t>(v.begin(), v.end());
}

static int fails = 0;
static long cases = 0;

static void run_case(uint32_t q, uint32_t n, const std::vector<int64_t>& x) {
  std::vector<uint8_t> w = widths_of(q, n);
  const uint32_t block = n < 64 ? n : 64, nb = n / block;
  std::vector<uint64_t> out(n);
  std::vector<int64_t> bc(nb);
  std::vector<uint8_t> bf(nb);
  std::vector<int8_t> bcin(nb);
  uint32_t flags = 0;
  CanonDesc D{};
  D.x = x.data(); D.carry = nullptr; D.widths = w.data(); D.out = out.data();
  D.blk_carry = bc.data(); D.blk_fn = bf.data(); D.blk_cin = bcin.data(); D.flags = &flags;
  D.n = n; D.block = block; D.nblocks = nb;
  for (uint32_t b = 0; b < nb; ++b) canon_local_block(D, b);
  bool ok = true;
  for (uint32_t b = 0; b < nb; ++b) ok = canon_hop_block(D, b) && ok;
  uint32_t total = canon_chunk_fn(D, 0, nb);
  int c;
  ok = canon_wrap_carry(total, c) && ok;
  canon_chunk_cin(D, 0, nb, c);
  bool nam = false, hnz = false;
  for (uint32_t b = 0; b < nb; ++b) canon_apply_block(D, b, nam, hnz);
  std::vector<uint64_t> ref = reference(x, w);
  ++cases;
  if (!ok || out != ref) {
    if (fails++ < 5) {
      std::printf("mismatch q=%u n=%u ok=%d\n got:", q, n, (int)ok);
      for (uint32_t j = 0; j < n && j < 8; ++j) std::printf(" %llu", (unsigned long long)out[j]);
      std::printf("\n ref:");
      for (uint32_t j = 0; j < n && j < 8; ++j) std::printf(" %llu", (unsigned long long)ref[j]);
      std::printf("\n");
    }
  }
}

int main() {
  // the state that exposed the readout fault: q = 89, n = 4 after 4 LL squarings
  run_case(89, 4, {-1356798, 169, 0, 0});
  std::mt19937_64 rng(7);
  const uint32_t qs[] = {89, 127, 1009, 9973, 44497, 160001};
  const uint32_t ns[] = {4, 8, 64, 512, 2048, 8192};
  for (int t = 0; t < 6; ++t) {
    uint32_t q = qs[t], n = ns[t];
    std::vector<uint8_t> w = widths_of(q, n);
    for (int rep = 0; rep < 200; ++rep) {
      std::vector<int64_t> x(n);
      int mode = rep % 5;
      for (uint32_t j = 0; j < n; ++j) {
        int64_t half = int64_t(1) << (w[j] - 1);
        if (mode == 0) x[j] = (int64_t)(rng() % (2 * half)) - half;     // balanced
        else if (mode == 1) x[j] = 0;                                   // zero ...
        else if (mode == 2) x[j] = (int64_t(1) << w[j]) - 1;            // all maximal (M)
        else if (mode == 3) x[j] = (int64_t)(rng() % (2 * half + 3)) - half - 1;  // excess 1
        else x[j] = (rng() % 16 == 0) ? (int64_t)(rng() % (2 * half)) - half : 0; // sparse
      }
      if (mode == 1) x[rng() % n] = -(int64_t)(rng() % 5) - 1;  // ... with one small negative
      run_case(q, n, x);
    }
  }
  if (fails) { std::printf("FAILED %d of %ld\n", fails, cases); return 1; }
  std::printf("ok %ld\n", cases);
  return 0;
}

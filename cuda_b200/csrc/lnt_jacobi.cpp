// Jacobi symbol of a Lucas-Lehmer residue, for the LL error check.
//
// No counterpart in the reference, which checks nothing during a test
// (lucas_prp.cu:137-195).  With u_0 = 4 and u_{k+1} = u_k^2 - 2 (mod M_q):
// u_k - 2 = (u_{k-1} - 2)(u_{k-1} + 2) and u_{k-1} + 2 = u_{k-2}^2, so the
// Jacobi symbol (u_k - 2 | M_q) is the same for every k >= 1, namely
// (12 | M_q) = (3 | M_q) = -1 (M_q = 1 mod 3 and (M_q - 1) / 2 is odd).  A
// residue whose symbol is +1 is wrong; an error leaves the symbol at -1 about
// half of the time, so the check finds about half of all errors.
//
// The symbol of a q-bit number needs a subquadratic big-integer algorithm;
// this file calls GMP's mpz_jacobi through its documented C interface, loaded
// at run time from libgmp.so.10 (no GMP headers are needed to build).
#include <dlfcn.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

namespace lnt {

namespace {

// mpz_t's layout in GMP's public interface: allocated limbs, signed size, limbs.
struct Mpz {
  int alloc;
  int size;
  void* d;
};

struct Gmp {
  void (*init)(Mpz*) = nullptr;
  void (*clear)(Mpz*) = nullptr;
  void (*import)(Mpz*, size_t, int, size_t, int, size_t, const void*) = nullptr;
  int (*jacobi)(const Mpz*, const Mpz*) = nullptr;
  void (*setbit)(Mpz*, unsigned long) = nullptr;
  void (*sub_ui)(Mpz*, const Mpz*, unsigned long) = nullptr;
  void (*add)(Mpz*, const Mpz*, const Mpz*) = nullptr;
  bool ok = false;
  std::string why;
};

const Gmp& gmp() {
  static Gmp g;
  static std::once_flag once;
  std::call_once(once, [] {
    void* h = dlopen("libgmp.so.10", RTLD_NOW | RTLD_LOCAL);
    if (!h) {
      g.why = std::string("libgmp.so.10 not found: ") + dlerror();
      return;
    }
    g.init = reinterpret_cast<void (*)(Mpz*)>(dlsym(h, "__gmpz_init"));
    g.clear = reinterpret_cast<void (*)(Mpz*)>(dlsym(h, "__gmpz_clear"));
    g.import = reinterpret_cast<void (*)(Mpz*, size_t, int, size_t, int, size_t, const void*)>(
        dlsym(h, "__gmpz_import"));
    g.jacobi = reinterpret_cast<int (*)(const Mpz*, const Mpz*)>(dlsym(h, "__gmpz_jacobi"));
    g.setbit = reinterpret_cast<void (*)(Mpz*, unsigned long)>(dlsym(h, "__gmpz_setbit"));
    g.sub_ui = reinterpret_cast<void (*)(Mpz*, const Mpz*, unsigned long)>(dlsym(h, "__gmpz_sub_ui"));
    g.add = reinterpret_cast<void (*)(Mpz*, const Mpz*, const Mpz*)>(dlsym(h, "__gmpz_add"));
    g.ok = g.init && g.clear && g.import && g.jacobi && g.setbit && g.sub_ui && g.add;
    if (!g.ok) g.why = "libgmp.so.10 lacks an mpz function";
  });
  return g;
}

}  // namespace

bool jacobi_available(std::string* why) {
  const Gmp& g = gmp();
  if (!g.ok && why) *why = g.why;
  return g.ok;
}

// (s - 2 | 2^q - 1) for the residue s given by canonical digits (digit j has
// width widths[j]; the value is sum d_j 2^(w_0 + ... + w_{j-1}), in [0, M]).
// Returns -1, 0 or +1; 2 when GMP is unavailable (*why says why).
int jacobi_of_ll_residue(const uint64_t* digits, const uint8_t* widths, uint32_t n, uint32_t q,
                         std::string* why) {
  const Gmp& g = gmp();
  if (!g.ok) {
    if (why) *why = g.why;
    return 2;
  }
  // pack the variable-width digits into 64-bit limbs, least significant first
  std::vector<uint64_t> limbs((q + 63) / 64 + 1, 0);
  uint64_t pos = 0;
  for (uint32_t j = 0; j < n; ++j) {
    const uint64_t d = digits[j];
    const uint32_t w = widths[j];
    if (w == 0) continue;
    const size_t li = (size_t)(pos >> 6);
    const uint32_t sh = (uint32_t)(pos & 63);
    limbs[li] |= d << sh;
    if (sh + w > 64) limbs[li + 1] |= d >> (64 - sh);
    pos += w;
  }
  Mpz s, m, a;
  g.init(&s);
  g.init(&m);
  g.init(&a);
  g.import(&s, limbs.size(), -1, 8, 0, 0, limbs.data());
  g.setbit(&m, q);
  g.sub_ui(&m, &m, 1);  // M = 2^q - 1
  // s - 2 mod M, as a non-negative number
  g.add(&a, &s, &m);
  g.sub_ui(&a, &a, 2);
  const int r = g.jacobi(&a, &m);
  g.clear(&a);
  g.clear(&m);
  g.clear(&s);
  return r;
}

}  // namespace lnt

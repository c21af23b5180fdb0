// Length policy and plan choice (host).
//
// lnt_secured_log2_length / lnt_length_candidates reproduce the reference's
// NttLengths::GetNttSecuredLength and GetCandidates (ntt_lengths.cu:88-128)
// bit for bit, including the double-precision arithmetic and the
// std::to_string(double) spelling of the candidates.  make_plan replaces the
// autotuned choice among pools (lucas_prp.cu:36-70, kernel_pool.cu:17-142).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/lucasntt.h"
#include "lnt_internal.h"

namespace lnt {

static const double kModulus = 18446744069414584321.0;  // p = 2^64 - 2^32 + 1 as a double

uint32_t secured_log2(uint32_t exponent) {
  double log_n = std::ceil(std::log2(1.0 * exponent / 32));
  double m = std::exp2(std::ceil(1.0 * exponent / std::exp2(log_n))) - 1;
  if (m * m >= kModulus / (2 * std::exp2(log_n))) log_n++;
  return (uint32_t)log_n;
}

std::vector<std::string> candidates(uint32_t exponent) {
  std::vector<std::string> c;
  uint32_t l = secured_log2(exponent);
  c.push_back(std::to_string(std::exp2(l)));
  if (l >= 10 && l <= 24) {
    uint32_t a = l / 2;
    c.push_back(std::to_string(std::exp2(a)) + ":" + std::to_string(std::exp2(l - a)));
    if (l - a != a) c.push_back(std::to_string(std::exp2(l - a)) + ":" + std::to_string(std::exp2(a)));
  }
  if (l == 23) { c.push_back("256:256:128"); c.push_back("512:256:64"); }
  if (l == 24) { c.push_back("512:256:128"); c.push_back("512:512:64"); }
  if (l == 25) { c.push_back("512:512:128"); c.push_back("1024:256:128"); c.push_back("1024:512:64"); }
  if (l == 26) { c.push_back("512:512:256"); c.push_back("1024:256:256"); c.push_back("1024:512:128"); }
  return c;
}

// StringToLength + FillLength (ntt_lengths.cu:32-68): one factor of a
// description, with an optional K / M suffix; 2^a 3^b 5^c with b, c <= 1.
struct Factor { uint32_t n, log2, log3, log5; };

static bool parse_factor(std::string d, Factor& f) {
  uint32_t mult = 1;
  if (d.empty()) return false;
  if (std::toupper((unsigned char)d.back()) == 'K') { mult = 1024; d.pop_back(); }
  if (!d.empty() && std::toupper((unsigned char)d.back()) == 'M') { mult = 1024 * 1024; d.pop_back(); }
  long v;
  try { v = std::stol(d); } catch (...) { return false; }
  if (v <= 0) return false;
  uint64_t n = (uint64_t)v * mult;
  if (n > 0xFFFFFFFFull) return false;
  f = {(uint32_t)n, 0, 0, 0};
  uint32_t m = f.n;
  while (m % 2 == 0) { f.log2++; m /= 2; }
  while (m % 3 == 0) { f.log3++; m /= 3; }
  while (m % 5 == 0) { f.log5++; m /= 5; }
  return m == 1 && f.log3 <= 1 && f.log5 <= 1;
}

static bool parse_description(const char* s, std::vector<Factor>& out) {
  if (!s) return false;
  std::string str(s), item;
  size_t start = 0;
  while (true) {
    size_t pos = str.find(':', start);
    item = str.substr(start, pos == std::string::npos ? std::string::npos : pos - start);
    Factor f;
    if (!parse_factor(item, f)) return false;
    out.push_back(f);
    if (pos == std::string::npos) break;
    start = pos + 1;
  }
  return !out.empty();
}

static void name_plan(Plan& plan) {
  if (plan.kind == PlanKind::Resident) {
    plan.name = "RESIDENT_" + std::to_string(plan.n);
    return;
  }
  plan.name = "TWOPASS_" + std::to_string(plan.n2) + "x" +
              (plan.five ? "5x" + std::to_string(plan.n1 / 5) : std::to_string(plan.n1)) +
              (plan.fast ? "_R" + std::to_string(plan.radix) : std::string("_R2")) + "_T" +
              std::to_string(plan.tile) + (plan.fused ? "_F" : "");
}

// Column tiles the kernels can stage: radix-16 columns of 4096 words only fit
// shared memory four columns wide; radix-2 columns longer than 2048 likewise.
static bool tile_fits(bool fast, uint32_t log2n2, uint32_t tile) {
  if (tile != 4 && tile != 8) return false;
  if (fast) return tile == 4 || log2n2 < 12;
  return tile == 4 || log2n2 <= 11;
}

bool five_length(uint32_t n) {
  return n >= 5 && n % 5 == 0 && ((n / 5) & (n / 5 - 1)) == 0;
}

// n = 5 * 2^k: register-pass two-pass plans only.  Rows hold n1 = 5 L words (the
// five stride-5 planes of L words each take the L-point passes, then a radix-5
// step), columns n2 words as for 2^k; 2^7 <= L <= 2^12, 2^6 <= n2 <= 2^12.
// Policy: rows of L = 2^11 (87 KB of shared memory) where the columns allow.
static bool make_five_plan(uint32_t n, uint32_t exponent, PlanOptions o, Plan& plan,
                           std::string* why) {
  auto reject = [&](const char* msg) {
    if (why) *why = msg;
    return false;
  };
  uint32_t k = 0;
  while ((5u << k) < n) ++k;
  if (k < 13 || k > 24) return reject("length 5 * 2^k needs 13 <= k <= 24");
  if (o.kind != 0 && o.kind != 2) return reject("lengths 5 * 2^k run on the register-pass plan only");
  if (o.radix != 0 && o.radix != 8) return reject("lengths 5 * 2^k take radix-8 passes");
  if (o.fused > 2) return reject("fused must be 0 (policy), 1 (fused) or 2 (two launches)");
  plan = Plan();
  plan.n = n;
  while ((1ull << plan.log2n) < n) plan.log2n++;
  plan.kind = PlanKind::TwoPass;
  plan.fast = true;
  plan.five = true;
  uint32_t l2 = o.log2_rows, l1;
  if (l2 == 0) {
    l1 = k - 6 < 11 ? k - 6 : 11;
    l2 = k - l1;
    if (l2 > 12) {
      l2 = 12;
      l1 = k - 12;
    }
  } else {
    if (l2 >= k) return reject("column length exceeds the length");
    l1 = k - l2;
  }
  if (l2 < 6 || l2 > 12 || l1 < 7 || l1 > 12 || (5u << l1) < (1u << l2))
    return reject("5 * 2^k plan needs 2^6 <= n2 <= 2^12, 2^7 <= L <= 2^12, 5 L >= n2");
  const uint32_t run_words = exponent ? r16_run_words_needed(exponent, n) : 8;
  uint32_t tile = o.tile;
  if (tile == 0) {
    tile = (run_words <= 4 && tile_fits(true, l2, 4)) ? 4 : 8;
    if (!tile_fits(true, l2, tile)) tile = 4;
  } else if (!tile_fits(true, l2, tile)) {
    return reject("column tile must be 4 or 8 and fit shared memory");
  } else if (exponent && tile < run_words && tile < 8 && tile_fits(true, l2, 8)) {
    // as the policy: 4-word runs where 8-word tiles do not fit (the kernels' carry check
    // reports a carry that outruns them)
    return reject("carry runs of this tile are too short for the exponent");
  }
  plan.log2n1 = l1;  // log2 L: the transform length of each plane
  plan.log2n2 = l2;
  plan.n1 = 5u << l1;
  plan.n2 = 1u << l2;
  plan.tile = tile;
  plan.ntiles = plan.n1 / tile;
  plan.radix = 8;
  plan.fused = o.fused ? o.fused == 1 : plan.log2n >= 19;
  name_plan(plan);
  return true;
}

bool make_plan(uint32_t n, uint32_t exponent, const PlanOptions* opt, Plan& plan,
               std::string* why) {
  auto reject = [&](const char* msg) {
    if (why) *why = msg;
    return false;
  };
  PlanOptions o = opt ? *opt : PlanOptions();
  if (five_length(n)) return make_five_plan(n, exponent, o, plan, why);
  if (n < 2 || (n & (n - 1)) || n > (1u << kMaxLog2))
    return reject("length must be 2^k (1 <= k <= 26) or 5 * 2^k (13 <= k <= 24)");
  if (o.kind > 3) return reject("unknown plan kind");
  if (o.radix != 0 && o.radix != 8 && o.radix != 16) return reject("pass radix must be 8 or 16");
  if (o.fused > 2) return reject("fused must be 0 (policy), 1 (fused) or 2 (two launches)");
  plan = Plan();
  plan.n = n;
  while ((1u << plan.log2n) < n) plan.log2n++;
  if (o.kind == 0) o.kind = plan.log2n <= kResidentMaxLog2 ? 1 : 0;
  if (o.kind == 1) {
    if (plan.log2n > kResidentMaxLog2) return reject("resident plan needs n <= 4096");
    if (o.log2_rows || o.tile || o.radix || o.fused)
      return reject("resident plan takes no split, tile, radix or fusion choice");
    plan.kind = PlanKind::Resident;
    name_plan(plan);
    return true;
  }
  if (plan.log2n <= kResidentMaxLog2) return reject("two-pass plans need n >= 8192");
  plan.kind = PlanKind::TwoPass;
  const uint32_t run_words = exponent ? r16_run_words_needed(exponent, n) : 8;
  uint32_t l2 = o.log2_rows, l1;
  if (o.kind == 0) {
    // policy: radix-16 with the most square split the kernels take
    const uint32_t p2 = plan.log2n / 2 < 12 ? plan.log2n / 2 : 12;
    if (l2 == 0 ? r16_supported(plan.log2n - p2, p2) : r16_supported(plan.log2n - l2, l2))
      o.kind = 2;
    else
      o.kind = 3;
  }
  plan.fast = o.kind == 2;
  if (!plan.fast && (o.radix || o.fused)) return reject("radix and fusion choices need the register-pass kernels");
  if (plan.fast) {
    if (l2 == 0) l2 = plan.log2n / 2 < 12 ? plan.log2n / 2 : 12;
    l1 = plan.log2n - l2;
    if (!r16_supported(l1, l2)) return reject("radix-16 plan needs 2^6 <= n2 <= n1 <= 2^12, n1 >= 2^7");
  } else {
    if (l2 == 0) {
      l2 = plan.log2n / 2;
      if (l2 > 11) l2 = 11;
      l1 = plan.log2n - l2;
      if (l1 > 14) { l1 = 14; l2 = plan.log2n - 14; }
    } else {
      l1 = plan.log2n - l2;
    }
    if (l2 < 1 || l1 < 1 || l1 > 14 || l2 > 12) return reject("radix-2 plan needs n1 <= 2^14, n2 <= 2^12");
  }
  uint32_t tile = o.tile;
  if (tile == 0) {
    // narrowest tile whose runs absorb every carry (more CTAs per SM)
    tile = (run_words <= 4 && tile_fits(plan.fast, l2, 4)) ? 4 : 8;
    if (!tile_fits(plan.fast, l2, tile)) tile = 4;
  } else if (!tile_fits(plan.fast, l2, tile)) {
    return reject("column tile must be 4 or 8 and fit shared memory");
  } else if (exponent && tile < run_words && tile < 8 && tile_fits(plan.fast, l2, 8)) {
    // as the policy: 4-word runs where 8-word tiles do not fit (the kernels' carry check
    // reports a carry that outruns them)
    return reject("carry runs of this tile are too short for the exponent");
  }
  if ((1u << l1) < tile) return reject("rows shorter than the tile");
  plan.log2n1 = l1;
  plan.log2n2 = l2;
  plan.n1 = 1u << l1;
  plan.n2 = 1u << l2;
  plan.tile = tile;
  plan.ntiles = plan.n1 / plan.tile;
  if (plan.fast) {
    plan.radix = o.radix ? o.radix : 8;
    // policy: the carry-fused column kernel from 2^19 words, where its tiles
    // fill the GPU; the autotuner may choose either way at any length
    plan.fused = o.fused ? o.fused == 1 : plan.log2n >= 19;
  }
  name_plan(plan);
  return true;
}

static PlanOptions options_of(const Plan& p) {
  PlanOptions o;
  if (p.kind == PlanKind::Resident) {
    o.kind = 1;
    return o;
  }
  o.kind = p.fast ? 2 : 3;
  o.log2_rows = p.log2n2;
  o.tile = p.tile;
  if (p.fast) {
    o.radix = p.radix;
    o.fused = p.fused ? 1 : 2;
  }
  return o;
}

std::vector<PlanOptions> plan_candidates(uint32_t n, uint32_t exponent) {
  std::vector<PlanOptions> out;
  auto add = [&](const PlanOptions& o) {
    for (const PlanOptions& c : out)
      if (c.kind == o.kind && c.log2_rows == o.log2_rows && c.tile == o.tile && c.radix == o.radix &&
          c.fused == o.fused)
        return;
    out.push_back(o);
  };
  Plan plan;
  if (!make_plan(n, exponent, nullptr, plan)) return out;
  add(options_of(plan));  // the policy's plan first
  if (plan.kind == PlanKind::Resident) return out;
  const bool r16 = plan.fast;
  for (uint32_t l2 = 1; l2 <= 12 && l2 < plan.log2n; ++l2)
    for (uint32_t tile : {4u, 8u})
      for (uint32_t radix : {8u, 16u})
        for (uint32_t fused : {1u, 2u}) {
          // radix-2 only where no register-pass plan exists, with splits near square
          PlanOptions o;
          o.kind = r16 ? 2 : 3;
          o.log2_rows = l2;
          o.tile = tile;
          if (r16) {
            o.radix = radix;
            o.fused = fused;
          } else if (radix != 8 || fused != 1) {
            continue;
          }
          Plan p;
          if (!make_plan(n, exponent, &o, p)) continue;
          const int skew = (int)p.log2n1 - (int)p.log2n2;
          if (!r16 && (skew < 0 || skew > 3)) continue;
          add(o);
        }
  return out;
}

void word_widths(uint32_t exponent, uint32_t n, uint8_t* widths) {
  uint64_t start = 0;  // ceil(qj/n)
  for (uint32_t j = 0; j < n; ++j) {
    const uint64_t next = ((uint64_t)exponent * (j + 1) + n - 1) / n;
    widths[j] = (uint8_t)(next - start);
    start = next;
  }
}

std::vector<uint32_t> shifted_words(uint32_t exponent, uint32_t n) {
  std::vector<uint32_t> out;
  for (uint32_t j = 1; j < n; ++j) {
    // the reference's start bit: its double widths telescope to ceil_double(qj/n)
    const double ref = std::ceil(1.0 * exponent * (double)j / n);
    if ((uint64_t)ref != ((uint64_t)exponent * j + n - 1) / n) out.push_back(j);
  }
  return out;
}

}  // namespace lnt

extern "C" {

int lnt_smallest_length(uint32_t exponent, uint32_t* n_out) {
  if (!n_out || exponent < 3) return LNT_ERR_INVALID_ARGUMENT;
  std::vector<uint32_t> cand;
  for (uint32_t k = 1; k <= lnt::kMaxLog2; ++k) cand.push_back(1u << k);
  for (uint32_t k = 13; k <= 24; ++k) cand.push_back(5u << k);
  std::sort(cand.begin(), cand.end());
  for (uint32_t n : cand) {
    if (n > exponent) break;
    // the reference's bound (ntt_lengths.cu:94): 2 n (2^W - 1)^2 < p, W = ceil(q / n)
    const double w = std::ceil(1.0 * exponent / n), m = std::exp2(w) - 1;
    if (w > 30 || m * m >= lnt::kModulus / (2.0 * n)) continue;
    lnt::Plan plan;
    if (!lnt::make_plan(n, exponent, nullptr, plan)) continue;
    *n_out = n;
    return LNT_OK;
  }
  return LNT_ERR_UNSUPPORTED_LENGTH;
}

int lnt_shifted_words(uint32_t exponent, uint32_t n, uint32_t* count, uint32_t* first) {
  if (!count || exponent < 3 || n < 2 || (n & (n - 1)) || n > (1u << lnt::kMaxLog2))
    return LNT_ERR_INVALID_ARGUMENT;
  const std::vector<uint32_t> s = lnt::shifted_words(exponent, n);
  *count = (uint32_t)s.size();
  if (first) *first = s.empty() ? 0 : s[0];
  return LNT_OK;
}

uint32_t lnt_secured_log2_length(uint32_t exponent) { return lnt::secured_log2(exponent); }

int lnt_length_candidates(uint32_t exponent, char* out, size_t outlen) {
  std::vector<std::string> c = lnt::candidates(exponent);
  if (out && outlen) {
    std::string joined;
    for (auto& s : c) joined += s + ";";
    size_t k = joined.size() < outlen - 1 ? joined.size() : outlen - 1;
    std::memcpy(out, joined.data(), k);
    out[k] = 0;
  }
  return (int)c.size();
}

int lnt_parse_length(const char* description, uint32_t* n_out) {
  std::vector<lnt::Factor> fs;
  if (!n_out || !lnt::parse_description(description, fs)) return LNT_ERR_INVALID_ARGUMENT;
  uint64_t n = 1;
  uint32_t l3 = 0, l5 = 0;
  for (auto& f : fs) { n *= f.n; l3 += f.log3; l5 += f.log5; }
  if (n > 0xFFFFFFFFull) return LNT_ERR_INVALID_ARGUMENT;
  *n_out = (uint32_t)n;
  if (l3 || l5 > 1) return LNT_ERR_UNSUPPORTED_LENGTH;  // 5 * 2^k has a kernel, 3 * 2^k none
  return LNT_OK;
}

int lnt_check_provided_length(uint32_t exponent, const char* description, int* diff) {
  std::vector<lnt::Factor> fs;
  if (!diff || !lnt::parse_description(description, fs)) return LNT_ERR_INVALID_ARGUMENT;
  int log_n = 0;
  for (auto& f : fs) log_n += (int)f.log2;
  *diff = (int)lnt::secured_log2(exponent) - log_n;
  return LNT_OK;
}

}  // extern "C"

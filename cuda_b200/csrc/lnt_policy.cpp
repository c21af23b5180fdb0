// Length policy and plan choice (host).
//
// lnt_secured_log2_length / lnt_length_candidates reproduce the reference's
// NttLengths::GetNttSecuredLength and GetCandidates (ntt_lengths.cu:88-128)
// bit for bit, including the double-precision arithmetic and the
// std::to_string(double) spelling of the candidates.  make_plan replaces the
// autotuned choice among pools (lucas_prp.cu:36-70, kernel_pool.cu:17-142).
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

bool make_plan(uint32_t n, Plan& plan) {
  if (n < 2 || (n & (n - 1)) || n > (1u << kMaxLog2)) return false;
  plan = Plan();
  plan.n = n;
  while ((1u << plan.log2n) < n) plan.log2n++;
  if (plan.log2n <= kResidentMaxLog2) {
    plan.kind = PlanKind::Resident;
    plan.name = "RESIDENT_" + std::to_string(n);
    return true;
  }
  plan.kind = PlanKind::TwoPass;
  uint32_t l2 = plan.log2n / 2;
  uint32_t l1 = plan.log2n - l2;
  if (r16_supported(l1, l2)) {
    // radix-16 pass kernels
    plan.fast = true;
    plan.tile = r16_tile(l2);
  } else {
    if (l2 > 11) l2 = 11;
    l1 = plan.log2n - l2;
    if (l1 > 14) { l1 = 14; l2 = plan.log2n - 14; }
    plan.tile = l2 <= 11 ? 8 : 4;
  }
  plan.log2n1 = l1;
  plan.log2n2 = l2;
  plan.n1 = 1u << l1;
  plan.n2 = 1u << l2;
  plan.ntiles = plan.n1 / plan.tile;
  plan.name = "TWOPASS_" + std::to_string(plan.n2) + "x" + std::to_string(plan.n1) +
              (plan.fast ? "_R16" : "_R2");
  return true;
}

}  // namespace lnt

extern "C" {

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
  if (l3 || l5) return LNT_ERR_UNSUPPORTED_LENGTH;
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

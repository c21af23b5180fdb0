#include "residue_files.h"

#include <cinttypes>
#include <cstdio>
#include <cstring>

namespace lucasntt {

bool WriteResidueFile(const std::string& path, const std::vector<uint64_t>& digits) {
  FILE* fp = std::fopen(path.c_str(), "w+");
  if (!fp) return false;
  // one buffered pass: 19 bytes per word
  std::vector<char> buf(19 * 4096 + 1);
  size_t used = 0;
  bool ok = true;
  for (size_t i = 0; i < digits.size(); ++i) {
    used += (size_t)std::snprintf(buf.data() + used, 20, "0x%016" PRIX64 "\n", digits[i]);
    if (used + 19 > 19 * 4096) {
      ok &= std::fwrite(buf.data(), 1, used, fp) == used;
      used = 0;
    }
  }
  if (used) ok &= std::fwrite(buf.data(), 1, used, fp) == used;
  ok &= std::fclose(fp) == 0;
  return ok;
}

namespace {

int hexval(char c) {
  if (c >= '0' && c <= '9') return c - '0';
  if (c >= 'A' && c <= 'F') return c - 'A' + 10;
  if (c >= 'a' && c <= 'f') return c - 'a' + 10;
  return -1;
}

}  // namespace

bool ReadResidueFile(const std::string& path, const std::vector<uint8_t>& widths,
                     std::vector<uint64_t>& digits, std::string* why) {
  auto reject = [&](const std::string& msg) {
    if (why) *why = msg;
    return false;
  };
  FILE* fp = std::fopen(path.c_str(), "rb");
  if (!fp) return reject("cannot open " + path);
  const size_t n = widths.size();
  digits.assign(n, 0);
  char rec[19];
  size_t i = 0;
  bool ok = true;
  std::string msg;
  while (ok) {
    const size_t got = std::fread(rec, 1, sizeof rec, fp);
    if (got == 0) break;
    if (got != sizeof rec) { ok = false; msg = "truncated record " + std::to_string(i); break; }
    if (i >= n) { ok = false; msg = "more than " + std::to_string(n) + " records"; break; }
    if (rec[0] != '0' || (rec[1] != 'x' && rec[1] != 'X') || rec[18] != '\n') {
      ok = false;
      msg = "malformed record " + std::to_string(i);
      break;
    }
    uint64_t v = 0;
    for (int k = 2; k < 18; ++k) {
      const int h = hexval(rec[k]);
      if (h < 0) { ok = false; msg = "malformed record " + std::to_string(i); break; }
      v = (v << 4) | (uint64_t)h;
    }
    if (!ok) break;
    if (widths[i] < 64 && (v >> widths[i]) != 0) {
      ok = false;
      msg = "digit " + std::to_string(i) + " exceeds its width";
      break;
    }
    digits[i++] = v;
  }
  std::fclose(fp);
  if (!ok) return reject(msg);
  if (i != n) return reject("expected " + std::to_string(n) + " records, found " + std::to_string(i));
  return true;
}

bool WriteStatsFile(const std::string& path, const StatsRecord& r) {
  FILE* fp = std::fopen(path.c_str(), "w+");
  if (!fp) return false;
  std::fprintf(fp, "Exponent = %u\n", r.exponent);
  if (r.is_prime) std::fprintf(fp, "Conclusion = %sPrime\n", r.prp ? "Probably " : "");
  if (r.is_composite) std::fprintf(fp, "Conclusion = Composite\n");
  if (!r.is_prime && !r.is_composite) std::fprintf(fp, "Conclusion = Partial\n");
  std::fprintf(fp, "PRP = %d\n", r.prp ? 1 : 0);
  std::fprintf(fp, "Iterations = %u\n", r.iterations);
  std::fprintf(fp, "fft = %s\n", r.fft.c_str());
  std::fprintf(fp, "n = %u\n", r.n);
  std::fprintf(fp, "log2_n = %u\n", r.log2_n);
  std::fprintf(fp, "log3_n = %u\n", r.log3_n);
  std::fprintf(fp, "log5_n = %u\n", r.log5_n);
  for (const auto& p : r.performances)
    std::fprintf(fp, "Candidate Performance (in ms for %ld loops): %s = %g\n", r.performance_loops,
                 p.first.c_str(), p.second);
  std::fprintf(fp, "Pool = %s\n", r.pool.c_str());
  for (size_t i = 0; i < r.kernels.size(); ++i)
    std::fprintf(fp, "Kernel%zu = %s\n", i, r.kernels[i].c_str());
  std::fprintf(fp, "Interrupted = %d\n", r.interrupted ? 1 : 0);
  std::fprintf(fp, "currentIteration = %u\n", r.current_iteration);
  std::fprintf(fp, "Per iteration (ms) = %g\n", r.per_iteration_ms);
  if (r.was_interrupted)
    std::fprintf(fp, "Warning! total time is not relevant since the full process has been interrupted by CTRL-C\n");
  std::fprintf(fp, "Total time (sec) = %g\n", r.total_seconds);
  if (r.has_res64) std::fprintf(fp, "Res64 = %016" PRIX64 "\n", r.res64);
  if (r.has_gerbicz) {
    std::fprintf(fp, "Gerbicz checks = %" PRIu64 "\n", r.gerbicz_checks);
    std::fprintf(fp, "Gerbicz errors = %" PRIu64 "\n", r.gerbicz_errors);
  }
  if (r.has_jacobi) {
    std::fprintf(fp, "Jacobi checks = %" PRIu64 "\n", r.jacobi_checks);
    std::fprintf(fp, "Jacobi errors = %" PRIu64 "\n", r.jacobi_errors);
  }
  return std::fclose(fp) == 0;
}

bool WriteTextFile(const std::string& path, const std::string& text) {
  FILE* fp = std::fopen(path.c_str(), "w+");
  if (!fp) return false;
  const bool ok = std::fwrite(text.data(), 1, text.size(), fp) == text.size();
  return (std::fclose(fp) == 0) && ok;
}

}  // namespace lucasntt

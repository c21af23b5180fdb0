#include "lucas_prp.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <stdexcept>

#include "logger.h"
#include "residue_files.h"

namespace lucasntt {

volatile std::sig_atomic_t g_interrupted = 0;

namespace {

using Clock = std::chrono::steady_clock;

double ms_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

// Res64 of canonical digits: the low 64 bits of sum d_j 2^(w_0 + ... + w_{j-1})
uint64_t res64_of(const std::vector<uint64_t>& d, const std::vector<uint8_t>& w) {
  uint64_t r = 0;
  unsigned off = 0;
  for (size_t j = 0; j < d.size() && off < 64; off += w[j], ++j) r |= d[j] << off;
  return r;
}

}  // namespace

LucasPRP::LucasPRP(MainOptions& options, const lnt_plan_options& plan, uint32_t n,
                   std::vector<Candidate> performances)
    : o_(options), plan_(plan), n_(n), performances_(std::move(performances)) {
  char buf[128];
  if (lnt_plan_describe(&plan_, o_.exponent, n_, buf, sizeof buf) == LNT_OK)
    Name = std::string("LucasPRP ") + buf;
  else
    Name = "LucasPRP";
}

LucasPRP::~LucasPRP() { Finalize(); }

void LucasPRP::Check(int status, const char* what) {
  if (status == LNT_OK) return;
  throw std::runtime_error(std::string(what) + " failed: " + lnt_status_string(status) + " (" +
                           lnt_last_error() + ")");
}

bool LucasPRP::Initialize() {
  const int st = lnt_create_with_plan(o_.exponent, n_, o_.prp ? 1 : 0, o_.gpu, &plan_, &t_);
  if (st != LNT_OK) {
    LOG_NORMAL("Cannot create the test: %s (%s)", lnt_status_string(st), lnt_last_error());
    return false;
  }
  widths_.resize(n_);
  Check(lnt_get_widths(t_, widths_.data(), n_), "lnt_get_widths");
  host_x_.assign(n_, 0);
  return true;
}

void LucasPRP::Finalize() {
  if (t_) lnt_destroy(t_);
  t_ = nullptr;
}

void LucasPRP::InitializeTest() { Check(lnt_init_test(t_), "lnt_init_test"); }

void LucasPRP::Run() {
  if (o_.was_interrupted) {
    if (LoadResidue()) {
      LOG_NORMAL("Previous residue successfully loaded!");
    } else {
      LOG_NORMAL("Failed to restore previous residue, restarting from iteration 1!");
      InitializeTest();
      o_.from_iteration = 1;
    }
  } else {
    InitializeTest();
  }
  EnableChecks();
  const Clock::time_point t0 = Clock::now();
  MainLoop();
  Check(lnt_synchronize(t_), "lnt_synchronize");
  total_ms_ = ms_since(t0);

  Check(lnt_get_digits(t_, host_x_.data(), n_), "lnt_get_digits");
  if (current_iteration_ > MaxIterations(o_)) {
    // verdict of lucas_prp.cu:167-184 on the final residue
    is_prime_ = host_x_[0] == (o_.prp ? 9u : 0u);
    for (uint32_t i = 1; i < n_ && is_prime_; ++i) is_prime_ = host_x_[i] == 0;
    if (is_prime_) {
      LOG_NORMAL("\n\nM(%u) is %sprime!\n", o_.exponent, o_.prp ? "probably " : "");
    } else {
      is_composite_ = true;
      LOG_NORMAL("\n\nM(%u) is composite!\n", o_.exponent);
    }
  } else {
    LOG_NORMAL("\n\n%u loops performed with M(%u)\n", current_iteration_ - o_.from_iteration,
               o_.exponent);
  }
  LOG_VERBOSE("Res64 = %016llX", (unsigned long long)res64_of(host_x_, widths_));

  if (o_.dump_residue || interrupted_ || current_iteration_ + 2 <= o_.exponent) DumpResidue();
  if (o_.dump_environment) DumpEnvironment();
  if (o_.dump_stats) DumpStats(total_ms_);
}

// The error checks (extensions): the Gerbicz-Li check of PRP tests
// (GerbiczBlock) or the Jacobi check of LL tests (JacobiCheck), on the residue the loop
// starts from: a fresh test or the residue a resume loaded.
void LucasPRP::EnableChecks() {
  if (!o_.prp && o_.jacobi_interval) {
    // the Jacobi check of LL tests (JacobiCheck, an extension): the symbol is
    // defined from the first squaring on, so the check starts from the residue
    // the loop begins with (a fresh start or a resumed one)
    const int st = lnt_jacobi_enable(t_, o_.jacobi_interval);
    jacobi_ = st == LNT_OK;
    if (jacobi_)
      LOG_VERBOSE("Jacobi check every %llu squarings", (unsigned long long)o_.jacobi_interval);
    else
      LOG_NORMAL("Jacobi check not available for this test: %s", lnt_last_error());
    return;
  }
  if (!o_.prp || o_.gerbicz_block == 0) return;
  const int st = lnt_gerbicz_enable(t_, o_.gerbicz_block);
  gerbicz_ = st == LNT_OK;
  if (gerbicz_)
    LOG_VERBOSE("Gerbicz check every %u squarings", o_.gerbicz_block * o_.gerbicz_block);
  else
    LOG_NORMAL("Gerbicz check not available for this test: %s", lnt_last_error());
}

void LucasPRP::MainLoop() {
  // iterations per minute (progress) and per safety period (residue dump),
  // from the evaluated performance, 2 % early as lucas_prp.cu:198-203
  double per_it = Performance > 0 && o_.performance_loops > 0 ? Performance / o_.performance_loops : 0;
  if (per_it <= 0) per_it = 1.0;
  const uint64_t pit_stop = std::max<uint64_t>(1, (uint64_t)(60.0 * 1000.0 / per_it * 0.98));
  const uint64_t dump_every =
      std::max<uint64_t>(1, (uint64_t)(o_.safety_dump_seconds * 1000.0 / per_it * 0.98));
  // squarings per chunk between checks of the interrupt flag: about 50 ms
  const uint64_t chunk = std::max<uint64_t>(1, (uint64_t)(50.0 / per_it));
  const Clock::time_point t0 = Clock::now();
  uint64_t since_dump = 0, since_pit = 0;
  uint64_t cur = o_.from_iteration;
  while (cur <= o_.iterations) {
    if (g_interrupted) {
      interrupted_ = true;
      break;
    }
    const uint64_t todo = std::min({(uint64_t)o_.iterations - cur + 1, chunk, dump_every - since_dump,
                                    pit_stop - since_pit});
    int st = lnt_iterate(t_, todo);
    if (st == LNT_OK) st = lnt_synchronize(t_);
    if (st != LNT_OK) {
      // which squarings failed, for the user's report
      const std::string where = "squarings " + std::to_string(cur) + " to " + std::to_string(cur + todo - 1);
      Check(st, where.c_str());
    }
    cur += todo;
    since_dump += todo;
    since_pit += todo;
    current_iteration_ = (uint32_t)cur;
    if (since_dump >= dump_every && cur <= o_.iterations) {
      since_dump = 0;
      LOG_NORMAL("\nNow dumping intermediate residue for safety reasons...\n");
      Check(lnt_get_digits(t_, host_x_.data(), n_), "lnt_get_digits");
      DumpResidue();
      DumpStats(ms_since(t0));
    }
    if (since_pit >= pit_stop) {
      since_pit = 0;
      if (Logger::Get().GetVerbosity() != Verbosity::Silent) DisplayPitStop(ms_since(t0));
    }
  }
  current_iteration_ = (uint32_t)cur;
}

// LucasPRP::DisplayPitStop (lucas_prp.cu:231-252)
void LucasPRP::DisplayPitStop(double elapsed) {
  const long long h = (long long)(elapsed / 3600000.0);
  const long long m = (long long)((elapsed / 1000.0 - h * 3600) / 60);
  const long long s = (long long)(elapsed / 1000.0) - h * 3600 - m * 60;
  const double done = (double)current_iteration_ - (double)o_.from_iteration;
  const double per = done > 0 ? elapsed / done : 0;
  const double remaining = per * ((double)o_.iterations - (double)current_iteration_ + 1);
  const long long h2 = (long long)(remaining / 3600000.0);
  const long long m2 = (long long)((remaining / 1000.0 - h2 * 3600) / 60);
  const long long s2 = (long long)(remaining / 1000.0) - h2 * 3600 - m2 * 60;
  const double pct = 100.0 * ((double)current_iteration_ - 1) / (double)o_.iterations;
  LOG_NORMAL("%d%% - Elapsed %02lld:%02lld:%02lld - Remaining %02lld:%02lld:%02lld - Per iteration %.4f ms",
             (int)pct, h, m, s, h2, m2, s2, per);
}

void LucasPRP::DumpResidue() {
  if (!WriteResidueFile(o_.dump_filename, host_x_))
    LOG_NORMAL("Cannot write the residue to %s", o_.dump_filename.c_str());
}

bool LucasPRP::LoadResidue() {
  std::vector<uint64_t> d;
  std::string why;
  if (!ReadResidueFile(o_.dump_filename, widths_, d, &why)) {
    LOG_VERBOSE("Residue file %s not usable: %s", o_.dump_filename.c_str(), why.c_str());
    return false;
  }
  std::remove(o_.dump_filename.c_str());  // as the reference, lucas_prp.cu:342
  Check(lnt_set_digits(t_, d.data(), d.size()), "lnt_set_digits");
  host_x_ = d;
  return true;
}

void LucasPRP::DumpEnvironment() {
  std::vector<char> buf(1 << 16);
  if (lnt_environment(buf.data(), buf.size()) != LNT_OK ||
      !WriteTextFile(o_.env_filename, std::string(buf.data())))
    LOG_NORMAL("Cannot write the environment to %s", o_.env_filename.c_str());
}

void LucasPRP::DumpStats(double total_ms) {
  StatsRecord r;
  r.exponent = o_.exponent;
  r.prp = o_.prp;
  r.is_prime = is_prime_;
  r.is_composite = is_composite_;
  r.iterations = o_.iterations;
  r.n = n_;
  while ((1u << r.log2_n) < n_) r.log2_n++;
  lnt_plan_options used{};
  if (lnt_get_plan(t_, &used) == LNT_OK && used.kind != LNT_PLAN_RESIDENT) {
    const uint32_t n2 = 1u << used.log2_rows;
    r.fft = std::to_string(n2) + ":" + std::to_string(n_ / n2);
    const std::string t = std::to_string(used.tile);
    if (used.kind == LNT_PLAN_RADIX16)
      r.kernels = {"col_forward_r16<" + t + ">", n_ % 5 == 0 ? "row5_r16" : "row_square_r16",
                   "col_inverse_r16<" + t + ">"};
    else
      r.kernels = {"col_forward", "row_square", "col_inverse"};
  } else {
    r.fft = std::to_string(n_);
    r.kernels = {"resident_square_loop"};
  }
  r.performance_loops = o_.performance_loops;
  for (const Candidate& c : performances_)
    if (c.ms >= 0) r.performances.emplace_back(c.name, c.ms);
  char name[128] = {0};
  lnt_plan_name(t_, name, sizeof name);
  r.pool = name;
  r.interrupted = interrupted_ || current_iteration_ < o_.iterations;
  r.current_iteration = current_iteration_;
  const double done = (double)current_iteration_ - (double)o_.from_iteration + 1;
  r.per_iteration_ms = done > 0 ? total_ms / done : 0;
  r.was_interrupted = o_.was_interrupted;
  r.total_seconds = total_ms / 1000.0;
  r.has_res64 = true;
  r.res64 = res64_of(host_x_, widths_);
  if (gerbicz_ && lnt_gerbicz_stats(t_, nullptr, &r.gerbicz_checks, &r.gerbicz_errors) == LNT_OK)
    r.has_gerbicz = true;
  if (jacobi_ && lnt_jacobi_stats(t_, nullptr, &r.jacobi_checks, &r.jacobi_errors) == LNT_OK)
    r.has_jacobi = true;
  if (!WriteStatsFile(o_.stat_filename, r))
    LOG_NORMAL("Cannot write the statistics to %s", o_.stat_filename.c_str());
}

}  // namespace lucasntt

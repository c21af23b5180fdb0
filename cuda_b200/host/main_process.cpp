#include "main_process.h"

#include <cctype>
#include <csignal>
#include <iostream>
#include <stdexcept>

#include "logger.h"

namespace lucasntt {

namespace {

void on_sigint(int) {
  g_interrupted = 1;  // the loop reports "Process interrupted!" when it stops
}

// The reference's pool names (LucasNTT.ini) mapped onto this library's plan
// kinds: FFT_1SMEM is the resident plan, the FFT_2SMEM family the two-pass
// plans.  Other pools have no counterpart; then every plan stays a candidate.
int kind_for_pool(const std::string& pool) {
  if (pool == "FFT_1SMEM") return LNT_PLAN_RESIDENT;
  if (pool.rfind("FFT_2SMEM", 0) == 0) return LNT_PLAN_RADIX16;
  return LNT_PLAN_AUTO;
}

}  // namespace

bool Confirm(const std::string& question) {
  std::string answer;
  while (true) {
    std::cout << question << " (Y/N) : " << std::flush;
    if (!std::getline(std::cin, answer)) return false;
    if (!answer.empty()) {
      const char c = (char)std::toupper((unsigned char)answer[0]);
      if (c == 'Y') return true;
      if (c == 'N') return false;
    }
    std::cout << "Please enter Y or N.\n";
  }
}

MainProcess::MainProcess(int argc, char** argv) {
  Name = "MainProcess";
  o_ = ResolveOptions(argc, argv);
  Logger::Get().SetVerbosity(o_.verbosity);
  LOG_NORMAL("Welcome to LucasNTT, a pure-integer Lucas-Lehmer and PRP primality test for Mersenne numbers running on GPU.");
  LOG_NORMAL("------------------------------------------------------------------------------------------------------------");
  LOG_NORMAL("%s", "");
  LOG_VERBOSE("Filename for final results: %s", o_.stat_filename.c_str());
  if (o_.was_interrupted)
    LOG_NORMAL("Last execution was interrupted, trying to restore last execution status...");
  LOG_NORMAL("Exponent = %u", o_.exponent);

  if (o_.provided_length.empty()) {
    n_ = 1u << lnt_secured_log2_length(o_.exponent);
  } else {
    int st = lnt_parse_length(o_.provided_length.c_str(), &n_);
    if (st != LNT_OK)
      throw std::runtime_error("Invalid FFT length " + o_.provided_length + ": " + lnt_status_string(st));
    int diff = 0;
    lnt_check_provided_length(o_.exponent, o_.provided_length.c_str(), &diff);
    uint32_t best = 0;
    if (n_ % 5 == 0 && lnt_smallest_length(o_.exponent, &best) == LNT_OK)
      diff = n_ < best ? 1 : (n_ > best ? -1 : 0);  // 5 * 2^k: this library's bound, not log2 alone
    if (diff != 0 &&
        !Confirm(diff > 0 ? "\n\nThe provided length is too small. Due to the risk of overflow, the result will not be reliable.\nDo you still want to process?"
                          : "\n\nThe provided length is not optimal. The process can be accelerated.\nDo you still want to process?"))
      throw std::runtime_error("Process cancelled by user. Invalid FFT length.");
  }

  // candidate plans of this length (the reference's candidate lengths x pools)
  std::vector<lnt_plan_options> plans(128);
  int count = 0;
  const int st = lnt_plan_candidates(o_.exponent, n_, plans.data(), (int)plans.size(), &count);
  if (st != LNT_OK)
    throw std::runtime_error(std::string("No plan for this length: ") + lnt_last_error());
  plans.resize((size_t)std::min(count, 128));
  std::vector<lnt_plan_options> chosen;
  const std::string& pool = o_.preferred_pool;
  if (!pool.empty()) {
    const int kind = kind_for_pool(pool);
    for (const lnt_plan_options& p : plans) {
      char name[128];
      lnt_plan_describe(&p, o_.exponent, n_, name, sizeof name);
      const bool same_family = kind != LNT_PLAN_AUTO &&
                               (p.kind == (uint32_t)kind || (kind == LNT_PLAN_RADIX16 && p.kind == LNT_PLAN_RADIX2));
      if (pool == name || same_family) chosen.push_back(p);
    }
    if (chosen.empty())
      LOG_NORMAL("Pool %s has no counterpart for this length; every plan is a candidate.", pool.c_str());
  }
  if (chosen.empty()) chosen = plans;
  if (o_.preferred_kernels != ";;")
    LOG_VERBOSE("Kernels preference %s ignored: kernels are chosen with the plan.", o_.preferred_kernels.c_str());
  for (const lnt_plan_options& p : chosen) {
    char name[128];
    lnt_plan_describe(&p, o_.exponent, n_, name, sizeof name);
    candidates_.push_back({p, std::string("LucasPRP ") + name, -1});
  }
  LOG_NORMAL("%s", "");
}

void MainProcess::Run() {
  LOG_VERBOSE("Here are the candidates to run this test:");
  for (size_t i = 0; i < candidates_.size(); ++i)
    LOG_VERBOSE("    [Candidate %zu] %s", i + 1, candidates_[i].name.c_str());

  // Process::GetBestPerformers (process.cu:45-127): time every candidate
  std::vector<lnt_plan_options> plans;
  for (const Candidate& c : candidates_) plans.push_back(c.plan);
  std::vector<float> ms(plans.size(), -1.0f);
  const int loops = o_.performance_loops > 0 ? (int)o_.performance_loops : 500;
  const int st = lnt_time_plans(o_.exponent, n_, o_.prp ? 1 : 0, o_.gpu, (uint32_t)loops, plans.data(),
                                (int)plans.size(), ms.data());
  if (st == LNT_ERR_NO_DEVICE || st == LNT_ERR_CUDA)
    throw std::runtime_error(std::string("cudaSetDevice failed!  Do you have a CUDA-capable GPU installed? (") +
                             lnt_last_error() + ")");
  int best = -1;
  for (size_t i = 0; i < candidates_.size(); ++i) {
    candidates_[i].ms = ms[i];
    if (ms[i] >= 0 && (best < 0 || ms[i] < ms[(size_t)best])) best = (int)i;
  }
  LOG_NORMAL("\nSummary of the performances of the different processes on %d loops:", loops);
  size_t width = 0;
  for (const Candidate& c : candidates_) width = std::max(width, c.name.size());
  for (const Candidate& c : candidates_)
    if (c.ms >= 0) LOG_NORMAL("%-*s = %8.3fms", (int)width, c.name.c_str(), c.ms);
  if (best < 0) {
    LOG_VERBOSE("%s: cannot find a suitable candidate to run with this configuration.", Name.c_str());
    return;
  }

  LucasPRP test(o_, candidates_[(size_t)best].plan, n_, candidates_);
  test.Performance = candidates_[(size_t)best].ms;
  LOG_NORMAL("\nThis test will run using the following processes:");
  LOG_NORMAL("%s", Name.c_str());
  LOG_NORMAL("    %s", test.Name.c_str());
  LOG_NORMAL("\n\n----------------------------------------------");
  LOG_NORMAL("Now testing M(q) = 2^q - 1 where q = %u", o_.exponent);
  LOG_NORMAL(o_.prp ? "With PRP pseudo-primality test" : "With Lucas-Lehmer primality test");
  LOG_NORMAL("From iteration %u to %u\n", o_.from_iteration, o_.iterations);
  if (!test.Initialize()) throw std::runtime_error("Cannot initialize the test on the GPU");
  std::signal(SIGINT, on_sigint);
  test.Run();
  std::signal(SIGINT, SIG_DFL);
  if (g_interrupted) LOG_NORMAL("\nProcess interrupted!");
  LOG_VERBOSE("\nFinalization...");
  test.Finalize();
  LOG_VERBOSE("End.");
}

}  // namespace lucasntt

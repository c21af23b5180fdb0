// Console output with the reference's three verbosity levels
// (common/common.cuh:32-60, common/common.cu:19-81): a message is printed when
// the configured level is at or below the message's level.
#pragma once
#include <cstdarg>
#include <cstdio>

namespace lucasntt {

enum class Verbosity { Verbose = 0, Normal = 1, Silent = 2 };

class Logger {
 public:
  static Logger& Get() {
    static Logger instance;
    return instance;
  }
  void SetVerbosity(Verbosity v) { level_ = v; }
  Verbosity GetVerbosity() const { return level_; }

  void WriteLine(Verbosity at, const char* fmt, ...) __attribute__((format(printf, 3, 4))) {
    if ((int)level_ > (int)at) return;
    va_list ap;
    va_start(ap, fmt);
    std::vprintf(fmt, ap);
    va_end(ap);
    std::printf("\n");
    std::fflush(stdout);
  }

 private:
  Verbosity level_ = Verbosity::Normal;
};

#define LOG_NORMAL(...) ::lucasntt::Logger::Get().WriteLine(::lucasntt::Verbosity::Normal, __VA_ARGS__)
#define LOG_VERBOSE(...) ::lucasntt::Logger::Get().WriteLine(::lucasntt::Verbosity::Verbose, __VA_ARGS__)

}  // namespace lucasntt

// The reference's Process seam (process.cuh:16-35): a named step that can be
// initialised, run, finalised and timed.  MainProcess and LucasPRP implement
// it here as in the reference; the squaring itself is the library's
// (include/lucasntt.h), so there is no KernelPool level below LucasPRP.
#pragma once
#include <string>

namespace lucasntt {

class Process {
 public:
  virtual ~Process() = default;
  virtual bool Initialize() { return true; }
  virtual void Run() = 0;
  virtual void Finalize() {}
  std::string Name;
  float Performance = 0;  // ms for PerformanceLoops iterations (Process::EvaluatePerformance)
};

}  // namespace lucasntt

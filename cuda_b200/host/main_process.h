// MainProcess (main_process.cu:57-190): options, candidate plans, autotune
// over them, then one LucasPRP test.
#pragma once
#include <vector>

#include "lucas_prp.h"
#include "options.h"
#include "process.h"

namespace lucasntt {

class MainProcess : public Process {
 public:
  MainProcess(int argc, char** argv);
  void Run() override;
  const MainOptions& options() const { return o_; }

 private:
  MainOptions o_;
  uint32_t n_ = 0;
  std::vector<Candidate> candidates_;
};

// Confirm (main_process.cu:49-62): Y/N on standard input; end of input = N.
bool Confirm(const std::string& question);

}  // namespace lucasntt

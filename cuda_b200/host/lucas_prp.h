// One Lucas-Lehmer or PRP test driven through the C ABI: the host side of the
// reference's LucasPRP (lucas_prp.cu:24-352) with the same console messages,
// pit stops, safety dumps, resume and result files.
#pragma once
#include <csignal>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/lucasntt.h"
#include "options.h"
#include "process.h"

namespace lucasntt {

// Set by the SIGINT handler (main_process.cu:35-47); the loop stops at the
// next chunk boundary and the residue is dumped for a later resume.
extern volatile std::sig_atomic_t g_interrupted;

struct Candidate {
  lnt_plan_options plan;
  std::string name;  // "LucasPRP <plan>"
  float ms = -1;     // ms for PerformanceLoops squarings, -1 = failed
};

class LucasPRP : public Process {
 public:
  LucasPRP(MainOptions& options, const lnt_plan_options& plan, uint32_t n,
           std::vector<Candidate> performances);
  ~LucasPRP() override;
  bool Initialize() override;  // allocate the test on the GPU (LucasPRP::Initialize)
  void Run() override;         // LucasPRP::Run: resume or start, main loop, verdict, files
  void Finalize() override;

  bool is_prime() const { return is_prime_; }
  bool is_composite() const { return is_composite_; }

 private:
  void InitializeTest();
  void MainLoop();
  void DisplayPitStop(double elapsed_ms);
  void DumpResidue();
  bool LoadResidue();
  void DumpStats(double total_ms);
  void DumpEnvironment();
  void Check(int status, const char* what);
  void EnableChecks();

  MainOptions& o_;
  lnt_plan_options plan_;
  uint32_t n_;
  std::vector<Candidate> performances_;
  lnt_test* t_ = nullptr;
  std::vector<uint8_t> widths_;
  std::vector<uint64_t> host_x_;
  uint32_t current_iteration_ = 0;
  bool interrupted_ = false;
  bool is_prime_ = false, is_composite_ = false;
  double total_ms_ = 0;
  double ms_per_iteration_estimate_ = 0;
  bool gerbicz_ = false;
  bool jacobi_ = false;
};

}  // namespace lucasntt

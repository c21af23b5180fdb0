// Run options of the lucasntt program: LucasNTT.ini, the command line and,
// after an interruption, the stats file of the interrupted run.
//
// Same keys, defaults and precedence as MainProcess::MainProcess
// (main_process.cu:64-147): argv = exponent iterations prefix fft; when the
// stats file says Interrupted = 1 it replaces LucasNTT.ini and its
// currentIteration becomes the first iteration to run.
#pragma once
#include <cstdint>
#include <string>

#include "logger.h"

namespace lucasntt {

struct MainOptions {
  Verbosity verbosity = Verbosity::Normal;
  int gpu = 0;
  long performance_loops = 500;
  std::string dump_filename = "LucasNTT_results.dat";
  std::string stat_filename = "LucasNTT_results.txt";
  std::string env_filename = "LucasNTT_results.env";
  bool dump_residue = false;
  bool dump_stats = true;
  bool dump_environment = false;
  bool was_interrupted = false;  // the stats file said Interrupted = 1
  bool prp = false;
  uint32_t exponent = 9689;
  uint32_t iterations = 9687;     // last iteration to run (1-based)
  uint32_t from_iteration = 1;    // first iteration to run
  std::string preferred_pool;     // "" = autotune
  std::string preferred_kernels;  // ";a;b;" as the reference stores it
  std::string provided_length;    // "" = the length policy's candidates
  // Extension: seconds between safety dumps of residue + stats (the
  // reference's fixed hour, lucas_prp.cu:201-215).  Key SafetyDumpSeconds.
  double safety_dump_seconds = 3600.0;
  // Extension: GerbiczBlock = B turns on the Gerbicz-Li check of PRP tests
  // (lnt_gerbicz_enable; a verification every B^2 squarings).  0 = off.
  uint32_t gerbicz_block = 0;
  // Extension: JacobiCheck = K turns on the Jacobi check of LL tests
  // (lnt_jacobi_enable; the symbol of the residue every K squarings).  0 = off.
  uint64_t jacobi_interval = 0;
};

// Resolve the options.  `ini_path` is LucasNTT.ini in the working directory
// for the program; tests pass their own.  Throws std::runtime_error on a
// malformed number on the command line (as std::stoi does in the reference).
MainOptions ResolveOptions(int argc, char** argv, const std::string& ini_path = "LucasNTT.ini");

// Largest iteration of a full test: q - 2 for LL, q for PRP (lucas_prp.cu:167).
inline uint32_t MaxIterations(const MainOptions& o) { return o.prp ? o.exponent : o.exponent - 2; }

}  // namespace lucasntt

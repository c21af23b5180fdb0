#include "options.h"

#include <stdexcept>

#include "ini_file.h"

namespace lucasntt {

namespace {

// std::stoi on an argv word, as main_process.cu:116 and :120 do
long parse_int(const char* word, const char* what) {
  try {
    size_t used = 0;
    const long v = std::stol(word, &used, 10);
    return v;
  } catch (const std::exception&) {
    throw std::runtime_error(std::string("invalid ") + what + " on the command line: " + word);
  }
}

}  // namespace

MainOptions ResolveOptions(int argc, char** argv, const std::string& ini_path) {
  MainOptions o;
  IniFile file;
  const IniFile* ini = file.Load(ini_path) ? &file : nullptr;

  const std::string verbosity = ini ? ini->GetValue("Verbosity", "Normal") : "Normal";
  if (verbosity == "Verbose") o.verbosity = Verbosity::Verbose;
  if (verbosity == "Silent") o.verbosity = Verbosity::Silent;
  o.gpu = ini ? (int)ini->GetLongValue("GPU", 0) : 0;
  o.performance_loops = ini ? ini->GetLongValue("PerformanceLoops", 500) : 500;

  if (argc > 3) {
    const std::string prefix = argv[3];
    o.dump_filename = prefix + ".dat";
    o.stat_filename = prefix + ".txt";
    o.env_filename = prefix + ".env";
  } else if (ini) {
    o.dump_filename = ini->GetValue("Dump", "LucasNTT_results.dat");
    o.stat_filename = ini->GetValue("Stats", "LucasNTT_results.txt");
    o.env_filename = ini->GetValue("Env", "LucasNTT_results.env");
  }
  o.dump_residue = ini ? ini->GetLongValue("dumpResidue", 0) == 1 : false;
  o.dump_stats = ini ? ini->GetLongValue("dumpStats", 1) == 1 : true;
  o.dump_environment = ini ? ini->GetLongValue("dumpEnvironment", 0) == 1 : false;
  o.safety_dump_seconds = ini ? (double)ini->GetLongValue("SafetyDumpSeconds", 3600) : 3600.0;
  if (o.safety_dump_seconds <= 0) o.safety_dump_seconds = 3600.0;
  {
    const long b = ini ? ini->GetLongValue("GerbiczBlock", 0) : 0;
    o.gerbicz_block = b > 0 && b < (1L << 20) ? (uint32_t)b : 0;
    const long j = ini ? ini->GetLongValue("JacobiCheck", 0) : 0;
    o.jacobi_interval = j > 0 ? (uint64_t)j : 0;
  }

  // an interrupted run's stats file replaces LucasNTT.ini (main_process.cu:98-106)
  IniFile last;
  o.was_interrupted = last.Load(o.stat_filename) && last.GetLongValue("Interrupted", 0) == 1;
  if (o.was_interrupted) ini = &last;

  o.prp = ini ? ini->GetLongValue("PRP", 0) == 1 : false;
  long q = argc > 1 ? parse_int(argv[1], "exponent") : (ini ? ini->GetLongValue("Exponent", 9689) : 9689);
  if (q < 3 || q > 0x7FFFFFFFL) throw std::runtime_error("exponent out of range: " + std::to_string(q));
  o.exponent = (uint32_t)q;

  const long max_it = (long)MaxIterations(o);
  long it = argc > 2 ? parse_int(argv[2], "iterations")
                     : (ini ? ini->GetLongValue("Iterations", max_it) : max_it);
  if (it > max_it || it <= 0) it = max_it;  // main_process.cu:121-122
  o.iterations = (uint32_t)it;
  long from = o.was_interrupted && ini ? ini->GetLongValue("currentIteration", 1) : 1;
  if (from < 1) from = 1;
  o.from_iteration = (uint32_t)from;

  o.preferred_pool = ini ? ini->GetValue("Pool", "") : "";
  o.preferred_kernels = ";" + (ini ? ini->GetValue("Kernels", "") : std::string()) + ";";
  o.provided_length = argc > 4 ? std::string(argv[4]) : (ini ? ini->GetValue("fft", "") : "");
  return o;
}

}  // namespace lucasntt

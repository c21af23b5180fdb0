// Host-only checks of the lucasntt program's option resolution and result
// files (no GPU).  Built by tests/test_cli.py together with the program's
// sources; argv[1] is an empty scratch directory to work in.
#include <unistd.h>

#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../cuda_b200/host/ini_file.h"
#include "../../cuda_b200/host/options.h"
#include "../../cuda_b200/host/residue_files.h"

using namespace lucasntt;

static int failures = 0;
#define CHECK(cond)                                                     \
  do {                                                                  \
    if (!(cond)) {                                                      \
      std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #cond);       \
      ++failures;                                                       \
    }                                                                   \
  } while (0)

static void write_file(const std::string& path, const std::string& text) {
  std::ofstream(path) << text;
}

static std::string read_file(const std::string& path) {
  std::ifstream in(path);
  std::stringstream ss;
  ss << in.rdbuf();
  return ss.str();
}

static MainOptions resolve(std::vector<std::string> args, const std::string& ini = "LucasNTT.ini") {
  std::vector<char*> argv;
  args.insert(args.begin(), "lucasntt");
  for (auto& a : args) argv.push_back(&a[0]);
  return ResolveOptions((int)argv.size(), argv.data(), ini);
}

static void test_defaults() {
  std::remove("LucasNTT.ini");
  std::remove("LucasNTT_results.txt");
  MainOptions o = resolve({});
  CHECK(o.exponent == 9689 && o.iterations == 9687 && o.from_iteration == 1 && !o.prp);
  CHECK(o.dump_filename == "LucasNTT_results.dat" && o.stat_filename == "LucasNTT_results.txt" &&
        o.env_filename == "LucasNTT_results.env");
  CHECK(o.dump_stats && !o.dump_residue && !o.dump_environment && !o.was_interrupted);
  CHECK(o.performance_loops == 500 && o.gpu == 0 && o.verbosity == Verbosity::Normal);
  CHECK(o.gerbicz_block == 0 && o.jacobi_interval == 0);
  CHECK(o.provided_length.empty() && o.preferred_pool.empty() && o.preferred_kernels == ";;");
}

static void test_ini_and_argv() {
  write_file("LucasNTT.ini",
             "## comment\n# Exponent = 1\n ; other comment\n"
             "exponent = 44497\nPRP = 1\nIterations=1000\nperformanceloops = 77\n"
             "Verbosity = Silent\nGPU = 0\ndumpResidue = 1\ndumpStats = 0\ndumpEnvironment = 1\n"
             "Dump = r.dat\nStats = r.txt\nEnv = r.env\nfft = 4096\nPool = FFT_1SMEM\nKernels = a;b\n"
             "GerbiczBlock = 64\nJacobiCheck = 250000\n"
             "[Section]\nExponent = 3\n");
  MainOptions o = resolve({});
  CHECK(o.exponent == 44497 && o.prp && o.iterations == 1000 && o.performance_loops == 77);
  CHECK(o.verbosity == Verbosity::Silent && o.dump_residue && !o.dump_stats && o.dump_environment);
  CHECK(o.dump_filename == "r.dat" && o.stat_filename == "r.txt" && o.env_filename == "r.env");
  CHECK(o.provided_length == "4096" && o.preferred_pool == "FFT_1SMEM" && o.preferred_kernels == ";a;b;");
  CHECK(o.gerbicz_block == 64 && o.jacobi_interval == 250000);
  // command line: exponent iterations prefix fft
  o = resolve({"9941", "50", "run1", "1024"});
  CHECK(o.exponent == 9941 && o.iterations == 50 && o.provided_length == "1024");
  CHECK(o.dump_filename == "run1.dat" && o.stat_filename == "run1.txt" && o.env_filename == "run1.env");
  // iterations beyond the full test or <= 0 become the full test (PRP: q)
  CHECK(resolve({"9941", "99999"}).iterations == 9941);
  CHECK(resolve({"9941", "0"}).iterations == 9941);
  CHECK(resolve({"9941", "-5"}).iterations == 9941);
  bool threw = false;
  try {
    resolve({"abc"});
  } catch (const std::exception&) {
    threw = true;
  }
  CHECK(threw);
  std::remove("LucasNTT.ini");
  CHECK(resolve({"9941"}).iterations == 9939);  // LL: q - 2
}

static void test_resume_from_stats() {
  std::remove("LucasNTT.ini");
  write_file("LucasNTT_results.txt",
             "Exponent = 86243\nConclusion = Partial\nPRP = 1\nIterations = 5000\nfft = 4096\n"
             "n = 4096\nPool = RESIDENT_4096\nInterrupted = 1\ncurrentIteration = 1234\n"
             "Per iteration (ms) = 0.01\nWarning! total time is not relevant\nTotal time (sec) = 3\n");
  MainOptions o = resolve({});
  CHECK(o.was_interrupted && o.prp && o.exponent == 86243 && o.iterations == 5000);
  CHECK(o.from_iteration == 1234 && o.provided_length == "4096" && o.preferred_pool == "RESIDENT_4096");
  // a finished run is not resumed
  write_file("LucasNTT_results.txt", "Exponent = 86243\nInterrupted = 0\ncurrentIteration = 1234\n");
  o = resolve({});
  CHECK(!o.was_interrupted && o.from_iteration == 1 && o.exponent == 9689);
  // the prefix on the command line names the stats file that is checked
  write_file("p.txt", "Exponent = 110503\nInterrupted = 1\ncurrentIteration = 7\nIterations = 100\n");
  o = resolve({"110503", "100", "p"});
  CHECK(o.was_interrupted && o.from_iteration == 7 && o.iterations == 100);
  std::remove("LucasNTT_results.txt");
  std::remove("p.txt");
}

static void test_residue_files() {
  const std::vector<uint8_t> widths = {5, 4, 5, 4};
  const std::vector<uint64_t> d = {31, 0, 17, 15};
  CHECK(WriteResidueFile("x.dat", d));
  CHECK(read_file("x.dat") ==
        "0x000000000000001F\n0x0000000000000000\n0x0000000000000011\n0x000000000000000F\n");
  std::vector<uint64_t> back;
  std::string why;
  CHECK(ReadResidueFile("x.dat", widths, back, &why) && back == d);
  // truncated, malformed, too long, a digit over its width, missing file
  write_file("t.dat", "0x000000000000001F\n0x0000000000000000\n0x00000000000");
  CHECK(!ReadResidueFile("t.dat", widths, back, &why) && !why.empty());
  write_file("t.dat", "0x000000000000001F\n0x00000000000000G0\n0x0000000000000011\n0x000000000000000F\n");
  CHECK(!ReadResidueFile("t.dat", widths, back, &why));
  write_file("t.dat", read_file("x.dat") + "0x0000000000000001\n");
  CHECK(!ReadResidueFile("t.dat", widths, back, &why));
  write_file("t.dat", "0x0000000000000020\n0x0000000000000000\n0x0000000000000011\n0x000000000000000F\n");
  CHECK(!ReadResidueFile("t.dat", widths, back, &why));
  write_file("t.dat", "0x000000000000001F\n0x0000000000000000\n");
  CHECK(!ReadResidueFile("t.dat", widths, back, &why));
  CHECK(!ReadResidueFile("missing.dat", widths, back, &why));
  std::remove("x.dat");
  std::remove("t.dat");
}

static void test_stats_file() {
  StatsRecord r;
  r.exponent = 44497;
  r.prp = false;
  r.is_prime = true;
  r.iterations = 44495;
  r.fft = "2048";
  r.n = 2048;
  r.log2_n = 11;
  r.performance_loops = 500;
  r.performances = {{"LucasPRP RESIDENT_2048", 9.5f}};
  r.pool = "RESIDENT_2048";
  r.kernels = {"resident_square_loop"};
  r.current_iteration = 44496;
  r.per_iteration_ms = 0.0125;
  r.total_seconds = 0.5;
  r.has_res64 = true;
  r.res64 = 0;
  CHECK(WriteStatsFile("s.txt", r));
  const std::string s = read_file("s.txt");
  CHECK(s.rfind("Exponent = 44497\nConclusion = Prime\nPRP = 0\nIterations = 44495\nfft = 2048\n"
                "n = 2048\nlog2_n = 11\nlog3_n = 0\nlog5_n = 0\n"
                "Candidate Performance (in ms for 500 loops): LucasPRP RESIDENT_2048 = 9.5\n"
                "Pool = RESIDENT_2048\nKernel0 = resident_square_loop\nInterrupted = 0\n"
                "currentIteration = 44496\nPer iteration (ms) = 0.0125\nTotal time (sec) = 0.5\n"
                "Res64 = 0000000000000000\n", 0) == 0);
  IniFile ini;
  CHECK(ini.Load("s.txt") && ini.GetLongValue("Interrupted", 7) == 0 &&
        ini.GetLongValue("currentIteration", 0) == 44496 && ini.GetValue("Pool", "") == "RESIDENT_2048");
  r.is_prime = false;
  r.prp = true;
  r.interrupted = true;
  r.was_interrupted = true;
  CHECK(WriteStatsFile("s.txt", r));
  const std::string s2 = read_file("s.txt");
  CHECK(s2.find("Conclusion = Partial\n") != std::string::npos);
  CHECK(s2.find("Interrupted = 1\n") != std::string::npos);
  CHECK(s2.find("Warning! total time is not relevant") != std::string::npos);
  std::remove("s.txt");
}

int main(int argc, char** argv) {
  if (argc < 2 || chdir(argv[1]) != 0) {
    std::printf("usage: cli_selftest <scratch dir>\n");
    return 2;
  }
  test_defaults();
  test_ini_and_argv();
  test_resume_from_stats();
  test_residue_files();
  test_stats_file();
  if (failures) {
    std::printf("%d failures\n", failures);
    return 1;
  }
  std::printf("cli selftest ok\n");
  return 0;
}

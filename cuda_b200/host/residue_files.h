// The reference's result files, byte for byte (lucas_prp.cu:254-346):
//   .dat  residue dump: one "0x%016llX\n" record (19 bytes) per word, natural order
//   .txt  stats: key = value lines read back on resume (Interrupted, currentIteration)
//   .env  CUDA version and device properties
#pragma once
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace lucasntt {

// DumpResidue (lucas_prp.cu:254-263).  False if the file cannot be written.
bool WriteResidueFile(const std::string& path, const std::vector<uint64_t>& digits);

// LoadResidue (lucas_prp.cu:326-346) with validation the reference lacks: the
// file must hold exactly widths.size() well-formed records and every digit must
// fit its width; otherwise false with the reason in *why (the caller restarts
// from iteration 1, as the reference does for a missing file).
bool ReadResidueFile(const std::string& path, const std::vector<uint8_t>& widths,
                     std::vector<uint64_t>& digits, std::string* why);

struct StatsRecord {
  uint32_t exponent = 0;
  bool prp = false;
  bool is_prime = false, is_composite = false;
  uint32_t iterations = 0;
  std::string fft;  // the lengths of the plan ("2048:4096")
  uint32_t n = 0, log2_n = 0, log3_n = 0, log5_n = 0;
  long performance_loops = 500;
  std::vector<std::pair<std::string, float>> performances;  // candidate -> ms for the loops
  std::string pool;
  std::vector<std::string> kernels;
  bool interrupted = false;
  uint32_t current_iteration = 0;
  double per_iteration_ms = 0;
  bool was_interrupted = false;
  double total_seconds = 0;
  bool has_res64 = false;
  uint64_t res64 = 0;
  bool has_gerbicz = false;
  uint64_t gerbicz_checks = 0, gerbicz_errors = 0;
  bool has_jacobi = false;
  uint64_t jacobi_checks = 0, jacobi_errors = 0;
};

// DumpStats (lucas_prp.cu:293-324): same keys, same order, same %g formats;
// adds a Res64 line (the reference prints none).
bool WriteStatsFile(const std::string& path, const StatsRecord& r);

bool WriteTextFile(const std::string& path, const std::string& text);

}  // namespace lucasntt

// Minimal reader for LucasNTT.ini and the stats file (key = value lines).
//
// The reference reads both with SimpleIni (main_process.cu:72-126): keys in
// the unnamed section, matched without regard to case, '#' and ';' comment
// lines, values trimmed.  Only that subset is needed here, so this is a small
// parser of its own rather than the third-party library.
#pragma once
#include <map>
#include <string>

namespace lucasntt {

class IniFile {
 public:
  // false when the file cannot be opened (the reference then runs on defaults)
  bool Load(const std::string& path);
  bool Has(const std::string& key) const;
  std::string GetValue(const std::string& key, const std::string& def) const;
  // SimpleIni's GetLongValue: decimal or 0x-prefixed hex; def when absent or
  // not a number
  long GetLongValue(const std::string& key, long def) const;

 private:
  std::map<std::string, std::string> values_;  // lower-cased key -> value
};

}  // namespace lucasntt

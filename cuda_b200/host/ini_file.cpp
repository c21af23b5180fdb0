#include "ini_file.h"

#include <cctype>
#include <cerrno>
#include <cstdlib>
#include <fstream>

namespace lucasntt {

namespace {

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

std::string lower(std::string s) {
  for (char& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

}  // namespace

bool IniFile::Load(const std::string& path) {
  std::ifstream in(path);
  if (!in) return false;
  values_.clear();
  std::string line;
  bool in_unnamed = true;
  bool first = true;
  while (std::getline(in, line)) {
    if (first && line.size() >= 3 && (unsigned char)line[0] == 0xEF &&
        (unsigned char)line[1] == 0xBB && (unsigned char)line[2] == 0xBF)
      line = line.substr(3);  // UTF-8 byte order mark
    first = false;
    const std::string t = trim(line);
    if (t.empty() || t[0] == '#' || t[0] == ';') continue;
    if (t[0] == '[') {
      in_unnamed = false;  // named sections are not used by LucasNTT
      continue;
    }
    const size_t eq = t.find('=');
    if (eq == std::string::npos || !in_unnamed) continue;
    const std::string key = lower(trim(t.substr(0, eq)));
    if (key.empty()) continue;
    values_[key] = trim(t.substr(eq + 1));  // a repeated key replaces the earlier value
  }
  return true;
}

bool IniFile::Has(const std::string& key) const { return values_.count(lower(key)) != 0; }

std::string IniFile::GetValue(const std::string& key, const std::string& def) const {
  auto it = values_.find(lower(key));
  return it == values_.end() ? def : it->second;
}

long IniFile::GetLongValue(const std::string& key, long def) const {
  auto it = values_.find(lower(key));
  if (it == values_.end() || it->second.empty()) return def;
  const std::string& v = it->second;
  const char* s = v.c_str();
  char* end = nullptr;
  errno = 0;
  long r;
  if (v.size() > 2 && v[0] == '0' && (v[1] == 'x' || v[1] == 'X'))
    r = std::strtol(s + 2, &end, 16);
  else
    r = std::strtol(s, &end, 10);
  if (end == s || *end != '\0' || errno) return def;
  return r;
}

}  // namespace lucasntt

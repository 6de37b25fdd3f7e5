// The autotuners' persistent table (host code, header-only so that the CPU
// tests can compile it alone).
//
// One line per (device, tuner, problem class):
//
//   ccfj-tune-v1 <device> <kind> <class key> <choice> <ms>
//
// <device> is the CUDA device name with blanks replaced by '_', <kind> the
// tuner ("fj": single-set transform, "batch": ragged batch), <class key> the
// tuner's integer class of the problem, <choice> the winning tile choice in
// the tuner's encoding and <ms> its measured time. Unknown or malformed
// lines are kept as they are and otherwise ignored. Writes go to a
// temporary file renamed over the table, so a reader never sees half of one.
#pragma once

#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace ccfj {
namespace tune {

constexpr const char* kMagic = "ccfj-tune-v1";

struct Entry {
  std::string device;
  std::string kind;
  long long key = 0;
  int choice = 0;
  float ms = 0.f;
};

inline bool parse_line(const std::string& line, Entry* e) {
  std::istringstream in(line);
  std::string magic, extra;
  Entry t;
  if (!(in >> magic >> t.device >> t.kind >> t.key >> t.choice >> t.ms)) return false;
  if (magic != kMagic || (in >> extra)) return false;
  *e = t;
  return true;
}

inline std::string format_line(const Entry& e) {
  char ms[32];
  std::snprintf(ms, sizeof(ms), "%.6g", (double)e.ms);
  std::ostringstream out;
  out << kMagic << ' ' << e.device << ' ' << e.kind << ' ' << e.key << ' ' << e.choice << ' ' << ms;
  return out.str();
}

inline std::string device_token(const std::string& name) {
  std::string t = name.empty() ? std::string("unknown") : name;
  for (char& ch : t)
    if (ch == ' ' || ch == '\t' || ch == '\n') ch = '_';
  return t;
}

inline std::vector<std::string> read_lines(const std::string& path) {
  std::vector<std::string> lines;
  std::ifstream in(path);
  std::string line;
  while (std::getline(in, line)) lines.push_back(line);
  return lines;
}

// Every well-formed entry of the table (a missing file has none).
inline std::vector<Entry> read_file(const std::string& path) {
  std::vector<Entry> out;
  for (const std::string& line : read_lines(path)) {
    Entry e;
    if (parse_line(line, &e)) out.push_back(e);
  }
  return out;
}

// Replaces the line of (device, kind, key) with e, or appends it.
inline bool upsert_file(const std::string& path, const Entry& e) {
  std::vector<std::string> lines = read_lines(path);
  bool replaced = false;
  for (std::string& line : lines) {
    Entry old;
    if (parse_line(line, &old) && old.device == e.device && old.kind == e.kind && old.key == e.key) {
      line = format_line(e);
      replaced = true;
    }
  }
  if (!replaced) lines.push_back(format_line(e));
  const std::string tmp = path + ".tmp";
  {
    std::ofstream out(tmp, std::ios::trunc);
    if (!out) return false;
    for (const std::string& line : lines) out << line << '\n';
    if (!out) return false;
  }
  return std::rename(tmp.c_str(), path.c_str()) == 0;
}

}  // namespace tune
}  // namespace ccfj

// CPU harness for the autotuners' persistent table (csrc/tune_cache.h):
// exported so that tests/test_tune_cache.py can drive it through ctypes.
#include <cstring>
#include <string>

#include "tune_cache.h"

extern "C" int tc_upsert(const char* path, const char* device, const char* kind, long long key,
                         int choice, float ms) {
  ccfj::tune::Entry e;
  e.device = ccfj::tune::device_token(device);
  e.kind = kind;
  e.key = key;
  e.choice = choice;
  e.ms = ms;
  return ccfj::tune::upsert_file(path, e) ? 0 : 1;
}

// The choice recorded for (device, kind, key), or -1.
extern "C" int tc_lookup(const char* path, const char* device, const char* kind, long long key) {
  const std::string dev = ccfj::tune::device_token(device);
  for (const ccfj::tune::Entry& e : ccfj::tune::read_file(path))
    if (e.device == dev && e.kind == kind && e.key == key) return e.choice;
  return -1;
}

extern "C" int tc_count(const char* path) { return (int)ccfj::tune::read_file(path).size(); }

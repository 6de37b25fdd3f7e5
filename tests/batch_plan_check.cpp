// CPU harness for the planner of large host batches (csrc/batch_plan.h):
// exported so that tests/test_batch_plan.py can drive it through ctypes.
#include "batch_plan.h"

// Writes (b0, b1, row_lo, row_hi) per group into out (4 values per group,
// at most max_groups groups) and returns the group count (0: one pass).
extern "C" int bp_plan(const long long* off, int nsets, const long long* perm, long long total,
                       int nin, unsigned long long ubytes, long long* out, int max_groups) {
  const std::vector<ccfj::SetGroup> g =
      ccfj::plan_set_groups(off, nsets, perm, total, nin, (size_t)ubytes);
  for (int i = 0; i < (int)g.size() && i < max_groups; ++i) {
    out[4 * i] = g[i].b0;
    out[4 * i + 1] = g[i].b1;
    out[4 * i + 2] = g[i].row_lo;
    out[4 * i + 3] = g[i].row_hi;
  }
  return (int)g.size();
}

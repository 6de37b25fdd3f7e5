// Groups of sets for a large host-memory batch (fj_batch.cu): host code
// only, so that a CPU test can check it (tests/batch_plan_check.cpp).
//
// A large batch from host memory is run in groups of consecutive sets, the
// copy of group g + 1 on a stream of its own while group g computes, so
// that only the first group's copy is exposed. Group g ends at the first set
// boundary at or past kGroupEnd[g] of the pairs (the first group is small:
// its copy is the part that cannot overlap).
#pragma once

#include <algorithm>
#include <climits>
#include <cstddef>
#include <vector>

namespace ccfj {

constexpr double kGroupEnd[] = {1.0 / 16, 0.25, 0.5, 0.75, 1.0};
constexpr size_t kPipelineBytes = (size_t)256 << 20;  // inputs below this: one copy, one pass

struct SetGroup {
  int b0, b1;                // sets [b0, b1)
  long long row_lo, row_hi;  // rows of the input its pairs read, [row_lo, row_hi]
};

// Groups of a host batch of nsets sets (pair offsets off[0..nsets], pair i
// reading input row perm[i], or i without perm) with one input of ubytes
// bytes, or none (one pass) where the input has two parts, is small, holds
// one set, or the groups' rows are not disjoint and increasing (a
// permutation that mixes sets).
inline std::vector<SetGroup> plan_set_groups(const long long* off, int nsets,
                                             const long long* perm, long long total, int nin,
                                             size_t ubytes) {
  std::vector<SetGroup> g;
  if (nin != 1 || nsets < 2 || ubytes < kPipelineBytes) return g;
  int b = 0;
  for (double end : kGroupEnd) {
    const long long target = (long long)(end * (double)total);
    const int b0 = b;
    while (b < nsets && (off[b + 1] <= target || b == b0)) ++b;
    if (end == 1.0) b = nsets;
    if (b <= b0) continue;
    long long lo = LLONG_MAX, hi = -1;
    for (long long i = off[b0]; i < off[b]; ++i) {
      const long long row = perm ? perm[i] : i;
      lo = std::min(lo, row);
      hi = std::max(hi, row);
    }
    if (!g.empty() && lo <= g.back().row_hi) return {};
    g.push_back({b0, b, lo, hi});
    if (b == nsets) break;
  }
  return g.size() > 1 ? g : std::vector<SetGroup>{};
}

}  // namespace ccfj

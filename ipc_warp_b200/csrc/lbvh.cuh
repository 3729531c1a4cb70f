// LBVH node access and stack traversal shared by the DCD and CCD kernels.
#pragma once
#include "common.cuh"

namespace ipcb {

constexpr int kStackDepth = 64;

IPCB_D bool box_overlap(f3 alo, f3 ahi, float4 blo, float4 bhi) {
  return alo.x <= bhi.x && blo.x <= ahi.x && alo.y <= bhi.y && blo.y <= ahi.y && alo.z <= bhi.z && blo.z <= ahi.z;
}

// Visit every leaf whose box overlaps [qlo, qhi]; leaf(prim) is called per hit.
// Each node load brings both child boxes (64 B), so one dependent load per
// level.  Returns false if the stack overflowed (result incomplete).
template <class Leaf>
IPCB_D bool traverse(const float4* __restrict__ nodes, int n, f3 qlo, f3 qhi, Leaf&& leaf) {
  if (n <= 0) return true;
  int stack[kStackDepth];
  int sp = 0;
  int node = 0;
  bool ok = true;
  // A well-formed tree visits each internal node at most once per query; the
  // bound only protects against a corrupted hierarchy.
  const int max_visits = 2 * n + 64;
  for (int visits = 0;; ++visits) {
    if (visits >= max_visits) return false;
    const float4* nd = nodes + 4 * node;
    float4 llo = __ldg(nd), lhi = __ldg(nd + 1), rlo = __ldg(nd + 2), rhi = __ldg(nd + 3);
    int lc = __float_as_int(llo.w), rc = __float_as_int(rlo.w);
    bool hl = box_overlap(qlo, qhi, llo, lhi);
    bool hr = box_overlap(qlo, qhi, rlo, rhi);
    if (hl && lc < 0) leaf(~lc);
    if (hr && rc < 0) leaf(~rc);
    bool tl = hl && lc >= 0, tr = hr && rc >= 0;
    if (tl || tr) {
      node = tl ? lc : rc;
      if (tl && tr) {
        if (sp < kStackDepth) stack[sp++] = rc;
        else ok = false;
      }
    } else {
      if (sp == 0) break;
      node = stack[--sp];
    }
  }
  return ok;
}

}  // namespace ipcb

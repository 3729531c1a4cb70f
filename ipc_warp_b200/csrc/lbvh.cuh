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

// 4-wide view of the hierarchy: wide node b (for every internal binary node b)
// holds the boxes of b's grandchildren -- or of a child directly when that
// child is a leaf -- in SoA order: lo.x[4] lo.y[4] lo.z[4] hi.x[4] hi.y[4]
// hi.z[4] code[4] last[4] (8 float4 = 128 B).  code >= 0: continue at wide
// node `code`; code < 0: leaf ~primitive; empty slots have an empty box.
// last: the largest leaf rank (position in Morton order) below the slot (-1
// when empty); a slot covers the contiguous ranks up to it.  One visit tests
// four boxes, so a query's chain of dependent loads is about half as long as
// in the binary tree.
constexpr int kWideStack = 128;

// traverse4 restricted to leaves of rank > after: slots whose last rank is
// <= after are skipped whole.  A self-query of the hierarchy's own leaf at
// rank r with after = r meets every overlapping pair once (from its
// lower-ranked member) instead of twice; leaf(prim, rank) gets both.
template <class Leaf>
IPCB_D bool traverse4_after(const float4* __restrict__ wide, int n, int after, f3 qlo, f3 qhi, Leaf&& leaf) {
  if (n <= 0) return true;
  int stack[kWideStack];
  int sp = 0;
  int node = 0;
  bool ok = true;
  const int max_visits = n + 64;
  for (int visits = 0;; ++visits) {
    if (visits >= max_visits) return false;
    const float4* w = wide + 8 * node;
    const int4 ls = __ldg(reinterpret_cast<const int4*>(w + 7));
    const int last[4] = {ls.x, ls.y, ls.z, ls.w};
    float4 lx = __ldg(w), ly = __ldg(w + 1), lz = __ldg(w + 2), hx = __ldg(w + 3), hy = __ldg(w + 4),
           hz = __ldg(w + 5);
    int4 cd = __ldg(reinterpret_cast<const int4*>(w + 6));
    const float alx[4] = {lx.x, lx.y, lx.z, lx.w}, aly[4] = {ly.x, ly.y, ly.z, ly.w}, alz[4] = {lz.x, lz.y, lz.z, lz.w};
    const float ahx[4] = {hx.x, hx.y, hx.z, hx.w}, ahy[4] = {hy.x, hy.y, hy.z, hy.w}, ahz[4] = {hz.x, hz.y, hz.z, hz.w};
    const int code[4] = {cd.x, cd.y, cd.z, cd.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (last[k] <= after) continue;
      bool hit = alx[k] <= qhi.x && qlo.x <= ahx[k] && aly[k] <= qhi.y && qlo.y <= ahy[k] && alz[k] <= qhi.z &&
                 qlo.z <= ahz[k];
      if (!hit) continue;
      if (code[k] < 0) {
        leaf(~code[k], last[k]);
      } else if (sp < kWideStack) {
        stack[sp++] = code[k];
      } else {
        ok = false;
      }
    }
    if (sp == 0) break;
    node = stack[--sp];
  }
  return ok;
}

template <class Leaf>
IPCB_D bool traverse4(const float4* __restrict__ wide, int n, f3 qlo, f3 qhi, Leaf&& leaf) {
  if (n <= 0) return true;
  int stack[kWideStack];
  int sp = 0;
  int node = 0;
  bool ok = true;
  const int max_visits = n + 64;
  for (int visits = 0;; ++visits) {
    if (visits >= max_visits) return false;
    const float4* w = wide + 8 * node;
    float4 lx = __ldg(w), ly = __ldg(w + 1), lz = __ldg(w + 2), hx = __ldg(w + 3), hy = __ldg(w + 4),
           hz = __ldg(w + 5);
    int4 cd = __ldg(reinterpret_cast<const int4*>(w + 6));
    const float alx[4] = {lx.x, lx.y, lx.z, lx.w}, aly[4] = {ly.x, ly.y, ly.z, ly.w}, alz[4] = {lz.x, lz.y, lz.z, lz.w};
    const float ahx[4] = {hx.x, hx.y, hx.z, hx.w}, ahy[4] = {hy.x, hy.y, hy.z, hy.w}, ahz[4] = {hz.x, hz.y, hz.z, hz.w};
    const int code[4] = {cd.x, cd.y, cd.z, cd.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      bool hit = alx[k] <= qhi.x && qlo.x <= ahx[k] && aly[k] <= qhi.y && qlo.y <= ahy[k] && alz[k] <= qhi.z &&
                 qlo.z <= ahz[k];
      if (!hit) continue;
      if (code[k] < 0) {
        leaf(~code[k]);
      } else if (sp < kWideStack) {
        stack[sp++] = code[k];
      } else {
        ok = false;
      }
    }
    if (sp == 0) break;
    node = stack[--sp];
  }
  return ok;
}

}  // namespace ipcb

// Exact float32 proximity predicates (the acceptance tests of the broad phase,
// the narrow-phase gate and the feature dispatch).  All arithmetic goes through
// the correctly rounded x* helpers so the results do not depend on FMA
// contraction.
#pragma once
#include "common.cuh"

namespace ipcb {

// Point-triangle closest point by Voronoi region, in the region order of
// contact.py:230-302 (vertex A, vertex B, edge AB, vertex C, edge AC, edge BC,
// face).  type: 0 A, 1 B, 2 C, 3 AB, 4 AC, 5 BC, 6 face.
struct CPT {
  float u, v, d;
  int type;
};
IPCB_D CPT closest_point_triangle(f3 p, f3 a, f3 b, f3 c) {
  CPT r{0.f, 0.f, 0.f, -1};
  f3 ab = esub(b, a), ac = esub(c, a), ap = esub(p, a);
  float d1 = edot(ab, ap), d2 = edot(ac, ap);
  if (d1 <= 0.f && d2 <= 0.f) r = CPT{1.f, 0.f, elength(esub(p, a)), 0};
  f3 bp = esub(p, b);
  float d3 = edot(ab, bp), d4 = edot(ac, bp);
  if (d3 >= 0.f && d4 <= d3 && r.type == -1) r = CPT{0.f, 1.f, elength(esub(p, b)), 1};
  float vc = xsub(xmul(d1, d4), xmul(d3, d2));
  if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f && r.type == -1) {
    float v = xdiv(d1, xsub(d1, d3));
    f3 pt = eadd(a, escale(ab, v));
    r = CPT{xsub(1.f, v), v, elength(esub(p, pt)), 3};
  }
  f3 cp = esub(p, c);
  float d5 = edot(ab, cp), d6 = edot(ac, cp);
  if (d6 >= 0.f && d5 <= d6 && r.type == -1) r = CPT{0.f, 0.f, elength(esub(p, c)), 2};
  float vb = xsub(xmul(d5, d2), xmul(d1, d6));
  if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f && r.type == -1) {
    float w = xdiv(d2, xsub(d2, d6));
    f3 pt = eadd(a, escale(ac, w));
    r = CPT{xsub(1.f, w), 0.f, elength(esub(p, pt)), 4};
  }
  float va = xsub(xmul(d3, d6), xmul(d5, d4));
  float d43 = xsub(d4, d3), d56 = xsub(d5, d6);
  if (va <= 0.f && d43 >= 0.f && d56 >= 0.f && r.type == -1) {
    float w = xdiv(d43, xadd(d43, d56));
    f3 pt = eadd(b, escale(esub(c, b), w));
    r = CPT{0.f, xsub(1.f, w), elength(esub(p, pt)), 5};
  }
  if (r.type == -1) {
    float denom = xdiv(1.f, xadd(xadd(va, vb), vc));
    float v = xmul(vb, denom), w = xmul(vc, denom);
    float u = xsub(xsub(1.f, v), w);
    f3 pt = eadd(eadd(a, escale(ab, v)), escale(ac, w));
    r = CPT{u, v, elength(esub(p, pt)), 6};
  }
  return r;
}

// Closest points between segments p1q1 and p2q2 (s on the first, t on the
// second) and their distance: the clamped segment-segment method of Ericson,
// Real-Time Collision Detection (2005) 5.1.9, with the degenerate-segment
// threshold `eps` on squared lengths.
struct CPEE {
  float s, t, d;
};
IPCB_D CPEE closest_point_edge_edge(f3 p1, f3 q1, f3 p2, f3 q2, float eps) {
  f3 d1 = esub(q1, p1), d2 = esub(q2, p2), r = esub(p1, p2);
  float a = edot(d1, d1), e = edot(d2, d2), f = edot(d2, r);
  float s = 0.f, t = 0.f;
  if (a <= eps && e <= eps) {
    s = 0.f;
    t = 0.f;
  } else if (a <= eps) {
    s = 0.f;
    t = clampv(xdiv(f, e), 0.f, 1.f);
  } else {
    float c = edot(d1, r);
    if (e <= eps) {
      t = 0.f;
      s = clampv(xdiv(-c, a), 0.f, 1.f);
    } else {
      float b = edot(d1, d2);
      float denom = xsub(xmul(a, e), xmul(b, b));
      s = (denom != 0.f) ? clampv(xdiv(xsub(xmul(b, f), xmul(c, e)), denom), 0.f, 1.f) : 0.f;
      t = xdiv(xadd(xmul(b, s), f), e);
      if (t < 0.f) {
        t = 0.f;
        s = clampv(xdiv(-c, a), 0.f, 1.f);
      } else if (t > 1.f) {
        t = 1.f;
        s = clampv(xdiv(xsub(b, c), a), 0.f, 1.f);
      }
    }
  }
  f3 c1 = eadd(p1, escale(d1, s)), c2 = eadd(p2, escale(d2, t));
  return CPEE{s, t, elength(esub(c1, c2))};
}

}  // namespace ipcb

// ORACLE -- test infrastructure, not product code.
//
// A second CPU restatement of the reference's P1 and P4 formulas
// (subgraph_matching/pattern_kernels.cuh:6-133 and :855-963, combined as in
// subgraph_matching/sm_multigpu.cu:206-232), for graphs whose hubs make the
// literal restatement in patterns_oracle.cpp take hours: the same per-edge
// sets and sizes, counted through the symmetry of the graph with position
// marks instead of one binary search per pair.
//
// P1 star term of v0, N0 = N(v0) sorted, position i of N0:
//   c_i    = #{x < i : N0[x] not adjacent to N0[i]} = i - lo_i
//   freq_i = #{j > i : N0[j] not adjacent to N0[i]} = (d0 - 1 - i) - hi_i
//   with lo_i / hi_i the neighbours of N0[i] inside N0 before / after i;
//   star += wrap32(c_i * freq_i)                      (:68-133)
// P1 correction of the directed edge (v0, v1), v0 != v1:
//   A = {x in N0 : x < v1, x notin N1}, B = {x in N0 : x < v1, x in N1}
//   corr += sum over v2 in B of #{k in A : k > v2, k notin N(v2)}   (:6-66)
//         = (pos0(v1) - pos0(v2) - 1) - #{x in B : x > v2}
//           - #{k in N(v2) : v2 < k < v1, k in N0, k notin N1}
// P4 of the directed edge (v0, v1), v1 < v0:
//   A = N0 - N1, B = N1 - N0;  c1 += |A| |B| - #{(a, b) : a ~ b}
//   (the reference's pair loop of :898-958), the adjacent pairs counted from
//   whichever side has the smaller degree sum.
// wrap32 is the reference's 32-bit int product, as in patterns_oracle.cpp;
// every other quantity is a count of the same sets, so the results equal the
// literal restatement exactly (tests/test_oracle.py checks that).
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <vector>

namespace {

inline uint64_t wrap_mul32(int64_t a, int64_t b) {
  const uint32_t p = (uint32_t)a * (uint32_t)b;
  return (uint64_t)(int64_t)(int32_t)p;
}

struct Csr {
  int64_t n;
  const int64_t *rp;
  const int32_t *ci;
  int64_t deg(int64_t v) const { return rp[v + 1] - rp[v]; }
};

// Per-thread marks: pos0[v] = position of v in N(v0) (or -1), seen1[v] ==
// stamp iff v in N(v1) for the current edge.
struct Marks {
  std::vector<int32_t> pos0;
  std::vector<int64_t> seen1;
  int64_t stamp = 0;
  explicit Marks(int64_t n) : pos0(n, -1), seen1(n, -1) {}
};

uint64_t p1_vertex(const Csr &g, int64_t v0, Marks &mk, std::vector<int32_t> &B,
                   uint64_t &corr) {
  const int64_t d0 = g.deg(v0);
  const int32_t *n0 = g.ci + g.rp[v0];
  for (int64_t i = 0; i < d0; ++i) mk.pos0[n0[i]] = (int32_t)i;
  uint64_t star = 0;
  for (int64_t i = 0; i < d0; ++i) {
    const int32_t x = n0[i];
    int64_t lo = 0, hi = 0;
    for (int64_t e = g.rp[x]; e < g.rp[x + 1]; ++e) {
      const int32_t p = mk.pos0[g.ci[e]];
      if (p < 0) continue;
      if (p < i) ++lo;
      else if (p > i) ++hi;
    }
    star += wrap_mul32(i - lo, (d0 - 1 - i) - hi);
  }
  for (int64_t p1 = 0; p1 < d0; ++p1) {
    const int32_t v1 = n0[p1];
    if (v1 == v0) continue;
    const int64_t stamp = ++mk.stamp;
    const int32_t *n1 = g.ci + g.rp[v1];
    const int64_t d1 = g.deg(v1);
    for (int64_t e = 0; e < d1; ++e) mk.seen1[n1[e]] = stamp;
    // B = N0 & N1 below v1, ascending: the shorter of the two lists drives.
    B.clear();
    const int64_t below0 = p1;  // entries of N0 below v1
    const int64_t below1 = std::lower_bound(n1, n1 + d1, v1) - n1;
    if (below0 <= below1) {
      for (int64_t i = 0; i < below0; ++i)
        if (mk.seen1[n0[i]] == stamp) B.push_back(n0[i]);
    } else {
      for (int64_t i = 0; i < below1; ++i)
        if (mk.pos0[n1[i]] >= 0) B.push_back(n1[i]);
    }
    const int64_t nb = (int64_t)B.size();
    for (int64_t t = 0; t < nb; ++t) {
      const int32_t v2 = B[t];
      int64_t term = (int64_t)(p1 - mk.pos0[v2] - 1) - (nb - 1 - t);
      const int32_t *l = g.ci + g.rp[v2], *le = g.ci + g.rp[v2 + 1];
      for (const int32_t *k = std::upper_bound(l, le, v2); k != le && *k < v1; ++k)
        if (mk.pos0[*k] >= 0 && mk.seen1[*k] != stamp) --term;
      corr += (uint64_t)term;
    }
  }
  for (int64_t i = 0; i < d0; ++i) mk.pos0[n0[i]] = -1;
  return star;
}

uint64_t p4_vertex(const Csr &g, int64_t v0, Marks &mk) {
  const int64_t d0 = g.deg(v0);
  const int32_t *n0 = g.ci + g.rp[v0];
  for (int64_t i = 0; i < d0; ++i) mk.pos0[n0[i]] = (int32_t)i;
  uint64_t c1 = 0;
  for (int64_t p1 = 0; p1 < d0; ++p1) {
    const int32_t v1 = n0[p1];
    if (!(v1 < v0)) break;  // N0 ascending: the rest are larger
    const int64_t stamp = ++mk.stamp;
    const int32_t *n1 = g.ci + g.rp[v1];
    const int64_t d1 = g.deg(v1);
    int64_t common = 0;
    for (int64_t e = 0; e < d1; ++e) {
      mk.seen1[n1[e]] = stamp;
      common += mk.pos0[n1[e]] >= 0;
    }
    const int64_t na = d0 - common, nb = d1 - common;
    // Degree sums of A = N0 - N1 and B = N1 - N0.
    int64_t sa = 0, sb = 0;
    for (int64_t i = 0; i < d0; ++i)
      if (mk.seen1[n0[i]] != stamp) sa += g.deg(n0[i]);
    for (int64_t e = 0; e < d1; ++e)
      if (mk.pos0[n1[e]] < 0) sb += g.deg(n1[e]);
    int64_t adj = 0;
    if (sa <= sb) {
      for (int64_t i = 0; i < d0; ++i) {
        const int32_t a = n0[i];
        if (mk.seen1[a] == stamp) continue;
        for (int64_t e = g.rp[a]; e < g.rp[a + 1]; ++e) {
          const int32_t y = g.ci[e];
          adj += mk.seen1[y] == stamp && mk.pos0[y] < 0;
        }
      }
    } else {
      for (int64_t e1 = 0; e1 < d1; ++e1) {
        const int32_t b = n1[e1];
        if (mk.pos0[b] >= 0) continue;
        for (int64_t e = g.rp[b]; e < g.rp[b + 1]; ++e) {
          const int32_t y = g.ci[e];
          adj += mk.pos0[y] >= 0 && mk.seen1[y] != stamp;
        }
      }
    }
    c1 += (uint64_t)(na * nb - adj);
  }
  for (int64_t i = 0; i < d0; ++i) mk.pos0[n0[i]] = -1;
  return c1;
}

}  // namespace

extern "C" {

// P1 (c1 - c2) or P4 (c1) of a simple symmetric CSR; c12 (optional) gets
// (c1, c2).  Returns 0 with c12 untouched for any other pattern.
uint64_t orc_pattern_fast(int64_t n, const int64_t *rowptr, const int32_t *col, int pattern,
                          uint64_t *c12) {
  if (pattern != 1 && pattern != 4) return 0;
  const Csr g{n, rowptr, col};
  uint64_t c1 = 0, c2 = 0;
#pragma omp parallel reduction(+ : c1, c2)
  {
    Marks mk(n);
    std::vector<int32_t> B;
#pragma omp for schedule(dynamic, 1)
    for (int64_t v0 = 0; v0 < n; ++v0) {
      if (pattern == 1) c1 += p1_vertex(g, v0, mk, B, c2);
      else c1 += p4_vertex(g, v0, mk);
    }
  }
  if (c12) {
    c12[0] = c1;
    c12[1] = c2;
  }
  return pattern == 4 ? c1 : c1 - c2;
}

}  // extern "C"

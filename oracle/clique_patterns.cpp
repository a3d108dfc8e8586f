// ORACLE -- test infrastructure, not product code.
//
// A second CPU restatement of the reference's P7 and P8 formulas
// (subgraph_matching/pattern_kernels.cuh:352-459 and :461-572, combined as
// in subgraph_matching/sm_multigpu.cu:206-232), for graphs whose hubs make
// the literal restatement in patterns_oracle.cpp take days.
//
// P7.  Per directed edge
// (v0, v1) the formula counts the triples of A = N(v0) & N(v1) that are
// pairwise non-adjacent, I3(A) (its frequency term less its correction).
// By inclusion-exclusion over the edges inside A,
//   I3(A) = C(a, 3) - e_A (a - 2) + sum over x in A of C(d_A(x), 2) - t_A,
// where a = |A| (the edge's triangles), e_A = the edges inside A (the K4s on
// the edge), d_A(x) = x's neighbours inside A (the K4s on the triangle
// {v0, v1, x}) and t_A = the triangles inside A (the K5s on the edge).  Both
// directions of an undirected edge have the same A; each triangle appears
// for its three edges and each K5 holds ten edges, so over the graph
//   P7 = 2 [ sum_e C(a_e, 3) - sum_e k4_e (a_e - 2)
//            + 3 sum_tau C(k4_tau, 2) - 10 K5 ].
//
// P8.  The formula counts, per directed edge (v0, v1), the pairs of
// adjacent x < v2 in A with a v4 in N(v1) - N(v0) adjacent to neither: a K4
// {v0, v1, v2, x} with a vertex hung on v1 alone, an induced tailed K4, once
// for each of the three other K4 vertices as v0.  For a K4 Q and q in Q,
// inclusion-exclusion over N(q) gives the vertices hung on q alone:
//   d(q) - 3 - sum_p (a_qp - 2) + sum_{p,r} (k_qpr - 1) - k5_Q
// (p, r the other vertices, a the triangles on an edge, k the K4s on a
// triangle, k5_Q the K5s on Q).  Summed over q and over every K4 (a
// triangle lies in k_tau K4s, an edge's K4s are half the k of its
// triangles, a vertex's a third, a K5 holds five K4s):
//   P8 = sum_tau k_tau (d_x + d_y + d_z) - 3 sum_tau k_tau (a_e1 + a_e2 + a_e3)
//        + 9 sum_tau k_tau^2 - 60 K5.
//
// The counts come from listing every triangle, K4 and K5 once on the
// degree-ordered DAG (u -> v iff d(v) > d(u), or equal and v > u).  The
// reference multiplies two 32-bit ints per term (:411, :526); the
// identities hold while those products cannot wrap, i.e. for a maximum
// degree of at most 46,340, and the function refuses larger graphs.
// tests/test_oracle.py checks both against the literal restatement on
// random graphs, the fixtures and graphs with hubs.
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <vector>

namespace {

using u128 = unsigned __int128;

inline int64_t index_in(const int32_t *b, const int32_t *e, int32_t v) {
  return std::lower_bound(b, e, v) - b;
}

}  // namespace

extern "C" {

// Returns 0 and writes P7 and P8 (mod 2^64) to result[0..1], or -1 when the
// maximum degree exceeds 46,340.  terms (optional, 7 doubles): triangles,
// K4, K5, sum_e C(a_e,3), sum_e k4_e (a_e - 2), 3 sum C(k4_tau,2), 10 K5.
int orc_clique_patterns(int64_t n, const int64_t *rp, const int32_t *ci, uint64_t *result,
                        double *terms) {
  for (int64_t v = 0; v < n; ++v)
    if (rp[v + 1] - rp[v] > 46340) return -1;
  auto keep = [&](int64_t u, int32_t v) {
    const int64_t du = rp[u + 1] - rp[u], dv = rp[v + 1] - rp[v];
    return dv > du || (dv == du && v > u);
  };
  // The DAG, rows ascending.
  std::vector<int64_t> drp(n + 1, 0);
  for (int64_t u = 0; u < n; ++u) {
    int64_t c = 0;
    for (int64_t e = rp[u]; e < rp[u + 1]; ++e) c += keep(u, ci[e]);
    drp[u + 1] = drp[u] + c;
  }
  const int64_t m = drp[n];
  std::vector<int32_t> dcol(m);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t u = 0; u < n; ++u) {
    int64_t o = drp[u];
    for (int64_t e = rp[u]; e < rp[u + 1]; ++e)
      if (keep(u, ci[e])) dcol[o++] = ci[e];
  }
  auto row = [&](int64_t u) { return dcol.data() + drp[u]; };
  auto row_end = [&](int64_t u) { return dcol.data() + drp[u + 1]; };
  auto eid = [&](int64_t u, int32_t v) { return drp[u] + index_in(row(u), row_end(u), v); };
  // Triangle lists T_i = N+(u) & N+(v) for each DAG edge i = (u -> v).
  std::vector<int64_t> toff(m + 1, 0);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t u = 0; u < n; ++u)
    for (int64_t i = drp[u]; i < drp[u + 1]; ++i) {
      const int32_t v = dcol[i];
      const int32_t *a = row(u), *ae = row_end(u), *b = row(v), *be = row_end(v);
      int64_t c = 0;
      while (a < ae && b < be) {
        if (*a < *b) ++a;
        else if (*b < *a) ++b;
        else { ++c; ++a; ++b; }
      }
      toff[i + 1] = c;
    }
  for (int64_t i = 0; i < m; ++i) toff[i + 1] += toff[i];
  const int64_t ntri = toff[m];
  std::vector<int32_t> tcol(ntri);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t u = 0; u < n; ++u)
    for (int64_t i = drp[u]; i < drp[u + 1]; ++i) {
      const int32_t v = dcol[i];
      std::set_intersection(row(u), row_end(u), row(v), row_end(v), tcol.begin() + toff[i]);
    }
  auto tri = [&](int64_t i) { return tcol.data() + toff[i]; };
  auto tri_end = [&](int64_t i) { return tcol.data() + toff[i + 1]; };
  // a_e, k4_e per DAG edge; k4_tau per triangle; K4 and K5 totals.
  std::vector<int64_t> a(m, 0), k4e(m, 0);
  std::vector<int32_t> k4t(ntri, 0);
  double k4_total = 0, k5_total = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : k4_total, k5_total)
  for (int64_t u = 0; u < n; ++u) {
    std::vector<int32_t> S;
    for (int64_t i = drp[u]; i < drp[u + 1]; ++i) {
      const int32_t v = dcol[i];
      for (const int32_t *pw = tri(i); pw != tri_end(i); ++pw) {
        const int32_t w = *pw;  // triangle (u, v, w) in DAG order
        const int64_t uw = eid(u, w), vw = eid(v, w);
        __atomic_fetch_add(&a[i], 1, __ATOMIC_RELAXED);
        __atomic_fetch_add(&a[uw], 1, __ATOMIC_RELAXED);
        __atomic_fetch_add(&a[vw], 1, __ATOMIC_RELAXED);
        // K4s (u, v, w, x): x in T_i & N+(w).
        S.clear();
        std::set_intersection(tri(i), tri_end(i), row(w), row_end(w), std::back_inserter(S));
        if (S.empty()) continue;
        const int64_t s = (int64_t)S.size();
        k4_total += (double)s;
        __atomic_fetch_add(&k4e[i], s, __ATOMIC_RELAXED);
        __atomic_fetch_add(&k4e[uw], s, __ATOMIC_RELAXED);
        __atomic_fetch_add(&k4e[vw], s, __ATOMIC_RELAXED);
        __atomic_fetch_add(&k4t[toff[i] + (pw - tri(i))], (int32_t)s, __ATOMIC_RELAXED);
        for (const int32_t x : S) {
          __atomic_fetch_add(&k4e[eid(u, x)], 1, __ATOMIC_RELAXED);
          __atomic_fetch_add(&k4e[eid(v, x)], 1, __ATOMIC_RELAXED);
          __atomic_fetch_add(&k4e[eid(w, x)], 1, __ATOMIC_RELAXED);
          __atomic_fetch_add(&k4t[toff[i] + index_in(tri(i), tri_end(i), x)], 1, __ATOMIC_RELAXED);
          __atomic_fetch_add(&k4t[toff[uw] + index_in(tri(uw), tri_end(uw), x)], 1,
                             __ATOMIC_RELAXED);
          __atomic_fetch_add(&k4t[toff[vw] + index_in(tri(vw), tri_end(vw), x)], 1,
                             __ATOMIC_RELAXED);
          // K5s (u, v, w, x, y): y in S & N+(x).
          int64_t c = 0;
          const int32_t *b = row(x), *be = row_end(x);
          for (const int32_t y : S)
            if (y != x && std::binary_search(b, be, y)) ++c;
          k5_total += (double)c;
        }
      }
    }
  }
  u128 s1 = 0, s2 = 0, s3 = 0;
  for (int64_t i = 0; i < m; ++i) {
    const u128 t = (u128)a[i];
    if (t >= 3) s1 += t * (t - 1) * (t - 2) / 6;
    if (t >= 2) s2 += (u128)k4e[i] * (t - 2);
  }
  for (int64_t j = 0; j < ntri; ++j) {
    const u128 k = (u128)k4t[j];
    if (k >= 2) s3 += 3 * (k * (k - 1) / 2);
  }
  const u128 s4 = 10 * (u128)(uint64_t)k5_total;
  // The true values are non-negative; the reference's u64 result is each
  // modulo 2^64.
  const u128 p7 = 2 * (s1 + s3 - s2 - s4);
  // P8's triangle terms: k (d_x + d_y + d_z), 3 k (a_e1 + a_e2 + a_e3), 9 k^2.
  u128 t_deg = 0, t_a = 0, t_k2 = 0;
#pragma omp parallel
  {
    u128 dg = 0, ta = 0, k2 = 0;
#pragma omp for schedule(dynamic, 256)
    for (int64_t u = 0; u < n; ++u)
      for (int64_t i = drp[u]; i < drp[u + 1]; ++i) {
        const int32_t v = dcol[i];
        for (int64_t j = toff[i]; j < toff[i + 1]; ++j) {
          const int32_t w = tcol[j];
          const u128 k = (u128)k4t[j];
          if (k == 0) continue;
          const u128 d = (u128)((rp[u + 1] - rp[u]) + (rp[v + 1] - rp[v]) + (rp[w + 1] - rp[w]));
          const u128 s = (u128)(a[i] + a[eid(u, w)] + a[eid(v, w)]);
          dg += k * d;
          ta += k * s;
          k2 += k * k;
        }
      }
#pragma omp critical
    {
      t_deg += dg;
      t_a += ta;
      t_k2 += k2;
    }
  }
  const u128 p8 = t_deg + 9 * t_k2 - 3 * t_a - 60 * (u128)(uint64_t)k5_total;
  result[0] = (uint64_t)p7;
  result[1] = (uint64_t)p8;
  if (terms) {
    const double v[] = {(double)ntri, k4_total, k5_total, (double)s1, (double)s2, (double)s3,
                        (double)s4};
    for (int k = 0; k < 7; ++k) terms[k] = v[k];
  }
  return 0;
}

}  // extern "C"

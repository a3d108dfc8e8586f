// ORACLE -- test infrastructure, not product code.
//
// A CPU restatement of the reference's counting path, used only as the
// checker of the CUDA path (tests/, the smoke check) and as the timed CPU
// baseline of bench.py.  Nothing in mercury_b200/ links or calls it.
//
// Restated reference behaviour (paths relative to the reference project):
//   * orc_orient     -- Graph::orientation_with_division, DAG part
//                       (graph.cc:196-235): u->v iff deg v > deg u, or equal
//                       degrees and v > u; rows keep ascending id order.
//   * orc_division   -- the small/large split of the same function
//                       (graph.cc:237-312, REVERSE_DAG at graph.cc:4) and the
//                       task lists of TCSolver (tc_challenge.cu:20-46).
//   * orc_tc_*       -- the quantity TCSolver computes: sum over DAG edges
//                       (u->v) of |N+(u) & N+(v)|, by the two-pointer merge of
//                       Graph::intersect_num (graph.cc:396-411, labels
//                       dropped).  Parity pinned in tests/test_oracle.py
//                       against brute-force triangle enumeration and the
//                       fixtures in tests/golden/.
//   * orc_tc_by_label -- the labelled two-pointer merge of
//                       Graph::intersect_num(v, u, label) (graph.cc:396-411,
//                       counted only when vlabels[a] == label), summed over
//                       the DAG edges v->u for every label at once: counts[l]
//                       = triangles whose common out-neighbour has label l.
//   * orc_pattern    -- the P1..P8 formulas of
//                       subgraph_matching/pattern_kernels.cuh (see the
//                       comment above each case below).
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

struct Csr {
  int64_t n;
  const int64_t *rp;
  const int32_t *ci;
  int32_t deg(int64_t v) const { return (int32_t)(rp[v + 1] - rp[v]); }
  const int32_t *begin(int64_t v) const { return ci + rp[v]; }
  const int32_t *end(int64_t v) const { return ci + rp[v + 1]; }
};

bool dag_keep(const Csr &g, int64_t src, int32_t dst) {
  int32_t ds = g.deg(src), dd = g.deg(dst);
  return dd > ds || (dd == ds && dst > src);
}

uint64_t merge_count(const int32_t *a, int64_t na, const int32_t *b, int64_t nb) {
  int64_t i = 0, j = 0;
  uint64_t c = 0;
  while (i < na && j < nb) {
    int32_t x = a[i], y = b[j];
    if (x <= y) ++i;
    if (y <= x) ++j;
    if (x == y) ++c;
  }
  return c;
}

}  // namespace

extern "C" {

int orc_num_threads(void) { return omp_get_max_threads(); }

// DAG out-degrees d+[v] and the DAG CSR (dag_rowptr[n+1], dag_col[m+]).
// Pass dag_col == nullptr to get only the row offsets (and m+ at [n]).
void orc_orient(int64_t n, const int64_t *rowptr, const int32_t *col, int64_t *dag_rowptr,
                int32_t *dag_col) {
  Csr g{n, rowptr, col};
  std::vector<int64_t> nd(n, 0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < n; ++v) {
    int64_t c = 0;
    for (const int32_t *p = g.begin(v); p != g.end(v); ++p) c += dag_keep(g, v, *p);
    nd[v] = c;
  }
  dag_rowptr[0] = 0;
  for (int64_t v = 0; v < n; ++v) dag_rowptr[v + 1] = dag_rowptr[v] + nd[v];
  if (!dag_col) return;
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < n; ++v) {
    int64_t o = dag_rowptr[v];
    for (const int32_t *p = g.begin(v); p != g.end(v); ++p)
      if (dag_keep(g, v, *p)) dag_col[o++] = *p;
  }
}

// The reference's small/large division counts: out[0] small edges,
// out[1] large edges, out[2] small tasks, out[3] large tasks.
void orc_division(int64_t n, const int64_t *rowptr, const int32_t *col, int deg_thd,
                  int64_t *out) {
  Csr g{n, rowptr, col};
  std::vector<int64_t> drp(n + 1);
  orc_orient(n, rowptr, col, drp.data(), nullptr);
  auto nd = [&](int64_t v) { return drp[v + 1] - drp[v]; };
  int64_t small = 0, large = 0, st = 0, lt = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : small, large, st, lt)
  for (int64_t src = 0; src < n; ++src) {
    int64_t s_src = 0, l_src = 0;
    const int64_t ns = nd(src);
    for (const int32_t *p = g.begin(src); p != g.end(src); ++p) {
      const int32_t dst = *p;
      const int64_t ndst = nd(dst);
      if (std::min(ns, ndst) < 1) continue;
      if (std::max(ns, ndst) <= deg_thd) {
        if (dag_keep(g, src, dst)) ++s_src;
      } else if (ns >= deg_thd || ndst >= deg_thd) {
        if (ns > ndst || (ndst == ns && src > dst)) ++l_src;
      }
    }
    small += s_src;
    large += l_src;
    st += s_src != 0;
    lt += l_src != 0;
  }
  out[0] = small;
  out[1] = large;
  out[2] = st;
  out[3] = lt;
}

// Triangle count over a prebuilt DAG, restricted to sources [v0, v1)
// (the whole graph with v0 = 0, v1 = n).
uint64_t orc_tc_dag(int64_t n, const int64_t *dag_rowptr, const int32_t *dag_col, int64_t v0,
                    int64_t v1) {
  Csr d{n, dag_rowptr, dag_col};
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total)
  for (int64_t u = v0; u < v1; ++u) {
    const int32_t *a = d.begin(u);
    const int64_t na = d.deg(u);
    for (int64_t i = 0; i < na; ++i) {
      const int32_t v = a[i];
      total += merge_count(a, na, d.begin(v), d.deg(v));
    }
  }
  return total;
}

// Triangle count over the sources u with mix(u ^ seed) % modulus == 0 (a
// hash-sampled 1/modulus of the vertices, for a bounded CPU timing);
// *edges_out receives the number of DAG edges those sources own.
uint64_t orc_tc_sample(int64_t n, const int64_t *dag_rowptr, const int32_t *dag_col,
                       uint64_t modulus, uint64_t seed, int64_t *edges_out) {
  Csr d{n, dag_rowptr, dag_col};
  uint64_t total = 0;
  int64_t edges = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total, edges)
  for (int64_t u = 0; u < n; ++u) {
    uint64_t h = (uint64_t)u ^ seed;
    h = (h ^ (h >> 33)) * 0xff51afd7ed558ccdull;
    h = (h ^ (h >> 33)) * 0xc4ceb9fe1a85ec53ull;
    h ^= h >> 33;
    if (h % modulus) continue;
    const int32_t *a = d.begin(u);
    const int64_t na = d.deg(u);
    edges += na;
    for (int64_t i = 0; i < na; ++i) total += merge_count(a, na, d.begin(a[i]), d.deg(a[i]));
  }
  *edges_out = edges;
  return total;
}

// Sum over DAG edges (u->v) of (d+u + d+v): the merge volume of the count.
double orc_merge_volume(int64_t n, const int64_t *dag_rowptr, const int32_t *dag_col) {
  double s = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : s)
  for (int64_t u = 0; u < n; ++u)
    for (int64_t e = dag_rowptr[u]; e < dag_rowptr[u + 1]; ++e) {
      int32_t v = dag_col[e];
      s += (double)(dag_rowptr[u + 1] - dag_rowptr[u]) + (double)(dag_rowptr[v + 1] - dag_rowptr[v]);
    }
  return s;
}

// Whole triangle count of a symmetric CSR.
// counts[0..max_label]; labels[v] <= max_label.
void orc_tc_by_label(int64_t n, const int64_t *rowptr, const int32_t *col, const uint8_t *labels,
                     int max_label, uint64_t *counts) {
  std::vector<int64_t> drp(n + 1);
  orc_orient(n, rowptr, col, drp.data(), nullptr);
  std::vector<int32_t> dcol(std::max<int64_t>(drp[n], 1));
  orc_orient(n, rowptr, col, drp.data(), dcol.data());
  const int L1 = max_label + 1;
  std::vector<uint64_t> total(L1, 0);
#pragma omp parallel
  {
    std::vector<uint64_t> mine(L1, 0);
#pragma omp for schedule(dynamic, 256)
    for (int64_t v = 0; v < n; ++v) {
      for (int64_t e = drp[v]; e < drp[v + 1]; ++e) {
        const int32_t u = dcol[e];
        const int32_t *a = dcol.data() + drp[v], *b = dcol.data() + drp[u];
        const int64_t na = drp[v + 1] - drp[v], nb = drp[u + 1] - drp[u];
        int64_t i = 0, j = 0;
        while (i < na && j < nb) {  // intersect_num's merge, label per hit
          const int32_t x = a[i], y = b[j];
          if (x <= y) ++i;
          if (y <= x) ++j;
          if (x == y) ++mine[labels[x]];
        }
      }
    }
#pragma omp critical
    for (int l = 0; l < L1; ++l) total[l] += mine[l];
  }
  for (int l = 0; l < L1; ++l) counts[l] = total[l];
}

uint64_t orc_tc(int64_t n, const int64_t *rowptr, const int32_t *col) {
  std::vector<int64_t> drp(n + 1);
  orc_orient(n, rowptr, col, drp.data(), nullptr);
  std::vector<int32_t> dcol(std::max<int64_t>(drp[n], 1));
  orc_orient(n, rowptr, col, drp.data(), dcol.data());
  return orc_tc_dag(n, drp.data(), dcol.data(), 0, n);
}

}  // extern "C"

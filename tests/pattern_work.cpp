// Test infrastructure, not product code: the set sizes that set the cost of
// the reference's pattern formulas on a graph (subgraph_matching/
// pattern_kernels.cuh), counted on the CPU.  Per directed edge (v0, v1):
// A = N(v0) & N(v1) (|A| = the edge's triangles), B = N(v1) - N(v0)
// (|B| = d(v1) - |A|, v0 included).  The per-edge triangle counts come from
// listing every triangle once on the degree-ordered DAG (u -> v iff
// d(v) > d(u), or equal and v > u) and adding one to each of its three edges.
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <vector>

extern "C" {

// out[0..5]: triangles, sum over vertices of d^3, sum over directed edges
// of |A|^3, directed edges with |A| > 32, sum over directed edges of
// |A| * |B|, sum over vertices of d^2.
void pattern_work(int64_t n, const int64_t *rp, const int32_t *ci, double *out) {
  std::vector<int64_t> drp(n + 1, 0);
  auto keep = [&](int64_t u, int32_t v) {
    const int64_t du = rp[u + 1] - rp[u], dv = rp[v + 1] - rp[v];
    return dv > du || (dv == du && v > u);
  };
  for (int64_t u = 0; u < n; ++u) {
    int64_t c = 0;
    for (int64_t e = rp[u]; e < rp[u + 1]; ++e) c += keep(u, ci[e]);
    drp[u + 1] = drp[u] + c;
  }
  std::vector<int32_t> dcol(drp[n]);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t u = 0; u < n; ++u) {
    int64_t o = drp[u];
    for (int64_t e = rp[u]; e < rp[u + 1]; ++e)
      if (keep(u, ci[e])) dcol[o++] = ci[e];
  }
  // Triangles per DAG edge (an undirected edge), by listing.
  std::vector<std::atomic<int64_t>> tri(drp[n]);
  for (auto &t : tri) t.store(0, std::memory_order_relaxed);
  auto edge_id = [&](int64_t u, int32_t v) {
    const int32_t *b = dcol.data() + drp[u], *e = dcol.data() + drp[u + 1];
    return (int64_t)(std::lower_bound(b, e, v) - dcol.data());
  };
  double triangles = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : triangles)
  for (int64_t u = 0; u < n; ++u) {
    for (int64_t i = drp[u]; i < drp[u + 1]; ++i) {
      const int32_t v = dcol[i];
      int64_t a = drp[u], ae = drp[u + 1], b = drp[v], be = drp[v + 1];
      while (a < ae && b < be) {
        if (dcol[a] < dcol[b]) ++a;
        else if (dcol[b] < dcol[a]) ++b;
        else {
          const int32_t w = dcol[a];
          tri[i].fetch_add(1, std::memory_order_relaxed);
          tri[edge_id(u, w)].fetch_add(1, std::memory_order_relaxed);
          tri[edge_id(v, w)].fetch_add(1, std::memory_order_relaxed);
          triangles += 1;
          ++a;
          ++b;
        }
      }
    }
  }
  double d3 = 0, d2 = 0, a3 = 0, big = 0, ab = 0;
#pragma omp parallel for schedule(static) reduction(+ : d3, d2)
  for (int64_t v = 0; v < n; ++v) {
    const double d = (double)(rp[v + 1] - rp[v]);
    d3 += d * d * d;
    d2 += d * d;
  }
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : a3, big, ab)
  for (int64_t u = 0; u < n; ++u) {
    for (int64_t i = drp[u]; i < drp[u + 1]; ++i) {
      const int32_t v = dcol[i];
      const double t = (double)tri[i].load(std::memory_order_relaxed);
      const double du = (double)(rp[u + 1] - rp[u]), dv = (double)(rp[v + 1] - rp[v]);
      a3 += 2 * t * t * t;  // both directions have the same A
      big += t > 32 ? 2 : 0;
      ab += t * (dv - t) + t * (du - t);  // (u, v) and (v, u)
    }
  }
  const double o[] = {triangles, d3, a3, big, ab, d2};
  for (int k = 0; k < 6; ++k) out[k] = o[k];
}

}  // extern "C"

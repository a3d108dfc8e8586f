// ORACLE -- test infrastructure, not product code.
//
// CPU restatement of the reference's pattern kernels
// (subgraph_matching/pattern_kernels.cuh) and of the host combine step
// (subgraph_matching/sm_multigpu.cu:206-232).  Each kernel runs over the 2m
// directed edges (v0, v1) of the COO list built by Graph::init_edgelist
// (graph.cc:336-365: every CSR entry in row order, self-loops skipped in
// the source list) and accumulates into counters[1] and counters[2]; the
// result is counters[1] for P4/P6, counters[1] - counters[2] otherwise
// (unsigned 64-bit arithmetic).
//
// The reference's warp set operations are restated by their results:
//   difference_set(a, b[, bound])  = {x in a : [x < bound,] x not in b}
//   intersect(a, b[, bound])       = {x in a & b : [x < bound]}
//   difference_num / intersect_num = sizes of the same sets
// (gpu_kernels/set_difference.cuh:41-237, gpu_kernels/set_intersect.cuh:
// 107-433; the materialising forms compact with ballot+popc in input order,
// so outputs stay sorted, which the bounded forms' early exit relies on).
// Membership tests "binary_search(N(k), x)" keep the reference's direction
// (x searched in k's list).  Where the reference multiplies two `int`s
// before adding to the 64-bit counter (P1 :120, P2 :199, P3 :304, P5 :671,
// P7 :411, P8 :526), the product is wrapped to 32 bits and sign-extended,
// as the GPU integer multiply does.
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <vector>

namespace {

using V = std::vector<int32_t>;

struct G {
  int64_t n;
  const int64_t *rp;
  const int32_t *ci;
  int32_t deg(int64_t v) const { return (int32_t)(rp[v + 1] - rp[v]); }
  const int32_t *b(int64_t v) const { return ci + rp[v]; }
  const int32_t *e(int64_t v) const { return ci + rp[v + 1]; }
  // binary_search(g.N(k), x, k_size)
  bool in(int32_t k, int32_t x) const { return std::binary_search(b(k), e(k), x); }
};

inline uint64_t wrap_mul(int64_t a, int64_t b) {
  const uint32_t p = (uint32_t)a * (uint32_t)b;
  return (uint64_t)(int64_t)(int32_t)p;
}

// {x in a : x < bound, x not in list(k)}; bound < 0 means no bound.
void diff_list(const int32_t *a, const int32_t *ae, const G &g, int32_t k, int64_t bound, V &out) {
  out.clear();
  for (const int32_t *p = a; p != ae; ++p) {
    if (bound >= 0 && *p >= bound) break;
    if (!std::binary_search(g.b(k), g.e(k), *p)) out.push_back(*p);
  }
}
void diff_vec(const V &a, const G &g, int32_t k, int64_t bound, V &out) {
  diff_list(a.data(), a.data() + a.size(), g, k, bound, out);
}
// {x in a & list(k) : x < bound}
void inter_list(const int32_t *a, const int32_t *ae, const G &g, int32_t k, int64_t bound, V &out) {
  out.clear();
  for (const int32_t *p = a; p != ae; ++p) {
    if (bound >= 0 && *p >= bound) break;
    if (std::binary_search(g.b(k), g.e(k), *p)) out.push_back(*p);
  }
}
void inter_vec(const V &a, const G &g, int32_t k, int64_t bound, V &out) {
  inter_list(a.data(), a.data() + a.size(), g, k, bound, out);
}
int64_t count_diff(const V &a, const G &g, int32_t k, int64_t bound) {
  int64_t c = 0;
  for (int32_t x : a) {
    if (bound >= 0 && x >= bound) break;
    c += !g.in(k, x);
  }
  return c;
}
int64_t count_inter(const V &a, const G &g, int32_t k, int64_t bound) {
  int64_t c = 0;
  for (int32_t x : a) {
    if (bound >= 0 && x >= bound) break;
    c += g.in(k, x);
  }
  return c;
}

struct Acc {
  uint64_t c1 = 0, c2 = 0;
};

// freq[j] = #{i > j : a[j] not in N(a[i])}   (P3 :280-292, P7 :386-398)
void pair_freq(const G &g, const V &a, std::vector<int64_t> &freq) {
  freq.assign(a.size(), 0);
  for (size_t i = 0; i < a.size(); ++i)
    for (size_t j = 0; j < i; ++j)
      if (!g.in(a[i], a[j])) ++freq[j];
}

// Correction of P3/P7 (:310-340, :417-449): sum over v2 in A of
// #{(c in A & N(v2), key in A - N(v2), key < v2) : key > c, c not in N(key)}.
uint64_t bounded_correction(const G &g, const V &A, V &D, V &C) {
  uint64_t corr = 0;
  for (int32_t v2 : A) {
    diff_vec(A, g, v2, v2, D);
    inter_vec(A, g, v2, -1, C);
    for (int32_t c : C)
      for (int32_t key : D)
        if (key > c && !g.in(key, c)) ++corr;
  }
  return corr;
}

void edge_pattern(const G &g, int pattern, int32_t v0, int32_t v1, Acc &acc, V &A, V &B, V &C,
                  V &D, V &E, std::vector<int64_t> &freq) {
  const int32_t *n0 = g.b(v0), *n0e = g.e(v0), *n1 = g.b(v1), *n1e = g.e(v1);
  switch (pattern) {
    case 1: {  // P1_count_correction (:6-66)
      if (v0 == v1) return;
      diff_list(n0, n0e, g, v1, v1, A);   // dif, bounded by v1
      inter_list(n0, n0e, g, v1, v1, B);  // int, bounded by v1
      for (int32_t v2 : B)
        for (int32_t key : A)
          if (key > v2 && !g.in(key, v2)) ++acc.c2;
      return;
    }
    case 2: {  // P2_subgraph_matching (:135-243)
      diff_list(n0, n0e, g, v1, -1, A);
      diff_list(n1, n1e, g, v0, -1, B);
      freq.assign(A.size(), 0);
      for (int32_t v4 : B)
        for (size_t j = 0; j < A.size(); ++j)
          if (!g.in(v4, A[j])) ++freq[j];
      for (size_t i = 0; i < A.size(); ++i)
        acc.c1 += wrap_mul(count_diff(A, g, A[i], A[i]), freq[i]);
      for (int32_t v4 : B) {
        diff_vec(A, g, v4, -1, D);
        inter_vec(A, g, v4, -1, C);
        for (int32_t v2 : C)
          for (int32_t key : D)
            if (key > v2 && !g.in(key, v2)) ++acc.c2;
      }
      return;
    }
    case 3: {  // P3_subgraph_matching (:245-350)
      diff_list(n0, n0e, g, v1, -1, A);
      pair_freq(g, A, freq);
      for (size_t i = 0; i < A.size(); ++i)
        acc.c1 += wrap_mul(count_diff(A, g, A[i], A[i]), freq[i]);
      acc.c2 += bounded_correction(g, A, D, C);
      return;
    }
    case 4: {  // P4_subgraph_matching (:855-963), only v1 < v0
      if (v1 >= v0) return;
      diff_list(n0, n0e, g, v1, -1, A);
      diff_list(n1, n1e, g, v0, -1, B);
      if (A.size() < B.size()) {
        for (int32_t v2 : A)
          for (int32_t key : B) acc.c1 += !g.in(v2, key);
      } else {
        for (int32_t v2 : B)
          for (int32_t key : A) acc.c1 += !g.in(v2, key);
      }
      return;
    }
    case 5: {  // P5_subgraph_matching (:574-734)
      inter_list(n0, n0e, g, v1, -1, A);
      diff_list(n0, n0e, g, v1, -1, B);
      diff_list(n1, n1e, g, v0, -1, C);
      freq.assign(B.size(), 0);
      for (int32_t v2 : A)
        for (size_t j = 0; j < B.size(); ++j)
          if (!g.in(v2, B[j])) ++freq[j];
      for (size_t i = 0; i < B.size(); ++i) {
        if (freq[i] == 0) continue;
        int64_t t = 0;
        for (int32_t key : C) t += !g.in(B[i], key);
        acc.c1 += wrap_mul(t, freq[i]);
      }
      for (int32_t v2 : A) {
        inter_vec(C, g, v2, -1, D);  // list 5
        diff_vec(B, g, v2, -1, E);   // list 4
        for (int32_t c : D)
          for (int32_t key : E) acc.c2 += !g.in(c, key);
      }
      return;
    }
    case 6: {  // P6_subgraph_matching (:736-853)
      inter_list(n0, n0e, g, v1, -1, A);
      diff_list(n1, n1e, g, v0, -1, B);
      for (int32_t v2 : A) {
        diff_vec(A, g, v2, -1, D);  // list 2
        diff_vec(B, g, v2, -1, E);  // list 3
        if (D.size() < E.size()) {
          for (int32_t v3 : D)
            for (int32_t key : E) acc.c1 += !g.in(v3, key);
        } else {
          for (int32_t v3 : E)
            for (int32_t key : D) acc.c1 += !g.in(v3, key);
        }
      }
      return;
    }
    case 7: {  // P7_subgraph_matching (:352-459)
      inter_list(n0, n0e, g, v1, -1, A);
      pair_freq(g, A, freq);
      for (size_t i = 0; i < A.size(); ++i)
        acc.c1 += wrap_mul(count_diff(A, g, A[i], A[i]), freq[i]);
      acc.c2 += bounded_correction(g, A, D, C);
      return;
    }
    case 8: {  // P8_subgraph_matching (:461-572)
      inter_list(n0, n0e, g, v1, -1, A);
      diff_list(n1, n1e, g, v0, -1, B);
      freq.assign(A.size(), 0);
      for (int32_t v4 : B)
        for (size_t j = 0; j < A.size(); ++j)
          if (!g.in(v4, A[j])) ++freq[j];
      for (size_t i = 0; i < A.size(); ++i)
        acc.c1 += wrap_mul(count_inter(A, g, A[i], A[i]), freq[i]);
      for (int32_t v4 : B) {
        diff_vec(A, g, v4, -1, D);
        inter_vec(A, g, v4, -1, C);
        for (int32_t v2 : C)
          for (int32_t key : D)
            if (key > v2 && g.in(key, v2)) ++acc.c2;
      }
      return;
    }
  }
}

// P1_frequency_count (:68-133): per vertex v0, the star count that the
// correction pass is subtracted from.
uint64_t p1_star(const G &g, int32_t v0, std::vector<int64_t> &freq) {
  const int32_t d = g.deg(v0);
  const int32_t *nb = g.b(v0);
  freq.assign(d, 0);
  for (int32_t j = 0; j < d; ++j)
    for (int32_t i = 0; i < d; ++i)
      if (nb[i] < nb[j] && !g.in(nb[j], nb[i])) ++freq[i];
  uint64_t s = 0;
  for (int32_t i = 0; i < d; ++i) {
    const int32_t v2 = nb[i];
    int64_t c = 0;
    for (int32_t x = 0; x < d && nb[x] < v2; ++x) c += !g.in(v2, nb[x]);
    s += wrap_mul(c, freq[i]);
  }
  return s;
}

}  // namespace

extern "C" {

// Reference result of pattern P<pattern> (1..8); counters[1], counters[2]
// are written to c12 when it is non-null.
uint64_t orc_pattern(int64_t n, const int64_t *rowptr, const int32_t *col, int pattern,
                     uint64_t *c12) {
  G g{n, rowptr, col};
  uint64_t c1 = 0, c2 = 0;
#pragma omp parallel reduction(+ : c1, c2)
  {
    V A, B, C, D, E;
    std::vector<int64_t> freq;
    Acc acc;
    // Threads share out single directed edges, not vertices: the hubs of a
    // power-law graph hold most of the work (the sums wrap mod 2^64, so the
    // order of the additions does not change the result).
    if (pattern == 1) {
#pragma omp for schedule(dynamic, 16)
      for (int64_t v0 = 0; v0 < n; ++v0) acc.c1 += p1_star(g, (int32_t)v0, freq);
    }
    const int64_t nnz = rowptr[n];
#pragma omp for schedule(dynamic, 4)
    for (int64_t e = 0; e < nnz; ++e) {
      const int64_t v0 = std::upper_bound(rowptr, rowptr + n + 1, e) - rowptr - 1;
      const int32_t v1 = col[e];
      if (v1 == v0) continue;  // init_edgelist skips self-loops
      edge_pattern(g, pattern, (int32_t)v0, v1, acc, A, B, C, D, E, freq);
    }
    c1 += acc.c1;
    c2 += acc.c2;
  }
  if (c12) {
    c12[0] = c1;
    c12[1] = c2;
  }
  if (pattern == 4 || pattern == 6) return c1;
  return c1 - c2;
}

}  // extern "C"

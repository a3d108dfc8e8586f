// Test infrastructure, not product code: a CPU count of the work the hub
// triangle kernel (mercury_b200/csrc/tc.cu, tc_hub_kernel) schedules on a
// graph, used to check that its scheduling choices do what they claim and to
// reproduce the work figures quoted for RMAT scale 22.
//
// It restates the kernel's task decomposition: owners with d+ > 64 (the leaf
// limit) in tasks of 512 symmetric-row entries; a neighbour y is a partner
// when d+(y) >= 1 and (d+(x) > d+(y) or equal and x > y); a partner of 64+
// entries is dense when the owner keeps a bitmap (degree rank <= the bitmap
// capacity), rank(y) < the core size and the AND over the words below both
// ranks takes at most dense_factor words per list entry; other partners of
// 64+ entries are long, the rest short.
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <numeric>
#include <vector>

namespace {

// Largest j with off[j] <= f (off ascending, off[0] = 0 <= f).
int list_of(const std::vector<int> &off, int f) {
  return (int)(std::upper_bound(off.begin(), off.end(), f) - off.begin()) - 1;
}

// Pair batches of 128 entries: a pair streams for as many batches as its
// longer list needs.
double pair_batches(const std::vector<int> &lists) {
  double b = 0;
  for (size_t i = 0; i < lists.size(); i += 2) {
    int mx = lists[i];
    if (i + 1 < lists.size()) mx = std::max(mx, lists[i + 1]);
    b += (mx + 127) / 128;
  }
  return b;
}

}  // namespace

extern "C" {

// out[0..15]: hub tasks, short lists, short entries, long lists, long
// entries, dense partners, dense probes replaced (their list entries), dense
// words, list steps between interleaved windows, list steps inside
// interleaved windows, list steps of the contiguous ranges (inside plus one
// binary search per warp and task), pair batches in row order, pair batches
// with the length classes, pair batches fully sorted by length, the dense
// AND's (partner, quad) slots as claims of four partners stream them (64
// quads per lane pass, to the claim's longest partner), and the slots of
// the (partner, 32-quad group) pairs below each partner's own end.
void hub_work(int64_t n, const int64_t *rp, const int32_t *ci, int bitmap_bits, int core_ranks,
              int dense_factor, double *out) {
  std::vector<int32_t> deg(n), dp(n), rank(n);
  for (int64_t v = 0; v < n; ++v) deg[v] = (int32_t)(rp[v + 1] - rp[v]);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t v = 0; v < n; ++v) {
    int c = 0;
    for (int64_t e = rp[v]; e < rp[v + 1]; ++e) {
      const int32_t w = ci[e];
      c += deg[w] > deg[v] || (deg[w] == deg[v] && w > v);
    }
    dp[v] = c;
  }
  std::vector<int32_t> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::sort(ord.begin(), ord.end(),
            [&](int a, int b) { return deg[a] != deg[b] ? deg[a] > deg[b] : a > b; });
  for (int64_t i = 0; i < n; ++i) rank[ord[i]] = (int32_t)i;

  constexpr int kChunk = 512, kLong = 64, kWarps = 8, kWin = 128;
  double tasks = 0, ns = 0, ts = 0, nl = 0, tl = 0, nd = 0, dprobe = 0, dword = 0;
  double walk_between = 0, walk_inside = 0, walk_ranges = 0, b_row = 0, b_class = 0, b_sort = 0;
  double dq_claims = 0, dq_own = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : tasks, ns, ts, nl, tl, nd, dprobe, \
    dword, walk_between, walk_inside, walk_ranges, b_row, b_class, b_sort, dq_claims, dq_own)
  for (int64_t x = 0; x < n; ++x) {
    const int px = dp[x];
    if (px <= kLong) continue;
    const int R = rank[x];
    const bool bitmap = R <= bitmap_bits;
    std::vector<int> sl, ll, dq;
    for (int64_t e0 = rp[x]; e0 < rp[x + 1]; e0 += kChunk) {
      tasks += 1;
      sl.clear();
      ll.clear();
      dq.clear();
      const int64_t e1 = std::min(rp[x + 1], e0 + (int64_t)kChunk);
      for (int64_t e = e0; e < e1; ++e) {
        const int y = ci[e], py = dp[y];
        if (!(py >= 1 && (px > py || (px == py && x > y)))) continue;
        if (py >= kLong && bitmap) {
          const int ry = rank[y];
          const int words = (std::min(ry, R) + 31) >> 5;
          if (ry < core_ranks && words <= dense_factor * py) {
            nd += 1;
            dprobe += py;
            dword += words;
            dq.push_back((std::min(ry, R) + 127) >> 7);  // 16-byte quads
            continue;
          }
        }
        if (py >= kLong) ll.push_back(py);
        else sl.push_back(py);
      }
      // Dense partners in claims of four, 64 quads per lane pass.
      for (size_t i = 0; i < dq.size(); i += 4) {
        int mx = 0;
        for (size_t k = i; k < std::min(dq.size(), i + 4); ++k) mx = std::max(mx, dq[k]);
        dq_claims += 4.0 * ((mx + 63) / 64) * 64;
      }
      for (int q : dq) dq_own += ((q + 31) / 32) * 32.0;
      // Long lists: row order, then the two length classes, then sorted.
      nl += ll.size();
      for (int v : ll) tl += v;
      b_row += pair_batches(ll);
      std::vector<int> cls;
      for (int v : ll)
        if (v < 2 * kLong) cls.push_back(v);
      for (int v : ll)
        if (v >= 2 * kLong) cls.push_back(v);
      b_class += pair_batches(cls);
      std::sort(ll.begin(), ll.end());
      b_sort += pair_batches(ll);
      // Short stream: list offsets, then the list steps of both forms.
      ns += sl.size();
      std::vector<int> off(sl.size() + 1, 0);
      for (size_t j = 0; j < sl.size(); ++j) off[j + 1] = off[j] + sl[j];
      const int total = off.back();
      ts += total;
      if (total == 0) continue;
      // Interleaved windows: warp w takes windows w, w + 8, ...; its list
      // pointer j steps to each window's first list, then every lane walks
      // from j to its entry's list (a warp step costs the longest lane walk).
      for (int w = 0; w < kWarps; ++w) {
        int j = 0;
        for (int wb = w * kWin; wb < total; wb += kWarps * kWin) {
          const int jw = list_of(off, wb);
          walk_between += jw - j;
          j = jw;
          std::vector<int> lane(32, j);
          for (int u = 0; u < 4; ++u) {
            int mx = 0;
            for (int l = 0; l < 32; ++l) {
              const int f = wb + u * 32 + l;
              if (f >= total) continue;
              const int lf = list_of(off, f);
              mx = std::max(mx, lf - lane[l]);
              lane[l] = lf;
            }
            walk_inside += mx;
          }
        }
      }
      // Contiguous ranges: warp w takes [lo, hi), an eighth rounded to whole
      // windows; one binary search, then the lanes walk forward.
      const int span = (total + kWarps * kWin - 1) / (kWarps * kWin) * kWin;
      for (int w = 0; w < kWarps; ++w) {
        const int lo = w * span, hi = std::min(total, lo + span);
        if (lo >= hi) continue;
        int steps = 0;
        for (int len = (int)sl.size(); len > 1; len = (len + 1) / 2) ++steps;
        walk_ranges += steps;
        std::vector<int> lane(32, list_of(off, lo));
        for (int wb = lo; wb < hi; wb += kWin)
          for (int u = 0; u < 4; ++u) {
            int mx = 0;
            for (int l = 0; l < 32; ++l) {
              const int f = wb + u * 32 + l;
              if (f >= hi) continue;
              const int lf = list_of(off, f);
              mx = std::max(mx, lf - lane[l]);
              lane[l] = lf;
            }
            walk_ranges += mx;
          }
      }
    }
  }
  const double v[] = {tasks, ns, ts, nl, tl, nd, dprobe, dword, walk_between, walk_inside,
                      walk_ranges, b_row, b_class, b_sort, dq_claims, dq_own};
  for (int i = 0; i < 16; ++i) out[i] = v[i];
}

}  // extern "C"

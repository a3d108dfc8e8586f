// ORACLE -- test infrastructure, not product code.
//
// CPU restatement of the dataset preparation the reference does offline:
// datasets/tsv2mtx.py:13 reads the edge list into a networkx Graph (a set of
// unordered vertex pairs: duplicates and reversed duplicates collapse), and
// the converter (datasets/converter.sh:5) writes that graph as the symmetric
// CSR triple the loader reads (graph.cc:6-35: rows ascending, no self-loops,
// as the loader's contract requires). Restated here as: every pair u != v
// yields the directed entries (u, v) and (v, u); the entries are sorted as
// packed keys u * n + v and made unique; rows and offsets follow.
// Used only by tests/ and by bench.py's CPU baseline of the CSR build.
#include <omp.h>
#include <parallel/algorithm>

#include <algorithm>
#include <cstdint>
#include <vector>

extern "C" {

// src/dst: m pairs of ids in [0, n). rowptr_out: n + 1 entries. col_out: room
// for 2m entries. Returns the entry count, or -1 when an id is out of range.
int64_t orc_csr_build(int64_t n, int64_t m, const int32_t *src, const int32_t *dst,
                      int64_t *rowptr_out, int32_t *col_out) {
  for (int64_t i = 0; i < m; ++i)
    if (src[i] < 0 || src[i] >= n || dst[i] < 0 || dst[i] >= n) return -1;
  std::vector<int64_t> keys(2 * (size_t)m);
  int64_t live = 0;
  {
    std::vector<int64_t> pos(m + 1, 0);
    for (int64_t i = 0; i < m; ++i) pos[i + 1] = pos[i] + (src[i] != dst[i] ? 2 : 0);
    live = pos[m];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) {
      if (src[i] == dst[i]) continue;
      keys[pos[i]] = (int64_t)src[i] * n + dst[i];
      keys[pos[i] + 1] = (int64_t)dst[i] * n + src[i];
    }
  }
  keys.resize(live);
  __gnu_parallel::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  const int64_t nnz = (int64_t)keys.size();
  std::fill(rowptr_out, rowptr_out + n + 1, 0);
  for (int64_t j = 0; j < nnz; ++j) {
    ++rowptr_out[keys[j] / n + 1];
    col_out[j] = (int32_t)(keys[j] % n);
  }
  for (int64_t v = 0; v < n; ++v) rowptr_out[v + 1] += rowptr_out[v];
  return nnz;
}

}  // extern "C"

// Internal declarations shared by the host and device translation units.
#pragma once
#include <cstdint>
#include <vector>
#include "mercury.h"

struct mc_graph {
  int64_t n = 0;
  int64_t nnz = 0;
  int64_t max_degree = 0;
  std::vector<int64_t> rowptr;  // n + 1
  std::vector<int32_t> col;     // nnz
  std::vector<uint8_t> vlabels; // n, or empty (mc_graph_load_vlabels)
};

namespace mc {

// splitmix64 finaliser: the counter-based generator behind every seeded draw,
// so a graph depends only on (seed, draw index) and never on thread timing.
inline uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Builds a sorted, deduplicated, self-loop-free symmetric CSR from undirected
// endpoint pairs (each pair contributes both directions).
int build_symmetric_csr(int64_t n, const std::vector<int32_t> &src,
                        const std::vector<int32_t> &dst, mc_graph *g);

// Raw endpoint draws of the seeded generators (before any symmetrising).
int rmat_draws(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
               int64_t *n_out, std::vector<int32_t> &src, std::vector<int32_t> &dst);
int chung_lu_draws(int64_t n, double gamma, double mean_degree, double max_weight,
                   uint64_t seed, std::vector<int32_t> &src, std::vector<int32_t> &dst);

}  // namespace mc

struct mc_edges {
  int64_t n = 0;  // vertex count (ids in [0, n))
  std::vector<int32_t> src, dst;
};

namespace mc {

}  // namespace mc

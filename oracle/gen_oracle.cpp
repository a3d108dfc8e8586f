// ORACLE -- test infrastructure, not product code.
//
// CPU restatement of the seeded synthetic inputs the benchmarks use (the
// GraphChallenge sets the reference was timed on are not available here):
//  * RMAT: per-level quadrant draws with probabilities (a, b, c, 1-a-b-c),
//    top bit first, from a counter-based splitmix64 stream, so the pair of
//    draw i depends only on (seed, i);
//  * Chung-Lu: expected-degree weights (i+1)^(-1/(gamma-1)) scaled to the
//    mean degree and capped, n*mean/2 endpoint pairs each drawn with
//    probability proportional to the weight.
// The pairs then go through orc_csr_build (csr_oracle.cpp) to the symmetric,
// sorted, deduplicated CSR.  bench.py's CPU arm builds its graph with these,
// so the timed CPU path loads nothing of the product library; the tests check
// that both generators give the library's graphs array for array.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

uint64_t splitmix_fin(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

}  // namespace

extern "C" {

// Writes n * edge_factor pairs (n = 2^scale) into src/dst.  Returns the pair
// count, or -1 for arguments outside the generator's range.
int64_t orc_rmat_draws(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                       int32_t *src, int32_t *dst) {
  if (scale < 1 || scale > 30 || edge_factor < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
    return -1;
  const int64_t pairs = (int64_t(1) << scale) * edge_factor;
  if (!src || !dst) return pairs;
  const double two32 = 4294967296.0;
  const uint64_t cut0 = (uint64_t)(a * two32), cut1 = (uint64_t)((a + b) * two32),
                 cut2 = (uint64_t)((a + b + c) * two32);
  const uint64_t stream = splitmix_fin(seed ^ 0x52D4A7ull);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < pairs; ++i) {
    uint32_t u = 0, v = 0;
    uint64_t word = 0;
    for (int level = 0; level < scale; ++level) {
      // One 64-bit draw serves two levels: low half first, then high half.
      if (level % 2 == 0)
        word = splitmix_fin(stream + (uint64_t)i * 0x1000193ull + (uint64_t)(level / 2));
      const uint64_t r = level % 2 ? (word >> 32) : (word & 0xFFFFFFFFull);
      const uint32_t ub = r >= cut1 ? 1u : 0u;
      const uint32_t vb = (r >= cut0 && r < cut1) || r >= cut2 ? 1u : 0u;
      u = (u << 1) | ub;
      v = (v << 1) | vb;
    }
    src[i] = (int32_t)u;
    dst[i] = (int32_t)v;
  }
  return pairs;
}

// Writes round(n * mean / 2) pairs into src/dst.  Returns the pair count, or
// -1 for arguments outside the generator's range.
int64_t orc_chung_lu_draws(int64_t n, double gamma, double mean_degree, double max_weight,
                           uint64_t seed, int32_t *src, int32_t *dst) {
  if (n < 2 || n > INT32_MAX || gamma <= 1.0 || mean_degree <= 0 || max_weight <= 0) return -1;
  const int64_t pairs = (int64_t)std::llround((double)n * mean_degree / 2.0);
  if (!src || !dst) return pairs;
  const double expo = -1.0 / (gamma - 1.0);
  double raw = 0;
  for (int64_t i = 0; i < n; ++i) raw += std::pow((double)(i + 1), expo);
  const double to_mean = mean_degree * (double)n / raw;
  std::vector<double> cum(n);
  double run = 0;
  for (int64_t i = 0; i < n; ++i) {
    run += std::min(to_mean * std::pow((double)(i + 1), expo), max_weight);
    cum[i] = run;
  }
  const uint64_t stream = splitmix_fin(seed ^ 0xC1u);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < pairs; ++i) {
    const uint64_t r = splitmix_fin(stream + (uint64_t)i);
    const double x0 = (double)(r >> 32) * (1.0 / 4294967296.0) * run;
    const double x1 = (double)(r & 0xFFFFFFFFull) * (1.0 / 4294967296.0) * run;
    const int64_t p = std::upper_bound(cum.begin(), cum.end(), x0) - cum.begin();
    const int64_t q = std::upper_bound(cum.begin(), cum.end(), x1) - cum.begin();
    src[i] = (int32_t)std::min(p, n - 1);
    dst[i] = (int32_t)std::min(q, n - 1);
  }
  return pairs;
}

}  // extern "C"

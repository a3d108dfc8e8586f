// Host CSR graphs: the reference's on-disk format, the input contract check
// and the seeded generators that stand in for the closed dataset converter.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <new>
#include <string>
#include <omp.h>

#include "mc_internal.h"

namespace {

template <typename T>
int read_exact(const std::string &path, std::vector<T> &out, size_t count) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) return MC_ERR_IO;
  try {
    out.resize(count);
  } catch (const std::bad_alloc &) {
    std::fclose(f);
    return MC_ERR_OOM;
  }
  size_t got = count ? std::fread(out.data(), sizeof(T), count, f) : 0;
  std::fclose(f);
  return got == count ? MC_OK : MC_ERR_FORMAT;  // truncated file
}

template <typename T>
int write_exact(const std::string &path, const T *data, size_t count) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) return MC_ERR_IO;
  size_t put = count ? std::fwrite(data, sizeof(T), count, f) : 0;
  int rc = (std::fclose(f) == 0 && put == count) ? MC_OK : MC_ERR_IO;
  return rc;
}

int64_t max_row_degree(const mc_graph *g) {
  int64_t md = 0;
#pragma omp parallel for reduction(max : md) schedule(static)
  for (int64_t v = 0; v < g->n; ++v)
    md = std::max<int64_t>(md, g->rowptr[v + 1] - g->rowptr[v]);
  return md;
}

}  // namespace

namespace mc {

int build_symmetric_csr(int64_t n, const std::vector<int32_t> &src,
                        const std::vector<int32_t> &dst, mc_graph *g) {
  const int64_t pairs = (int64_t)src.size();
  try {
    std::vector<std::atomic<int64_t>> deg(n + 1);
    for (int64_t v = 0; v <= n; ++v) deg[v].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < pairs; ++i) {
      if (src[i] == dst[i]) continue;
      deg[src[i]].fetch_add(1, std::memory_order_relaxed);
      deg[dst[i]].fetch_add(1, std::memory_order_relaxed);
    }
    std::vector<int64_t> start(n + 1, 0);
    for (int64_t v = 0; v < n; ++v)
      start[v + 1] = start[v] + deg[v].load(std::memory_order_relaxed);
    std::vector<int32_t> raw(start[n]);
    std::vector<std::atomic<int64_t>> &fill = deg;  // reuse as cursors
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < n; ++v) fill[v].store(start[v], std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < pairs; ++i) {
      int32_t s = src[i], d = dst[i];
      if (s == d) continue;
      raw[fill[s].fetch_add(1, std::memory_order_relaxed)] = d;
      raw[fill[d].fetch_add(1, std::memory_order_relaxed)] = s;
    }
    std::vector<int64_t> uniq(n + 1, 0);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < n; ++v) {
      int32_t *b = raw.data() + start[v], *e = raw.data() + start[v + 1];
      std::sort(b, e);
      uniq[v] = std::unique(b, e) - b;
    }
    g->n = n;
    g->rowptr.assign(n + 1, 0);
    for (int64_t v = 0; v < n; ++v) g->rowptr[v + 1] = g->rowptr[v] + uniq[v];
    g->nnz = g->rowptr[n];
    g->col.resize(g->nnz);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < n; ++v)
      std::memcpy(g->col.data() + g->rowptr[v], raw.data() + start[v],
                  sizeof(int32_t) * uniq[v]);
    g->max_degree = max_row_degree(g);
  } catch (const std::bad_alloc &) {
    return MC_ERR_OOM;
  }
  return MC_OK;
}


int rmat_draws(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
               int64_t *n_out, std::vector<int32_t> &src, std::vector<int32_t> &dst) {
  if (scale < 1 || scale > 30 || edge_factor < 1) return MC_ERR_ARG;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return MC_ERR_ARG;
  const int64_t n = int64_t(1) << scale;
  const int64_t draws = n * edge_factor;
  // Quadrant thresholds on a 32-bit uniform: [0,a) -> (0,0), [a,a+b) -> (0,1),
  // [a+b,a+b+c) -> (1,0), rest -> (1,1) for (src bit, dst bit), top bit first.
  const double s32 = 4294967296.0;
  const uint64_t ta = (uint64_t)(a * s32), tb = (uint64_t)((a + b) * s32),
                 tc = (uint64_t)((a + b + c) * s32);
  try {
    src.resize(draws);
    dst.resize(draws);
  } catch (const std::bad_alloc &) {
    return MC_ERR_OOM;
  }
  const uint64_t key = mix64(seed ^ 0x52D4A7ull);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < draws; ++i) {
    uint32_t s = 0, d = 0;
    uint64_t bits = 0;
    for (int l = 0; l < scale; ++l) {
      if ((l & 1) == 0) bits = mix64(key + (uint64_t)i * 0x1000193ull + (uint64_t)(l >> 1));
      uint64_t r = (l & 1) ? (bits >> 32) : (bits & 0xFFFFFFFFull);
      uint32_t sb = 0, db = 0;
      if (r < ta) { sb = 0; db = 0; }
      else if (r < tb) { sb = 0; db = 1; }
      else if (r < tc) { sb = 1; db = 0; }
      else { sb = 1; db = 1; }
      s = (s << 1) | sb;
      d = (d << 1) | db;
    }
    src[i] = (int32_t)s;
    dst[i] = (int32_t)d;
  }
  *n_out = n;
  return MC_OK;
}

int chung_lu_draws(int64_t n, double gamma, double mean_degree, double max_weight,
                   uint64_t seed, std::vector<int32_t> &src, std::vector<int32_t> &dst) {
  if (n < 2 || n > INT32_MAX || gamma <= 1.0 || mean_degree <= 0 || max_weight <= 0)
    return MC_ERR_ARG;
  std::vector<double> cdf;
  const int64_t pairs = (int64_t)std::llround((double)n * mean_degree / 2.0);
  try {
    cdf.resize(n);
    src.resize(pairs);
    dst.resize(pairs);
  } catch (const std::bad_alloc &) {
    return MC_ERR_OOM;
  }
  // Expected-degree weights w_i = (i+1)^(-1/(gamma-1)), scaled to the mean,
  // then capped.
  const double expo = -1.0 / (gamma - 1.0);
  double sum = 0;
  for (int64_t i = 0; i < n; ++i) sum += std::pow((double)(i + 1), expo);
  const double scale = mean_degree * (double)n / sum;
  double acc = 0;
  for (int64_t i = 0; i < n; ++i) {
    double w = std::min(scale * std::pow((double)(i + 1), expo), max_weight);
    acc += w;
    cdf[i] = acc;
  }
  const double total = acc;
  const uint64_t key = mix64(seed ^ 0xC1u);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < pairs; ++i) {
    uint64_t r = mix64(key + (uint64_t)i);
    double u0 = (double)(r >> 32) * (1.0 / 4294967296.0) * total;
    double u1 = (double)(r & 0xFFFFFFFFull) * (1.0 / 4294967296.0) * total;
    src[i] = (int32_t)(std::upper_bound(cdf.begin(), cdf.end(), u0) - cdf.begin());
    dst[i] = (int32_t)(std::upper_bound(cdf.begin(), cdf.end(), u1) - cdf.begin());
    if (src[i] >= n) src[i] = (int32_t)(n - 1);
    if (dst[i] >= n) dst[i] = (int32_t)(n - 1);
  }
  return MC_OK;
}

}  // namespace mc

namespace {
int finish_generated(int64_t n, const std::vector<int32_t> &src, const std::vector<int32_t> &dst,
                     mc_graph_t **out) {
  mc_graph *g = new (std::nothrow) mc_graph();
  if (!g) return MC_ERR_OOM;
  int rc = mc::build_symmetric_csr(n, src, dst, g);
  if (rc != MC_OK) {
    delete g;
    return rc;
  }
  *out = g;
  return MC_OK;
}
}  // namespace

extern "C" {

int mc_graph_load(const char *prefix, mc_graph_t **out) {
  if (!prefix || !out) return MC_ERR_ARG;
  *out = nullptr;
  std::string p(prefix);
  std::ifstream meta(p + ".meta.txt");
  if (!meta) return MC_ERR_IO;
  long long nv = 0, ne = 0, vid_size = 0, eid_size = 0, vl = 0, el = 0, md = 0,
            feat = 0, nvc = 0, nec = 0;
  meta >> nv >> ne >> vid_size >> eid_size >> vl >> el >> md >> feat >> nvc >> nec;
  if (!meta) return MC_ERR_FORMAT;
  // The reference asserts these (graph.cc:24-28).
  if (vid_size != 4 || eid_size != 8 || vl != 1 || el != 2) return MC_ERR_FORMAT;
  if (!(md > 0 && md < nv)) return MC_ERR_FORMAT;
  if (nv <= 0 || nv > INT32_MAX || ne < 0) return MC_ERR_FORMAT;
  mc_graph *g = new (std::nothrow) mc_graph();
  if (!g) return MC_ERR_OOM;
  int rc = read_exact(p + ".vertex.bin", g->rowptr, (size_t)nv + 1);
  if (rc == MC_OK) rc = read_exact(p + ".edge.bin", g->col, (size_t)ne);
  if (rc == MC_OK && (g->rowptr[0] != 0 || g->rowptr[nv] != ne)) rc = MC_ERR_FORMAT;
  if (rc != MC_OK) {
    delete g;
    return rc;
  }
  g->n = nv;
  g->nnz = ne;
  g->max_degree = md;
  *out = g;
  return MC_OK;
}

int mc_graph_write(const mc_graph_t *g, const char *prefix) {
  if (!g || !prefix) return MC_ERR_ARG;
  std::string p(prefix);
  FILE *f = std::fopen((p + ".meta.txt").c_str(), "w");
  if (!f) return MC_ERR_IO;
  // nv ne vid_size eid_size vlabel_size elabel_size max_degree feat_len
  // n_vclasses n_eclasses -- the field order graph.cc:22-23 reads.
  std::fprintf(f, "%lld %lld 4 8 1 2 %lld 0 0 0\n", (long long)g->n,
               (long long)g->nnz, (long long)g->max_degree);
  if (std::fclose(f) != 0) return MC_ERR_IO;
  int rc = write_exact(p + ".vertex.bin", g->rowptr.data(), g->rowptr.size());
  if (rc == MC_OK) rc = write_exact(p + ".edge.bin", g->col.data(), g->col.size());
  return rc;
}

int mc_graph_load_vlabels(mc_graph_t *g, const char *prefix) {
  if (!g || !prefix) return MC_ERR_ARG;
  const std::string path = std::string(prefix) + ".vlabel.bin";
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) return MC_ERR_IO;
  std::fseek(f, 0, SEEK_END);
  const long size = std::ftell(f);
  std::fclose(f);
  if (size != (long)g->n) return MC_ERR_FORMAT;  // one uint8 per vertex
  std::vector<uint8_t> labels;
  try {
    const int rc = read_exact(path, labels, (size_t)g->n);
    if (rc != MC_OK) return rc;
  } catch (const std::bad_alloc &) {
    return MC_ERR_OOM;
  }
  g->vlabels.swap(labels);
  return MC_OK;
}

int mc_graph_vlabels(const mc_graph_t *g, const uint8_t **labels) {
  if (!g || !labels) return MC_ERR_ARG;
  *labels = g->vlabels.empty() ? nullptr : g->vlabels.data();
  return MC_OK;
}

int mc_graph_from_csr(const int64_t *rowptr, const int32_t *col, int64_t n,
                      int64_t nnz, mc_graph_t **out) {
  if (!out || n < 0 || nnz < 0 || !rowptr || (nnz > 0 && !col)) return MC_ERR_ARG;
  if (n > INT32_MAX) return MC_ERR_UNSUPPORTED;
  *out = nullptr;
  mc_graph *g = new (std::nothrow) mc_graph();
  if (!g) return MC_ERR_OOM;
  try {
    g->rowptr.assign(rowptr, rowptr + n + 1);
    g->col.assign(col, col + nnz);
  } catch (const std::bad_alloc &) {
    delete g;
    return MC_ERR_OOM;
  }
  g->n = n;
  g->nnz = nnz;
  if (g->rowptr[0] != 0 || g->rowptr[n] != nnz) {
    delete g;
    return MC_ERR_FORMAT;
  }
  for (int64_t v = 0; v < n; ++v)
    if (g->rowptr[v + 1] < g->rowptr[v]) {
      delete g;
      return MC_ERR_FORMAT;
    }
  g->max_degree = max_row_degree(g);
  *out = g;
  return MC_OK;
}

int mc_graph_info(const mc_graph_t *g, int64_t *n, int64_t *nnz, int64_t *max_degree) {
  if (!g) return MC_ERR_ARG;
  if (n) *n = g->n;
  if (nnz) *nnz = g->nnz;
  if (max_degree) *max_degree = g->max_degree;
  return MC_OK;
}

const int64_t *mc_graph_rowptr(const mc_graph_t *g) { return g ? g->rowptr.data() : nullptr; }
const int32_t *mc_graph_col(const mc_graph_t *g) { return g ? g->col.data() : nullptr; }

int mc_graph_validate(const mc_graph_t *g, int check_symmetry) {
  if (!g) return MC_ERR_ARG;
  const int64_t n = g->n;
  if ((int64_t)g->rowptr.size() != n + 1 || g->rowptr[0] != 0 || g->rowptr[n] != g->nnz)
    return MC_ERR_FORMAT;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(| : bad)
  for (int64_t v = 0; v < n; ++v) {
    int64_t b = g->rowptr[v], e = g->rowptr[v + 1];
    if (e < b || e > g->nnz) { bad |= 1; continue; }
    for (int64_t i = b; i < e; ++i) {
      int32_t u = g->col[i];
      if (u < 0 || u >= n || u == v || (i > b && g->col[i - 1] >= u)) bad |= 1;
      else if (check_symmetry) {
        const int32_t *rb = g->col.data() + g->rowptr[u], *re = g->col.data() + g->rowptr[u + 1];
        if (!std::binary_search(rb, re, (int32_t)v)) bad |= 1;
      }
    }
  }
  return bad ? MC_ERR_FORMAT : MC_OK;
}

void mc_graph_free(mc_graph_t *g) { delete g; }

int mc_gen_rmat(int scale, int edge_factor, double a, double b, double c,
                uint64_t seed, mc_graph_t **out) {
  if (!out) return MC_ERR_ARG;
  *out = nullptr;
  std::vector<int32_t> src, dst;
  int64_t n = 0;
  int rc = mc::rmat_draws(scale, edge_factor, a, b, c, seed, &n, src, dst);
  if (rc != MC_OK) return rc;
  return finish_generated(n, src, dst, out);
}

int mc_gen_chung_lu(int64_t n, double gamma, double mean_degree, double max_weight,
                    uint64_t seed, mc_graph_t **out) {
  if (!out) return MC_ERR_ARG;
  *out = nullptr;
  std::vector<int32_t> src, dst;
  int rc = mc::chung_lu_draws(n, gamma, mean_degree, max_weight, seed, src, dst);
  if (rc != MC_OK) return rc;
  return finish_generated(n, src, dst, out);
}

}  // extern "C"

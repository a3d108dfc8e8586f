// Edge-list input: the text formats the reference's dataset preparation
// reads (Matrix Market for datasets/converter.sh:5, GraphChallenge TSV for
// datasets/tsv2mtx.py:10), SNAP edge lists, and the seeded generators' raw
// draws.  Parsing runs on the host over a memory-mapped file, split into
// newline-aligned chunks parsed by OpenMP threads; the CSR itself is built on
// the device (build.cu).
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <climits>
#include <cstring>
#include <new>
#include <string>
#include <vector>
#include <omp.h>

#include "mc_internal.h"

namespace {

// Largest id accepted after the base shift: handles take n <= INT32_MAX - 1.
constexpr int64_t kMaxVertexId = (int64_t)INT32_MAX - 2;

struct Mapped {
  const char *p = nullptr;
  size_t size = 0;
  int fd = -1;
  ~Mapped() {
    if (p && size) munmap(const_cast<char *>(p), size);
    if (fd >= 0) close(fd);
  }
};

int map_file(const char *path, Mapped &m) {
  m.fd = open(path, O_RDONLY);
  if (m.fd < 0) return MC_ERR_IO;
  struct stat st;
  if (fstat(m.fd, &st) != 0) return MC_ERR_IO;
  m.size = (size_t)st.st_size;
  if (m.size == 0) return MC_OK;
  void *p = mmap(nullptr, m.size, PROT_READ, MAP_PRIVATE, m.fd, 0);
  if (p == MAP_FAILED) {
    m.size = 0;
    return MC_ERR_IO;
  }
  madvise(p, m.size, MADV_SEQUENTIAL);
  m.p = static_cast<const char *>(p);
  return MC_OK;
}

inline bool is_blank(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// One unsigned decimal field at p; false when the field is not a plain
// non-negative integer (a sign, a fraction, an exponent) or exceeds 2^62.
inline bool parse_field(const char *&p, const char *end, int64_t &v) {
  while (p < end && is_blank(*p)) ++p;
  if (p >= end || *p < '0' || *p > '9') return false;
  constexpr int64_t kMax = int64_t(1) << 62;
  int64_t x = 0;
  while (p < end && *p >= '0' && *p <= '9') {
    const int64_t d = *p - '0';
    if (x > (kMax - d) / 10) return false;  // x * 10 + d would exceed 2^62
    x = x * 10 + d;
    ++p;
  }
  if (p < end && !is_blank(*p) && *p != '\n') return false;
  v = x;
  return true;
}

// Line kinds of the body of every format.
enum LineKind { kSkip, kPair, kBad };

// Reads the line starting at p (advancing p past its newline): blank lines
// and lines whose first non-blank character is '%' or '#' are skipped; a
// data line yields its first two fields (any further fields, such as an MTX
// value or a TSV weight, are ignored).
inline LineKind parse_line(const char *&p, const char *end, int64_t &a, int64_t &b) {
  const char *q = p;
  while (q < end && is_blank(*q)) ++q;
  const char *eol = static_cast<const char *>(std::memchr(q, '\n', (size_t)(end - q)));
  if (!eol) eol = end;
  LineKind kind;
  if (q == eol || *q == '%' || *q == '#') {
    kind = kSkip;
  } else {
    const char *r = q;
    kind = (parse_field(r, eol, a) && parse_field(r, eol, b)) ? kPair : kBad;
  }
  p = eol < end ? eol + 1 : end;
  return kind;
}

struct Chunk {
  std::vector<int32_t> src, dst;
  int64_t max_id = -1;
  int64_t lines = 0;
  int status = MC_OK;
};

// Parses [begin, end) into per-thread chunks split at line boundaries and
// concatenates them in file order.
int parse_body(const char *begin, const char *end, int64_t base, mc_edges &e,
               int64_t *max_id, int64_t *lines) {
  const size_t len = (size_t)(end - begin);
  int threads = std::max(1, omp_get_max_threads());
  if (len < (size_t)1 << 20) threads = 1;
  std::vector<const char *> cut(threads + 1);
  cut[0] = begin;
  cut[threads] = end;
  for (int t = 1; t < threads; ++t) {
    const char *c = begin + len / threads * t;
    if (c < cut[t - 1]) c = cut[t - 1];
    const char *nl = static_cast<const char *>(std::memchr(c, '\n', (size_t)(end - c)));
    cut[t] = nl ? nl + 1 : end;
  }
  std::vector<Chunk> parts(threads);
#pragma omp parallel for num_threads(threads) schedule(static, 1)
  for (int t = 0; t < threads; ++t) {
    Chunk &ck = parts[t];
    const char *p = cut[t], *q = cut[t + 1];
    try {
      ck.src.reserve((size_t)(q - p) / 8);
      ck.dst.reserve((size_t)(q - p) / 8);
      while (p < q) {
        int64_t a = 0, b = 0;
        LineKind k = parse_line(p, q, a, b);
        if (k == kSkip) continue;
        if (k == kBad || a < base || b < base) {
          ck.status = MC_ERR_FORMAT;
          break;
        }
        a -= base;
        b -= base;
        if (a > kMaxVertexId || b > kMaxVertexId) {
          ck.status = MC_ERR_UNSUPPORTED;
          break;
        }
        ck.src.push_back((int32_t)a);
        ck.dst.push_back((int32_t)b);
        ck.max_id = std::max(ck.max_id, std::max(a, b));
        ++ck.lines;
      }
    } catch (const std::bad_alloc &) {
      ck.status = MC_ERR_OOM;
    }
  }
  int64_t total = 0, mx = -1;
  for (const Chunk &ck : parts) {
    if (ck.status != MC_OK) return ck.status;
    total += (int64_t)ck.src.size();
    mx = std::max(mx, ck.max_id);
  }
  try {
    e.src.resize(total);
    e.dst.resize(total);
  } catch (const std::bad_alloc &) {
    return MC_ERR_OOM;
  }
  std::vector<int64_t> off(threads + 1, 0);
  for (int t = 0; t < threads; ++t) off[t + 1] = off[t] + (int64_t)parts[t].src.size();
#pragma omp parallel for num_threads(threads) schedule(static, 1)
  for (int t = 0; t < threads; ++t) {
    std::copy(parts[t].src.begin(), parts[t].src.end(), e.src.begin() + off[t]);
    std::copy(parts[t].dst.begin(), parts[t].dst.end(), e.dst.begin() + off[t]);
  }
  *max_id = mx;
  *lines = total;
  return MC_OK;
}

bool starts_with_nocase(const char *p, const char *end, const char *word) {
  for (; *word; ++word, ++p)
    if (p >= end || std::tolower((unsigned char)*p) != std::tolower((unsigned char)*word))
      return false;
  return true;
}

// Matrix Market: the banner line, then '%' comments, then the size line
// "rows cols entries"; *body points past the size line.
int parse_mtx_header(const char *p, const char *end, const char **body, int64_t *rows,
                     int64_t *cols, int64_t *entries) {
  if (!starts_with_nocase(p, end, "%%MatrixMarket")) return MC_ERR_FORMAT;
  const char *eol = static_cast<const char *>(std::memchr(p, '\n', (size_t)(end - p)));
  if (!eol) return MC_ERR_FORMAT;
  std::string banner(p, eol);
  for (char &c : banner) c = (char)std::tolower((unsigned char)c);
  if (banner.find("array") != std::string::npos) return MC_ERR_UNSUPPORTED;
  if (banner.find("coordinate") == std::string::npos) return MC_ERR_FORMAT;
  p = eol + 1;
  while (p < end) {
    const char *q = p;
    while (q < end && is_blank(*q)) ++q;
    const char *e2 = static_cast<const char *>(std::memchr(q, '\n', (size_t)(end - q)));
    if (!e2) e2 = end;
    if (q == e2 || *q == '%') {
      p = e2 < end ? e2 + 1 : end;
      continue;
    }
    const char *r = q;
    if (!parse_field(r, e2, *rows) || !parse_field(r, e2, *cols) || !parse_field(r, e2, *entries))
      return MC_ERR_FORMAT;
    *body = e2 < end ? e2 + 1 : end;
    return MC_OK;
  }
  return MC_ERR_FORMAT;  // no size line
}

int adopt(mc_edges *e, mc_edges_t **out) {
  *out = e;
  return MC_OK;
}

}  // namespace

extern "C" {

int mc_edges_load(const char *path, int format, int id_base, mc_edges_t **out) {
  if (!path || !out) return MC_ERR_ARG;
  *out = nullptr;
  if (format != MC_EDGES_MTX && format != MC_EDGES_TSV && format != MC_EDGES_SNAP)
    return MC_ERR_ARG;
  if (id_base > 1) return MC_ERR_ARG;
  const int64_t base = id_base >= 0 ? id_base : (format == MC_EDGES_SNAP ? 0 : 1);
  Mapped m;
  int rc = map_file(path, m);
  if (rc != MC_OK) return rc;
  const char *p = m.p, *end = m.p + m.size;
  mc_edges *e = new (std::nothrow) mc_edges();
  if (!e) return MC_ERR_OOM;
  int64_t rows = 0, cols = 0, entries = -1;
  if (format == MC_EDGES_MTX) {
    if (m.size == 0) rc = MC_ERR_FORMAT;
    else rc = parse_mtx_header(p, end, &p, &rows, &cols, &entries);
    if (rc == MC_OK && (rows > kMaxVertexId + 1 || cols > kMaxVertexId + 1))
      rc = MC_ERR_UNSUPPORTED;
  }
  int64_t max_id = -1, lines = 0;
  if (rc == MC_OK && p < end) rc = parse_body(p, end, base, *e, &max_id, &lines);
  if (rc == MC_OK && entries >= 0 && lines != entries) rc = MC_ERR_FORMAT;
  if (rc != MC_OK) {
    delete e;
    return rc;
  }
  e->n = std::max(std::max(rows, cols), max_id + 1);
  return adopt(e, out);
}

int mc_edges_from_arrays(const int32_t *src, const int32_t *dst, int64_t num_edges, int64_t n,
                         mc_edges_t **out) {
  if (!out || num_edges < 0 || n < 0 || (num_edges > 0 && (!src || !dst))) return MC_ERR_ARG;
  *out = nullptr;
  if (n > kMaxVertexId + 1) return MC_ERR_UNSUPPORTED;
  mc_edges *e = new (std::nothrow) mc_edges();
  if (!e) return MC_ERR_OOM;
  try {
    e->src.assign(src, src + num_edges);
    e->dst.assign(dst, dst + num_edges);
  } catch (const std::bad_alloc &) {
    delete e;
    return MC_ERR_OOM;
  }
  e->n = n;
  return adopt(e, out);
}

int mc_edges_info(const mc_edges_t *e, int64_t *num_edges, int64_t *n) {
  if (!e) return MC_ERR_ARG;
  if (num_edges) *num_edges = (int64_t)e->src.size();
  if (n) *n = e->n;
  return MC_OK;
}

const int32_t *mc_edges_src(const mc_edges_t *e) { return e ? e->src.data() : nullptr; }
const int32_t *mc_edges_dst(const mc_edges_t *e) { return e ? e->dst.data() : nullptr; }
void mc_edges_free(mc_edges_t *e) { delete e; }

int mc_gen_rmat_edges(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                      mc_edges_t **out) {
  if (!out) return MC_ERR_ARG;
  *out = nullptr;
  mc_edges *e = new (std::nothrow) mc_edges();
  if (!e) return MC_ERR_OOM;
  int rc = mc::rmat_draws(scale, edge_factor, a, b, c, seed, &e->n, e->src, e->dst);
  if (rc != MC_OK) {
    delete e;
    return rc;
  }
  return adopt(e, out);
}

int mc_gen_chung_lu_edges(int64_t n, double gamma, double mean_degree, double max_weight,
                          uint64_t seed, mc_edges_t **out) {
  if (!out) return MC_ERR_ARG;
  *out = nullptr;
  mc_edges *e = new (std::nothrow) mc_edges();
  if (!e) return MC_ERR_OOM;
  int rc = mc::chung_lu_draws(n, gamma, mean_degree, max_weight, seed, e->src, e->dst);
  if (rc != MC_OK) {
    delete e;
    return rc;
  }
  e->n = n;
  return adopt(e, out);
}

}  // extern "C"

// C ABI of the device graph handle and the triangle-count entry points.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <new>

#include "dgraph.cuh"
#include "device_common.cuh"
#include "scan.cuh"

namespace mc {

namespace {
thread_local cudaError_t t_last_cuda = cudaSuccess;

double elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) return 0.0;
  return (double)ms;
}

void release(mc_dgraph *g) {
  if (!g) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(g->device);
  void *bufs[] = {g->rowptr,     g->col,        g->key,      g->dag_rowptr,
                  g->dag_col,    g->keep,       g->tile_counts, g->tile_offsets,
                  g->hub_cnt,    g->leaf_cnt,   g->hub_off,  g->leaf_off,  g->hub_tasks,
                  g->leaf_tasks, g->scan_temp,  g->counters, g->err, g->pat_scratch,
                  g->mega_cnt,   g->mega_off,   g->mega_tasks, g->rank,
                  g->dag_rank,   g->rank_keys,  g->rank_counts, g->rank_offsets,
                  g->center_scratch, g->stage, g->chunk_offsets, g->core_bits, g->pinfo,
                  g->hop_scratch, g->hub_bits, g->vlabels, g->tile_rows};
  if (g->col_host) bufs[1] = nullptr;  // pinned host memory, freed below
  if (g->dag_host)  // DAG entries and ranks: pinned host memory, freed below
    for (void *&p : bufs)
      if (p == g->dag_col || p == g->dag_rank) p = nullptr;
  // Stream-ordered frees: no device-wide synchronisation, so other handles'
  // work keeps running while this one is released.
  for (void *p : bufs)
    if (p) dev_free(p, g->stream);
  if (g->stream) cudaStreamSynchronize(g->stream);
  if (g->col_host && g->col_h) cudaFreeHost(g->col_h);
  if (g->dag_col_h) cudaFreeHost(g->dag_col_h);
  if (g->dag_rank_h) cudaFreeHost(g->dag_rank_h);
  delete[] g->h_counters;
  for (cudaEvent_t e : g->ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : g->stage_ev)
    if (e) cudaEventDestroy(e);
  if (g->copy_stream) cudaStreamDestroy(g->copy_stream);
  if (g->own_stream && g->stream) cudaStreamDestroy(g->stream);
  if (prev >= 0) cudaSetDevice(prev);
  delete g;
}

// Free device memory for the placement decision: what the driver reports
// plus what this process's pool holds unused. MERCURY_DEVICE_BYTES replaces
// the figure (tests reach the host-column fallback with it on small graphs).
int device_bytes_available(int device, int64_t *avail) {
  size_t free_b = 0, total_b = 0;
  MC_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
  int64_t a = (int64_t)free_b;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t reserved = 0, used = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess &&
        reserved > used)
      a += (int64_t)(reserved - used);
  }
  if (const char *env = std::getenv("MERCURY_DEVICE_BYTES")) {
    const long long v = std::atoll(env);
    if (v > 0) a = v;
  }
  *avail = a;
  return MC_OK;
}

// Where a graph's column array goes. In device memory when the device can
// hold it together with the triangle-count scratch (and a margin);
// otherwise, or when the caller asks, in pinned host memory that the
// kernels read through the device's mapping of it.
constexpr int64_t kPlacementMargin = 256ll << 20;
constexpr unsigned kDeviceColumns = 0x80000000u;  // internal: skip the decision
// The DAG goes to host memory too (dag_host) when asked, or when the device
// cannot hold it even with the columns on the host.
int columns_on_host(int device, int64_t n, int64_t nnz, unsigned flags, bool *host,
                    bool *dag_host = nullptr) {
  const bool want_dag = (flags & MC_HOST_DAG) != 0;
  *host = want_dag || (flags & MC_HOST_COLUMNS) != 0;
  if (dag_host) *dag_host = want_dag;
  if (want_dag || nnz == 0 || (flags & kDeviceColumns)) return MC_OK;
  // MERCURY_PLACEMENT=columns / dag forces the automatic choice (benchmarks
  // of the host placements use it).
  if (const char *env = std::getenv("MERCURY_PLACEMENT")) {
    if (std::strcmp(env, "columns") == 0 || std::strcmp(env, "dag") == 0) {
      *host = true;
      if (dag_host) *dag_host = std::strcmp(env, "dag") == 0;
      return MC_OK;
    }
  }
  int64_t avail = 0;
  const int rc = device_bytes_available(device, &avail);
  if (rc != MC_OK) return rc;
  const int64_t in_core = 8 * (n + 1) + 4 * nnz + tc_device_bytes(n, nnz, false);
  if (!*host) *host = in_core + kPlacementMargin > avail;
  if (*host && dag_host) {
    const int64_t with_dag = 8 * (n + 1) + tc_device_bytes(n, nnz, true, false);
    *dag_host = with_dag + kPlacementMargin > avail;
  }
  return MC_OK;
}

// Host-to-pinned copy of a large column array, split over the host threads.
void copy_to_pinned(int32_t *dst, const int32_t *src, int64_t count) {
  constexpr int64_t kPiece = 1 << 22;  // 16 MB of entries per piece
  const int64_t pieces = (count + kPiece - 1) / kPiece;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < pieces; ++p) {
    const int64_t a = p * kPiece, b = std::min(count, a + kPiece);
    std::memcpy(dst + a, src + a, sizeof(int32_t) * (size_t)(b - a));
  }
}

int create_common(int64_t n, int64_t nnz, void *stream, mc_dgraph **out, mc_dgraph **gp,
                  unsigned flags = 0) {
  if (!out || n < 0 || nnz < 0) return MC_ERR_ARG;
  if (n > INT32_MAX - 1) return MC_ERR_UNSUPPORTED;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MC_ERR_NO_DEVICE;
  mc_dgraph *g = new (std::nothrow) mc_dgraph();
  if (!g) return MC_ERR_OOM;
  *gp = g;
  MC_CUDA_TRY(cudaGetDevice(&g->device));
  MC_CUDA_TRY(cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, g->device));
  retain_pool_memory(g->device);
  if (stream) {
    g->stream = static_cast<cudaStream_t>(stream);
  } else {
    MC_CUDA_TRY(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    g->own_stream = true;
  }
  g->n = n;
  g->nnz = nnz;
  MC_CUDA_TRY(dev_alloc((void **)&g->rowptr, sizeof(int64_t) * (size_t)(n + 1), g->stream));
  const int rc = columns_on_host(g->device, n, nnz, flags, &g->col_host, &g->dag_host);
  if (rc != MC_OK) return rc;
  const size_t col_bytes = sizeof(int32_t) * (size_t)std::max<int64_t>(nnz, 1);
  if (g->col_host) {
    MC_CUDA_TRY(cudaHostAlloc((void **)&g->col_h, col_bytes, cudaHostAllocMapped));
    MC_CUDA_TRY(cudaHostGetDevicePointer((void **)&g->col, g->col_h, 0));
  } else {
    MC_CUDA_TRY(dev_alloc((void **)&g->col, col_bytes, g->stream));
  }
  MC_CUDA_TRY(dev_alloc((void **)&g->counters, sizeof(unsigned long long) * 8, g->stream));
  MC_CUDA_TRY(dev_alloc((void **)&g->err, sizeof(unsigned), g->stream));
  // Host mirror of the counters (read after a stream synchronisation).
  g->h_counters = new (std::nothrow) unsigned long long[16]();
  if (!g->h_counters) return MC_ERR_OOM;
  g->h_err = reinterpret_cast<unsigned *>(g->h_counters + 8);
  for (cudaEvent_t &e : g->ev) MC_CUDA_TRY(cudaEventCreate(&e));
  return MC_OK;
}

int finish_create(mc_dgraph *g, unsigned flags, mc_dgraph **out, int rc) {
  if (rc == MC_OK) rc = validate_graph(g, flags);
  if (rc != MC_OK) {
    release(g);
    return rc;
  }
  *out = g;
  return MC_OK;
}

// Per-thread cache for the one-shot entry point: the handle is kept and its
// buffers reused while later graphs fit in its capacity.
struct HostCache {
  mc_dgraph *g = nullptr;
  int64_t cap_n = -1, cap_nnz = -1;
  // Pinned staging for callers that pass pageable arrays: two column slots
  // of one upload chunk each, and the row offsets.
  int32_t *pin_col[2] = {nullptr, nullptr};
  int64_t pin_col_entries = 0;
  int64_t *pin_rowptr = nullptr;
  int64_t pin_rowptr_entries = 0;
  cudaEvent_t pin_done[2] = {nullptr, nullptr};
  void drop_pins() {
    for (auto &p : pin_col) {
      if (p) cudaFreeHost(p);
      p = nullptr;
    }
    if (pin_rowptr) cudaFreeHost(pin_rowptr);
    pin_rowptr = nullptr;
    pin_col_entries = pin_rowptr_entries = 0;
    for (auto &e : pin_done) {
      if (e) cudaEventDestroy(e);
      e = nullptr;
    }
  }
  ~HostCache() {
    release(g);
    drop_pins();
  }
};

bool is_pageable(const void *p) {
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeUnregistered;
}
thread_local HostCache t_cache;

}  // namespace

void set_last_cuda_error(cudaError_t e) { t_last_cuda = e; }
cudaError_t last_cuda_error() { return t_last_cuda; }

void retain_pool_memory(int device) {
  static std::atomic<unsigned long long> done{0};  // one bit per device (first 64)
  const unsigned long long bit = device < 64 ? 1ull << device : 0ull;
  if (bit && (done.load(std::memory_order_relaxed) & bit)) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  done.fetch_or(bit, std::memory_order_relaxed);
}

int tc_stats(mc_dgraph *g, mc_tc_stats_t *st) {
  std::memset(st, 0, sizeof(*st));
  st->n = g->n;
  st->nnz = g->nnz;
  if (!g->tc_ready || g->n == 0) return MC_OK;
  int64_t v[4] = {0, 0, 0, 0};
  const int64_t *src[4] = {g->dag_rowptr + g->n, g->hub_off + g->n, g->leaf_off + g->n,
                           g->mega_off + g->n};
  for (int i = 0; i < 4; ++i)
    MC_CUDA_TRY(cudaMemcpyAsync(&v[i], src[i], sizeof(int64_t), cudaMemcpyDeviceToHost, g->stream));
  unsigned long long maxd = 0;
  MC_CUDA_TRY(cudaMemcpyAsync(&maxd, g->counters + 3, sizeof(maxd), cudaMemcpyDeviceToHost,
                              g->stream));
  MC_CUDA_TRY(cudaStreamSynchronize(g->stream));
  unsigned long long pe = 0, work = 0;
  const int rc = tc_partner_stats(g, &pe, &work);
  if (rc != MC_OK) return rc;
  st->dag_edges = v[0];
  st->hub_tasks = v[1] + v[3];  // both table-size classes
  st->leaf_tasks = v[2];
  st->partner_edges = (int64_t)pe;
  st->max_out_degree = (int64_t)maxd;
  st->probe_work = (double)work;
  return MC_OK;
}

}  // namespace mc

using mc::release;

extern "C" {

const char *mc_strerror(int status) {
  switch (status) {
    case MC_OK: return "ok";
    case MC_ERR_ARG: return "invalid argument";
    case MC_ERR_IO: return "file could not be opened, read or written";
    case MC_ERR_FORMAT: return "input breaks the CSR contract";
    case MC_ERR_OOM: return "out of host or device memory";
    case MC_ERR_CUDA: return "CUDA runtime error";
    case MC_ERR_DEVICE: return "a kernel raised its error flag";
    case MC_ERR_UNSUPPORTED: return "size beyond a documented limit";
    case MC_ERR_NO_DEVICE: return "no CUDA device visible";
    case MC_ERR_BUDGET: return "refused by the HBM budget";
    case MC_ERR_TIMEOUT: return "a bounded wait expired";
    default: return "unknown status";
  }
}

const char *mc_version(void) { return "mercury_b200 0.1.0 sm_100a"; }

int mc_dgraph_create(const int64_t *rowptr, const int32_t *col, int64_t n, int64_t nnz,
                     void *stream, unsigned flags, mc_dgraph_t **out) {
  mc::NvtxRange range("mc_dgraph_create");
  if (!rowptr || (nnz > 0 && !col)) return MC_ERR_ARG;
  mc_dgraph *g = nullptr;
  int rc = mc::create_common(n, nnz, stream, out, &g, flags);
  if (rc != MC_OK) {
    release(g);
    return rc;
  }
  auto up = [&]() -> int {
    MC_CUDA_TRY(cudaMemcpyAsync(g->rowptr, rowptr, sizeof(int64_t) * (size_t)(n + 1),
                                cudaMemcpyHostToDevice, g->stream));
    if (nnz > 0 && g->col_host)
      mc::copy_to_pinned(g->col_h, col, nnz);
    else if (nnz > 0)
      MC_CUDA_TRY(cudaMemcpyAsync(g->col, col, sizeof(int32_t) * (size_t)nnz,
                                  cudaMemcpyHostToDevice, g->stream));
    return MC_OK;
  };
  return mc::finish_create(g, flags, out, up());
}

int mc_dgraph_create_device(const int64_t *d_rowptr, const int32_t *d_col, int64_t n, int64_t nnz,
                            void *stream, unsigned flags, mc_dgraph_t **out) {
  if (!d_rowptr || (nnz > 0 && !d_col)) return MC_ERR_ARG;
  mc_dgraph *g = nullptr;
  int rc = mc::create_common(n, nnz, stream, out, &g, flags);
  if (rc != MC_OK) {
    release(g);
    return rc;
  }
  auto up = [&]() -> int {
    MC_CUDA_TRY(cudaMemcpyAsync(g->rowptr, d_rowptr, sizeof(int64_t) * (size_t)(n + 1),
                                cudaMemcpyDeviceToDevice, g->stream));
    if (nnz > 0)
      MC_CUDA_TRY(cudaMemcpyAsync(g->col_host ? g->col_h : g->col, d_col,
                                  sizeof(int32_t) * (size_t)nnz,
                                  g->col_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                  g->stream));
    return MC_OK;
  };
  return mc::finish_create(g, flags, out, up());
}

int mc_dgraph_from_edges(const int32_t *src, const int32_t *dst, int64_t num_edges, int64_t n,
                         unsigned flags, void *stream, mc_dgraph_t **out, mc_timing_t *timing) {
  mc::NvtxRange range("mc_dgraph_from_edges");
  if (!out || num_edges < 0 || (num_edges > 0 && (!src || !dst))) return MC_ERR_ARG;
  if (timing) std::memset(timing, 0, sizeof(*timing));
  mc_dgraph *g = nullptr;
  // The handle starts with an empty column array; it is sized once the
  // build has counted the distinct entries.
  int rc = mc::create_common(n, 0, stream, out, &g, mc::kDeviceColumns);
  if (rc != MC_OK) {
    release(g);
    return rc;
  }
  mc::CsrBuild *b = nullptr;
  auto run = [&]() -> int {
    MC_CUDA_TRY(cudaEventRecord(g->ev[0], g->stream));
    int r = mc::csr_build_create(num_edges, n, g->stream, &b);
    if (r != MC_OK) return r;
    r = mc::csr_build_input(b, src, dst, (flags & MC_BUILD_DEVICE_INPUT) != 0);
    if (r != MC_OK) return r;
    MC_CUDA_TRY(cudaEventRecord(g->ev[1], g->stream));
    int64_t nnz = 0, max_degree = 0;
    r = mc::csr_build_sort(b, &nnz);
    if (r != MC_OK) return r;
    mc::dev_free(g->col, g->stream);
    g->col = nullptr;
    MC_CUDA_TRY(mc::dev_alloc((void **)&g->col, sizeof(int32_t) * (size_t)std::max<int64_t>(nnz, 1),
                              g->stream));
    g->nnz = nnz;
    r = mc::csr_build_emit(b, g->rowptr, g->col, &max_degree);
    if (r != MC_OK) return r;
    MC_CUDA_TRY(cudaEventRecord(g->ev[2], g->stream));
    return MC_OK;
  };
  rc = run();
  const int64_t launches = mc::csr_build_launches(b);
  mc::csr_build_free(b);
  // The contract check of every handle (and its max degree) runs on the
  // built CSR too.
  g->launches = 0;
  rc = mc::finish_create(g, flags & MC_VALIDATE_SYMMETRY, out, rc);
  if (rc != MC_OK) return rc;
  if (timing) {
    MC_CUDA_TRY(cudaEventRecord(g->ev[3], g->stream));
    MC_CUDA_TRY(cudaEventSynchronize(g->ev[3]));
    timing->h2d_ms = mc::elapsed(g->ev[0], g->ev[1]);
    timing->count_ms = mc::elapsed(g->ev[1], g->ev[2]);
    timing->total_ms = mc::elapsed(g->ev[0], g->ev[3]);
    timing->launches = launches + g->launches;
  }
  return MC_OK;
}

int mc_dgraph_info(const mc_dgraph_t *g, int64_t *n, int64_t *nnz, int64_t *max_degree) {
  if (!g) return MC_ERR_ARG;
  if (n) *n = g->n;
  if (nnz) *nnz = g->nnz;
  if (max_degree) *max_degree = g->max_degree;
  return MC_OK;
}

int mc_dgraph_export_csr(const mc_dgraph_t *g, int64_t *rowptr_out, int32_t *col_out) {
  if (!g || !rowptr_out) return MC_ERR_ARG;
  MC_CUDA_TRY(cudaSetDevice(g->device));
  MC_CUDA_TRY(cudaMemcpyAsync(rowptr_out, g->rowptr, sizeof(int64_t) * (size_t)(g->n + 1),
                              cudaMemcpyDeviceToHost, g->stream));
  MC_CUDA_TRY(cudaStreamSynchronize(g->stream));
  if (col_out && g->nnz > 0 && g->col_host) {
    std::memcpy(col_out, g->col_h, sizeof(int32_t) * (size_t)g->nnz);
  } else if (col_out && g->nnz > 0) {
    MC_CUDA_TRY(cudaMemcpyAsync(col_out, g->col, sizeof(int32_t) * (size_t)g->nnz,
                                cudaMemcpyDeviceToHost, g->stream));
    MC_CUDA_TRY(cudaStreamSynchronize(g->stream));
  }
  return MC_OK;
}

int mc_dgraph_dag_on_host(const mc_dgraph_t *g, int *on_host) {
  if (!g || !on_host) return MC_ERR_ARG;
  *on_host = g->dag_host ? 1 : 0;
  return MC_OK;
}

int mc_dgraph_columns_on_host(const mc_dgraph_t *g, int *on_host) {
  if (!g || !on_host) return MC_ERR_ARG;
  *on_host = g->col_host ? 1 : 0;
  return MC_OK;
}

int mc_dgraph_stream(const mc_dgraph_t *g, void **stream) {
  if (!g || !stream) return MC_ERR_ARG;
  *stream = (void *)g->stream;
  return MC_OK;
}

void mc_dgraph_free(mc_dgraph_t *g) { release(g); }

int mc_tc_count(mc_dgraph_t *g, uint64_t *count, mc_timing_t *timing) {
  return mc_tc_count_shard(g, 0, 1, count, timing);
}

}  // extern "C"

namespace mc {
namespace {
// The triangle count of a handle; upload (host memory, or null) streams the
// column array into the handle during orientation (see tc_orient).
int tc_count_impl(mc_dgraph_t *g, int shard, int num_shards, uint64_t *count,
                  mc_timing_t *timing, const int32_t *upload) {
  NvtxRange range("mc_tc_count");
  if (!g || !count || num_shards < 1 || shard < 0 || shard >= num_shards) return MC_ERR_ARG;
  MC_CUDA_TRY(cudaSetDevice(g->device));
  int rc = tc_alloc(g);
  if (rc != MC_OK) return rc;
  cudaStream_t s = g->stream;
  const int64_t launches_before = g->launches;
  MC_CUDA_TRY(cudaEventRecord(g->ev[0], s));
  rc = tc_orient(g, upload);
  if (rc != MC_OK) return rc;
  MC_CUDA_TRY(cudaEventRecord(g->ev[1], s));
  // The hub table size follows the largest DAG out-degree (load <= 1/4).
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_counters + 3, g->counters + 3, sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_err, g->err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  // An exact-size DAG (host columns) that the rows overran (the input is not
  // symmetric), or a streamed chunk that failed its contract checks: the DAG
  // was left unwritten.
  if (*g->h_err & (kErrDagCapacity | kErrContract)) return MC_ERR_FORMAT;
  const long long maxd = (long long)g->h_counters[3];
  // MERCURY_TC_TABLE_LOG2_MAX (8..15) lowers the shared-memory table cap;
  // owners whose list no longer fits are then probed by binary search in
  // global memory (tests use it to reach that path on small graphs).
  int cap = mc::kHubTableLog2Max;
  if (const char *env = std::getenv("MERCURY_TC_TABLE_LOG2_MAX")) {
    const int v = std::atoi(env);
    if (v >= 8 && v <= mc::kHubTableLog2Max) cap = v;
  }
  int lg = 8;
  while (lg < cap && (1ll << lg) < 4 * maxd) ++lg;
  g->hub_table_log2 = lg;
  // MERCURY_TC_BITMAP_BITS caps the hub bitmaps (0: tables only), so that
  // tests reach the table paths on graphs whose ranks would all fit.
  g->bitmap_bits_cap = 0x7fffffff;
  if (const char *env = std::getenv("MERCURY_TC_BITMAP_BITS")) {
    const long v = std::atol(env);
    if (v >= 0) g->bitmap_bits_cap = (int)std::min<long>(v, 0x7fffffff);
  }
  // MERCURY_TC_DENSE_FACTOR (1..64): words of a core-bitmap AND allowed per
  // list entry it replaces.
  g->dense_factor = 2;
  if (const char *env = std::getenv("MERCURY_TC_DENSE_FACTOR")) {
    const int v = std::atoi(env);
    if (v >= 1 && v <= 64) g->dense_factor = v;
  }
  MC_CUDA_TRY(cudaEventRecord(g->ev[4], s));
  rc = mc::tc_count_launch(g, g->ev[2], shard, num_shards);
  if (rc != MC_OK) return rc;
  MC_CUDA_TRY(cudaEventRecord(g->ev[3], s));
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_counters, g->counters, sizeof(unsigned long long) * 8,
                              cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_err, g->err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  if (*g->h_err) return MC_ERR_DEVICE;
  *count = (uint64_t)g->h_counters[0];
  if (timing) {
    std::memset(timing, 0, sizeof(*timing));
    timing->orient_ms = mc::elapsed(g->ev[0], g->ev[1]);
    timing->hub_ms = mc::elapsed(g->ev[4], g->ev[2]);
    timing->leaf_ms = mc::elapsed(g->ev[2], g->ev[3]);
    timing->count_ms = mc::elapsed(g->ev[4], g->ev[3]);
    timing->total_ms = mc::elapsed(g->ev[0], g->ev[3]);
    timing->launches = g->launches - launches_before;
  }
  return MC_OK;
}

}  // namespace
}  // namespace mc

extern "C" {

int mc_tc_count_shard(mc_dgraph_t *g, int shard, int num_shards, uint64_t *count,
                      mc_timing_t *timing) {
  return mc::tc_count_impl(g, shard, num_shards, count, timing, nullptr);
}

int mc_tc_stats(const mc_dgraph_t *g, mc_tc_stats_t *stats) {
  if (!g || !stats) return MC_ERR_ARG;
  MC_CUDA_TRY(cudaSetDevice(g->device));
  return mc::tc_stats(const_cast<mc_dgraph *>(g), stats);
}

int mc_dgraph_export_dag(const mc_dgraph_t *g, int64_t *rowptr_out, int32_t *col_out) {
  if (!g || !rowptr_out) return MC_ERR_ARG;
  if (!g->tc_ready) return MC_ERR_ARG;
  MC_CUDA_TRY(cudaSetDevice(g->device));
  MC_CUDA_TRY(cudaMemcpyAsync(rowptr_out, g->dag_rowptr, sizeof(int64_t) * (size_t)(g->n + 1),
                              cudaMemcpyDeviceToHost, g->stream));
  MC_CUDA_TRY(cudaStreamSynchronize(g->stream));
  const int64_t m = rowptr_out[g->n];
  if (m > 0 && col_out) {
    MC_CUDA_TRY(cudaMemcpyAsync(col_out, g->dag_col, sizeof(int32_t) * (size_t)m,
                                cudaMemcpyDeviceToHost, g->stream));
    MC_CUDA_TRY(cudaStreamSynchronize(g->stream));
  }
  return MC_OK;
}

int mc_tc_count_host(const int64_t *rowptr, const int32_t *col, int64_t n, int64_t nnz,
                     uint64_t *count, mc_timing_t *timing) {
  if (!rowptr || (nnz > 0 && !col) || !count || n < 0 || nnz < 0) return MC_ERR_ARG;
  mc::HostCache &c = mc::t_cache;
  int dev = 0;
  MC_CUDA_TRY(cudaGetDevice(&dev));
  if (c.g && (c.g->device != dev || n > c.cap_n || nnz > c.cap_nnz)) {
    release(c.g);
    c.g = nullptr;
  }
  // A graph the device cannot hold is counted with its columns in host
  // memory. A cached handle of that kind is kept only while the graphs
  // still need it.
  bool host = false, dag_host = false;
  if (!c.g || c.g->col_host) {
    const int prc = mc::columns_on_host(dev, n, nnz, 0, &host, &dag_host);
    if (prc != MC_OK) return prc;
    if (c.g && (!host || c.g->dag_host != dag_host)) {
      release(c.g);
      c.g = nullptr;
    }
  }
  if (!c.g) {
    mc_dgraph *g = nullptr;
    mc_dgraph *tmp = nullptr;
    int rc = mc::create_common(n, nnz, nullptr, &tmp, &g,
                               dag_host ? MC_HOST_DAG
                                        : (host ? MC_HOST_COLUMNS : mc::kDeviceColumns));
    if (rc != MC_OK) {
      release(g);
      return rc;
    }
    c.g = g;
    c.cap_n = n;
    c.cap_nnz = nnz;
    rc = mc::tc_alloc(g);
    if (rc != MC_OK) {
      release(g);
      c.g = nullptr;
      return rc;
    }
  }
  mc_dgraph *g = c.g;
  g->n = n;
  g->nnz = nnz;
  // Pageable arrays (the reference loader's new[] arrays) cross the link
  // through pinned slots that the host threads fill (see staged_dag_passes).
  const bool pageable = !g->col_host && nnz > 0 && mc::is_pageable(col);
  g->pin_slot[0] = g->pin_slot[1] = nullptr;
  g->pin_entries = 0;
  if (pageable) {
    const int64_t want = g->chunk_edges;  // one upload chunk (whole tiles)
    if (c.pin_col_entries < want || c.pin_rowptr_entries < n + 1) {
      c.drop_pins();
      MC_CUDA_TRY(cudaHostAlloc((void **)&c.pin_col[0], sizeof(int32_t) * (size_t)want,
                                cudaHostAllocPortable));
      MC_CUDA_TRY(cudaHostAlloc((void **)&c.pin_col[1], sizeof(int32_t) * (size_t)want,
                                cudaHostAllocPortable));
      MC_CUDA_TRY(cudaHostAlloc((void **)&c.pin_rowptr, sizeof(int64_t) * (size_t)(n + 1),
                                cudaHostAllocPortable));
      MC_CUDA_TRY(cudaEventCreateWithFlags(&c.pin_done[0], cudaEventDisableTiming));
      MC_CUDA_TRY(cudaEventCreateWithFlags(&c.pin_done[1], cudaEventDisableTiming));
      c.pin_col_entries = want;
      c.pin_rowptr_entries = n + 1;
    }
    g->pin_slot[0] = c.pin_col[0];
    g->pin_slot[1] = c.pin_col[1];
    g->pin_entries = c.pin_col_entries;
    g->pin_done[0] = c.pin_done[0];
    g->pin_done[1] = c.pin_done[1];
  }
  cudaEvent_t e0, e1;
  MC_CUDA_TRY(cudaEventCreate(&e0));
  MC_CUDA_TRY(cudaEventCreate(&e1));
  MC_CUDA_TRY(cudaEventRecord(e0, g->stream));
  if (pageable) {
    // The previous call's copy out of the pinned offsets has finished (that
    // call synchronised its stream before returning).
    const int64_t *src = rowptr;
    int64_t *dst = c.pin_rowptr;
    const int64_t count = n + 1;
    constexpr int64_t kPiece = 1 << 17;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < (count + kPiece - 1) / kPiece; ++p) {
      const int64_t a = p * kPiece, b = std::min(count, a + kPiece);
      std::memcpy(dst + a, src + a, sizeof(int64_t) * (size_t)(b - a));
    }
    MC_CUDA_TRY(cudaMemcpyAsync(g->rowptr, c.pin_rowptr, sizeof(int64_t) * (size_t)(n + 1),
                                cudaMemcpyHostToDevice, g->stream));
  } else {
    MC_CUDA_TRY(cudaMemcpyAsync(g->rowptr, rowptr, sizeof(int64_t) * (size_t)(n + 1),
                                cudaMemcpyHostToDevice, g->stream));
  }
  if (nnz > 0 && g->col_host) mc::copy_to_pinned(g->col_h, col, nnz);  // while the offsets upload
  MC_CUDA_TRY(cudaEventRecord(e1, g->stream));
  g->launches = 0;
  int rc;
  int64_t validate_launches = 0;
  if (g->col_host) {
    rc = mc::validate_graph(g, 0);
    validate_launches = g->launches;
    if (rc == MC_OK) rc = mc_tc_count(g, count, timing);
  } else {
    // Device columns: the row offsets are checked first; the column array
    // then crosses in chunks during orientation, each chunk checked before
    // the passes that read it, so the copy overlaps the checks and passes.
    rc = mc::validate_rowptr(g);
    validate_launches = g->launches;
    if (rc == MC_OK) rc = mc::tc_count_impl(g, 0, 1, count, timing, nnz > 0 ? col : nullptr);
  }
  if (rc == MC_OK && timing) {
    timing->h2d_ms = mc::elapsed(e0, e1);
    timing->orient_ms += mc::elapsed(e1, g->ev[0]);  // validation on upload
    timing->total_ms = mc::elapsed(e0, g->ev[3]);
    timing->launches += validate_launches;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

}  // extern "C"

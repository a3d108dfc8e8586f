// Batched counting: many graphs, each tagged with a job (triangles or
// P1..P8), counted together.  The graphs are one device CSR (their disjoint
// union: graph g owns vertices [gptr[g], gptr[g+1]) and no edge crosses
// graphs).  One pass runs the device orientation over the union, the
// triangle kernels on the triangle graphs (each task adds its hits to its
// own graph), one persistent pattern kernel over every pattern graph's
// tasks, and a combine step -- captured once as a CUDA graph and replayed
// per count.  An autotuner picks, per degree bucket of the triangle graphs,
// the warp/CTA threshold on the owner's out-degree and the table slots per
// key.
//
// The reference has no batched mode; each graph there is a separate run of
// TCSolver (tc_challenge.cu:11) or SMSolverMultiGPU
// (subgraph_matching/sm_multigpu.cu:97).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "dgraph.cuh"
#include "device_common.cuh"

namespace mc {
namespace {

constexpr int kBuckets = 4;  // by the graph's largest degree: <64, <256, <1024, >=1024
constexpr int kLeafChoices[] = {16, 32, 64, 128};
constexpr int kSlotChoices[] = {1, 2, 3};  // log2 table slots per key

int degree_bucket(int64_t max_degree) {
  if (max_degree < 64) return 0;
  if (max_degree < 256) return 1;
  if (max_degree < 1024) return 2;
  return 3;
}

__global__ void fill_gid_kernel(const int64_t *gptr, int num_graphs, int64_t n, int32_t *gid) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  int lo = 0, hi = num_graphs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (gptr[mid] <= v) lo = mid;
    else hi = mid - 1;
  }
  gid[v] = lo;
}

// Rows are sorted, so the first and last neighbour bound the row.
__global__ void check_within_graph_kernel(const int64_t *rowptr, const int32_t *col,
                                          const int64_t *gptr, const int32_t *gid, int64_t n,
                                          unsigned *err) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const int64_t b = rowptr[v], e = rowptr[v + 1];
  if (b == e) return;
  const int g = gid[v];
  if (col[b] < gptr[g] || col[e - 1] >= gptr[g + 1]) atomicOr(err, (unsigned)kErrIdRange);
}

__global__ void combine_kernel(const int32_t *job, const unsigned long long *res, int num_graphs,
                               unsigned long long *out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= num_graphs) return;
  const int j = job[g];
  const unsigned long long tc = res[g], c1 = res[num_graphs + g], c2 = res[2 * num_graphs + g];
  out[g] = j == 0 ? tc : ((j == 4 || j == 6) ? c1 : c1 - c2);
}

unsigned blocks(int64_t items, int threads) {
  return (unsigned)std::max<int64_t>(1, (items + threads - 1) / threads);
}

int ceil_log2_i64(int64_t v) {
  int lg = 0;
  while ((int64_t(1) << lg) < v) ++lg;
  return lg;
}

}  // namespace
}  // namespace mc

struct mc_batch {
  mc_dgraph *g = nullptr;  // the union CSR and the triangle-count scratch
  int num_graphs = 0;
  std::vector<int64_t> gptr;
  std::vector<int32_t> job;
  std::vector<int> bucket;     // degree bucket of each triangle graph, -1 otherwise
  std::vector<int64_t> dplus_bound;  // per triangle graph: bound on d+
  std::vector<int2> param;     // per graph {leaf threshold, log2 slots per key}
  int64_t *d_gptr = nullptr;
  int32_t *d_gid = nullptr, *d_job = nullptr, *d_job_active = nullptr;
  int2 *d_param = nullptr;
  unsigned long long *d_res = nullptr;   // 3 x num_graphs: triangles, c1, c2
  unsigned long long *d_out = nullptr;   // num_graphs
  unsigned long long *h_out = nullptr;   // pinned
  bool has_tc = false, has_pat = false;
  mc::BatchPatternArgs pa{};
  int pat_grid = 0;
  int table_log2 = 8;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t graph_launches = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int32_t tuned[mc::kBuckets][2];
};

namespace mc {
namespace {

void batch_release(mc_batch *b) {
  if (!b) return;
  if (b->g) {
    cudaSetDevice(b->g->device);
    cudaStreamSynchronize(b->g->stream);
  }
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  void *bufs[] = {b->d_gptr, b->d_gid, b->d_job, b->d_job_active, b->d_param, b->d_res, b->d_out,
                  (void *)b->pa.graph, (void *)b->pa.job, (void *)b->pa.v0, (void *)b->pa.v1,
                  (void *)b->pa.star_off, (void *)b->pa.edge_off, b->pa.scratch, b->pa.queue};
  if (b->g)
    for (void *p : bufs)
      if (p) dev_free(p, b->g->stream);
  delete[] b->h_out;
  if (b->e0) cudaEventDestroy(b->e0);
  if (b->e1) cudaEventDestroy(b->e1);
  if (b->g) mc_dgraph_free(b->g);
  delete b;
}

// Slots-per-key of the largest table any triangle graph may build, sizing
// the hub kernel's shared memory (no host round trip inside the graph).
void size_tables(mc_batch *b) {
  int lg = 8;
  for (int i = 0; i < b->num_graphs; ++i) {
    if (b->job[i] != 0) continue;
    const int64_t want = b->dplus_bound[i] << b->param[i].y;
    lg = std::max(lg, std::min(kHubTableLog2Max, ceil_log2_i64(std::max<int64_t>(want, 1))));
  }
  b->table_log2 = lg;
}

// Enqueues one full count on the handle's stream (no host synchronisation).
int enqueue(mc_batch *b) {
  mc_dgraph *g = b->g;
  cudaStream_t s = g->stream;
  const int G = b->num_graphs;
  MC_CUDA_TRY(cudaMemsetAsync(b->d_res, 0, sizeof(unsigned long long) * 3 * G, s));
  if (b->has_tc) {
    g->batch.gid = b->d_gid;
    g->batch.job = b->d_job_active;
    g->batch.param = b->d_param;
    g->batch.res = b->d_res;
    int rc = tc_orient(g);
    if (rc != MC_OK) return rc;
    g->hub_table_log2 = b->table_log2;
    rc = tc_count_launch(g, nullptr, 0, 1);
    if (rc != MC_OK) return rc;
  }
  if (b->has_pat) {
    MC_CUDA_TRY(cudaMemsetAsync(b->pa.queue, 0, sizeof(unsigned long long), s));
    int rc = batch_pattern_launch(b->pa, b->pat_grid, s);
    if (rc != MC_OK) return rc;
    g->launches += 1;
  }
  combine_kernel<<<blocks(G, 256), 256, 0, s>>>(b->d_job, b->d_res, G, b->d_out);
  MC_CUDA_TRY(cudaGetLastError());
  g->launches += 1;
  return MC_OK;
}

// Counts and the error word to the host, after the stream reached them.
int read_back(mc_batch *b) {
  mc_dgraph *g = b->g;
  MC_CUDA_TRY(cudaMemcpyAsync(b->h_out, b->d_out, sizeof(unsigned long long) * b->num_graphs,
                              cudaMemcpyDeviceToHost, g->stream));
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_err, g->err, sizeof(unsigned), cudaMemcpyDeviceToHost,
                              g->stream));
  MC_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return MC_OK;
}

int capture(mc_batch *b) {
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  cudaStream_t s = b->g->stream;
  const int64_t before = b->g->launches;
  MC_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  const int rc = enqueue(b);
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(s, &graph);
  if (rc != MC_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  MC_CUDA_TRY(end);
  b->graph = graph;
  MC_CUDA_TRY(cudaGraphInstantiate(&b->exec, graph, 0));
  b->graph_launches = b->g->launches - before;
  return MC_OK;
}

int upload_params(mc_batch *b) {
  MC_CUDA_TRY(cudaMemcpyAsync(b->d_param, b->param.data(), sizeof(int2) * b->num_graphs,
                              cudaMemcpyHostToDevice, b->g->stream));
  return MC_OK;
}

}  // namespace
}  // namespace mc

using mc::batch_release;

namespace mc {

// Builds a batch from a union CSR held in host memory (device_csr false) or
// device memory (true), with each graph's largest degree and entry count
// given by the caller (gmaxdeg, gnnz); with do_capture the count sequence is
// captured as a CUDA graph, otherwise every count launches it directly.
int batch_create(const int64_t *rowptr, const int32_t *col, bool device_csr, int64_t n,
                 int64_t nnz, const int64_t *graph_vptr, int num_graphs, const int32_t *jobs,
                 const int64_t *gmaxdeg, const int64_t *gnnz_of, void *stream, bool do_capture,
                 mc_batch_t **out) {
  if (!out || !rowptr || !graph_vptr || !jobs || num_graphs < 1 || n < 0 || nnz < 0)
    return MC_ERR_ARG;
  *out = nullptr;
  if (graph_vptr[0] != 0 || graph_vptr[num_graphs] != n) return MC_ERR_ARG;
  for (int i = 0; i < num_graphs; ++i) {
    if (graph_vptr[i + 1] < graph_vptr[i] || jobs[i] < 0 || jobs[i] > 8) return MC_ERR_ARG;
  }
  mc_batch *b = new (std::nothrow) mc_batch();
  if (!b) return MC_ERR_OOM;
  b->num_graphs = num_graphs;
  b->gptr.assign(graph_vptr, graph_vptr + num_graphs + 1);
  b->job.assign(jobs, jobs + num_graphs);
  b->bucket.assign(num_graphs, -1);
  b->dplus_bound.assign(num_graphs, 0);
  // MERCURY_BATCH_LEAF_MAX (one of the autotuner's thresholds, 16..128)
  // overrides the default warp/CTA threshold, so that tests reach every
  // schedule the autotuner may pick.
  int leaf_max = kLeafMaxOut;
  if (const char *env = std::getenv("MERCURY_BATCH_LEAF_MAX")) {
    const int v = std::atoi(env);
    for (int c : kLeafChoices)
      if (v == c) leaf_max = v;
  }
  b->param.assign(num_graphs, make_int2(leaf_max, 2));
  for (auto &row : b->tuned) row[0] = row[1] = -1;
  auto fail = [&](int rc) {
    batch_release(b);
    return rc;
  };
  int rc = device_csr ? mc_dgraph_create_device(rowptr, col, n, nnz, stream, 0, &b->g)
                      : mc_dgraph_create(rowptr, col, n, nnz, stream, 0, &b->g);
  if (rc != MC_OK) return fail(rc);
  mc_dgraph *g = b->g;
  cudaStream_t s = g->stream;
  const int G = num_graphs;
  // Per-graph sizes: largest degree and a bound on d+ (d+(v)^2 <= the
  // graph's nnz, as every out-neighbour has degree >= d+(v)).
  int64_t pat_cap = 1;
  std::vector<int32_t> pg_graph, pg_job;
  std::vector<int64_t> pg_v0, pg_v1, star_off(1, 0), edge_off(1, 0);
  for (int i = 0; i < G; ++i) {
    const int64_t md = gmaxdeg[i];
    const int64_t gnnz = gnnz_of[i];
    if (jobs[i] == 0) {
      b->has_tc = true;
      b->bucket[i] = degree_bucket(md);
      b->dplus_bound[i] = std::min<int64_t>(md, (int64_t)std::sqrt((double)gnnz) + 1);
    } else {
      b->has_pat = true;
      pat_cap = std::max(pat_cap, md);
      pg_graph.push_back(i);
      pg_job.push_back(jobs[i]);
      pg_v0.push_back(graph_vptr[i]);
      pg_v1.push_back(graph_vptr[i + 1]);
      star_off.push_back(star_off.back() + (jobs[i] == 1 ? graph_vptr[i + 1] - graph_vptr[i] : 0));
      edge_off.push_back(edge_off.back() + gnnz);
    }
  }
  auto alloc = [s](void **p, size_t bytes) { return dev_alloc(p, bytes, s); };
#define MC_BALLOC(ptr, bytes) MC_CUDA_TRY(alloc((void **)&(ptr), (bytes)))
  try {
    MC_BALLOC(b->d_gptr, sizeof(int64_t) * (G + 1));
    MC_BALLOC(b->d_gid, sizeof(int32_t) * std::max<int64_t>(n, 1));
    MC_BALLOC(b->d_job, sizeof(int32_t) * G);
    MC_BALLOC(b->d_job_active, sizeof(int32_t) * G);
    MC_BALLOC(b->d_param, sizeof(int2) * G);
    MC_BALLOC(b->d_res, sizeof(unsigned long long) * 3 * G);
    MC_BALLOC(b->d_out, sizeof(unsigned long long) * G);
    b->h_out = new unsigned long long[G]();
    MC_CUDA_TRY(cudaEventCreate(&b->e0));
    MC_CUDA_TRY(cudaEventCreate(&b->e1));
    MC_CUDA_TRY(cudaMemcpyAsync(b->d_gptr, graph_vptr, sizeof(int64_t) * (G + 1),
                                cudaMemcpyHostToDevice, s));
    MC_CUDA_TRY(cudaMemcpyAsync(b->d_job, jobs, sizeof(int32_t) * G, cudaMemcpyHostToDevice, s));
    MC_CUDA_TRY(cudaMemcpyAsync(b->d_job_active, jobs, sizeof(int32_t) * G, cudaMemcpyHostToDevice,
                                s));
    rc = upload_params(b);
    if (rc != MC_OK) return fail(rc);
    if (n > 0) {
      fill_gid_kernel<<<blocks(n, 256), 256, 0, s>>>(b->d_gptr, G, n, b->d_gid);
      MC_CUDA_TRY(cudaGetLastError());
      MC_CUDA_TRY(cudaMemsetAsync(g->err, 0, sizeof(unsigned), s));
      check_within_graph_kernel<<<blocks(n, 256), 256, 0, s>>>(g->rowptr, g->col, b->d_gptr,
                                                               b->d_gid, n, g->err);
      MC_CUDA_TRY(cudaGetLastError());
      MC_CUDA_TRY(cudaMemcpyAsync(g->h_err, g->err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
      MC_CUDA_TRY(cudaStreamSynchronize(s));
      if (*g->h_err) return fail(MC_ERR_FORMAT);  // an edge crosses two graphs
    }
    if (b->has_tc) {
      g->batch.gid = b->d_gid;  // a batch handle: no degree ranks (see tc_alloc)
      rc = tc_alloc(g);
      if (rc != MC_OK) return fail(rc);
    }
    if (b->has_pat) {
      const int Gp = (int)pg_graph.size();
      mc::BatchPatternArgs &pa = b->pa;
      pa.rp = g->rowptr;
      pa.ci = g->col;
      pa.num_graphs = Gp;
      MC_BALLOC(pa.graph, sizeof(int32_t) * Gp);
      MC_BALLOC(pa.job, sizeof(int32_t) * Gp);
      MC_BALLOC(pa.v0, sizeof(int64_t) * Gp);
      MC_BALLOC(pa.v1, sizeof(int64_t) * Gp);
      MC_BALLOC(pa.star_off, sizeof(int64_t) * (Gp + 1));
      MC_BALLOC(pa.edge_off, sizeof(int64_t) * (Gp + 1));
      MC_BALLOC(pa.queue, sizeof(unsigned long long));
      MC_CUDA_TRY(cudaMemcpyAsync((void *)pa.graph, pg_graph.data(), sizeof(int32_t) * Gp,
                                  cudaMemcpyHostToDevice, s));
      MC_CUDA_TRY(cudaMemcpyAsync((void *)pa.job, pg_job.data(), sizeof(int32_t) * Gp,
                                  cudaMemcpyHostToDevice, s));
      MC_CUDA_TRY(cudaMemcpyAsync((void *)pa.v0, pg_v0.data(), sizeof(int64_t) * Gp,
                                  cudaMemcpyHostToDevice, s));
      MC_CUDA_TRY(cudaMemcpyAsync((void *)pa.v1, pg_v1.data(), sizeof(int64_t) * Gp,
                                  cudaMemcpyHostToDevice, s));
      MC_CUDA_TRY(cudaMemcpyAsync((void *)pa.star_off, star_off.data(), sizeof(int64_t) * (Gp + 1),
                                  cudaMemcpyHostToDevice, s));
      MC_CUDA_TRY(cudaMemcpyAsync((void *)pa.edge_off, edge_off.data(), sizeof(int64_t) * (Gp + 1),
                                  cudaMemcpyHostToDevice, s));
      int64_t warps = 0;
      b->pat_grid = batch_pattern_grid(g->num_sms, pat_cap, &warps);
      pa.cap = pat_cap;
      MC_BALLOC(pa.scratch, sizeof(int32_t) * (size_t)(warps * pattern_lists() * pat_cap));
      pa.c1 = b->d_res + G;
      pa.c2 = b->d_res + 2 * G;
    }
  } catch (...) {
    return fail(MC_ERR_OOM);
  }
#undef MC_BALLOC
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  size_tables(b);
  if (do_capture) {
    rc = capture(b);
    if (rc != MC_OK) return fail(rc);
  }
  *out = b;
  return MC_OK;
}

}  // namespace mc

extern "C" {

int mc_batch_create(const int64_t *rowptr, const int32_t *col, int64_t n, int64_t nnz,
                    const int64_t *graph_vptr, int num_graphs, const int32_t *jobs, void *stream,
                    mc_batch_t **out) {
  if (!rowptr || !graph_vptr || num_graphs < 1 || n < 0) return MC_ERR_ARG;
  if (graph_vptr[0] != 0 || graph_vptr[num_graphs] != n) return MC_ERR_ARG;
  for (int i = 0; i < num_graphs; ++i)
    if (graph_vptr[i + 1] < graph_vptr[i]) return MC_ERR_ARG;
  // Per-graph largest degree and entry count from the host arrays.
  std::vector<int64_t> md(num_graphs, 0), gnnz(num_graphs, 0);
  for (int i = 0; i < num_graphs; ++i) {
    for (int64_t v = graph_vptr[i]; v < graph_vptr[i + 1]; ++v)
      md[i] = std::max<int64_t>(md[i], rowptr[v + 1] - rowptr[v]);
    gnnz[i] = rowptr[graph_vptr[i + 1]] - rowptr[graph_vptr[i]];
  }
  return mc::batch_create(rowptr, col, false, n, nnz, graph_vptr, num_graphs, jobs, md.data(),
                          gnnz.data(), stream, true, out);
}

int mc_batch_count(mc_batch_t *b, uint64_t *counts, mc_timing_t *timing) {
  mc::NvtxRange range("mc_batch_count");
  if (!b || !counts) return MC_ERR_ARG;
  MC_CUDA_TRY(cudaSetDevice(b->g->device));
  cudaStream_t s = b->g->stream;
  MC_CUDA_TRY(cudaEventRecord(b->e0, s));
  if (b->exec) {
    MC_CUDA_TRY(cudaGraphLaunch(b->exec, s));
  } else {
    const int erc = mc::enqueue(b);
    if (erc != MC_OK) return erc;
  }
  MC_CUDA_TRY(cudaEventRecord(b->e1, s));
  const int rc = mc::read_back(b);
  if (rc != MC_OK) return rc;
  if (*b->g->h_err) return MC_ERR_DEVICE;
  std::memcpy(counts, b->h_out, sizeof(uint64_t) * b->num_graphs);
  if (timing) {
    std::memset(timing, 0, sizeof(*timing));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->e0, b->e1);
    timing->total_ms = ms;
    timing->count_ms = ms;
    timing->launches = b->graph_launches;
  }
  return MC_OK;
}

int mc_batch_autotune(mc_batch_t *b, int32_t *choice) {
  using namespace mc;
  if (!b) return MC_ERR_ARG;
  MC_CUDA_TRY(cudaSetDevice(b->g->device));
  cudaStream_t s = b->g->stream;
  const int G = b->num_graphs;
  std::vector<int32_t> active(G);
  for (int bk = 0; bk < kBuckets; ++bk) {
    bool any = false;
    for (int i = 0; i < G; ++i) {
      active[i] = (b->job[i] == 0 && b->bucket[i] == bk) ? 0 : -1;
      any |= active[i] == 0;
    }
    if (!any || !b->has_tc) continue;
    MC_CUDA_TRY(cudaMemcpyAsync(b->d_job_active, active.data(), sizeof(int32_t) * G,
                                cudaMemcpyHostToDevice, s));
    const bool had_pat = b->has_pat;
    b->has_pat = false;  // time the triangle part of this bucket alone
    float best = 1e30f;
    for (int leaf : kLeafChoices) {
      for (int slots : kSlotChoices) {
        for (int i = 0; i < G; ++i)
          if (active[i] == 0) b->param[i] = make_int2(leaf, slots);
        int rc = upload_params(b);
        if (rc == MC_OK) {
          size_tables(b);
          float ms = 0.f;
          for (int rep = 0; rep < 2 && rc == MC_OK; ++rep) {  // second run is timed
            MC_CUDA_TRY(cudaEventRecord(b->e0, s));
            rc = enqueue(b);
            MC_CUDA_TRY(cudaEventRecord(b->e1, s));
            if (rc == MC_OK) rc = read_back(b);
            cudaEventElapsedTime(&ms, b->e0, b->e1);
          }
          if (rc == MC_OK && *b->g->h_err) rc = MC_ERR_DEVICE;
          if (rc == MC_OK && ms < best) {
            best = ms;
            b->tuned[bk][0] = leaf;
            b->tuned[bk][1] = slots;
          }
        }
        if (rc != MC_OK) {
          b->has_pat = had_pat;
          return rc;
        }
      }
    }
    b->has_pat = had_pat;
  }
  for (int i = 0; i < G; ++i)
    if (b->job[i] == 0 && b->tuned[b->bucket[i]][0] > 0)
      b->param[i] = make_int2(b->tuned[b->bucket[i]][0], b->tuned[b->bucket[i]][1]);
  MC_CUDA_TRY(cudaMemcpyAsync(b->d_job_active, b->job.data(), sizeof(int32_t) * G,
                              cudaMemcpyHostToDevice, s));
  int rc = upload_params(b);
  if (rc != MC_OK) return rc;
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  size_tables(b);
  rc = capture(b);
  if (rc != MC_OK) return rc;
  if (choice)
    for (int bk = 0; bk < kBuckets; ++bk) {
      choice[2 * bk] = b->tuned[bk][0];
      choice[2 * bk + 1] = b->tuned[bk][1];
    }
  return MC_OK;
}

void mc_batch_free(mc_batch_t *b) { batch_release(b); }

}  // extern "C"

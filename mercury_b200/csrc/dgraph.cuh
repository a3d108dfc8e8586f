// Device-resident graph handle and the scratch layout of the counting path.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "mercury.h"

// Tunables of the triangle-count schedule (task classes and chunk sizes).
namespace mc {
constexpr int kTileThreads = 256;          // threads per orientation tile
constexpr int kEdgesPerThread = 16;        // consecutive CSR entries per thread
constexpr int64_t kTileEdges = (int64_t)kTileThreads * kEdgesPerThread;
constexpr int kLeafMaxOut = 64;            // d+(owner) <= this: warp task
constexpr int kLeafSlots = 256;            // per-warp hash slots for leaf owners
#ifndef MC_HUB_CHUNK
#define MC_HUB_CHUNK 512
#endif
constexpr int kHubChunk = MC_HUB_CHUNK;    // owner's neighbours per CTA (hub) task
constexpr int kLeafChunk = 64;             // owner's neighbours per warp (leaf) task
constexpr int kCountThreads = 256;         // threads per counting CTA
constexpr int kHubTableLog2Max = 15;       // at most 32768 slots (128 KB smem)
// Hub owners up to this d+ run in a launch with small tables (16 KB, high
// occupancy); larger ones in a launch sized for the largest table.
constexpr int kHubSmallMaxOut = 1024;
constexpr int kHubSmallTableLog2 = 12;
// Least shared memory of a hub CTA (also the bitmap capacity: 8 bits per
// byte, so owners of degree rank below 262144 use bitmaps).
constexpr int kHubBitmapBytes = 32768;
// Longest DAG out-list the P7/P8 clique route stages in shared memory.
constexpr int kCliqueMaxOut = 1024;
// Core bitmaps: N+(v) as a bitmap over ranks [0, rank(v)) for the vertices
// of the kCoreRanks lowest ranks (the highest degrees), so that a hub task
// intersects such a partner by a word-wise AND with its owner's bitmap.
constexpr int kCoreRanks = 32768;

// Word offset of rank r's core bitmap: rank t holds ceil(t / 128) quads (4
// words, 16-byte aligned) covering bits [0, t), so the offset is 4 times
// sum over t < r of ceil(t / 128) = 64 Q (Q + 1) + (r - 1 - 128 Q)(Q + 1),
// with Q = (r - 1) / 128.
__host__ __device__ __forceinline__ int64_t core_offset(int64_t r) {
  if (r <= 0) return 0;
  const int64_t q = (r - 1) >> 7;
  return 4 * (64 * q * (q + 1) + (r - 1 - 128 * q) * (q + 1));
}
}  // namespace mc

namespace mc {
// Per-graph data when one device CSR holds many graphs (a batch: the
// disjoint union, graph g owning vertices [gptr[g], gptr[g+1])).  All null
// for a single graph, which then uses the compile-time schedule.
struct BatchView {
  const int32_t *gid = nullptr;       // vertex -> graph
  const int32_t *job = nullptr;       // graph -> 0 (triangles) or 1..8 (pattern)
  const int2 *param = nullptr;        // graph -> {leaf d+ threshold, log2 table factor}
  unsigned long long *res = nullptr;  // graph -> triangle count
};
}  // namespace mc

struct mc_dgraph {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 0;
  int64_t n = 0, nnz = 0;
  int64_t max_degree = 0;     // set by validation on upload
  int64_t *rowptr = nullptr;  // n + 1
  int32_t *col = nullptr;     // nnz
  // Column placement: false, col is device memory; true, col is pinned host
  // memory mapped into the device's address space (graphs whose columns do
  // not fit the device; every kernel reads them over the host link).
  bool col_host = false;
  bool dag_host = false;      // DAG entries and ranks in pinned mapped host memory
  int32_t *dag_col_h = nullptr, *dag_rank_h = nullptr;  // their host views
  int32_t *col_h = nullptr;   // host view of col when col_host

  // ---- pattern-count scratch (frontier lists), grown on demand ----------
  void *pat_scratch = nullptr;
  size_t pat_scratch_bytes = 0;
  void *center_scratch = nullptr;  // center classes of the bitmap kernels
  size_t center_scratch_bytes = 0;
  void *hop_scratch = nullptr;     // two-hop rows of the centers (outer patterns)
  size_t hop_scratch_bytes = 0;
  void *hub_bits = nullptr;        // per-CTA id bitmaps of the large P1 centers
  size_t hub_bits_bytes = 0;

  // ---- vertex labels (mc_dgraph_set_vlabels), one uint8 per vertex -------
  uint8_t *vlabels = nullptr;
  int max_label = -1;

  // ---- triangle-count scratch, allocated on the first mc_tc_count -------
  bool tc_ready = false;
  int2 *key = nullptr;            // n      {symmetric degree, DAG out-degree}
  // n: {d+, rank (INT_MAX without ranks), DAG row start low, high}: what a
  // hub task needs of a neighbour, in one 16-byte load.
  int4 *pinfo = nullptr;
  int64_t *dag_rowptr = nullptr;  // n + 1
  int32_t *dag_col = nullptr;     // dag_cap (m+ used)
  int64_t dag_cap = 0;            // nnz; nnz / 2 + 1 with host columns
  // Degree rank: vertices sorted by (degree desc, id desc), so every entry
  // of N+(v) ranks below v. dag_rank holds dag_col's entries as ranks (a
  // single graph only; a batch leaves both null).
  int32_t *rank = nullptr;        // n
  int32_t *dag_rank = nullptr;    // dag_cap
  unsigned long long *rank_keys = nullptr;  // 2 n sort keys
  int32_t *rank_counts = nullptr;           // radix histograms
  int64_t *rank_offsets = nullptr;
  const unsigned long long *rank_sorted = nullptr;  // rank p -> key of vertex (see orient.cu)
  unsigned *core_bits = nullptr;  // core_offset(core_ranks) words
  int core_ranks = 0;             // capacity: core_offset(core_ranks) words
  int core_used = 0;              // ranks [0, core_used) have core bitmaps (<= n)
  int dense_factor = 2;           // AND when its words <= factor x list entries
  uint16_t *keep = nullptr;       // one DAG keep mask per orientation thread
  int32_t *tile_counts = nullptr; // tiles
  int64_t *tile_offsets = nullptr;// tiles + 1
  int64_t *tile_rows = nullptr;   // 2 x tiles: first and last row of each tile
  // Streamed upload from pageable host memory: two pinned slots of
  // pin_entries column entries (owned by the caller of the upload) and the
  // events that mark each slot's copy to the device done.
  int32_t *pin_slot[2] = {nullptr, nullptr};
  int64_t pin_entries = 0;
  cudaEvent_t pin_done[2] = {nullptr, nullptr};
  int32_t *hub_cnt = nullptr, *leaf_cnt = nullptr, *mega_cnt = nullptr;    // n
  int64_t *hub_off = nullptr, *leaf_off = nullptr, *mega_off = nullptr;    // n + 1
  uint64_t *hub_tasks = nullptr, *leaf_tasks = nullptr, *mega_tasks = nullptr;  // capacity
  int64_t task_capacity = 0;
  // Host columns: two DMA staging buffers of stage_edges entries each, the
  // stream that fills them, events {copied[2], drained[2]}, and the tile
  // offsets of one chunk.
  int32_t *stage = nullptr;
  int64_t stage_edges = 0;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t stage_ev[4] = {};
  int64_t chunk_edges = 0;  // entries per chunk of a streamed upload (fixed at allocation)
  int64_t *chunk_offsets = nullptr;  // chunk_edges / kTileEdges + 1
  void *scan_temp = nullptr;
  size_t scan_temp_size = 0;
  // 0: result, 1: hub queue, 2: leaf queue, 3: max d+, 4-5: partner
  // statistics, 6: large-table hub queue, 7: max degree (validation)
  unsigned long long *counters = nullptr;
  unsigned *err = nullptr;
  // pinned host mirror of counters + err
  unsigned long long *h_counters = nullptr;
  unsigned *h_err = nullptr;
  int hub_table_log2 = 10;
  int bitmap_bits_cap = 0x7fffffff;  // upper bound on hub bitmap capacity (bits)
  cudaEvent_t ev[6] = {};
  int64_t launches = 0;  // kernels launched by the current call
  mc::BatchView batch;   // set by a batch that owns this handle
};

namespace mc {
// orient.cu
int validate_graph(mc_dgraph *g, unsigned flags);
int tc_alloc(mc_dgraph *g);
// Device bytes tc_alloc takes for a single graph of n vertices and nnz
// entries (the DAG at half the entries when the columns are on the host).
int64_t tc_device_bytes(int64_t n, int64_t nnz, bool col_host, bool dag_host = false);
// upload (host memory, nnz entries): the column array is copied into the
// handle in chunks during the passes, each chunk checked against the CSR
// contract first (the row offsets must have been checked: validate_rowptr).
int tc_orient(mc_dgraph *g, const int32_t *upload = nullptr);
// P7 and P8 by clique counts (cliques.cu): whether the route applies
// (building the DAG if it does), and its launch, which adds the count to
// counters[0].
int clique_prepare(mc_dgraph *g, int pattern, bool *use, int64_t *dag_edges);
int clique_launch(mc_dgraph *g, int pattern, int64_t dag_edges, int shard, int num_shards,
                  const unsigned long long *deadline, unsigned long long *stop_flag);
// Contract checks of the row offsets alone; sets max_degree.
int validate_rowptr(mc_dgraph *g);
int tc_partner_stats(mc_dgraph *g, unsigned long long *partner_edges, unsigned long long *work);
// Contract checks of a caller-owned device CSR with caller-provided device
// words for the error flag and the maximum degree (nothing is allocated).
int validate_csr_words(const int64_t *rowptr, const int32_t *col, int64_t n, int64_t nnz,
                       unsigned *d_err, unsigned long long *d_max_deg, cudaStream_t s,
                       int64_t *max_degree);
// tc.cu
int tc_count_launch(mc_dgraph *g, cudaEvent_t after_hub, int shard, int num_shards);
// patterns.cu: result of P<pattern>; c12 (optional) receives counters 1 and 2.
// Shard `shard` of `num_shards` (0 of 1: the whole count); partial results
// of all shards sum to the count modulo 2^64.
// budget_ms > 0: slice the launches and stop with MC_ERR_TIMEOUT once the
// sliced launches have used more device time than that; progress (optional)
// receives the fraction of the sliced tasks done.
int pattern_count(mc_dgraph *g, int pattern, uint64_t *out, uint64_t *c12, mc_timing_t *timing,
                  int shard = 0, int num_shards = 1, double budget_ms = -1.0,
                  double *progress = nullptr);

// Pattern tasks of a batch (see batch.cu): pattern graphs 0..num_graphs-1.
struct BatchPatternArgs {
  const int64_t *rp;          // union CSR
  const int32_t *ci;
  int num_graphs;
  const int32_t *graph;       // pattern graph -> batch graph id
  const int32_t *job;         // pattern graph -> 1..8
  const int64_t *v0, *v1;     // pattern graph -> vertex range
  const int64_t *star_off;    // cumulative P1 star tasks, num_graphs + 1
  const int64_t *edge_off;    // cumulative directed-edge tasks, num_graphs + 1
  int32_t *scratch;           // frontier lists
  int64_t cap;                // list capacity (max degree over pattern graphs)
  unsigned long long *c1, *c2;  // per batch graph
  unsigned long long *queue;
};
int batch_pattern_launch(const BatchPatternArgs &b, int grid, cudaStream_t s);
// batch.cu: a batch over a host (device_csr false) or device union CSR.
int batch_create(const int64_t *rowptr, const int32_t *col, bool device_csr, int64_t n,
                 int64_t nnz, const int64_t *graph_vptr, int num_graphs, const int32_t *jobs,
                 const int64_t *gmaxdeg, const int64_t *gnnz_of, void *stream, bool do_capture,
                 mc_batch_t **out);
// Blocks of the batch pattern kernel whose frontier lists fit the scratch
// budget; *warps receives the resident warp count.
int batch_pattern_grid(int num_sms, int64_t cap, int64_t *warps);
int pattern_lists();

// build.cu: the device CSR build from an edge list, in steps so that callers
// can time them and place the output where they need it.
struct CsrBuild;
// Scratch for m pairs over n vertices, on stream s.
int csr_build_create(int64_t m, int64_t n, cudaStream_t s, CsrBuild **out);
// Pairs in: copied from the host, or read in place from device memory.
int csr_build_input(CsrBuild *b, const int32_t *src, const int32_t *dst, bool device_input);
// Sorts the packed keys and counts the distinct entries; waits for the
// stream. MC_ERR_FORMAT when an id is outside [0, n).
int csr_build_sort(CsrBuild *b, int64_t *nnz);
// Writes col[nnz] and rowptr[n + 1]; *max_degree gets the largest row.
int csr_build_emit(CsrBuild *b, int64_t *rowptr, int32_t *col, int64_t *max_degree);
int64_t csr_build_launches(const CsrBuild *b);
void csr_build_free(CsrBuild *b);
}  // namespace mc

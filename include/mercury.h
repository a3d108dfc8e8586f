/*
 * mercury.h -- C ABI of the B200 (sm_100a) counting path: triangle counting
 * and the P1..P8 pattern counts over an undirected CSR graph.
 *
 * Every entry point returns an int status (MC_OK == 0, negative on error)
 * and never exits or aborts the calling process; mc_strerror() names the
 * status.  Device buffers are owned by the handle that created them until
 * the matching *_free call.  Calls on distinct handles may run from distinct
 * host threads; calls on one handle must be serialised by the caller.
 *
 * Graph contract (the reference's input contract, graph.cc:18-35): vertex ids
 * are int32 in [0, n), row offsets are int64 with rowptr[0] == 0 and
 * rowptr[n] == nnz, each row is sorted strictly ascending (no duplicates), no
 * self-loops, and the adjacency is symmetric (nnz == 2m directed entries).
 * mc_dgraph_create() checks everything but symmetry on the device and
 * refuses a graph that breaks it with MC_ERR_FORMAT; MC_VALIDATE_SYMMETRY
 * adds the symmetry check.
 */
#ifndef MERCURY_B200_H
#define MERCURY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define MC_OK 0
#define MC_ERR_ARG (-1)         /* null pointer, bad size, bad pattern id      */
#define MC_ERR_IO (-2)          /* a file could not be opened/read/written     */
#define MC_ERR_FORMAT (-3)      /* input breaks the CSR contract above         */
#define MC_ERR_OOM (-4)         /* host or device allocation failed            */
#define MC_ERR_CUDA (-5)        /* a CUDA runtime call failed                  */
#define MC_ERR_DEVICE (-6)      /* a kernel raised its error flag              */
#define MC_ERR_UNSUPPORTED (-7) /* size beyond a documented limit              */
#define MC_ERR_NO_DEVICE (-8)   /* no CUDA device visible                      */
#define MC_ERR_BUDGET (-9)      /* request refused by the HBM budget           */
#define MC_ERR_TIMEOUT (-10)    /* a bounded wait expired                      */

/* ---- flags for mc_dgraph_create ----------------------------------------- */
#define MC_VALIDATE_SYMMETRY 0x1u
/* Keep the column array in pinned host memory that the device reads through
 * its mapping (the row offsets, the DAG and all scratch stay in device
 * memory).  mc_dgraph_create, mc_dgraph_create_device and mc_tc_count_host
 * choose this placement by themselves when the device's free memory cannot
 * hold the columns together with the triangle-count scratch.  Replaces the
 * reference's unified-memory fallback for graphs larger than the GPU
 * (include/graph_gpu.h:102-119).  Every pass over the columns then runs at
 * the host link's bandwidth instead of HBM's. */
#define MC_HOST_COLUMNS 0x2u
/* mc_dgraph_create* flag: keep the degree-ordered DAG (its entries and their
 * ranks) in pinned host memory as well, read by the counting kernels through
 * the device's mapping; implies MC_HOST_COLUMNS.  Chosen by itself when the
 * device cannot hold the DAG next to the per-vertex arrays even with the
 * columns on the host.  Only O(n) arrays (offsets, degrees, ranks, partner
 * records, task lists) and the core bitmaps stay in device memory: the
 * whole-CSR counterpart of the reference's unified-memory fallback
 * (include/graph_gpu.h:100-119).  Counting then reads partner lists across
 * the host link. */
#define MC_HOST_DAG 0x4u

/* Opaque handles. */
typedef struct mc_graph mc_graph_t;   /* host CSR (loaded or generated)      */
typedef struct mc_dgraph mc_dgraph_t; /* device-resident CSR + its scratch   */

/* Per-call device timings in milliseconds, measured with CUDA events on the
 * handle's stream.  Fields a call does not run are left at 0. */
typedef struct mc_timing {
  double h2d_ms;      /* host->device copy of the CSR (one-shot calls)       */
  double orient_ms;   /* degree order, DAG build, partner lists, task queue  */
  double count_ms;    /* counting kernels                                    */
  double d2h_ms;      /* device->host copy of the result                     */
  double total_ms;    /* first to last event of the call                     */
  double hub_ms;      /* share of count_ms spent in the hash (hub) kernel    */
  double leaf_ms;     /* share of count_ms spent in the warp (leaf) kernel   */
  int64_t launches;   /* kernels this call launched                          */
} mc_timing_t;

/* Sizes of the device preprocessing, for reporting and parity tests. */
typedef struct mc_tc_stats {
  int64_t n;             /* vertices                                         */
  int64_t nnz;           /* directed entries of the symmetric CSR (2m)       */
  int64_t dag_edges;     /* m+ = edges of the degree-ordered DAG             */
  int64_t max_out_degree;/* max d+ over the DAG                              */
  int64_t hub_tasks;     /* tasks routed to the CTA hash kernel              */
  int64_t leaf_tasks;    /* tasks routed to the warp kernel                  */
  int64_t partner_edges; /* DAG edges whose two ends both have d+ >= 1       */
  double probe_work;     /* sum over partner edges of the streamed list size */
} mc_tc_stats_t;

/* ---- status ------------------------------------------------------------- */
const char *mc_strerror(int status);
/* Library version string ("mercury_b200 <semver> sm_100a"). */
const char *mc_version(void);

/* ---- host graphs ---------------------------------------------------------
 * mc_graph_load replaces the reference loader Graph::Graph(prefix)
 * (graph.cc:6-35): reads <prefix>.meta.txt (10 whitespace fields: nv ne
 * vid_size eid_size vlabel_size elabel_size max_degree feat_len n_vclasses
 * n_eclasses), <prefix>.vertex.bin (int64[nv+1]) and <prefix>.edge.bin
 * (int32[ne]).  The reference asserts the field sizes and
 * 0 < max_degree < nv (graph.cc:24-28); this returns MC_ERR_FORMAT instead. */
int mc_graph_load(const char *prefix, mc_graph_t **out);
/* Writes the same three files (the layout the reference reader expects). */
int mc_graph_write(const mc_graph_t *g, const char *prefix);
/* Reads <prefix>.vlabel.bin, one uint8 label per vertex, into the graph:
 * the vertex-label part of the reference loader (graph.cc:37-58, with
 * use_vlabel).  MC_ERR_IO when the file is missing (the reference then draws
 * random labels; here the caller decides), MC_ERR_FORMAT when its size is
 * not n bytes. */
int mc_graph_load_vlabels(mc_graph_t *g, const char *prefix);
/* The graph's labels (n bytes, owned by the graph), or NULL if none. */
int mc_graph_vlabels(const mc_graph_t *g, const uint8_t **labels);
/* Wraps caller arrays into a host graph (copied; the caller keeps its own). */
int mc_graph_from_csr(const int64_t *rowptr, const int32_t *col, int64_t n,
                      int64_t nnz, mc_graph_t **out);
int mc_graph_info(const mc_graph_t *g, int64_t *n, int64_t *nnz,
                  int64_t *max_degree);
/* Borrowed pointers, valid until mc_graph_free. */
const int64_t *mc_graph_rowptr(const mc_graph_t *g);
const int32_t *mc_graph_col(const mc_graph_t *g);
/* Host-side contract check (sorted rows, ids in range, no self-loops and,
 * when check_symmetry != 0, symmetry).  MC_OK or MC_ERR_FORMAT. */
int mc_graph_validate(const mc_graph_t *g, int check_symmetry);
void mc_graph_free(mc_graph_t *g);

/* Seeded synthetic graphs (the reference ships only a closed converter
 * binary, datasets/converter.sh:5; these produce the same CSR layout).
 * RMAT: 2^scale vertices, edge_factor*2^scale draws of (a,b,c,1-a-b-c)
 * quadrant recursion, no noise, no relabelling; self-loops dropped,
 * symmetrised, deduplicated, sorted. */
int mc_gen_rmat(int scale, int edge_factor, double a, double b, double c,
                uint64_t seed, mc_graph_t **out);
/* Chung-Lu: weights w_i = (i+1)^(-1/(gamma-1)) scaled to mean_degree and
 * capped at max_weight; n*mean_degree/2 endpoint pairs drawn proportional to
 * w; self-loops and duplicates dropped. */
int mc_gen_chung_lu(int64_t n, double gamma, double mean_degree,
                    double max_weight, uint64_t seed, mc_graph_t **out);

/* ---- edge lists and the device CSR build --------------------------------
 * These replace the reference's dataset preparation. That is the closed
 * binary `converter mtx <file> <prefix> ...` (datasets/converter.sh:5), which
 * writes the CSR triple from a Matrix Market file, and datasets/tsv2mtx.py
 * (GraphChallenge TSV -> Matrix Market through a networkx Graph, i.e.
 * undirected with duplicates merged).
 * Parsing text is host work. Symmetrising, dropping self-loops, merging
 * duplicates, sorting rows and building the row offsets run on the device. */
typedef struct mc_edges mc_edges_t;   /* host edge list (pairs of int32 ids) */

#define MC_EDGES_MTX 1  /* Matrix Market "coordinate" file: '%' comment lines,
                           "rows cols entries", then one "i j [value]" per
                           entry; ids 1-based                              */
#define MC_EDGES_TSV 2  /* GraphChallenge TSV: "u<TAB>v[<TAB>w]" per line;
                           ids 1-based                                     */
#define MC_EDGES_SNAP 3 /* whitespace-separated "u v" per line, '#' comment
                           lines; ids 0-based                              */

/* Reads an edge list. id_base is the id of the first vertex in the file (0 or
 * 1); a negative id_base takes the format's default (1 for MTX and TSV, 0 for
 * SNAP). The reference's converter_vidfrom0 corresponds to MTX with
 * id_base 0.
 * The vertex count is max(rows, cols) from an MTX size line, or the
 * largest id seen + 1 - id_base when that is larger. Any id below id_base,
 * a value that is not an integer, a line with one field, or an MTX body
 * whose entry count differs from its size line is refused with
 * MC_ERR_FORMAT. "array" Matrix Market files are MC_ERR_UNSUPPORTED. */
int mc_edges_load(const char *path, int format, int id_base, mc_edges_t **out);
/* Copies caller arrays (ids already 0-based) into an edge list. */
int mc_edges_from_arrays(const int32_t *src, const int32_t *dst,
                         int64_t num_edges, int64_t n, mc_edges_t **out);
int mc_edges_info(const mc_edges_t *e, int64_t *num_edges, int64_t *n);
/* Borrowed pointers, valid until mc_edges_free. */
const int32_t *mc_edges_src(const mc_edges_t *e);
const int32_t *mc_edges_dst(const mc_edges_t *e);
void mc_edges_free(mc_edges_t *e);
/* The raw endpoint draws behind mc_gen_rmat / mc_gen_chung_lu, before any
 * symmetrising or merging (the same seed gives the same graph after a
 * CSR build). */
int mc_gen_rmat_edges(int scale, int edge_factor, double a, double b,
                      double c, uint64_t seed, mc_edges_t **out);
int mc_gen_chung_lu_edges(int64_t n, double gamma, double mean_degree,
                          double max_weight, uint64_t seed, mc_edges_t **out);

/* Flag of the CSR builds: src/dst are device pointers on the current device.
 * Otherwise they are host pointers and are copied in. */
#define MC_BUILD_DEVICE_INPUT 0x100u

/* Builds the symmetric CSR of the simple undirected graph on [0, n) given by
 * the pairs (src[i], dst[i]) on the current device, and returns it as a
 * host graph. Every pair u != v puts v in N(u) and u in N(v). Self-loops
 * are dropped, duplicates merged and rows sorted ascending, so the result
 * meets the graph contract above. An id outside [0, n) is refused with
 * MC_ERR_FORMAT. Replaces the converter's CSR construction. `stream` is a
 * cudaStream_t (NULL: a stream of the call's own). `timing` (may be NULL)
 * gets h2d_ms (input copy), count_ms (device build), d2h_ms (result copy),
 * total_ms and launches; its other fields are zero. */
int mc_csr_build(const int32_t *src, const int32_t *dst, int64_t num_edges,
                 int64_t n, unsigned flags, void *stream, mc_graph_t **out,
                 mc_timing_t *timing);
/* Same build, but the CSR stays on the device as a graph handle ready for
 * mc_tc_count / mc_pattern_count, with no host round trip. flags may also
 * hold MC_VALIDATE_SYMMETRY (the handle's contract check runs as in
 * mc_dgraph_create). timing->total_ms includes the handle's check. */
int mc_dgraph_from_edges(const int32_t *src, const int32_t *dst,
                         int64_t num_edges, int64_t n, unsigned flags,
                         void *stream, mc_dgraph_t **out,
                         mc_timing_t *timing);

/* ---- device graphs -------------------------------------------------------
 * mc_dgraph_create replaces GraphGPU::init / init_with_division
 * (include/graph_gpu.h:87-188): copies the symmetric CSR to the current
 * device and validates it there.  `stream` is a cudaStream_t (NULL: the
 * handle creates its own non-blocking stream).  The orientation
 * (Graph::orientation_with_division, graph.cc:196-321) is NOT done on the
 * host: mc_tc_count builds it on the device. */
int mc_dgraph_create(const int64_t *rowptr, const int32_t *col, int64_t n,
                     int64_t nnz, void *stream, unsigned flags,
                     mc_dgraph_t **out);
/* Same, from a CSR that already lives in device memory (copied into the
 * handle with device-to-device copies on the handle's stream). */
int mc_dgraph_create_device(const int64_t *d_rowptr, const int32_t *d_col,
                            int64_t n, int64_t nnz, void *stream,
                            unsigned flags, mc_dgraph_t **out);
/* The cudaStream_t every call on this handle is issued on. */
int mc_dgraph_stream(const mc_dgraph_t *g, void **stream);
/* Sizes of the handle's symmetric CSR (max_degree from its contract check). */
int mc_dgraph_info(const mc_dgraph_t *g, int64_t *n, int64_t *nnz,
                   int64_t *max_degree);
/* Copies the handle's symmetric CSR to host arrays of n+1 and nnz entries
 * (col_out may be NULL for the offsets only). */
int mc_dgraph_export_csr(const mc_dgraph_t *g, int64_t *rowptr_out,
                         int32_t *col_out);
/* *on_host = 1 when the handle's columns are in host memory
 * (MC_HOST_COLUMNS, asked for or chosen), else 0. */
int mc_dgraph_columns_on_host(const mc_dgraph_t *g, int *on_host);
/* *on_host = 1 if the handle keeps its DAG in host memory (MC_HOST_DAG,
 * asked for or chosen), else 0. */
int mc_dgraph_dag_on_host(const mc_dgraph_t *g, int *on_host);
void mc_dgraph_free(mc_dgraph_t *g);

/* Triangle count.  Replaces TCSolver(Graph&, uint64_t&) (tc_challenge.cu:11,
 * declared main.cc:3) and its two kernels hashIndex_for_large_degree and
 * binarySearch_for_small_degree (gpu_kernels/tc_challenge.cuh:4-303).
 * Device-side: degree-ordered DAG (u->v iff deg v > deg u, or equal degree
 * and v > u: graph.cc:207-214), then sum over DAG edges of
 * |N+(u) & N+(v)|.  Blocks until the count is on the host. */
int mc_tc_count(mc_dgraph_t *g, uint64_t *count, mc_timing_t *timing);
/* Partial triangle count over shard `shard` of `num_shards`: the counting
 * tasks are dealt round-robin to the shards, so the partial counts of
 * shards 0..num_shards-1 sum to mc_tc_count's result.  Each GPU of a
 * multi-GPU run holds the whole graph and counts its own shard; the partial
 * counts are then summed across ranks (the reference's MPI_Reduce,
 * tc_multigpu/tc_challenge_multigpu.cu:198-206). */
int mc_tc_count_shard(mc_dgraph_t *g, int shard, int num_shards,
                      uint64_t *partial, mc_timing_t *timing);
/* Preprocessing sizes of the last mc_tc_count on this handle. */
int mc_tc_stats(const mc_dgraph_t *g, mc_tc_stats_t *stats);
/* Copies the device-built DAG (after mc_tc_count) to host arrays of n+1
 * and dag_edges entries, for parity checks of the orientation.  With
 * col_out == NULL only the offsets are copied (rowptr_out[n] = dag_edges). */
int mc_dgraph_export_dag(const mc_dgraph_t *g, int64_t *rowptr_out,
                         int32_t *col_out);

/* Pattern count P<pattern> (1..8) over the symmetric graph.  Replaces the
 * single-rank path of SMSolverMultiGPU (subgraph_matching/sm_multigpu.cu:97,
 * kernels in subgraph_matching/pattern_kernels.cuh, combine at
 * sm_multigpu.cu:206-232): the same quantities over all 2m directed edges,
 * bit-exact, without MPI.  Uses per-warp frontier scratch of max_degree
 * entries per list, grown on first use and kept by the handle.  P7 and P8
 * on a graph with a vertex of degree above 4,096 (and none above 46,340,
 * where the reference's 32-bit products could wrap) are counted from the
 * triangles, K4s and K5s of the degree-ordered DAG instead of the per-edge
 * formulas: the same values, in time that grows with those clique counts
 * rather than with the cube of a hub's degree (MERCURY_CLIQUE_ROUTE=
 * cliques / formula forces either route). */
int mc_pattern_count(mc_dgraph_t *g, int pattern, uint64_t *count,
                     mc_timing_t *timing);
/* One shard of mc_pattern_count for multi-GPU runs with the graph
 * replicated on every GPU (the reference splits the edge list round-robin
 * across MPI ranks and reduces with MPI_Reduce, sm_multigpu.cu:12-95,
 * :206-232). Shard s of num_shards takes the centers v with
 * v mod num_shards == s, and the matching share of the remaining edge and
 * star tasks. Every pattern is c1 - c2 (or c1) of sums over edges and
 * vertices, so the num_shards partial results sum to the count modulo
 * 2^64. */
int mc_pattern_count_shard(mc_dgraph_t *g, int pattern, int shard,
                           int num_shards, uint64_t *partial,
                           mc_timing_t *timing);

/* mc_pattern_count with a time budget.  The count runs as a sequence of
 * launches over slices of its tasks, each sized from the previous one's
 * measured time to last about MERCURY_PATTERN_SLICE_MS (default 250 ms);
 * once the slices have used more than budget_ms of device time the count
 * stops between two slices and returns MC_ERR_TIMEOUT (count not written).
 * progress (optional) receives the fraction of the tasks done.  Graphs with
 * a maximum degree above 4,096 are counted in slices by mc_pattern_count too
 * (no budget): a hub edge alone can take seconds.  The reference has no
 * budget; its kernels run to the end (subgraph_matching/sm_multigpu.cu:
 * 150-200). */
int mc_pattern_count_budget(mc_dgraph_t *g, int pattern, double budget_ms,
                            uint64_t *count, double *progress,
                            mc_timing_t *timing);

/* Pattern count P<pattern> (1..8) of a symmetric CSR the caller already
 * holds in device memory (d_rowptr: int64[n+1], d_col: int32[nnz]), for
 * callers that cannot allocate device memory: a host application that owns
 * all of the GPU's memory through its own pool and forbids allocations
 * outside it, or a latency-bound caller that cannot afford cudaMalloc /
 * cudaFree (cudaFree waits for the whole device).  This entry point calls no
 * cudaMalloc, cudaFree or allocating library routine: its scratch (the
 * per-warp frontier lists and a few counter words) is a file-scope device
 * array of 32 MiB that every GPU loading this library holds until the
 * process exits.  Frontier lists need 6 x max_degree ints per warp, so
 * graphs whose maximum degree leaves room for fewer than 8 warps
 * (max_degree > 174762) are refused with MC_ERR_UNSUPPORTED; larger
 * degrees run fewer warps.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress) with that device current, and looks
 * it up again when the device's context has changed since (after a
 * cudaDeviceReset, which reloads the module holding the array); make the
 * first call on a device, and the first after a reset, before any stream
 * capture.  All calls share the array and its last contents (the counters
 * are cleared at the start of every call): calls whose work overlaps on the
 * GPU -- from two host threads, or on two streams -- race and must be
 * serialised by the caller.  `stream` is a cudaStream_t (NULL: the default
 * stream); the call returns after the count is on the host.  Vertex ids in
 * [0, n), ascending rows, no self-loops and monotone offsets are checked on
 * the device (MC_ERR_FORMAT); symmetry is NOT checked here, and the count of
 * a CSR that is not symmetric is meaningless (mc_graph_validate checks it on
 * the host).
 * No counterpart in the reference, which allocates its frontier with
 * cudaMalloc (subgraph_matching/sm_multigpu.cu:117-122). */
int mc_pattern_count_static(const int64_t *d_rowptr, const int32_t *d_col,
                            int64_t n, int64_t nnz, int pattern,
                            uint64_t *count, void *stream);

/* ---- batches ---------------------------------------------------------------
 * Many graphs counted in one captured CUDA-graph launch (no reference
 * counterpart: the reference runs TCSolver / SMSolverMultiGPU once per
 * graph).  The batch is one symmetric CSR, the disjoint union of the graphs:
 * graph g owns vertices [graph_vptr[g], graph_vptr[g+1]) (ids are global)
 * and no edge may join two graphs (MC_ERR_FORMAT).  jobs[g] is 0 for a
 * triangle count or 1..8 for pattern P1..P8.  Every count equals the
 * single-graph result (mc_tc_count / mc_pattern_count) of that graph. */
typedef struct mc_batch mc_batch_t;
int mc_batch_create(const int64_t *rowptr, const int32_t *col, int64_t n,
                    int64_t nnz, const int64_t *graph_vptr, int num_graphs,
                    const int32_t *jobs, void *stream, mc_batch_t **out);
/* Tunes the triangle schedule per degree bucket of the triangle graphs
 * (largest degree < 64, < 256, < 1024, >= 1024): the owner out-degree up to
 * which a task is one warp (else one CTA) and the table slots per key, each
 * from a small grid, by timing the bucket's graphs; re-captures the launch.
 * `choice` (optional, 8 ints) receives {threshold, log2 slots per key} per
 * bucket, -1 for empty buckets. */
int mc_batch_autotune(mc_batch_t *b, int32_t *choice);
/* counts[g] for every graph, from one replay of the captured launch. */
int mc_batch_count(mc_batch_t *b, uint64_t *counts, mc_timing_t *timing);
void mc_batch_free(mc_batch_t *b);

/* ---- vertex labels ----------------------------------------------------------
 * Labels live on the device beside the CSR, one uint8 per vertex, each at most
 * max_label (the reference's num_vertex_classes; vlabel_t is uint8,
 * include/common.h:33).  mc_dgraph_set_vlabels copies them (MC_ERR_FORMAT if
 * a label exceeds max_label).  The queries restate the reference's label
 * helpers on the device:
 *   mc_label_frequency: freq[l] = vertices of label l, l = 0..max_label
 *     (Graph::computeLabelsFrequency, graph.cc:440-460);
 *   mc_label_reverse_index: offsets[max_label + 2] and vertices[n], the
 *     vertices grouped by label in id order (Graph::BuildReverseIndex,
 *     graph.cc:413-436, getVerticesByLabel);
 *   mc_label_nlf: for v in [v_begin, v_end), row v - v_begin of
 *     (max_label + 1) counts of N(v)'s labels (Graph::BuildNLF,
 *     graph.cc:483-495, as a dense table instead of one map per vertex);
 *   mc_tc_count_by_label: counts[l] = the sum over DAG edges v -> u of
 *     |{w in N+(v) & N+(u) : label(w) = l}|, the reference's labelled
 *     intersection Graph::intersect_num(v, u, label) (graph.cc:396-411) over
 *     the degree-ordered DAG: triangles split by the label of their DAG sink
 *     (the vertex of largest (degree, id)), summing to the triangle count. */
int mc_dgraph_set_vlabels(mc_dgraph_t *g, const uint8_t *labels, int max_label);
int mc_label_frequency(mc_dgraph_t *g, uint64_t *freq);
int mc_label_reverse_index(mc_dgraph_t *g, int64_t *offsets, int32_t *vertices);
int mc_label_nlf(mc_dgraph_t *g, int64_t v_begin, int64_t v_end, uint32_t *nlf);
int mc_tc_count_by_label(mc_dgraph_t *g, uint64_t *counts, mc_timing_t *timing);

/* ---- serving ---------------------------------------------------------------
 * A request loop with continuous batching (no reference counterpart).
 * Worker threads (each with its own stream) take every queued request that
 * fits the HBM budget -- up to max_batch per batch, in arrival order, and
 * closing a batch once its estimated work (n + nnz per triangle job, the sum
 * of squared degrees per pattern job) would pass 2^23 entry visits
 * (MERCURY_SERVE_BATCH_WORK), or the queued work's share per worker when
 * that is larger; a request above 2^23 runs alone --
 * assemble the batch on the device, count it with the batch kernels and
 * deliver each graph's count; requests that arrive while batches run are
 * admitted as memory is returned, and batches of different workers overlap
 * on the device.  A request with a non-zero key leaves its CSR resident on
 * the device (within the budget, least recently used evicted first); later
 * requests with that key may pass NULL arrays.  A request that cannot fit
 * the budget even alone fails with MC_ERR_BUDGET.  Counts equal the
 * single-graph results. */
typedef struct mc_server mc_server_t;
typedef struct mc_server_stats {
  int64_t submitted, completed, failed, batches, cache_hits;
  int64_t cache_bytes, cached_graphs, queued, max_batch_seen;
} mc_server_stats_t;
int mc_server_create(int64_t hbm_budget_bytes, int max_batch, int workers,
                     mc_server_t **out);
/* Copies the graph (unless `key` is resident) and queues it; *ticket names
 * the request for mc_server_wait.  job: 0 triangles, 1..8 pattern P1..P8. */
int mc_server_submit(mc_server_t *s, const int64_t *rowptr, const int32_t *col,
                     int64_t n, int64_t nnz, int job, uint64_t key,
                     uint64_t *ticket);
/* Waits up to timeout_ms (MC_ERR_TIMEOUT after that; the ticket stays
 * valid); on completion returns the request's status, its count and its
 * latency from submission to result. */
int mc_server_wait(mc_server_t *s, uint64_t ticket, int timeout_ms,
                   uint64_t *count, double *latency_ms);
int mc_server_stats(mc_server_t *s, mc_server_stats_t *stats);
/* Finishes the queued requests, stops the workers, frees the cache. */
void mc_server_free(mc_server_t *s);

/* One-shot drop-in for TCSolver: host CSR in, count out.  Uploads, orients,
 * counts and copies the result back inside the call (timing->h2d_ms etc.).
 * Device buffers are cached in a per-thread context and reused while the
 * graph fits, so repeated calls do not re-allocate.  A graph the device
 * cannot hold is counted with its columns in host memory (MC_HOST_COLUMNS);
 * that context is kept while later graphs also need it. */
int mc_tc_count_host(const int64_t *rowptr, const int32_t *col, int64_t n,
                     int64_t nnz, uint64_t *count, mc_timing_t *timing);

#ifdef __cplusplus
}
#endif
#endif /* MERCURY_B200_H */

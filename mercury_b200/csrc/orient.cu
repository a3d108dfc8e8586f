// Device preprocessing of the triangle-count path: contract validation,
// degree-ordered DAG build and the owner->partner lists, all as streaming
// row-aware compactions of the symmetric CSR.
//
// Reference behaviour restated here: Graph::orientation_with_division
// (graph.cc:196-321) runs on the host with OpenMP in five passes.  The DAG
// rule is the same (u->v iff deg v > deg u, or equal and v > u:
// graph.cc:207-214).  The reference then splits edges into a "small" CSR
// (DAG direction, both out-degrees <= 128) and a "large" CSR (REVERSE_DAG:
// from the endpoint with the larger DAG out-degree, ties to the larger id,
// graph.cc:238-263), skipping edges with an endpoint of out-degree 0
// (graph.cc:246).  Here every DAG edge with both out-degrees >= 1 goes to the
// owner list of its larger-out-degree end (the reference's "large" rule for
// all edges), because the counting kernels always hash the owner's list and
// stream the partner's shorter list; the small/large routing is made per
// owner instead (d+ <= kLeafMaxOut: warp task, else CTA task).
#include <algorithm>
#include <cstdio>

#include "dgraph.cuh"
#include "device_common.cuh"
#include "scan.cuh"

namespace mc {
namespace {

// ---- predicates over one CSR entry (v -> u) ------------------------------

// Degree-ordered orientation: keep u in N+(v).
struct DagPred {
  const int32_t *deg;
  __device__ __forceinline__ int32_t row_value(int64_t v) const { return __ldg(deg + v); }
  __device__ __forceinline__ bool operator()(int64_t v, int32_t dv, int32_t u) const {
    int32_t du = __ldg(deg + u);
    return du > dv || (du == dv && u > (int32_t)v);
  }
};

// Owner rule: the end with the larger DAG out-degree owns the edge (ties to
// the larger id); edges touching an out-degree-0 end are dropped.
struct OwnerPred {
  const int32_t *dplus;
  __device__ __forceinline__ int32_t row_value(int64_t v) const { return __ldg(dplus + v); }
  __device__ __forceinline__ bool operator()(int64_t v, int32_t pv, int32_t u) const {
    if (pv < 1) return false;
    int32_t pu = __ldg(dplus + u);
    return pu >= 1 && (pv > pu || (pv == pu && (int32_t)v > u));
  }
};

__device__ __forceinline__ void load_span(const int32_t *__restrict__ col, int64_t s, int64_t nnz,
                                          int32_t (&vals)[kEdgesPerThread]) {
  if (s + kEdgesPerThread <= nnz) {
    const int4 *p = reinterpret_cast<const int4 *>(col + s);
#pragma unroll
    for (int k = 0; k < kEdgesPerThread / 4; ++k) {
      int4 q = __ldg(p + k);
      vals[4 * k] = q.x;
      vals[4 * k + 1] = q.y;
      vals[4 * k + 2] = q.z;
      vals[4 * k + 3] = q.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < kEdgesPerThread; ++k) vals[k] = s + k < nnz ? __ldg(col + s + k) : 0;
  }
}

// Row range [lo, hi] that covers the CSR entries of this tile.
__device__ __forceinline__ void tile_rows(const int64_t *rowptr, int64_t n, int64_t t0, int64_t t1,
                                          int64_t *lo, int64_t *hi) {
  __shared__ int64_t sh[2];
  if (threadIdx.x == 0) sh[0] = upper_row(rowptr, 0, n - 1, t0);
  if (threadIdx.x == kTileThreads - 1) sh[1] = upper_row(rowptr, 0, n - 1, t1 - 1);
  __syncthreads();
  *lo = sh[0];
  *hi = sh[1];
}

__device__ __forceinline__ int block_sum_int(int v) {
  __shared__ int ws[kTileThreads / kWarp];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
  if (lane == 0) ws[wid] = v;
  __syncthreads();
  int t = 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < kTileThreads / kWarp; ++i) t += ws[i];
  return t;
}

__device__ __forceinline__ int block_exclusive_int(int v) {
  __shared__ int ws[kTileThreads / kWarp];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = warp_inclusive_scan(v, lane);
  if (lane == 31) ws[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int w = lane < kTileThreads / kWarp ? ws[lane] : 0;
    w = warp_inclusive_scan(w, lane);
    if (lane < kTileThreads / kWarp) ws[lane] = w;
  }
  __syncthreads();
  return (wid ? ws[wid - 1] : 0) + x - v;
}

// Pass 1 (kWrite == false): tile_counts[tile] = kept entries in the tile.
// Pass 2 (kWrite == true): stable compaction of the kept entries into
// out_col and out_rowptr[r] = kept entries before rowptr[r], for every row.
template <class Pred, bool kWrite>
__global__ void __launch_bounds__(kTileThreads)
    compact_kernel(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ col, int64_t n,
                   int64_t nnz, Pred pred, int32_t *tile_counts, const int64_t *tile_offsets,
                   int64_t *out_rowptr, int32_t *out_col) {
  const int64_t t0 = (int64_t)blockIdx.x * kTileEdges;
  const int64_t t1 = min(t0 + kTileEdges, nnz);
  int64_t rlo, rhi;
  tile_rows(rowptr, n, t0, t1, &rlo, &rhi);
  const int64_t s = t0 + (int64_t)threadIdx.x * kEdgesPerThread;
  const int64_t e_end = min(s + kEdgesPerThread, t1);
  int32_t vals[kEdgesPerThread];
  unsigned keep = 0;
  int64_t r = 0;
  if (s < t1) {
    load_span(col, s, nnz, vals);
    r = upper_row(rowptr, rlo, rhi, s);
    int64_t next = __ldg(rowptr + r + 1);
    int64_t v = r;
    int32_t pv = pred.row_value(v);
#pragma unroll
    for (int k = 0; k < kEdgesPerThread; ++k) {
      const int64_t e = s + k;
      if (e < e_end) {
        while (e == next) {
          ++v;
          next = __ldg(rowptr + v + 1);
          pv = pred.row_value(v);
        }
        if (pred(v, pv, vals[k])) keep |= 1u << k;
      }
    }
  }
  const int cnt = __popc(keep);
  if (!kWrite) {
    int t = block_sum_int(cnt);
    if (threadIdx.x == 0) tile_counts[blockIdx.x] = t;
    return;
  }
  int64_t pos = tile_offsets[blockIdx.x] + block_exclusive_int(cnt);
  if (s >= t1) return;
  // Rows that start exactly at s (empty rows before r included) start here.
  if (__ldg(rowptr + r) == s) {
    int64_t rf = lower_row(rowptr, 0, r, s);
    for (int64_t q = rf; q <= r; ++q) out_rowptr[q] = pos;
  }
  int64_t next = __ldg(rowptr + r + 1);
#pragma unroll
  for (int k = 0; k < kEdgesPerThread; ++k) {
    const int64_t e = s + k;
    if (e < e_end) {
      while (e == next) {
        ++r;
        out_rowptr[r] = pos;
        next = __ldg(rowptr + r + 1);
      }
      if (keep & (1u << k)) out_col[pos++] = vals[k];
    }
  }
  // Rows that start at nnz (trailing empty rows and r == n) get the total.
  if (e_end == nnz)
    for (int64_t q = r + 1; q <= n; ++q) out_rowptr[q] = pos;
}

// Contract checks that need the row of each entry: ids in range, strictly
// ascending rows, no self-loops, and (optionally) symmetry.
__global__ void __launch_bounds__(kTileThreads)
    validate_entries_kernel(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ col,
                            int64_t n, int64_t nnz, int check_sym, unsigned *err) {
  const int64_t t0 = (int64_t)blockIdx.x * kTileEdges;
  const int64_t t1 = min(t0 + kTileEdges, nnz);
  int64_t rlo, rhi;
  tile_rows(rowptr, n, t0, t1, &rlo, &rhi);
  const int64_t s = t0 + (int64_t)threadIdx.x * kEdgesPerThread;
  const int64_t e_end = min(s + kEdgesPerThread, t1);
  if (s >= t1) return;
  int64_t v = upper_row(rowptr, rlo, rhi, s);
  int64_t start = __ldg(rowptr + v), next = __ldg(rowptr + v + 1);
  unsigned bad = 0;
  for (int64_t e = s; e < e_end; ++e) {
    while (e == next) {
      ++v;
      start = next;
      next = __ldg(rowptr + v + 1);
    }
    const int32_t u = __ldg(col + e);
    if (u < 0 || (int64_t)u >= n) {
      bad |= kErrIdRange;
      continue;
    }
    if ((int64_t)u == v) bad |= kErrSelfLoop;
    if (e > start && __ldg(col + e - 1) >= u) bad |= kErrUnsorted;
    if (check_sym) {
      // v must appear in N(u) (binary search; rows are checked sorted).
      int64_t lo = __ldg(rowptr + u), hi = __ldg(rowptr + u + 1) - 1;
      bool found = false;
      while (lo <= hi && lo >= 0 && hi < nnz) {
        int64_t mid = lo + ((hi - lo) >> 1);
        int32_t m = __ldg(col + mid);
        if (m == (int32_t)v) { found = true; break; }
        if (m < (int32_t)v) lo = mid + 1; else hi = mid - 1;
      }
      if (!found) bad |= kErrAsymmetric;
    }
  }
  if (bad) atomicOr(err, bad);
}

__global__ void validate_rowptr_kernel(const int64_t *rowptr, int64_t n, int64_t nnz, unsigned *err) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v > n) return;
  const int64_t a = rowptr[v];
  bool bad = (v == 0 && a != 0) || (v == n && a != nnz) || a < 0 || a > nnz;
  if (v < n && rowptr[v + 1] < a) bad = true;
  if (bad) atomicOr(err, (unsigned)kErrRowptr);
}

__global__ void degree_kernel(const int64_t *rowptr, int64_t n, int32_t *deg) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) deg[v] = (int32_t)(rowptr[v + 1] - rowptr[v]);
}

__global__ void dplus_kernel(const int64_t *dag_rowptr, int64_t n, int32_t *dplus,
                             unsigned long long *max_out) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int32_t d = 0;
  if (v < n) {
    d = (int32_t)(dag_rowptr[v + 1] - dag_rowptr[v]);
    dplus[v] = d;
  }
  // Warp max, then one atomic per warp.
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) d = max(d, __shfl_down_sync(kFull, d, o));
  if ((threadIdx.x & 31) == 0 && d > 0) atomicMax(max_out, (unsigned long long)d);
}

// Number of tasks each owner contributes to the hub and leaf queues.
__global__ void task_count_kernel(const int64_t *prt_rowptr, const int32_t *dplus, int64_t n,
                                  int32_t *hub_cnt, int32_t *leaf_cnt) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const int64_t p = prt_rowptr[v + 1] - prt_rowptr[v];
  const int32_t d = dplus[v];
  int32_t h = 0, l = 0;
  if (p > 0) {
    if (d > kLeafMaxOut) h = (int32_t)((p + kHubChunk - 1) / kHubChunk);
    else l = (int32_t)((p + kLeafChunk - 1) / kLeafChunk);
  }
  hub_cnt[v] = h;
  leaf_cnt[v] = l;
}

// Task word: owner id in the high half, chunk index in the low half.
__global__ void task_fill_kernel(const int32_t *hub_cnt, const int64_t *hub_off,
                                 const int32_t *leaf_cnt, const int64_t *leaf_off, int64_t n,
                                 uint64_t *hub_tasks, uint64_t *leaf_tasks) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const uint64_t hi = (uint64_t)v << 32;
  for (int32_t c = 0, h = hub_cnt[v]; c < h; ++c) hub_tasks[hub_off[v] + c] = hi | (uint32_t)c;
  for (int32_t c = 0, l = leaf_cnt[v]; c < l; ++c) leaf_tasks[leaf_off[v] + c] = hi | (uint32_t)c;
}

unsigned grid_for(int64_t items, int threads) {
  return (unsigned)std::max<int64_t>(1, (items + threads - 1) / threads);
}

template <class Pred>
int compact(mc_dgraph *g, Pred pred, int64_t *out_rowptr, int32_t *out_col) {
  const int64_t tiles = (g->nnz + kTileEdges - 1) / kTileEdges;
  if (tiles == 0) {
    MC_CUDA_TRY(cudaMemsetAsync(out_rowptr, 0, sizeof(int64_t) * (g->n + 1), g->stream));
    return MC_OK;
  }
  g->launches += 2 + scan_launches(tiles);
  compact_kernel<Pred, false><<<(unsigned)tiles, kTileThreads, 0, g->stream>>>(
      g->rowptr, g->col, g->n, g->nnz, pred, g->tile_counts, nullptr, nullptr, nullptr);
  MC_CUDA_TRY(cudaGetLastError());
  MC_CUDA_TRY(exclusive_scan(g->tile_counts, g->tile_offsets, tiles, g->scan_temp, g->stream));
  compact_kernel<Pred, true><<<(unsigned)tiles, kTileThreads, 0, g->stream>>>(
      g->rowptr, g->col, g->n, g->nnz, pred, nullptr, g->tile_offsets, out_rowptr, out_col);
  MC_CUDA_TRY(cudaGetLastError());
  return MC_OK;
}

}  // namespace

int validate_graph(mc_dgraph *g, unsigned flags) {
  MC_CUDA_TRY(cudaMemsetAsync(g->err, 0, sizeof(unsigned), g->stream));
  validate_rowptr_kernel<<<grid_for(g->n + 1, 256), 256, 0, g->stream>>>(g->rowptr, g->n, g->nnz,
                                                                        g->err);
  MC_CUDA_TRY(cudaGetLastError());
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_err, g->err, sizeof(unsigned), cudaMemcpyDeviceToHost, g->stream));
  MC_CUDA_TRY(cudaStreamSynchronize(g->stream));
  if (*g->h_err) return MC_ERR_FORMAT;  // the entry walk needs monotone offsets
  const int64_t tiles = (g->nnz + kTileEdges - 1) / kTileEdges;
  g->launches += 1 + (tiles > 0 ? 1 : 0);
  if (tiles > 0) {
    validate_entries_kernel<<<(unsigned)tiles, kTileThreads, 0, g->stream>>>(
        g->rowptr, g->col, g->n, g->nnz, (flags & MC_VALIDATE_SYMMETRY) ? 1 : 0, g->err);
    MC_CUDA_TRY(cudaGetLastError());
  }
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_err, g->err, sizeof(unsigned), cudaMemcpyDeviceToHost, g->stream));
  MC_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return *g->h_err ? MC_ERR_FORMAT : MC_OK;
}

int tc_alloc(mc_dgraph *g) {
  if (g->tc_ready) return MC_OK;
  const int64_t n = g->n, cap = std::max<int64_t>(g->nnz, 1);
  const int64_t tiles = std::max<int64_t>((g->nnz + kTileEdges - 1) / kTileEdges, 1);
  // Each owner contributes at most ceil(p / chunk) <= 1 + p / chunk tasks.
  g->task_capacity = n + cap / std::min(kHubChunk, kLeafChunk) + 1;
  g->scan_temp_size = std::max(scan_temp_bytes(n + 1), scan_temp_bytes(tiles + 1));
#define MC_ALLOC(ptr, count) MC_CUDA_TRY(cudaMalloc((void **)&(ptr), sizeof(*(ptr)) * (size_t)(count)))
  MC_ALLOC(g->deg, n + 1);
  MC_ALLOC(g->dplus, n + 1);
  MC_ALLOC(g->dag_rowptr, n + 1);
  MC_ALLOC(g->dag_col, cap);
  MC_ALLOC(g->prt_rowptr, n + 1);
  MC_ALLOC(g->prt_col, cap);
  MC_ALLOC(g->tile_counts, tiles);
  MC_ALLOC(g->tile_offsets, tiles + 1);
  MC_ALLOC(g->hub_cnt, n + 1);
  MC_ALLOC(g->leaf_cnt, n + 1);
  MC_ALLOC(g->hub_off, n + 1);
  MC_ALLOC(g->leaf_off, n + 1);
  MC_ALLOC(g->hub_tasks, g->task_capacity);
  MC_ALLOC(g->leaf_tasks, g->task_capacity);
  MC_CUDA_TRY(cudaMalloc(&g->scan_temp, g->scan_temp_size));
#undef MC_ALLOC
  g->tc_ready = true;
  return MC_OK;
}

int tc_orient(mc_dgraph *g) {
  const int64_t n = g->n;
  cudaStream_t s = g->stream;
  MC_CUDA_TRY(cudaMemsetAsync(g->counters, 0, sizeof(unsigned long long) * 8, s));
  if (n == 0) return MC_OK;
  g->launches += 4 + 2 * scan_launches(n);  // degree, d+, task count/fill, 2 scans
  degree_kernel<<<grid_for(n, 256), 256, 0, s>>>(g->rowptr, n, g->deg);
  MC_CUDA_TRY(cudaGetLastError());
  int rc = compact(g, DagPred{g->deg}, g->dag_rowptr, g->dag_col);
  if (rc != MC_OK) return rc;
  dplus_kernel<<<grid_for(n, 256), 256, 0, s>>>(g->dag_rowptr, n, g->dplus, g->counters + 3);
  MC_CUDA_TRY(cudaGetLastError());
  rc = compact(g, OwnerPred{g->dplus}, g->prt_rowptr, g->prt_col);
  if (rc != MC_OK) return rc;
  task_count_kernel<<<grid_for(n, 256), 256, 0, s>>>(g->prt_rowptr, g->dplus, n, g->hub_cnt,
                                                     g->leaf_cnt);
  MC_CUDA_TRY(cudaGetLastError());
  MC_CUDA_TRY(exclusive_scan(g->hub_cnt, g->hub_off, n, g->scan_temp, s));
  MC_CUDA_TRY(exclusive_scan(g->leaf_cnt, g->leaf_off, n, g->scan_temp, s));
  task_fill_kernel<<<grid_for(n, 256), 256, 0, s>>>(g->hub_cnt, g->hub_off, g->leaf_cnt,
                                                    g->leaf_off, n, g->hub_tasks, g->leaf_tasks);
  MC_CUDA_TRY(cudaGetLastError());
  return MC_OK;
}

}  // namespace mc

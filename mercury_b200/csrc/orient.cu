// Device preprocessing of the triangle-count path: contract validation and
// the degree-ordered DAG, built by two streaming row-aware passes over the
// symmetric CSR, plus the counting task queues.
//
// Reference behaviour restated here: Graph::orientation_with_division
// (graph.cc:196-321) runs on the host with OpenMP in five passes.  The DAG
// rule is the same (u->v iff deg v > deg u, or equal and v > u:
// graph.cc:207-214).  The reference then splits edges into a "small" CSR
// (DAG direction, both out-degrees <= 128) and a "large" CSR (REVERSE_DAG:
// from the endpoint with the larger DAG out-degree, ties to the larger id,
// graph.cc:238-263), skipping edges with an endpoint of out-degree 0
// (graph.cc:246).  Here every DAG edge with both out-degrees >= 1 belongs to
// its larger-out-degree end (the reference's "large" rule for all edges);
// the counting kernels find an owner's partners by filtering the owner's own
// symmetric row, so no partner CSR is written.  Routing is per owner
// (d+ <= kLeafMaxOut: warp task, else CTA task).
//
// Passes (each CTA owns a tile of kTileEdges consecutive CSR entries and
// stages the tile's row offsets in shared memory):
//   A  DAG keep masks, per-tile DAG counts, d+ of every row by atomics
//   B  DAG entries and row offsets written from the keep masks
// Each vertex's (degree, d+) pair is one 8-byte word (key[]).
#include <algorithm>
#include <cstring>
#include <climits>
#include <cstdio>
#include <cstdlib>

#include "dgraph.cuh"
#include "device_common.cuh"
#include "radix.cuh"
#include "scan.cuh"

namespace mc {
namespace {

constexpr int kSegMax = 2048;  // row offsets of a tile kept in shared memory

// The span's entries from p (16-byte aligned), `avail` of them valid.
__device__ __forceinline__ void load_span(const int32_t *__restrict__ p32, int64_t avail,
                                          int32_t (&vals)[kEdgesPerThread]) {
  if (avail >= kEdgesPerThread) {
    const int4 *p = reinterpret_cast<const int4 *>(p32);
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
    for (int k = 0; k < kEdgesPerThread; ++k) vals[k] = k < avail ? __ldg(p32 + k) : 0;
  }
}

// Row offsets of one tile: rows [lo, hi] hold the tile's entries; when the
// segment rowptr[lo .. hi+1] fits it is read from shared memory.
struct TileRows {
  const int64_t *g;
  const int64_t *s;
  int64_t lo, hi;
  __device__ __forceinline__ int64_t at(int64_t r) const { return s ? s[r - lo] : __ldg(g + r); }
  // Largest r in [lo, hi] with rowptr[r] <= key.
  __device__ __forceinline__ int64_t row_of(int64_t key) const {
    int64_t a = lo, b = hi;
    while (a < b) {
      int64_t mid = a + ((b - a + 1) >> 1);
      if (at(mid) <= key) a = mid;
      else b = mid - 1;
    }
    return a;
  }
  // Smallest r in [a, b] with rowptr[r] >= key (rowptr[b] >= key).
  __device__ __forceinline__ int64_t first_at(int64_t a, int64_t b, int64_t key) const {
    while (a < b) {
      int64_t mid = a + ((b - a) >> 1);
      if (at(mid) >= key) b = mid;
      else a = mid + 1;
    }
    return a;
  }
};

// rows (optional): {first row, last row} of this tile, precomputed by
// tile_rows_kernel; without it two threads binary-search rowptr (22
// dependent loads at n = 4 M, which the rest of the CTA waits for).
__device__ __forceinline__ TileRows load_tile_rows(const int64_t *rowptr, int64_t n, int64_t t0,
                                                   int64_t t1, int64_t *seg,
                                                   const int64_t *rows = nullptr) {
  __shared__ int64_t sh[2];
  if (rows) {
    if (threadIdx.x < 2) sh[threadIdx.x] = __ldg(rows + threadIdx.x);
  } else {
    if (threadIdx.x == 0) sh[0] = upper_row(rowptr, 0, n - 1, t0);
    if (threadIdx.x == kTileThreads - 1) sh[1] = upper_row(rowptr, 0, n - 1, t1 - 1);
  }
  __syncthreads();
  TileRows tr{rowptr, nullptr, sh[0], sh[1]};
  const int64_t len = tr.hi - tr.lo + 2;
  if (len <= kSegMax) {
    for (int64_t i = threadIdx.x; i < len; i += kTileThreads) seg[i] = __ldg(rowptr + tr.lo + i);
    __syncthreads();
    tr.s = seg;
  }
  return tr;
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

// Exclusive prefix of v over the block; *total receives the block sum.
__device__ __forceinline__ int block_exclusive_int(int v, int *total) {
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
  *total = ws[kTileThreads / kWarp - 1];
  return (wid ? ws[wid - 1] : 0) + x - v;
}

// Writes the kept entries of this thread's span [s, e_end) (row r holds s)
// from position pos on, and out_rowptr[q] = position for every row q that
// starts inside the span.  Rows starting at nnz are written by the caller.
// kStage: the entries go to stage[pos - stage_base] in shared memory (the
// caller copies the tile's range out, coalesced, and gathers the ranks
// there); otherwise straight to out_col / out_rank.
template <bool kStage>
__device__ __forceinline__ void write_span(const TileRows &tr, const int64_t *rowptr, int64_t t0,
                                           int64_t s, int64_t e_end, int64_t r,
                                           const int32_t (&vals)[kEdgesPerThread], unsigned keep,
                                           int64_t pos, int64_t *out_rowptr, int32_t *out_col,
                                           const int32_t *__restrict__ rank, int32_t *out_rank,
                                           int32_t *stage, int64_t stage_base) {
  if (tr.at(r) == s) {
    // Rows starting exactly at s: row r and the empty rows just before it.
    // For s > t0 they all lie in the staged range; the tile's first span may
    // share its start with rows before the range.
    const int64_t rf = s == t0 ? lower_row(rowptr, 0, r, s) : tr.first_at(tr.lo, r, s);
    for (int64_t q = rf; q <= r; ++q) out_rowptr[q] = pos;
  }
  // The ranks of the kept entries, gathered before the row walk so that
  // they are all in flight at once.
  int32_t ranks[kEdgesPerThread];
  if (!kStage) {
#pragma unroll
    for (int k = 0; k < kEdgesPerThread; ++k)
      ranks[k] = out_rank && (keep & (1u << k)) ? __ldg(rank + vals[k]) : 0;
  }
  int64_t next = tr.at(r + 1);
#pragma unroll
  for (int k = 0; k < kEdgesPerThread; ++k) {
    const int64_t e = s + k;
    if (e < e_end) {
      while (e == next) {
        ++r;
        out_rowptr[r] = pos;
        next = tr.at(r + 1);
      }
      if (keep & (1u << k)) {
        if (kStage) {
          stage[pos - stage_base] = vals[k];
        } else {
          out_col[pos] = vals[k];
          if (out_rank) out_rank[pos] = ranks[k];
        }
        ++pos;
      }
    }
  }
}

// Where a pass finds its tiles' column entries: the whole array (col_base
// 0, tile_base 0), or a staged chunk of it holding entries from col_base on
// for the tiles from tile_base on (chunks start on tile boundaries).
struct ColumnChunk {
  const int32_t *col;
  int64_t col_base;
  int64_t tile_base;
};

// Pass A (kWrite == false): DAG entries of every thread's span as a 16-bit
// mask in keep[], per-tile counts, and d+ of every row by atomics on
// key[].y (which starts at 0).  Pass B (kWrite == true): the kept entries
// compacted into out_col (and, when rank is given, their ranks into
// out_rank) and out_rowptr[r] = kept entries before rowptr[r].  With
// chunk_end given, pass B writes nothing when *chunk_end (the DAG entries
// up to the end of this chunk) exceeds cap; with stop given, neither pass
// does anything once a contract bit is set there.
template <bool kWrite, bool kStage = false>
__global__ void __launch_bounds__(kTileThreads)
    dag_pass_kernel(const int64_t *__restrict__ rowptr, ColumnChunk cc,
                    const int32_t *__restrict__ deg, int64_t n, int64_t nnz, int2 *key,
                    uint16_t *keep_masks, int32_t *counts_out,
                    const int64_t *__restrict__ offs_in, int64_t *out_rowptr, int32_t *out_col,
                    const int32_t *__restrict__ rank, int32_t *out_rank,
                    const int64_t *chunk_end, int64_t cap, const unsigned *stop,
                    const int64_t *__restrict__ tile_rows) {
  __shared__ int64_t seg[kSegMax];
  // Both checks read one word, the same for the whole CTA.  `stop`: the
  // contract checks of a chunk validated just before found a bad entry, so
  // no id is gathered or written.
  if (stop && (*(volatile const unsigned *)stop & kErrContract)) return;
  if (kWrite && chunk_end && *chunk_end > cap) return;
  const int64_t tile = cc.tile_base + blockIdx.x;
  const int64_t t0 = tile * kTileEdges;
  const int64_t t1 = min(t0 + kTileEdges, nnz);
  const TileRows tr =
      load_tile_rows(rowptr, n, t0, t1, seg, tile_rows ? tile_rows + 2 * tile : nullptr);
  const int64_t s = t0 + (int64_t)threadIdx.x * kEdgesPerThread;
  const int64_t e_end = min(s + kEdgesPerThread, t1);
  const int64_t slot = tile * kTileThreads + threadIdx.x;
  int32_t vals[kEdgesPerThread];
  unsigned keep = 0;
  int64_t r = 0;
  if (s < t1) {
    load_span(cc.col + (s - cc.col_base), nnz - s, vals);
    r = tr.row_of(s);
    if (!kWrite) {
      // All sixteen degree gathers are issued before the row walk below
      // (whose loop would otherwise serialise them); entries past the span
      // hold id 0, a valid vertex.
      int du[kEdgesPerThread];
#pragma unroll
      for (int k = 0; k < kEdgesPerThread; ++k) du[k] = __ldg(deg + vals[k]);
      int64_t v = r, next = tr.at(r + 1);
      int dv = __ldg(deg + v);
      int run = 0;  // DAG entries of row v seen in this span
#pragma unroll
      for (int k = 0; k < kEdgesPerThread; ++k) {
        const int64_t e = s + k;
        if (e < e_end) {
          while (e == next) {
            if (run) {
              atomicAdd(&key[v].y, run);
              run = 0;
            }
            ++v;
            next = tr.at(v + 1);
            dv = __ldg(deg + v);
          }
          const int u = vals[k];
          if (du[k] > dv || (du[k] == dv && u > (int)v)) {
            keep |= 1u << k;
            ++run;
          }
        }
      }
      if (run) atomicAdd(&key[v].y, run);
      keep_masks[slot] = (uint16_t)keep;
    } else {
      keep = keep_masks[slot];
    }
  }
  if (!kWrite) {
    const int t = block_sum_int(__popc(keep));
    if (threadIdx.x == 0) counts_out[tile] = t;
    return;
  }
  int total = 0;
  const int64_t base = offs_in[tile];
  const int64_t pos = base + block_exclusive_int(__popc(keep), &total);
  if (kStage) {
    // The tile's DAG entries are the range [base, base + total): staged in
    // shared memory, then written with whole-line stores, the rank gathers
    // issued four per thread at a time.
    __shared__ int32_t stage[kTileEdges];
    if (s < t1)
      write_span<true>(tr, rowptr, t0, s, e_end, r, vals, keep, pos, out_rowptr, nullptr,
                       nullptr, nullptr, stage, base);
    __syncthreads();
#pragma unroll 4
    for (int i = threadIdx.x; i < total; i += kTileThreads) {
      const int32_t c = stage[i];
      out_col[base + i] = c;
      if (out_rank) out_rank[base + i] = __ldg(rank + c);
    }
  } else if (s < t1) {
    write_span<false>(tr, rowptr, t0, s, e_end, r, vals, keep, pos, out_rowptr, out_col, rank,
                      out_rank, nullptr, 0);
  }
  // Rows after the last entry (trailing empty rows and q == n) start at nnz.
  if (t1 == nnz)
    for (int64_t q = tr.hi + 1 + threadIdx.x; q <= n; q += kTileThreads) out_rowptr[q] = base + total;
}

// rows[2t] / rows[2t + 1] = the rows holding the first and the last entry of
// tile t: each non-empty row marks the tiles whose first or last entry it
// holds (rowptr validated: monotone, ends at nnz).
__global__ void tile_rows_kernel(const int64_t *__restrict__ rowptr, int64_t n, int64_t nnz,
                                 int64_t tiles, int64_t *rows) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const int64_t b = rowptr[v], e = rowptr[v + 1];
  if (b >= e) return;
  for (int64_t t = b / kTileEdges; t <= (e - 1) / kTileEdges && t < tiles; ++t) {
    const int64_t first = t * kTileEdges;
    const int64_t last = min(first + kTileEdges, nnz) - 1;
    if (first >= b && first < e) rows[2 * t] = v;
    if (last >= b && last < e) rows[2 * t + 1] = v;
  }
}

// Tile offsets of one staged chunk: offs[0] holds the DAG entries of the
// earlier chunks; offs[i] = offs[0] + local[i] for i in [0, count] (local is
// the chunk's exclusive scan, local[0] = 0, so offs[0] is rewritten with its
// own value). The chunk's end above cap raises kErrDagCapacity.
__global__ void chunk_offsets_kernel(const int64_t *__restrict__ local, int64_t count,
                                     int64_t *offs, int64_t cap, unsigned *err) {
  const int64_t base = offs[0];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > count) return;
  const int64_t v = base + local[i];
  offs[i] = v;
  if (i == count && v > cap) atomicOr(err, (unsigned)kErrDagCapacity);
}

// Contract checks that need the row of each entry: ids in range, strictly
// ascending rows, no self-loops, and (optionally) symmetry.
__global__ void __launch_bounds__(kTileThreads)
    validate_entries_kernel(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ col,
                            int64_t n, int64_t nnz, int check_sym, unsigned *err,
                            int64_t tile_base, const int64_t *__restrict__ tile_rows = nullptr) {
  __shared__ int64_t seg[kSegMax];
  const int64_t tile = tile_base + blockIdx.x;
  const int64_t t0 = tile * kTileEdges;
  const int64_t t1 = min(t0 + kTileEdges, nnz);
  const TileRows tr =
      load_tile_rows(rowptr, n, t0, t1, seg, tile_rows ? tile_rows + 2 * tile : nullptr);
  const int64_t s = t0 + (int64_t)threadIdx.x * kEdgesPerThread;
  const int64_t e_end = min(s + kEdgesPerThread, t1);
  if (s >= t1) return;
  int64_t v = tr.row_of(s);
  int64_t start = tr.at(v), next = tr.at(v + 1);
  unsigned bad = 0;
  for (int64_t e = s; e < e_end; ++e) {
    while (e == next) {
      ++v;
      start = next;
      next = tr.at(v + 1);
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
        if (m == (int32_t)v) {
          found = true;
          break;
        }
        if (m < (int32_t)v) lo = mid + 1;
        else hi = mid - 1;
      }
      if (!found) bad |= kErrAsymmetric;
    }
  }
  if (bad) atomicOr(err, bad);
}

// Offsets monotone with the right ends; *max_deg receives the largest row.
__global__ void validate_rowptr_kernel(const int64_t *rowptr, int64_t n, int64_t nnz,
                                       unsigned *err, unsigned long long *max_deg) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  long long d = 0;
  if (v <= n) {
    const int64_t a = rowptr[v];
    bool bad = (v == 0 && a != 0) || (v == n && a != nnz) || a < 0 || a > nnz;
    if (v < n) {
      d = rowptr[v + 1] - a;
      if (d < 0) bad = true;
    }
    if (bad) atomicOr(err, (unsigned)kErrRowptr);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) d = max(d, __shfl_down_sync(kFull, d, o));
  if ((threadIdx.x & 31) == 0 && d > 0) atomicMax(max_deg, (unsigned long long)d);
}

// Degree-rank sort keys: position i holds vertex n-1-i, keyed by
// (max_degree - degree) in the high word. A stable sort of the high word
// keeps equal degrees in descending id order, so the sorted position is the
// rank in (degree desc, id desc) order.
__global__ void rank_keys_kernel(const int2 *__restrict__ key, int64_t n, int max_degree,
                                 unsigned long long *__restrict__ keys) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    keys[i] = ((unsigned long long)(unsigned)(max_degree - key[n - 1 - i].x) << 32) |
              (unsigned long long)i;
}

__global__ void rank_scatter_kernel(const unsigned long long *__restrict__ sorted, int64_t n,
                                    int32_t *__restrict__ rank) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) rank[n - 1 - (int64_t)(uint32_t)sorted[p]] = (int32_t)p;
}

// Core bitmaps: warp per rank p < core_ranks; its vertex is the one whose
// sort key sits at position p. Every entry z of N+(v) ranks below p, so it
// sets bit z of the words from core_offset(p) (which start
// cleared; the row's last quad pads to a multiple of 128 bits with zeros).
// Nothing runs when an exact-size DAG was overrun: its rows were
// then never written.
__global__ void core_bits_kernel(const unsigned long long *__restrict__ sorted, int64_t n,
                                 int core_ranks, const int64_t *__restrict__ dag_rowptr,
                                 const int32_t *__restrict__ dag_rank, unsigned *core,
                                 unsigned *err) {
  const int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
  const int lane = threadIdx.x & (kWarp - 1);
  if (p >= core_ranks || (*(volatile unsigned *)err & (kErrDagCapacity | kErrContract))) return;
  const int64_t v = n - 1 - (int64_t)(uint32_t)sorted[p];
  unsigned *row = core + core_offset(p);
  for (int64_t e = dag_rowptr[v] + lane; e < dag_rowptr[v + 1]; e += kWarp) {
    const int z = __ldg(dag_rank + e);
    if (z >= 0 && z < p) atomicOr(row + (z >> 5), 1u << (z & 31));
    else atomicOr(err, (unsigned)kErrRank);
  }
}

// pinfo[v] = {d+(v), rank(v) (INT_MAX without ranks), dag_rowptr[v]}.
__global__ void partner_info_kernel(const int2 *__restrict__ key, const int32_t *__restrict__ rank,
                                    const int64_t *__restrict__ dag_rowptr, int64_t n,
                                    int4 *__restrict__ pinfo) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const long long st = dag_rowptr[v];
  pinfo[v] = make_int4(key[v].y, rank ? rank[v] : INT_MAX, (int)(unsigned)(st & 0xffffffffll),
                       (int)(st >> 32));
}

// key[v] = {degree, 0}; deg[v] = degree alone (4 bytes per gather in pass A).
__global__ void init_key_kernel(const int64_t *rowptr, int64_t n, int2 *key, int32_t *deg) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) {
    const int d = (int)(rowptr[v + 1] - rowptr[v]);
    key[v] = make_int2(d, 0);
    deg[v] = d;
  }
}

// Tasks each owner contributes to the hub, large-table hub and leaf queues
// (chunks of its symmetric row), and the largest DAG out-degree.
__global__ void task_count_kernel(const int2 *key, int64_t n, int32_t *hub_cnt,
                                  int32_t *leaf_cnt, int32_t *mega_cnt,
                                  unsigned long long *max_out, BatchView bv) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int32_t d = 0;
  if (v < n) {
    const int2 kv = key[v];
    d = kv.y;
    int32_t h = 0, l = 0, m = 0;
    int leaf_max = kLeafMaxOut;
    bool counted = true;
    if (bv.gid) {  // batch: only triangle jobs get tasks, with their graph's threshold
      const int g = bv.gid[v];
      counted = bv.job[g] == 0;
      if (bv.param) leaf_max = bv.param[g].x;
    }
    // Owners need d+ >= 1; every neighbour of the row may be a partner.
    if (counted && d >= 1) {
      if (d <= leaf_max) l = (kv.x + kLeafChunk - 1) / kLeafChunk;
      else if (d <= kHubSmallMaxOut) h = (kv.x + kHubChunk - 1) / kHubChunk;
      else m = (kv.x + kHubChunk - 1) / kHubChunk;
    }
    hub_cnt[v] = h;
    leaf_cnt[v] = l;
    mega_cnt[v] = m;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) d = max(d, __shfl_down_sync(kFull, d, o));
  if ((threadIdx.x & 31) == 0 && d > 0) atomicMax(max_out, (unsigned long long)d);
}

// Task word: owner id in the high half, chunk index in the low half.
__global__ void task_fill_kernel(const int32_t *hub_cnt, const int64_t *hub_off,
                                 const int32_t *leaf_cnt, const int64_t *leaf_off,
                                 const int32_t *mega_cnt, const int64_t *mega_off, int64_t n,
                                 uint64_t *hub_tasks, uint64_t *leaf_tasks, uint64_t *mega_tasks) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const uint64_t hi = (uint64_t)v << 32;
  for (int32_t c = 0, h = hub_cnt[v]; c < h; ++c) hub_tasks[hub_off[v] + c] = hi | (uint32_t)c;
  for (int32_t c = 0, l = leaf_cnt[v]; c < l; ++c) leaf_tasks[leaf_off[v] + c] = hi | (uint32_t)c;
  for (int32_t c = 0, m = mega_cnt[v]; c < m; ++c) mega_tasks[mega_off[v] + c] = hi | (uint32_t)c;
}

// Partner edges (owner rule) and their streamed-list work, for statistics:
// one warp per row, lanes over its entries.
__global__ void partner_stats_kernel(const int64_t *rowptr, const int32_t *col, const int2 *key,
                                     int64_t n, unsigned long long *out) {
  unsigned long long pe = 0, work = 0;
  const int lane = threadIdx.x & (kWarp - 1);
  const int64_t warps = (int64_t)gridDim.x * blockDim.x / kWarp;
  for (int64_t x = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; x < n; x += warps) {
    const int px = key[x].y;
    if (px < 1) continue;
    for (int64_t e = rowptr[x] + lane; e < rowptr[x + 1]; e += kWarp) {
      const int y = col[e];
      const int py = key[y].y;
      if (py >= 1 && (px > py || (px == py && (int)x > y))) {
        ++pe;
        work += (unsigned long long)py;
      }
    }
  }
  pe = warp_sum_u64(pe);
  work = warp_sum_u64(work);
  if ((threadIdx.x & 31) == 0) {
    if (pe) atomicAdd(out, pe);
    if (work) atomicAdd(out + 1, work);
  }
}

unsigned grid_for(int64_t items, int threads) {
  return (unsigned)std::max<int64_t>(1, (items + threads - 1) / threads);
}

}  // namespace

int validate_graph(mc_dgraph *g, unsigned flags) {
  NvtxRange range("validate_graph");
  MC_CUDA_TRY(cudaMemsetAsync(g->err, 0, sizeof(unsigned), g->stream));
  MC_CUDA_TRY(cudaMemsetAsync(g->counters + 7, 0, sizeof(unsigned long long), g->stream));
  validate_rowptr_kernel<<<grid_for(g->n + 1, 256), 256, 0, g->stream>>>(
      g->rowptr, g->n, g->nnz, g->err, g->counters + 7);
  MC_CUDA_TRY(cudaGetLastError());
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_err, g->err, sizeof(unsigned), cudaMemcpyDeviceToHost, g->stream));
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_counters + 7, g->counters + 7, sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, g->stream));
  MC_CUDA_TRY(cudaStreamSynchronize(g->stream));
  if (*g->h_err) return MC_ERR_FORMAT;  // the entry walk needs monotone offsets
  g->max_degree = (int64_t)g->h_counters[7];
  const int64_t tiles = (g->nnz + kTileEdges - 1) / kTileEdges;
  g->launches += 1 + (tiles > 0 ? 1 : 0);
  if (tiles > 0) {
    validate_entries_kernel<<<(unsigned)tiles, kTileThreads, 0, g->stream>>>(
        g->rowptr, g->col, g->n, g->nnz, (flags & MC_VALIDATE_SYMMETRY) ? 1 : 0, g->err, 0);
    MC_CUDA_TRY(cudaGetLastError());
  }
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_err, g->err, sizeof(unsigned), cudaMemcpyDeviceToHost, g->stream));
  MC_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return *g->h_err ? MC_ERR_FORMAT : MC_OK;
}

int validate_rowptr(mc_dgraph *g) {
  MC_CUDA_TRY(cudaMemsetAsync(g->err, 0, sizeof(unsigned), g->stream));
  MC_CUDA_TRY(cudaMemsetAsync(g->counters + 7, 0, sizeof(unsigned long long), g->stream));
  validate_rowptr_kernel<<<grid_for(g->n + 1, 256), 256, 0, g->stream>>>(
      g->rowptr, g->n, g->nnz, g->err, g->counters + 7);
  MC_CUDA_TRY(cudaGetLastError());
  g->launches += 1;
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_err, g->err, sizeof(unsigned), cudaMemcpyDeviceToHost, g->stream));
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_counters + 7, g->counters + 7, sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, g->stream));
  MC_CUDA_TRY(cudaStreamSynchronize(g->stream));
  if (*g->h_err) return MC_ERR_FORMAT;
  g->max_degree = (int64_t)g->h_counters[7];
  return MC_OK;
}

int validate_csr_words(const int64_t *rowptr, const int32_t *col, int64_t n, int64_t nnz,
                       unsigned *d_err, unsigned long long *d_max_deg, cudaStream_t s,
                       int64_t *max_degree) {
  unsigned h_err = 0;
  unsigned long long h_max = 0;
  MC_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(unsigned), s));
  MC_CUDA_TRY(cudaMemsetAsync(d_max_deg, 0, sizeof(unsigned long long), s));
  validate_rowptr_kernel<<<grid_for(n + 1, 256), 256, 0, s>>>(rowptr, n, nnz, d_err, d_max_deg);
  MC_CUDA_TRY(cudaGetLastError());
  MC_CUDA_TRY(cudaMemcpyAsync(&h_err, d_err, sizeof(h_err), cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaMemcpyAsync(&h_max, d_max_deg, sizeof(h_max), cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  if (h_err) return MC_ERR_FORMAT;  // the entry walk needs monotone offsets
  const int64_t tiles = (nnz + kTileEdges - 1) / kTileEdges;
  if (tiles > 0) {
    validate_entries_kernel<<<(unsigned)tiles, kTileThreads, 0, s>>>(rowptr, col, n, nnz, 0, d_err,
                                                                   0);
    MC_CUDA_TRY(cudaGetLastError());
    MC_CUDA_TRY(cudaMemcpyAsync(&h_err, d_err, sizeof(h_err), cudaMemcpyDeviceToHost, s));
    MC_CUDA_TRY(cudaStreamSynchronize(s));
  }
  *max_degree = (int64_t)h_max;
  return h_err ? MC_ERR_FORMAT : MC_OK;
}

namespace {
// DAG capacity: every entry in device memory; with host columns the exact
// m+ = nnz / 2 of a symmetric simple graph (tc_orient refuses more).
int64_t dag_capacity(int64_t nnz, bool col_host) {
  return col_host ? nnz / 2 + 1 : std::max<int64_t>(nnz, 1);
}
}  // namespace

// Column entries per staging buffer with host columns (two buffers): 64 MB,
// or MERCURY_STAGE_EDGES rounded down to whole tiles (tests use it to run
// many chunks on small graphs).
int64_t stage_capacity(int64_t nnz) {
  int64_t stage = 1ll << 24;
  if (const char *env = std::getenv("MERCURY_STAGE_EDGES")) {
    const long long v = std::atoll(env);
    if (v > 0) stage = std::max<int64_t>(kTileEdges, v / kTileEdges * kTileEdges);
  }
  return std::min(stage, std::max<int64_t>((nnz + kTileEdges - 1) / kTileEdges, 1) * kTileEdges);
}

// Ranks with core bitmaps: kCoreRanks, or MERCURY_TC_CORE_RANKS (0 turns
// them off; tests move the boundary with it), at most n.
int core_rank_count(int64_t n) {
  int64_t k = kCoreRanks;
  if (const char *env = std::getenv("MERCURY_TC_CORE_RANKS")) {
    const long long v = std::atoll(env);
    if (v >= 0) k = std::min<long long>(v, 1 << 18);
  }
  return (int)std::min<int64_t>(k, n);
}

int64_t tc_device_bytes(int64_t n, int64_t nnz, bool col_host, bool dag_host) {
  const int64_t cap = std::max<int64_t>(nnz, 1);
  const int64_t tiles = std::max<int64_t>((nnz + kTileEdges - 1) / kTileEdges, 1);
  const int64_t tasks = n + cap / std::min(kHubChunk, kLeafChunk) + 1;
  const int64_t scan = (int64_t)std::max(std::max(scan_temp_bytes(n + 1), scan_temp_bytes(tiles + 1)),
                                         radix_temp_bytes(n));
  const int64_t staging =
      col_host ? 2 * 4 * stage_capacity(nnz) + 8 * (stage_capacity(nnz) / kTileEdges + 1) : 0;
  return (n + 1) * (8 + 16 + 8 + 3 * 4 + 3 * 8 + 4 + 16) + 3 * 8 * tasks +
         (dag_host ? 0 : 2 * 4 * (dag_capacity(nnz, col_host) + 4)) +
         tiles * (2 * kTileThreads + 28) +
         2 * 12 * (radix_entries(n) + 1) + scan + staging + 4 * core_offset(core_rank_count(n));
}

int tc_alloc(mc_dgraph *g) {
  if (g->tc_ready) return MC_OK;
  const int64_t n = g->n, cap = std::max<int64_t>(g->nnz, 1);
  const int64_t tiles = std::max<int64_t>((g->nnz + kTileEdges - 1) / kTileEdges, 1);
  g->dag_cap = dag_capacity(g->nnz, g->col_host);
  // Each owner contributes ceil(deg / chunk) <= 1 + deg / chunk tasks.
  g->task_capacity = n + cap / std::min(kHubChunk, kLeafChunk) + 1;
  g->scan_temp_size = std::max(scan_temp_bytes(n + 1), scan_temp_bytes(tiles + 1));
  const bool ranked = g->batch.gid == nullptr;
  if (ranked) g->scan_temp_size = std::max(g->scan_temp_size, radix_temp_bytes(n));
#define MC_ALLOC(ptr, count) \
  MC_CUDA_TRY(dev_alloc((void **)&(ptr), sizeof(*(ptr)) * (size_t)(count), g->stream))
  MC_ALLOC(g->key, n + 1);
  MC_ALLOC(g->pinfo, n + 1);
  MC_ALLOC(g->dag_rowptr, n + 1);
  // 4 entries of padding: the staged hub kernel copies whole 16-byte groups.
  // With the DAG on the host, its entries and ranks live in pinned memory
  // that the kernels reach through the device's mapping.
  auto dag_alloc = [&](int32_t **dev, int32_t **host) -> cudaError_t {
    if (!g->dag_host) return dev_alloc((void **)dev, sizeof(int32_t) * (size_t)(g->dag_cap + 4), g->stream);
    cudaError_t e = cudaHostAlloc((void **)host, sizeof(int32_t) * (size_t)(g->dag_cap + 4),
                                  cudaHostAllocMapped);
    if (e != cudaSuccess) return e;
    return cudaHostGetDevicePointer((void **)dev, *host, 0);
  };
  MC_CUDA_TRY(dag_alloc(&g->dag_col, &g->dag_col_h));
  MC_ALLOC(g->keep, tiles * kTileThreads);
  MC_ALLOC(g->tile_counts, tiles);
  MC_ALLOC(g->tile_offsets, tiles + 1);
  MC_ALLOC(g->tile_rows, 2 * tiles);
  MC_ALLOC(g->hub_cnt, n + 1);
  MC_ALLOC(g->leaf_cnt, n + 1);
  MC_ALLOC(g->hub_off, n + 1);
  MC_ALLOC(g->leaf_off, n + 1);
  MC_ALLOC(g->hub_tasks, g->task_capacity);
  MC_ALLOC(g->leaf_tasks, g->task_capacity);
  MC_ALLOC(g->mega_cnt, n + 1);
  MC_ALLOC(g->mega_off, n + 1);
  MC_ALLOC(g->mega_tasks, g->task_capacity);
  if (ranked) {
    MC_ALLOC(g->rank, n + 1);
    MC_CUDA_TRY(dag_alloc(&g->dag_rank, &g->dag_rank_h));
    MC_ALLOC(g->rank_keys, 2 * n + 2);
    MC_ALLOC(g->rank_counts, radix_entries(n) + 1);
    MC_ALLOC(g->rank_offsets, radix_entries(n) + 1);
    g->core_ranks = core_rank_count(n);
    if (g->core_ranks > 0) MC_ALLOC(g->core_bits, core_offset(g->core_ranks));
  }
  // Chunked column passes (host columns, or a streamed upload of a single
  // graph): the copy stream, its events and one chunk's tile offsets.
  if (ranked) {
    g->chunk_edges = stage_capacity(g->nnz);
    MC_ALLOC(g->chunk_offsets, g->chunk_edges / kTileEdges + 1);
    MC_CUDA_TRY(cudaStreamCreateWithFlags(&g->copy_stream, cudaStreamNonBlocking));
    for (cudaEvent_t &e : g->stage_ev)
      MC_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  if (g->col_host && ranked) {
    g->stage_edges = g->chunk_edges;
    MC_ALLOC(g->stage, 2 * g->stage_edges);
  }
  MC_CUDA_TRY(dev_alloc(&g->scan_temp, g->scan_temp_size, g->stream));
#undef MC_ALLOC
  g->tc_ready = true;
  return MC_OK;
}

// Host copy of count entries by all host threads, in 1 MB pieces.
static void parallel_copy(int32_t *dst, const int32_t *src, int64_t count) {
  constexpr int64_t kPiece = 1 << 18;
  const int64_t pieces = (count + kPiece - 1) / kPiece;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < pieces; ++p) {
    const int64_t a = p * kPiece, b = std::min(count, a + kPiece);
    std::memcpy(dst + a, src + a, sizeof(int32_t) * (size_t)(b - a));
  }
}

// Passes A and B over a column array that crosses from host memory in
// chunks of whole tiles, copied by DMA on a copy stream while the passes run
// on the previous chunk.  Each chunk runs A, the scan of its tile counts on
// top of the earlier chunks' total, and B, so no pass waits for the whole
// array.  Two forms:
//  * host columns (in_place false): chunks go to two staging buffers; the
//    columns were validated when the handle was made;
//  * streamed upload (in_place true): chunks land in the handle's own device
//    column array, and each chunk's contract checks run before its passes,
//    which do nothing once a check has failed (no gather of an unchecked id).
// The DAG holds dag_cap entries; a chunk that would end past it raises
// kErrDagCapacity and writes nothing.  The caller reads the flags before
// counting.
// Pass B stages each tile's DAG entries in shared memory and writes them
// out with whole-line stores (MERCURY_DAG_STAGE=0: each thread writes its
// own kept entries directly).
static bool stage_dag_writes() {
  const char *env = std::getenv("MERCURY_DAG_STAGE");
  return env ? std::atoi(env) != 0 : true;
}

static int staged_dag_passes(mc_dgraph *g, const int32_t *deg, const int32_t *src, bool in_place) {
  const int64_t n = g->n, nnz = g->nnz;
  cudaStream_t s = g->stream, cs = g->copy_stream;
  cudaEvent_t *copied = g->stage_ev, *drained = g->stage_ev + 2;
  const int64_t chunk = in_place ? g->chunk_edges : g->stage_edges;
  const unsigned *stop = in_place ? g->err : nullptr;
  // A streamed upload from pageable memory goes through the pinned slots when
  // the caller provided them (the driver's own pageable copies are slower).
  bool pageable = false;
  if (in_place && g->pin_slot[0] && g->pin_slot[1] && g->pin_entries >= chunk) {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, src) == cudaSuccess)
      pageable = attr.type == cudaMemoryTypeUnregistered;
    else
      cudaGetLastError();  // an unknown pointer: plain copies
  }
  MC_CUDA_TRY(cudaMemsetAsync(g->tile_offsets, 0, sizeof(int64_t), s));
  // Copies start after the work already queued on the handle's stream.
  MC_CUDA_TRY(cudaEventRecord(drained[0], s));
  MC_CUDA_TRY(cudaStreamWaitEvent(cs, drained[0], 0));
  const int64_t chunks = (nnz + chunk - 1) / chunk;
  for (int64_t c = 0; c < chunks; ++c) {
    const int slot = (int)(c & 1);
    const int64_t e0 = c * chunk, e1 = std::min(nnz, e0 + chunk);
    const int64_t tb = e0 / kTileEdges, ct = (e1 - e0 + kTileEdges - 1) / kTileEdges;
    int32_t *buf = in_place ? g->col + e0 : g->stage + (int64_t)slot * g->stage_edges;
    if (!in_place && c >= 2) MC_CUDA_TRY(cudaStreamWaitEvent(cs, drained[slot], 0));
    if (pageable) {
      // The host threads copy the chunk into a pinned slot (free once its
      // previous copy to the device is done), then the DMA engine takes it,
      // while the threads fill the other slot.
      if (c >= 2) MC_CUDA_TRY(cudaEventSynchronize(g->pin_done[slot]));
      parallel_copy(g->pin_slot[slot], src + e0, e1 - e0);
      MC_CUDA_TRY(cudaMemcpyAsync(buf, g->pin_slot[slot], sizeof(int32_t) * (size_t)(e1 - e0),
                                  cudaMemcpyHostToDevice, cs));
      MC_CUDA_TRY(cudaEventRecord(g->pin_done[slot], cs));
    } else {
      MC_CUDA_TRY(cudaMemcpyAsync(buf, src + e0, sizeof(int32_t) * (size_t)(e1 - e0),
                                  cudaMemcpyHostToDevice, cs));
    }
    MC_CUDA_TRY(cudaEventRecord(copied[slot], cs));
    MC_CUDA_TRY(cudaStreamWaitEvent(s, copied[slot], 0));
    if (in_place) {
      validate_entries_kernel<<<(unsigned)ct, kTileThreads, 0, s>>>(g->rowptr, g->col, n, nnz, 0,
                                                                    g->err, tb, g->tile_rows);
      MC_CUDA_TRY(cudaGetLastError());
      g->launches += 1;
    }
    const ColumnChunk cc = in_place ? ColumnChunk{g->col, 0, tb} : ColumnChunk{buf, e0, tb};
    dag_pass_kernel<false><<<(unsigned)ct, kTileThreads, 0, s>>>(
        g->rowptr, cc, deg, n, nnz, g->key, g->keep, g->tile_counts, nullptr, nullptr, nullptr,
        nullptr, nullptr, nullptr, 0, stop, g->tile_rows);
    MC_CUDA_TRY(cudaGetLastError());
    MC_CUDA_TRY(exclusive_scan(g->tile_counts + tb, g->chunk_offsets, ct, g->scan_temp, s));
    chunk_offsets_kernel<<<grid_for(ct + 1, 256), 256, 0, s>>>(g->chunk_offsets, ct,
                                                               g->tile_offsets + tb, g->dag_cap,
                                                               g->err);
    MC_CUDA_TRY(cudaGetLastError());
    (stage_dag_writes() ? dag_pass_kernel<true, true> : dag_pass_kernel<true, false>)
        <<<(unsigned)ct, kTileThreads, 0, s>>>(
        g->rowptr, cc, deg, n, nnz, g->key, g->keep, nullptr, g->tile_offsets, g->dag_rowptr,
        g->dag_col, g->rank, g->dag_rank, g->tile_offsets + tb + ct, g->dag_cap, stop,
        g->tile_rows);
    MC_CUDA_TRY(cudaGetLastError());
    MC_CUDA_TRY(cudaEventRecord(drained[slot], s));
    g->launches += 3 + scan_launches(ct);
  }
  return MC_OK;
}

int tc_orient(mc_dgraph *g, const int32_t *upload) {
  NvtxRange range("tc_orient");
  const int64_t n = g->n, nnz = g->nnz;
  cudaStream_t s = g->stream;
  MC_CUDA_TRY(cudaMemsetAsync(g->counters, 0, sizeof(unsigned long long) * 7, s));
  g->core_used = 0;
  if (n == 0) return MC_OK;
  const int64_t tiles = (nnz + kTileEdges - 1) / kTileEdges;
  // The degrees alone, for pass A's gathers, in mega_cnt (unused until the
  // task counts are written after pass B).
  int32_t *deg = g->mega_cnt;
  init_key_kernel<<<grid_for(n, 256), 256, 0, s>>>(g->rowptr, n, g->key, deg);
  MC_CUDA_TRY(cudaGetLastError());
  g->launches += 1;
  if (g->rank && !g->batch.gid) {
    // Degree ranks (the hub kernel's bitmaps are indexed by them).
    rank_keys_kernel<<<grid_for(n, 256), 256, 0, s>>>(g->key, n, (int)g->max_degree, g->rank_keys);
    MC_CUDA_TRY(cudaGetLastError());
    unsigned long long *sorted = nullptr;
    MC_CUDA_TRY(radix_sort_u64(g->rank_keys, g->rank_keys + n, n, 32,
                               32 + bit_width((uint64_t)g->max_degree), g->rank_counts,
                               g->rank_offsets, g->scan_temp, s, &sorted, &g->launches));
    rank_scatter_kernel<<<grid_for(n, 256), 256, 0, s>>>(sorted, n, g->rank);
    MC_CUDA_TRY(cudaGetLastError());
    g->rank_sorted = sorted;
    g->launches += 2;
  }
  if (tiles > 0) {
    tile_rows_kernel<<<grid_for(n, 256), 256, 0, s>>>(g->rowptr, n, nnz, tiles, g->tile_rows);
    MC_CUDA_TRY(cudaGetLastError());
    g->launches += 1;
  }
  if (tiles == 0) {
    MC_CUDA_TRY(cudaMemsetAsync(g->dag_rowptr, 0, sizeof(int64_t) * (n + 1), s));
  } else if (upload) {
    // A streamed upload needs the chunk machinery of a single-graph handle.
    if (!g->copy_stream || !g->chunk_offsets || g->chunk_edges <= 0) return MC_ERR_ARG;
    const int rc = staged_dag_passes(g, deg, upload, true);
    if (rc != MC_OK) return rc;
  } else if (g->col_host) {
    if (!g->copy_stream || !g->stage || g->stage_edges <= 0) return MC_ERR_ARG;
    const int rc = staged_dag_passes(g, deg, g->col_h, false);
    if (rc != MC_OK) return rc;
  } else {
    const unsigned grid = (unsigned)tiles;
    const ColumnChunk all{g->col, 0, 0};
    dag_pass_kernel<false><<<grid, kTileThreads, 0, s>>>(
        g->rowptr, all, deg, n, nnz, g->key, g->keep, g->tile_counts, nullptr, nullptr, nullptr,
        nullptr, nullptr, nullptr, 0, nullptr, g->tile_rows);
    MC_CUDA_TRY(cudaGetLastError());
    MC_CUDA_TRY(exclusive_scan(g->tile_counts, g->tile_offsets, tiles, g->scan_temp, s));
    (stage_dag_writes() ? dag_pass_kernel<true, true> : dag_pass_kernel<true, false>)
        <<<grid, kTileThreads, 0, s>>>(
        g->rowptr, all, deg, n, nnz, g->key, g->keep, nullptr, g->tile_offsets, g->dag_rowptr,
        g->dag_col, g->batch.gid ? nullptr : g->rank, g->batch.gid ? nullptr : g->dag_rank,
        nullptr, 0, nullptr, g->tile_rows);
    MC_CUDA_TRY(cudaGetLastError());
    g->launches += 2 + scan_launches(tiles);
  }
  // A handle reused for a smaller graph keeps its capacity: only the ranks
  // of this graph get core bitmaps.
  if (g->core_bits && g->rank_sorted && !g->batch.gid) {
    g->core_used = (int)std::min<int64_t>(g->core_ranks, n);
    MC_CUDA_TRY(cudaMemsetAsync(g->core_bits, 0, sizeof(unsigned) * core_offset(g->core_used), s));
    core_bits_kernel<<<grid_for((int64_t)g->core_used * kWarp, 256), 256, 0, s>>>(
        g->rank_sorted, n, g->core_used, g->dag_rowptr, g->dag_rank, g->core_bits, g->err);
    MC_CUDA_TRY(cudaGetLastError());
    g->launches += 1;
  }
  partner_info_kernel<<<grid_for(n, 256), 256, 0, s>>>(
      g->key, g->batch.gid ? nullptr : g->rank, g->dag_rowptr, n, g->pinfo);
  MC_CUDA_TRY(cudaGetLastError());
  g->launches += 1;
  task_count_kernel<<<grid_for(n, 256), 256, 0, s>>>(g->key, n, g->hub_cnt, g->leaf_cnt,
                                                     g->mega_cnt, g->counters + 3, g->batch);
  MC_CUDA_TRY(cudaGetLastError());
  MC_CUDA_TRY(exclusive_scan(g->hub_cnt, g->hub_off, n, g->scan_temp, s));
  MC_CUDA_TRY(exclusive_scan(g->leaf_cnt, g->leaf_off, n, g->scan_temp, s));
  MC_CUDA_TRY(exclusive_scan(g->mega_cnt, g->mega_off, n, g->scan_temp, s));
  task_fill_kernel<<<grid_for(n, 256), 256, 0, s>>>(g->hub_cnt, g->hub_off, g->leaf_cnt,
                                                    g->leaf_off, g->mega_cnt, g->mega_off, n,
                                                    g->hub_tasks, g->leaf_tasks, g->mega_tasks);
  MC_CUDA_TRY(cudaGetLastError());
  g->launches += 2 + 3 * scan_launches(n);
  return MC_OK;
}

int tc_partner_stats(mc_dgraph *g, unsigned long long *partner_edges, unsigned long long *work) {
  *partner_edges = *work = 0;
  if (!g->tc_ready || g->n == 0) return MC_OK;
  MC_CUDA_TRY(cudaMemsetAsync(g->counters + 4, 0, sizeof(unsigned long long) * 2, g->stream));
  partner_stats_kernel<<<g->num_sms * 8, 256, 0, g->stream>>>(g->rowptr, g->col, g->key, g->n,
                                                              g->counters + 4);
  MC_CUDA_TRY(cudaGetLastError());
  unsigned long long c[2];
  MC_CUDA_TRY(cudaMemcpyAsync(c, g->counters + 4, sizeof(c), cudaMemcpyDeviceToHost, g->stream));
  MC_CUDA_TRY(cudaStreamSynchronize(g->stream));
  *partner_edges = c[0];
  *work = c[1];
  return MC_OK;
}

}  // namespace mc

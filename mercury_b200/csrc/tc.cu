// Triangle-count kernels.  count = sum over DAG edges {x, y} of
// |N+(x) & N+(y)|, where x is the edge's owner (larger d+, ties to the larger
// id) and y its partner.  A task is (owner, chunk of the owner's symmetric
// row): N+(owner) goes into a shared-memory open-addressing table, the
// chunk's neighbours are filtered down to partners (owner rule on d+), and
// each partner's list N+(y) -- never longer than N+(owner) -- is streamed
// through the table.
//
// Reference counterparts: hashIndex_for_large_degree (CTA per large vertex,
// 1019-bin hash staged through a 256 MiB global scratch,
// gpu_kernels/tc_challenge.cuh:4-192) and binarySearch_for_small_degree
// (warp per small vertex, binary search in shared memory,
// gpu_kernels/tc_challenge.cuh:195-303), each with an atomic work counter
// (DYNAMIC_MODE, gpu_kernels/tuning_schedules.cuh:1-21).  Here the queues hold
// bounded (owner, row-chunk) tasks, the tables live in shared memory only,
// and the hash needs no global scratch.
#include <algorithm>

#include "dgraph.cuh"
#include "device_common.cuh"

namespace mc {
namespace {

constexpr int kClaim = 16;  // owner-row entries a hub warp claims at a time

struct CountArgs {
  const int64_t *__restrict__ rowptr;      // symmetric CSR
  const int32_t *__restrict__ col;
  const int2 *__restrict__ key;            // {deg, d+}
  const int64_t *__restrict__ dag_rowptr;  // N+ lists
  const int32_t *__restrict__ dag_col;
  const uint64_t *__restrict__ tasks;
  const int64_t *__restrict__ ntasks;  // device scalar (end of the offsets)
  unsigned long long *queue;
  unsigned long long *result;
  unsigned *err;
  int table_log2_max;
  int shard, num_shards;  // this call counts tasks shard, shard + num_shards, ...
};

// Tasks of this shard: queue position t maps to task t * num_shards + shard.
__device__ __forceinline__ int64_t shard_tasks(const CountArgs &a) {
  const int64_t total = *a.ntasks;
  return total > a.shard ? (total - a.shard + a.num_shards - 1) / a.num_shards : 0;
}
__device__ __forceinline__ uint64_t shard_task(const CountArgs &a, unsigned long long t) {
  return a.tasks[(int64_t)t * a.num_shards + a.shard];
}

// Probe of an open-addressing table (empty slot = -1, linear probing).  The
// tables are filled to at most half, so a probe meets an empty slot; the
// bound only guards against a corrupted table.
struct TableProbe {
  const int *tab;
  unsigned mask;
  int shift;
  __device__ __forceinline__ unsigned operator()(int w) const {
    unsigned h = hash_slot(w, shift);
    int t = tab[h];
    if (t == w) return 1u;
#pragma unroll 1
    for (unsigned it = 0; t >= 0 && it < mask; ++it) {
      h = (h + 1) & mask;
      t = tab[h];
      if (t == w) return 1u;
    }
    return 0u;
  }
};

// Binary search in a sorted global list (owners too large for the table).
struct ListProbe {
  const int32_t *list;
  int len;
  __device__ __forceinline__ unsigned operator()(int w) const {
    int lo = 0, hi = len - 1;
    while (lo <= hi) {
      int mid = (lo + hi) >> 1;
      int m = __ldg(list + mid);
      if (m == w) return 1u;
      if (m < w) lo = mid + 1; else hi = mid - 1;
    }
    return 0u;
  }
};

__device__ __forceinline__ void table_insert(int *tab, unsigned mask, int shift, int key,
                                             unsigned *err) {
  unsigned h = hash_slot(key, shift);
  for (unsigned it = 0;; ++it) {
    const int prev = atomicCAS(tab + h, -1, key);
    if (prev == -1 || prev == key) return;
    h = (h + 1) & mask;
    if (it >= mask) {
      atomicOr(err, (unsigned)kErrHashFull);
      return;
    }
  }
}

// Partner test for neighbour y of owner x (px = d+(x), py = d+(y)).
__device__ __forceinline__ bool owns(int x, int px, int y, int py) {
  return py >= 1 && (px > py || (px == py && x > y));
}

// One warp streams one list col[st, st+len) through `probe`: 8-byte loads
// (two probes per lane) with a scalar head/tail for odd ends.  Returns this
// lane's hits.
template <class Probe>
__device__ __forceinline__ unsigned stream_list(const int32_t *__restrict__ col, int64_t st,
                                                int len, int lane, const Probe &probe) {
  unsigned hits = 0;
  const int head = (int)(st & 1) & (len > 0 ? 1 : 0);
  if (lane == 0 && head) hits += probe(__ldg(col + st));
  const int64_t a = st + head;
  const int rest = len - head;
  const int body = rest >> 1;
  const int2 *v = reinterpret_cast<const int2 *>(col + a);
  for (int k = lane; k < body; k += kWarp) {
    const int2 q = __ldg(v + k);
    hits += probe(q.x) + probe(q.y);
  }
  if (lane == 0 && (rest & 1)) hits += probe(__ldg(col + a + 2 * body));
  return hits;
}

// ---- table probes with deferred collisions ---------------------------------
// Every key gets one probe of its home slot.  A key that finds another key
// there is appended to a per-warp queue in shared memory; the queue is worked
// off 32 entries at a time, one slot per entry per step (entries that meet
// yet another key are re-queued), so no lane waits on another lane's chain.
constexpr int kQueueCap = 64;

struct ProbeQueue {
  int2 *q;  // this warp's kQueueCap entries {key, next slot}
  int cnt;  // same value on every lane
};

__device__ __forceinline__ void queue_push(ProbeQueue &Q, bool need, int w, unsigned slot,
                                           int lane) {
  const unsigned m = __ballot_sync(kFull, need);
  if (need) Q.q[Q.cnt + __popc(m & ((1u << lane) - 1u))] = make_int2(w, (int)slot);
  Q.cnt += __popc(m);
}

// One step over the newest min(cnt, 32) queued keys.
__device__ __forceinline__ unsigned queue_step(ProbeQueue &Q, const int *tab, unsigned mask,
                                               int lane) {
  __syncwarp();
  const int take = min(Q.cnt, kWarp);
  const int base = Q.cnt - take;
  const bool act = lane < take;
  const int2 e = act ? Q.q[base + lane] : make_int2(0, 0);
  __syncwarp();
  Q.cnt = base;
  unsigned hit = 0;
  bool more = false;
  if (act) {
    const int t = tab[e.y];
    hit = t == e.x;
    more = t >= 0 && t != e.x;
  }
  queue_push(Q, more, e.x, ((unsigned)e.y + 1u) & mask, lane);
  return hit;
}

// Steps until at most keep_below keys wait.  Every queued key reaches an
// empty slot or itself within mask + 1 steps (tables are at most half
// full); the bound only guards against a corrupted table, which raises the
// error flag and drops the queue.
__device__ __forceinline__ unsigned queue_drain(ProbeQueue &Q, const int *tab, unsigned mask,
                                                int lane, int keep_below, unsigned *err) {
  unsigned hits = 0;
  const int limit = 4 * (int)(mask + 1) + 8;
  for (int it = 0; Q.cnt > keep_below; ++it) {
    if (it >= limit) {
      if (lane == 0) atomicOr(err, (unsigned)kErrHashFull);
      Q.cnt = 0;
      break;
    }
    hits += queue_step(Q, tab, mask, lane);
  }
  return hits;
}

// Home-slot probe of key w (valid lanes only); collisions are queued.
__device__ __forceinline__ unsigned home_probe(ProbeQueue &Q, const int *tab, unsigned mask,
                                               int shift, int w, bool valid, int lane) {
  const unsigned h = hash_slot(w, shift);
  const int t = valid ? tab[h] : -1;
  queue_push(Q, t >= 0 && t != w, w, (h + 1u) & mask, lane);
  return valid && t == w;
}

// One warp streams col[st, st+len) through the table: each lane keeps four
// 8-byte loads in flight, then probes the eight keys.  The queue holds at
// most 31 keys between push rounds, so one round (<= 32 keys) never
// overflows its kQueueCap entries.
__device__ __forceinline__ unsigned stream_list_q(const int32_t *__restrict__ col, int64_t st,
                                                  int len, int lane, const int *tab,
                                                  unsigned mask, int shift, ProbeQueue &Q,
                                                  unsigned *err) {
  constexpr int kU = 4;
  unsigned hits = 0;
  const int head = (int)(st & 1) & (len > 0 ? 1 : 0);
  const int64_t a = st + head;
  const int rest = len - head;
  const int body = rest >> 1;
  // the scalar ends: head (odd start) on lane 0, odd tail on lane 1
  {
    const bool h = lane == 0 && head;
    const bool t = lane == 1 && (rest & 1);
    const int w = h ? __ldg(col + st) : (t ? __ldg(col + a + 2 * body) : 0);
    hits += home_probe(Q, tab, mask, shift, w, h || t, lane);
    hits += queue_drain(Q, tab, mask, lane, kWarp - 1, err);
  }
  const int2 *v = reinterpret_cast<const int2 *>(col + a);
  for (int k0 = 0; k0 < body; k0 += kWarp * kU) {
    int2 q[kU];
    bool ok[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int k = k0 + u * kWarp + lane;
      ok[u] = k < body;
      q[u] = ok[u] ? __ldg(v + k) : make_int2(0, 0);
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      hits += home_probe(Q, tab, mask, shift, q[u].x, ok[u], lane);
      hits += queue_drain(Q, tab, mask, lane, kWarp - 1, err);
      hits += home_probe(Q, tab, mask, shift, q[u].y, ok[u], lane);
      hits += queue_drain(Q, tab, mask, lane, kWarp - 1, err);
    }
  }
  return hits;
}

// Hub task over entries [e0, e0 + nc) of owner x's symmetric row: the CTA's
// warps claim entries from the shared counter *next (smaller claims as the
// chunk runs out); each claimed neighbour that is a partner has its list
// streamed through the owner's table by the whole warp.
__device__ __forceinline__ unsigned long long claim_and_stream_table(
    const CountArgs &a, int x, int px, int64_t e0, int nc, int *next, int lane, const int *tab,
    unsigned mask, int shift, ProbeQueue &Q) {
  unsigned long long hits = 0;
  for (;;) {
    int g = 0;
    if (lane == 0) {
      const int seen = *(volatile int *)next;
      const int size = max(1, min(kClaim, (nc - seen) / 16));
      g = atomicAdd(next, size) | (size << 20);
    }
    g = __shfl_sync(kFull, g, 0);
    const int size = g >> 20;
    g &= (1 << 20) - 1;
    if (g >= nc) break;
    bool part = false;
    int64_t st = 0;
    int len = 0;
    if (lane < size && g + lane < nc) {
      const int y = __ldg(a.col + e0 + g + lane);
      const int py = __ldg(&a.key[y].y);
      if (owns(x, px, y, py)) {
        part = true;
        st = __ldg(a.dag_rowptr + y);
        len = py;
      }
    }
    unsigned m = __ballot_sync(kFull, part);
    unsigned h = 0;
    while (m) {
      const int p = __ffs(m) - 1;
      m &= m - 1;
      const int64_t s = __shfl_sync(kFull, st, p);
      const int l = __shfl_sync(kFull, len, p);
      h += stream_list_q(a.dag_col, s, l, lane, tab, mask, shift, Q, a.err);
    }
    h += queue_drain(Q, tab, mask, lane, 0, a.err);
    hits += h;
  }
  return hits;
}

// Entries [e0, e0 + nc) of owner x's symmetric row, claimed by the CTA's warps
// kClaim at a time from the shared counter *next; each claimed neighbour that
// is a partner has its list streamed by the whole warp (binary-search probe
// for owners too large for the shared-memory table).
template <class Probe>
__device__ __forceinline__ unsigned long long claim_and_stream(const CountArgs &a, int x, int px,
                                                               int64_t e0, int nc, int *next,
                                                               int lane, const Probe &probe) {
  unsigned long long hits = 0;
  for (;;) {
    int g = 0;
    if (lane == 0) g = atomicAdd(next, kClaim);
    g = __shfl_sync(kFull, g, 0);
    if (g >= nc) break;
    bool part = false;
    int64_t st = 0;
    int len = 0;
    if (lane < kClaim && g + lane < nc) {
      const int y = __ldg(a.col + e0 + g + lane);
      const int py = __ldg(&a.key[y].y);
      if (owns(x, px, y, py)) {
        part = true;
        st = __ldg(a.dag_rowptr + y);
        len = py;
      }
    }
    unsigned m = __ballot_sync(kFull, part);
    unsigned h = 0;
    while (m) {
      const int p = __ffs(m) - 1;
      m &= m - 1;
      const int64_t s = __shfl_sync(kFull, st, p);
      const int l = __shfl_sync(kFull, len, p);
      h += stream_list(a.dag_col, s, l, lane, probe);
    }
    hits += h;
  }
  return hits;
}

// Short lists: lanes 0..k-1 hold one non-empty list each (st, len; the other
// lanes len 0) and the warp walks the concatenated lists 32 entries at a
// time; lane L of window F handles flat entry F + L, whose list is found by
// counting the list starts inside the window.
template <class Probe>
__device__ __forceinline__ unsigned long long stream_flat(const int32_t *__restrict__ col,
                                                          int64_t st, int len, int lane,
                                                          const Probe &probe) {
  unsigned long long hits = 0;
  const int incl = warp_inclusive_scan(len, lane);
  const int excl = incl - len;
  const int total = __shfl_sync(kFull, incl, kWarp - 1);
  const unsigned upto = lane == kWarp - 1 ? kFull : ((2u << lane) - 1u);
  int base = 0;  // lists started before window F
  for (int F = 0; F < total; F += kWarp) {
    const unsigned bit = (len > 0 && excl >= F && excl < F + kWarp) ? (1u << (excl - F)) : 0u;
    const unsigned starts = __reduce_or_sync(kFull, bit);
    const int p = max(base + __popc(starts & upto) - 1, 0);
    const int64_t pst = __shfl_sync(kFull, st, p);
    const int pex = __shfl_sync(kFull, excl, p);
    const int f = F + lane;
    if (f < total) hits += probe(__ldg(col + pst + (f - pex)));
    base += __popc(starts);
  }
  return hits;
}

__device__ __forceinline__ int ceil_log2(int v) { return v <= 1 ? 0 : 32 - __clz(v - 1); }

// One CTA per hub task: N+(owner) into a table of 2^lg slots (load <= 1/4
// when it fits, <= 1/2 at the size cap; owners beyond the cap use binary
// search in global memory), then the 8 warps claim the row chunk kClaim
// entries at a time and stream each partner's list through the table.
__global__ void __launch_bounds__(kCountThreads, 5) tc_hub_kernel(CountArgs a) {
  extern __shared__ int table[];
  __shared__ unsigned long long s_task;
  __shared__ int s_next;
  __shared__ int2 s_queue[kCountThreads / kWarp][kQueueCap];
  const int lane = threadIdx.x & (kWarp - 1);
  ProbeQueue Q{s_queue[threadIdx.x / kWarp], 0};
  const int64_t ntasks = shard_tasks(a);
  unsigned long long hits = 0;
  for (;;) {
    if (threadIdx.x == 0) {
      s_task = atomicAdd(a.queue, 1ull);
      s_next = 0;
    }
    __syncthreads();
    const unsigned long long t = s_task;
    if ((int64_t)t >= ntasks) break;
    const uint64_t task = shard_task(a, t);
    const int x = (int)(task >> 32);
    const int chunk = (int)(task & 0xffffffffu);
    const int64_t a0 = a.dag_rowptr[x];
    const int d = a.key[x].y;
    const int64_t e0 = a.rowptr[x] + (int64_t)chunk * kHubChunk;
    const int nc = (int)min((int64_t)kHubChunk, a.rowptr[x + 1] - e0);
    int lg = max(8, ceil_log2(4 * d));
    if (lg > a.table_log2_max && 2 * d <= (1 << a.table_log2_max)) lg = a.table_log2_max;
    if (lg <= a.table_log2_max) {
      const int size = 1 << lg;
      const unsigned mask = (unsigned)size - 1u;
      const int shift = 32 - lg;
      int4 *t4 = reinterpret_cast<int4 *>(table);
      for (int i = threadIdx.x; i < size / 4; i += blockDim.x) t4[i] = make_int4(-1, -1, -1, -1);
      __syncthreads();
      for (int i = threadIdx.x; i < d; i += blockDim.x)
        table_insert(table, mask, shift, __ldg(a.dag_col + a0 + i), a.err);
      __syncthreads();
      hits += claim_and_stream_table(a, x, d, e0, nc, &s_next, lane, table, mask, shift, Q);
    } else {
      hits += claim_and_stream(a, x, d, e0, nc, &s_next, lane, ListProbe{a.dag_col + a0, d});
    }
    __syncthreads();  // table, s_task and s_next are rewritten by the next task
  }
  hits = warp_sum_u64(hits);
  if (lane == 0 && hits) atomicAdd(a.result, hits);
}

// One warp per leaf task (owner d+ <= kLeafMaxOut): a private 256-slot table;
// the chunk's neighbours, 32 at a time, are filtered to partners whose
// (short) lists are walked flat.
__global__ void __launch_bounds__(kCountThreads) tc_leaf_kernel(CountArgs a) {
  __shared__ int tables[kCountThreads / kWarp][kLeafSlots];
  __shared__ int64_t c_st[kCountThreads / kWarp][kWarp];
  __shared__ int c_len[kCountThreads / kWarp][kWarp];
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x / kWarp;
  int *tab = tables[warp];
  constexpr int lg = 8;  // log2(kLeafSlots)
  static_assert((1 << lg) == kLeafSlots, "leaf table size");
  const TableProbe probe{tab, kLeafSlots - 1, 32 - lg};
  const int64_t ntasks = shard_tasks(a);
  unsigned long long hits = 0;
  for (;;) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(a.queue, 1ull);
    t = __shfl_sync(kFull, t, 0);
    if ((int64_t)t >= ntasks) break;
    const uint64_t task = shard_task(a, t);
    const int x = (int)(task >> 32);
    const int chunk = (int)(task & 0xffffffffu);
    const int64_t a0 = a.dag_rowptr[x];
    const int d = a.key[x].y;
    const int64_t e0 = a.rowptr[x] + (int64_t)chunk * kLeafChunk;
    const int nc = (int)min((int64_t)kLeafChunk, a.rowptr[x + 1] - e0);
    // Partners of the chunk first (kLeafChunk / 32 per lane); no table is
    // built for a chunk without partners.
    static_assert(kLeafChunk == 2 * kWarp, "two neighbours per lane");
    int64_t pst[2] = {0, 0};
    int plen[2] = {0, 0};
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int i = r * kWarp + lane;
      if (i < nc) {
        const int y = __ldg(a.col + e0 + i);
        const int py = __ldg(&a.key[y].y);
        if (owns(x, d, y, py)) {
          pst[r] = __ldg(a.dag_rowptr + y);
          plen[r] = py;
        }
      }
    }
    if (!__any_sync(kFull, plen[0] > 0 || plen[1] > 0)) continue;
    int4 *t4 = reinterpret_cast<int4 *>(tab);
    for (int i = lane; i < kLeafSlots / 4; i += kWarp) t4[i] = make_int4(-1, -1, -1, -1);
    __syncwarp();
    for (int i = lane; i < d; i += kWarp)
      table_insert(tab, kLeafSlots - 1, 32 - lg, __ldg(a.dag_col + a0 + i), a.err);
    __syncwarp();
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      int64_t st = pst[r];
      int len = plen[r];
      // Compact the partners into lanes 0..k-1.
      const unsigned m = __ballot_sync(kFull, len > 0);
      if (len > 0) {
        const int r = __popc(m & ((1u << lane) - 1u));
        c_st[warp][r] = st;
        c_len[warp][r] = len;
      }
      __syncwarp();
      const int k = __popc(m);
      st = lane < k ? c_st[warp][lane] : 0;
      len = lane < k ? c_len[warp][lane] : 0;
      __syncwarp();
      hits += stream_flat(a.dag_col, st, len, lane, probe);
    }
    __syncwarp();
  }
  hits = warp_sum_u64(hits);
  if (lane == 0 && hits) atomicAdd(a.result, hits);
}

int resident_blocks(const void *kernel, int threads, size_t smem) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess)
    per_sm = 1;
  return std::max(per_sm, 1);
}

}  // namespace

int tc_count_launch(mc_dgraph *g, cudaEvent_t after_hub, int shard, int num_shards) {
  if (g->n == 0) {
    if (after_hub) MC_CUDA_TRY(cudaEventRecord(after_hub, g->stream));
    return MC_OK;
  }
  CountArgs a{};
  a.rowptr = g->rowptr;
  a.col = g->col;
  a.key = g->key;
  a.dag_rowptr = g->dag_rowptr;
  a.dag_col = g->dag_col;
  a.result = g->counters + 0;
  a.err = g->err;
  a.table_log2_max = g->hub_table_log2;
  a.shard = shard;
  a.num_shards = num_shards;

  const size_t hub_smem = sizeof(int) << g->hub_table_log2;
  MC_CUDA_TRY(cudaFuncSetAttribute(tc_hub_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)hub_smem));
  const int hub_grid = g->num_sms * resident_blocks((const void *)tc_hub_kernel, kCountThreads, hub_smem);
  a.tasks = g->hub_tasks;
  a.ntasks = g->hub_off + g->n;
  a.queue = g->counters + 1;
  g->launches += 2;
  tc_hub_kernel<<<hub_grid, kCountThreads, hub_smem, g->stream>>>(a);
  MC_CUDA_TRY(cudaGetLastError());
  if (after_hub) MC_CUDA_TRY(cudaEventRecord(after_hub, g->stream));

  const int leaf_grid = g->num_sms * resident_blocks((const void *)tc_leaf_kernel, kCountThreads, 0);
  a.tasks = g->leaf_tasks;
  a.ntasks = g->leaf_off + g->n;
  a.queue = g->counters + 2;
  tc_leaf_kernel<<<leaf_grid, kCountThreads, 0, g->stream>>>(a);
  MC_CUDA_TRY(cudaGetLastError());
  return MC_OK;
}

}  // namespace mc

// Triangle-count kernels.  count = sum over DAG edges {x, y} of
// |N+(x) & N+(y)|, where x is the edge's owner (larger d+, ties to the larger
// id) and y its partner.  A task is (owner, chunk of the owner's symmetric
// row): N+(owner) goes into shared memory (a degree-rank bitmap or a cuckoo
// table), the chunk's neighbours are filtered down to partners (owner rule
// on d+), and each partner's list N+(y) -- never longer than N+(owner) -- is
// streamed through it.
//
// Reference counterparts: hashIndex_for_large_degree (CTA per large vertex,
// 1019-bin hash staged through a 256 MiB global scratch, bin scanned
// linearly per probe, gpu_kernels/tc_challenge.cuh:4-192) and
// binarySearch_for_small_degree (warp per small vertex, binary search in
// shared memory, gpu_kernels/tc_challenge.cuh:195-303), each with an atomic
// work counter (DYNAMIC_MODE, gpu_kernels/tuning_schedules.cuh:1-21).  Here
// the queues hold bounded (owner, row-chunk) tasks, the tables live in shared
// memory only, and a probe is one bitmap word or two fixed table reads with
// no branch.
#include <algorithm>
#include <climits>
#include <cstdlib>

#include "dgraph.cuh"
#include "device_common.cuh"

namespace mc {
namespace {

constexpr int kMaxKicks = 64;  // cuckoo displacements allowed per inserted key
constexpr int kNoKey = INT_MIN;  // probe value that matches no slot

struct CountArgs {
  const int64_t *__restrict__ rowptr;      // symmetric CSR
  const int32_t *__restrict__ col;
  const int2 *__restrict__ key;            // {deg, d+}
  const int4 *__restrict__ pinfo;          // {d+, rank, DAG row start (2 words)}
  const int64_t *__restrict__ dag_rowptr;  // N+ lists
  const int32_t *__restrict__ dag_col;
  const uint64_t *__restrict__ tasks;
  const int64_t *__restrict__ ntasks;  // device scalar (end of the offsets)
  unsigned long long *queue;
  unsigned long long *result;
  unsigned *err;
  int table_log2_max;
  // Degree ranks: every entry of N+(v) ranks below v, so an owner x whose
  // rank fits the launch's bitmap capacity keeps N+(x) as a bitmap of
  // rank(x) bits (null rank: a batch, tables only).
  const int32_t *__restrict__ rank;
  const int32_t *__restrict__ dag_rank;  // N+ lists as ranks
  int bitmap_bits;
  // Core bitmaps of the ranks [0, core_ranks) (null: none), laid out by
  // core_offset().
  const unsigned *__restrict__ core;
  int core_ranks;
  int dense_factor;  // dense when the AND's words <= dense_factor x list length
  int shard, num_shards;  // this call counts tasks shard, shard + num_shards, ...
  BatchView bv;           // per-graph table factor and counts of a batch
  int stage_off;          // staged hub kernel: start of the copy slots (ints)
  int64_t nnz;            // entries of col (the row prefetch never copies past them)
  int short_ranges;       // short stream: one contiguous range per warp (else windows)
  int long_classes;       // long lists of one batch placed before the longer ones
};

// log2 of the table slots per key of owner x's graph (4 slots per key by
// default: load <= 1/4).
__device__ __forceinline__ int table_factor_log2(const CountArgs &a, int x) {
  return a.bv.param ? a.bv.param[a.bv.gid[x]].y : 2;
}

// A batch adds each task's hits to its graph's count (one atomic per warp).
__device__ __forceinline__ void flush_task(const CountArgs &a, int x, unsigned long long task_hits,
                                           int lane) {
  if (!a.bv.res) return;
  task_hits = warp_sum_u64(task_hits);
  if (lane == 0 && task_hits) atomicAdd(a.bv.res + a.bv.gid[x], task_hits);
}

// Tasks of this shard: queue position t maps to task t * num_shards + shard.
__device__ __forceinline__ int64_t shard_tasks(const CountArgs &a) {
  const int64_t total = *a.ntasks;
  return total > a.shard ? (total - a.shard + a.num_shards - 1) / a.num_shards : 0;
}
__device__ __forceinline__ uint64_t shard_task(const CountArgs &a, unsigned long long t) {
  return a.tasks[(int64_t)t * a.num_shards + a.shard];
}

// ---- cuckoo tables ---------------------------------------------------------
// A table of 2^lg int slots (empty = -1).  Key k lives in one of two slots:
// s1 (multiplicative hash) or s2 = s1 ^ (odd second hash), so s2 != s1 and
// each slot names the other.  Lookup reads both slots.
__device__ __forceinline__ void cuckoo_slots(int key, int shift, unsigned &s1, unsigned &s2) {
  s1 = ((unsigned)key * 2654435769u) >> shift;
  s2 = s1 ^ ((((unsigned)key * 0x85EBCA77u) >> shift) | 1u);
}

// A key always enters at s1 and moves to s2 only when another key takes s1,
// and a filled slot never empties: so an empty s1 means the key is absent,
// and s2 is read only when s1 holds a different key.
struct CuckooProbe {
  const int *tab;
  int shift;
  __device__ __forceinline__ unsigned operator()(int w) const {
    unsigned s1, s2;
    cuckoo_slots(w, shift, s1, s2);
    const int t1 = tab[s1];
    unsigned hit = t1 == w;
    if (t1 >= 0 && t1 != w) hit = tab[s2] == w;
    return hit;
  }
};

// Concurrent insertion: exchange the key into a slot and carry the evicted
// key to its other slot.  Every key stays in exactly one carrier (a slot or
// a thread), so with all threads done each inserted key sits in s1 or s2 --
// unless a thread ran out of displacements, in which case the key it carries
// is not stored and the function returns false.
__device__ __forceinline__ bool cuckoo_insert(int *tab, int shift, int key) {
  unsigned s1, s2;
  cuckoo_slots(key, shift, s1, s2);
  unsigned pos = s1;
  int k = key;
  for (int kick = 0; kick < kMaxKicks; ++kick) {
    const int old = atomicExch(tab + pos, k);
    if (old < 0) return true;
    k = old;
    cuckoo_slots(k, shift, s1, s2);
    pos = pos == s1 ? s2 : s1;
  }
  return false;
}

// Membership in the owner's bitmap over ranks [0, R), by a clamped word
// index and no range test: bits at or above R are never set, and word
// `zero` (the first word of the quad cleared after the bitmap's own quads)
// is all zero, so every rank at or above R -- kNoKey included -- reads a
// zero bit.  The probe is straight-line code with no branch.
struct BitmapProbe {
  const unsigned *bits;
  unsigned zero;
  __device__ __forceinline__ unsigned operator()(int w) const {
    const unsigned u = (unsigned)w;
    return (bits[min(u >> 5, zero)] >> (u & 31)) & 1u;
  }
};

// Binary search in a sorted global list: owners too large for the table, or
// whose table could not be built.
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

// Partner test for neighbour y of owner x (px = d+(x), py = d+(y)).
__device__ __forceinline__ bool owns(int x, int px, int y, int py) {
  return py >= 1 && (px > py || (px == py && x > y));
}

// Partner lists at least this long are streamed by one warp each; shorter
// ones are concatenated and streamed flat by the whole CTA.
constexpr int kLongList = 64;

// Partners of one hub task, compacted in row order.  Thread t examines
// neighbours 2t and 2t+1 of the chunk; one block scan of (long partners of
// one batch, longer long partners, short partners, dense partners, short
// list lengths) packed in 64 bits places every partner: four 11-bit counts
// (a chunk has at most 1024 partners) and a 16-bit length sum (at most
// 1024 x 63).  Long list j (j < nl): start base[j], length off[j].  Short
// list j: elements [off[nl+j], off[nl+j+1]) of the short stream, element f
// of it at lists[base[nl+j] + f] (base = list start - offset).  Dense
// partner j (j < nd): its rank at base[kHubChunk - 1 - j], above every long
// and short entry.
//
// A long partner y is dense when the owner keeps a bitmap (owner_bits, its
// rank) and y has a core bitmap whose AND with it over the words below both
// ranks takes at most dense_factor words per entry of y's list.
struct Partners {
  int nl;     // long lists
  int total;  // elements of the short stream
  int nd;     // dense partners
  int ns;     // short lists
};

// Fields of the partner scan's 64-bit word.
constexpr int kLenShift = 0, kDenseShift = 16, kShortShift = 27, kLongAShift = 38,
              kLongBShift = 49;
constexpr unsigned long long kLenMask = 0xffffull, kCountMask = 0x7ffull;
static_assert(kLongBShift + 11 <= 64 && kHubChunk <= 1024 && kHubChunk * 63 <= 0xffff,
              "partner scan fields hold a chunk's counts and short lengths");

// The chunk's neighbours come from the row prefetch in shared memory where
// it holds them (entries [ca, cend) of col at s_col[0 ..)), else from global
// memory.
struct ChunkSource {
  const int *s_col;  // null: every neighbour from global memory
  long long ca, cend;
};

__device__ __forceinline__ Partners find_partners(const CountArgs &a, int x, int px, int64_t e0,
                                                  int nc, long long *s_base, int *s_off,
                                                  unsigned long long *s_warp, int owner_bits,
                                                  ChunkSource src = ChunkSource{nullptr, 0, 0}) {
  constexpr int kR = kHubChunk / kCountThreads;  // neighbours per thread
  static_assert(kR * kCountThreads == kHubChunk && kHubChunk <= 1024,
                "whole neighbours per thread; 16-bit scan fields");
  constexpr int kWarps = kCountThreads / kWarp;
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x / kWarp;
  int len[kR] = {};
  long long st[kR] = {};
  bool dense[kR] = {};
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    const int i = kR * threadIdx.x + r;
    if (i < nc) {
      const long long e = e0 + i;
      const int y = src.s_col && e < src.cend ? src.s_col[e - src.ca] : __ldg(a.col + e);
      const int4 pi = __ldg(a.pinfo + y);
      const int py = pi.x;
      if (owns(x, px, y, py)) {
        len[r] = py;
        if (py >= kLongList && owner_bits > 0) {
          const int ry = pi.y;
          const int words = (min(ry, owner_bits) + 31) >> 5;
          dense[r] = ry < a.core_ranks && words <= a.dense_factor * py;
          if (dense[r]) st[r] = ry;
        }
        if (!dense[r]) st[r] = ((long long)pi.w << 32) | (unsigned)pi.z;
      }
    }
  }
  // Long lists of one 128-entry batch (64..127 entries) take the slots
  // before the longer ones, so a claimed pair mostly streams two lists of
  // the same batch count (at RMAT scale 22, counted on the CPU: 22.8 M pair
  // batches against 25.8 M in row order).  Off (long_classes 0): every long
  // list in row order.
  const bool classes = a.long_classes != 0;
  unsigned long long mine = 0;
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    if (dense[r]) mine += 1ull << kDenseShift;
    else if (len[r] >= kLongList)
      mine += 1ull << (classes && len[r] >= 2 * kLongList ? kLongBShift : kLongAShift);
    else if (len[r] > 0) mine += (1ull << kShortShift) + ((unsigned long long)len[r] << kLenShift);
  }
  unsigned long long incl = mine;
#pragma unroll
  for (int o = 1; o < kWarp; o <<= 1) {
    const unsigned long long v = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == kWarp - 1) s_warp[warp] = incl;
  __syncthreads();
  unsigned long long before = 0, all = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    const unsigned long long v = s_warp[w];
    if (w < warp) before += v;
    all += v;
  }
  const unsigned long long excl = before + incl - mine;
  auto field = [](unsigned long long v, int shift) { return (int)((v >> shift) & kCountMask); };
  const int nla = field(all, kLongAShift);
  const int nl = nla + field(all, kLongBShift), ns = field(all, kShortShift);
  const int nd = field(all, kDenseShift);
  int aslot = field(excl, kLongAShift), bslot = nla + field(excl, kLongBShift);
  int sslot = nl + field(excl, kShortShift), off = (int)((excl >> kLenShift) & kLenMask);
  int dslot = field(excl, kDenseShift);
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    if (dense[r]) {
      s_base[kHubChunk - 1 - dslot] = st[r];
      ++dslot;
    } else if (len[r] >= kLongList) {
      const bool b = classes && len[r] >= 2 * kLongList;
      const int slot = b ? bslot++ : aslot++;
      s_base[slot] = st[r];
      s_off[slot] = len[r];
    } else if (len[r] > 0) {
      s_base[sslot] = st[r] - off;
      s_off[sslot] = off;
      ++sslot;
      off += len[r];
    }
  }
  const int total = (int)((all >> kLenShift) & kLenMask);
  if (threadIdx.x == 0) s_off[nl + ns] = total;
  __syncthreads();
  return Partners{nl, total, nd, ns};
}

// One warp streams N lists lists[st[i], st[i] + len[i]) together with
// lane-per-element loads (128 bytes per instruction): every load of a
// 128-element batch of every list is issued before the first probe, so a
// warp keeps 4 N loads in flight per lane.  Entries past a list's end probe
// as kNoKey, which costs less than a branch per 32-entry group.  Batch depth
// 4 with N = 2 measured best (depths 2..8 with N = 1, N = 3 slower, and
// 16-byte loads slower still, at RMAT scale 22).
template <int N, class Probe>
__device__ __forceinline__ unsigned stream_n(const int32_t *__restrict__ lists, const long long *st,
                                             const int *len, int lane, const Probe &probe) {
  constexpr int kB = 4;
  int mx = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) mx = max(mx, len[i]);
  unsigned h = 0;
  for (int base = 0; base < mx; base += kB * kWarp) {
    int w[N][kB];
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int k = base + u * kWarp + lane;
#pragma unroll
      for (int i = 0; i < N; ++i) w[i][u] = k < len[i] ? __ldg(lists + st[i] + k) : kNoKey;
    }
#pragma unroll
    for (int u = 0; u < kB; ++u)
#pragma unroll
      for (int i = 0; i < N; ++i) h += probe(w[i][u]);
  }
  return h;
}

// ---- bulk-copy staging of long partner lists (MERCURY_TC_TMA=1) -----------
// Each warp owns two 1 KB slots of shared memory and two mbarriers.  Lane 0
// copies the next chunk of the claimed lists (up to 252 entries) from global
// memory into one slot with cp.async.bulk (no multicast: this GPU's own
// memory, one CTA) while the warp probes the chunk already in the other
// slot.  A bulk copy starts and ends on 16-byte boundaries, so a chunk's
// start is rounded down to a multiple of 4 entries and its end up (the list
// arrays carry 4 entries of padding for that); the warp indexes the slot
// from the remainder.
constexpr int kStageInts = 256;
constexpr int kStageChunk = kStageInts - 4;
constexpr size_t kStageBytes = (size_t)(kCountThreads / kWarp) * 2 * kStageInts * sizeof(int);
constexpr int kWaitSpins = 1 << 20;  // try_wait rounds before a wait gives up

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
// Lane 0: expect `bytes` on bar, then copy them (16-byte aligned, multiple of 16).
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, unsigned bytes,
                                          unsigned long long *bar) {
  // The warp's earlier (generic) reads of dst are ordered before this
  // asynchronous write by the __syncwarp before the call and this fence.
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Waits for the phase of `parity` on bar; false after kWaitSpins rounds.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity) {
  for (int i = 0; i < kWaitSpins; ++i) {
    unsigned done = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

struct Stage {
  int *slot[2];                  // this warp's two slots
  unsigned long long *bar;       // this warp's two mbarriers
  unsigned phase;                // bit s: parity of slot s's next completion
  unsigned *err;
};

// The N claimed lists (starts st[i], lengths len[i]) as chunks through the
// two slots; returns this lane's hits.  A wait that gives up raises
// kErrWaitTimeout and waits once more for the copy before returning.
template <int N, class Probe>
__device__ __forceinline__ unsigned stream_n_staged(const int32_t *__restrict__ lists,
                                                    const long long *st, const int *len,
                                                    int lane, const Probe &probe, Stage &sg) {
  int ci = 0;
  while (ci < N && len[ci] <= 0) ++ci;
  if (ci >= N) return 0;
  int co = 0, s = 0;
  auto issue = [&](int i, int o, int slot) {
    if (lane == 0) {
      const long long first = st[i] + o;
      const long long a = first & ~3LL;
      const int cnt = min(kStageChunk, len[i] - o);
      const unsigned bytes = (unsigned)((((first - a) + cnt + 3) & ~3LL) * sizeof(int));
      bulk_copy(sg.slot[slot], lists + a, bytes, sg.bar + slot);
    }
  };
  issue(ci, co, s);
  unsigned h = 0;
  for (;;) {
    // The chunk after (ci, co), issued into the other slot before waiting.
    int ni = ci, no = co + kStageChunk;
    if (no >= len[ni]) {
      no = 0;
      ++ni;
      while (ni < N && len[ni] <= 0) ++ni;
    }
    if (ni < N) issue(ni, no, s ^ 1);
    const unsigned parity = (sg.phase >> s) & 1u;
    if (!mbar_wait(sg.bar + s, parity)) {
      if (lane == 0) atomicOr(sg.err, kErrWaitTimeout);
      mbar_wait(sg.bar + s, parity);
      if (ni < N) mbar_wait(sg.bar + (s ^ 1), (sg.phase >> (s ^ 1)) & 1u);
      return h;
    }
    sg.phase ^= 1u << s;
    const int shift = (int)((st[ci] + co) & 3LL);
    const int cnt = min(kStageChunk, len[ci] - co);
    const int *buf = sg.slot[s] + shift;
    for (int k = lane; k < cnt; k += kWarp) h += probe(buf[k]);
    __syncwarp();  // every lane is done with slot s before it is refilled
    if (ni >= N) break;
    ci = ni;
    co = no;
    s ^= 1;
  }
  return h;
}

// The short stream: warp w takes windows of 32 x kU consecutive elements
// (w, w + 8, ...), lane l element window + 32u + l, so every load
// instruction reads one 128-byte span and every lane has kU loads in
// flight.  An element's list is found by walking forward from the window's
// first list (lists are at least one element long).
template <class Probe>
__device__ __forceinline__ unsigned stream_short(const int32_t *__restrict__ lists,
                                                 const long long *s_base, const int *s_off,
                                                 int total, int warp, int lane,
                                                 const Probe &probe) {
  constexpr int kU = 4;
  constexpr int kWarps = kCountThreads / kWarp;
  unsigned hits = 0;
  int j = 0;  // list holding the warp's window start (the same on every lane)
  for (int wb = warp * kWarp * kU; wb < total; wb += kWarps * kWarp * kU) {
    while (s_off[j + 1] <= wb) ++j;
    int w[kU];
    int jj = j;
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int f = wb + u * kWarp + lane;
      w[u] = kNoKey;
      if (f < total) {
        while (s_off[jj + 1] <= f) ++jj;
        w[u] = __ldg(lists + s_base[jj] + f);
      }
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) hits += probe(w[u]);
  }
  return hits;
}

// The short stream in contiguous ranges: warp w takes elements [lo, hi), an
// eighth of the stream rounded to whole 128-element windows, so a lane's list
// pointer only ever moves forward across the warp's windows.  (With the
// windows w, w + 8, ... every warp steps over all lists of the task between
// its windows: at RMAT scale 22, counted on the CPU, 78 M list steps between
// windows and 24 M inside them, against 36 M for the ranges.)  The list
// holding lo is found by one binary search over the ns + 1 offsets.
template <class Probe>
__device__ __forceinline__ unsigned stream_short_ranges(const int32_t *__restrict__ lists,
                                                        const long long *s_base, const int *s_off,
                                                        int total, int ns, int warp, int lane,
                                                        const Probe &probe) {
  constexpr int kU = 4;
  constexpr int kWarps = kCountThreads / kWarp;
  constexpr int kWin = kWarp * kU;
  const int span = (total + kWarps * kWin - 1) / (kWarps * kWin) * kWin;
  const int lo = warp * span, hi = min(total, lo + span);
  unsigned hits = 0;
  if (lo >= hi) return hits;
  int l = 0, r = ns - 1;  // s_off[0] = 0 <= lo < total = s_off[ns]
  while (l < r) {
    const int m = (l + r + 1) >> 1;
    if (s_off[m] <= lo) l = m;
    else r = m - 1;
  }
  int jj = l;  // this lane's list, carried across the windows
  for (int wb = lo; wb < hi; wb += kWin) {
    int w[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int f = wb + u * kWarp + lane;
      w[u] = kNoKey;
      if (f < hi) {
        while (s_off[jj + 1] <= f) ++jj;
        w[u] = __ldg(lists + s_base[jj] + f);
      }
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) hits += probe(w[u]);
  }
  return hits;
}

// |N+(owner) & N+(y)| summed over N dense partners y of ranks ry[i] (-1:
// none): the AND of the owner's bitmap (shared memory, cleared to whole
// quads past its rank) and each y's core bitmap over the quads below both
// ranks, lane-per-quad (16-byte loads: 512 bytes per instruction, no bank
// conflict), 2 N loads in flight per lane (N = 4 measured best of 1, 2, 4).
template <int N>
__device__ __forceinline__ unsigned and_count_n(const unsigned *bits, int owner_bits,
                                                const unsigned *__restrict__ core, const int *ry,
                                                int lane) {
  const uint4 *o = reinterpret_cast<const uint4 *>(bits);
  const uint4 *q[N];
  int nq[N];
  int mx = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    q[i] = reinterpret_cast<const uint4 *>(core + core_offset(max(ry[i], 0)));
    nq[i] = ry[i] >= 0 ? (min(ry[i], owner_bits) + 127) >> 7 : 0;
    mx = max(mx, nq[i]);
  }
  unsigned h = 0;
  for (int base = 0; base < mx; base += 2 * kWarp) {
    uint4 v[N][2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int k = base + u * kWarp + lane;
#pragma unroll
      for (int i = 0; i < N; ++i) v[i][u] = k < nq[i] ? __ldg(q[i] + k) : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int k = base + u * kWarp + lane;
      const uint4 w = o[k < mx ? k : 0];
#pragma unroll
      for (int i = 0; i < N; ++i)
        h += __popc(w.x & v[i][u].x) + __popc(w.y & v[i][u].y) + __popc(w.z & v[i][u].z) +
             __popc(w.w & v[i][u].w);
    }
  }
  return h;
}

// All partner lists of the task: the long ones (two per claim) and the
// dense partners (four per claim) claimed by the warps, then the short
// stream.  Returns this thread's hits.
template <bool kStaged, class Probe>
__device__ __forceinline__ unsigned long long stream_partners(const int32_t *__restrict__ lists,
                                                              const long long *s_base,
                                                              const int *s_off, Partners pt,
                                                              int *s_next, int warp, int lane,
                                                              const Probe &probe, Stage &sg,
                                                              bool short_ranges,
                                                              const unsigned *bits = nullptr,
                                                              int owner_bits = 0,
                                                              const unsigned *core = nullptr) {
  unsigned long long hits = 0;
  constexpr int kNL = 2, kND = 4;
  const int lp = (pt.nl + kNL - 1) / kNL, dp = (pt.nd + kND - 1) / kND;
  for (;;) {
    int j = 0;
    if (lane == 0) j = atomicAdd(s_next, 1);
    j = __shfl_sync(kFull, j, 0);
    if (j >= lp + dp) break;
    if (j < lp) {
      long long st[kNL];
      int len[kNL];
#pragma unroll
      for (int i = 0; i < kNL; ++i) {
        const int a = kNL * j + i;
        st[i] = a < pt.nl ? s_base[a] : 0;
        len[i] = a < pt.nl ? s_off[a] : 0;
      }
      if constexpr (kStaged) hits += stream_n_staged<kNL>(lists, st, len, lane, probe, sg);
      else hits += stream_n<kNL>(lists, st, len, lane, probe);
    } else {
      int ry[kND];
#pragma unroll
      for (int i = 0; i < kND; ++i) {
        const int a = kND * (j - lp) + i;
        ry[i] = a < pt.nd ? (int)s_base[kHubChunk - 1 - a] : -1;
      }
      hits += and_count_n<kND>(bits, owner_bits, core, ry, lane);
    }
  }
  if (pt.total > 0) {
    if (short_ranges)
      hits += stream_short_ranges(lists, s_base + pt.nl, s_off + pt.nl, pt.total, pt.ns, warp,
                                  lane, probe);
    else
      hits += stream_short(lists, s_base + pt.nl, s_off + pt.nl, pt.total, warp, lane, probe);
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
    hits += probe(f < total ? __ldg(col + pst + (f - pex)) : kNoKey);
    base += __popc(starts);
  }
  return hits;
}

__device__ __forceinline__ int ceil_log2(int v) { return v <= 1 ? 0 : 32 - __clz(v - 1); }

// A hub task as its CTA reads it: owner x with d+ d and rank R, the start a0
// of N+(x), and the chunk [e0, e0 + nc) of x's symmetric row.  With the row
// prefetch, [ca, cend) is the part of the chunk, widened to 16-byte bounds,
// that a bulk copy brought into shared memory (cend <= ca: none).
struct HubTask {
  long long a0, e0, ca, cend;
  int x, d, nc, R;
};

__device__ __forceinline__ HubTask hub_task(const CountArgs &a, unsigned long long t) {
  HubTask h;
  const uint64_t task = shard_task(a, t);
  h.x = (int)(task >> 32);
  const int chunk = (int)(task & 0xffffffffu);
  h.a0 = a.dag_rowptr[h.x];
  h.d = a.key[h.x].y;
  h.e0 = a.rowptr[h.x] + (int64_t)chunk * kHubChunk;
  h.nc = (int)min((long long)kHubChunk, (long long)(a.rowptr[h.x + 1] - h.e0));
  h.R = a.rank ? __ldg(a.rank + h.x) : INT_MAX;
  h.ca = h.cend = 0;
  return h;
}

// Row prefetch: shared-memory ints for one chunk widened to 16-byte bounds
// (at most kHubChunk + 4 after rounding both ends).
constexpr int kRowStageInts = kHubChunk + 8;

// Thread 0, one task ahead: task t's header into *s_hdr and its row chunk
// into s_col by one cp.async.bulk (this GPU's own memory, no multicast)
// completing on bar.  The copy starts at the chunk's first entry rounded
// down to 16 bytes and ends at its last rounded up, but never past the
// column array's last whole 16 bytes: entries after cend come from global
// memory.
__device__ __forceinline__ void row_prefetch(const CountArgs &a, unsigned long long t,
                                             HubTask *s_hdr, int *s_col,
                                             unsigned long long *bar) {
  HubTask h = hub_task(a, t);
  const long long ca = h.e0 & ~3LL;
  const long long cend = min((long long)((h.e0 + h.nc + 3) & ~3LL), (long long)(a.nnz & ~3LL));
  if (cend > ca) {
    h.ca = ca;
    h.cend = cend;
    bulk_copy(s_col, a.col + ca, (unsigned)((cend - ca) * sizeof(int)), bar);
  }
  *s_hdr = h;
}

// One CTA per hub task: N+(owner) into shared memory; the chunk's partners
// are found in one pass and compacted; then the whole CTA streams their
// concatenated lists through it.  N+(owner) is kept as a bitmap over ranks
// [0, rank(owner)) when that fits the launch's shared memory (lists streamed
// as ranks), else as a cuckoo table of 2^lg slots (load <= 1/4 when it fits,
// <= 1/2 at the size cap).  Owners beyond the cap, or whose table could not
// be built, are probed by binary search in global memory instead.
// kStaged: long partner lists through the bulk-copy slots (stream_n_staged),
// which follow the table in dynamic shared memory at a.stage_off ints.
// (The copy slots' 16 KB leave room for 4 CTAs per SM, which the register
// bound then follows.)
// kRowStage (MERCURY_TC_ROW_STAGE=1, off by default): thread 0 reads the
// next task's header and bulk-copies its row chunk into shared memory while
// the current task streams, so a task starts with its owner, offsets and
// neighbour ids already on chip: the chain task -> owner row -> neighbours
// -> partner records shrinks to its last load.  It measured slower (the
// header loads hold warp 0 while the rest of the CTA waits for it at the
// end-of-task barrier).
template <bool kStaged, bool kRowStage>
__global__ void __launch_bounds__(kCountThreads, kStaged ? 4 : 5) tc_hub_kernel(CountArgs a) {
  extern __shared__ __align__(128) int table[];
  __shared__ unsigned long long s_task;
  __shared__ int s_fail, s_next;
  __shared__ long long s_base[kHubChunk];
  __shared__ int s_off[kHubChunk + 1];
  __shared__ unsigned long long s_warp[kCountThreads / kWarp];
  __shared__ unsigned long long s_bar[kStaged ? kCountThreads / kWarp * 2 : 1];
  __shared__ __align__(16) int s_col[kRowStage ? kRowStageInts : 4];
  __shared__ HubTask s_hdr;
  __shared__ unsigned long long s_cbar;
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x / kWarp;
  const int64_t ntasks = shard_tasks(a);
  unsigned long long hits = 0;
  Stage sg{{nullptr, nullptr}, s_bar + (kStaged ? 2 * warp : 0), 0u, a.err};
  if constexpr (kStaged) {
    int *base = table + a.stage_off + warp * 2 * kStageInts;
    sg.slot[0] = base;
    sg.slot[1] = base + kStageInts;
    if (lane == 0) {
      mbar_init(sg.bar);
      mbar_init(sg.bar + 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
  }
  // Parity of the row-prefetch barrier's next completion (the same on every
  // thread: each waits once per copied chunk).
  unsigned cphase = 0;
  // Thread 0 claims each task one task ahead, so the queue atomic's latency
  // overlaps the current task.
  unsigned long long t_next = 0;
  if (threadIdx.x == 0) {
    const unsigned long long t0 = atomicAdd(a.queue, 1ull);
    s_task = t0;
    if constexpr (kRowStage) {
      mbar_init(&s_cbar);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      if ((int64_t)t0 < ntasks) row_prefetch(a, t0, &s_hdr, s_col, &s_cbar);
    }
  }
  for (;;) {
    if (threadIdx.x == 0) {
      s_fail = 0;
      s_next = 0;
    }
    __syncthreads();
    const unsigned long long t = s_task;
    if ((int64_t)t >= ntasks) break;
    if (threadIdx.x == 0) t_next = atomicAdd(a.queue, 1ull);
    HubTask h;
    if constexpr (kRowStage) h = s_hdr;
    else h = hub_task(a, t);
    const int x = h.x, d = h.d, nc = h.nc, R = h.R;
    const int64_t a0 = h.a0, e0 = h.e0;
    const bool bitmap = R <= a.bitmap_bits;
    int lg = max(8, ceil_log2(d << table_factor_log2(a, x)));
    if (lg > a.table_log2_max && 2 * d <= (1 << a.table_log2_max)) lg = a.table_log2_max;
    bool use_table = !bitmap && lg <= a.table_log2_max;
    const int shift = 32 - lg;
    // Clear the bitmap / table, then find the partners (their loads overlap).
    int4 *t4 = reinterpret_cast<int4 *>(table);
    if (bitmap) {
      // The bitmap's quads and one more (the probe's zero word).
      for (int i = threadIdx.x; i <= (R + 127) >> 7; i += blockDim.x) t4[i] = make_int4(0, 0, 0, 0);
    } else if (use_table) {
      for (int i = threadIdx.x; i < (1 << lg) / 4; i += blockDim.x) t4[i] = make_int4(-1, -1, -1, -1);
    }
    // The owner's first kOwnAhead x 256 out-list entries are loaded now and
    // stored after the partner scan (whose barriers also order them after
    // the clear), so their loads overlap the scan's.
    constexpr int kOwnAhead = 4;
    int own[kOwnAhead];
    const int32_t *own_list = bitmap ? a.dag_rank + a0 : a.dag_col + a0;
#pragma unroll
    for (int r = 0; r < kOwnAhead; ++r) {
      const int i = threadIdx.x + r * kCountThreads;
      own[r] = (bitmap || use_table) && i < d ? __ldg(own_list + i) : -1;
    }
    // Dense partners need the owner's bitmap and the core bitmaps.
    const int owner_bits = bitmap && a.core ? R : 0;
    ChunkSource src{nullptr, 0, 0};
    if constexpr (kRowStage) {
      if (h.cend > h.ca) {
        // A wait that gives up raises kErrWaitTimeout (the call then fails),
        // waits once more for the copy, and reads the chunk from global memory.
        if (mbar_wait(&s_cbar, cphase)) {
          src = ChunkSource{s_col, h.ca, h.cend};
        } else {
          atomicOr(a.err, kErrWaitTimeout);
          mbar_wait(&s_cbar, cphase);
        }
        cphase ^= 1u;
      }
    }
    const Partners pt = find_partners(a, x, d, e0, nc, s_base, s_off, s_warp, owner_bits, src);
    // N+(x) into shared memory.
    if (bitmap) {
      unsigned *bits = reinterpret_cast<unsigned *>(table);
      auto set = [&](unsigned r) {
        if (r < (unsigned)R) atomicOr(bits + (r >> 5), 1u << (r & 31));
        else atomicOr(a.err, kErrRank);  // never written outside the bitmap
      };
#pragma unroll
      for (int r = 0; r < kOwnAhead; ++r)
        if (own[r] >= 0) set((unsigned)own[r]);
      for (int i = threadIdx.x + kOwnAhead * kCountThreads; i < d; i += blockDim.x)
        set((unsigned)__ldg(a.dag_rank + a0 + i));
    } else if (use_table) {
      bool ok = true;
#pragma unroll
      for (int r = 0; r < kOwnAhead; ++r)
        if (own[r] >= 0) ok &= cuckoo_insert(table, shift, own[r]);
      for (int i = threadIdx.x + kOwnAhead * kCountThreads; i < d; i += blockDim.x)
        ok &= cuckoo_insert(table, shift, __ldg(a.dag_col + a0 + i));
      if (!ok) s_fail = 1;
    }
    __syncthreads();
    if constexpr (kRowStage) {
      // Every thread has read this task's header and chunk (two barriers
      // ago): the next task's may replace them.
      if (threadIdx.x == 0 && (int64_t)t_next < ntasks)
        row_prefetch(a, t_next, &s_hdr, s_col, &s_cbar);
    }
    use_table = use_table && s_fail == 0;
    const bool ranges = a.short_ranges != 0;
    unsigned long long th = 0;
    if (bitmap)
      th = stream_partners<kStaged>(
          a.dag_rank, s_base, s_off, pt, &s_next, warp, lane,
          BitmapProbe{reinterpret_cast<const unsigned *>(table), (unsigned)(((R + 127) >> 7) << 2)},
          sg, ranges,
          reinterpret_cast<const unsigned *>(table), R, a.core);
    else if (use_table)
      th = stream_partners<kStaged>(a.dag_col, s_base, s_off, pt, &s_next, warp, lane,
                                    CuckooProbe{table, shift}, sg, ranges);
    else
      th = stream_partners<false>(a.dag_col, s_base, s_off, pt, &s_next, warp, lane,
                                  ListProbe{a.dag_col + a0, d}, sg, ranges);
    hits += th;
    flush_task(a, x, th, lane);
    if (threadIdx.x == 0) s_task = t_next;  // every thread read s_task two barriers ago
    __syncthreads();  // shared memory is rewritten by the next task
  }
  hits = warp_sum_u64(hits);
  if (lane == 0 && hits) atomicAdd(a.result, hits);
}

// One warp per leaf task (owner d+ <= kLeafMaxOut): a private 256-slot cuckoo
// table (load <= 1/4); the chunk's neighbours are filtered to partners whose
// (short) lists are walked flat.
// A leaf task as the warp holds it: the owner, the first 64 entries of its
// out-list (two per lane; kLeafMaxOut is 64, a batch may route up to 128)
// and the chunk's neighbours (two per lane).
struct LeafTask {
  bool valid;
  int x, d;
  int64_t a0;
  int y[2];   // neighbour ids, -1 past the chunk
  int ow[2];  // owner out-list entries, kNoKey past d+
};

__device__ __forceinline__ LeafTask leaf_fetch(const CountArgs &a, int64_t ntasks,
                                               unsigned long long t, int lane) {
  LeafTask k;
  k.valid = (int64_t)t < ntasks;
  k.x = 0;
  k.d = 0;
  k.a0 = 0;
  k.y[0] = k.y[1] = -1;
  k.ow[0] = k.ow[1] = kNoKey;
  if (!k.valid) return k;
  const uint64_t task = shard_task(a, t);
  k.x = (int)(task >> 32);
  const int chunk = (int)(task & 0xffffffffu);
  k.a0 = a.dag_rowptr[k.x];
  k.d = a.key[k.x].y;
  const int64_t e0 = a.rowptr[k.x] + (int64_t)chunk * kLeafChunk;
  const int nc = (int)min((int64_t)kLeafChunk, a.rowptr[k.x + 1] - e0);
  static_assert(kLeafChunk == 2 * kWarp, "two neighbours per lane");
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int i = r * kWarp + lane;
    if (i < nc) k.y[r] = __ldg(a.col + e0 + i);
    if (i < k.d) k.ow[r] = __ldg(a.dag_col + k.a0 + i);
  }
  return k;
}

// One warp per leaf task (owner d+ <= kLeafMaxOut): a private 256-slot cuckoo
// table (load <= 1/4); the chunk's neighbours are filtered to partners whose
// (short) lists are walked flat.  Every load of a task is a short dependent
// chain (task -> owner row -> neighbours -> their d+ -> their list start ->
// list entries), so the warp fetches the next task's owner, out-list and
// neighbours while it works on the current one.
__global__ void __launch_bounds__(kCountThreads) tc_leaf_kernel(CountArgs a) {
  __shared__ int tables[kCountThreads / kWarp][kLeafSlots];
  __shared__ int64_t c_st[kCountThreads / kWarp][kWarp];
  __shared__ int c_len[kCountThreads / kWarp][kWarp];
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x / kWarp;
  int *tab = tables[warp];
  constexpr int lg = 8;  // log2(kLeafSlots)
  static_assert((1 << lg) == kLeafSlots, "leaf table size");
  static_assert(4 * kLeafMaxOut <= kLeafSlots, "leaf table load <= 1/4");
  const CuckooProbe probe{tab, 32 - lg};
  const int64_t ntasks = shard_tasks(a);
  unsigned long long hits = 0;
  // Tasks are claimed kLeafClaim at a time: one queue atomic per 16 tasks
  // instead of per task (millions of them contend on one address).
  constexpr unsigned long long kLeafClaim = 16;
  unsigned long long batch = 0, used = kLeafClaim;
  auto next_ticket = [&]() {
    if (used == kLeafClaim) {
      unsigned long long b = 0;
      if (lane == 0) b = atomicAdd(a.queue, kLeafClaim);
      batch = __shfl_sync(kFull, b, 0);
      used = 0;
    }
    return batch + used++;
  };
  LeafTask cur = leaf_fetch(a, ntasks, next_ticket(), lane);
  while (cur.valid) {
    // Partners of the current chunk: d+ of each neighbour, then the list start.
    int4 pi[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) pi[r] = cur.y[r] >= 0 ? __ldg(a.pinfo + cur.y[r]) : make_int4(0, 0, 0, 0);
    // The next task (claimed while those loads are in flight).
    const unsigned long long tn = next_ticket();
    int64_t pst[2] = {0, 0};
    int plen[2] = {0, 0};
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      if (cur.y[r] >= 0 && owns(cur.x, cur.d, cur.y[r], pi[r].x)) {
        pst[r] = ((long long)pi[r].w << 32) | (unsigned)pi[r].z;
        plen[r] = pi[r].x;
      }
    }
    // The next task's owner row, out-list and neighbours.
    const LeafTask next = leaf_fetch(a, ntasks, tn, lane);
    if (__any_sync(kFull, plen[0] > 0 || plen[1] > 0)) {
      int4 *t4 = reinterpret_cast<int4 *>(tab);
      for (int i = lane; i < kLeafSlots / 4; i += kWarp) t4[i] = make_int4(-1, -1, -1, -1);
      __syncwarp();
      bool ok = true;
#pragma unroll
      for (int r = 0; r < 2; ++r)
        if (cur.ow[r] != kNoKey) ok &= cuckoo_insert(tab, 32 - lg, cur.ow[r]);
      // A batch's autotuner may route owners of d+ up to 128 here: the
      // entries past the 64 fetched ahead come from memory.
      for (int i = 2 * kWarp + lane; i < cur.d; i += kWarp)
        ok &= cuckoo_insert(tab, 32 - lg, __ldg(a.dag_col + cur.a0 + i));
      const bool use_table = __all_sync(kFull, ok);
      __syncwarp();
      unsigned long long th = 0;
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        int64_t st = pst[r];
        int len = plen[r];
        // Compact the partners into lanes 0..k-1.
        const unsigned m = __ballot_sync(kFull, len > 0);
        if (len > 0) {
          const int rank = __popc(m & ((1u << lane) - 1u));
          c_st[warp][rank] = st;
          c_len[warp][rank] = len;
        }
        __syncwarp();
        const int k = __popc(m);
        st = lane < k ? c_st[warp][lane] : 0;
        len = lane < k ? c_len[warp][lane] : 0;
        __syncwarp();
        if (use_table) th += stream_flat(a.dag_col, st, len, lane, probe);
        else th += stream_flat(a.dag_col, st, len, lane, ListProbe{a.dag_col + cur.a0, cur.d});
      }
      hits += th;
      flush_task(a, cur.x, th, lane);
      __syncwarp();
    }
    cur = next;
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
  NvtxRange range("tc_count_launch");
  if (g->n == 0) {
    if (after_hub) MC_CUDA_TRY(cudaEventRecord(after_hub, g->stream));
    return MC_OK;
  }
  CountArgs a{};
  a.rowptr = g->rowptr;
  a.col = g->col;
  a.key = g->key;
  a.pinfo = g->pinfo;
  a.dag_rowptr = g->dag_rowptr;
  a.dag_col = g->dag_col;
  a.result = g->counters + 0;
  a.err = g->err;
  a.table_log2_max = g->hub_table_log2;
  a.shard = shard;
  a.num_shards = num_shards;
  a.bv = g->batch;

  // Owners with d+ <= kHubSmallMaxOut: tables of at most 2^12 slots (16 KB),
  // so many CTAs share an SM; the few larger owners run in a second launch
  // whose shared memory fits the largest table.
  // Both launches get at least kHubBitmapBytes: at 5 CTAs per SM (the
  // register bound) that costs no occupancy and lets owners of rank up to
  // 8 x kHubBitmapBytes use bitmaps.
  const int small_lg = std::min(kHubSmallTableLog2, g->hub_table_log2);
  const int big_lg = std::max(kHubSmallTableLog2, g->hub_table_log2);
  const size_t small_smem = std::max<size_t>(sizeof(int) << small_lg, kHubBitmapBytes);
  const size_t big_smem = std::max<size_t>(sizeof(int) << big_lg, kHubBitmapBytes);
  const bool ranked = g->rank != nullptr && g->batch.gid == nullptr;
  a.rank = ranked ? g->rank : nullptr;
  a.dag_rank = ranked ? g->dag_rank : nullptr;
  a.core = ranked && g->core_used > 0 ? g->core_bits : nullptr;
  a.core_ranks = a.core ? g->core_used : 0;
  a.dense_factor = g->dense_factor;
  // MERCURY_TC_TMA=1: long partner lists staged by bulk copies (the table's
  // shared memory is followed by 16 KB of copy slots).
  const char *tma_env = std::getenv("MERCURY_TC_TMA");
  // (Lists in host memory, MC_HOST_DAG, always take the lane loads.)
  const bool staged = tma_env && std::atoi(tma_env) != 0 && !g->dag_host;
  // MERCURY_TC_ROW_STAGE=1: the row prefetch, which bulk-copies chunks of
  // the column array (device columns on a 16-byte boundary only).  Off by
  // default: at RMAT scale 22 it took the hub kernel from 9.26 to 10.38 ms,
  // as thread 0's header loads for the next task held warp 0 and the CTA's
  // end-of-task barrier waited for it.
  const char *row_env = std::getenv("MERCURY_TC_ROW_STAGE");
  const bool row_stage = !staged && !g->col_host &&
                         (reinterpret_cast<uintptr_t>(g->col) & 15u) == 0 && row_env &&
                         std::atoi(row_env) != 0;
  // MERCURY_TC_SHORT_RANGES=0: the short stream in interleaved windows.
  const char *ranges_env = std::getenv("MERCURY_TC_SHORT_RANGES");
  a.short_ranges = !(ranges_env && std::atoi(ranges_env) == 0);
  // MERCURY_TC_LONG_CLASSES=0: long partner lists paired in row order.
  const char *classes_env = std::getenv("MERCURY_TC_LONG_CLASSES");
  a.long_classes = !(classes_env && std::atoi(classes_env) == 0);
  a.nnz = g->nnz;
  auto kern = staged ? tc_hub_kernel<true, false>
                     : (row_stage ? tc_hub_kernel<false, true> : tc_hub_kernel<false, false>);
  const size_t extra = staged ? kStageBytes : 0;
  MC_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(big_smem + extra)));
  a.table_log2_max = small_lg;
  a.tasks = g->hub_tasks;
  a.ntasks = g->hub_off + g->n;
  a.queue = g->counters + 1;
  // (One quad of each bitmap's shared memory is the probe's zero word.)
  a.bitmap_bits = (int)std::min<size_t>(small_smem * 8 - 128, (size_t)g->bitmap_bits_cap);
  a.stage_off = (int)(small_smem / sizeof(int));
  const int small_grid =
      g->num_sms * resident_blocks((const void *)kern, kCountThreads, small_smem + extra);
  kern<<<small_grid, kCountThreads, small_smem + extra, g->stream>>>(a);
  MC_CUDA_TRY(cudaGetLastError());
  a.table_log2_max = big_lg;
  a.tasks = g->mega_tasks;
  a.ntasks = g->mega_off + g->n;
  a.queue = g->counters + 6;
  a.bitmap_bits = (int)std::min<size_t>(big_smem * 8 - 128, (size_t)g->bitmap_bits_cap);
  a.stage_off = (int)(big_smem / sizeof(int));
  const int big_grid =
      g->num_sms * resident_blocks((const void *)kern, kCountThreads, big_smem + extra);
  kern<<<big_grid, kCountThreads, big_smem + extra, g->stream>>>(a);
  MC_CUDA_TRY(cudaGetLastError());
  g->launches += 3;
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

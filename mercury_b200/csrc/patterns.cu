// P1..P8 pattern counts on the device.
//
// Reference: subgraph_matching/pattern_kernels.cuh (kernels P1_frequency_count,
// P1_count_correction, P2..P8_subgraph_matching) and the host combine of
// subgraph_matching/sm_multigpu.cu:206-232.  Every count is a sum over the
// 2m directed edges (v0, v1) of the symmetric CSR (graph.cc:336-365), plus
// P1's sum over vertices, of two 64-bit counters; the result is counters[1]
// for P4/P6 and counters[1] - counters[2] otherwise.  Two routes compute the
// same per-edge terms (each pattern takes the faster; see
// pattern_uses_centers):
//  * warp per directed edge: the frontier lists of the pattern materialised
//    in a per-warp slice of global scratch, membership by binary search or,
//    for the dominant terms of P4, P5, P6 and P8, by a per-warp hash set in
//    shared memory (counts restated as |N(x) & S| through the symmetry of
//    the graph; same integers, same 32-bit products), and for P7 and P8's
//    correction by 32-bit adjacency rows within A when |A| <= 32;
//  * center bitmaps: a group of warps per center v0 holds the adjacency among
//    N(v0) as bit rows in shared memory and reads each term off popcounts
//    (centers of degree above kCenterMaxDeg stay on the first route).
//
// The warp set operations return the same sets as the reference's
// difference_set / intersect / difference_num / intersect_num
// (gpu_kernels/set_difference.cuh, gpu_kernels/set_intersect.cuh): outputs
// are compacted with ballot + popc in input order so they stay sorted, and
// the bounded forms stop at the first key >= bound.  Membership tests keep
// the reference's direction (x searched in N(k)).  Where the reference
// multiplies two 32-bit ints before adding to its 64-bit counter (P1, P2,
// P3, P5, P7, P8), the product is formed the same way (wrapped to 32 bits,
// sign-extended).
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include <cuda.h>

#include "dgraph.cuh"
#include "device_common.cuh"
#include "scan.cuh"

namespace mc {
namespace {

constexpr int kPatThreads = 256;
constexpr int kLists = 6;  // frontier lists per warp, each max_degree long
// Frontier scratch is capped; graphs with huge degrees run fewer warps.
constexpr size_t kScratchBudget = size_t(2) << 30;

struct PatArgs {
  const int64_t *__restrict__ rp;
  const int32_t *__restrict__ ci;
  int64_t n, nnz;
  int32_t *scratch;      // kLists * cap ints per resident warp
  int64_t cap;           // list capacity (max degree)
  unsigned long long *counters;  // [0] = c1, [1] = c2
  unsigned long long *queue;
  // Optional restriction to the large centers (those the center-bitmap
  // kernels leave out): edge task t of center v is t in
  // [task_off[v], task_off[v+1]); star tasks skip vertices of degree <= skip_deg.
  const int64_t *task_off = nullptr;
  int skip_deg = -1;
  // Shard `shard` of `num_shards` takes queue positions t -> task
  // t * num_shards + shard (partial counts of all shards sum to the count).
  int shard = 0, num_shards = 1;
  // 0: the binary-search forms only (MERCURY_PATTERN_SETS=0; tests compare
  // both forms with it).
  int use_sets = 1;
  // Slice [task_begin, task_end) of this shard's queue positions (task_end
  // < 0: to the end); the queue counter starts at 0 for every slice.
  int64_t task_begin = 0, task_end = -1;
  // Budgeted count: stop at *deadline (globaltimer ns), raising *stop_flag.
  const unsigned long long *deadline = nullptr;
  unsigned long long *stop_flag = nullptr;
};

__device__ __forceinline__ unsigned long long wrap_mul(int a, int b) {
  return (unsigned long long)(long long)(int)((unsigned)a * (unsigned)b);
}

// Plain (coherent) loads: `list` may be a frontier list this warp wrote.
__device__ __forceinline__ bool bsearch(const int32_t *list, int len, int key) {
  int lo = 0, hi = len - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int m = list[mid];
    if (m == key) return true;
    if (m < key) lo = mid + 1;
    else hi = mid - 1;
  }
  return false;
}

// Per-warp hash set in shared memory: one table of kSetSlots ints (open
// addressing, linear probing) holding at most kSetMax distinct keys (load
// <= 1/2), each tagged 0 or 1: a key k is stored as k (tag 0) or -(k + 2)
// (tag 1), and -1 marks an empty slot, so two disjoint sets share the
// table.  Sets larger than that take the binary-search forms below.
constexpr int kSetSlots = 1024;
constexpr int kSetMax = kSetSlots / 2;
constexpr int kSetShift = 32 - 10;
static_assert((1 << (32 - kSetShift)) == kSetSlots, "set hash width");

struct WarpSet {
  int *tab;
  __device__ __forceinline__ static unsigned slot(int key) {
    return ((unsigned)key * 2654435769u) >> kSetShift;
  }
  __device__ void clear(int lane) const {
    int4 *t4 = reinterpret_cast<int4 *>(tab);
    for (int i = lane; i < kSetSlots / 4; i += kWarp) t4[i] = make_int4(-1, -1, -1, -1);
    __syncwarp();
  }
  // Inserts list[0, n) with the given tag (keys distinct from every key
  // already present; at most kSetMax keys in all).
  __device__ void insert(const int32_t *list, int n, int tag, int lane) const {
    for (int i = lane; i < n; i += kWarp) {
      const int key = list[i];
      const int code = tag ? -(key + 2) : key;
      unsigned sl = slot(key);
      for (int probe = 0; probe < kSetSlots; ++probe) {
        if (atomicCAS(tab + sl, -1, code) == -1) break;
        sl = (sl + 1) & (kSetSlots - 1);
      }
    }
    __syncwarp();
  }
  // 0: absent, 1: present with tag 0, 2: present with tag 1.
  __device__ __forceinline__ int lookup(int key) const {
    const int alt = -(key + 2);
    unsigned sl = slot(key);
    for (int probe = 0; probe < kSetSlots; ++probe) {
      const int v = tab[sl];
      if (v == key) return 1;
      if (v == alt) return 2;
      if (v == -1) return 0;
      sl = (sl + 1) & (kSetSlots - 1);
    }
    return 0;
  }
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

struct Warp {
  const int64_t *__restrict__ rp;
  const int32_t *__restrict__ ci;
  int lane;
  int *H = nullptr;  // this warp's kSetSlots-int set table (null: none)
  unsigned *M = nullptr;  // this warp's 32 words of row masks
  // A budgeted count: past *deadline (globaltimer ns) the warp stops and
  // raises *stop_flag (the count is then incomplete and refused).
  const unsigned long long *deadline = nullptr;
  unsigned long long *stop_flag = nullptr;
  // Warp-uniform: lane 0's clock decides (call from every lane).
  __device__ __forceinline__ bool out_of_time() const {
    if (!deadline) return false;
    unsigned long long t = lane == 0 ? global_ns() : 0ull;
    t = __shfl_sync(kFull, t, 0);
    const bool late = t > *deadline;
    if (late && lane == 0) atomicOr(stop_flag, 1ull);
    return late;
  }
  // One lane's own check, for loops whose trip counts differ across lanes.
  __device__ __forceinline__ bool lane_out_of_time() const {
    return deadline && global_ns() > *deadline;
  }
  __device__ __forceinline__ int deg(int v) const { return (int)(__ldg(rp + v + 1) - __ldg(rp + v)); }
  __device__ __forceinline__ const int32_t *N(int v) const { return ci + __ldg(rp + v); }
  // x in N(k), searched in k's list.
  __device__ __forceinline__ bool in(int k, int x) const { return bsearch(N(k), deg(k), x); }

  // out = {x in a[0, na) : x < bound, (x in list) == want}, in a's order;
  // bound < 0: no bound.  Returns the size (the same on every lane).
  __device__ int filter(const int32_t *a, int na, const int32_t *list, int nl, int bound,
                        bool want, int32_t *out) const {
    int cnt = 0;
    for (int base = 0; base < na; base += kWarp) {
      const int i = base + lane;
      const bool inr = i < na;
      const int x = inr ? a[i] : 0;
      const bool below = inr && (bound < 0 || x < bound);
      const bool keep = below && (bsearch(list, nl, x) == want);
      const unsigned m = __ballot_sync(kFull, keep);
      if (keep) out[cnt + __popc(m & ((1u << lane) - 1u))] = x;
      cnt += __popc(m);
      if (__any_sync(kFull, inr && !below)) break;
    }
    __syncwarp();
    return cnt;
  }
  // difference_set(a, N(k)[, bound])
  __device__ __forceinline__ int diff(const int32_t *a, int na, int k, int bound,
                                      int32_t *out) const {
    return filter(a, na, N(k), deg(k), bound, false, out);
  }
  // intersect(a, N(k)[, bound]): the shorter list drives the loop.
  __device__ __forceinline__ int inter(const int32_t *a, int na, int k, int bound,
                                       int32_t *out) const {
    const int nk = deg(k);
    return nk < na ? filter(N(k), nk, a, na, bound, true, out)
                   : filter(a, na, N(k), nk, bound, true, out);
  }
  // #{x in a : x < bound, (x in N(k)) == want}, summed over the warp.
  __device__ int count(const int32_t *a, int na, int k, int bound, bool want) const {
    const int32_t *list = N(k);
    const int nl = deg(k);
    int c = 0;
    for (int base = 0; base < na; base += kWarp) {
      const int i = base + lane;
      const bool inr = i < na;
      const int x = inr ? a[i] : 0;
      const bool below = inr && (bound < 0 || x < bound);
      if (below && bsearch(list, nl, x) == want) ++c;
      if (__any_sync(kFull, inr && !below)) break;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
    return c;
  }
};

struct Acc {
  unsigned long long c1 = 0, c2 = 0;
};

// Index of y in the ascending list[0, n) (y present).
__device__ __forceinline__ int pos_of(const int32_t *list, int n, int y) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (list[mid] < y) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int ceil_log2_int(int v) { return v <= 1 ? 1 : 32 - __clz(v - 1); }

// |N(x) & S| by the whole warp (every lane gets the total), S the set's
// tag-0 keys and also given as its list of nS entries: lanes stream
// N(x) probing the set (ceil(d / 32) steps), or search S's entries in N(x)
// (ceil(nS / 32) binary searches), whichever takes fewer warp steps.
__device__ __forceinline__ int warp_common(const Warp &w, int x, const WarpSet &S,
                                           const int32_t *list, int nS) {
  const int32_t *p = w.N(x);
  const int d = w.deg(x);
  int c = 0;
  if ((d + kWarp - 1) / kWarp <= ((nS + kWarp - 1) / kWarp) * ceil_log2_int(d)) {
    for (int k = w.lane; k < d; k += kWarp) c += S.lookup(__ldg(p + k)) == 1;
  } else {
    for (int k = w.lane; k < nS; k += kWarp) c += bsearch(p, d, list[k]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
  return c;
}


// freq[j] = #{i > j : a[j] not in N(a[i])}   (P3 :280-292, P7 :386-398)
__device__ void pair_freq(const Warp &w, const int32_t *a, int na, int32_t *freq) {
  for (int j = w.lane; j < na; j += kWarp) {
    const int x = a[j];
    int f = 0;
    for (int i = j + 1; i < na; ++i) {
      if ((i & 1023) == 0 && w.lane_out_of_time()) break;
      f += !w.in(a[i], x);
    }
    freq[j] = f;
  }
  __syncwarp();
}

// freq[j] = #{v in list : a[j] not in N(v)}   (P2 :175-187, P5 :628-640, P8 :501-514)
__device__ void cross_freq(const Warp &w, const int32_t *a, int na, const int32_t *list, int nl,
                           int32_t *freq) {
  for (int j = w.lane; j < na; j += kWarp) {
    const int x = a[j];
    int f = 0;
    for (int i = 0; i < nl; ++i) {
      if ((i & 1023) == 1023 && w.lane_out_of_time()) break;
      f += !w.in(list[i], x);
    }
    freq[j] = f;
  }
  __syncwarp();
}

// Correction of P3/P7 (:310-340, :417-449): for v2 in A,
// #{(c in A & N(v2), key in A - N(v2), key < v2) : key > c, c not in N(key)}.
__device__ void bounded_correction(const Warp &w, const int32_t *A, int nA, int32_t *D,
                                   int32_t *C, Acc &acc) {
  for (int i = 0; i < nA; ++i) {
    if ((i & 15) == 15 && w.out_of_time()) return;
    const int v2 = A[i];
    const int nD = w.diff(A, nA, v2, v2, D);
    const int nC = w.inter(A, nA, v2, -1, C);
    for (int ii = 0; ii < nC; ++ii) {
      const int c = C[ii];
      for (int j = w.lane; j < nD; j += kWarp) {
        const int key = D[j];
        if (key > c && !w.in(key, c)) ++acc.c2;
      }
    }
  }
}

template <int P>
__device__ void edge_pattern(const Warp &w, int v0, int v1, int32_t *L, int64_t cap, Acc &acc) {
  int32_t *L0 = L, *L1 = L + cap, *L2 = L + 2 * cap, *L3 = L + 3 * cap, *L4 = L + 4 * cap,
          *L5 = L + 5 * cap;
  const int32_t *n0 = w.N(v0), *n1 = w.N(v1);
  const int d0 = w.deg(v0), d1 = w.deg(v1);
  if (P == 1) {  // P1_count_correction (:6-66)
    if (v0 == v1) return;
    const int nA = w.diff(n0, d0, v1, v1, L0);   // dif, bounded by v1
    const int nB = w.inter(n0, d0, v1, v1, L1);  // int, bounded by v1
    for (int i = 0; i < nB; ++i) {
      if ((i & 15) == 15 && w.out_of_time()) return;
      const int v2 = L1[i];
      for (int j = w.lane; j < nA; j += kWarp) {
        const int key = L0[j];
        if (key > v2 && !w.in(key, v2)) ++acc.c2;
      }
    }
  } else if (P == 2) {  // P2_subgraph_matching (:135-243)
    const int nA = w.diff(n0, d0, v1, -1, L0);
    const int nB = w.diff(n1, d1, v0, -1, L1);
    cross_freq(w, L0, nA, L1, nB, L4);
    for (int i = 0; i < nA; ++i) {
      if ((i & 15) == 15 && w.out_of_time()) return;
      const int c = w.count(L0, nA, L0[i], L0[i], false);
      if (w.lane == 0) acc.c1 += wrap_mul(c, L4[i]);
    }
    for (int i = 0; i < nB; ++i) {
      if ((i & 15) == 15 && w.out_of_time()) return;
      const int v4 = L1[i];
      const int nD = w.diff(L0, nA, v4, -1, L2);
      const int nC = w.inter(L0, nA, v4, -1, L3);
      for (int ii = 0; ii < nC; ++ii) {
        const int v2 = L3[ii];
        for (int j = w.lane; j < nD; j += kWarp) {
          const int key = L2[j];
          if (key > v2 && !w.in(key, v2)) ++acc.c2;
        }
      }
    }
  } else if (P == 3) {  // P3_subgraph_matching (:245-350)
    const int nA = w.diff(n0, d0, v1, -1, L0);
    pair_freq(w, L0, nA, L4);
    for (int i = 0; i < nA; ++i) {
      if ((i & 15) == 15 && w.out_of_time()) return;
      const int c = w.count(L0, nA, L0[i], L0[i], false);
      if (w.lane == 0) acc.c1 += wrap_mul(c, L4[i]);
    }
    bounded_correction(w, L0, nA, L1, L2, acc);
  } else if (P == 4) {  // P4_subgraph_matching (:855-963), only v1 < v0
    if (v1 >= v0) return;
    const int nA = w.diff(n0, d0, v1, -1, L0);
    const int nB = w.diff(n1, d1, v0, -1, L1);
    const int32_t *outer = nA < nB ? L0 : L1, *inner = nA < nB ? L1 : L0;
    const int no = nA < nB ? nA : nB, ni = nA < nB ? nB : nA;
    if (w.H && ni <= kSetMax) {
      // Per v2 in outer, the whole warp: ni - |N(v2) & inner|, streaming
      // N(v2) against `inner` in the shared-memory set, or searching inner's
      // entries in N(v2) when that takes fewer warp steps.
      const WarpSet s0{w.H};
      s0.clear(w.lane);
      s0.insert(inner, ni, 0, w.lane);
      for (int i = 0; i < no; ++i) {
        if ((i & 15) == 15 && w.out_of_time()) return;
        const int common = warp_common(w, outer[i], s0, inner, ni);
        if (w.lane == 0) acc.c1 += (unsigned long long)(ni - common);
      }
      __syncwarp();
      return;
    }
    for (int i = 0; i < no; ++i) {
      if ((i & 15) == 15 && w.out_of_time()) return;
      const int v2 = outer[i];
      const int dv2 = w.deg(v2);
      if (dv2 < ni) {
        // #{y in inner : y not in N(v2)} = ni - |N(v2) & inner|, searching the
        // shorter N(v2) in `inner` (the reference's size switch, :898-958).
        const int32_t *nv2 = w.N(v2);
        unsigned long long common = 0;
        for (int j = w.lane; j < dv2; j += kWarp) common += bsearch(inner, ni, __ldg(nv2 + j));
        acc.c1 += (w.lane == 0 ? (unsigned long long)ni : 0ull) - common;
      } else {
        for (int j = w.lane; j < ni; j += kWarp) acc.c1 += !w.in(v2, inner[j]);
      }
    }
  } else if (P == 5) {  // P5_subgraph_matching (:574-734)
    const int nA = w.inter(n0, d0, v1, -1, L0);
    const int nB = w.diff(n0, d0, v1, -1, L1);
    const int nC = w.diff(n1, d1, v0, -1, L2);
    if (w.H && nA + nC <= kSetMax && nB <= kSetMax) {
      // The same per-edge terms through the hash set.  For b in B the
      // reference's f = #{a in A : b not in N(a)} = nA - |N(b) & A| and
      // t = #{c in C : c not in N(b)} = nC - |N(b) & C| (the graph is
      // symmetric): one lane per b walks N(b) once for both, A and C
      // sharing the table with tags 0 and 1 (they are disjoint), or
      // searches A and C in N(b) when that is shorter.
      const WarpSet s0{w.H};
      if (nA > 0) {  // with A empty every f is 0
        s0.clear(w.lane);
        s0.insert(L0, nA, 0, w.lane);
        s0.insert(L2, nC, 1, w.lane);
        // Groups of kGroup lanes per b (kWarp / kGroup b's at a time): short
        // and hub neighbourhoods alike keep the group's lanes busy.
        constexpr int kGroup = 8;
        const int grp = w.lane / kGroup, sub = w.lane % kGroup;
        const int nb_round = (nB + kWarp / kGroup - 1) / (kWarp / kGroup) * (kWarp / kGroup);
        for (int j0 = 0; j0 < nb_round; j0 += kWarp / kGroup) {
          if ((j0 & 255) == 252 && w.out_of_time()) return;
          const int j = j0 + grp;
          int ca = 0, cc = 0;
          if (j < nB) {
            const int b = L1[j];
            const int32_t *p = w.N(b);
            const int db = w.deg(b);
            if ((db + kGroup - 1) / kGroup <=
                ((nA + nC + kGroup - 1) / kGroup) * ceil_log2_int(db)) {
              for (int k = sub; k < db; k += kGroup) {
                const int r = s0.lookup(__ldg(p + k));
                ca += r == 1;
                cc += r == 2;
              }
            } else {
              for (int k = sub; k < nA; k += kGroup) ca += bsearch(p, db, L0[k]);
              for (int k = sub; k < nC; k += kGroup) cc += bsearch(p, db, L2[k]);
            }
          }
#pragma unroll
          for (int o = kGroup / 2; o > 0; o >>= 1) {
            ca += __shfl_xor_sync(kFull, ca, o);
            cc += __shfl_xor_sync(kFull, cc, o);
          }
          const int f = nA - ca;
          if (j < nB && sub == 0 && f) acc.c1 += wrap_mul(nC - cc, f);
        }
        __syncwarp();
      }
      // Correction: for v2 in A, D = C & N(v2), E = B - N(v2), and
      // #{e in E : e not in N(c)} = nE - |N(c) & E| for c in D (the whole
      // warp per c: D is short).
      for (int i = 0; i < nA; ++i) {
        if ((i & 15) == 15 && w.out_of_time()) return;
        const int v2 = L0[i];
        const int nD = w.inter(L2, nC, v2, -1, L3);
        if (nD == 0) continue;
        const int nE = w.diff(L1, nB, v2, -1, L4);
        s0.clear(w.lane);
        s0.insert(L4, nE, 0, w.lane);
        for (int j = 0; j < nD; ++j) {
          const int common = warp_common(w, L3[j], s0, L4, nE);
          if (w.lane == 0) acc.c2 += (unsigned long long)(nE - common);
        }
        __syncwarp();
      }
      __syncwarp();
      return;
    }
    // freq over B of the A vertices not adjacent to it
    for (int j = w.lane; j < nB; j += kWarp) {
      const int x = L1[j];
      int f = 0;
      for (int i = 0; i < nA; ++i) f += !w.in(L0[i], x);
      L5[j] = f;
    }
    __syncwarp();
    for (int i = 0; i < nB; ++i) {
      if ((i & 15) == 15 && w.out_of_time()) return;
      const int f = L5[i];
      if (f == 0) continue;
      const int b = L1[i];
      int t = 0;
      for (int j = w.lane; j < nC; j += kWarp) t += !w.in(b, L2[j]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(kFull, t, o);
      if (w.lane == 0) acc.c1 += wrap_mul(t, f);
    }
    for (int i = 0; i < nA; ++i) {
      if ((i & 15) == 15 && w.out_of_time()) return;
      const int v2 = L0[i];
      const int nD = w.inter(L2, nC, v2, -1, L3);  // C & N(v2)
      const int nE = w.diff(L1, nB, v2, -1, L4);   // B - N(v2)
      for (int ii = 0; ii < nD; ++ii) {
        const int c = L3[ii];
        for (int j = w.lane; j < nE; j += kWarp) acc.c2 += !w.in(c, L4[j]);
      }
    }
  } else if (P == 6) {  // P6_subgraph_matching (:736-853)
    const int nA = w.inter(n0, d0, v1, -1, L0);
    const int nB = w.diff(n1, d1, v0, -1, L1);
    if (nA == 0) {
      __syncwarp();
      return;
    }
    if (w.H && w.M && nA <= kWarp && nA + nB <= kSetMax) {
      // Bit-mask form.  Lane j walks N(A[j]) once against B (tag 0) and A
      // (tag 1) in the shared-memory set, recording the B positions it holds
      // (row j of mask, ceil(nB / 32) words in the warp's scratch) and the A
      // positions (M[j]).  For v2 = A[j] the reference's D = A - N(v2) is
      // ~M[j] and E = B - N(v2) is ~mask[j]; its count for v3 in D,
      // #{key in E : key not in N(v3)}, is popc(~mask[j] & ~mask[v3]) over
      // B's positions (the graph is symmetric).
      const int wb = (nB + kWarp - 1) / kWarp;
      unsigned *mask = reinterpret_cast<unsigned *>(L2);
      const WarpSet s0{w.H};
      s0.clear(w.lane);
      s0.insert(L1, nB, 0, w.lane);
      s0.insert(L0, nA, 1, w.lane);
      unsigned mrow = 0;
      if (w.lane < nA) {
        const int j = w.lane;
        unsigned *mj = mask + j * wb;
        for (int k = 0; k < wb; ++k) mj[k] = 0u;
        const int x = L0[j];
        const int32_t *p = w.N(x);
        const int dx = w.deg(x);
        if (dx <= (nB + nA) * ceil_log2_int(dx)) {
          for (int k = 0; k < dx; ++k) {
            const int y = __ldg(p + k);
            const int r = s0.lookup(y);
            if (r == 1) {
              const int q = pos_of(L1, nB, y);
              mj[q >> 5] |= 1u << (q & 31);
            } else if (r == 2) {
              mrow |= 1u << pos_of(L0, nA, y);
            }
          }
        } else {
          for (int k = 0; k < nB; ++k)
            if (bsearch(p, dx, L1[k])) mj[k >> 5] |= 1u << (k & 31);
          for (int k = 0; k < nA; ++k)
            if (k != j && bsearch(p, dx, L0[k])) mrow |= 1u << k;
        }
      }
      w.M[w.lane] = mrow;
      __syncwarp();
      if (w.lane < nA) {
        const int j = w.lane;
        const unsigned *mj = mask + j * wb;
        const unsigned valid_a = nA == kWarp ? kFull : ((1u << nA) - 1u);
        unsigned dset = ~mrow & valid_a;  // D = A - N(v2), v2 itself included
        unsigned long long c = 0;
        while (dset) {
          const int t = __ffs(dset) - 1;
          dset &= dset - 1u;
          const unsigned *mt = mask + t * wb;
          for (int k = 0; k < wb; ++k) {
            const int left = nB - 32 * k;
            const unsigned valid = left >= 32 ? kFull : ((1u << left) - 1u);
            c += (unsigned long long)__popc(valid & ~(mj[k] | mt[k]));
          }
        }
        acc.c1 += c;
      }
      __syncwarp();
      return;
    }
    for (int i = 0; i < nA; ++i) {
      if ((i & 15) == 15 && w.out_of_time()) return;
      const int v2 = L0[i];
      const int nD = w.diff(L0, nA, v2, -1, L2);
      const int nE = w.diff(L1, nB, v2, -1, L3);
      const int32_t *outer = nD < nE ? L2 : L3, *inner = nD < nE ? L3 : L2;
      const int no = nD < nE ? nD : nE, ni = nD < nE ? nE : nD;
      if (w.H && ni <= kSetMax && no > 0) {
        // #{x in inner : x not in N(v3)} = ni - |N(v3) & inner| by the
        // whole warp, `inner` in the shared-memory set.
        const WarpSet s0{w.H};
        s0.clear(w.lane);
        s0.insert(inner, ni, 0, w.lane);
        for (int ii = 0; ii < no; ++ii) {
          const int common = warp_common(w, outer[ii], s0, inner, ni);
          if (w.lane == 0) acc.c1 += (unsigned long long)(ni - common);
        }
        __syncwarp();
        continue;
      }
      for (int ii = 0; ii < no; ++ii) {
        const int v3 = outer[ii];
        for (int j = w.lane; j < ni; j += kWarp) acc.c1 += !w.in(v3, inner[j]);
      }
    }
  } else if (P == 7) {  // P7_subgraph_matching (:352-459)
    const int nA = w.inter(n0, d0, v1, -1, L0);
    if (w.M && nA <= kWarp) {
      // Every set of P7 lies inside A (ascending, at most 32 entries): lane
      // i holds M[i] = {k : A[k] in N(A[i])}, and by the graph's symmetry
      // freq[i] = #{k > i : A[i] not in N(A[k])} = popc(~M[i] above i),
      // c = #{x in A : x < A[i], x not in N(A[i])} = popc(~M[i] below i),
      // and the correction for v2 = A[i] (D = ~M[i] below i, C = M[i]) is
      // the sum over t in C of popc(D above t & ~M[t]).  With |A| <= 2 every
      // term is 0.
      if (nA < 3) {
        __syncwarp();
        return;
      }
      unsigned row = 0;
      if (w.lane < nA) {
        const int32_t *p = w.N(L0[w.lane]);
        const int dx = w.deg(L0[w.lane]);
        for (int k = 0; k < nA; ++k)
          if (k != w.lane && bsearch(p, dx, L0[k])) row |= 1u << k;
      }
      w.M[w.lane] = row;
      __syncwarp();
      if (w.lane < nA) {
        const int i = w.lane;
        const unsigned valid = nA == kWarp ? kFull : ((1u << nA) - 1u);
        const unsigned below = (1u << i) - 1u;
        const unsigned above = valid & ~below & ~(1u << i);
        const int freq = __popc(~row & above);
        const int c = __popc(~row & below);
        acc.c1 += wrap_mul(c, freq);
        const unsigned dmask = ~row & below;
        unsigned cm = row;
        int c2 = 0;
        while (cm) {
          const int t = __ffs(cm) - 1;
          cm &= cm - 1u;
          const unsigned above_t = t == kWarp - 1 ? 0u : ~((2u << t) - 1u);
          c2 += __popc(dmask & above_t & ~w.M[t]);
        }
        acc.c2 += (unsigned long long)c2;
      }
      __syncwarp();
      return;
    }
    pair_freq(w, L0, nA, L4);
    for (int i = 0; i < nA; ++i) {
      if ((i & 15) == 15 && w.out_of_time()) return;
      const int c = w.count(L0, nA, L0[i], L0[i], false);
      if (w.lane == 0) acc.c1 += wrap_mul(c, L4[i]);
    }
    bounded_correction(w, L0, nA, L1, L2, acc);
  } else if (P == 8) {  // P8_subgraph_matching (:461-572)
    const int nA = w.inter(n0, d0, v1, -1, L0);
    const int nB = w.diff(n1, d1, v0, -1, L1);
    if (w.H && w.M && nA + nB <= kSetMax && nA <= kWarp) {
      // For a = A[j] the reference's freq = #{v in B : a not in N(v)} =
      // nB - |N(a) & B| and c = #{x in A : x < a, x in N(a)} (symmetric
      // graph): lane j walks N(a) once against B (tag 0) and A (tag 1,
      // disjoint from B), or searches B and A in N(a) when that is shorter.
      // The same pass records which B entries N(a) holds (bit j of
      // mask_C[p] for B[p]) and M[j] = {k > j : A[k] in N(a)}; then the
      // correction, for v4 = B[p] with C = A & N(v4) (mask_C[p]) and D =
      // A - N(v4), is #{(v2, key) : v2 in C, key in D, key > v2, key in
      // N(v2)} = sum over i in C of popc(M[i] & ~mask_C[p]).
      const WarpSet s0{w.H};
      s0.clear(w.lane);
      s0.insert(L1, nB, 0, w.lane);
      s0.insert(L0, nA, 1, w.lane);
      unsigned *maskc = reinterpret_cast<unsigned *>(L2);
      for (int p = w.lane; p < nB; p += kWarp) maskc[p] = 0u;
      __syncwarp();
      unsigned mrow = 0;
      if (w.lane < nA) {
        const int j = w.lane;
        const int x = L0[j];
        const int32_t *p = w.N(x);
        const int dx = w.deg(x);
        int hb = 0, ca = 0;
        if (dx <= (nB + nA) * ceil_log2_int(dx)) {
          for (int k = 0; k < dx; ++k) {
            const int y = __ldg(p + k);
            const int r = s0.lookup(y);
            if (r == 1) {
              ++hb;
              atomicOr(maskc + pos_of(L1, nB, y), 1u << j);
            } else if (r == 2) {
              if (y < x) ++ca;
              else mrow |= 1u << pos_of(L0, nA, y);
            }
          }
        } else {
          for (int k = 0; k < nB; ++k)
            if (bsearch(p, dx, L1[k])) {
              ++hb;
              atomicOr(maskc + k, 1u << j);
            }
          for (int k = 0; k < nA; ++k)
            if (k != j && bsearch(p, dx, L0[k])) {
              if (k < j) ++ca;
              else mrow |= 1u << k;
            }
        }
        acc.c1 += wrap_mul(ca, nB - hb);
      }
      w.M[w.lane] = mrow;
      __syncwarp();
      for (int p = w.lane; p < nB; p += kWarp) {
        const unsigned mc = __ldcg(maskc + p);  // set by atomics: read at L2
        unsigned rest = mc;
        int t = 0;
        while (rest) {
          const int i = __ffs(rest) - 1;
          rest &= rest - 1u;
          t += __popc(w.M[i] & ~mc);
        }
        acc.c2 += (unsigned long long)t;
      }
      __syncwarp();
      return;
    }
    cross_freq(w, L0, nA, L1, nB, L4);
    for (int i = 0; i < nA; ++i) {
      if ((i & 15) == 15 && w.out_of_time()) return;
      const int c = w.count(L0, nA, L0[i], L0[i], true);
      if (w.lane == 0) acc.c1 += wrap_mul(c, L4[i]);
    }
    for (int i = 0; i < nB; ++i) {
      if ((i & 15) == 15 && w.out_of_time()) return;
      const int v4 = L1[i];
      const int nD = w.diff(L0, nA, v4, -1, L2);
      const int nC = w.inter(L0, nA, v4, -1, L3);
      for (int ii = 0; ii < nC; ++ii) {
        const int v2 = L3[ii];
        for (int j = w.lane; j < nD; j += kWarp) {
          const int key = L2[j];
          if (key > v2 && w.in(key, v2)) ++acc.c2;
        }
      }
    }
  }
  __syncwarp();
}

// P1_frequency_count (:68-133): per vertex v0, the star term.
__device__ void vertex_star(const Warp &w, int v0, int32_t *L, Acc &acc) {
  const int d = w.deg(v0);
  const int32_t *nb = w.N(v0);
  int32_t *freq = L;
  for (int i = w.lane; i < d; i += kWarp) {
    const int x = nb[i];
    int f = 0;
    for (int j = i + 1; j < d; ++j) {
      if ((j & 1023) == 0 && w.lane_out_of_time()) break;
      f += !w.in(nb[j], x);  // x < nb[j] iff j > i
    }
    freq[i] = f;
  }
  __syncwarp();
  for (int i = 0; i < d; ++i) {
    if ((i & 15) == 15 && w.out_of_time()) return;
    const int c = w.count(nb, d, nb[i], nb[i], false);
    if (w.lane == 0) acc.c1 += wrap_mul(c, freq[i]);
  }
  __syncwarp();
}

// Persistent warps take directed edges (or, for the P1 star pass, vertices)
// from the queue one at a time.
template <int P, bool kStar>
__global__ void __launch_bounds__(kPatThreads) pattern_kernel(PatArgs a) {
  __shared__ __align__(16) int s_sets[kPatThreads / kWarp][kSetSlots];
  __shared__ unsigned s_rows[kPatThreads / kWarp][kWarp];
  const int lane = threadIdx.x & (kWarp - 1);
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
  int32_t *L = a.scratch + gw * kLists * a.cap;
  const Warp w{a.rp, a.ci, lane, a.use_sets ? s_sets[threadIdx.x / kWarp] : nullptr,
               a.use_sets ? s_rows[threadIdx.x / kWarp] : nullptr, a.deadline, a.stop_flag};
  const int64_t all = kStar ? a.n : (a.task_off ? a.task_off[a.n] : a.nnz);
  const int64_t ntasks = all > a.shard ? (all - a.shard + a.num_shards - 1) / a.num_shards : 0;
  const int64_t t_end = a.task_end >= 0 && a.task_end < ntasks ? a.task_end : ntasks;
  const int64_t span = t_end - a.task_begin;
  Acc acc;
  for (;;) {
    if (w.out_of_time()) break;
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(a.queue, 1ull);
    t = __shfl_sync(kFull, t, 0);
    if ((int64_t)t >= span) break;
    t += (unsigned long long)a.task_begin;
    t = t * (unsigned long long)a.num_shards + (unsigned long long)a.shard;
    if (kStar) {
      if (w.deg((int)t) > a.skip_deg) vertex_star(w, (int)t, L, acc);
    } else if (a.task_off) {
      const int v0 = (int)upper_row(a.task_off, 0, a.n - 1, (int64_t)t);
      const int64_t e = __ldg(a.rp + v0) + ((int64_t)t - a.task_off[v0]);
      edge_pattern<P>(w, v0, __ldg(a.ci + e), L, a.cap, acc);
    } else {
      const int v0 = (int)upper_row(a.rp, 0, a.n - 1, (int64_t)t);
      const int v1 = __ldg(a.ci + t);
      edge_pattern<P>(w, v0, v1, L, a.cap, acc);
    }
  }
  unsigned long long c1 = warp_sum_u64(acc.c1), c2 = warp_sum_u64(acc.c2);
  if (lane == 0) {
    if (c1) atomicAdd(a.counters + 0, c1);
    if (c2) atomicAdd(a.counters + 1, c2);
  }
}


// ---- center bitmaps (P1, P3, P7) -------------------------------------------
// Every edge (v0, v1) is taken with v0 as its center.  For these three
// patterns every set of the reference's formula lies inside N0 = N(v0), so a
// group of warps first builds M, the adjacency among N0: d0 rows of W words,
// bit j of row i set iff N0[j] ~ N0[i].  v1 = N0[p] and, with A a mask over
// N0 and below(q) / above(q) the positions before / after q:
//   P3  A = N0 - N1 = ~M[p];   P7  A = N0 & N1 = M[p]
//       count(q) = |A & ~M[q] & below(q)|, freq(q) = |A & ~M[q] & above(q)|
//       c1 += count(q) * freq(q) (32-bit product) for q in A;
//       c2 += sum over r in A & M[q] of |D & above(r) & ~M[r]|,
//             D = A & ~M[q] & below(q)      (pattern_kernels.cuh:280-340, :386-449)
//   P1  star: c1 += |~M[i] & below(i)| * |~M[i] & above(i)| over i
//       correction: A = ~M[p] & below(p), B = M[p] & below(p),
//       c2 += sum over r in B of |A & above(r) & ~M[r]|   (:6-133)
// These are the reference's per-edge counts exactly (the same sets, sizes
// and products), read off popcounts instead of binary searches.
constexpr int kCenterMaxDeg = 1024;  // larger centers use pattern_kernel
constexpr int kCenterClasses = 6;    // W = 1, 2, 4, 8, 16, 32 words per row

__host__ __device__ constexpr int center_words(int cls) { return 1 << cls; }
// Warps per center: one for small rows, the whole CTA from W = 16 on.
__host__ __device__ constexpr int center_group(int W) { return W >= 16 ? kPatThreads / kWarp : 1; }
// Patterns whose formulas also look outside N0: for every y in N1 - N0 - {v0}
// they need R(y) = N(y) & N0 as a mask over N0.
__host__ __device__ constexpr bool center_outer(int P) {
  return P == 2 || P == 4 || P == 5 || P == 6 || P == 8;
}
// Shared memory of one group: M (32W rows of W words), N0 (32W ints) and,
// for the outer patterns, per warp one R row per lane (32 x W words) and a
// counter per N0 position (32W ints).
// (Per warp, the outer patterns keep 32 R rows, 32W counters and 32 vertex
// slots.)  Outer patterns with rows of 4+ words also keep a position hash of N0
// (64W slots: keys, then positions), so that R(y) looks each neighbour of y
// up in about one read instead of a binary search.
__host__ __device__ constexpr bool center_hash(int P, int W) { return center_outer(P) && W >= 4; }
__host__ __device__ constexpr size_t center_group_bytes(int P, int W) {
  return sizeof(unsigned) * ((size_t)(32 * W) * W + (size_t)(32 * W) +
                             (center_outer(P) ? (size_t)center_group(W) * (64 * W + 32) : 0) +
                             (center_hash(P, W) ? (size_t)(128 * W) : 0));
}

struct CenterArgs {
  const int64_t *__restrict__ rp;
  const int32_t *__restrict__ ci;
  const int32_t *__restrict__ centers;  // this class's centers
  const int32_t *__restrict__ count;    // how many
  unsigned long long *queue;
  unsigned long long *counters;         // [0] = c1, [1] = c2
  // Slice [c_begin, c_end) of the class's centers (c_end < 0: to the end);
  // the queue counter starts at 0 for every slice.
  int64_t c_begin = 0, c_end = -1;
  // Outer patterns: hop_words words of global scratch per group (block b's
  // group g at (b * groups + g) * hop_words) for the center's two-hop rows;
  // null: rows are built per edge.
  unsigned *hop = nullptr;
  int64_t hop_words = 0;
  int64_t hop_walk = 0;  // host side: the class's largest two-hop walk (0: no rows)
  unsigned long long *hop_misses = nullptr;  // centers whose rows did not fit
  // Budgeted count: stop at *deadline (globaltimer ns), raising *stop_flag.
  const unsigned long long *deadline = nullptr;
  unsigned long long *stop_flag = nullptr;
};

// Warp-uniform deadline check (lane 0's clock decides; call from every lane).
__device__ __forceinline__ bool warp_late(const unsigned long long *deadline,
                                          unsigned long long *flag, int lane) {
  if (!deadline) return false;
  unsigned long long t = lane == 0 ? global_ns() : 0ull;
  t = __shfl_sync(kFull, t, 0);
  const bool late = t > *deadline;
  if (late && lane == 0) atomicOr(flag, 1ull);
  return late;
}

// Two-hop rows of a center v0: for every vertex y outside N0 + {v0} with a
// neighbour in N0, R(y) = N(y) & N0 as W words over N0's positions, built
// once per center by walking the lists of N0's members (sum over x in N0 of
// d(x) entries) instead of once per edge (v0, v1) for each y in N(v1) (sum
// over y in N(v1) of d(y) entries per edge).  keys/vals: an open-addressing
// map y -> row (2^lg slots, load <= 1/2).
struct HopRows {
  const int *keys;
  const int *vals;
  const unsigned *rows;
  int lg;
  int words;
  __device__ __forceinline__ const unsigned *row_of(int y) const {
    const unsigned mask = (1u << lg) - 1u;
    unsigned h = ((unsigned)y * 2654435769u) >> (32 - lg);
    for (int step = 0; step <= (int)mask; ++step) {
      const int k = keys[h];
      if (k == y) return rows + (int64_t)vals[h] * words;
      if (k < 0) break;
      h = (h + 1u) & mask;
    }
    return nullptr;  // not reached for a y with a neighbour in N0
  }
};

// Word k of the mask of positions below q (q in [0, 32W)).
__device__ __forceinline__ unsigned below_word(int k, int q) {
  const int qw = q >> 5;
  return k < qw ? ~0u : (k == qw ? ((1u << (q & 31)) - 1u) : 0u);
}
// Word k of the mask of positions above q.
__device__ __forceinline__ unsigned above_word(int k, int q) {
  const int qw = q >> 5;
  return k > qw ? ~0u : (k == qw ? ~((2u << (q & 31)) - 1u) : 0u);
}
__device__ __forceinline__ unsigned full_word(int k, int d) {
  const int b = d - 32 * k;
  return b >= 32 ? ~0u : (b <= 0 ? 0u : ((1u << b) - 1u));
}

// Position of y in the sorted n0[0, d0), or -1.
__device__ __forceinline__ int find_pos(const int32_t *n0, int d0, int y) {
  int lo = 0, hi = d0 - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int m = n0[mid];
    if (m == y) return mid;
    if (m < y) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

// Where y sits in N0 (-1: absent): the group's position hash when it has
// one (linear probing, load <= 1/2, so an empty slot ends every probe),
// else a binary search of n0.
struct PosIndex {
  const int32_t *n0;
  int d0;
  const int *hkeys;  // null: no hash
  const int *hpos;
  int lg;
  __device__ __forceinline__ int find(int y) const {
    if (!hkeys) return find_pos(n0, d0, y);
    const unsigned mask = (1u << lg) - 1u;
    unsigned h = ((unsigned)y * 2654435769u) >> (32 - lg);
    for (int step = 0; step <= (int)mask; ++step) {
      const int k = hkeys[h];
      if (k == y) return hpos[h];
      if (k < 0) return -1;
      h = (h + 1u) & mask;
    }
    return -1;
  }
};

// Row of x over N0: bit j set iff N0[j] in N(x).  One lane owns the row (no
// other lane writes it).  The cheapest of three walks is taken: each
// neighbour of x searched in N0 (shared memory), each N0[j] searched in N(x)
// (global), or a merge of the two sorted lists.
template <int W>
__device__ __forceinline__ void build_row(const int64_t *__restrict__ rp,
                                          const int32_t *__restrict__ ci, const PosIndex &idx,
                                          int x, unsigned *row) {
  const int32_t *n0 = idx.n0;
  const int d0 = idx.d0;
#pragma unroll
  for (int k = 0; k < W; ++k) row[k] = 0;
  const int64_t b = __ldg(rp + x), e = __ldg(rp + x + 1);
  const int dx = (int)(e - b);
  const int by_x = dx * ceil_log2_int(d0 + 1);
  const int by_n0 = d0 * ceil_log2_int(dx + 1);
  const int merge = dx + d0;
  if (by_x <= by_n0 && by_x <= merge) {
    for (int64_t t = b; t < e; ++t) {
      const int j = idx.find(__ldg(ci + t));
      if (j >= 0) row[j >> 5] |= 1u << (j & 31);
    }
  } else if (by_n0 <= merge) {
    for (int j = 0; j < d0; ++j) {
      const int y = n0[j];
      int64_t lo = b, hi = e - 1;
      while (lo <= hi) {
        const int64_t mid = (lo + hi) >> 1;
        const int m = __ldg(ci + mid);
        if (m == y) {
          row[j >> 5] |= 1u << (j & 31);
          break;
        }
        if (m < y) lo = mid + 1;
        else hi = mid - 1;
      }
    }
  } else {
    int j = 0;
    for (int64_t t = b; t < e && j < d0; ++t) {
      const int y = __ldg(ci + t);
      while (j < d0 && n0[j] < y) ++j;
      if (j < d0 && n0[j] == y) row[j >> 5] |= 1u << (j & 31);
    }
  }
}

__device__ __forceinline__ bool bit_of(const unsigned *row, int j) {
  return (row[j >> 5] >> (j & 31)) & 1u;
}

// Warp wg of the center's G warps takes edges p = wg, wg + G, ...; its lanes
// split the positions q (P3, P7) or r (P1) of each edge.  Membership in A
// and B is read from M's row p; the fully unrolled word loops keep A and D
// in registers.
template <int P, int W>
__device__ __forceinline__ void center_edges(const unsigned *M, int d0, int wg, int G, int lane,
                                             Acc &acc) {
  for (int p = wg; p < d0; p += G) {
    const unsigned *mp = M + p * W;
    if (P == 1) {
      unsigned A[W];
#pragma unroll
      for (int k = 0; k < W; ++k) A[k] = ~mp[k] & below_word(k, p) & full_word(k, d0);
      for (int r = lane; r < p; r += kWarp) {
        if (!bit_of(mp, r)) continue;  // r in B = N0 & N1 below p
        const unsigned *mr = M + r * W;
        int c = 0;
#pragma unroll
        for (int k = 0; k < W; ++k) c += __popc(A[k] & above_word(k, r) & ~mr[k]);
        acc.c2 += (unsigned long long)c;
      }
    } else {
      unsigned A[W];
#pragma unroll
      for (int k = 0; k < W; ++k) A[k] = (P == 3 ? ~mp[k] : mp[k]) & full_word(k, d0);
      for (int q = lane; q < d0; q += kWarp) {
        if (bit_of(mp, q) != (P == 7)) continue;  // q in A
        const unsigned *mq = M + q * W;
        unsigned D[W];
        int cnt = 0, freq = 0;
#pragma unroll
        for (int k = 0; k < W; ++k) {
          const unsigned nq = A[k] & ~mq[k];
          D[k] = nq & below_word(k, q);
          cnt += __popc(D[k]);
          freq += __popc(nq & above_word(k, q));
        }
        acc.c1 += wrap_mul(cnt, freq);
        if (cnt == 0) continue;  // D empty: no correction term
        for (int k = 0; k < W; ++k) {
          unsigned cw = (P == 3 ? ~mp[k] : mp[k]) & mq[k] & full_word(k, d0);  // A & N(q)
          while (cw) {
            const int r = 32 * k + __ffs(cw) - 1;
            cw &= cw - 1;
            const unsigned *mr = M + r * W;
            int c = 0;
#pragma unroll
            for (int k2 = 0; k2 < W; ++k2) c += __popc(D[k2] & above_word(k2, r) & ~mr[k2]);
            acc.c2 += (unsigned long long)c;
          }
        }
      }
    }
  }
}

// P2, P4, P5, P6, P8 for the edges p = wg, wg + G, ... of center v0.  The
// lanes split y over N1 = N(v1); each y outside N0 and other than v0 gets
// its row R(y) in the lane's own scratch row, then (A, B masks over N0 in
// registers, M in shared memory):
//   P2/P8  A = N0 - N1 (P2) or N0 & N1 (P8): cnt[r]++ and
//          c2 += |(A & ~R) & above(r) & ~M[r] (P2) / M[r] (P8)| for r in A & R;
//          afterwards c1 += |A & ~M[q] / M[q] & below(q)| * ((|N1 - N0| - 1) - cnt[q])
//          for q in A                             (:135-243, :461-572)
//   P5     A = N0 & N1, B = N0 - N1: cnt[b]++ for b in B & R,
//          c2 += |B & ~M[v2] & ~R| for v2 in A & R; afterwards
//          c1 += ((|N1 - N0| - 1) - cnt[b]) * |A & ~M[b]| for b in B   (:574-734)
//   P6     A = N0 & N1: c1 += |A & ~R & ~M[v2]| for v2 in A & ~R       (:736-853)
//   P4     (v1 < v0 only) A = N0 - N1: c1 += |A & ~R|                 (:855-963)
// v0 itself (in N1 - N0) is adjacent to every vertex of N0 and adds nothing
// to any term, which the "- 1" accounts for.
template <int P, int W>
__device__ __forceinline__ void center_outer_edges(const int64_t *__restrict__ rp,
                                                   const int32_t *__restrict__ ci,
                                                   const unsigned *M, const PosIndex &idx,
                                                   int v0, int wg, int G, int lane,
                                                   unsigned *Rw, int *cnt, int *slots,
                                                   const HopRows *hop,
                                                   const unsigned long long *deadline,
                                                   unsigned long long *stop_flag, Acc &acc) {
  const int32_t *n0 = idx.n0;
  const int d0 = idx.d0;
  unsigned *Rl = Rw + lane * W;
  const unsigned upto = lane == kWarp - 1 ? kFull : ((2u << lane) - 1u);
  for (int p = wg; p < d0; p += G) {
    if (warp_late(deadline, stop_flag, lane)) break;
    const int v1 = n0[p];
    if (P == 4 && !(v1 < v0)) continue;
    const unsigned *mp = M + p * W;
    unsigned A[W], B[W];
    int in_both = 0;
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const unsigned f = full_word(k, d0);
      const bool a_out = (P == 2 || P == 4);  // A = N0 - N1
      A[k] = (a_out ? ~mp[k] : mp[k]) & f;
      B[k] = ~mp[k] & f;
      in_both += __popc(mp[k]);
    }
    const bool counts = (P == 2 || P == 5 || P == 8);
    if (counts) {
      for (int i = lane; i < d0; i += kWarp) cnt[i] = 0;
      __syncwarp();
    }
    const int64_t b1 = __ldg(rp + v1);
    const int d1 = (int)(__ldg(rp + v1 + 1) - b1);
    // N1 in chunks of 32: the outer neighbours y of a chunk are compacted
    // into lanes 0..nu-1, their rows R(y) built by a flat walk of their
    // concatenated lists (every lane one entry per step, entry -> owner lane
    // by counting the list starts in the window), then each lane applies
    // its y's terms.
    for (int c0 = 0; c0 < d1; c0 += kWarp) {
      bool use = false;
      int y = 0;
      if (c0 + lane < d1) {
        y = __ldg(ci + b1 + c0 + lane);
        use = y != v0 && idx.find(y) < 0;
      }
      const unsigned um = __ballot_sync(kFull, use);
      if (use) slots[__popc(um & ((1u << lane) - 1u))] = y;
      const int nu = __popc(um);
      __syncwarp();
      const bool mine = lane < nu;
      if (hop) {
        // R(y) from the center's two-hop rows: each lane copies its own.
        if (mine) {
          const unsigned *r = hop->row_of(slots[lane]);
#pragma unroll
          for (int k = 0; k < W; ++k) Rl[k] = r ? r[k] : 0u;
        }
        __syncwarp();
      } else {
#pragma unroll
      for (int k = 0; k < W; ++k) Rl[k] = 0;
      int64_t ys = 0;
      int dy = 0;
      if (mine) {
        const int yl = slots[lane];
        ys = __ldg(rp + yl);
        dy = (int)(__ldg(rp + yl + 1) - ys);  // >= 1: yl is adjacent to v1
      }
      const int incl = warp_inclusive_scan(dy, lane);
      const int excl = incl - dy;
      const int total = __shfl_sync(kFull, incl, kWarp - 1);
      __syncwarp();  // rows cleared before other lanes set their bits
      int started = 0;  // lists started before window F
      for (int F = 0; F < total; F += kWarp) {
        const unsigned bit = (dy > 0 && excl >= F && excl < F + kWarp) ? (1u << (excl - F)) : 0u;
        const unsigned starts = __reduce_or_sync(kFull, bit);
        const int o = max(started + __popc(starts & upto) - 1, 0);
        const int64_t oys = __shfl_sync(kFull, ys, o);
        const int oex = __shfl_sync(kFull, excl, o);
        const int f = F + lane;
        if (f < total) {
          const int pos = idx.find(__ldg(ci + oys + (f - oex)));
          if (pos >= 0) atomicOr(Rw + o * W + (pos >> 5), 1u << (pos & 31));
        }
        started += __popc(starts);
      }
      __syncwarp();
      }  // per-edge rows
      if (mine) {
      if (P == 4) {
        int c = 0;
#pragma unroll
        for (int k = 0; k < W; ++k) c += __popc(A[k] & ~Rl[k]);
        acc.c1 += (unsigned long long)c;
      } else if (P == 6) {
        for (int k = 0; k < W; ++k) {
          unsigned sw = mp[k] & full_word(k, d0) & ~Rl[k];  // A & ~R
          while (sw) {
            const int v2 = 32 * k + __ffs(sw) - 1;
            sw &= sw - 1;
            const unsigned *m2 = M + v2 * W;
            int c = 0;
#pragma unroll
            for (int k2 = 0; k2 < W; ++k2) c += __popc(A[k2] & ~Rl[k2] & ~m2[k2]);
            acc.c1 += (unsigned long long)c;
          }
        }
      } else if (P == 5) {
        for (int k = 0; k < W; ++k) {
          unsigned bw = (~mp[k] & full_word(k, d0)) & Rl[k];  // B & R
          while (bw) {
            const int bpos = 32 * k + __ffs(bw) - 1;
            bw &= bw - 1;
            atomicAdd(cnt + bpos, 1);
          }
          unsigned aw = mp[k] & Rl[k];  // A & R
          while (aw) {
            const int v2 = 32 * k + __ffs(aw) - 1;
            aw &= aw - 1;
            const unsigned *m2 = M + v2 * W;
            int c = 0;
#pragma unroll
            for (int k2 = 0; k2 < W; ++k2) c += __popc(B[k2] & ~m2[k2] & ~Rl[k2]);
            acc.c2 += (unsigned long long)c;
          }
        }
      } else {  // P2, P8
        for (int k = 0; k < W; ++k) {
          unsigned cw = ((P == 2 ? ~mp[k] : mp[k]) & full_word(k, d0)) & Rl[k];  // A & R
          while (cw) {
            const int r = 32 * k + __ffs(cw) - 1;
            cw &= cw - 1;
            atomicAdd(cnt + r, 1);
            const unsigned *mr = M + r * W;
            int c = 0;
#pragma unroll
            for (int k2 = 0; k2 < W; ++k2)
              c += __popc(A[k2] & ~Rl[k2] & above_word(k2, r) & (P == 2 ? ~mr[k2] : mr[k2]));
            acc.c2 += (unsigned long long)c;
          }
        }
      }
      }  // mine
      __syncwarp();  // rows and slots are rewritten by the next chunk
    }
    if (counts) {
      __syncwarp();
      const int others = (d1 - in_both) - 1;  // |N1 - N0| without v0
      if (P == 5) {
        for (int q = lane; q < d0; q += kWarp) {
          if (bit_of(mp, q)) continue;  // q in B = N0 - N1
          const unsigned *mq = M + q * W;
          int f = 0;
#pragma unroll
          for (int k = 0; k < W; ++k) f += __popc(A[k] & ~mq[k]);
          acc.c1 += wrap_mul(others - cnt[q], f);
        }
      } else {
        for (int q = lane; q < d0; q += kWarp) {
          if (bit_of(mp, q) != (P == 8)) continue;  // q in A
          const unsigned *mq = M + q * W;
          int c = 0;
#pragma unroll
          for (int k = 0; k < W; ++k)
            c += __popc(A[k] & (P == 2 ? ~mq[k] : mq[k]) & below_word(k, q));
          acc.c1 += wrap_mul(c, others - cnt[q]);
        }
      }
      __syncwarp();  // cnt is cleared for the next edge
    }
  }
}

__device__ __forceinline__ void group_sync(int G) {
  if (G == 1) __syncwarp();
  else __syncthreads();
}

// Builds the two-hop rows of center v0 in this group's scratch.  Returns
// false (every thread of the group alike) when they do not fit; the edges
// then build their rows per edge.
template <int W, int G>
__device__ bool build_hop_rows(const CenterArgs &a, const PosIndex &idx, int v0, int grp, int gl,
                               int wg, int lane, unsigned long long *s_walk, int *s_keys,
                               int *s_rows, HopRows *out) {
  constexpr int kGroups = kPatThreads / kWarp / G;
  const int32_t *n0 = idx.n0;
  const int d0 = idx.d0;
  if (gl == 0) {
    *s_walk = 0;
    *s_keys = 0;
    *s_rows = 0;
  }
  group_sync(G);
  unsigned long long walk = 0;
  for (int i = gl; i < d0; i += G * kWarp) {
    const int x = n0[i];
    walk += (unsigned long long)(__ldg(a.rp + x + 1) - __ldg(a.rp + x));
  }
  walk = warp_sum_u64(walk);
  if (lane == 0 && walk) atomicAdd(s_walk, walk);
  group_sync(G);
  const unsigned long long B = *s_walk;
  int lg = 6;
  while ((1ull << lg) < 2 * B) ++lg;
  const int64_t cap = int64_t(1) << lg;
  if (lg > 30 || 2 * cap > a.hop_words) return false;  // the same on every thread
  unsigned *base = a.hop + ((int64_t)blockIdx.x * kGroups + grp) * a.hop_words;
  int *keys = reinterpret_cast<int *>(base);
  int *vals = keys + cap;
  unsigned *rows = reinterpret_cast<unsigned *>(vals + cap);
  const unsigned mask = (unsigned)cap - 1u;
  for (int64_t j = gl; j < cap; j += G * kWarp) keys[j] = -1;
  group_sync(G);
  // Keys: every y outside N0 + {v0} adjacent to a member of N0 (at most B
  // distinct, so the map's load stays <= 1/2 and every probe ends).
  for (int i = wg; i < d0; i += G) {
    const int x = n0[i];
    const int64_t b = __ldg(a.rp + x), e = __ldg(a.rp + x + 1);
    for (int64_t t = b + lane; t < e; t += kWarp) {
      const int y = __ldg(a.ci + t);
      if (y == v0 || idx.find(y) >= 0) continue;
      unsigned h = ((unsigned)y * 2654435769u) >> (32 - lg);
      for (int64_t step = 0; step < cap; ++step) {
        const int old = atomicCAS(keys + h, -1, y);
        if (old == -1) {
          atomicAdd(s_keys, 1);
          break;
        }
        if (old == y) break;
        h = (h + 1u) & mask;
      }
    }
  }
  group_sync(G);
  const int64_t nkeys = *s_keys;
  if (2 * cap + nkeys * W > a.hop_words) return false;  // the same on every thread
  for (int64_t j = gl; j < cap; j += G * kWarp)
    if (keys[j] >= 0) vals[j] = atomicAdd(s_rows, 1);
  for (int64_t j = gl; j < nkeys * W; j += G * kWarp) rows[j] = 0u;
  group_sync(G);
  const HopRows hr{keys, vals, rows, lg, W};
  for (int i = wg; i < d0; i += G) {
    const int x = n0[i];
    const int64_t b = __ldg(a.rp + x), e = __ldg(a.rp + x + 1);
    for (int64_t t = b + lane; t < e; t += kWarp) {
      const int y = __ldg(a.ci + t);
      if (y == v0 || idx.find(y) >= 0) continue;
      const unsigned *r = hr.row_of(y);
      if (r) atomicOr(const_cast<unsigned *>(r) + (i >> 5), 1u << (i & 31));
    }
  }
  group_sync(G);
  *out = hr;
  return true;
}

// Persistent groups of G warps take centers of this class from the queue.
template <int P, int W>
__global__ void __launch_bounds__(kPatThreads) center_kernel(CenterArgs a) {
  constexpr int G = center_group(W);
  constexpr int kGroups = kPatThreads / kWarp / G;
  extern __shared__ unsigned char smem[];
  __shared__ int s_center[kGroups];
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x / kWarp;
  const int grp = warp / G, wg = warp % G, gl = wg * kWarp + lane;  // lane within the group
  unsigned *M = reinterpret_cast<unsigned *>(smem + grp * center_group_bytes(P, W));
  int32_t *n0 = reinterpret_cast<int32_t *>(M + 32 * W * W);
  // Outer patterns: this warp's R rows (one per lane) and position counters.
  unsigned *Rw = reinterpret_cast<unsigned *>(n0 + 32 * W) + wg * (64 * W + 32);
  int *cnt = reinterpret_cast<int *>(Rw + 32 * W);
  int *slots = cnt + 32 * W;
  // Position hash of N0 (outer patterns, W >= 4), after all warps' scratch.
  int *hkeys = reinterpret_cast<int *>(n0 + 32 * W) +
               (center_outer(P) ? center_group(W) * (64 * W + 32) : 0);
  const int64_t count = *a.count;
  const int64_t limit = a.c_end >= 0 && a.c_end < count ? a.c_end : count;
  __shared__ unsigned long long s_hop_walk[kGroups];
  __shared__ int s_hop_keys[kGroups], s_hop_rows[kGroups];
  Acc acc;
  for (;;) {
    if (gl == 0) {
      if (a.deadline && global_ns() > *a.deadline) {
        atomicOr(a.stop_flag, 1ull);
        s_center[grp] = -1;
      } else {
        const int64_t t = a.c_begin + (int64_t)atomicAdd(a.queue, 1ull);
        s_center[grp] = t < limit ? a.centers[t] : -1;
      }
    }
    if (G == 1) __syncwarp(); else __syncthreads();
    const int v0 = s_center[grp];
    if (v0 < 0) break;
    const int64_t b0 = __ldg(a.rp + v0);
    const int d0 = (int)(__ldg(a.rp + v0 + 1) - b0);
    for (int i = gl; i < d0; i += G * kWarp) n0[i] = __ldg(a.ci + b0 + i);
    PosIndex idx{n0, d0, nullptr, nullptr, 0};
    if constexpr (center_hash(P, W)) {
      constexpr int kLg = 6 + (W >= 8) + (W >= 16) + (W >= 32) + 2;  // 64W slots
      static_assert((1 << kLg) == 64 * W, "hash size");
      for (int i = gl; i < (1 << kLg); i += G * kWarp) hkeys[i] = -1;
      if (G == 1) __syncwarp(); else __syncthreads();
      for (int i = gl; i < d0; i += G * kWarp) {
        const int y = n0[i];
        unsigned h = ((unsigned)y * 2654435769u) >> (32 - kLg);
        // Keys are distinct and the load is <= 1/2: an empty slot is found.
        for (int step = 0; step < (1 << kLg); ++step) {
          if (atomicCAS(hkeys + h, -1, y) == -1) {
            hkeys[(1 << kLg) + h] = i;
            break;
          }
          h = (h + 1u) & ((1u << kLg) - 1u);
        }
      }
      idx = PosIndex{n0, d0, hkeys, hkeys + (1 << kLg), kLg};
    }
    if (G == 1) __syncwarp(); else __syncthreads();
    for (int i = gl; i < d0; i += G * kWarp) build_row<W>(a.rp, a.ci, idx, n0[i], M + i * W);
    if (G == 1) __syncwarp(); else __syncthreads();
    if (P == 1) {  // star term of v0 (P1_frequency_count)
      for (int i = gl; i < d0; i += G * kWarp) {
        const unsigned *mi = M + i * W;
        int c = 0, f = 0;
#pragma unroll
        for (int k = 0; k < W; ++k) {
          const unsigned non = ~mi[k] & full_word(k, d0);
          c += __popc(non & below_word(k, i));
          f += __popc(non & above_word(k, i));
        }
        acc.c1 += wrap_mul(c, f);
      }
    }
    if constexpr (center_outer(P)) {
      const HopRows *hop = nullptr;
      HopRows hr{};
      if (a.hop) {
        if (build_hop_rows<W, G>(a, idx, v0, grp, gl, wg, lane, s_hop_walk + grp,
                                 s_hop_keys + grp, s_hop_rows + grp, &hr))
          hop = &hr;
        else if (gl == 0)
          atomicAdd(a.hop_misses, 1ull);
      }
      center_outer_edges<P, W>(a.rp, a.ci, M, idx, v0, wg, G, lane, Rw, cnt, slots, hop,
                               a.deadline, a.stop_flag, acc);
    } else
      center_edges<P, W>(M, d0, wg, G, lane, acc);
    if (G == 1) __syncwarp(); else __syncthreads();  // M and n0 are rewritten next
  }
  const unsigned long long c1 = warp_sum_u64(acc.c1), c2 = warp_sum_u64(acc.c2);
  if (lane == 0) {
    if (c1) atomicAdd(a.counters + 0, c1);
    if (c2) atomicAdd(a.counters + 1, c2);
  }
}

// ---- P1 on the centers above kCenterMaxDeg ----------------------------------
// One CTA per (center v0, chunk of kHubEdgeChunk of its edges), persistent
// over an atomic queue.  The CTA marks N0 = N(v0) in its own bitmap over the
// vertex ids (global memory, n bits, cleared again after the task), so that
// "x in N0" is one bit read.  Chunk c also adds the star terms of positions
// [256c, 256c + 256) of N0.  With
// positions in N0 equal to id order (N0 is sorted):
//   star  (P1_frequency_count, pattern_kernels.cuh:68-133): for x = N0[i],
//         lo / hi = neighbours of x in N0 below / above x;
//         c1 += wrap32((i - lo) * ((d0 - 1 - i) - hi))
//   edge (v0, v1 = N0[p]) (P1_count_correction, :6-66): B = N1 & N0 below v1
//         (ascending), and for v2 = B[t]
//         c2 += #{k in N0 : v2 < k < v1, k notin N1, k notin N(v2)}
//             = (p - pos(v2) - 1) - (|B| - 1 - t)
//               - #{k in N(v2) : v2 < k < v1, k in N0, k notin N1}
// These are the sizes of the reference's sets A = N0 - N1 and B = N0 & N1
// (both below v1) and its pair test, counted through the symmetry of the
// graph; the per-vertex products are the same 32-bit products.
constexpr int kHubEdgeChunk = 256;

struct HubP1Args {
  const int64_t *__restrict__ rp;
  const int32_t *__restrict__ ci;
  int64_t n;
  const int64_t *chunk_off;  // exclusive scan of the chunks per vertex (n + 1)
  unsigned *bits;            // per CTA: ceil(n / 32) words, all zero between tasks
  int32_t *scratch;          // per warp: cap ints (the list B)
  int64_t cap;
  unsigned long long *queue;
  unsigned long long *counters;  // [0] c1, [1] c2
  int shard, num_shards;
  const unsigned long long *deadline = nullptr;
  unsigned long long *stop_flag = nullptr;
  int64_t task_begin = 0, task_end = -1;  // slice of the queue positions
  int lane_scan = 64;  // ranges up to this many entries are scanned by one lane
};

__device__ __forceinline__ int warp_sum_int(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ bool bit_set(const unsigned *bits, int v) {
  return (bits[v >> 5] >> (v & 31)) & 1u;
}

// Position of y in the ascending list[0, n) (y present).
__device__ __forceinline__ int lower_pos(const int32_t *__restrict__ list, int n, int y) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(list + mid) < y) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(kPatThreads) hub_p1_kernel(HubP1Args a) {
  constexpr int kWarps = kPatThreads / kWarp;
  __shared__ long long s_task;
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x / kWarp;
  unsigned *bits = a.bits + (int64_t)blockIdx.x * ((a.n + 31) >> 5);
  int32_t *B = a.scratch + ((int64_t)blockIdx.x * kWarps + warp) * a.cap;
  const int64_t all = __ldg(a.chunk_off + a.n);
  const int64_t ntasks = all > a.shard ? (all - a.shard + a.num_shards - 1) / a.num_shards : 0;
  const int64_t t_end = a.task_end >= 0 && a.task_end < ntasks ? a.task_end : ntasks;
  const int64_t span = t_end - a.task_begin;
  Acc acc;
  for (;;) {
    if (threadIdx.x == 0) {
      long long t = (long long)atomicAdd(a.queue, 1ull);
      if (a.deadline && global_ns() > *a.deadline) {
        atomicOr(a.stop_flag, 1ull);
        t = span;
      }
      s_task = t;
    }
    __syncthreads();
    const int64_t q = s_task;
    if (q >= span) break;
    const int64_t t = (a.task_begin + q) * a.num_shards + a.shard;
    const int v0 = (int)upper_row(a.chunk_off, 0, a.n - 1, t);
    const int chunk = (int)(t - __ldg(a.chunk_off + v0));
    const int64_t b0 = __ldg(a.rp + v0);
    const int d0 = (int)(__ldg(a.rp + v0 + 1) - b0);
    const int32_t *n0 = a.ci + b0;
    for (int i = threadIdx.x; i < d0; i += kPatThreads) {
      const int y = __ldg(n0 + i);
      atomicOr(bits + (y >> 5), 1u << (y & 31));
    }
    __syncthreads();
    {  // the star term of v0 over this chunk's positions (balanced with the edges)
      const int i_end = min(d0, (chunk + 1) * kHubEdgeChunk);
      for (int i = chunk * kHubEdgeChunk + warp; i < i_end; i += kWarps) {
        const int x = __ldg(n0 + i);
        const int64_t bx = __ldg(a.rp + x), ex = __ldg(a.rp + x + 1);
        int lo = 0, hi = 0;
        for (int64_t k = bx + lane; k < ex; k += kWarp) {
          const int y = __ldg(a.ci + k);
          if (bit_set(bits, y)) {
            if (y < x) ++lo;
            else ++hi;
          }
        }
        lo = warp_sum_int(lo);
        hi = warp_sum_int(hi);
        if (lane == 0) acc.c1 += wrap_mul(i - lo, (d0 - 1 - i) - hi);
      }
    }
    const int p_end = min(d0, (chunk + 1) * kHubEdgeChunk);
    for (int p = chunk * kHubEdgeChunk + warp; p < p_end; p += kWarps) {
      const int v1 = __ldg(n0 + p);
      const int64_t b1 = __ldg(a.rp + v1);
      const int d1 = (int)(__ldg(a.rp + v1 + 1) - b1);
      const int32_t *n1 = a.ci + b1;
      // B = N1 & N0 below v1, in order (ballot compaction).
      int nb = 0;
      for (int base = 0; base < d1; base += kWarp) {
        const int k = base + lane;
        const int y = k < d1 ? __ldg(n1 + k) : INT_MAX;
        const bool keep = y < v1 && bit_set(bits, y);
        const unsigned m = __ballot_sync(kFull, keep);
        if (keep) B[nb + __popc(m & ((1u << lane) - 1u))] = y;
        nb += __popc(m);
        if (__any_sync(kFull, y >= v1)) break;
      }
      __syncwarp();
      // For v2 in B: #{k : v2 < k < v1, k in N0 & N(v2), k notin N1}, over the
      // shorter of N(v2) and N0 within (v2, v1).  Lane t takes B[t], B[t + 32],
      // ... and scans a short range itself; ranges above kLaneScan entries
      // are scanned by the whole warp, one after the other.
      const int kLaneScan = a.lane_scan;
      long long c2 = 0;
      for (int base = 0; base < nb; base += kWarp) {
        const int tb = base + lane;
        int q2 = 0, side = 0;  // side 1: scan N(v2) [lo, top); 0: N0 (q2, p)
        int64_t lo = 0, top = 0, b2 = 0;
        int d2 = 0, len = 0;
        if (tb < nb) {
          const int v2 = B[tb];
          q2 = lower_pos(n0, d0, v2);
          b2 = __ldg(a.rp + v2);
          const int64_t e2 = __ldg(a.rp + v2 + 1);
          d2 = (int)(e2 - b2);
          lo = b2;
          int64_t hi = e2;  // first entry of N(v2) above v2
          while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (__ldg(a.ci + mid) <= v2) lo = mid + 1;
            else hi = mid;
          }
          top = lo;
          hi = e2;  // first entry at or above v1
          while (top < hi) {
            const int64_t mid = (top + hi) >> 1;
            if (__ldg(a.ci + mid) < v1) top = mid + 1;
            else hi = mid;
          }
          side = top - lo <= p - q2 - 1;
          len = side ? (int)(top - lo) : p - q2 - 1;
          c2 += (long long)(p - q2 - 1) - (nb - 1 - tb);
          if (len <= kLaneScan) {
            int drop = 0;
            if (side) {
              for (int64_t k = lo; k < top; ++k) {
                const int y = __ldg(a.ci + k);
                drop += bit_set(bits, y) && !bsearch(n1, d1, y);
              }
            } else {
              for (int j = q2 + 1; j < p; ++j) {
                const int y = __ldg(n0 + j);
                drop += bsearch(a.ci + b2, d2, y) && !bsearch(n1, d1, y);
              }
            }
            c2 -= drop;
          }
        }
        unsigned longs = __ballot_sync(kFull, tb < nb && len > kLaneScan);
        while (longs) {
          const int src = __ffs(longs) - 1;
          longs &= longs - 1u;
          const int s_side = __shfl_sync(kFull, side, src);
          const int64_t s_lo = __shfl_sync(kFull, lo, src), s_top = __shfl_sync(kFull, top, src);
          const int64_t s_b2 = __shfl_sync(kFull, b2, src);
          const int s_d2 = __shfl_sync(kFull, d2, src), s_q2 = __shfl_sync(kFull, q2, src);
          int drop = 0;
          if (s_side) {
            for (int64_t k = s_lo + lane; k < s_top; k += kWarp) {
              const int y = __ldg(a.ci + k);
              drop += bit_set(bits, y) && !bsearch(n1, d1, y);
            }
          } else {
            for (int j = s_q2 + 1 + lane; j < p; j += kWarp) {
              const int y = __ldg(n0 + j);
              drop += bsearch(a.ci + s_b2, s_d2, y) && !bsearch(n1, d1, y);
            }
          }
          c2 -= drop;
        }
      }
      acc.c2 += (unsigned long long)c2;
      __syncwarp();  // B is rewritten by the warp's next edge
    }
    __syncthreads();
    for (int i = threadIdx.x; i < d0; i += kPatThreads) bits[__ldg(n0 + i) >> 5] = 0u;
    __syncthreads();
  }
  const unsigned long long c1 = warp_sum_u64(acc.c1), c2 = warp_sum_u64(acc.c2);
  if (lane == 0) {
    if (c1) atomicAdd(a.counters + 0, c1);
    if (c2) atomicAdd(a.counters + 1, c2);
  }
}

// chunks[v] = ceil(big_deg[v] / kHubEdgeChunk).
__global__ void hub_chunks_kernel(const int32_t *__restrict__ big_deg, int64_t n,
                                  int32_t *__restrict__ chunks) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) chunks[v] = (big_deg[v] + kHubEdgeChunk - 1) / kHubEdgeChunk;
}

// Splits the vertices into the six center classes (1 <= degree <= 1024;
// class c holds degrees in (16 * 2^c, 32 * 2^c], class 0 from 1) and marks
// the larger ones: big_deg[v] = degree if above kCenterMaxDeg, else 0.
__global__ void center_classes_kernel(const int64_t *__restrict__ rp, int64_t n, int shard,
                                      int num_shards, int32_t *__restrict__ lists,
                                      int32_t *__restrict__ counts,
                                      int32_t *__restrict__ big_deg) {
  __shared__ int h[kCenterClasses], base[kCenterClasses];
  if (threadIdx.x < kCenterClasses) h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int cls = -1, slot = 0;
  if (v < n) {
    const int d = (int)(rp[v + 1] - rp[v]);
    big_deg[v] = d > kCenterMaxDeg ? d : 0;
    // A shard keeps the centers v = shard (mod num_shards); the large
    // centers' edge tasks are split by pattern_kernel itself.
    if (d >= 1 && d <= kCenterMaxDeg && v % num_shards == shard) {
      cls = 0;
      while (32 * center_words(cls) < d) ++cls;
      slot = atomicAdd(&h[cls], 1);
    }
  }
  __syncthreads();
  if (threadIdx.x < kCenterClasses) base[threadIdx.x] = atomicAdd(counts + threadIdx.x, h[threadIdx.x]);
  __syncthreads();
  if (cls >= 0) lists[(int64_t)cls * n + base[cls] + slot] = (int32_t)v;
}

// Long pattern counts run in slices of their task range, each a launch of
// bounded length, so that no kernel runs for minutes and a caller's time
// budget can end the count between two slices.  Slices are sized from the
// previous slice's measured time (first slice: one task per resident warp or
// group, then x(target / measured), clamped to [1/4, 4]).
struct Slicer {
  bool on = false;
  double budget_ms = -1.0;  // < 0: no budget
  double target_ms = 250.0;
  bool trace = false;
  double used_ms = 0.0;     // device time of the sliced launches so far
  int64_t tasks_total = 0, tasks_done = 0, slices = 0;
  // With a budget the kernels also stop by themselves at a device deadline
  // (a single hub edge can outlast any slice); stop_flag is the device word
  // they raise, and h_stop its host copy.
  unsigned long long *stop_flag = nullptr;
  unsigned long long *h_stop = nullptr;
};

__global__ void set_deadline_kernel(unsigned long long *deadline, unsigned long long budget_ns) {
  *deadline = global_ns() + budget_ns;
}

// launch(begin, end) runs tasks [begin, end) of a launch whose queue counter
// is `queue`; total = the launch's task count, first = first slice size.
template <class Launch>
int run_slices(mc_dgraph *g, Slicer &sl, const char *what, int64_t total, int64_t first,
               unsigned long long *queue, Launch launch) {
  if (!sl.on) return launch(0, -1);
  if (total <= 0) return MC_OK;
  cudaStream_t s = g->stream;
  sl.tasks_total += total;
  int64_t b = 0, size = std::max<int64_t>(first, 1);
  while (b < total) {
    const int64_t e = std::min(total, b + size);
    MC_CUDA_TRY(cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s));
    MC_CUDA_TRY(cudaEventRecord(g->ev[4], s));
    const int rc = launch(b, e);
    if (rc != MC_OK) return rc;
    if (sl.stop_flag)
      MC_CUDA_TRY(cudaMemcpyAsync(sl.h_stop, sl.stop_flag, sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, s));
    MC_CUDA_TRY(cudaEventRecord(g->ev[5], s));
    MC_CUDA_TRY(cudaEventSynchronize(g->ev[5]));
    float ms = 0.f;
    MC_CUDA_TRY(cudaEventElapsedTime(&ms, g->ev[4], g->ev[5]));
    sl.used_ms += ms;
    sl.tasks_done += e - b;
    sl.slices += 1;
    if (sl.trace)
      std::fprintf(stderr, "mercury: %s slice [%lld, %lld) of %lld: %.3f ms (total %.1f ms)\n",
                   what, (long long)b, (long long)e, (long long)total, ms, sl.used_ms);
    b = e;
    if (sl.h_stop && *sl.h_stop) return MC_ERR_TIMEOUT;  // stopped at the deadline
    if (sl.budget_ms > 0 && sl.used_ms > sl.budget_ms && b < total) return MC_ERR_TIMEOUT;
    // Never below one task per resident warp or group: a smaller slice
    // leaves the GPU idle.
    const double f = ms > 0.01f ? std::min(4.0, std::max(0.25, sl.target_ms / ms)) : 4.0;
    size = std::max<int64_t>(std::max<int64_t>(first, 1), (int64_t)((double)size * f));
  }
  return MC_OK;
}

// Largest two-hop walk (sum over x in N(v) of d(x)) among the centers of each
// class: sizes the two-hop row maps (walk[c], c = class).
__global__ void hop_need_kernel(const int64_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                int64_t n, int shard, int num_shards,
                                unsigned long long *__restrict__ walk) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const int64_t b = rp[v], e = rp[v + 1];
  const int d = (int)(e - b);
  if (d < 1 || d > kCenterMaxDeg || v % num_shards != shard) return;
  int cls = 0;
  while (32 * center_words(cls) < d) ++cls;
  unsigned long long sum = 0;
  for (int64_t k = b; k < e; ++k) {
    const int x = __ldg(ci + k);
    sum += (unsigned long long)(__ldg(rp + x + 1) - __ldg(rp + x));
  }
  atomicMax(walk + cls, sum);
}

// Words of two-hop scratch one group needs for a center whose walk is B
// (the map of build_hop_rows plus at most B rows of W words).
__host__ __device__ inline int64_t hop_group_words(int64_t B, int W) {
  int lg = 6;
  while ((int64_t(1) << lg) < 2 * B) ++lg;
  return 2 * (int64_t(1) << lg) + B * W;
}

template <int P, int W>
int launch_center(mc_dgraph *g, const CenterArgs &a, int num_sms, int64_t total, Slicer *sl) {
  constexpr int G = center_group(W);
  const size_t smem = center_group_bytes(P, W) * (kPatThreads / kWarp / G);
  auto kern = center_kernel<P, W>;
  MC_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPatThreads, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const int grid = num_sms * per_sm;
  CenterArgs ha = a;
  if (center_outer(P) && a.hop_walk > 0) {
    // Each resident group gets the words its largest center needs, within
    // 4 GiB (or a quarter of the free memory) in all; centers that do not
    // fit build their rows per edge.
    const int64_t groups = (int64_t)grid * (kPatThreads / kWarp / G);
    const int64_t need = hop_group_words(a.hop_walk, W);
    size_t free_b = 0, total_b = 0;
    MC_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    const int64_t cap_words =
        (int64_t)(std::min<size_t>(size_t(4) << 30, free_b / 4) / sizeof(unsigned));
    int64_t per_group = std::min<int64_t>(need, cap_words / groups);
    // MERCURY_HOP_WORDS lowers the share (tests use it to send the larger
    // centers to the per-edge rows).
    if (const char *env = std::getenv("MERCURY_HOP_WORDS"))
      per_group = std::min<int64_t>(per_group, std::atoll(env));
    const size_t bytes = (size_t)(per_group * groups) * sizeof(unsigned);
    if (per_group > 0 && bytes > g->hop_scratch_bytes) {
      if (g->hop_scratch) dev_free(g->hop_scratch, g->stream);
      g->hop_scratch = nullptr;
      g->hop_scratch_bytes = 0;
      MC_CUDA_TRY(dev_alloc(&g->hop_scratch, bytes, g->stream));
      g->hop_scratch_bytes = bytes;
    }
    ha.hop = per_group > 0 ? static_cast<unsigned *>(g->hop_scratch) : nullptr;
    ha.hop_words = per_group;
  } else {
    ha.hop = nullptr;
  }
  return run_slices(g, *sl, "centers", total, (int64_t)grid * (kPatThreads / kWarp / G), a.queue,
                    [&](int64_t b, int64_t e) {
                      CenterArgs sa = ha;
                      sa.c_begin = b;
                      sa.c_end = e;
                      kern<<<grid, kPatThreads, smem, g->stream>>>(sa);
                      MC_CUDA_TRY(cudaGetLastError());
                      g->launches += 1;
                      return MC_OK;
                    });
}

template <int P>
int launch_center_class(mc_dgraph *g, const CenterArgs &a, int cls, int64_t total, Slicer *sl) {
  switch (cls) {
    case 0: return launch_center<P, 1>(g, a, g->num_sms, total, sl);
    case 1: return launch_center<P, 2>(g, a, g->num_sms, total, sl);
    case 2: return launch_center<P, 4>(g, a, g->num_sms, total, sl);
    case 3: return launch_center<P, 8>(g, a, g->num_sms, total, sl);
    case 4: return launch_center<P, 16>(g, a, g->num_sms, total, sl);
    default: return launch_center<P, 32>(g, a, g->num_sms, total, sl);
  }
}

// all: task count before sharding (n for star tasks, the restricted edge
// count with task_off, else nnz).
template <int P, bool kStar>
int launch_pattern(mc_dgraph *g, const PatArgs &a, int grid, int64_t all, Slicer *sl) {
  const int64_t ntasks =
      all > a.shard ? (all - a.shard + a.num_shards - 1) / a.num_shards : 0;
  return run_slices(g, *sl, kStar ? "stars" : "edges", ntasks,
                    (int64_t)grid * (kPatThreads / kWarp), a.queue,
                    [&](int64_t b, int64_t e) {
                      PatArgs sa = a;
                      sa.task_begin = b;
                      sa.task_end = e;
                      pattern_kernel<P, kStar><<<grid, kPatThreads, 0, g->stream>>>(sa);
                      MC_CUDA_TRY(cudaGetLastError());
                      g->launches += 1;
                      return MC_OK;
                    });
}

int grid_blocks(mc_dgraph *g, int64_t cap) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pattern_kernel<3, false>, kPatThreads,
                                                    0) != cudaSuccess)
    per_sm = 4;
  const int64_t resident = (int64_t)g->num_sms * std::max(per_sm, 1);
  const int64_t block_bytes = (int64_t)(kPatThreads / kWarp) * kLists * cap * 4;
  // The frontier scratch a handle keeps grows with its graph (256 bytes per
  // CSR entry, 8 MiB at least, kScratchBudget at most), so that thousands of
  // small resident graphs do not each hold the full budget.
  const int64_t budget = std::min<int64_t>(
      (int64_t)kScratchBudget, std::max<int64_t>(int64_t(8) << 20, 256 * std::max<int64_t>(g->nnz, 1)));
  const int64_t fit = std::max<int64_t>(1, budget / block_bytes);
  return (int)std::min(resident, fit);
}

// ---- batches: many graphs, each with its own pattern ----------------------
// Largest i in [0, count) with off[i] <= t (off ascending, off[0] == 0).
__device__ __forceinline__ int find_graph(const int64_t *off, int count, int64_t t) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(off + mid) <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int P>
__device__ __forceinline__ void batch_edge(const Warp &w, int v0, int v1, int32_t *L, int64_t cap,
                                           Acc &acc) {
  edge_pattern<P>(w, v0, v1, L, cap, acc);
}

// Persistent warps over the pattern tasks of a batch: first the P1 star
// tasks (one per vertex of every P1 graph), then one task per directed edge
// of every pattern graph; each task's counters go to its own graph.
__global__ void __launch_bounds__(kPatThreads) batch_pattern_kernel(BatchPatternArgs b) {
  __shared__ __align__(16) int s_sets[kPatThreads / kWarp][kSetSlots];
  __shared__ unsigned s_rows[kPatThreads / kWarp][kWarp];
  const int lane = threadIdx.x & (kWarp - 1);
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
  int32_t *L = b.scratch + gw * kLists * b.cap;
  const Warp w{b.rp, b.ci, lane, s_sets[threadIdx.x / kWarp], s_rows[threadIdx.x / kWarp]};
  const int64_t n_star = b.star_off[b.num_graphs], n_edge = b.edge_off[b.num_graphs];
  for (;;) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(b.queue, 1ull);
    t = __shfl_sync(kFull, t, 0);
    if ((int64_t)t >= n_star + n_edge) break;
    Acc acc;
    int pg;
    if ((int64_t)t < n_star) {
      pg = find_graph(b.star_off, b.num_graphs, (int64_t)t);
      vertex_star(w, (int)(b.v0[pg] + ((int64_t)t - b.star_off[pg])), L, acc);
    } else {
      const int64_t te = (int64_t)t - n_star;
      pg = find_graph(b.edge_off, b.num_graphs, te);
      const int64_t vb = b.v0[pg], ve = b.v1[pg];
      const int64_t e = __ldg(b.rp + vb) + (te - b.edge_off[pg]);
      const int v0 = (int)upper_row(b.rp, vb, ve - 1, e);
      const int v1 = __ldg(b.ci + e);
      switch (b.job[pg]) {
        case 1: batch_edge<1>(w, v0, v1, L, b.cap, acc); break;
        case 2: batch_edge<2>(w, v0, v1, L, b.cap, acc); break;
        case 3: batch_edge<3>(w, v0, v1, L, b.cap, acc); break;
        case 4: batch_edge<4>(w, v0, v1, L, b.cap, acc); break;
        case 5: batch_edge<5>(w, v0, v1, L, b.cap, acc); break;
        case 6: batch_edge<6>(w, v0, v1, L, b.cap, acc); break;
        case 7: batch_edge<7>(w, v0, v1, L, b.cap, acc); break;
        default: batch_edge<8>(w, v0, v1, L, b.cap, acc); break;
      }
    }
    const unsigned long long c1 = warp_sum_u64(acc.c1), c2 = warp_sum_u64(acc.c2);
    if (lane == 0) {
      const int g = b.graph[pg];
      if (c1) atomicAdd(b.c1 + g, c1);
      if (c2) atomicAdd(b.c2 + g, c2);
    }
  }
}

}  // namespace

int batch_pattern_launch(const BatchPatternArgs &b, int grid, cudaStream_t s) {
  batch_pattern_kernel<<<grid, kPatThreads, 0, s>>>(b);
  MC_CUDA_TRY(cudaGetLastError());
  return MC_OK;
}

int batch_pattern_grid(int num_sms, int64_t cap, int64_t *warps) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_pattern_kernel, kPatThreads,
                                                    0) != cudaSuccess)
    per_sm = 4;
  const int64_t resident = (int64_t)num_sms * std::max(per_sm, 1);
  const int64_t block_bytes = (int64_t)(kPatThreads / kWarp) * kLists * cap * 4;
  const int64_t fit = std::max<int64_t>(1, (int64_t)kScratchBudget / block_bytes);
  const int grid = (int)std::min(resident, fit);
  *warps = (int64_t)grid * (kPatThreads / kWarp);
  return grid;
}

int pattern_lists() { return kLists; }

namespace {

// P1, P3, P7: centers of degree <= kCenterMaxDeg through the bitmap kernels
// (one launch per class), the edges (and P1 stars) of larger centers
// through pattern_kernel restricted to them.
// Default route per pattern, from timings on a Chung-Lu graph (n 100,000,
// mean degree 10, cap 200) on a B200: the center bitmaps win for P1 (2.1x
// over the warp-per-edge kernel), P2 (1.4x) and P3 (17x).  P7's sets are
// small, so building M costs more than its probes save, and for P4, P5, P6,
// P8 building R(y) for every outer neighbour costs 6-30x more than the
// warp-per-edge kernel's searches.
bool pattern_uses_centers(int pattern) { return pattern == 1 || pattern == 2 || pattern == 3; }

int center_path(mc_dgraph *g, int pattern, PatArgs a, int grid, Slicer *sl) {
  cudaStream_t s = g->stream;
  const int64_t n = g->n;
  // Scratch: class lists (kCenterClasses * n), class counts and queues,
  // big_deg (n), big_off (n + 1), scan temporary.
  const size_t lists_b = sizeof(int32_t) * (size_t)(kCenterClasses * n);
  const size_t words_b = 256;
  const size_t deg_b = sizeof(int32_t) * (size_t)(n + 1);
  const size_t off_b = sizeof(int64_t) * (size_t)(n + 1);
  const size_t temp_b = scan_temp_bytes(n);
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  // P1: per-vertex chunk counts of the large centers and their scan.
  const size_t need = up(lists_b) + words_b + up(deg_b) + up(off_b) + up(temp_b) +
                      (pattern == 1 ? up(deg_b) + up(off_b) : 0);
  if (need > g->center_scratch_bytes) {
    if (g->center_scratch) dev_free(g->center_scratch, s);
    g->center_scratch = nullptr;
    g->center_scratch_bytes = 0;
    MC_CUDA_TRY(dev_alloc(&g->center_scratch, need, s));
    g->center_scratch_bytes = need;
  }
  char *base = static_cast<char *>(g->center_scratch);
  int32_t *lists = reinterpret_cast<int32_t *>(base);
  char *words = base + up(lists_b);
  int32_t *counts = reinterpret_cast<int32_t *>(words);                       // 6 ints
  unsigned long long *queues = reinterpret_cast<unsigned long long *>(words + 64);  // 6 words
  int32_t *big_deg = reinterpret_cast<int32_t *>(words + words_b);
  int64_t *big_off = reinterpret_cast<int64_t *>(reinterpret_cast<char *>(big_deg) + up(deg_b));
  void *temp = reinterpret_cast<char *>(big_off) + up(off_b);

  // Two-hop rows of the outer patterns: 4 GiB of scratch (or a quarter of the
  // free memory, if less) shared out among the resident groups of each class
  // launch.  MERCURY_HOP_ROWS=0: rows per edge only.
  const char *hop_env = std::getenv("MERCURY_HOP_ROWS");
  const bool hop_on = center_outer(pattern) && !(hop_env && std::atoi(hop_env) == 0);
  unsigned long long *hop_walk = reinterpret_cast<unsigned long long *>(words + 128);  // 6 words
  MC_CUDA_TRY(cudaMemsetAsync(words, 0, words_b, s));
  if (hop_on) {
    hop_need_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(g->rowptr, g->col, n, a.shard,
                                                                a.num_shards, hop_walk);
    MC_CUDA_TRY(cudaGetLastError());
    g->launches += 1;
  }
  center_classes_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
      g->rowptr, n, a.shard, a.num_shards, lists, counts, big_deg);
  MC_CUDA_TRY(cudaGetLastError());
  MC_CUDA_TRY(exclusive_scan(big_deg, big_off, n, temp, s));
  g->launches += 1 + scan_launches(n);
  int32_t h_counts[kCenterClasses];
  unsigned long long h_walk[kCenterClasses];
  int64_t big_total = 0;
  MC_CUDA_TRY(cudaMemcpyAsync(h_counts, counts, sizeof(h_counts), cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaMemcpyAsync(h_walk, hop_walk, sizeof(h_walk), cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaMemcpyAsync(&big_total, big_off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  for (int c = 0; c < kCenterClasses; ++c) {
    if (h_counts[c] == 0) continue;
    CenterArgs ca{g->rowptr, g->col, lists + (int64_t)c * n, counts + c, queues + c, g->counters};
    ca.hop_walk = hop_on ? (int64_t)h_walk[c] : 0;
    ca.hop_misses = g->counters + 7;
    ca.deadline = a.deadline;
    ca.stop_flag = a.stop_flag;
    int rc = MC_OK;
    const int64_t tc = h_counts[c];
    switch (pattern) {
      case 1: rc = launch_center_class<1>(g, ca, c, tc, sl); break;
      case 2: rc = launch_center_class<2>(g, ca, c, tc, sl); break;
      case 3: rc = launch_center_class<3>(g, ca, c, tc, sl); break;
      case 4: rc = launch_center_class<4>(g, ca, c, tc, sl); break;
      case 5: rc = launch_center_class<5>(g, ca, c, tc, sl); break;
      case 6: rc = launch_center_class<6>(g, ca, c, tc, sl); break;
      case 7: rc = launch_center_class<7>(g, ca, c, tc, sl); break;
      default: rc = launch_center_class<8>(g, ca, c, tc, sl); break;
    }
    if (rc != MC_OK) return rc;
  }
  // P1 on the larger centers: hub_p1_kernel (MERCURY_HUB_P1=0: the
  // warp-per-edge kernel, as for the other patterns).
  const char *hub_env = std::getenv("MERCURY_HUB_P1");
  if (pattern == 1 && big_total > 0 && !(hub_env && std::atoi(hub_env) == 0)) {
    int32_t *chunks = reinterpret_cast<int32_t *>(reinterpret_cast<char *>(temp) + up(temp_b));
    int64_t *chunk_off = reinterpret_cast<int64_t *>(reinterpret_cast<char *>(chunks) + up(deg_b));
    hub_chunks_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(big_deg, n, chunks);
    MC_CUDA_TRY(cudaGetLastError());
    MC_CUDA_TRY(exclusive_scan(chunks, chunk_off, n, temp, s));
    g->launches += 1 + scan_launches(n);
    int64_t total_chunks = 0;
    MC_CUDA_TRY(cudaMemcpyAsync(&total_chunks, chunk_off + n, sizeof(int64_t),
                                cudaMemcpyDeviceToHost, s));
    MC_CUDA_TRY(cudaStreamSynchronize(s));
    // Grid: every resident CTA, as far as the frontier scratch allows (each
    // warp of this kernel needs cap ints of it, the edge kernel kLists x cap).
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hub_p1_kernel, kPatThreads, 0) !=
            cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    const int hub_grid = (int)std::min<int64_t>((int64_t)g->num_sms * per_sm, (int64_t)grid * kLists);
    // One id bitmap per CTA, zero between tasks (cleared here as well, in
    // case an earlier count stopped at its deadline mid-task).
    const size_t bits_b = sizeof(unsigned) * (size_t)((n + 31) / 32) * (size_t)hub_grid;
    if (bits_b > g->hub_bits_bytes) {
      if (g->hub_bits) dev_free(g->hub_bits, s);
      g->hub_bits = nullptr;
      g->hub_bits_bytes = 0;
      MC_CUDA_TRY(dev_alloc(&g->hub_bits, bits_b, s));
      g->hub_bits_bytes = bits_b;
    }
    MC_CUDA_TRY(cudaMemsetAsync(g->hub_bits, 0, bits_b, s));
    HubP1Args ha{g->rowptr, g->col, n, chunk_off, static_cast<unsigned *>(g->hub_bits),
                 a.scratch, a.cap, g->counters + 3, g->counters, a.shard, a.num_shards,
                 a.deadline, a.stop_flag};
    // MERCURY_HUB_LANE_SCAN: longest range one lane scans alone (0: every
    // range by the whole warp).
    if (const char *env = std::getenv("MERCURY_HUB_LANE_SCAN")) ha.lane_scan = std::max(0, std::atoi(env));
    const int64_t ntasks = total_chunks > a.shard
                               ? (total_chunks - a.shard + a.num_shards - 1) / a.num_shards
                               : 0;
    return run_slices(g, *sl, "hub P1", ntasks, hub_grid, ha.queue, [&](int64_t b, int64_t e) {
      HubP1Args sa = ha;
      sa.task_begin = b;
      sa.task_end = e;
      hub_p1_kernel<<<hub_grid, kPatThreads, 0, s>>>(sa);
      MC_CUDA_TRY(cudaGetLastError());
      g->launches += 1;
      return MC_OK;
    });
  }
  // Larger centers: the warp-per-edge kernel over their edges only.
  a.skip_deg = kCenterMaxDeg;
  if (pattern == 1) {
    int rc = launch_pattern<1, true>(g, a, grid, n, sl);  // stars of degree > kCenterMaxDeg
    if (rc != MC_OK) return rc;
    a.queue = g->counters + 3;
  }
  if (big_total > 0) {
    a.task_off = big_off;
    switch (pattern) {
      case 1: return launch_pattern<1, false>(g, a, grid, big_total, sl);
      case 2: return launch_pattern<2, false>(g, a, grid, big_total, sl);
      case 3: return launch_pattern<3, false>(g, a, grid, big_total, sl);
      case 4: return launch_pattern<4, false>(g, a, grid, big_total, sl);
      case 5: return launch_pattern<5, false>(g, a, grid, big_total, sl);
      case 6: return launch_pattern<6, false>(g, a, grid, big_total, sl);
      case 7: return launch_pattern<7, false>(g, a, grid, big_total, sl);
      default: return launch_pattern<8, false>(g, a, grid, big_total, sl);
    }
  }
  return MC_OK;
}

}  // namespace

// Graphs whose largest degree exceeds this run their pattern launches in
// slices (hub edges can take seconds each; see Slicer).
constexpr int64_t kSliceDegree = 4096;

namespace {
int pattern_count_body(mc_dgraph *g, int pattern, uint64_t *out, uint64_t *c12,
                       mc_timing_t *timing, int shard, int num_shards, double budget_ms,
                       double *progress);

// The pattern scratch (frontier lists, center classes, two-hop rows, hub
// bitmaps) goes back to the stream-ordered pool after every count: a later
// count on any handle reuses it from the pool, and a process that keeps
// thousands of small graphs resident holds their CSRs only.
void release_pattern_scratch(mc_dgraph *g) {
  void **bufs[] = {&g->pat_scratch, &g->center_scratch, &g->hop_scratch, &g->hub_bits};
  size_t *sizes[] = {&g->pat_scratch_bytes, &g->center_scratch_bytes, &g->hop_scratch_bytes,
                     &g->hub_bits_bytes};
  for (int i = 0; i < 4; ++i) {
    if (*bufs[i]) dev_free(*bufs[i], g->stream);
    *bufs[i] = nullptr;
    *sizes[i] = 0;
  }
}
}  // namespace

int pattern_count(mc_dgraph *g, int pattern, uint64_t *out, uint64_t *c12, mc_timing_t *timing,
                  int shard, int num_shards, double budget_ms, double *progress) {
  const int rc = pattern_count_body(g, pattern, out, c12, timing, shard, num_shards, budget_ms,
                                    progress);
  release_pattern_scratch(g);
  return rc;
}

namespace {
int pattern_count_body(mc_dgraph *g, int pattern, uint64_t *out, uint64_t *c12,
                       mc_timing_t *timing, int shard, int num_shards, double budget_ms,
                       double *progress) {
  NvtxRange range("pattern_count");
  if (pattern < 1 || pattern > 8) return MC_ERR_ARG;
  // P7 and P8 on graphs with hubs: by clique counts over the degree-ordered
  // DAG (cliques.cu), which is built first; its time counts as the pattern's.
  bool cliques = false;
  int64_t dag_edges = 0;
  if (pattern == 7 || pattern == 8) {
    MC_CUDA_TRY(cudaEventRecord(g->ev[0], g->stream));
    const int rc = clique_prepare(g, pattern, &cliques, &dag_edges);
    if (rc != MC_OK) return rc;
  }
  // MERCURY_PATTERN_SLICE=1/0 forces slicing on/off (the tests compare both);
  // MERCURY_PATTERN_SLICE_MS sets the target slice length; MERCURY_TRACE_SLICES
  // prints each slice to stderr.
  Slicer sl;
  sl.budget_ms = budget_ms;
  sl.on = budget_ms > 0 || g->max_degree > kSliceDegree;
  if (const char *env = std::getenv("MERCURY_PATTERN_SLICE")) sl.on = std::atoi(env) != 0 || budget_ms > 0;
  if (const char *env = std::getenv("MERCURY_PATTERN_SLICE_MS")) sl.target_ms = std::max(0.01, std::atof(env));
  sl.trace = std::getenv("MERCURY_TRACE_SLICES") != nullptr;
  cudaStream_t s = g->stream;
  const int64_t launches_before = g->launches;
  MC_CUDA_TRY(cudaMemsetAsync(g->counters, 0, sizeof(unsigned long long) * 8, s));
  // The frontier lists hold at most max_degree vertices.
  const int64_t cap = std::max<int64_t>(g->max_degree, 1);
  const int grid = grid_blocks(g, cap);
  const int64_t warps = (int64_t)grid * (kPatThreads / kWarp);
  const size_t need = sizeof(int32_t) * (size_t)(warps * kLists * cap);
  if (need > g->pat_scratch_bytes) {
    if (g->pat_scratch) dev_free(g->pat_scratch, s);
    g->pat_scratch = nullptr;
    g->pat_scratch_bytes = 0;
    MC_CUDA_TRY(dev_alloc(&g->pat_scratch, need, s));
    g->pat_scratch_bytes = need;
  }
  PatArgs a{g->rowptr, g->col, g->n, g->nnz, static_cast<int32_t *>(g->pat_scratch), cap,
            g->counters + 0, g->counters + 2};
  a.shard = shard;
  a.num_shards = num_shards;
  if (budget_ms > 0) {
    // counters[5]: the deadline, counters[6]: the stop flag (zeroed above).
    set_deadline_kernel<<<1, 1, 0, s>>>(g->counters + 5,
                                        (unsigned long long)(budget_ms * 1e6));
    MC_CUDA_TRY(cudaGetLastError());
    a.deadline = g->counters + 5;
    a.stop_flag = g->counters + 6;
    sl.stop_flag = g->counters + 6;
    sl.h_stop = g->h_counters + 6;
    g->h_counters[6] = 0;
  }
  if (const char *env = std::getenv("MERCURY_PATTERN_SETS")) a.use_sets = std::atoi(env) != 0;
  if (!cliques) MC_CUDA_TRY(cudaEventRecord(g->ev[0], s));
  int rc = MC_OK;
  if (cliques) {
    rc = clique_launch(g, pattern, dag_edges, shard, num_shards, a.deadline, a.stop_flag);
  } else if (g->n > 0 && g->nnz > 0) {
    // MERCURY_PATTERN_KERNEL=edge / =centers forces one route for every
    // pattern (the tests run all three settings; timing comparisons use it).
    const char *route = std::getenv("MERCURY_PATTERN_KERNEL");
    bool centers = pattern_uses_centers(pattern);
    if (route && std::strcmp(route, "edge") == 0) centers = false;
    if (route && std::strcmp(route, "centers") == 0) centers = true;
    if (pattern < 1 || pattern > 8) return MC_ERR_ARG;
    const int64_t n = g->n, nnz = g->nnz;
    if (centers) {
      rc = center_path(g, pattern, a, grid, &sl);
    } else {
      switch (pattern) {
        case 1:
          rc = launch_pattern<1, true>(g, a, grid, n, &sl);
          if (rc == MC_OK) {
            a.queue = g->counters + 3;
            rc = launch_pattern<1, false>(g, a, grid, nnz, &sl);
          }
          break;
        case 2: rc = launch_pattern<2, false>(g, a, grid, nnz, &sl); break;
        case 3: rc = launch_pattern<3, false>(g, a, grid, nnz, &sl); break;
        case 4: rc = launch_pattern<4, false>(g, a, grid, nnz, &sl); break;
        case 5: rc = launch_pattern<5, false>(g, a, grid, nnz, &sl); break;
        case 6: rc = launch_pattern<6, false>(g, a, grid, nnz, &sl); break;
        case 7: rc = launch_pattern<7, false>(g, a, grid, nnz, &sl); break;
        default: rc = launch_pattern<8, false>(g, a, grid, nnz, &sl); break;
      }
    }
  }
  if (progress)
    *progress = sl.tasks_total > 0 ? (double)sl.tasks_done / (double)sl.tasks_total : 1.0;
  if (rc != MC_OK) {
    cudaStreamSynchronize(s);  // nothing of this call is left running
    return rc;
  }
  MC_CUDA_TRY(cudaEventRecord(g->ev[3], s));
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_counters, g->counters, sizeof(unsigned long long) * 8,
                              cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  if (sl.trace && g->h_counters[7])
    std::fprintf(stderr, "mercury: %llu centers built their outer rows per edge\n",
                 (unsigned long long)g->h_counters[7]);
  if (budget_ms > 0 && g->h_counters[6]) {  // a kernel stopped early
    if (cliques && progress) *progress = 0.0;  // the clique route keeps no task fraction
    return MC_ERR_TIMEOUT;
  }
  const unsigned long long c1 = g->h_counters[0], c2 = g->h_counters[1];
  *out = (pattern == 4 || pattern == 6) ? c1 : c1 - c2;
  if (c12) {
    c12[0] = c1;
    c12[1] = c2;
  }
  if (timing) {
    std::memset(timing, 0, sizeof(*timing));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev[0], g->ev[3]);
    timing->count_ms = ms;
    timing->total_ms = ms;
    timing->launches = g->launches - launches_before;
  }
  return MC_OK;
}

}  // namespace
}  // namespace mc

extern "C" int mc_pattern_count(mc_dgraph_t *g, int pattern, uint64_t *count, mc_timing_t *timing) {
  return mc_pattern_count_shard(g, pattern, 0, 1, count, timing);
}

extern "C" int mc_pattern_count_shard(mc_dgraph_t *g, int pattern, int shard, int num_shards,
                                      uint64_t *partial, mc_timing_t *timing) {
  if (!g || !partial || pattern < 1 || pattern > 8) return MC_ERR_ARG;
  if (num_shards < 1 || shard < 0 || shard >= num_shards) return MC_ERR_ARG;
  MC_CUDA_TRY(cudaSetDevice(g->device));
  return mc::pattern_count(g, pattern, partial, nullptr, timing, shard, num_shards);
}

extern "C" int mc_pattern_count_budget(mc_dgraph_t *g, int pattern, double budget_ms,
                                       uint64_t *count, double *progress, mc_timing_t *timing) {
  if (!g || !count || pattern < 1 || pattern > 8 || !(budget_ms > 0)) return MC_ERR_ARG;
  MC_CUDA_TRY(cudaSetDevice(g->device));
  return mc::pattern_count(g, pattern, count, nullptr, timing, 0, 1, budget_ms, progress);
}

// ---- pattern count without allocation --------------------------------------
// mc_pattern_count_static: the same kernels as mc_pattern_count over a CSR the
// caller already holds in device memory, with every byte of scratch taken from
// file-scope device arrays instead of cudaMalloc.  The arrays exist once per
// GPU that loads this library and stay until the process exits.
namespace mc {
namespace {

// Frontier lists of all warps: kLists lists of max_degree entries per warp.
constexpr int64_t kStaticFrontierInts = int64_t(8) << 20;  // 32 MiB
static __device__ __align__(256) int32_t g_static_frontier[kStaticFrontierInts];
// [0] c1, [1] c2, [2] star queue, [3] edge queue, [4] max degree, [5] error
static __device__ __align__(256) unsigned long long g_static_words[8];

constexpr int kMaxStaticDevices = 64;
struct StaticScratch {
  int32_t *frontier = nullptr;
  unsigned long long *words = nullptr;
  unsigned long long ctx_id = 0;  // context the addresses belong to (0: none)
};
StaticScratch g_static_scratch[kMaxStaticDevices];
std::mutex g_static_mu;

// Unique id of the calling thread's current CUDA context (0 if none), read
// through the driver entry points the runtime exposes, so the library links
// no driver library.  A device's primary context is destroyed by
// cudaDeviceReset and created anew on the next runtime call; the module
// holding the arrays is then loaded again and their addresses may change.
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext *);
  using GetId = CUresult (*)(CUcontext, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
    void *f1 = nullptr, *f2 = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
      get_current = reinterpret_cast<GetCurrent>(f1);
      get_id = reinterpret_cast<GetId>(f2);
    }
    looked_up = true;
  }
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device addresses of the file-scope arrays on device `dev` (the current
// device).  The host-side names are stand-ins, not device addresses; the
// addresses come from cudaGetSymbolAddress, looked up once per device and
// again whenever the device's context is not the one they were taken in
// (after a cudaDeviceReset, for example).
int static_scratch(int dev, StaticScratch *out) {
  if (dev < 0 || dev >= kMaxStaticDevices) return MC_ERR_UNSUPPORTED;
  // cudaSetDevice makes the device's primary context current (creating it
  // if needed), so the context id below is the one the kernels will use.
  MC_CUDA_TRY(cudaSetDevice(dev));
  const unsigned long long ctx = current_context_id();  // 0: unknown, look up again
  std::lock_guard<std::mutex> lock(g_static_mu);
  StaticScratch &s = g_static_scratch[dev];
  if (!s.frontier || ctx == 0 || s.ctx_id != ctx) {
    MC_CUDA_TRY(cudaGetSymbolAddress((void **)&s.frontier, g_static_frontier));
    MC_CUDA_TRY(cudaGetSymbolAddress((void **)&s.words, g_static_words));
    s.ctx_id = ctx;
  }
  *out = s;
  return MC_OK;
}

template <int P, bool kStar>
int launch_static(cudaStream_t s, const PatArgs &a, int grid) {
  pattern_kernel<P, kStar><<<grid, kPatThreads, 0, s>>>(a);
  MC_CUDA_TRY(cudaGetLastError());
  return MC_OK;
}

}  // namespace
}  // namespace mc

extern "C" int mc_pattern_count_static(const int64_t *d_rowptr, const int32_t *d_col, int64_t n,
                                       int64_t nnz, int pattern, uint64_t *count, void *stream) {
  using namespace mc;
  if (!d_rowptr || (nnz > 0 && !d_col) || !count || n < 0 || nnz < 0) return MC_ERR_ARG;
  if (pattern < 1 || pattern > 8) return MC_ERR_ARG;
  if (n > INT32_MAX - 1) return MC_ERR_UNSUPPORTED;
  int dev = 0;
  MC_CUDA_TRY(cudaGetDevice(&dev));
  StaticScratch sc;
  int rc = static_scratch(dev, &sc);
  if (rc != MC_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // Contract checks (ids in range, sorted rows, no self-loops) and the largest
  // degree, which sizes the frontier lists; both use the static words.
  int64_t max_degree = 0;
  rc = validate_csr_words(d_rowptr, d_col, n, nnz, reinterpret_cast<unsigned *>(sc.words + 5),
                          sc.words + 4, s, &max_degree);
  if (rc != MC_OK) return rc;
  const int64_t cap = std::max<int64_t>(max_degree, 1);
  // Whole blocks of warps that fit in the static frontier array.
  const int64_t per_block = (int64_t)(kPatThreads / kWarp) * kLists * cap;
  const int64_t fit_blocks = kStaticFrontierInts / per_block;
  if (fit_blocks < 1) return MC_ERR_UNSUPPORTED;  // max degree beyond the static capacity
  int dev_sms = 0, per_sm = 0;
  MC_CUDA_TRY(cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, dev));
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pattern_kernel<3, false>, kPatThreads,
                                                    0) != cudaSuccess)
    per_sm = 4;
  const int grid = (int)std::min<int64_t>(fit_blocks, (int64_t)dev_sms * std::max(per_sm, 1));
  // The words keep the previous call's values: the counters and queues must
  // start at zero.
  MC_CUDA_TRY(cudaMemsetAsync(sc.words, 0, sizeof(unsigned long long) * 4, s));
  PatArgs a{d_rowptr, d_col, n, nnz, sc.frontier, cap, sc.words + 0, sc.words + 2};
  if (n > 0 && nnz > 0) {
    switch (pattern) {
      case 1:
        rc = launch_static<1, true>(s, a, grid);
        if (rc == MC_OK) {
          a.queue = sc.words + 3;
          rc = launch_static<1, false>(s, a, grid);
        }
        break;
      case 2: rc = launch_static<2, false>(s, a, grid); break;
      case 3: rc = launch_static<3, false>(s, a, grid); break;
      case 4: rc = launch_static<4, false>(s, a, grid); break;
      case 5: rc = launch_static<5, false>(s, a, grid); break;
      case 6: rc = launch_static<6, false>(s, a, grid); break;
      case 7: rc = launch_static<7, false>(s, a, grid); break;
      default: rc = launch_static<8, false>(s, a, grid); break;
    }
    if (rc != MC_OK) return rc;
  }
  unsigned long long c[2] = {0, 0};
  MC_CUDA_TRY(cudaMemcpyAsync(c, sc.words, sizeof(c), cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  *count = (pattern == 4 || pattern == 6) ? c[0] : c[0] - c[1];
  return MC_OK;
}

// P1..P8 pattern counts on the device.
//
// Reference: subgraph_matching/pattern_kernels.cuh (kernels P1_frequency_count,
// P1_count_correction, P2..P8_subgraph_matching) and the host combine of
// subgraph_matching/sm_multigpu.cu:206-232.  Each kernel walks the 2m
// directed edges (v0, v1) of the symmetric CSR (graph.cc:336-365) with one
// warp per edge, materialises the frontier lists of the pattern in a
// per-warp slice of global scratch and accumulates two 64-bit counters; the
// result is counters[1] for P4/P6 and counters[1] - counters[2] otherwise.
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
#include <cstring>
#include <mutex>

#include "dgraph.cuh"
#include "device_common.cuh"

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

struct Warp {
  const int64_t *__restrict__ rp;
  const int32_t *__restrict__ ci;
  int lane;
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

// freq[j] = #{i > j : a[j] not in N(a[i])}   (P3 :280-292, P7 :386-398)
__device__ void pair_freq(const Warp &w, const int32_t *a, int na, int32_t *freq) {
  for (int j = w.lane; j < na; j += kWarp) {
    const int x = a[j];
    int f = 0;
    for (int i = j + 1; i < na; ++i) f += !w.in(a[i], x);
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
    for (int i = 0; i < nl; ++i) f += !w.in(list[i], x);
    freq[j] = f;
  }
  __syncwarp();
}

// Correction of P3/P7 (:310-340, :417-449): for v2 in A,
// #{(c in A & N(v2), key in A - N(v2), key < v2) : key > c, c not in N(key)}.
__device__ void bounded_correction(const Warp &w, const int32_t *A, int nA, int32_t *D,
                                   int32_t *C, Acc &acc) {
  for (int i = 0; i < nA; ++i) {
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
      const int c = w.count(L0, nA, L0[i], L0[i], false);
      if (w.lane == 0) acc.c1 += wrap_mul(c, L4[i]);
    }
    for (int i = 0; i < nB; ++i) {
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
    for (int i = 0; i < no; ++i) {
      const int v2 = outer[i];
      for (int j = w.lane; j < ni; j += kWarp) acc.c1 += !w.in(v2, inner[j]);
    }
  } else if (P == 5) {  // P5_subgraph_matching (:574-734)
    const int nA = w.inter(n0, d0, v1, -1, L0);
    const int nB = w.diff(n0, d0, v1, -1, L1);
    const int nC = w.diff(n1, d1, v0, -1, L2);
    // freq over B of the A vertices not adjacent to it
    for (int j = w.lane; j < nB; j += kWarp) {
      const int x = L1[j];
      int f = 0;
      for (int i = 0; i < nA; ++i) f += !w.in(L0[i], x);
      L5[j] = f;
    }
    __syncwarp();
    for (int i = 0; i < nB; ++i) {
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
    for (int i = 0; i < nA; ++i) {
      const int v2 = L0[i];
      const int nD = w.diff(L0, nA, v2, -1, L2);
      const int nE = w.diff(L1, nB, v2, -1, L3);
      const int32_t *outer = nD < nE ? L2 : L3, *inner = nD < nE ? L3 : L2;
      const int no = nD < nE ? nD : nE, ni = nD < nE ? nE : nD;
      for (int ii = 0; ii < no; ++ii) {
        const int v3 = outer[ii];
        for (int j = w.lane; j < ni; j += kWarp) acc.c1 += !w.in(v3, inner[j]);
      }
    }
  } else if (P == 7) {  // P7_subgraph_matching (:352-459)
    const int nA = w.inter(n0, d0, v1, -1, L0);
    pair_freq(w, L0, nA, L4);
    for (int i = 0; i < nA; ++i) {
      const int c = w.count(L0, nA, L0[i], L0[i], false);
      if (w.lane == 0) acc.c1 += wrap_mul(c, L4[i]);
    }
    bounded_correction(w, L0, nA, L1, L2, acc);
  } else if (P == 8) {  // P8_subgraph_matching (:461-572)
    const int nA = w.inter(n0, d0, v1, -1, L0);
    const int nB = w.diff(n1, d1, v0, -1, L1);
    cross_freq(w, L0, nA, L1, nB, L4);
    for (int i = 0; i < nA; ++i) {
      const int c = w.count(L0, nA, L0[i], L0[i], true);
      if (w.lane == 0) acc.c1 += wrap_mul(c, L4[i]);
    }
    for (int i = 0; i < nB; ++i) {
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
    for (int j = i + 1; j < d; ++j) f += !w.in(nb[j], x);  // x < nb[j] iff j > i
    freq[i] = f;
  }
  __syncwarp();
  for (int i = 0; i < d; ++i) {
    const int c = w.count(nb, d, nb[i], nb[i], false);
    if (w.lane == 0) acc.c1 += wrap_mul(c, freq[i]);
  }
  __syncwarp();
}

// Persistent warps take directed edges (or, for the P1 star pass, vertices)
// from the queue one at a time.
template <int P, bool kStar>
__global__ void __launch_bounds__(kPatThreads) pattern_kernel(PatArgs a) {
  const int lane = threadIdx.x & (kWarp - 1);
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
  int32_t *L = a.scratch + gw * kLists * a.cap;
  const Warp w{a.rp, a.ci, lane};
  const int64_t ntasks = kStar ? a.n : a.nnz;
  Acc acc;
  for (;;) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(a.queue, 1ull);
    t = __shfl_sync(kFull, t, 0);
    if ((int64_t)t >= ntasks) break;
    if (kStar) {
      vertex_star(w, (int)t, L, acc);
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

template <int P, bool kStar>
int launch_pattern(mc_dgraph *g, const PatArgs &a, int grid) {
  pattern_kernel<P, kStar><<<grid, kPatThreads, 0, g->stream>>>(a);
  MC_CUDA_TRY(cudaGetLastError());
  g->launches += 1;
  return MC_OK;
}

int grid_blocks(mc_dgraph *g, int64_t cap) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pattern_kernel<3, false>, kPatThreads,
                                                    0) != cudaSuccess)
    per_sm = 4;
  const int64_t resident = (int64_t)g->num_sms * std::max(per_sm, 1);
  const int64_t block_bytes = (int64_t)(kPatThreads / kWarp) * kLists * cap * 4;
  const int64_t fit = std::max<int64_t>(1, (int64_t)kScratchBudget / block_bytes);
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
  const int lane = threadIdx.x & (kWarp - 1);
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
  int32_t *L = b.scratch + gw * kLists * b.cap;
  const Warp w{b.rp, b.ci, lane};
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

int pattern_count(mc_dgraph *g, int pattern, uint64_t *out, uint64_t *c12, mc_timing_t *timing) {
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
  MC_CUDA_TRY(cudaEventRecord(g->ev[0], s));
  int rc = MC_OK;
  if (g->n > 0 && g->nnz > 0) {
    switch (pattern) {
      case 1:
        rc = launch_pattern<1, true>(g, a, grid);
        if (rc == MC_OK) {
          a.queue = g->counters + 3;
          rc = launch_pattern<1, false>(g, a, grid);
        }
        break;
      case 2: rc = launch_pattern<2, false>(g, a, grid); break;
      case 3: rc = launch_pattern<3, false>(g, a, grid); break;
      case 4: rc = launch_pattern<4, false>(g, a, grid); break;
      case 5: rc = launch_pattern<5, false>(g, a, grid); break;
      case 6: rc = launch_pattern<6, false>(g, a, grid); break;
      case 7: rc = launch_pattern<7, false>(g, a, grid); break;
      case 8: rc = launch_pattern<8, false>(g, a, grid); break;
      default: return MC_ERR_ARG;
    }
  }
  if (rc != MC_OK) return rc;
  MC_CUDA_TRY(cudaEventRecord(g->ev[3], s));
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_counters, g->counters, sizeof(unsigned long long) * 8,
                              cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaStreamSynchronize(s));
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

}  // namespace mc

extern "C" int mc_pattern_count(mc_dgraph_t *g, int pattern, uint64_t *count, mc_timing_t *timing) {
  if (!g || !count || pattern < 1 || pattern > 8) return MC_ERR_ARG;
  MC_CUDA_TRY(cudaSetDevice(g->device));
  return mc::pattern_count(g, pattern, count, nullptr, timing);
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
  bool ready = false;
};
StaticScratch g_static_scratch[kMaxStaticDevices];
std::mutex g_static_mu;

// Device addresses of the file-scope arrays on device `dev` (the current
// device).  The host-side names are stand-ins, not device addresses; the
// addresses come from cudaGetSymbolAddress, once per device.
int static_scratch(int dev, StaticScratch *out) {
  if (dev < 0 || dev >= kMaxStaticDevices) return MC_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_static_mu);
  StaticScratch &s = g_static_scratch[dev];
  if (!s.ready) {
    MC_CUDA_TRY(cudaGetSymbolAddress((void **)&s.frontier, g_static_frontier));
    MC_CUDA_TRY(cudaGetSymbolAddress((void **)&s.words, g_static_words));
    s.ready = true;
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

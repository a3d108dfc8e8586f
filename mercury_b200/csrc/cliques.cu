// P7 and P8 by clique counts: a second device route for the reference's P7
// and P8 (subgraph_matching/pattern_kernels.cuh:352-459 and :461-572,
// combined as in subgraph_matching/sm_multigpu.cu:206-232) on graphs whose
// hubs make the per-edge formulas cubic in a hub's degree.
//
// P7.  Per directed edge (v0, v1) the formula counts I3(A), the pairwise
// non-adjacent triples of A = N(v0) & N(v1).  By inclusion-exclusion over
// the edges inside A,
//   I3(A) = C(a, 3) - e_A (a - 2) + sum over x in A of C(d_A(x), 2) - t_A,
// with a = |A|, e_A the K4s on the edge, d_A(x) the K4s on the triangle
// {v0, v1, x} and t_A the K5s on the edge.  Summed over both directions of
// every edge (each triangle appears for its three edges, each K5 holds ten):
//   P7 = 2 sum_e C(a_e, 3) - sum_tau k_tau (a_e1 + a_e2 + a_e3 - 6)
//        + 6 sum_tau C(k_tau, 2) - 20 K5,
// k_tau = |N(x) & N(y) & N(z)| for the triangle tau = {x, y, z}.
// P8.  The formula counts each induced tailed K4 (a K4 with a vertex hung on
// one of its vertices alone) three times; inclusion-exclusion over the hung
// vertex's neighbours, summed over every K4, gives
//   P8 = sum_tau k_tau (d_x + d_y + d_z) - 3 sum_tau k_tau (a_e1 + a_e2 + a_e3)
//        + 9 sum_tau k_tau^2 - 60 K5.
// Every term is a sum over edges or triangles, so each is accumulated modulo 2^64
// as the reference's u64 counter is, and shards of the edges sum to the
// whole.  The identity holds while the reference's 32-bit products cannot
// wrap: the route runs only for a maximum degree of at most 46,340.
//
// Triangles are listed once on the degree-ordered DAG (the one the triangle
// count builds): for the DAG edge (u -> v), T = N+(u) & N+(v) in shared
// memory; for w in T, S = T & N+(w) lists the K4s (u, v, w, x) and each
// x in S the K5s (u, v, w, x, y) with y in S & N+(x).  u has the smallest
// degree of its triangle, so k_tau walks N(u).  DAG out-lists are staged in
// shared memory up to kCliqueMaxOut entries; the host sends larger graphs to
// the formula route.
#include <climits>
#include <cstdlib>
#include <cstring>

#include "dgraph.cuh"
#include "device_common.cuh"

namespace mc {
namespace {

constexpr int kCliqueWarps = 4;  // warps per CTA of the triangle kernel
constexpr int kCliqueClaim = 4;  // DAG edges claimed per queue atomic

struct CliqueArgs {
  const int64_t *__restrict__ rowptr;  // symmetric CSR
  const int32_t *__restrict__ col;
  const int64_t *__restrict__ drp;  // DAG rows (ascending)
  const int32_t *__restrict__ dcol;
  int64_t n, m;  // vertices, DAG edges
  int32_t *tri;  // triangles per DAG edge (the edge kernel writes them)
  unsigned long long *acc;    // the count, modulo 2^64
  unsigned long long *queue;  // claims of the running kernel
  int shard, num_shards;
  const unsigned long long *deadline;  // budgeted count: globaltimer ns, or null
  unsigned long long *stop_flag;
  int pattern;  // 7 or 8
};

__device__ __forceinline__ unsigned long long clique_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Warp-uniform: past the deadline (lane 0's clock), raise the flag.
__device__ __forceinline__ bool clique_late(const CliqueArgs &a, int lane) {
  if (!a.deadline) return false;
  unsigned long long t = lane == 0 ? clique_ns() : 0ull;
  t = __shfl_sync(kFull, t, 0);
  const bool late = t > *a.deadline;
  if (late && lane == 0) atomicOr(a.stop_flag, 1ull);
  return late;
}

// First index of a sorted list holding a value >= x (len if none).
__device__ __forceinline__ int lower_index(const int32_t *__restrict__ p, int len, int32_t x) {
  int lo = 0, hi = len;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(p + mid) < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ bool in_sorted(const int32_t *__restrict__ p, int len, int32_t x) {
  const int i = lower_index(p, len, x);
  return i < len && __ldg(p + i) == x;
}

__device__ __forceinline__ int warp_sum_int(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ unsigned long long choose2(unsigned long long k) {
  return k < 2 ? 0ull : k * (k - 1) / 2;
}

__device__ __forceinline__ unsigned long long choose3(unsigned long long k) {
  return k < 3 ? 0ull : k * (k - 1) / 2 * (k - 2) / 3;
}

// The DAG edge queue position t of this shard -> DAG edge index.
__device__ __forceinline__ int64_t shard_edge(const CliqueArgs &a, unsigned long long t) {
  return (int64_t)t * a.num_shards + a.shard;
}

// Triangles per DAG edge (u -> v): a = |N(u) & N(v)| over the symmetric rows,
// by walking the shorter row and searching the longer (warp per edge, every
// edge: the triangle kernel reads the counts of all three edges of its
// triangles).  For P7, edges of this shard add 2 C(a, 3).
__global__ void __launch_bounds__(256) clique_edge_kernel(CliqueArgs a) {
  const int lane = threadIdx.x & (kWarp - 1);
  unsigned long long mine = 0;
  for (;;) {
    unsigned long long t0 = 0;
    if (lane == 0) t0 = atomicAdd(a.queue, (unsigned long long)kCliqueClaim);
    t0 = __shfl_sync(kFull, t0, 0);
    if ((int64_t)t0 >= a.m || clique_late(a, lane)) break;
    for (int c = 0; c < kCliqueClaim; ++c) {
      const int64_t i = (int64_t)t0 + c;
      if (i >= a.m) break;
      const int64_t u = upper_row(a.drp, 0, a.n - 1, i);
      const int32_t v = __ldg(a.dcol + i);
      const int64_t bu = a.rowptr[u], du = a.rowptr[u + 1] - bu;
      const int64_t bv = a.rowptr[v], dv = a.rowptr[v + 1] - bv;
      const bool u_short = du <= dv;
      const int32_t *ps = a.col + (u_short ? bu : bv), *pl = a.col + (u_short ? bv : bu);
      const int ls = (int)(u_short ? du : dv), ll = (int)(u_short ? dv : du);
      int hits = 0;
      for (int k = lane; k < ls; k += kWarp) hits += in_sorted(pl, ll, __ldg(ps + k));
      hits = warp_sum_int(hits);
      if (lane == 0) {
        a.tri[i] = hits;
        if (a.pattern == 7 && i % a.num_shards == a.shard)
          mine += 2ull * choose3((unsigned long long)hits);
      }
    }
  }
  if (lane == 0 && mine) atomicAdd(a.acc, mine);
}

// The triangle terms of this shard's DAG edges (u -> v): for each w in
// T = N+(u) & N+(v), the triangle's k = |N(u) & N(v) & N(w)|, its edges'
// triangle counts, its vertices' degrees (P8) and the K5s on it as the
// first three of their DAG order.
__global__ void __launch_bounds__(kCliqueWarps * kWarp) clique_triangle_kernel(CliqueArgs a) {
  __shared__ int32_t s_t[kCliqueWarps][kCliqueMaxOut];
  __shared__ int32_t s_s[kCliqueWarps][kCliqueMaxOut];
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x / kWarp;
  int32_t *T = s_t[warp], *S = s_s[warp];
  const unsigned below = (1u << lane) - 1u;
  const int64_t edges = a.m > a.shard ? (a.m - a.shard + a.num_shards - 1) / a.num_shards : 0;
  unsigned long long mine = 0;  // lane 0's sum, modulo 2^64
  for (;;) {
    unsigned long long t0 = 0;
    if (lane == 0) t0 = atomicAdd(a.queue, (unsigned long long)kCliqueClaim);
    t0 = __shfl_sync(kFull, t0, 0);
    if ((int64_t)t0 >= edges || clique_late(a, lane)) break;
    for (int c = 0; c < kCliqueClaim; ++c) {
      if ((int64_t)(t0 + c) >= edges) break;
      const int64_t i = shard_edge(a, t0 + c);
      const int64_t u = upper_row(a.drp, 0, a.n - 1, i);
      const int32_t v = __ldg(a.dcol + i);
      const int32_t *ou = a.dcol + a.drp[u], *ov = a.dcol + a.drp[v];
      const int lu = (int)(a.drp[u + 1] - a.drp[u]), lv = (int)(a.drp[v + 1] - a.drp[v]);
      // T = N+(u) & N+(v), in ascending order (lu <= kCliqueMaxOut).
      int nt = 0;
      for (int base = 0; base < lu; base += kWarp) {
        const int k = base + lane;
        const int32_t x = k < lu ? __ldg(ou + k) : 0;
        const bool hit = k < lu && in_sorted(ov, lv, x);
        const unsigned mask = __ballot_sync(kFull, hit);
        if (hit) T[nt + __popc(mask & below)] = x;
        nt += __popc(mask);
      }
      __syncwarp();
      if (nt == 0) continue;
      const long long a_uv = __ldg(a.tri + i);
      const int32_t *nu = a.col + a.rowptr[u];
      const int du = (int)(a.rowptr[u + 1] - a.rowptr[u]);
      const int32_t *nv = a.col + a.rowptr[v];
      const int dv = (int)(a.rowptr[v + 1] - a.rowptr[v]);
      for (int j = 0; j < nt; ++j) {
        const int32_t w = T[j];
        const int32_t *nw = a.col + a.rowptr[w];
        const int dw = (int)(a.rowptr[w + 1] - a.rowptr[w]);
        const int32_t *ow = a.dcol + a.drp[w];
        const int lw = (int)(a.drp[w + 1] - a.drp[w]);
        // k = |N(u) & N(v) & N(w)| (u has the smallest degree of the three).
        int kt = 0;
        for (int k = lane; k < du; k += kWarp) {
          const int32_t y = __ldg(nu + k);
          kt += in_sorted(nv, dv, y) && in_sorted(nw, dw, y);
        }
        kt = warp_sum_int(kt);
        // S = T & N+(w): the K4s (u, v, w, x).
        int ns = 0;
        for (int base = 0; base < nt; base += kWarp) {
          const int k = base + lane;
          const int32_t x = k < nt ? T[k] : 0;
          const bool hit = k < nt && in_sorted(ow, lw, x);
          const unsigned mask = __ballot_sync(kFull, hit);
          if (hit) S[ns + __popc(mask & below)] = x;
          ns += __popc(mask);
        }
        __syncwarp();
        // K5s (u, v, w, x, y): y in S & N+(x).
        int k5 = 0;
        for (int q = 0; q < ns; ++q) {
          const int32_t x = S[q];
          const int32_t *ox = a.dcol + a.drp[x];
          const int lx = (int)(a.drp[x + 1] - a.drp[x]);
          for (int k = lane; k < ns; k += kWarp) k5 += in_sorted(ox, lx, S[k]);
        }
        k5 = warp_sum_int(k5);
        __syncwarp();  // S is rewritten for the next w
        if (lane == 0) {
          const long long a_uw = __ldg(a.tri + a.drp[u] + lower_index(ou, lu, w));
          const long long a_vw = __ldg(a.tri + a.drp[v] + lower_index(ov, lv, w));
          const long long k = kt, sum_a = a_uv + a_uw + a_vw;
          if (a.pattern == 7) {
            mine += 6ull * choose2((unsigned long long)k);
            mine -= (unsigned long long)(k * (sum_a - 6));
            mine -= 20ull * (unsigned long long)k5;
          } else {
            mine += (unsigned long long)(k * ((long long)du + dv + dw));
            mine -= (unsigned long long)(3 * k * sum_a);
            mine += (unsigned long long)(9 * k * k);
            mine -= 60ull * (unsigned long long)k5;
          }
        }
      }
      __syncwarp();  // T is rewritten for the next edge
    }
  }
  if (lane == 0 && mine) atomicAdd(a.acc, mine);
}

int resident(const void *kernel, int threads) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess)
    per_sm = 1;
  return per_sm < 1 ? 1 : per_sm;
}

}  // namespace

// MERCURY_CLIQUE_ROUTE=cliques sends P7 and P8 here whenever the graph
// allows it, =formula never; unset, they take this route on graphs with a
// vertex of degree above 4,096 (where the formulas' per-edge loops do not
// finish), unless MERCURY_PATTERN_KERNEL forces a formula route.  The
// degree-ordered DAG is built here; *use is false when the graph does not
// allow the route (a degree above 46,340, where the reference's products
// wrap, or a DAG out-list longer than kCliqueMaxOut).
int clique_prepare(mc_dgraph *g, int pattern, bool *use, int64_t *dag_edges) {
  *use = false;
  *dag_edges = 0;
  if (pattern != 7 && pattern != 8) return MC_OK;
  const char *env = std::getenv("MERCURY_CLIQUE_ROUTE");
  const bool forced = env && std::strcmp(env, "cliques") == 0;
  if (env && std::strcmp(env, "formula") == 0) return MC_OK;
  if (!forced && (std::getenv("MERCURY_PATTERN_KERNEL") || g->max_degree <= 4096)) return MC_OK;
  if (g->max_degree > 46340 || g->n == 0 || g->nnz == 0 || g->batch.gid) return MC_OK;
  int rc = tc_alloc(g);
  if (rc != MC_OK) return rc;
  rc = tc_orient(g);
  if (rc != MC_OK) return rc;
  cudaStream_t s = g->stream;
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_counters + 3, g->counters + 3, sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_err, g->err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  int64_t edges = 0;  // the DAG's entries as written (not assumed from nnz)
  MC_CUDA_TRY(cudaMemcpyAsync(&edges, g->dag_rowptr + g->n, sizeof(int64_t),
                              cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  if (*g->h_err & (kErrDagCapacity | kErrContract)) return MC_ERR_FORMAT;
  *use = g->h_counters[3] <= (unsigned long long)kCliqueMaxOut && edges > 0;
  *dag_edges = edges;
  return MC_OK;
}

// Adds P7 or P8 of this shard's DAG edges to counters[0] (zeroed by the
// caller, with counters[2] and counters[3], the kernels' queues).  The DAG
// and its m entries come from clique_prepare.
int clique_launch(mc_dgraph *g, int pattern, int64_t m, int shard, int num_shards,
                  const unsigned long long *deadline, unsigned long long *stop_flag) {
  NvtxRange range("clique_patterns");
  cudaStream_t s = g->stream;
  int32_t *tri = nullptr;
  MC_CUDA_TRY(dev_alloc(reinterpret_cast<void **>(&tri), sizeof(int32_t) * (size_t)(m + 1), s));
  CliqueArgs a{g->rowptr, g->col, g->dag_rowptr, g->dag_col, g->n, m, tri,
               g->counters + 0, g->counters + 2, shard, num_shards, deadline, stop_flag,
               pattern};
  const int edge_grid = g->num_sms * resident((const void *)clique_edge_kernel, 256);
  clique_edge_kernel<<<edge_grid, 256, 0, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    a.queue = g->counters + 3;
    const int tri_grid =
        g->num_sms * resident((const void *)clique_triangle_kernel, kCliqueWarps * kWarp);
    clique_triangle_kernel<<<tri_grid, kCliqueWarps * kWarp, 0, s>>>(a);
    e = cudaGetLastError();
  }
  dev_free(tri, s);
  g->launches += 2;
  MC_CUDA_TRY(e);
  return MC_OK;
}

}  // namespace mc

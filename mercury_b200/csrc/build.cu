// Device CSR construction from an edge list: the work of the reference's
// dataset converter (datasets/converter.sh:5, a closed binary) and of the
// networkx step in datasets/tsv2mtx.py:13, redone on the GPU.
//
// 1. Each pair (u, v) becomes two packed keys (u << col_bits | v) and
//    (v << col_bits | u); a self-loop becomes two "dead" keys whose row field
//    is n, so they sort after every real entry.
// 2. An LSD radix sort orders the keys, 8 bits per pass, over exactly the
//    bits the packing uses (2 * ceil(log2 n) + 1 bits).
// 3. One pass drops the dead keys and the duplicates, writes the column array
//    and adds each row's entry count into a degree array; a scan of the
//    degrees gives the row offsets.
//
// Every pass streams the keys through HBM with coalesced loads; the radix
// scatter stages each 4096-key tile in shared memory so that the stores to
// each digit's bucket are contiguous.
#include <algorithm>
#include <cstring>
#include <new>

#include "dgraph.cuh"
#include "device_common.cuh"
#include "mc_internal.h"
#include "radix.cuh"
#include "scan.cuh"

namespace mc {

namespace {

using u64 = unsigned long long;

// Pairs -> packed keys, two per pair.
__global__ void edge_keys_kernel(const int32_t *__restrict__ src, const int32_t *__restrict__ dst,
                                 int64_t m, int64_t n, int col_bits, ulonglong2 *__restrict__ keys,
                                 unsigned *err) {
  const u64 dead = (u64)n << col_bits;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
    const int32_t u = __ldg(src + i), v = __ldg(dst + i);
    ulonglong2 k = make_ulonglong2(dead, dead);
    if (u < 0 || v < 0 || u >= n || v >= n) {
      atomicOr(err, kErrIdRange);
    } else if (u != v) {
      k.x = ((u64)u << col_bits) | (u64)(uint32_t)v;
      k.y = ((u64)v << col_bits) | (u64)(uint32_t)u;
    }
    keys[i] = k;
  }
}

// Per-lane view of the sorted keys used by the two duplicate passes.
struct KeyRound {
  bool valid;   // a real entry (not past the end, not a dead key)
  bool fresh;   // valid and different from the previous key
};

__device__ __forceinline__ KeyRound classify(const u64 *__restrict__ keys, int64_t i,
                                             int64_t count, u64 key, u64 dead, int lane,
                                             u64 carry, bool have_carry) {
  // The previous key comes from the lane below; lane 0 takes the previous
  // round's lane 31 (carry) or, at a warp's first key, reads it from memory.
  u64 prev = __shfl_up_sync(kFull, key, 1);
  if (lane == 0) prev = have_carry ? carry : (i > 0 && i < count ? __ldg(keys + i - 1) : ~0ull);
  KeyRound kr;
  kr.valid = i < count && key < dead;
  kr.fresh = kr.valid && (i == 0 || prev != key);
  return kr;
}

// Distinct real entries per tile.
__global__ void __launch_bounds__(kSortThreads) unique_count_kernel(const u64 *__restrict__ keys,
                                                                    int64_t count, u64 dead,
                                                                    int32_t *__restrict__ tile_counts) {
  __shared__ int total;
  if (threadIdx.x == 0) total = 0;
  __syncthreads();
  const int lane = threadIdx.x & (kWarp - 1), w = threadIdx.x / kWarp;
  const int64_t first = (int64_t)blockIdx.x * kSortTile + (int64_t)w * kWarpSpan + lane;
  u64 k[kSortRounds];
  load_warp_keys(keys, count, first, k);
  int c = 0;
  u64 carry = 0;
#pragma unroll
  for (int r = 0; r < kSortRounds; ++r) {
    const KeyRound kr = classify(keys, first + r * kWarp, count, k[r], dead, lane, carry, r > 0);
    c += __popc(__ballot_sync(kFull, kr.fresh));
    carry = __shfl_sync(kFull, k[r], kWarp - 1);
  }
  if (lane == 0) atomicAdd(&total, c);
  __syncthreads();
  if (threadIdx.x == 0) tile_counts[blockIdx.x] = total;
}

// Writes the distinct entries' columns and the row entry counts.
// Entry counts: a row's keys inside one warp's 512-key span form a piece;
// its first key adds -p(first) and its last key adds p(last) + fresh(last)
// to deg[row], where p(i) is the number of distinct entries before key i.
// Summed over a row's pieces this is the row's distinct entry count, with
// two atomics per piece instead of one per entry.
__global__ void __launch_bounds__(kSortThreads) unique_emit_kernel(
    const u64 *__restrict__ keys, int64_t count, u64 dead, int col_bits,
    const int64_t *__restrict__ tile_off, int32_t *__restrict__ col, u64 *__restrict__ deg) {
  __shared__ int warp_tot[kSortWarps];
  const int lane = threadIdx.x & (kWarp - 1), w = threadIdx.x / kWarp;
  const int64_t first = (int64_t)blockIdx.x * kSortTile + (int64_t)w * kWarpSpan + lane;
  u64 k[kSortRounds];
  unsigned fresh_bits[kSortRounds];
  load_warp_keys(keys, count, first, k);
  int c = 0;
  u64 carry = 0;
#pragma unroll
  for (int r = 0; r < kSortRounds; ++r) {
    const KeyRound kr = classify(keys, first + r * kWarp, count, k[r], dead, lane, carry, r > 0);
    fresh_bits[r] = __ballot_sync(kFull, kr.fresh);
    c += __popc(fresh_bits[r]);
    carry = __shfl_sync(kFull, k[r], kWarp - 1);
  }
  if (lane == 0) warp_tot[w] = c;
  __syncthreads();
  int64_t p = tile_off[blockIdx.x];
  for (int x = 0; x < w; ++x) p += warp_tot[x];
  const unsigned lt = lanemask_lt();
  const u64 col_mask = (1ull << col_bits) - 1;
#pragma unroll
  for (int r = 0; r < kSortRounds; ++r) {
    const int64_t i = first + r * kWarp;
    const u64 key = k[r];
    const bool valid = i < count && key < dead;
    const bool fresh = (fresh_bits[r] >> lane) & 1u;
    const int64_t pi = p + __popc(fresh_bits[r] & lt);
    if (fresh) col[pi] = (int32_t)(key & col_mask);
    const u64 row = key >> col_bits;
    // Piece boundaries: neighbours in the same warp span with another row.
    // (All lanes take part in every shuffle; lane 0 / lane 31 then pick.)
    u64 prev_row = __shfl_up_sync(kFull, row, 1);
    const u64 prev_lane31 = __shfl_sync(kFull, k[r > 0 ? r - 1 : 0], kWarp - 1) >> col_bits;
    if (lane == 0) prev_row = r > 0 ? prev_lane31 : ~0ull;
    u64 next_row = __shfl_down_sync(kFull, row, 1);
    const u64 next_lane0 = __shfl_sync(kFull, k[r + 1 < kSortRounds ? r + 1 : r], 0) >> col_bits;
    if (lane == kWarp - 1) next_row = r + 1 < kSortRounds ? next_lane0 : ~0ull;
    if (i + 1 >= count) next_row = ~0ull;
    const bool is_first = valid && prev_row != row;
    const bool is_last = valid && next_row != row;
    if (is_first || is_last) {
      u64 delta = 0;
      if (is_last) delta += (u64)pi + (fresh ? 1ull : 0ull);
      if (is_first) delta -= (u64)pi;
      atomicAdd(deg + row, delta);
    }
    p += __popc(fresh_bits[r]);
  }
}

__global__ void max_degree_kernel(const u64 *__restrict__ deg, int64_t n,
                                  unsigned long long *__restrict__ out) {
  u64 m = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
    m = max(m, deg[v]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(kFull, m, o));
  if ((threadIdx.x & (kWarp - 1)) == 0) atomicMax(out, m);
}

unsigned stream_grid(int64_t items, int threads, int num_sms) {
  const int64_t want = (items + threads - 1) / threads;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)num_sms * 8));
}

}  // namespace

struct CsrBuild {
  cudaStream_t s = nullptr;
  int num_sms = 148;
  int64_t m = 0, n = 0, count = 0, tiles = 0;
  int col_bits = 1, key_bits = 2;
  const int32_t *src = nullptr, *dst = nullptr;  // device pairs (input or owned copy)
  int32_t *own_src = nullptr, *own_dst = nullptr;
  u64 *keys[2] = {nullptr, nullptr};
  int cur = 0;                       // keys[cur] holds the sorted keys
  int32_t *counts = nullptr;         // kRadixBins * tiles (then tiles) counters
  int64_t *offsets = nullptr;        // their exclusive scan
  void *temp = nullptr;              // scan scratch
  u64 *deg = nullptr;                // n entry counts
  unsigned *flags = nullptr;         // [0] error bits, [2..3] max degree (u64)
  unsigned *h_flags = nullptr;       // host mirror: err, pad, max degree, total
  int64_t launches = 0;
};

int csr_build_create(int64_t m, int64_t n, cudaStream_t s, CsrBuild **out) {
  *out = nullptr;
  if (m < 0 || n < 0) return MC_ERR_ARG;
  if (n > (int64_t)INT32_MAX - 1) return MC_ERR_UNSUPPORTED;
  CsrBuild *b = new (std::nothrow) CsrBuild();
  if (!b) return MC_ERR_OOM;
  *out = b;
  b->s = s;
  b->m = m;
  b->n = n;
  b->count = 2 * m;
  b->tiles = (b->count + kSortTile - 1) / kSortTile;
  b->col_bits = std::max(1, bit_width(n > 0 ? (uint64_t)(n - 1) : 0));
  b->key_bits = b->col_bits + bit_width((uint64_t)n);  // the row field also holds n
  int dev = 0;
  MC_CUDA_TRY(cudaGetDevice(&dev));
  MC_CUDA_TRY(cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, dev));
  retain_pool_memory(dev);
  b->h_flags = new (std::nothrow) unsigned[8]();
  if (!b->h_flags) return MC_ERR_OOM;
  MC_CUDA_TRY(dev_alloc((void **)&b->flags, sizeof(unsigned) * 4, s));
  MC_CUDA_TRY(dev_alloc((void **)&b->deg, sizeof(u64) * (size_t)std::max<int64_t>(n, 1), s));
  if (b->count > 0) {
    MC_CUDA_TRY(dev_alloc((void **)&b->keys[0], sizeof(u64) * (size_t)b->count, s));
    MC_CUDA_TRY(dev_alloc((void **)&b->keys[1], sizeof(u64) * (size_t)b->count, s));
    const int64_t entries = (int64_t)kRadixBins * b->tiles;
    MC_CUDA_TRY(dev_alloc((void **)&b->counts, sizeof(int32_t) * (size_t)entries, s));
    MC_CUDA_TRY(dev_alloc((void **)&b->offsets, sizeof(int64_t) * (size_t)(entries + 1), s));
  }
  const int64_t scan_max = std::max<int64_t>((int64_t)kRadixBins * b->tiles, n);
  MC_CUDA_TRY(dev_alloc(&b->temp, scan_temp_bytes(scan_max), s));
  return MC_OK;
}

int csr_build_input(CsrBuild *b, const int32_t *src, const int32_t *dst, bool device_input) {
  if (b->m == 0) return MC_OK;
  if (device_input) {
    b->src = src;
    b->dst = dst;
    return MC_OK;
  }
  const size_t bytes = sizeof(int32_t) * (size_t)b->m;
  MC_CUDA_TRY(dev_alloc((void **)&b->own_src, bytes, b->s));
  MC_CUDA_TRY(dev_alloc((void **)&b->own_dst, bytes, b->s));
  MC_CUDA_TRY(cudaMemcpyAsync(b->own_src, src, bytes, cudaMemcpyHostToDevice, b->s));
  MC_CUDA_TRY(cudaMemcpyAsync(b->own_dst, dst, bytes, cudaMemcpyHostToDevice, b->s));
  b->src = b->own_src;
  b->dst = b->own_dst;
  return MC_OK;
}

int csr_build_sort(CsrBuild *b, int64_t *nnz) {
  NvtxRange range("csr_build_sort");
  cudaStream_t s = b->s;
  MC_CUDA_TRY(cudaMemsetAsync(b->flags, 0, sizeof(unsigned) * 4, s));
  *nnz = 0;
  if (b->count == 0) return MC_OK;
  const u64 dead = (u64)b->n << b->col_bits;
  edge_keys_kernel<<<stream_grid(b->m, 256, b->num_sms), 256, 0, s>>>(
      b->src, b->dst, b->m, b->n, b->col_bits, reinterpret_cast<ulonglong2 *>(b->keys[0]),
      b->flags);
  MC_CUDA_TRY(cudaGetLastError());
  ++b->launches;
  b->cur = 0;
  u64 *sorted = nullptr;
  MC_CUDA_TRY(radix_sort_u64(b->keys[0], b->keys[1], b->count, 0, b->key_bits, b->counts,
                             b->offsets, b->temp, s, &sorted, &b->launches));
  b->cur = sorted == b->keys[0] ? 0 : 1;
  const unsigned grid = (unsigned)b->tiles;
  unique_count_kernel<<<grid, kSortThreads, 0, s>>>(b->keys[b->cur], b->count, dead, b->counts);
  MC_CUDA_TRY(cudaGetLastError());
  MC_CUDA_TRY(exclusive_scan(b->counts, b->offsets, b->tiles, b->temp, s));
  b->launches += 1 + scan_launches(b->tiles);
  MC_CUDA_TRY(cudaMemcpyAsync(b->h_flags, b->flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaMemcpyAsync(b->h_flags + 4, b->offsets + b->tiles, sizeof(int64_t),
                              cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  if (b->h_flags[0] & kErrIdRange) return MC_ERR_FORMAT;
  int64_t total = 0;
  std::memcpy(&total, b->h_flags + 4, sizeof(total));
  *nnz = total;
  return MC_OK;
}

int csr_build_emit(CsrBuild *b, int64_t *rowptr, int32_t *col, int64_t *max_degree) {
  NvtxRange range("csr_build_emit");
  cudaStream_t s = b->s;
  *max_degree = 0;
  if (b->n == 0) {
    MC_CUDA_TRY(cudaMemsetAsync(rowptr, 0, sizeof(int64_t), s));
    MC_CUDA_TRY(cudaStreamSynchronize(s));
    return MC_OK;
  }
  MC_CUDA_TRY(cudaMemsetAsync(b->deg, 0, sizeof(u64) * (size_t)b->n, s));
  if (b->count > 0) {
    unique_emit_kernel<<<(unsigned)b->tiles, kSortThreads, 0, s>>>(
        b->keys[b->cur], b->count, (u64)b->n << b->col_bits, b->col_bits, b->offsets, col, b->deg);
    MC_CUDA_TRY(cudaGetLastError());
    ++b->launches;
  }
  MC_CUDA_TRY(exclusive_scan(reinterpret_cast<const int64_t *>(b->deg), rowptr, b->n, b->temp, s));
  u64 *d_max = reinterpret_cast<u64 *>(b->flags + 2);
  max_degree_kernel<<<stream_grid(b->n, 256, b->num_sms), 256, 0, s>>>(b->deg, b->n, d_max);
  MC_CUDA_TRY(cudaGetLastError());
  b->launches += 1 + scan_launches(b->n);
  u64 h_max = 0;
  MC_CUDA_TRY(cudaMemcpyAsync(b->h_flags + 2, d_max, sizeof(u64), cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  std::memcpy(&h_max, b->h_flags + 2, sizeof(h_max));
  *max_degree = (int64_t)h_max;
  return MC_OK;
}

int64_t csr_build_launches(const CsrBuild *b) { return b ? b->launches : 0; }

void csr_build_free(CsrBuild *b) {
  if (!b) return;
  void *bufs[] = {b->own_src, b->own_dst, b->keys[0], b->keys[1], b->counts,
                  b->offsets, b->temp,    b->deg,     b->flags};
  for (void *p : bufs)
    if (p) dev_free(p, b->s);
  cudaStreamSynchronize(b->s);
  delete[] b->h_flags;
  delete b;
}

}  // namespace mc

namespace {

// Resources of one mc_csr_build call, released on every exit path.
struct HostBuildCall {
  cudaStream_t s = nullptr;
  bool own_stream = false;
  cudaEvent_t ev[4] = {};
  mc::CsrBuild *b = nullptr;
  int64_t *rowptr = nullptr;
  int32_t *col = nullptr;
  ~HostBuildCall() {
    if (rowptr) mc::dev_free(rowptr, s);
    if (col) mc::dev_free(col, s);
    mc::csr_build_free(b);
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
    if (own_stream && s) cudaStreamDestroy(s);
  }
};

float span_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  return cudaEventElapsedTime(&ms, a, b) == cudaSuccess ? ms : 0.f;
}

}  // namespace

extern "C" int mc_csr_build(const int32_t *src, const int32_t *dst, int64_t num_edges, int64_t n,
                            unsigned flags, void *stream, mc_graph_t **out, mc_timing_t *timing) {
  mc::NvtxRange range("mc_csr_build");
  if (!out || num_edges < 0 || n < 0 || (num_edges > 0 && (!src || !dst))) return MC_ERR_ARG;
  *out = nullptr;
  if (timing) std::memset(timing, 0, sizeof(*timing));
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MC_ERR_NO_DEVICE;
  HostBuildCall c;
  if (stream) {
    c.s = static_cast<cudaStream_t>(stream);
  } else {
    MC_CUDA_TRY(cudaStreamCreateWithFlags(&c.s, cudaStreamNonBlocking));
    c.own_stream = true;
  }
  for (cudaEvent_t &e : c.ev) MC_CUDA_TRY(cudaEventCreate(&e));
  int rc = mc::csr_build_create(num_edges, n, c.s, &c.b);
  if (rc != MC_OK) return rc;
  MC_CUDA_TRY(cudaEventRecord(c.ev[0], c.s));
  rc = mc::csr_build_input(c.b, src, dst, (flags & MC_BUILD_DEVICE_INPUT) != 0);
  if (rc != MC_OK) return rc;
  MC_CUDA_TRY(cudaEventRecord(c.ev[1], c.s));
  int64_t nnz = 0, max_degree = 0;
  rc = mc::csr_build_sort(c.b, &nnz);
  if (rc != MC_OK) return rc;
  MC_CUDA_TRY(mc::dev_alloc((void **)&c.rowptr, sizeof(int64_t) * (size_t)(n + 1), c.s));
  MC_CUDA_TRY(mc::dev_alloc((void **)&c.col, sizeof(int32_t) * (size_t)std::max<int64_t>(nnz, 1), c.s));
  rc = mc::csr_build_emit(c.b, c.rowptr, c.col, &max_degree);
  if (rc != MC_OK) return rc;
  MC_CUDA_TRY(cudaEventRecord(c.ev[2], c.s));
  mc_graph *g = new (std::nothrow) mc_graph();
  if (!g) return MC_ERR_OOM;
  try {
    g->rowptr.resize((size_t)n + 1);
    g->col.resize((size_t)nnz);
  } catch (const std::bad_alloc &) {
    delete g;
    return MC_ERR_OOM;
  }
  g->n = n;
  g->nnz = nnz;
  g->max_degree = max_degree;
  cudaError_t e = cudaMemcpyAsync(g->rowptr.data(), c.rowptr, sizeof(int64_t) * (size_t)(n + 1),
                                  cudaMemcpyDeviceToHost, c.s);
  if (e == cudaSuccess && nnz > 0)
    e = cudaMemcpyAsync(g->col.data(), c.col, sizeof(int32_t) * (size_t)nnz,
                        cudaMemcpyDeviceToHost, c.s);
  if (e == cudaSuccess) e = cudaEventRecord(c.ev[3], c.s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.s);
  if (e != cudaSuccess) {
    delete g;
    mc::set_last_cuda_error(e);
    return e == cudaErrorMemoryAllocation ? MC_ERR_OOM : MC_ERR_CUDA;
  }
  if (timing) {
    timing->h2d_ms = span_ms(c.ev[0], c.ev[1]);
    timing->count_ms = span_ms(c.ev[1], c.ev[2]);
    timing->d2h_ms = span_ms(c.ev[2], c.ev[3]);
    timing->total_ms = span_ms(c.ev[0], c.ev[3]);
    timing->launches = mc::csr_build_launches(c.b);
  }
  *out = g;
  return MC_OK;
}

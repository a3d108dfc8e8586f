// Stable LSD radix sort of 64-bit keys (reduce-then-scan per pass): an
// upsweep writes every tile's digit histogram digit-major, one exclusive scan
// turns the histograms into each (digit, tile) run's first output slot, and a
// downsweep ranks the tile's keys stably, stages them in shared memory in
// digit order and stores each digit's run contiguously.
#include <algorithm>

#include "radix.cuh"
#include "scan.cuh"

namespace mc {
namespace {

using u64 = unsigned long long;

__device__ __forceinline__ unsigned digit_of(u64 key, int shift) {
  return (unsigned)(key >> shift) & (kRadixBins - 1);
}

// Lanes of the warp holding a real key with the same digit as this lane: the
// intersection over the digit's 8 bits of each bit's ballot (or its
// complement), restricted to the lanes with a key.  The same set that
// __match_any_sync returns, from plain votes.
__device__ __forceinline__ unsigned digit_peers(unsigned d, bool ok) {
  unsigned peers = __ballot_sync(kFull, ok);
#pragma unroll
  for (int b = 0; b < kRadixBits; ++b) {
    const unsigned bit = (d >> b) & 1u;
    const unsigned m = __ballot_sync(kFull, bit);
    peers &= bit ? m : ~m;
  }
  return peers;
}

// Upsweep: the digit histogram of every tile (shared-memory atomics into a
// per-warp row), stored as counts[d * tiles + t] so that one exclusive scan
// orders the runs digit-major, tile-minor.
__global__ void __launch_bounds__(kSortThreads) radix_count_kernel(const u64 *__restrict__ keys,
                                                                   int64_t count, int shift,
                                                                   int64_t tiles,
                                                                   int32_t *__restrict__ counts) {
  __shared__ int hist[kSortWarps][kRadixBins];
  for (int i = threadIdx.x; i < kSortWarps * kRadixBins; i += kSortThreads) (&hist[0][0])[i] = 0;
  __syncthreads();
  const int lane = threadIdx.x & (kWarp - 1), w = threadIdx.x / kWarp;
  const int64_t first = (int64_t)blockIdx.x * kSortTile + (int64_t)w * kWarpSpan + lane;
  u64 k[kSortRounds];
  load_warp_keys(keys, count, first, k);
#pragma unroll
  for (int r = 0; r < kSortRounds; ++r)
    if (first + r * kWarp < count) atomicAdd(&hist[w][digit_of(k[r], shift)], 1);
  __syncthreads();
  int s = 0;
#pragma unroll
  for (int x = 0; x < kSortWarps; ++x) s += hist[x][threadIdx.x];
  counts[(int64_t)threadIdx.x * tiles + blockIdx.x] = s;
}

// Downsweep: ranks every key of the tile stably by digit (warp order, then
// round, then lane = input order), stages the tile in shared memory in digit
// order, then stores each digit's run to its slot range.
__global__ void __launch_bounds__(kSortThreads, 3) radix_scatter_kernel(
    const u64 *__restrict__ keys_in, u64 *__restrict__ keys_out, int64_t count, int shift,
    int64_t tiles, const int64_t *__restrict__ offsets) {
  __shared__ int hist[kSortWarps][kRadixBins];  // running counts, then warp prefixes
  __shared__ int bin_start[kRadixBins];         // tile-local first slot per digit
  __shared__ long long bin_dest[kRadixBins];    // global slot - tile-local slot
  __shared__ int warp_tot[kSortWarps];
  __shared__ u64 stage[kSortTile];
  for (int i = threadIdx.x; i < kSortWarps * kRadixBins; i += kSortThreads) (&hist[0][0])[i] = 0;
  __syncthreads();
  const int lane = threadIdx.x & (kWarp - 1), w = threadIdx.x / kWarp;
  const int64_t tile_first = (int64_t)blockIdx.x * kSortTile;
  const int64_t first = tile_first + (int64_t)w * kWarpSpan + lane;
  u64 k[kSortRounds];
  int rank[kSortRounds];
  load_warp_keys(keys_in, count, first, k);
  const unsigned lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < kSortRounds; ++r) {
    const bool ok = first + r * kWarp < count;
    const unsigned d = ok ? digit_of(k[r], shift) : 0u;
    const unsigned peers = digit_peers(d, ok);
    const int before = ok ? hist[w][d] : 0;
    __syncwarp();
    if (ok && lane == __ffs(peers) - 1) hist[w][d] = before + __popc(peers);
    __syncwarp();
    rank[r] = before + __popc(peers & lt);
  }
  __syncthreads();
  // Thread t owns digit t: exclusive prefix over warps, then over digits.
  const int t = threadIdx.x;
  int tot = 0;
#pragma unroll
  for (int x = 0; x < kSortWarps; ++x) {
    const int c = hist[x][t];
    hist[x][t] = tot;
    tot += c;
  }
  const int incl = warp_inclusive_scan(tot, lane);
  if (lane == kWarp - 1) warp_tot[w] = incl;
  __syncthreads();
  int wbase = 0;
  for (int x = 0; x < w; ++x) wbase += warp_tot[x];
  const int start = wbase + incl - tot;
  bin_start[t] = start;
  bin_dest[t] = (long long)offsets[(int64_t)t * tiles + blockIdx.x] - start;
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortRounds; ++r) {
    if (first + r * kWarp < count) {
      const unsigned d = digit_of(k[r], shift);
      stage[bin_start[d] + hist[w][d] + rank[r]] = k[r];
    }
  }
  __syncthreads();
  const int in_tile = (int)min((int64_t)kSortTile, count - tile_first);
  for (int j = t; j < in_tile; j += kSortThreads) {
    const u64 key = stage[j];
    keys_out[bin_dest[digit_of(key, shift)] + j] = key;
  }
}

}  // namespace

int64_t radix_entries(int64_t count) { return (int64_t)kRadixBins * sort_tiles(count); }

size_t radix_temp_bytes(int64_t count) { return scan_temp_bytes(radix_entries(count)); }

cudaError_t radix_sort_u64(u64 *keys, u64 *alt, int64_t count, int begin_bit, int end_bit,
                           int32_t *counts, int64_t *offsets, void *temp, cudaStream_t s,
                           u64 **sorted, int64_t *launches) {
  u64 *buf[2] = {keys, alt};
  int cur = 0;
  if (count > 0) {
    const int64_t tiles = sort_tiles(count);
    const int64_t entries = radix_entries(count);
    for (int shift = begin_bit; shift < end_bit; shift += kRadixBits) {
      radix_count_kernel<<<(unsigned)tiles, kSortThreads, 0, s>>>(buf[cur], count, shift, tiles,
                                                                  counts);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return e;
      e = exclusive_scan(counts, offsets, entries, temp, s);
      if (e != cudaSuccess) return e;
      radix_scatter_kernel<<<(unsigned)tiles, kSortThreads, 0, s>>>(buf[cur], buf[cur ^ 1], count,
                                                                    shift, tiles, offsets);
      e = cudaGetLastError();
      if (e != cudaSuccess) return e;
      cur ^= 1;
      *launches += 2 + scan_launches(entries);
    }
  }
  *sorted = buf[cur];
  return cudaSuccess;
}

}  // namespace mc

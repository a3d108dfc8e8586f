// Stable LSD radix sort of 64-bit keys on the device (8 bits per pass over a
// chosen bit range), and the warp-striped tile layout its kernels share with
// the CSR build: a CTA owns kSortTile consecutive keys, each warp a span of
// kWarpSpan, read in kSortRounds rounds of 32 consecutive keys.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "device_common.cuh"

namespace mc {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / kWarp;
constexpr int kSortRounds = 16;                          // keys per thread
constexpr int kSortTile = kSortThreads * kSortRounds;    // keys per CTA
constexpr int kWarpSpan = kWarp * kSortRounds;           // keys per warp
constexpr int kRadixBits = 8;
constexpr int kRadixBins = 1 << kRadixBits;
static_assert(kRadixBins == kSortThreads, "one thread per digit in the digit scans");

inline int bit_width(uint64_t x) {
  int b = 0;
  while (x) {
    ++b;
    x >>= 1;
  }
  return b;
}

inline int64_t sort_tiles(int64_t count) { return (count + kSortTile - 1) / kSortTile; }

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Round r, lane l of a warp whose span starts at `first - lane` holds key
// first + 32 r: every load instruction reads 256 contiguous bytes.
__device__ __forceinline__ void load_warp_keys(const unsigned long long *__restrict__ keys,
                                               int64_t count, int64_t first,
                                               unsigned long long (&k)[kSortRounds]) {
#pragma unroll
  for (int r = 0; r < kSortRounds; ++r) {
    const int64_t i = first + r * kWarp;
    k[r] = i < count ? __ldg(keys + i) : 0ull;
  }
}

// Scratch of one radix sort of `count` keys: counts (int32) and offsets
// (int64) of kRadixBins * tiles entries (+1), and the scan's temporary bytes.
int64_t radix_entries(int64_t count);
size_t radix_temp_bytes(int64_t count);

// Sorts keys[0, count) by bits [begin_bit, end_bit), stably, using `alt` as
// the other buffer of each pass; *sorted receives the buffer holding the
// result (keys or alt). Asynchronous on `s`; *launches counts the kernels.
cudaError_t radix_sort_u64(unsigned long long *keys, unsigned long long *alt, int64_t count,
                           int begin_bit, int end_bit, int32_t *counts, int64_t *offsets,
                           void *temp, cudaStream_t s, unsigned long long **sorted,
                           int64_t *launches);

}  // namespace mc

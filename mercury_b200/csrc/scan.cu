// Reduce-then-scan exclusive prefix sum.  Each block owns kScanTile
// consecutive inputs; pass 1 writes one sum per block, the block sums are
// scanned recursively, pass 2 rescans each tile with its block offset.
#include "scan.cuh"
#include "device_common.cuh"

namespace mc {
namespace {

template <typename T>
__device__ __forceinline__ int64_t block_sum_items(const T *in, int64_t count, int64_t base,
                                                   int64_t *items) {
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    int64_t v = i < count ? (int64_t)in[i] : 0;
    items[k] = v;
    s += v;
  }
  return s;
}

// Block-wide exclusive scan of one int64 per thread; returns the block total
// through *total.
__device__ __forceinline__ int64_t block_exclusive(int64_t v, int64_t *total) {
  __shared__ int64_t warp_tot[kScanThreads / kWarp];
  const int lane = threadIdx.x & (kWarp - 1), wid = threadIdx.x / kWarp;
  int64_t x = v;
#pragma unroll
  for (int o = 1; o < kWarp; o <<= 1) {
    int64_t t = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += t;
  }
  if (lane == kWarp - 1) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int64_t w = lane < kScanThreads / kWarp ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1) {
      int64_t t = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += t;
    }
    if (lane < kScanThreads / kWarp) warp_tot[lane] = w;  // inclusive
  }
  __syncthreads();
  int64_t warp_off = wid ? warp_tot[wid - 1] : 0;
  *total = warp_tot[kScanThreads / kWarp - 1];
  __syncthreads();
  return warp_off + x - v;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const T *in, int64_t count,
                                                                   int64_t *block_sums) {
  int64_t items[kScanItems];
  int64_t s = block_sum_items(in, count, (int64_t)blockIdx.x * kScanTile, items);
  int64_t total;
  block_exclusive(s, &total);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const T *in, int64_t count,
                                                                  const int64_t *block_offsets,
                                                                  int64_t *out) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  int64_t items[kScanItems];
  int64_t s = block_sum_items(in, count, base, items);
  int64_t total;
  int64_t run = block_exclusive(s, &total) + (block_offsets ? block_offsets[blockIdx.x] : 0);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    if (i < count) out[i] = run;
    run += items[k];
  }
  // The thread holding the last real item writes the grand total to
  // out[count]; its `run` already includes that item (padding items are 0).
  const int64_t first = base + (int64_t)threadIdx.x * kScanItems;
  if (count - 1 >= first && count - 1 < first + kScanItems) out[count] = run;
}

int64_t blocks_for(int64_t count) { return (count + kScanTile - 1) / kScanTile; }

template <typename T>
cudaError_t scan_impl(const T *in, int64_t *out, int64_t count, char *temp, cudaStream_t s) {
  if (count <= 0) {
    return cudaMemsetAsync(out, 0, sizeof(int64_t), s);
  }
  const int64_t nb = blocks_for(count);
  if (nb == 1) {
    scan_apply_kernel<T><<<1, kScanThreads, 0, s>>>(in, count, nullptr, out);
    return cudaGetLastError();
  }
  int64_t *sums = reinterpret_cast<int64_t *>(temp);
  int64_t *offs = sums + nb;
  char *rest = reinterpret_cast<char *>(offs + nb + 1);
  scan_reduce_kernel<T><<<(unsigned)nb, kScanThreads, 0, s>>>(in, count, sums);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = scan_impl<int64_t>(sums, offs, nb, rest, s);
  if (e != cudaSuccess) return e;
  scan_apply_kernel<T><<<(unsigned)nb, kScanThreads, 0, s>>>(in, count, offs, out);
  return cudaGetLastError();
}

}  // namespace

int scan_launches(int64_t count) {
  if (count <= 0) return 0;
  const int64_t nb = blocks_for(count);
  return nb == 1 ? 1 : 2 + scan_launches(nb);
}

size_t scan_temp_bytes(int64_t count) {
  size_t bytes = 0;
  int64_t c = count;
  while (c > kScanTile) {
    int64_t nb = blocks_for(c);
    bytes += sizeof(int64_t) * (2 * nb + 1);
    c = nb;
  }
  return bytes + 256;
}

cudaError_t exclusive_scan(const int32_t *in, int64_t *out, int64_t count, void *temp,
                           cudaStream_t stream) {
  return scan_impl<int32_t>(in, out, count, static_cast<char *>(temp), stream);
}

cudaError_t exclusive_scan(const int64_t *in, int64_t *out, int64_t count, void *temp,
                           cudaStream_t stream) {
  return scan_impl<int64_t>(in, out, count, static_cast<char *>(temp), stream);
}

}  // namespace mc

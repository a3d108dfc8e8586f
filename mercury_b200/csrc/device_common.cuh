// Device-side helpers shared by the counting-path kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include "mercury.h"

namespace mc {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// Error bits a kernel raises in the handle's device flag word.
enum DeviceError : unsigned {
  kErrIdRange = 1u << 0,      // neighbour id outside [0, n)
  kErrUnsorted = 1u << 1,     // row not strictly ascending (or duplicate)
  kErrSelfLoop = 1u << 2,     // v listed in N(v)
  kErrRowptr = 1u << 3,       // row offsets not monotone / wrong ends
  kErrAsymmetric = 1u << 4,   // u in N(v) but v not in N(u)
  kErrHashFull = 1u << 5,     // a shared-memory table had no free slot
  kErrCapacity = 1u << 6,     // a scratch list exceeded its capacity
  kErrRank = 1u << 7,         // an out-list entry not ranked below its owner
  kErrDagCapacity = 1u << 8,  // more DAG entries than an exact-size DAG holds
  kErrWaitTimeout = 1u << 9,  // a bounded wait for an asynchronous copy gave up
};
// Bits of the CSR contract checks.
constexpr unsigned kErrContract = kErrIdRange | kErrUnsorted | kErrSelfLoop | kErrRowptr |
                                  kErrAsymmetric;

#define MC_CUDA_TRY(expr)                                   \
  do {                                                      \
    cudaError_t mc_e_ = (expr);                             \
    if (mc_e_ != cudaSuccess) {                             \
      mc::set_last_cuda_error(mc_e_);                       \
      return mc_e_ == cudaErrorMemoryAllocation ? MC_ERR_OOM \
                                                : MC_ERR_CUDA; \
    }                                                       \
  } while (0)

void set_last_cuda_error(cudaError_t e);
// The calling thread's last CUDA error seen by MC_CUDA_TRY.
cudaError_t last_cuda_error();

// A named NVTX range for the lifetime of the object: the library's phases
// (upload, orientation, counting, builds, batches) show up by name in a
// timeline profiler; without a tool attached a range costs a few ns.
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

// Device buffers come from the stream-ordered allocator on the owning
// handle's stream: freeing one never waits for the whole device.
// retain_pool_memory() makes the device's default pool keep freed memory
// mapped (the default threshold of 0 hands it back to the driver at every
// synchronisation, and the next allocation maps it again), so repeated
// calls reuse their buffers. The pool stays private to this process.
void retain_pool_memory(int device);

inline cudaError_t dev_alloc(void **p, size_t bytes, cudaStream_t s) {
  return cudaMallocAsync(p, bytes < 8 ? 8 : bytes, s);
}
inline void dev_free(void *p, cudaStream_t s) { cudaFreeAsync(p, s); }

__device__ __forceinline__ int warp_inclusive_scan(int v, int lane) {
#pragma unroll
  for (int o = 1; o < kWarp; o <<= 1) {
    int t = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
  return v;
}

// Largest r in [lo, hi] with a[r] <= key (a non-decreasing, a[lo] <= key).
__device__ __forceinline__ int64_t upper_row(const int64_t *__restrict__ a, int64_t lo,
                                             int64_t hi, int64_t key) {
  while (lo < hi) {
    int64_t mid = lo + ((hi - lo + 1) >> 1);
    if (__ldg(a + mid) <= key) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Smallest r in [lo, hi] with a[r] >= key (a[hi] >= key).
__device__ __forceinline__ int64_t lower_row(const int64_t *__restrict__ a, int64_t lo,
                                             int64_t hi, int64_t key) {
  while (lo < hi) {
    int64_t mid = lo + ((hi - lo) >> 1);
    if (__ldg(a + mid) >= key) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// Multiplicative (Fibonacci) hash of a vertex id to `bits` bits.
__device__ __forceinline__ unsigned hash_slot(int key, int shift) {
  return ((unsigned)key * 2654435769u) >> shift;
}

}  // namespace mc

// Exclusive prefix sums on the device (reduce-then-scan, recursive over
// block sums).  out[i] = in[0] + ... + in[i-1] for i in [0, count], so
// out[count] is the total: the layout of a CSR row-offset array.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mc {

// Elements handled by one scan block.
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int64_t kScanTile = (int64_t)kScanThreads * kScanItems;

// Bytes of temporary storage exclusive_scan needs for `count` inputs.
size_t scan_temp_bytes(int64_t count);

// Kernels one exclusive_scan of `count` inputs launches.
int scan_launches(int64_t count);

// in: int32 counts (non-negative); out: int64[count + 1].  Asynchronous on
// `stream`; `temp` must hold scan_temp_bytes(count) bytes.
cudaError_t exclusive_scan(const int32_t *in, int64_t *out, int64_t count, void *temp,
                           cudaStream_t stream);
// Same for int64 inputs.
cudaError_t exclusive_scan(const int64_t *in, int64_t *out, int64_t count, void *temp,
                           cudaStream_t stream);

}  // namespace mc

// Vertex labels on the device: the reference's label bookkeeping
// (graph.cc:37-82 reads graph.vlabel.bin, one uint8 per vertex;
// Graph::computeLabelsFrequency, graph.cc:440-460; Graph::BuildReverseIndex,
// graph.cc:413-436; Graph::BuildNLF, graph.cc:483-495) and its labelled
// intersection Graph::intersect_num(v, u, label) (graph.cc:396-411), used
// here for a triangle count split by label: counts[l] = the sum over DAG
// edges v -> u of #{w in N+(v) & N+(u) : label(w) == l}, i.e. the triangles
// whose DAG sink (the vertex of largest (degree, id), to which the other two
// point) has label l.  The counts sum to the triangle count.
#include <algorithm>
#include <cstring>
#include <vector>

#include "dgraph.cuh"
#include "device_common.cuh"
#include "scan.cuh"

namespace mc {
namespace {

constexpr int kLabelThreads = 256;

// labels[v] <= max_label for every v, else the error flag.
__global__ void check_labels_kernel(const uint8_t *__restrict__ labels, int64_t n, int max_label,
                                    unsigned *err) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x)
    if (labels[v] > max_label) atomicOr(err, (unsigned)kErrIdRange);
}

// freq[l] = #{v : label(v) == l}, through a per-block histogram.
__global__ void label_frequency_kernel(const uint8_t *__restrict__ labels, int64_t n,
                                       unsigned long long *freq) {
  __shared__ unsigned h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(h + labels[v], 1u);
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (h[i]) atomicAdd(freq + i, (unsigned long long)h[i]);
}

// Reverse index: vertices grouped by label, ascending ids within a label
// (the reference's sequential loop order).  One block per label walks the
// labels in windows of 256 vertices and places its matches in id order.
__global__ void reverse_index_kernel(const uint8_t *__restrict__ labels, int64_t n,
                                     const int64_t *__restrict__ offsets, int32_t *out) {
  const int l = blockIdx.x;
  __shared__ int s_warp[kLabelThreads / kWarp];
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x / kWarp;
  int64_t base = offsets[l];
  for (int64_t v0 = 0; v0 < n; v0 += blockDim.x) {
    const int64_t v = v0 + threadIdx.x;
    const bool mine = v < n && labels[v] == l;
    // Block-wide exclusive rank of the matches of this window, in id order.
    const unsigned m = __ballot_sync(kFull, mine);
    if (lane == 0) s_warp[warp] = __popc(m);
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < kLabelThreads / kWarp; ++w) {
      const int c = s_warp[w];
      if (w < warp) before += c;
      total += c;
    }
    if (mine) out[base + before + __popc(m & ((1u << lane) - 1u))] = (int32_t)v;
    base += total;
    __syncthreads();
  }
}

// nlf[(v - v0) * L1 + l] = #{u in N(v) : label(u) == l} for v in [v0, v1).
__global__ void nlf_kernel(const int64_t *__restrict__ rp, const int32_t *__restrict__ ci,
                           const uint8_t *__restrict__ labels, int64_t v0, int64_t v1, int L1,
                           unsigned *__restrict__ nlf) {
  const int lane = threadIdx.x & (kWarp - 1);
  const int64_t warps = (int64_t)gridDim.x * blockDim.x / kWarp;
  for (int64_t v = v0 + ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; v < v1;
       v += warps) {
    unsigned *row = nlf + (v - v0) * L1;
    for (int64_t k = rp[v] + lane; k < rp[v + 1]; k += kWarp) {
      const int l = labels[ci[k]];
      if (l < L1) atomicAdd(row + l, 1u);
    }
  }
}

// Triangles split by the label of the DAG sink: warp per owner v, each
// out-neighbour u's list intersected with N+(v) by searching the shorter
// list's entries in the longer one.
__global__ void __launch_bounds__(kLabelThreads)
    tc_label_kernel(const int64_t *__restrict__ drp, const int32_t *__restrict__ dcol,
                    const uint8_t *__restrict__ labels, int64_t n, int L1,
                    unsigned long long *queue, unsigned long long *counts) {
  __shared__ unsigned long long h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const int lane = threadIdx.x & (kWarp - 1);
  for (;;) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(queue, 1ull);
    t = __shfl_sync(kFull, t, 0);
    if ((int64_t)t >= n) break;
    const int v = (int)t;
    const int64_t bv = drp[v], ev = drp[v + 1];
    const int dv = (int)(ev - bv);
    for (int64_t e = bv; e < ev; ++e) {
      const int u = dcol[e];
      const int64_t bu = drp[u];
      const int du = (int)(drp[u + 1] - bu);
      const int32_t *small = du < dv ? dcol + bu : dcol + bv;
      const int32_t *large = du < dv ? dcol + bv : dcol + bu;
      const int ns = du < dv ? du : dv, nl = du < dv ? dv : du;
      for (int i = lane; i < ns; i += kWarp) {
        const int w = small[i];
        int lo = 0, hi = nl - 1;
        bool hit = false;
        while (lo <= hi) {
          const int mid = (lo + hi) >> 1;
          const int m = large[mid];
          if (m == w) {
            hit = true;
            break;
          }
          if (m < w) lo = mid + 1;
          else hi = mid - 1;
        }
        if (hit) atomicAdd(h + labels[w], 1ull);
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < L1; i += blockDim.x)
    if (h[i]) atomicAdd(counts + i, h[i]);
}

double ms_between(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) return 0.0;
  return (double)ms;
}

int grid_for_n(int64_t n, int threads) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 148 * 32));
}

}  // namespace
}  // namespace mc

extern "C" {

int mc_dgraph_set_vlabels(mc_dgraph_t *g, const uint8_t *labels, int max_label) {
  if (!g || (!labels && g->n > 0) || max_label < 0 || max_label > 255) return MC_ERR_ARG;
  MC_CUDA_TRY(cudaSetDevice(g->device));
  cudaStream_t s = g->stream;
  if (g->vlabels) mc::dev_free(g->vlabels, s);
  g->vlabels = nullptr;
  g->max_label = -1;
  MC_CUDA_TRY(mc::dev_alloc((void **)&g->vlabels, (size_t)std::max<int64_t>(g->n, 1), s));
  if (g->n > 0)
    MC_CUDA_TRY(cudaMemcpyAsync(g->vlabels, labels, (size_t)g->n, cudaMemcpyHostToDevice, s));
  MC_CUDA_TRY(cudaMemsetAsync(g->err, 0, sizeof(unsigned), s));
  if (g->n > 0) {
    mc::check_labels_kernel<<<mc::grid_for_n(g->n, 256), 256, 0, s>>>(g->vlabels, g->n,
                                                                      max_label, g->err);
    MC_CUDA_TRY(cudaGetLastError());
  }
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_err, g->err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  if (*g->h_err) {
    mc::dev_free(g->vlabels, s);
    g->vlabels = nullptr;
    cudaMemsetAsync(g->err, 0, sizeof(unsigned), s);
    cudaStreamSynchronize(s);
    return MC_ERR_FORMAT;
  }
  g->max_label = max_label;
  return MC_OK;
}

int mc_label_frequency(mc_dgraph_t *g, uint64_t *freq) {
  if (!g || !freq) return MC_ERR_ARG;
  if (!g->vlabels) return MC_ERR_ARG;
  MC_CUDA_TRY(cudaSetDevice(g->device));
  cudaStream_t s = g->stream;
  unsigned long long *d = nullptr;
  MC_CUDA_TRY(mc::dev_alloc((void **)&d, sizeof(unsigned long long) * 256, s));
  MC_CUDA_TRY(cudaMemsetAsync(d, 0, sizeof(unsigned long long) * 256, s));
  if (g->n > 0) {
    mc::label_frequency_kernel<<<mc::grid_for_n(g->n, 256), 256, 0, s>>>(g->vlabels, g->n, d);
    MC_CUDA_TRY(cudaGetLastError());
  }
  MC_CUDA_TRY(cudaMemcpyAsync(freq, d, sizeof(uint64_t) * (g->max_label + 1),
                              cudaMemcpyDeviceToHost, s));
  mc::dev_free(d, s);
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  return MC_OK;
}

int mc_label_reverse_index(mc_dgraph_t *g, int64_t *offsets, int32_t *vertices) {
  if (!g || !offsets || (!vertices && g->n > 0) || !g->vlabels) return MC_ERR_ARG;
  const int L1 = g->max_label + 1;
  std::vector<uint64_t> freq(L1);
  int rc = mc_label_frequency(g, freq.data());
  if (rc != MC_OK) return rc;
  offsets[0] = 0;
  for (int l = 0; l < L1; ++l) offsets[l + 1] = offsets[l] + (int64_t)freq[l];
  if (g->n == 0) return MC_OK;
  cudaStream_t s = g->stream;
  int64_t *d_off = nullptr;
  int32_t *d_out = nullptr;
  MC_CUDA_TRY(mc::dev_alloc((void **)&d_off, sizeof(int64_t) * (L1 + 1), s));
  MC_CUDA_TRY(mc::dev_alloc((void **)&d_out, sizeof(int32_t) * (size_t)g->n, s));
  MC_CUDA_TRY(cudaMemcpyAsync(d_off, offsets, sizeof(int64_t) * (L1 + 1), cudaMemcpyHostToDevice, s));
  mc::reverse_index_kernel<<<L1, mc::kLabelThreads, 0, s>>>(g->vlabels, g->n, d_off, d_out);
  MC_CUDA_TRY(cudaGetLastError());
  MC_CUDA_TRY(cudaMemcpyAsync(vertices, d_out, sizeof(int32_t) * (size_t)g->n,
                              cudaMemcpyDeviceToHost, s));
  mc::dev_free(d_off, s);
  mc::dev_free(d_out, s);
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  return MC_OK;
}

int mc_label_nlf(mc_dgraph_t *g, int64_t v_begin, int64_t v_end, uint32_t *nlf) {
  if (!g || !g->vlabels || v_begin < 0 || v_end < v_begin || v_end > g->n) return MC_ERR_ARG;
  if (v_end == v_begin) return MC_OK;
  if (!nlf) return MC_ERR_ARG;
  MC_CUDA_TRY(cudaSetDevice(g->device));
  cudaStream_t s = g->stream;
  const int L1 = g->max_label + 1;
  const size_t bytes = sizeof(unsigned) * (size_t)(v_end - v_begin) * L1;
  unsigned *d = nullptr;
  MC_CUDA_TRY(mc::dev_alloc((void **)&d, bytes, s));
  MC_CUDA_TRY(cudaMemsetAsync(d, 0, bytes, s));
  mc::nlf_kernel<<<mc::grid_for_n((v_end - v_begin) * mc::kWarp, 256), 256, 0, s>>>(
      g->rowptr, g->col, g->vlabels, v_begin, v_end, L1, d);
  MC_CUDA_TRY(cudaGetLastError());
  MC_CUDA_TRY(cudaMemcpyAsync(nlf, d, bytes, cudaMemcpyDeviceToHost, s));
  mc::dev_free(d, s);
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  return MC_OK;
}

int mc_tc_count_by_label(mc_dgraph_t *g, uint64_t *counts, mc_timing_t *timing) {
  if (!g || !counts || !g->vlabels) return MC_ERR_ARG;
  MC_CUDA_TRY(cudaSetDevice(g->device));
  int rc = mc::tc_alloc(g);
  if (rc != MC_OK) return rc;
  cudaStream_t s = g->stream;
  const int L1 = g->max_label + 1;
  const int64_t launches_before = g->launches;
  MC_CUDA_TRY(cudaEventRecord(g->ev[0], s));
  rc = mc::tc_orient(g, nullptr);
  if (rc != MC_OK) return rc;
  MC_CUDA_TRY(cudaEventRecord(g->ev[1], s));
  unsigned long long *d = nullptr;
  MC_CUDA_TRY(mc::dev_alloc((void **)&d, sizeof(unsigned long long) * 257, s));
  MC_CUDA_TRY(cudaMemsetAsync(d, 0, sizeof(unsigned long long) * 257, s));
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mc::tc_label_kernel,
                                                    mc::kLabelThreads, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  if (g->n > 0) {
    mc::tc_label_kernel<<<g->num_sms * per_sm, mc::kLabelThreads, 0, s>>>(
        g->dag_rowptr, g->dag_col, g->vlabels, g->n, L1, d + 256, d);
    MC_CUDA_TRY(cudaGetLastError());
    g->launches += 1;
  }
  MC_CUDA_TRY(cudaEventRecord(g->ev[3], s));
  MC_CUDA_TRY(cudaMemcpyAsync(counts, d, sizeof(uint64_t) * L1, cudaMemcpyDeviceToHost, s));
  MC_CUDA_TRY(cudaMemcpyAsync(g->h_err, g->err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  mc::dev_free(d, s);
  MC_CUDA_TRY(cudaStreamSynchronize(s));
  if (*g->h_err & (mc::kErrDagCapacity | mc::kErrContract)) return MC_ERR_FORMAT;
  if (timing) {
    std::memset(timing, 0, sizeof(*timing));
    timing->orient_ms = mc::ms_between(g->ev[0], g->ev[1]);
    timing->count_ms = mc::ms_between(g->ev[1], g->ev[3]);
    timing->total_ms = mc::ms_between(g->ev[0], g->ev[3]);
    timing->launches = g->launches - launches_before;
  }
  return MC_OK;
}

}  // extern "C"

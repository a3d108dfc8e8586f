// Serving: a request loop with continuous batching.  Clients submit counting
// requests (a graph and a job) and wait on tickets.  Worker threads, each
// with its own stream, repeatedly take every queued request that fits the HBM
// budget (up to max_batch), assemble the batch on the device from the
// resident CSR cache, count it with the batch kernels and deliver each
// graph's count.  While one worker's batch runs, the others admit the
// requests that arrived meanwhile, so batches overlap on the device; memory
// is returned to the budget as each batch finishes.
//
// The reference has no serving mode (one graph per program run).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <list>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "dgraph.cuh"
#include "device_common.cuh"

namespace mc {
namespace {

using Clock = std::chrono::steady_clock;

// A graph resident on the device: the symmetric CSR, reused by every request
// that names the same cache key.
struct Resident {
  int64_t *rowptr = nullptr;
  int32_t *col = nullptr;
  int64_t n = 0, nnz = 0, max_degree = 0;
  int64_t sumsq = 0;  // sum of squared degrees (the pattern work estimate)
  int64_t bytes = 0;
  int pins = 0;  // batches currently using it
  cudaStream_t owner = nullptr;
};

struct Request {
  uint64_t ticket = 0;
  int job = 0;
  uint64_t key = 0;  // 0: not cached
  std::vector<int64_t> rowptr;
  std::vector<int32_t> col;
  int64_t n = 0, nnz = 0, max_degree = 0;
  int64_t sumsq = 0;
  Clock::time_point submitted;
  bool prepinned = false;  // resident graph pinned at submission (no arrays copied)
  bool done = false;
  int status = MC_OK;
  uint64_t count = 0;
  double latency_ms = 0;
};

struct Piece {
  const int64_t *rp;
  const int32_t *col;
  int64_t n, nnz, v0, e0;
};

// Concatenates the batch's graphs into one CSR with global ids: piece p
// (blockIdx.y) copies its rows with entry offset e0 and ids shifted by v0.
__global__ void assemble_kernel(const Piece *pieces, int64_t *urp, int32_t *ucol) {
  const Piece p = pieces[blockIdx.y];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t first = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t v = first; v < p.n; v += stride) urp[p.v0 + v] = p.rp[v] + p.e0;
  for (int64_t e = first; e < p.nnz; e += stride) ucol[p.e0 + e] = p.col[e] + (int32_t)p.v0;
}

__global__ void set_last_kernel(int64_t *urp, int64_t n, int64_t nnz) { urp[n] = nnz; }

int64_t csr_bytes(int64_t n, int64_t nnz) { return 8 * (n + 1) + 4 * nnz; }

// Estimated device work of a request, in entry visits: a triangle job
// streams its CSR (n + nnz); a pattern job's per-edge sets grow with the
// degrees at both ends (sum of squared degrees).  A batch is closed once
// its estimate would pass the server's cap, and a request above the cap on
// its own runs in a batch of its own, so one large graph never holds a
// whole batch of small ones behind it.
int64_t work_of(const Request &r) { return r.job == 0 ? r.n + r.nnz : std::max(r.sumsq, r.nnz); }

// Device memory one request needs inside a batch: its CSR three times
// (resident copy, batch union, handle copy) and the orientation scratch of a
// triangle job.  Pattern jobs also share the batch's frontier lists
// (pattern_scratch).
int64_t footprint(const Request &r) {
  const int64_t csr = csr_bytes(r.n, r.nnz);
  int64_t f = 3 * csr + 64 * 1024;
  if (r.job == 0) f += 40 * (r.n + 1) + 6 * r.nnz;
  return f;
}

// Frontier lists of the batch pattern kernel for list capacity `cap`: six
// lists of cap ints for at most 148 x 64 resident warps, capped like the
// kernel's own scratch budget.
int64_t pattern_scratch(int64_t cap) {
  return std::min<int64_t>(int64_t(2) << 30, 24 * 148 * 64 * std::max<int64_t>(cap, 1));
}

}  // namespace
}  // namespace mc

struct mc_server {
  int device = 0;
  int64_t budget = 0;
  int max_batch = 0;
  int64_t batch_work = 0;  // cap on a batch's estimated work (see work_of)
  int64_t pending_work = 0;  // estimated work of the queued requests
  int num_workers = 1;
  std::mutex mu;
  std::condition_variable work_cv, done_cv;
  std::deque<std::shared_ptr<mc::Request>> pending;
  std::unordered_map<uint64_t, std::shared_ptr<mc::Request>> tickets;
  std::unordered_map<uint64_t, mc::Resident> cache;
  std::list<uint64_t> lru;  // cache keys, most recent first
  int64_t in_use = 0;       // reserved by running batches
  int64_t cache_bytes = 0;
  uint64_t next_ticket = 1;
  bool stop = false;
  std::vector<std::thread> workers;
  mc_server_stats_t stats{};
};

namespace mc {
namespace {

double ms_since(Clock::time_point t) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t).count();
}

// Drops unpinned cache entries (least recently used first) until `need`
// more bytes fit in the budget.  Caller holds the lock.
void evict_for(mc_server *s, int64_t need, cudaStream_t stream) {
  for (auto it = s->lru.rbegin(); it != s->lru.rend() && s->in_use + s->cache_bytes + need > s->budget;) {
    auto c = s->cache.find(*it);
    if (c != s->cache.end() && c->second.pins == 0) {
      dev_free(c->second.rowptr, stream);
      dev_free(c->second.col, stream);
      s->cache_bytes -= c->second.bytes;
      s->cache.erase(c);
      it = decltype(it)(s->lru.erase(std::next(it).base()));
    } else {
      ++it;
    }
  }
}

void finish(mc_server *s, const std::vector<std::shared_ptr<Request>> &batch,
            const std::vector<uint64_t> &counts, int status) {
  std::lock_guard<std::mutex> lock(s->mu);
  for (size_t i = 0; i < batch.size(); ++i) {
    Request &r = *batch[i];
    r.status = status;
    r.count = status == MC_OK ? counts[i] : 0;
    r.latency_ms = ms_since(r.submitted);
    r.done = true;
    r.rowptr.clear();
    r.rowptr.shrink_to_fit();
    r.col.clear();
    r.col.shrink_to_fit();
    if (status == MC_OK) ++s->stats.completed;
    else ++s->stats.failed;
  }
  s->done_cv.notify_all();
}

// Runs one batch: device CSRs (resident or uploaded), union assembly, batch
// count, delivery.  `reserved` bytes were taken from the budget by the
// caller and are returned here.
void run_batch(mc_server *s, std::vector<std::shared_ptr<Request>> &batch, int64_t reserved,
               cudaStream_t stream) {
  const int G = (int)batch.size();
  std::vector<Piece> pieces(G);
  std::vector<void *> temps;
  struct Upload {
    int index;
    int64_t *rowptr;
    int32_t *col;
  };
  std::vector<Upload> uploads;  // keyed graphs uploaded by this batch
  std::vector<uint64_t> pinned;  // cache entries this batch pinned
  std::vector<int64_t> vptr(G + 1, 0), maxdeg(G), gnnz(G);
  std::vector<int32_t> jobs(G);
  std::vector<uint64_t> counts(G, 0);
  int status = MC_OK;
  auto cuda_ok = [&](cudaError_t e) {
    if (e != cudaSuccess && status == MC_OK) {
      status = e == cudaErrorMemoryAllocation ? MC_ERR_OOM : MC_ERR_CUDA;
      set_last_cuda_error(e);
    }
    return status == MC_OK;
  };
  int64_t e_total = 0;
  for (int i = 0; i < G; ++i) {
    Request &r = *batch[i];
    const int64_t *rp = nullptr;
    const int32_t *col = nullptr;
    bool cached = false;
    if (r.key) {
      std::lock_guard<std::mutex> lock(s->mu);
      auto it = s->cache.find(r.key);
      if (it != s->cache.end()) {
        rp = it->second.rowptr;
        col = it->second.col;
        r.n = it->second.n;
        r.nnz = it->second.nnz;
        r.max_degree = it->second.max_degree;
        if (!r.prepinned) ++it->second.pins;  // a prepinned request holds its pin already
        pinned.push_back(r.key);
        cached = true;
        ++s->stats.cache_hits;
        s->lru.remove(r.key);
        s->lru.push_front(r.key);
      }
    }
    if (!cached && status == MC_OK) {
      int64_t *drp = nullptr;
      int32_t *dcol = nullptr;
      if (cuda_ok(dev_alloc((void **)&drp, 8 * (r.n + 1), stream)) &&
          cuda_ok(dev_alloc((void **)&dcol, 4 * std::max<int64_t>(r.nnz, 1), stream)) &&
          cuda_ok(cudaMemcpyAsync(drp, r.rowptr.data(), 8 * (r.n + 1), cudaMemcpyHostToDevice, stream)) &&
          (r.nnz == 0 || cuda_ok(cudaMemcpyAsync(dcol, r.col.data(), 4 * r.nnz, cudaMemcpyHostToDevice, stream)))) {
        rp = drp;
        col = dcol;
        // Offered to the cache only once the copy has completed (below).
        if (r.key) uploads.push_back({i, drp, dcol});
        else {
          temps.push_back(drp);
          temps.push_back(dcol);
        }
      } else {
        if (drp) dev_free(drp, stream);
        if (dcol) dev_free(dcol, stream);
      }
    }
    pieces[i] = Piece{rp, col, r.n, r.nnz, vptr[i], e_total};
    vptr[i + 1] = vptr[i] + r.n;
    e_total += r.nnz;
    maxdeg[i] = r.max_degree;
    gnnz[i] = r.nnz;
    jobs[i] = r.job;
  }
  const int64_t n = vptr[G];
  int64_t *urp = nullptr;
  int32_t *ucol = nullptr;
  Piece *dpieces = nullptr;
  mc_batch_t *b = nullptr;
  if (status == MC_OK && cuda_ok(dev_alloc((void **)&urp, 8 * (n + 1), stream)) &&
      cuda_ok(dev_alloc((void **)&ucol, 4 * std::max<int64_t>(e_total, 1), stream)) &&
      cuda_ok(dev_alloc((void **)&dpieces, sizeof(Piece) * G, stream)) &&
      cuda_ok(cudaMemcpyAsync(dpieces, pieces.data(), sizeof(Piece) * G, cudaMemcpyHostToDevice, stream))) {
    int64_t longest = 1;
    for (const Piece &p : pieces) longest = std::max(longest, std::max(p.n, p.nnz));
    const unsigned gx = (unsigned)std::min<int64_t>((longest + 255) / 256, 256);
    assemble_kernel<<<dim3(gx, G), 256, 0, stream>>>(dpieces, urp, ucol);
    set_last_kernel<<<1, 1, 0, stream>>>(urp, n, e_total);
    if (cuda_ok(cudaGetLastError()) && cuda_ok(cudaStreamSynchronize(stream))) {
      // The uploads are complete: keyed graphs become resident for later
      // requests (pinned by this batch until it finishes).
      std::lock_guard<std::mutex> lock(s->mu);
      for (const Upload &u : uploads) {
        const Request &r = *batch[u.index];
        const int64_t bytes = csr_bytes(r.n, r.nnz);
        evict_for(s, bytes, stream);
        if (!s->cache.count(r.key) && s->in_use + s->cache_bytes + bytes <= s->budget) {
          Resident res;
          res.rowptr = u.rowptr;
          res.col = u.col;
          res.n = r.n;
          res.nnz = r.nnz;
          res.max_degree = r.max_degree;
          res.sumsq = r.sumsq;
          res.bytes = bytes;
          res.pins = 1;
          s->cache[r.key] = res;
          s->lru.push_front(r.key);
          s->cache_bytes += bytes;
          pinned.push_back(r.key);
        } else {
          temps.push_back(u.rowptr);
          temps.push_back(u.col);
        }
      }
      uploads.clear();
    }
    if (status == MC_OK) {
      status = batch_create(urp, ucol, true, n, e_total, vptr.data(), G, jobs.data(), maxdeg.data(),
                            gnnz.data(), stream, false, &b);
      if (status == MC_OK) status = mc_batch_count(b, counts.data(), nullptr);
    }
  }
  if (b) mc_batch_free(b);
  if (urp) dev_free(urp, stream);
  if (ucol) dev_free(ucol, stream);
  if (dpieces) dev_free(dpieces, stream);
  for (const Upload &u : uploads) {  // a failure before the cache step
    dev_free(u.rowptr, stream);
    dev_free(u.col, stream);
  }
  for (void *p : temps) dev_free(p, stream);
  cudaStreamSynchronize(stream);
  {
    std::lock_guard<std::mutex> lock(s->mu);
    for (uint64_t key : pinned) {
      auto it = s->cache.find(key);
      if (it != s->cache.end() && it->second.pins > 0) --it->second.pins;
    }
    s->in_use -= reserved;
    ++s->stats.batches;
    s->stats.max_batch_seen = std::max<int64_t>(s->stats.max_batch_seen, G);
  }
  s->work_cv.notify_all();  // memory came back: queued requests may now fit
  if (status == MC_ERR_CUDA) {
    const cudaError_t e = last_cuda_error() != cudaSuccess ? last_cuda_error() : cudaGetLastError();
    std::fprintf(stderr, "mercury server: a batch of %d requests failed: %s\n", G,
                 cudaGetErrorString(e));
  }
  finish(s, batch, counts, status);
}

void worker_main(mc_server *s) {
  cudaSetDevice(s->device);
  cudaStream_t stream = nullptr;
  cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
  for (;;) {
    std::vector<std::shared_ptr<Request>> batch;
    int64_t reserved = 0, pattern_cap = 0, work = 0;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      for (;;) {
        if (s->stop && s->pending.empty()) break;
        // Admit queued requests in arrival order while they fit the budget
        // and the batch's work cap.
        // The cap grows with the backlog (its share per worker), so a queue
        // that builds up is drained in larger batches; a request above the
        // base cap still runs alone.
        const int64_t cap = std::max(s->batch_work, s->pending_work / s->num_workers);
        while (!s->pending.empty() && (int)batch.size() < s->max_batch) {
          auto &r = s->pending.front();
          const int64_t w = work_of(*r);
          if (!batch.empty() && (work + w > cap || w > s->batch_work)) break;  // next batch
          int64_t f = footprint(*r);
          const int64_t cap_deg = r->job != 0 ? std::max(pattern_cap, r->max_degree) : pattern_cap;
          if (cap_deg > pattern_cap)
            f += pattern_scratch(cap_deg) - (pattern_cap ? pattern_scratch(pattern_cap) : 0);
          if (f > s->budget) {  // can never fit: refuse it
            if (r->prepinned) {
              auto c = s->cache.find(r->key);
              if (c != s->cache.end() && c->second.pins > 0) --c->second.pins;
            }
            r->status = MC_ERR_BUDGET;
            r->done = true;
            r->latency_ms = ms_since(r->submitted);
            ++s->stats.failed;
            s->pending_work -= w;
            s->pending.pop_front();
            s->done_cv.notify_all();
            continue;
          }
          if (s->in_use + reserved + f > s->budget) evict_for(s, reserved + f, stream);
          if (s->in_use + s->cache_bytes + reserved + f > s->budget && (!batch.empty() || s->in_use > 0))
            break;  // wait for memory from running batches
          reserved += f;
          pattern_cap = cap_deg;
          work += w;
          s->pending_work -= w;
          batch.push_back(r);
          s->pending.pop_front();
          if (w > s->batch_work) break;  // a large request runs alone
        }
        if (!batch.empty()) break;
        s->work_cv.wait(lock);
      }
      if (batch.empty()) break;  // stopping
      s->in_use += reserved;
    }
    run_batch(s, batch, reserved, stream);
  }
  cudaStreamSynchronize(stream);
  cudaStreamDestroy(stream);
}

}  // namespace
}  // namespace mc

extern "C" {

int mc_server_create(int64_t hbm_budget_bytes, int max_batch, int workers, mc_server_t **out) {
  if (!out || hbm_budget_bytes <= 0 || max_batch < 1 || workers < 1 || workers > 16)
    return MC_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MC_ERR_NO_DEVICE;
  mc_server *s = new (std::nothrow) mc_server();
  if (!s) return MC_ERR_OOM;
  cudaGetDevice(&s->device);
  s->budget = hbm_budget_bytes;
  s->max_batch = max_batch;
  // MERCURY_SERVE_BATCH_WORK overrides the default cap of 2^23 entry visits
  // (about 4 ms of batch kernels on a B200).
  s->batch_work = int64_t(1) << 23;
  if (const char *env = std::getenv("MERCURY_SERVE_BATCH_WORK"))
    s->batch_work = std::max<int64_t>(1, std::atoll(env));
  s->num_workers = workers;
  for (int i = 0; i < workers; ++i) s->workers.emplace_back(mc::worker_main, s);
  *out = s;
  return MC_OK;
}

int mc_server_submit(mc_server_t *s, const int64_t *rowptr, const int32_t *col, int64_t n,
                     int64_t nnz, int job, uint64_t key, uint64_t *ticket) {
  if (!s || !ticket || job < 0 || job > 8) return MC_ERR_ARG;
  auto r = std::make_shared<mc::Request>();
  r->job = job;
  r->key = key;
  bool cached = false;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = key ? s->cache.find(key) : s->cache.end();
    if (it != s->cache.end()) {
      // Resident: pin it now so it cannot be evicted before a worker runs
      // this request (the batch that runs it drops the pin).
      cached = true;
      r->n = it->second.n;
      r->nnz = it->second.nnz;
      r->max_degree = it->second.max_degree;
      r->sumsq = it->second.sumsq;
      ++it->second.pins;
      r->prepinned = true;
    }
  }
  if (!cached) {
    if (!rowptr || n < 0 || nnz < 0 || (nnz > 0 && !col)) return MC_ERR_ARG;
    if (rowptr[0] != 0 || rowptr[n] != nnz) return MC_ERR_FORMAT;
    try {
      r->rowptr.assign(rowptr, rowptr + n + 1);
      r->col.assign(col, col + nnz);
    } catch (const std::bad_alloc &) {
      return MC_ERR_OOM;
    }
    r->n = n;
    r->nnz = nnz;
    for (int64_t v = 0; v < n; ++v) {
      const int64_t d = rowptr[v + 1] - rowptr[v];
      r->max_degree = std::max(r->max_degree, d);
      r->sumsq += d * d;
    }
  }
  r->submitted = mc::Clock::now();
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stop) {
      if (r->prepinned) {
        auto c = s->cache.find(key);
        if (c != s->cache.end() && c->second.pins > 0) --c->second.pins;
      }
      return MC_ERR_ARG;
    }
    r->ticket = s->next_ticket++;
    s->tickets[r->ticket] = r;
    s->pending_work += mc::work_of(*r);
    s->pending.push_back(r);
    ++s->stats.submitted;
    *ticket = r->ticket;
  }
  s->work_cv.notify_one();
  return MC_OK;
}

int mc_server_wait(mc_server_t *s, uint64_t ticket, int timeout_ms, uint64_t *count,
                   double *latency_ms) {
  if (!s) return MC_ERR_ARG;
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return MC_ERR_ARG;
  std::shared_ptr<mc::Request> r = it->second;
  const bool ok = s->done_cv.wait_for(lock, std::chrono::milliseconds(std::max(timeout_ms, 0)),
                                      [&] { return r->done; });
  if (!ok) return MC_ERR_TIMEOUT;
  s->tickets.erase(ticket);
  if (count) *count = r->count;
  if (latency_ms) *latency_ms = r->latency_ms;
  return r->status;
}

int mc_server_stats(mc_server_t *s, mc_server_stats_t *out) {
  if (!s || !out) return MC_ERR_ARG;
  std::lock_guard<std::mutex> lock(s->mu);
  *out = s->stats;
  out->cache_bytes = s->cache_bytes;
  out->cached_graphs = (int64_t)s->cache.size();
  out->queued = (int64_t)s->pending.size();
  return MC_OK;
}

void mc_server_free(mc_server_t *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
  }
  s->work_cv.notify_all();
  for (auto &t : s->workers) t.join();
  cudaSetDevice(s->device);
  for (auto &kv : s->cache) {  // workers have stopped: a synchronous free is fine
    cudaFree(kv.second.rowptr);
    cudaFree(kv.second.col);
  }
  cudaDeviceSynchronize();
  delete s;
}

}  // extern "C"

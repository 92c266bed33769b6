// Internal interface of the B200 block-sparse engine: tensor metadata, the context (stream, HBM
// pool, descriptor staging, kernel accounting) and the planners every host module calls.
//
// A tensor keeps its block table on the host (sorted keys, shapes, offsets) and its payload in
// one HBM allocation from the device's stream-ordered memory pool. Every operation plans on the
// host from the block tables, ships one descriptor array per kernel through a pinned staging
// ring, and launches a handful of kernels on the context stream; only operations whose result
// the host must read (norms, inner products, singular values, downloads) synchronise.
#pragma once

#include "../../include/bug_b200.h"
#include "kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

using bugk::CopyDesc;
using bugk::DotDesc;
using bugk::GemmOut;
using bugk::GemmPair;
using bugk::GemmTile;
using bugk::LinOut;
using bugk::LinSrc;
using bugk::QrDesc;
using bugk::ScaleDesc;
using bugk::SvdDesc;

namespace bugi {

extern thread_local std::string g_err;

struct BugError : std::runtime_error {
  int code;
  BugError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define BUG_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      throw ::bugi::BugError(e_ == cudaErrorMemoryAllocation ? BUG_ENOMEM : BUG_EDEVICE,         \
                     std::string(#call) + ": " + cudaGetErrorString(e_));                \
  } while (0)

inline void require(bool ok, const std::string& msg) {
  if (!ok) throw BugError(BUG_EINVAL, msg);
}

using Key = std::array<int, BUG_MAX_RANK>;

struct Leg {
  int dir = 1;
  std::vector<int> q;  // ascending charges
  std::vector<int> d;  // dimensions
  int dim_of(int c) const {
    auto it = std::lower_bound(q.begin(), q.end(), c);
    return (it != q.end() && *it == c) ? d[it - q.begin()] : 0;
  }
  int index_of(int c) const {
    auto it = std::lower_bound(q.begin(), q.end(), c);
    return (it != q.end() && *it == c) ? int(it - q.begin()) : -1;
  }
  int64_t total() const {
    int64_t s = 0;
    for (int x : d) s += x;
    return s;
  }
};

struct Block {
  Key key{};
  std::array<int, BUG_MAX_RANK> shape{};
  int64_t off = 0;
  int64_t size = 0;
};

}  // namespace bugi

struct bug_ctx;

namespace bugi {

// Merges the stage lists of several contexts that share one stream into single launches (one
// cluster per list, bugk::launch_stage_lists). A context hands over its drained list and waits
// until a launch holding it has been issued: at once when every context that could still submit
// has submitted, else after a short spin. Contexts that are waiting on the device (a read-back) or
// have no job do not hold a launch back. Stream order keeps each context's operations in its own
// program order, because a context issues nothing else while its list is pending.
struct Combiner {
  cudaStream_t stream = nullptr;
  int cluster = 0;
  std::mutex mu;
  std::vector<std::pair<const bugk::Stage*, int>> pending;
  std::atomic<uint64_t> launched_upto{0};  // tickets below this were launched
  uint64_t next_ticket = 0;
  int active = 0;   // contexts running a job
  int blocked = 0;  // of those, waiting on the device
  int64_t launches = 0, lists = 0;
  cudaError_t err = cudaSuccess;
  static constexpr double kSpinSeconds = 25e-6;

  // caller holds mu
  void flush_locked() {
    if (pending.empty()) return;
    bugk::ListTable lt{};
    const int n = int(pending.size());
    for (int i = 0; i < n; ++i) {
      lt.stages[i] = pending[i].first;
      lt.n[i] = pending[i].second;
    }
    const cudaError_t e = bugk::launch_stage_lists(lt, n, cluster, stream);
    if (e != cudaSuccess && err == cudaSuccess) err = e;
    ++launches;
    lists += n;
    pending.clear();
    launched_upto.store(next_ticket, std::memory_order_release);
  }
  void maybe_flush_locked() {
    if (!pending.empty() && int(pending.size()) >= std::max(1, active - blocked)) flush_locked();
  }
  void submit(const bugk::Stage* st, int n) {
    uint64_t ticket;
    {
      std::lock_guard<std::mutex> lk(mu);
      ticket = next_ticket++;
      pending.push_back({st, n});
      if (int(pending.size()) >= bugk::kMaxLists) flush_locked();
      else maybe_flush_locked();
    }
    const auto t0 = std::chrono::steady_clock::now();
    while (launched_upto.load(std::memory_order_acquire) <= ticket) {
      if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > kSpinSeconds) {
        std::lock_guard<std::mutex> lk(mu);
        if (launched_upto.load(std::memory_order_relaxed) <= ticket) flush_locked();
      }
    }
    std::lock_guard<std::mutex> lk(mu);
    if (err != cudaSuccess) {
      const cudaError_t e = err;
      err = cudaSuccess;
      throw BugError(BUG_EDEVICE, std::string("stage-list launch: ") + cudaGetErrorString(e));
    }
  }
  void job_begin() {
    std::lock_guard<std::mutex> lk(mu);
    ++active;
  }
  void job_end() {
    std::lock_guard<std::mutex> lk(mu);
    --active;
    maybe_flush_locked();
  }
  void block_begin() {
    std::lock_guard<std::mutex> lk(mu);
    ++blocked;
    maybe_flush_locked();
  }
  void block_end() {
    std::lock_guard<std::mutex> lk(mu);
    --blocked;
  }
};

// The context whose scratch the current C-ABI call queued for release (freed, stream-ordered,
// when the call returns).
extern thread_local bug_ctx* g_active_ctx;


struct Buffer {
  double2* ptr = nullptr;
  int64_t n = 0;
  bug_ctx* ctx = nullptr;
  ~Buffer();
};

}  // namespace bugi

struct bug_tensor {
  int rank = 0;
  std::vector<bugi::Leg> legs;
  std::vector<bugi::Block> blocks;  // ascending keys, payload laid out in this order
  int64_t nelem = 0;
  std::shared_ptr<bugi::Buffer> buf;

  // index of the block with key k (binary search over the sorted keys), or -1
  int find(const bugi::Key& k) const {
    auto it = std::lower_bound(blocks.begin(), blocks.end(), k,
                               [](const bugi::Block& b, const bugi::Key& key) { return b.key < key; });
    return (it != blocks.end() && it->key == k) ? int(it - blocks.begin()) : -1;
  }
  const double2* data(int b) const { return buf->ptr + blocks[b].off; }
  double2* mdata(int b) { return buf->ptr + blocks[b].off; }
};

struct bug_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t launches = 0;
  std::atomic<int64_t> bytes{0};  // payload bytes of the live tensors (released from either stream's thread)
  // per kernel family: launches, algorithmic flops and bytes, device time (profiling only)
  int64_t k_launches[BUG_K_NFAMILIES] = {};
  double k_flops[BUG_K_NFAMILIES] = {};
  double k_bytes[BUG_K_NFAMILIES] = {};
  double k_ms[BUG_K_NFAMILIES] = {};
  bool profiling = false;
  // host-side accounting: synchronisations the host waited on and the time spent waiting, time
  // inside kernel-launch calls, and time inside the stream-ordered allocator
  int64_t syncs = 0;
  double sync_wait_s = 0.0, launch_s = 0.0, alloc_s = 0.0;
  std::chrono::steady_clock::time_point launch_t0;
  static double since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  // Wait for everything issued so far (the host is about to read a result).
  void wait() {
    drain();
    const auto t0 = std::chrono::steady_clock::now();
    sync_stream();
    sync_wait_s += since(t0);
    ++syncs;
    check_tc_error();
  }
  // Contexts of a job server or batch share one stream and a Combiner; a context then waits for
  // its own work by an event (recorded after it), not for the whole shared stream.
  bugi::Combiner* combiner = nullptr;
  cudaEvent_t sync_ev = nullptr;
  bool owns_stream = true;
  void sync_stream() {
    if (!combiner) {
      BUG_CUDA(cudaStreamSynchronize(stream));
      return;
    }
    combiner->block_begin();
    cudaError_t e = cudaEventRecord(sync_ev, stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(sync_ev);
    combiner->block_end();
    BUG_CUDA(e);
  }
  // Mixed precision: output blocks with both extents >= mixed_min_dim go to the tensor-core GEMM
  // (0: off). Its kernels report a timed-out pipeline wait in a host-mapped flag.
  int mixed_min_dim = 0;
  int* tc_err_host = nullptr;
  int* tc_err_dev = nullptr;
  int* tc_error_flag() {
    if (!tc_err_host) {
      BUG_CUDA(cudaHostAlloc((void**)&tc_err_host, sizeof(int), cudaHostAllocMapped));
      *tc_err_host = 0;
      BUG_CUDA(cudaHostGetDevicePointer((void**)&tc_err_dev, tc_err_host, 0));
    }
    return tc_err_dev;
  }
  void check_tc_error() {
    if (tc_err_host && *tc_err_host) {
      *tc_err_host = 0;
      throw bugi::BugError(BUG_ETIMEOUT, "tensor-core GEMM: a pipeline wait ran out its bound");
    }
  }
  // Device memory: a caching allocator over the stream-ordered pool. Every kernel of the context
  // runs in order on its one stream, so a block released after its last enqueued use may be handed
  // to any later enqueued operation at once; released blocks wait in per-size-class free lists
  // (classes 1.25x apart) instead of going back through cudaFreeAsync/cudaMallocAsync.
  static constexpr size_t kCacheCap = size_t(8) << 30;  // bytes parked in free lists at most
  std::unordered_map<void*, size_t> live_;                // allocation -> its size class
  std::unordered_map<size_t, std::vector<void*>> free_;   // size class -> released blocks
  size_t cached_bytes = 0;
  static size_t size_class(size_t b) {
    if (b <= 256) return 256;
    const int e = 63 - __builtin_clzll(b - 1);  // 2^e < b <= 2^(e+1)
    const size_t step = (size_t(1) << e) / 4;
    return ((b + step - 1) / step) * step;
  }
  //
  // Concurrent half-sweeps (`parallel`): a second context, `child`, with its own stream, stage
  // queue and descriptor staging, drives one half on a thread of its own and allocates from THIS
  // context's allocator (`alloc_owner` on the child; `alloc_mu` serialises the two threads). A
  // block handed out during the fork was released before it began, so its last use precedes the
  // fork event both streams are ordered after; every release during the fork (`forking`) is
  // parked in `fork_frees` until the join, where the parent stream has waited for the child's,
  // so the blocks return to the free lists with both streams' uses behind them.
  bug_ctx* child = nullptr;
  bug_ctx* alloc_owner = nullptr;
  cudaEvent_t fork_ev = nullptr;  // parent: the fork point; child: the end of its half
  bool forking = false;
  std::mutex alloc_mu;
  std::vector<void*> fork_frees;
  bug_ctx* allocator() { return alloc_owner ? alloc_owner : this; }
  void* dev_alloc(size_t bytes) {
    const auto t0 = std::chrono::steady_clock::now();
    void* p = allocator()->alloc_on(bytes, stream);
    alloc_s += since(t0);
    return p;
  }
  // (on the allocator) a block of at least `bytes`; a new one is ordered on stream `s`
  void* alloc_on(size_t bytes, cudaStream_t s) {
    std::unique_lock<std::mutex> lk(alloc_mu, std::defer_lock);
    if (child) lk.lock();
    const size_t cls = size_class(bytes);
    void* p = nullptr;
    auto it = free_.find(cls);
    if (it != free_.end() && !it->second.empty()) {
      p = it->second.back();
      it->second.pop_back();
      cached_bytes -= cls;
    } else {
      cudaError_t e = cudaMallocAsync(&p, cls, s);
      if (e == cudaErrorMemoryAllocation) {  // give the parked blocks back and retry once
        cudaGetLastError();
        release_cached_on(s);
        e = cudaMallocAsync(&p, cls, s);
      }
      BUG_CUDA(e);
    }
    live_[p] = cls;
    return p;
  }
  void dev_free(void* p) {
    bug_ctx* o = allocator();
    if (o->forking) {
      std::lock_guard<std::mutex> g(o->alloc_mu);
      o->fork_frees.push_back(p);
      return;
    }
    if (!queue.empty()) {  // a queued stage may still read it: reusable once the queue is launched
      pending_free.push_back(p);
      return;
    }
    const auto t0 = std::chrono::steady_clock::now();
    o->free_now(p);
    alloc_s += since(t0);
  }
  // (on the allocator, no fork running) back to the free lists, or to the pool on this stream
  void free_now(void* p) {
    auto it = live_.find(p);
    size_t cls = 0;
    if (it != live_.end()) {
      cls = it->second;
      live_.erase(it);
    }
    if (cls > 0 && cached_bytes + cls <= kCacheCap) {
      free_[cls].push_back(p);
      cached_bytes += cls;
    } else {
      cudaFreeAsync(p, stream);
    }
  }
  void release_cached() { release_cached_on(stream); }
  void release_cached_on(cudaStream_t s) {
    for (auto& kv : free_)
      for (void* p : kv.second) cudaFreeAsync(p, s);
    free_.clear();
    cached_bytes = 0;
  }
  struct Pending {
    int fam;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> event_pool;
  cudaEvent_t cur_start = nullptr;
  cudaEvent_t take_event() {
    if (event_pool.empty()) {
      cudaEvent_t e;
      BUG_CUDA(cudaEventCreate(&e));
      return e;
    }
    cudaEvent_t e = event_pool.back();
    event_pool.pop_back();
    return e;
  }
  void harvest() {
    if (pending.empty()) return;
    BUG_CUDA(cudaEventSynchronize(pending.back().b));
    for (auto& p : pending) {
      float ms = 0.f;
      BUG_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
      k_ms[p.fam] += ms;
      event_pool.push_back(p.a);
      event_pool.push_back(p.b);
    }
    pending.clear();
  }
  // Called right before a launch: hands the launch its descriptors, inline in the kernel
  // parameters when they fit, else committed to the arena by one copy.
  bugk::Blob begin() {
    drain(true);  // queued stages come first in stream order (their descriptors share the batch)
    bugk::Blob b{nullptr, 0, arena};
    if (!batch.empty() && batch.size() <= bugk::kInlineMax) {
      b.host = batch.data();
      b.bytes = batch.size();
    } else {
      commit();
    }
    if (profiling) {
      cur_start = take_event();
      BUG_CUDA(cudaEventRecord(cur_start, stream));
    }
    launch_t0 = std::chrono::steady_clock::now();
    return b;
  }
  // pinned staging ring for descriptor uploads
  static constexpr int kSlots = 32;
  void* stage_ptr[kSlots] = {};
  size_t stage_cap[kSlots] = {};
  cudaEvent_t stage_ev[kSlots] = {};
  bool stage_used[kSlots] = {};
  int stage_next = 0;
  std::vector<void*> deferred;  // device scratch to free after the next launch
  // Small pinned buffer for results the host reads. Pinned memory from cudaHostAlloc is mapped into
  // the device's address space under unified addressing, so kernels write results here directly
  // and the host reads them after a stream synchronisation, with no copy in between.
  double* pinned_out = nullptr;
  size_t pinned_out_cap = 0;
  // SVDs taken ahead of their check (svd_ahead): their singular values and sweep counts
  static constexpr size_t kAheadCap = size_t(1) << 20;  // doubles
  double* ahead_host = nullptr;
  size_t ahead_used = 0;
  struct Ahead {
    size_t off, nsv, nsweeps;
  };
  std::vector<Ahead> ahead;

  void* stage(size_t bytes) {
    int s = stage_next;
    stage_next = (stage_next + 1) % kSlots;
    if (stage_used[s]) BUG_CUDA(cudaEventSynchronize(stage_ev[s]));
    if (stage_cap[s] < bytes) {
      if (stage_ptr[s]) BUG_CUDA(cudaFreeHost(stage_ptr[s]));
      size_t cap = std::max<size_t>(bytes, 1 << 16);
      BUG_CUDA(cudaHostAlloc(&stage_ptr[s], cap, cudaHostAllocDefault));
      stage_cap[s] = cap;
    }
    cur_slot = s;
    return stage_ptr[s];
  }
  int cur_slot = 0;
  void stage_done() {
    BUG_CUDA(cudaEventRecord(stage_ev[cur_slot], stream));
    stage_used[cur_slot] = true;
  }
  // Descriptor arena: the arrays of ONE launch are appended to a host batch and go to the device
  // in one pinned copy + one H2D transfer (commit, run by begin() right before the launch). The
  // arena is reused by every launch: the next transfer into it is stream-ordered after the kernel
  // that read it.
  char* arena = nullptr;
  size_t arena_cap = 0;
  std::vector<char> batch;
  template <class T>
  T* push(const std::vector<T>& v) {
    const size_t bytes = (std::max<size_t>(v.size() * sizeof(T), 16) + 15) & ~size_t(15);
    if (!arena) {
      arena_cap = size_t(64) << 20;
      BUG_CUDA(cudaMallocAsync((void**)&arena, arena_cap, stream));  // lives until destroy
    }
    const size_t off = batch.size();
    if (off + bytes > arena_cap) {  // a launch larger than the arena: its own buffer
      void* h = stage(bytes);
      if (!v.empty()) std::memcpy(h, v.data(), v.size() * sizeof(T));
      void* dptr = dev_alloc(bytes);
      BUG_CUDA(cudaMemcpyAsync(dptr, h, bytes, cudaMemcpyHostToDevice, stream));
      stage_done();
      deferred.push_back(dptr);
      bugi::g_active_ctx = this;
      return static_cast<T*>(dptr);
    }
    batch.resize(off + bytes);
    if (!v.empty()) std::memcpy(batch.data() + off, v.data(), v.size() * sizeof(T));
    return reinterpret_cast<T*>(arena + off);
  }
  void commit() {
    if (batch.empty()) return;
    void* h = stage(batch.size());
    std::memcpy(h, batch.data(), batch.size());
    BUG_CUDA(cudaMemcpyAsync(arena, h, batch.size(), cudaMemcpyHostToDevice, stream));
    stage_done();
    batch.clear();
  }
  // ── launching one operation ──
  unsigned int* dot_counter = nullptr;  // last-CTA counter of the dot stage (zero between launches)
  unsigned int* counter() {
    if (!dot_counter) {
      BUG_CUDA(cudaMalloc((void**)&dot_counter, sizeof(unsigned int)));
      BUG_CUDA(cudaMemsetAsync(dot_counter, 0, sizeof(unsigned int), stream));
    }
    return dot_counter;
  }
  // ── deferred stages ──
  // A small stage is not launched on its own: it joins the queue, and the queue runs as ONE
  // launch of one thread-block cluster (bugk::launch_stage_list) when the host next needs the
  // device: a read-back, any other launch or stream operation, a full queue, or the end of the
  // C-ABI call. The queued stages' descriptors stay in `batch` (their arena offsets are final),
  // and memory released while stages are queued is parked in `pending_free` until the queue is
  // launched, so no later operation can be handed a block a queued stage still reads.
  bool queue_enabled = true;
  int list_cluster = 0;  // CTAs of the stage-list cluster (0: no cluster launch; never queue)
  std::vector<bugk::Stage> queue;
  std::vector<void*> pending_free;
  int64_t list_launches = 0, queued_stages = 0;
  // Stages a queue holds before it is launched: small enough that the device starts on them while
  // the host plans the next ones (a queue held back until a read-back leaves the device idle
  // meanwhile), large enough to save most launches.
  size_t queue_max_stages = 4;
  static constexpr size_t kQueueMaxBytes = size_t(2) << 20;
  // Only stages the cluster finishes in `queue_rounds` rounds are queued (a gemm tile or dot
  // descriptor per CTA per round; 4 elements per thread per round for the element-wise kinds):
  // a larger stage runs faster as its own full-grid launch than on one cluster.
  int queue_rounds = 1;
  static constexpr double kQueueMaxFlops = 2e7;       // gemm algorithmic flops
  bool queueable(const bugk::Stage& st, double flops) const {
    if (!queue_enabled || profiling || list_cluster <= 0) return false;
    const int64_t items = int64_t(queue_rounds) * list_cluster;
    switch (st.kind) {
      case bugk::kStageCopy:
      case bugk::kStageLincomb:
      case bugk::kStageScale:
        return st.total <= items * bugk::kStageThreads * 4;
      case bugk::kStageGemm:
        return st.n <= items && flops <= kQueueMaxFlops;
      case bugk::kStageDot:
        return st.n <= items;
      default:
        return false;
    }
  }
  // Launch the queued stages (in order) as one cluster launch. keep_batch: the caller has pushed
  // descriptors of its own launch after the queued ones and launches next (begin()).
  void drain(bool keep_batch = false) {
    if (queue.empty()) return;
    launch_t0 = std::chrono::steady_clock::now();
    bugk::Stage* d = push(queue);
    const int n = int(queue.size());
    cudaError_t e = cudaSuccess;
    if (combiner) {
      // descriptors to this context's arena (a merged launch carries nothing inline), then one
      // launch with the other contexts' lists
      commit();
      queue.clear();
      combiner->submit(d, n);
    } else {
      bugk::Blob b{nullptr, 0, arena};
      if (batch.size() <= bugk::kInlineMax) {
        b.host = batch.data();
        b.bytes = batch.size();
      } else {
        commit();  // copies every descriptor pushed so far (the caller's too) into the arena
      }
      e = bugk::launch_stage_list(b, d, n, list_cluster, stream);
      queue.clear();
      if (!keep_batch) batch.clear();
      ++launches;
    }
    launch_s += since(launch_t0);
    ++list_launches;
    std::vector<void*> freed;
    freed.swap(pending_free);
    for (void* p : freed) dev_free(p);
    BUG_CUDA(e);
  }
  // Drop the queue without launching it (the C-ABI call failed; its results are not used).
  void discard_queue() {
    queue.clear();
    batch.clear();
    std::vector<void*> freed;
    freed.swap(pending_free);
    for (void* p : freed) dev_free(p);
  }
  // Launch one stage whose descriptor arrays were pushed since the last launch, and account it.
  void run_stage(const bugk::Stage& st, int fam, double flops, double bytes_moved) {
    if (queueable(st, flops)) {
      queue.push_back(st);
      ++queued_stages;
      k_launches[fam] += 1;
      k_flops[fam] += flops;
      k_bytes[fam] += bytes_moved;
      bugi::g_active_ctx = this;  // the C-ABI call drains the queue when it returns
      if (queue.size() >= queue_max_stages || batch.size() >= kQueueMaxBytes) drain();
      return;
    }
    const bugk::Blob b = begin();
    bugk::launch_stage(b, st, stream);
    launched(fam, flops, bytes_moved);
  }
  void* scratch(size_t bytes) {
    void* dptr = dev_alloc(std::max<size_t>(bytes, 16));
    deferred.push_back(dptr);
    bugi::g_active_ctx = this;
    return dptr;
  }
  void launched(int fam, double flops, double bytes_moved) {
    launch_s += since(launch_t0);
    batch.clear();  // an inline launch has copied its descriptors into the launch
    ++launches;
    BUG_CUDA(cudaGetLastError());
    k_launches[fam] += 1;
    k_flops[fam] += flops;
    k_bytes[fam] += bytes_moved;
    if (profiling && cur_start) {
      cudaEvent_t e = take_event();
      BUG_CUDA(cudaEventRecord(e, stream));
      pending.push_back({fam, cur_start, e});
      cur_start = nullptr;
      if (pending.size() > 8192) harvest();
    }
  }
  void flush() {
    for (void* p : deferred) dev_free(p);
    deferred.clear();
  }
  double* readback(size_t n) {
    if (pinned_out_cap < n) {
      if (pinned_out) BUG_CUDA(cudaFreeHost(pinned_out));
      pinned_out_cap = std::max<size_t>(n, 4096);
      BUG_CUDA(cudaHostAlloc((void**)&pinned_out, pinned_out_cap * sizeof(double),
                             cudaHostAllocDefault));
    }
    return pinned_out;
  }
};

namespace bugi {

using TensorPtr = std::unique_ptr<bug_tensor>;

std::shared_ptr<Buffer> alloc_buffer(bug_ctx* c, int64_t n, bool zero);
TensorPtr make_tensor(bug_ctx* c, int rank, std::vector<Leg> legs, std::vector<Key> keys, bool zero);
Leg flipped(const Leg& l);
Leg merged(const Leg& a, const Leg& b);
TensorPtr permute_impl(bug_ctx* c, const bug_tensor& t, const int* perm);
TensorPtr contract_impl(bug_ctx* c, const bug_tensor& A, int n, const int* ia, const bug_tensor& B,
                        const int* ib, bool conja, bool conjb);
// want: 1 = U, 2 = Vd, 4 = U*S (into *US), 8 = S*Vd (into *SVd); all produced by one unpack launch
int svd_impl(bug_ctx* c, const bug_tensor& t, int nleft, const int* left, double cutoff, int nkeep,
             TensorPtr& U, TensorPtr& Vd, std::vector<double>& sv_sorted, std::vector<int>& sv_q,
             int& nkept, int want = 3, TensorPtr* US = nullptr, TensorPtr* SVd = nullptr);
// One tensor's SVD request for svd_many (svd_impl's arguments).
struct SvdReq {
  const bug_tensor* t;
  int nleft;
  const int* left;
  double cutoff;
  int nkeep;
  int want;
  TensorPtr* U;
  TensorPtr* Vd;
  std::vector<double>* sv_sorted;
  std::vector<int>* sv_q;
  int* nkept;
  TensorPtr* USo;
  TensorPtr* SVdo;
};
// Several tensors' SVDs (each as svd_impl) in one launch and one read-back.
void svd_many(bug_ctx* c, const std::vector<SvdReq>& reqs);
// SVDs with cutoff 0 and no Nkeep taken AHEAD of their read-back: every charge sector keeps all
// min(m, n) columns, which is what svd_many returns whenever no singular value is exactly zero
// (or non-finite) and every sector converged. Their singular values and sweep counts go to the
// context's pinned `ahead` region; svd_ahead_check waits for the stream and says whether every
// SVD taken ahead since the last check met that assumption, so a caller whose work is a pure
// function of its inputs can redo it the exact way when it did not. Returns false, launching
// nothing, when the region is full.
bool svd_ahead(bug_ctx* c, const std::vector<SvdReq>& reqs);
bool svd_ahead_check(bug_ctx* c);
void dots(bug_ctx* c, const std::vector<std::pair<const bug_tensor*, const bug_tensor*>>& pairs,
          double* out_re_im);
// sum_i coef_i t_i; with cmode[i] != 0 the coefficient of t_i is computed on the device from the
// dot product at cref[i] (bugk::LinSrc)
TensorPtr lincomb_impl(bug_ctx* c, int n, const double* coef, const bug_tensor* const* ts,
                       const double* const* cref = nullptr, const int* cmode = nullptr);
// <a_o, b_o> for every pair written (re, im) to device memory `q`, no host wait
void dots_device(bug_ctx* c, const std::vector<std::pair<const bug_tensor*, const bug_tensor*>>& pairs,
                 double2* q);
std::vector<double> sector_norms2(bug_ctx* c, const bug_tensor& t, int leg);
void sector_norms2_device(bug_ctx* c, const bug_tensor& t, int leg, double2* q);
// A context's stream, queue and staging, set up for `device` / released after its stream finished.
void ctx_init(bug_ctx* c, int device);
void ctx_release(bug_ctx* c);
// Two halves on two streams: fork_begin returns the second context (made on first use), ordered
// after everything the parent issued; the half on it ends with fork_child_done on its own thread;
// fork_end (parent thread, after that thread joined) orders the parent after it and returns the
// releases parked meanwhile.
bug_ctx* fork_begin(bug_ctx* c);
void fork_child_done(bug_ctx* ch, bool ok);
void fork_end(bug_ctx* c);
TensorPtr thin_qr_impl(bug_ctx* c, const bug_tensor& t, int fl, int ref_dir, double thr);
TensorPtr scale_leg_impl(bug_ctx* c, const bug_tensor& t, int leg, const double* w);
TensorPtr conj_impl(bug_ctx* c, const bug_tensor& t);
TensorPtr flip_leg_impl(bug_ctx* c, const bug_tensor& t, int leg);
TensorPtr oplus_impl(bug_ctx* c, int n, const bug_tensor* const* ts, int leg);
TensorPtr trim_impl(bug_ctx* c, const bug_tensor& t, int leg, const int* counts);
TensorPtr upload_impl(bug_ctx* c, int rank, const std::vector<Leg>& legs, const std::vector<Key>& keys,
                      const double* data);
int guard(const std::function<void()>& f);

}  // namespace bugi


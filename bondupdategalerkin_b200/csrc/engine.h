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
#include <cmath>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

using bugk::CopyDesc;
using bugk::DotDesc;
using bugk::GemmOut;
using bugk::GemmPair;
using bugk::GemmTile;
using bugk::LinOut;
using bugk::LinSrc;
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
  std::map<bugi::Key, int> index;
  int64_t nelem = 0;
  std::shared_ptr<bugi::Buffer> buf;

  int find(const bugi::Key& k) const {
    auto it = index.find(k);
    return it == index.end() ? -1 : it->second;
  }
  const double2* data(int b) const { return buf->ptr + blocks[b].off; }
  double2* mdata(int b) { return buf->ptr + blocks[b].off; }
};

struct bug_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t launches = 0;
  int64_t bytes = 0;
  // per kernel family: launches, algorithmic flops and bytes, device time (profiling only)
  int64_t k_launches[BUG_K_NFAMILIES] = {};
  double k_flops[BUG_K_NFAMILIES] = {};
  double k_bytes[BUG_K_NFAMILIES] = {};
  double k_ms[BUG_K_NFAMILIES] = {};
  bool profiling = false;
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
  void begin() {
    commit();
    if (profiling) {
      cur_start = take_event();
      BUG_CUDA(cudaEventRecord(cur_start, stream));
    }
  }
  // pinned staging ring for descriptor uploads
  static constexpr int kSlots = 32;
  void* stage_ptr[kSlots] = {};
  size_t stage_cap[kSlots] = {};
  cudaEvent_t stage_ev[kSlots] = {};
  bool stage_used[kSlots] = {};
  int stage_next = 0;
  std::vector<void*> deferred;  // device scratch to free after the next launch
  double* pinned_out = nullptr;  // small pinned buffer for results read back by the host
  size_t pinned_out_cap = 0;

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
  unsigned int* dot_counter = nullptr;  // last-block counter of the fused reduction
  char* arena = nullptr;
  size_t arena_cap = 0;
  std::vector<char> batch;
  template <class T>
  T* push(const std::vector<T>& v) {
    const size_t bytes = (std::max<size_t>(v.size() * sizeof(T), 16) + 15) & ~size_t(15);
    if (!arena) {
      arena_cap = size_t(64) << 20;
      BUG_CUDA(cudaMallocAsync((void**)&arena, arena_cap, stream));
    }
    const size_t off = batch.size();
    if (off + bytes > arena_cap) {  // a launch larger than the arena: its own buffer
      void* h = stage(bytes);
      if (!v.empty()) std::memcpy(h, v.data(), v.size() * sizeof(T));
      void* dptr = nullptr;
      BUG_CUDA(cudaMallocAsync(&dptr, bytes, stream));
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
  void* scratch(size_t bytes) {
    void* dptr = nullptr;
    BUG_CUDA(cudaMallocAsync(&dptr, std::max<size_t>(bytes, 16), stream));
    deferred.push_back(dptr);
    bugi::g_active_ctx = this;
    return dptr;
  }
  void launched(int fam, double flops, double bytes_moved) {
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
    for (void* p : deferred) BUG_CUDA(cudaFreeAsync(p, stream));
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
void dots(bug_ctx* c, const std::vector<std::pair<const bug_tensor*, const bug_tensor*>>& pairs,
          double* out_re_im);
TensorPtr lincomb_impl(bug_ctx* c, int n, const double* coef, const bug_tensor* const* ts);
std::vector<double> sector_norms2(bug_ctx* c, const bug_tensor& t, int leg);
TensorPtr scale_leg_impl(bug_ctx* c, const bug_tensor& t, int leg, const double* w);
TensorPtr conj_impl(bug_ctx* c, const bug_tensor& t);
TensorPtr flip_leg_impl(bug_ctx* c, const bug_tensor& t, int leg);
TensorPtr oplus_impl(bug_ctx* c, int n, const bug_tensor* const* ts, int leg);
TensorPtr trim_impl(bug_ctx* c, const bug_tensor& t, int leg, const int* counts);
TensorPtr upload_impl(bug_ctx* c, int rank, const std::vector<Leg>& legs, const std::vector<Key>& keys,
                      const double* data);
int guard(const std::function<void()>& f);

}  // namespace bugi


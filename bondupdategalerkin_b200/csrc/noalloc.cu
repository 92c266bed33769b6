// Inner product of two device vectors with no allocation of any kind.
//
// Who needs this: callers that may not allocate GPU memory at the point of the call -- code that
// runs under a memory budget fixed up front (a serving process that reserved its pool), code
// inside a host callback or a library hook where cudaMalloc is forbidden or would deadlock on the
// caller's allocator, and code that must not touch the engine's context (whose creation and
// operations allocate from the stream-ordered pool). For them `bug_inner_noalloc` computes
// <a|b> = sum_i conj(a_i) b_i with the reduction's scratch (per-block partial sums and the
// last-block counter) held in one file-scope device array that the library image carries.
//
// Facts a caller must know:
//   * The scratch array is `kScratchBytes` bytes and lives on EVERY device that loads this
//     library until the process exits.
//   * n is limited to kMaxElems complex elements (kMaxChunks blocks of kChunk elements); larger n
//     is rejected with BUG_EINVAL and nothing runs.
//   * The first call on a device looks up the array's device address with cudaGetSymbolAddress
//     (a host-side lookup, once per device, made with that device current). Make that first call
//     before any stream capture. The address is kept for the life of the process, so the entry
//     point assumes the device's primary context (the runtime's default) and no cudaDeviceReset
//     between calls; a caller that resets the device or makes another context current must not
//     use it afterwards.
//   * a, b and out must be 16-byte aligned (the kernel moves whole complex doubles); a misaligned
//     pointer is rejected with BUG_EINVAL before anything runs.
//   * All calls on a device share its one array, and the array keeps the last call's contents:
//     each call clears the counter that must start at zero, but two calls whose kernels overlap on
//     the GPU (issued on different streams of one device with nothing ordering them) race on the
//     partial sums and the counter. Serialise the calls on a device.
//   * No cudaMalloc, cudaFree or allocating library routine is called.
#include "engine.h"

#include <mutex>

namespace {

constexpr int kThreadsNA = 256;
constexpr int64_t kChunk = 2048;             // elements per block
constexpr int kMaxChunks = 4096;             // blocks per call
constexpr int64_t kMaxElems = kChunk * kMaxChunks;  // 8,388,608 complex elements
constexpr size_t kScratchBytes = size_t(kMaxChunks) * sizeof(double2) + 256;  // partials + counter

// The whole scratch of the entry point: kMaxChunks partial sums, then the counter at byte offset
// kMaxChunks * 16.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

__device__ __forceinline__ double warp_sum_na(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(kThreadsNA)
inner_noalloc_kernel(const double2* __restrict__ a, const double2* __restrict__ b, int64_t n,
                     double2* __restrict__ out, unsigned char* scratch) {
  double2* partial = reinterpret_cast<double2*>(scratch);
  unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + size_t(kMaxChunks) * sizeof(double2));
  __shared__ double sr[kThreadsNA / 32], si[kThreadsNA / 32];
  __shared__ bool last;
  const int64_t begin = int64_t(blockIdx.x) * kChunk;
  const int64_t end = begin + kChunk < n ? begin + kChunk : n;
  double re = 0.0, im = 0.0;
  for (int64_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
    const double2 x = a[i], y = b[i];
    re = fma(x.x, y.x, fma(x.y, y.y, re));
    im = fma(x.x, y.y, fma(-x.y, y.x, im));
  }
  re = warp_sum_na(re);
  im = warp_sum_na(im);
  if ((threadIdx.x & 31) == 0) {
    sr[threadIdx.x >> 5] = re;
    si[threadIdx.x >> 5] = im;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tr = 0.0, ti = 0.0;
    for (int w = 0; w < kThreadsNA / 32; ++w) {
      tr += sr[w];
      ti += si[w];
    }
    partial[blockIdx.x] = make_double2(tr, ti);
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  double tr = 0.0, ti = 0.0;
  for (unsigned int k = 0; k < gridDim.x; ++k) {  // fixed order: deterministic
    const double2 p = __ldcg(&partial[k]);
    tr += p.x;
    ti += p.y;
  }
  *out = make_double2(tr, ti);
  *counter = 0u;
}

__global__ void zero_out_kernel(double2* out) { *out = make_double2(0.0, 0.0); }

// The device address of the scratch array on the current device (looked up once per device).
unsigned char* scratch_address() {
  int dev = 0;
  BUG_CUDA(cudaGetDevice(&dev));
  bugi::require(dev >= 0 && dev < kMaxDevices, "device index out of range for the no-alloc scratch table");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    BUG_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_scratch_addr[dev] = p;
  }
  return static_cast<unsigned char*>(g_scratch_addr[dev]);
}

}  // namespace

extern "C" int bug_inner_noalloc(const double* a, const double* b, int64_t n, double* out,
                                 void* stream) {
  return bugi::guard([&] {
    bugi::require(out != nullptr, "bug_inner_noalloc: null output pointer");
    bugi::require(n >= 0, "bug_inner_noalloc: negative length");
    bugi::require(n <= kMaxElems, "bug_inner_noalloc: n = " + std::to_string(n) +
                                      " exceeds the no-alloc limit of " + std::to_string(kMaxElems) +
                                      " complex elements");
    bugi::require(n == 0 || (a != nullptr && b != nullptr), "bug_inner_noalloc: null input pointer");
    // the kernel reads and writes whole complex doubles (16-byte loads and stores)
    bugi::require(reinterpret_cast<uintptr_t>(out) % 16 == 0,
                  "bug_inner_noalloc: out is not 16-byte aligned");
    bugi::require(n == 0 || (reinterpret_cast<uintptr_t>(a) % 16 == 0 &&
                             reinterpret_cast<uintptr_t>(b) % 16 == 0),
                  "bug_inner_noalloc: a or b is not 16-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* scratch = scratch_address();
    double2* o = reinterpret_cast<double2*>(out);
    if (n == 0) {
      zero_out_kernel<<<1, 1, 0, s>>>(o);
      BUG_CUDA(cudaGetLastError());
      return;
    }
    // the counter must start at zero whatever the previous call left
    BUG_CUDA(cudaMemsetAsync(scratch + size_t(kMaxChunks) * sizeof(double2), 0, sizeof(unsigned int), s));
    const int blocks = int((n + kChunk - 1) / kChunk);
    inner_noalloc_kernel<<<blocks, kThreadsNA, 0, s>>>(reinterpret_cast<const double2*>(a),
                                                       reinterpret_cast<const double2*>(b), n, o,
                                                       scratch);
    BUG_CUDA(cudaGetLastError());
  });
}

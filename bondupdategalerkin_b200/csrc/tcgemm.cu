// Mixed-precision grouped complex GEMM on tcgen05 tensor cores; see tcgemm.cuh for the method.
#include "tcgemm.cuh"

#include "engine.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

namespace bugtc {

namespace {

constexpr int kSlabRows = 128;
constexpr int kSlabBytes = kSlabRows * kSlotK * 4;  // 16 KiB: 128 rows of 128 bytes
constexpr int kStages = 3;
constexpr int kStageBytes = 4 * kSlabBytes;           // A hi, A lo, B hi, B lo
constexpr int kTcThreads = 128;                       // 4 warps: TMEM lanes 0-127
constexpr uint32_t kTmemCols = 128;                   // FP32 accumulator: 128 lanes x 128 columns
constexpr int kTcSmem = kStages * kStageBytes + 1024;  // + alignment slack to 1024 bytes
constexpr int kPackThreads = 256;
constexpr long long kSpinLimit = 1ll << 22;           // bounded waits: a stuck pipeline errors out

// Instruction descriptor of tcgen05.mma kind::tf32: D FP32 (bits 4-5 = 1), A and B TF32 (bits 7-9
// and 10-12 = 2), both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(kTileNr >> 3) << 17) |
                            (uint32_t(kTileM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for the completion of the barrier phase with this parity; false if the bound ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (long long i = 0; i < kSpinLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// 2-D TMA tile load (box 32 x 128 of 4-byte elements, 128-byte swizzle) into shared memory,
// completing its bytes on the barrier. Coordinates: x = element in the row (always 0: 16-byte
// aligned), y = row.
__device__ __forceinline__ void tma_load(void* dst, const CUtensorMap* map, uint64_t* bar, int x,
                                         int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
      "%4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major operand in the 128-byte swizzled layout: rows of
// 128 bytes, 8-row groups 1024 bytes apart (stride byte offset), version 1, swizzle mode 2.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= uint64_t((saddr & 0x3FFFFu) >> 4);
  d |= uint64_t(1) << 16;            // leading byte offset (unused by swizzled K-major layouts)
  d |= uint64_t(1024 >> 4) << 32;    // stride byte offset
  d |= uint64_t(1) << 46;            // descriptor version of sm_100
  d |= uint64_t(2) << 61;            // SWIZZLE_128B
  return d;
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %3, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %4, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(accumulate), "r"(kIdesc)
      : "memory");
}

// Arrive on the barrier once every tcgen05.mma this thread issued so far has completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Round to TF32 (10 explicit mantissa bits, to nearest, ties away), kept in an FP32 container.
__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ void split3(double x, float& hi, float& lo) {
  hi = to_tf32(float(x));
  lo = to_tf32(float(x - double(hi)));
}

__device__ __forceinline__ int64_t grp_off(int idx, int n, const int* d, const int64_t* s) {
  if (n == 0) return 0;
  if (n == 1) return int64_t(idx) * s[0];
  int64_t off = 0;
  for (int j = n - 1; j >= 0; --j) {
    const int q = idx % d[j];
    idx /= d[j];
    off += int64_t(q) * s[j];
  }
  return off;
}

// The pair of group g whose K range holds complex index k (pairs' ranges laid end to end).
__device__ __forceinline__ int pair_of(const TcGroup& g, const int* koff, int k) {
  int lo = g.pair_begin, hi = g.pair_end - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (koff[mid] <= k) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// ── pack: operands into hi/lo TF32 slabs (one CTA per slab pair) ──────────────────────────────
// The CTA evaluates its 128 x 32 values in the order that reads the source contiguously (along
// rows or along K, from the first pair's layout), keeps them in shared memory, and writes both
// slabs row by row.
__global__ void __launch_bounds__(kPackThreads) tc_pack_kernel(const TcGroup* __restrict__ groups,
                                                               const bugk::GemmPair* __restrict__ pairs,
                                                               const int* __restrict__ koff,
                                                               const TcPack* __restrict__ items,
                                                               float* __restrict__ apk,
                                                               float* __restrict__ bpk) {
  __shared__ float shi[kSlabRows][kSlotK + 1], slo[kSlabRows][kSlotK + 1];
  const TcPack it = items[blockIdx.x];
  const TcGroup g = groups[it.group];
  const bool isA = it.which == 0;
  const bugk::Operand& first = isA ? pairs[g.pair_begin].A : pairs[g.pair_begin].B;
  // A: contiguous along rows when its row group is fast; B: contiguous along K when its row
  // (contracted) group is fast
  const bool along_rows = isA ? (first.row_fast != 0) : (first.row_fast == 0);
  for (int e = threadIdx.x; e < kSlabRows * kSlotK; e += kPackThreads) {
    const int r = along_rows ? (e % kSlabRows) : (e / kSlotK);
    const int cc = along_rows ? (e / kSlabRows) : (e % kSlotK);
    const int kap = it.slot * kSlotK + cc;  // real K index
    const int k = kap >> 1, part = kap & 1;
    double x = 0.0;
    if (isA) {
      const int row = it.tile * kTileM + r;
      if (row < g.m && k < g.K) {
        const int p = pair_of(g, koff, k);
        const bugk::Operand& A = pairs[p].A;
        const double2 v = __ldg(A.p + grp_off(row, A.nr, A.rd, A.rs) +
                                grp_off(k - koff[p], A.nc, A.cd, A.cs));
        x = part ? (A.conj ? -v.y : v.y) : v.x;
      }
    } else {
      const int rho = it.tile * kTileNr + r;  // real output column
      const int j = rho >> 1, c = rho & 1;
      if (j < g.n && k < g.K) {
        const int p = pair_of(g, koff, k);
        const bugk::Operand& B = pairs[p].B;
        const double2 v = __ldg(B.p + grp_off(k - koff[p], B.nr, B.rd, B.rs) +
                                grp_off(j, B.nc, B.cd, B.cs));
        const double br = v.x, bi = B.conj ? -v.y : v.y;
        x = c == 0 ? (part == 0 ? br : -bi) : (part == 0 ? bi : br);
      }
    }
    float h, l;
    split3(x, h, l);
    shi[r][cc] = h;
    slo[r][cc] = l;
  }
  __syncthreads();
  const int64_t slab = isA ? g.a_slab0 + 2 * (int64_t(it.tile) * g.ks + it.slot)
                           : g.b_slab0 + 2 * (int64_t(it.tile) * g.ks + it.slot);
  float* dst = (isA ? apk : bpk) + slab * int64_t(kSlabRows) * kSlotK;
  for (int e = threadIdx.x; e < kSlabRows * kSlotK; e += kPackThreads) {
    const int r = e / kSlotK, cc = e % kSlotK;
    dst[e] = shi[r][cc];
    dst[kSlabRows * kSlotK + e] = slo[r][cc];
  }
}

// ── the tensor-core GEMM: one 128 x 64 (complex) output tile per CTA ─────────────────────────
// Thread 0 streams the K slots through the 3-stage ring (TMA into shared memory) and issues the
// MMAs: per slot and per 8-wide K step, lo*hi, hi*lo, hi*hi into the TMEM accumulator; a slot is
// refilled once the MMAs that read it have completed (tcgen05.commit on its empty barrier). The
// final commit releases the four warps, which read their 32 TMEM lanes (one output row per thread)
// and store the tile in FP64. Every wait is bounded: on a timeout the CTA records the error, waits
// (bounded) for its own loads still in flight, frees its TMEM and returns.
__global__ void __launch_bounds__(kTcThreads, 1)
    tc_cgemm_kernel(const __grid_constant__ CUtensorMap amap, const __grid_constant__ CUtensorMap bmap,
                    const TcGroup* __restrict__ groups, const TcTile* __restrict__ tiles, int* err) {
  extern __shared__ unsigned char dsm_raw[];
  __shared__ __align__(8) uint64_t full[kStages], empty[kStages], accum;
  __shared__ uint32_t tmem_base;
  const uint32_t raw = smem_u32(dsm_raw);
  unsigned char* dsm = dsm_raw + (((raw + 1023u) & ~1023u) - raw);
  const TcTile t = tiles[blockIdx.x];
  const TcGroup g = groups[t.group];
  const int KS = g.ks;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&accum, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;

  if (threadIdx.x == 0) {
    auto load_slot = [&](int ks) {
      const int s = ks % kStages;
      unsigned char* st = dsm + s * kStageBytes;
      const int64_t as = g.a_slab0 + 2 * (int64_t(t.tm) * KS + ks);
      const int64_t bs = g.b_slab0 + 2 * (int64_t(t.tn) * KS + ks);
      mbar_expect_tx(&full[s], uint32_t(kStageBytes));
      tma_load(st, &amap, &full[s], 0, int(as * kSlabRows));
      tma_load(st + kSlabBytes, &amap, &full[s], 0, int((as + 1) * kSlabRows));
      tma_load(st + 2 * kSlabBytes, &bmap, &full[s], 0, int(bs * kSlabRows));
      tma_load(st + 3 * kSlabBytes, &bmap, &full[s], 0, int((bs + 1) * kSlabRows));
    };
    bool ok = true;
    int issued = KS < kStages ? KS : kStages;
    for (int ks = 0; ks < issued; ++ks) load_slot(ks);
    int consumed = 0;  // slots whose loads were waited on
    for (int ks = 0; ks < KS; ++ks) {
      const int s = ks % kStages;
      if (!mbar_wait(&full[s], uint32_t((ks / kStages) & 1))) {
        ok = false;
        break;
      }
      consumed = ks + 1;
      tc_fence_after();
      const uint32_t base = smem_u32(dsm + s * kStageBytes);
      const uint64_t ahi = sw128_desc(base), alo = sw128_desc(base + kSlabBytes);
      const uint64_t bhi = sw128_desc(base + 2 * kSlabBytes), blo = sw128_desc(base + 3 * kSlabBytes);
#pragma unroll
      for (int kk = 0; kk < kSlotK / 8; ++kk) {
        const uint64_t adv = uint64_t(kk * 32) >> 4;  // 8 TF32 values = 32 bytes along K
        umma_tf32(tmem, alo + adv, bhi + adv, (ks > 0 || kk > 0) ? 1u : 0u);
        umma_tf32(tmem, ahi + adv, blo + adv, 1u);
        umma_tf32(tmem, ahi + adv, bhi + adv, 1u);
      }
      umma_commit(&empty[s]);
      // refill the previous slot's stage once its MMAs are done (this slot's are still queued)
      if (ks >= 1 && issued < KS) {
        const int sp = (ks - 1) % kStages;
        if (!mbar_wait(&empty[sp], uint32_t(((ks - 1) / kStages) & 1))) {
          ok = false;
          break;
        }
        load_slot(issued);
        ++issued;
      }
    }
    umma_commit(&accum);
    if (!ok) {
      atomicExch(err, 1);
      for (int ks = consumed; ks < issued; ++ks)  // loads still in flight land before we leave
        mbar_wait(&full[ks % kStages], uint32_t((ks / kStages) & 1));
    }
  }
  __syncwarp();
  const bool done = mbar_wait(&accum, 0u);
  if (!done && lane == 0) atomicExch(err, 1);
  tc_fence_after();
  const int row = t.tm * kTileM + warp * 32 + lane;
  const uint32_t lane_addr = tmem + (uint32_t(warp * 32) << 16);
  for (int c0 = 0; c0 < kTileNr; c0 += 16) {
    uint32_t v[16];
    tmem_ld16(lane_addr + uint32_t(c0), v);
    if (done && row < g.m) {
      double2* crow = g.C + int64_t(row) * g.n;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int col = t.tn * kTileN + c0 / 2 + j;
        if (col < g.n)
          crow[col] = make_double2(double(__uint_as_float(v[2 * j])), double(__uint_as_float(v[2 * j + 1])));
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                 : "memory");
  }
}

// ── host: tensor maps ─────────────────────────────────────────────────────────────────────────

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static std::mutex mu;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    BUG_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    bugi::require(q == cudaDriverEntryPointSuccess && p != nullptr,
                  "cuTensorMapEncodeTiled is not available from the driver");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// A 2-D map over `rows` rows of 32 floats (128 bytes), box 32 x 128, 128-byte swizzle.
CUtensorMap slab_map(float* base, int64_t rows) {
  CUtensorMap m;
  const cuuint64_t dims[2] = {cuuint64_t(kSlotK), cuuint64_t(rows)};
  const cuuint64_t strides[1] = {cuuint64_t(kSlotK * 4)};
  const cuuint32_t box[2] = {cuuint32_t(kSlotK), cuuint32_t(kSlabRows)};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr,
                                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  bugi::require(r == CUDA_SUCCESS, "cuTensorMapEncodeTiled failed for the mixed GEMM operands");
  return m;
}

void smem_optin() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  std::lock_guard<std::mutex> lk(mu);
  if (!done[dev]) {
    BUG_CUDA(cudaFuncSetAttribute(tc_cgemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
    done[dev] = true;
  }
}

template <class T>
size_t append(std::vector<char>& blob, const std::vector<T>& v) {
  const size_t off = (blob.size() + 15) & ~size_t(15);
  blob.resize(off + std::max<size_t>(v.size() * sizeof(T), 16));
  if (!v.empty()) std::memcpy(blob.data() + off, v.data(), v.size() * sizeof(T));
  return off;
}

}  // namespace

double run_mixed(bug_ctx* c, const std::vector<bugk::GemmOut>& outs,
                 const std::vector<bugk::GemmPair>& pairs, const std::vector<int>& sel) {
  std::vector<TcGroup> groups;
  std::vector<bugk::GemmPair> gp;
  std::vector<int> koff;
  std::vector<TcTile> tiles;
  std::vector<TcPack> items;
  int64_t aslabs = 0, bslabs = 0;
  double flops = 0.0, bytes = 0.0;
  for (int o : sel) {
    const bugk::GemmOut& go = outs[o];
    TcGroup g{};
    g.C = go.C;
    g.m = go.m;
    g.n = go.n;
    g.pair_begin = int(gp.size());
    int64_t K = 0;
    for (int p = go.pair_begin; p < go.pair_end; ++p) {
      gp.push_back(pairs[p]);
      koff.push_back(int(K));
      K += pairs[p].k;
      flops += 8.0 * double(go.m) * double(go.n) * double(pairs[p].k);
      bytes += 16.0 * (double(go.m) + double(go.n)) * double(pairs[p].k);
    }
    bytes += 16.0 * double(go.m) * double(go.n);
    bugi::require(K < (int64_t(1) << 30), "mixed GEMM: contracted extent too large");
    g.pair_end = int(gp.size());
    g.K = int(K);
    g.ks = int((2 * K + kSlotK - 1) / kSlotK);
    g.mtiles = (go.m + kTileM - 1) / kTileM;
    g.ntiles = (go.n + kTileN - 1) / kTileN;
    g.a_slab0 = aslabs;
    aslabs += 2 * int64_t(g.mtiles) * g.ks;
    g.b_slab0 = bslabs;
    bslabs += 2 * int64_t(g.ntiles) * g.ks;
    const int gi = int(groups.size());
    groups.push_back(g);
    for (int tm = 0; tm < g.mtiles; ++tm)
      for (int tn = 0; tn < g.ntiles; ++tn) tiles.push_back(TcTile{gi, tm, tn});
    for (int tm = 0; tm < g.mtiles; ++tm)
      for (int s = 0; s < g.ks; ++s) items.push_back(TcPack{gi, tm, s, 0});
    for (int tn = 0; tn < g.ntiles; ++tn)
      for (int s = 0; s < g.ks; ++s) items.push_back(TcPack{gi, tn, s, 1});
  }
  if (tiles.empty()) return 0.0;
  // TMA row coordinates are 32-bit
  bugi::require(std::max(aslabs, bslabs) * kSlabRows < (int64_t(1) << 31),
                "mixed GEMM: operands too large for one launch");
  bugi::require(items.size() < (size_t(1) << 31) && tiles.size() < (size_t(1) << 31),
                "mixed GEMM: too many tiles for one launch");
  float* apk = static_cast<float*>(c->scratch(size_t(aslabs) * kSlabBytes));
  float* bpk = static_cast<float*>(c->scratch(size_t(bslabs) * kSlabBytes));
  std::vector<char> blob;
  const size_t o_groups = append(blob, groups), o_pairs = append(blob, gp),
               o_koff = append(blob, koff), o_tiles = append(blob, tiles), o_items = append(blob, items);
  char* dblob = static_cast<char*>(c->scratch(blob.size()));
  void* h = c->stage(blob.size());
  std::memcpy(h, blob.data(), blob.size());
  BUG_CUDA(cudaMemcpyAsync(dblob, h, blob.size(), cudaMemcpyHostToDevice, c->stream));
  c->stage_done();
  const auto* d_groups = reinterpret_cast<const TcGroup*>(dblob + o_groups);
  const auto* d_pairs = reinterpret_cast<const bugk::GemmPair*>(dblob + o_pairs);
  const auto* d_koff = reinterpret_cast<const int*>(dblob + o_koff);
  const auto* d_tiles = reinterpret_cast<const TcTile*>(dblob + o_tiles);
  const auto* d_items = reinterpret_cast<const TcPack*>(dblob + o_items);
  const CUtensorMap amap = slab_map(apk, aslabs * kSlabRows);
  const CUtensorMap bmap = slab_map(bpk, bslabs * kSlabRows);
  smem_optin();
  int* err = c->tc_error_flag();

  c->begin();  // launches the queued FP64 stages first (they may produce A and B)
  tc_pack_kernel<<<unsigned(items.size()), kPackThreads, 0, c->stream>>>(d_groups, d_pairs, d_koff,
                                                                         d_items, apk, bpk);
  c->launched(BUG_K_MIXED, 0.0, double(aslabs + bslabs) * kSlabBytes);
  c->begin();
  tc_cgemm_kernel<<<unsigned(tiles.size()), kTcThreads, kTcSmem, c->stream>>>(amap, bmap, d_groups,
                                                                             d_tiles, err);
  c->launched(BUG_K_MIXED, flops, bytes);
  return flops;
}

}  // namespace bugtc

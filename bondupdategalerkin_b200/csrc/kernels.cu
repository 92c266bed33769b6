// Device kernels of the B200 block-sparse engine. See kernels.cuh for the role of each kernel.
#include "kernels.cuh"

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

namespace bugk {

namespace {

constexpr int kThreads = kStageThreads;
constexpr int kSmCount = 148;  // B200: 2 dies x 74 SMs
constexpr int kElemUnroll = 4;  // elements per thread and pass of the element-wise stages

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename D>
__device__ __forceinline__ int find_desc(const D* d, int nd, int64_t e) {
  int lo = 0, hi = nd - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (d[mid].prefix <= e) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Tensor payloads are read through L2 only (ld.global.cg): a stage may read a block that an
// earlier stage of the same launch wrote on another SM, and a block may be reused for a new tensor
// within one launch, so no SM-local L1 copy may serve a later stage.
__device__ __forceinline__ double2 ldg2(const double2* p) { return __ldcg(p); }

// The descriptor bytes of an inline launch, passed by value in the kernel parameters.
template <int N>
struct ParamBlock {
  alignas(16) unsigned char b[N];
};

// Moves descriptor pointers formed against the arena onto the parameter block when the launch
// carried its descriptors inline (nb > 0); any other pointer is returned unchanged.
struct Rebase {
  const unsigned char* base;
  const char* arena;
  int64_t nb;
  template <class T>
  __device__ __forceinline__ const T* operator()(const T* p) const {
    const char* c = reinterpret_cast<const char*>(p);
    if (nb > 0 && c >= arena && c < arena + nb) return reinterpret_cast<const T*>(base + (c - arena));
    return p;
  }
};

#define BUG_BLOB_PARAMS(N) const __grid_constant__ ParamBlock<N> pb, const char* arena, int64_t nb

// ── copy stage: batched strided gather/scatter ───────────────────────────────────────────────

// `cta` / `ncta`: this CTA's rank among the CTAs that share the stage, and their number (the grid of
// a single-stage launch, or one cluster of a stage list).
__device__ void copy_stage(const Rebase& rb, const CopyDesc* d, int nd, int64_t total, int cta,
                           int ncta) {
  // a thread takes up to kElemUnroll elements per pass (a stride apart) and issues all their loads
  // before any store, so a small grid (one cluster of a stage list) waits for one L2 round trip per
  // pass instead of one per element; each element's arithmetic is unchanged
  const int64_t step = int64_t(ncta) * blockDim.x;
  for (int64_t e0 = cta * int64_t(blockDim.x) + threadIdx.x; e0 < total; e0 += step * kElemUnroll) {
    double2 v[kElemUnroll], o[kElemUnroll];
    double2* dp[kElemUnroll];
    bool acc[kElemUnroll];
#pragma unroll
    for (int u = 0; u < kElemUnroll; ++u) {
      const int64_t e = e0 + u * step;
      dp[u] = nullptr;
      acc[u] = false;
      if (e >= total) continue;
      const CopyDesc& c = d[find_desc(d, nd, e)];
      int64_t r = e - c.prefix;
      int64_t so = 0, dof = 0;
      int64_t widx = 0;
      for (int k = c.ndim - 1; k >= 0; --k) {
        int64_t i = r % c.dims[k];
        r /= c.dims[k];
        so += i * c.sstr[k];
        dof += i * c.dstr[k];
        if (k == c.wdim) widx = i;
      }
      double2 x = c.src ? ldg2(c.src + so) : make_double2(0.0, 0.0);
      if (c.conj) x.y = -x.y;
      if (c.w) {
        const double sc = __ldcg(rb(c.w) + widx);
        x.x *= sc;
        x.y *= sc;
      }
      v[u] = cmul(c.alpha, x);
      dp[u] = c.dst + dof;
      acc[u] = c.accumulate != 0;
      if (acc[u]) o[u] = ldg2(dp[u]);
    }
#pragma unroll
    for (int u = 0; u < kElemUnroll; ++u) {
      if (!dp[u]) continue;
      double2 w = v[u];
      if (acc[u]) {
        w.x += o[u].x;
        w.y += o[u].y;
      }
      *dp[u] = w;
    }
  }
}

// ── gemm stage: segmented grouped complex GEMM ───────────────────────────────────────────────
// Tile 32x32 per CTA, K chunks of 16, 256 threads each owning a 2x2 patch. Every output block is
// covered by its own tiles, and each tile sums over all block pairs of that output block.

constexpr int TM = 32, TN = 32, TK = 16;

__device__ __forceinline__ int64_t group_off(int idx, int n, const int* d, const int64_t* s) {
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

struct GemmSmem {
  double2 As[TM][TK + 1];
  double2 Bs[TK][TN + 1];
};

__device__ void gemm_tile(const GemmOut* outs, const GemmPair* pairs, const GemmTile& t,
                          GemmSmem& sm) {
  const GemmOut o = outs[t.out];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int row0 = t.tm * TM, col0 = t.tn * TN;
  double2 acc[2][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) acc[i][j] = make_double2(0.0, 0.0);

  for (int p = o.pair_begin; p < o.pair_end; ++p) {
    const Operand& A = pairs[p].A;
    const Operand& B = pairs[p].B;
    const int K = pairs[p].k;
    for (int k0 = 0; k0 < K; k0 += TK) {
      for (int i = threadIdx.x; i < TM * TK; i += kThreads) {
        int mm, kk;
        if (A.row_fast) { kk = i / TM; mm = i % TM; } else { mm = i / TK; kk = i % TK; }
        const int gm = row0 + mm, gk = k0 + kk;
        double2 v = make_double2(0.0, 0.0);
        if (gm < o.m && gk < K)
          v = ldg2(A.p + group_off(gm, A.nr, A.rd, A.rs) + group_off(gk, A.nc, A.cd, A.cs));
        if (A.conj) v.y = -v.y;
        sm.As[mm][kk] = v;
      }
      for (int i = threadIdx.x; i < TK * TN; i += kThreads) {
        int kk, nn;
        if (B.row_fast) { nn = i / TK; kk = i % TK; } else { kk = i / TN; nn = i % TN; }
        const int gk = k0 + kk, gn = col0 + nn;
        double2 v = make_double2(0.0, 0.0);
        if (gk < K && gn < o.n)
          v = ldg2(B.p + group_off(gk, B.nr, B.rd, B.rs) + group_off(gn, B.nc, B.cd, B.cs));
        if (B.conj) v.y = -v.y;
        sm.Bs[kk][nn] = v;
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < TK; ++kk) {
        const double2 a0 = sm.As[ty * 2][kk], a1 = sm.As[ty * 2 + 1][kk];
        const double2 b0 = sm.Bs[kk][tx * 2], b1 = sm.Bs[kk][tx * 2 + 1];
        cfma(acc[0][0], a0, b0);
        cfma(acc[0][1], a0, b1);
        cfma(acc[1][0], a1, b0);
        cfma(acc[1][1], a1, b1);
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int gm = row0 + ty * 2 + i;
    if (gm >= o.m) continue;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int gn = col0 + tx * 2 + j;
      if (gn < o.n) o.C[int64_t(gm) * o.n + gn] = acc[i][j];
    }
  }
}

// ── dot stages: deterministic two-phase inner products ──────────────────────────────────────

__device__ void dot_partial(const DotDesc& c, double2* out, double* sr, double* si) {
  double re = 0.0, im = 0.0;
  for (int64_t i = threadIdx.x; i < c.n; i += blockDim.x) {
    const double2 a = ldg2(c.a + i), b = ldg2(c.b + i);
    re = fma(a.x, b.x, fma(a.y, b.y, re));
    im = fma(a.x, b.y, fma(-a.y, b.x, im));
  }
  re = warp_sum(re);
  im = warp_sum(im);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sr[warp] = re;
    si[warp] = im;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tr = 0.0, ti = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) {
      tr += sr[w];
      ti += si[w];
    }
    *out = make_double2(tr, ti);
  }
  __syncthreads();
}

__device__ void dot_reduce(const int* seg, int nout, const double2* partial, double2* out) {
  for (int o = threadIdx.x; o < nout; o += blockDim.x) {
    double tr = 0.0, ti = 0.0;
    for (int k = seg[o]; k < seg[o + 1]; ++k) {
      const double2 p = ldg2(partial + k);
      tr += p.x;
      ti += p.y;
    }
    out[o] = make_double2(tr, ti);
  }
}

// ── lincomb and scale stages ────────────────────────────────────────────────────────────────

__device__ void lincomb_stage(const LinOut* outs, int nout, const LinSrc* srcs, int64_t total,
                              int cta, int ncta) {
  // as copy_stage: up to kElemUnroll elements per thread and pass, loads before stores
  const int64_t step = int64_t(ncta) * blockDim.x;
  for (int64_t e0 = cta * int64_t(blockDim.x) + threadIdx.x; e0 < total; e0 += step * kElemUnroll) {
    double2 res[kElemUnroll];
    double2* dp[kElemUnroll];
#pragma unroll
    for (int u = 0; u < kElemUnroll; ++u) {
      const int64_t e = e0 + u * step;
      dp[u] = nullptr;
      if (e >= total) continue;
      const LinOut& o = outs[find_desc(outs, nout, e)];
      const int64_t i = e - o.prefix;
      double2 acc = make_double2(0.0, 0.0);
      for (int s = o.src_begin; s < o.src_end; ++s) {
        double2 cf = srcs[s].coef;
        if (srcs[s].cmode == 4) {
          cf = make_double2(-__ldcg(srcs[s].cref), -__ldcg(srcs[s].cref + 1));
        } else if (srcs[s].cmode) {
          const double x = __ldcg(srcs[s].cref);
          const double r = sqrt(fmax(x, 0.0));
          cf = make_double2(srcs[s].cmode == 1 ? -x : (srcs[s].cmode == 2 ? 1.0 / r : -r), 0.0);
        }
        cfma(acc, cf, ldg2(srcs[s].src + i));
      }
      res[u] = acc;
      dp[u] = o.dst + i;
    }
#pragma unroll
    for (int u = 0; u < kElemUnroll; ++u)
      if (dp[u]) *dp[u] = res[u];
  }
}

__device__ void scale_stage(const Rebase& rb, const ScaleDesc* d, int nd, int64_t total, int cta,
                            int ncta) {
  for (int64_t e = cta * int64_t(blockDim.x) + threadIdx.x; e < total;
       e += int64_t(ncta) * blockDim.x) {
    const ScaleDesc& c = d[find_desc(d, nd, e)];
    const int64_t i = e - c.prefix;
    const int coord = int((i / c.leg_stride) % c.leg_dim);
    const double w = __ldcg(rb(c.w) + coord);
    const double2 v = ldg2(c.src + i);
    c.dst[i] = make_double2(v.x * w, v.y * w);
  }
}

// ── the stage kernel ─────────────────────────────────────────────────────────────────────────

// One launch = one stage. The dot stage reduces in the same launch: every CTA adds its partial
// sums, and the last CTA to finish (counted on a per-context counter that it resets) sums each
// output's partials in index order, so the result is deterministic.
template <int N>
__global__ void __launch_bounds__(kThreads) stage_kernel(BUG_BLOB_PARAMS(N), const Stage st) {
  __shared__ GemmSmem gsm;
  __shared__ double sr[kThreads / 32], si[kThreads / 32];
  __shared__ bool last;
  const Rebase rb{pb.b, arena, nb};
  switch (st.kind) {
    case kStageCopy:
      copy_stage(rb, rb(static_cast<const CopyDesc*>(st.a)), st.n, st.total, blockIdx.x, gridDim.x);
      break;
    case kStageGemm: {
      const GemmOut* outs = rb(static_cast<const GemmOut*>(st.a));
      const GemmPair* pairs = rb(static_cast<const GemmPair*>(st.b));
      const GemmTile* tiles = rb(static_cast<const GemmTile*>(st.c));
      for (int t = blockIdx.x; t < st.n; t += gridDim.x) gemm_tile(outs, pairs, tiles[t], gsm);
      break;
    }
    case kStageDot: {
      const DotDesc* d = rb(static_cast<const DotDesc*>(st.a));
      for (int i = blockIdx.x; i < st.n; i += gridDim.x) dot_partial(d[i], st.p + i, sr, si);
      unsigned int* counter = st.counter;
      if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
      }
      __syncthreads();
      if (!last) break;
      __threadfence();
      dot_reduce(rb(static_cast<const int*>(st.b)), int(st.total), st.p, st.q);
      if (threadIdx.x == 0) *counter = 0u;
      break;
    }
    case kStageLincomb:
      lincomb_stage(rb(static_cast<const LinOut*>(st.a)), st.n,
                    rb(static_cast<const LinSrc*>(st.b)), st.total, blockIdx.x, gridDim.x);
      break;
    case kStageScale:
      scale_stage(rb, rb(static_cast<const ScaleDesc*>(st.a)), st.n, st.total, blockIdx.x, gridDim.x);
      break;
    default:
      break;
  }
}

// ── stage lists: small stages in order, one cluster each, hardware barriers between them ─────

// One list on the CTAs of this cluster: `cta` is the CTA's rank in the cluster and `ncta` the
// cluster size, so the stage bodies stride over the cluster's CTAs. No CTA leaves early, so every
// CTA reaches every barrier. The barrier (barrier.cluster arrive.release / wait.acquire) orders
// each stage's global writes before the next stage's reads, which go through L2 (ld.global.cg).
__device__ void run_list(const Rebase& rb, const Stage* list, int nstages, int cta, int ncta,
                         GemmSmem& gsm, double* sr, double* si) {
  cooperative_groups::cluster_group cluster = cooperative_groups::this_cluster();
  for (int k = 0; k < nstages; ++k) {
    const Stage st = list[k];
    switch (st.kind) {
      case kStageCopy:
        copy_stage(rb, rb(static_cast<const CopyDesc*>(st.a)), st.n, st.total, cta, ncta);
        break;
      case kStageGemm: {
        const GemmOut* outs = rb(static_cast<const GemmOut*>(st.a));
        const GemmPair* pairs = rb(static_cast<const GemmPair*>(st.b));
        const GemmTile* tiles = rb(static_cast<const GemmTile*>(st.c));
        for (int t = cta; t < st.n; t += ncta) gemm_tile(outs, pairs, tiles[t], gsm);
        break;
      }
      case kStageDot: {
        const DotDesc* d = rb(static_cast<const DotDesc*>(st.a));
        for (int i = cta; i < st.n; i += ncta) dot_partial(d[i], st.p + i, sr, si);
        cluster.sync();  // every partial written before any is summed
        if (cta == 0) dot_reduce(rb(static_cast<const int*>(st.b)), int(st.total), st.p, st.q);
        break;
      }
      case kStageLincomb:
        lincomb_stage(rb(static_cast<const LinOut*>(st.a)), st.n,
                      rb(static_cast<const LinSrc*>(st.b)), st.total, cta, ncta);
        break;
      case kStageScale:
        scale_stage(rb, rb(static_cast<const ScaleDesc*>(st.a)), st.n, st.total, cta, ncta);
        break;
      default:
        break;
    }
    cluster.sync();
  }
}

// One list: the grid is exactly one cluster.
template <int N>
__global__ void __launch_bounds__(kThreads) stage_list_kernel(BUG_BLOB_PARAMS(N),
                                                              const Stage* stages, int nstages) {
  __shared__ GemmSmem gsm;
  __shared__ double sr[kThreads / 32], si[kThreads / 32];
  const Rebase rb{pb.b, arena, nb};
  run_list(rb, rb(stages), nstages, int(blockIdx.x), int(gridDim.x), gsm, sr, si);
}

// Several independent lists (of different contexts) in one launch: cluster i runs list i. The
// lists' descriptors are in their contexts' arenas (nothing inline, nothing to rebase).
__global__ void __launch_bounds__(kThreads) stage_lists_kernel(const __grid_constant__ ListTable lt) {
  __shared__ GemmSmem gsm;
  __shared__ double sr[kThreads / 32], si[kThreads / 32];
  cooperative_groups::cluster_group cluster = cooperative_groups::this_cluster();
  const int ncta = int(cluster.num_blocks());
  const int li = int(blockIdx.x) / ncta;
  const Rebase rb{nullptr, nullptr, 0};
  run_list(rb, lt.stages[li], lt.n[li], int(cluster.block_rank()), ncta, gsm, sr, si);
}

// ── batched one-sided Jacobi SVD ──────────────────────────────────────────────────────────────
// Problem: work = A (mm x r, column-major, mm >= r). Columns are orthogonalised pairwise in a
// round-robin order (r-1 rounds of disjoint pairs per sweep, one warp per pair) until no pair has
// |a_p^H a_q| > m eps |a_p||a_q| -- relative to BOTH columns, so the singular vectors of tiny
// singular values come out orthogonal too. Then sigma_j = |a_j|, sorted descending (ties by
// index), and the phase of each singular pair is fixed on the left vectors of M.

constexpr int kMaxSweeps = 60;
constexpr int kMaxR = 1024;
constexpr int kSvdThreads = 1024;  // launched with one warp per column pair, 8 to 32 warps

__device__ __forceinline__ void rr_pair(int i, int round, int re, int& a, int& b) {
  const int n1 = re - 1;
  if (i == 0) {
    a = round % n1;
    b = n1;
  } else {
    a = (round + i) % n1;
    b = (round + n1 - i) % n1;
  }
}

template <int N>
__global__ void __launch_bounds__(kSvdThreads) jacobi_svd_kernel(BUG_BLOB_PARAMS(N),
                                                              const SvdDesc* descs,
                                                              const CopyDesc* packs,
                                                              double tol_scale) {
  const Rebase rb{pb.b, arena, nb};
  descs = rb(descs);
  packs = rb(packs);
  extern __shared__ double2 dyn[];
  __shared__ double sig[kMaxR];
  __shared__ int perm[kMaxR];
  __shared__ int zero_col[kMaxR];  // 1: numerically zero column, completed orthonormally
  __shared__ double2 coef[kMaxR];
  __shared__ double maxn2, wnorm2;
  __shared__ int rotated;
  const SvdDesc d = descs[blockIdx.x];
  const int mm = d.m > d.n ? d.m : d.n;
  const int r = d.m < d.n ? d.m : d.n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  if (r <= 0) return;
  // gather the sector matrix from the tensor's blocks (column-major M, or M^H)
  for (int pk = d.pack_begin; pk < d.pack_end; ++pk) {
    const CopyDesc& c = packs[pk];
    for (int64_t e = tid; e < c.n; e += blockDim.x) {
      int64_t rr = e, so = 0, dof = 0;
      for (int k = c.ndim - 1; k >= 0; --k) {
        const int64_t i = rr % c.dims[k];
        rr /= c.dims[k];
        so += i * c.sstr[k];
        dof += i * c.dstr[k];
      }
      double2 v = c.src[so];
      if (c.conj) v.y = -v.y;
      c.dst[dof] = v;
    }
  }
  __syncthreads();
  double2* A = d.work;
  double2* V = d.vwork;
  if (d.use_smem) {  // 1: A in shared memory; 2: A and V
    A = dyn;
    if (d.use_smem == 2) V = dyn + int64_t(mm) * r;
    for (int64_t i = tid; i < int64_t(mm) * r; i += blockDim.x) A[i] = d.work[i];
  }
  for (int64_t i = tid; i < int64_t(r) * r; i += blockDim.x)
    V[i] = (i % (r + 1) == 0) ? make_double2(1.0, 0.0) : make_double2(0.0, 0.0);
  __syncthreads();
  // m * eps: the rounding error of the computed a_p^H a_q is itself of order m * eps |a_p||a_q|,
  // so a tighter test can keep near-degenerate or noise-level pairs rotating forever
  const double tol = tol_scale * double(mm);
  // a column at most tol * (largest column norm) long is numerically zero: rotating it against
  // the others only shrinks it further (its direction is rounding noise and never converges), so
  // no pair with such a column is rotated, and afterwards it is replaced by a unit vector
  // orthogonal to all other singular vectors (its singular value stays its tiny norm)
  for (int j = warp; j < r; j += nwarps) {
    const double2* aj = A + int64_t(j) * mm;
    double s2 = 0.0;
    for (int i = lane; i < mm; i += 32) s2 = fma(aj[i].x, aj[i].x, fma(aj[i].y, aj[i].y, s2));
    s2 = warp_sum(s2);
    if (lane == 0) sig[j] = s2;
  }
  __syncthreads();
  if (tid == 0) {
    double mx = 0.0;
    for (int j = 0; j < r; ++j) mx = fmax(mx, sig[j]);
    maxn2 = mx;
  }
  __syncthreads();
  const double negl = tol * tol * maxn2;
  const int re = r + (r & 1);
  int sweep = 0;
  bool converged = (r == 1);
  for (; sweep < kMaxSweeps && !converged; ++sweep) {
    if (tid == 0) rotated = 0;
    __syncthreads();
    for (int round = 0; round < re - 1; ++round) {
      for (int pi = warp; pi < re / 2; pi += nwarps) {
        int a, b;
        rr_pair(pi, round, re, a, b);
        const int p = a < b ? a : b, q = a < b ? b : a;
        if (q >= r) continue;
        double2* ap = A + int64_t(p) * mm;
        double2* aq = A + int64_t(q) * mm;
        double al = 0.0, be = 0.0, gr = 0.0, gi = 0.0;
        for (int i = lane; i < mm; i += 32) {
          const double2 x = ap[i], y = aq[i];
          al = fma(x.x, x.x, fma(x.y, x.y, al));
          be = fma(y.x, y.x, fma(y.y, y.y, be));
          gr = fma(x.x, y.x, fma(x.y, y.y, gr));
          gi = fma(x.x, y.y, fma(-x.y, y.x, gi));
        }
        al = warp_sum(al);
        be = warp_sum(be);
        gr = warp_sum(gr);
        gi = warp_sum(gi);
        // |a_p^H a_q| > tol |a_p| |a_q| tested on squares, so a pair that does not rotate (every
        // pair of the last sweep) costs no square root; the rotation then takes two reciprocal
        // square roots, one square root and one division in sequence. (tol^2 al) be is infinite
        // only where the threshold exceeds every finite g2, so the test is exact wherever g2 is
        // finite and normal, the range in which |a_p^H a_q| itself was computable before.
        const double g2 = gr * gr + gi * gi;
        if (al > negl && be > negl && g2 > (tol * tol * al) * be) {
          if (lane == 0) rotated = 1;
          const double ig = rsqrt(g2);  // 1 / |gamma|
          const double zeta = (be - al) * (0.5 * ig);
          const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
          const double c = rsqrt(1.0 + t * t), s = c * t;
          const double2 e = make_double2(gr * ig, -gi * ig);  // e^{-i phi}, gamma = |gamma| e^{i phi}
          for (int i = lane; i < mm; i += 32) {
            const double2 x = ap[i];
            const double2 ey = cmul(e, aq[i]);
            ap[i] = make_double2(c * x.x - s * ey.x, c * x.y - s * ey.y);
            aq[i] = make_double2(s * x.x + c * ey.x, s * x.y + c * ey.y);
          }
          double2* vp = V + int64_t(p) * r;
          double2* vq = V + int64_t(q) * r;
          for (int i = lane; i < r; i += 32) {
            const double2 x = vp[i];
            const double2 ey = cmul(e, vq[i]);
            vp[i] = make_double2(c * x.x - s * ey.x, c * x.y - s * ey.y);
            vq[i] = make_double2(s * x.x + c * ey.x, s * x.y + c * ey.y);
          }
        }
      }
      __syncthreads();
    }
    converged = (rotated == 0);
    __syncthreads();
  }
  if (tid == 0) *d.sweeps = converged ? sweep : -1;  // host-mapped
  // singular values
  for (int j = warp; j < r; j += nwarps) {
    const double2* aj = A + int64_t(j) * mm;
    double s2 = 0.0;
    for (int i = lane; i < mm; i += 32) s2 = fma(aj[i].x, aj[i].x, fma(aj[i].y, aj[i].y, s2));
    s2 = warp_sum(s2);
    if (lane == 0) {
      sig[j] = sqrt(s2);
      zero_col[j] = s2 <= negl ? 1 : 0;
    }
  }
  __syncthreads();
  // complete the numerically zero columns: for each in turn, two classical Gram-Schmidt passes of
  // a start vector (its own direction, else unit vectors e_k) against every other column's unit
  // vector; accepted when at least half of it survives, stored as a unit vector
  for (int j = 0; j < r; ++j) {
    if (!zero_col[j]) continue;
    double2* aj = A + int64_t(j) * mm;
    for (int attempt = 0; attempt <= mm; ++attempt) {
      const bool own = attempt == 0;
      if (own && !(sig[j] > 0.0)) continue;
      const double sc = own ? 1.0 / sig[j] : 0.0;
      for (int i = tid; i < mm; i += blockDim.x)
        aj[i] = own ? make_double2(aj[i].x * sc, aj[i].y * sc)
                    : make_double2(i == attempt - 1 ? 1.0 : 0.0, 0.0);
      __syncthreads();
      for (int pass = 0; pass < 2; ++pass) {
        for (int k = warp; k < r; k += nwarps) {  // coef_k = u_k^H w (zero for unfinished columns)
          double cr = 0.0, ci = 0.0;
          if (k != j && (!zero_col[k] || zero_col[k] == 2)) {
            const double2* ak = A + int64_t(k) * mm;
            const double inv = zero_col[k] == 2 ? 1.0 : 1.0 / sig[k];
            for (int i = lane; i < mm; i += 32) {
              const double2 u = ak[i], w = aj[i];
              cr = fma(u.x, w.x, fma(u.y, w.y, cr));
              ci = fma(u.x, w.y, fma(-u.y, w.x, ci));
            }
            cr = warp_sum(cr) * inv;
            ci = warp_sum(ci) * inv;
          }
          if (lane == 0) coef[k] = make_double2(cr, ci);
        }
        __syncthreads();
        for (int i = tid; i < mm; i += blockDim.x) {  // w -= sum_k coef_k u_k
          double2 w = aj[i];
          for (int k = 0; k < r; ++k) {
            const double2 c = coef[k];
            if (c.x == 0.0 && c.y == 0.0) continue;
            const double inv = zero_col[k] == 2 ? 1.0 : 1.0 / sig[k];
            const double2 u = A[int64_t(k) * mm + i];
            w.x -= inv * (c.x * u.x - c.y * u.y);
            w.y -= inv * (c.x * u.y + c.y * u.x);
          }
          aj[i] = w;
        }
        __syncthreads();
      }
      if (warp == 0) {
        double n2 = 0.0;
        for (int i = lane; i < mm; i += 32) n2 = fma(aj[i].x, aj[i].x, fma(aj[i].y, aj[i].y, n2));
        n2 = warp_sum(n2);
        if (lane == 0) wnorm2 = n2;
      }
      __syncthreads();
      if (wnorm2 >= 0.25) {
        const double inv = 1.0 / sqrt(wnorm2);
        for (int i = tid; i < mm; i += blockDim.x) aj[i] = make_double2(aj[i].x * inv, aj[i].y * inv);
        __syncthreads();
        if (tid == 0) zero_col[j] = 2;  // completed: a unit vector now
        __syncthreads();
        break;
      }
    }
  }
  for (int j = tid; j < r; j += blockDim.x) {
    const double sj = sig[j];
    int pos = 0;
    for (int k = 0; k < r; ++k) {
      const double sk = sig[k];
      pos += (sk > sj) || (sk == sj && k < j);
    }
    perm[pos] = j;
  }
  __syncthreads();
  const double phi = 1.6180339887498949;
  for (int o = warp; o < r; o += nwarps) {
    const int j = perm[o];
    const double sj = sig[j];
    const double inv = zero_col[j] == 2 ? 1.0 : (sj > 0.0 ? 1.0 / sj : 0.0);
    const double2* aj = A + int64_t(j) * mm;  // left vector of work (times sigma, or completed)
    const double2* vj = V + int64_t(j) * r;   // right vector of work
    double2* uo = d.U + int64_t(o) * d.m;
    double2* vo = d.V + int64_t(o) * d.n;
    // left vectors of M: work's left vectors (no transpose) or work's right vectors (M^H)
    double fr = 0.0, fi = 0.0;
    for (int i = lane; i < d.m; i += 32) {
      double2 u = d.trans ? vj[i] : make_double2(aj[i].x * inv, aj[i].y * inv);
      const double c = 1.0 / (double(i) + phi);
      fr = fma(c, u.x, fr);
      fi = fma(c, u.y, fi);
    }
    fr = warp_sum(fr);
    fi = warp_sum(fi);
    const double fa = sqrt(fr * fr + fi * fi);
    const double2 ph = fa > 0.0 ? make_double2(fr / fa, -fi / fa) : make_double2(1.0, 0.0);
    for (int i = lane; i < d.m; i += 32) {
      double2 u = d.trans ? vj[i] : make_double2(aj[i].x * inv, aj[i].y * inv);
      uo[i] = cmul(u, ph);
    }
    for (int i = lane; i < d.n; i += 32) {
      double2 v = d.trans ? make_double2(aj[i].x * inv, aj[i].y * inv) : vj[i];
      vo[i] = cmul(v, ph);
    }
    if (lane == 0) {
      d.S[o] = sj;
      d.S_host[o] = sj;
    }
  }
}

// ── column-pivoted Householder QR (thin, per charge sector) ────────────────────────────────
// Step k: the remaining column (index >= k) with the largest norm over rows k..m-1 is swapped to
// position k, columns whose squared norm is within kPivotTie (relative) of the largest counting as
// tied and the lowest index winning (the order of columns of numerically equal norm would
// otherwise follow rounding); its Householder reflector H_k = I - tau v v^H (v_k = 1,
// beta real, as LAPACK's zlarfg) zeroes it below the diagonal; H_k^H is applied to the columns
// right of k. Q = H_0 ... H_{kq-1} restricted to its first kq columns, each column scaled by
// sign(beta) so that R_kk >= 0.

constexpr int kQrMaxN = 1024;
constexpr int kQrThreads = 1024;  // launched with one warp per column of the widest sector, 8 to 32 warps
constexpr double kPivotTie = 1e-10;

template <int N>
__global__ void __launch_bounds__(kQrThreads) qr_kernel(BUG_BLOB_PARAMS(N), const QrDesc* descs,
                                                      const CopyDesc* packs) {
  const Rebase rb{pb.b, arena, nb};
  descs = rb(descs);
  packs = rb(packs);
  __shared__ double norms[kQrMaxN];
  __shared__ double2 tau[kQrMaxN];
  __shared__ double beta[kQrMaxN];
  __shared__ int pivot;
  __shared__ double xn2;
  const QrDesc d = descs[blockIdx.x];
  const int m = d.m, n = d.n, kq = m < n ? m : n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  if (kq <= 0 || n > kQrMaxN) return;
  for (int pk = d.pack_begin; pk < d.pack_end; ++pk) {  // gather the sector matrix
    const CopyDesc& c = packs[pk];
    for (int64_t e = tid; e < c.n; e += blockDim.x) {
      int64_t rr = e, so = 0, dof = 0;
      for (int k = c.ndim - 1; k >= 0; --k) {
        const int64_t i = rr % c.dims[k];
        rr /= c.dims[k];
        so += i * c.sstr[k];
        dof += i * c.dstr[k];
      }
      c.dst[dof] = c.src[so];
    }
  }
  __syncthreads();
  double2* A = d.work;
  for (int k = 0; k < kq; ++k) {
    for (int j = k + warp; j < n; j += nwarps) {  // remaining column norms
      const double2* aj = A + int64_t(j) * m;
      double s2 = 0.0;
      for (int i = k + lane; i < m; i += 32) s2 = fma(aj[i].x, aj[i].x, fma(aj[i].y, aj[i].y, s2));
      s2 = warp_sum(s2);
      if (lane == 0) norms[j] = s2;
    }
    __syncthreads();
    if (tid == 0) {  // the lowest index whose squared norm is within kPivotTie of the largest
      int p = k;
      for (int j = k + 1; j < n; ++j)
        if (norms[j] > norms[p]) p = j;
      const double lim = norms[p] * (1.0 - kPivotTie);
      int q = k;
      while (q < p && !(norms[q] >= lim)) ++q;
      pivot = q;
    }
    __syncthreads();
    const int p = pivot;
    if (p != k)
      for (int i = tid; i < m; i += blockDim.x) {
        const double2 t = A[int64_t(k) * m + i];
        A[int64_t(k) * m + i] = A[int64_t(p) * m + i];
        A[int64_t(p) * m + i] = t;
      }
    __syncthreads();
    double2* ak = A + int64_t(k) * m;
    if (warp == 0) {
      double s2 = 0.0;
      for (int i = k + 1 + lane; i < m; i += 32) s2 = fma(ak[i].x, ak[i].x, fma(ak[i].y, ak[i].y, s2));
      s2 = warp_sum(s2);
      if (lane == 0) xn2 = s2;
    }
    __syncthreads();
    const double2 alpha = ak[k];
    double bt, tr, ti;
    double2 scale = make_double2(0.0, 0.0);
    if (xn2 == 0.0 && alpha.y == 0.0) {
      bt = alpha.x;
      tr = 0.0;
      ti = 0.0;
    } else {
      const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2);
      bt = alpha.x >= 0.0 ? -nrm : nrm;
      tr = (bt - alpha.x) / bt;
      ti = -alpha.y / bt;
      const double2 den = make_double2(alpha.x - bt, alpha.y);  // 1 / (alpha - beta)
      const double dd = den.x * den.x + den.y * den.y;
      scale = make_double2(den.x / dd, -den.y / dd);
    }
    __syncthreads();
    if (!(tr == 0.0 && ti == 0.0)) {
      for (int i = k + 1 + tid; i < m; i += blockDim.x) ak[i] = cmul(ak[i], scale);
    }
    if (tid == 0) {
      tau[k] = make_double2(tr, ti);
      beta[k] = bt;
    }
    __syncthreads();
    if (!(tr == 0.0 && ti == 0.0)) {
      // A_j -= conj(tau) v (v^H A_j), j > k
      const double2 ctau = make_double2(tr, -ti);
      for (int j = k + 1 + warp; j < n; j += nwarps) {
        double2* aj = A + int64_t(j) * m;
        double wr = 0.0, wi = 0.0;
        for (int i = k + lane; i < m; i += 32) {
          const double2 v = i == k ? make_double2(1.0, 0.0) : ak[i];
          const double2 x = aj[i];
          wr = fma(v.x, x.x, fma(v.y, x.y, wr));
          wi = fma(v.x, x.y, fma(-v.y, x.x, wi));
        }
        wr = warp_sum(wr);
        wi = warp_sum(wi);
        const double2 f = cmul(ctau, make_double2(wr, wi));
        for (int i = k + lane; i < m; i += 32) {
          const double2 v = i == k ? make_double2(1.0, 0.0) : ak[i];
          const double2 fv = cmul(v, f);
          aj[i] = make_double2(aj[i].x - fv.x, aj[i].y - fv.y);
        }
      }
    }
    __syncthreads();
  }
  // Q columns: q_c = H_0 ... H_{kq-1} e_c, scaled by sign(beta_c)
  for (int c = warp; c < kq; c += nwarps) {
    double2* q = d.Q + int64_t(c) * m;
    for (int i = lane; i < m; i += 32) q[i] = make_double2(i == c ? 1.0 : 0.0, 0.0);
    __syncwarp();
    for (int k = (c < kq - 1 ? c : kq - 1); k >= 0; --k) {  // H_k e_c = e_c for k > c
      const double2 t = tau[k];
      if (t.x == 0.0 && t.y == 0.0) continue;
      const double2* vk = A + int64_t(k) * m;
      double wr = 0.0, wi = 0.0;
      for (int i = k + lane; i < m; i += 32) {
        const double2 v = i == k ? make_double2(1.0, 0.0) : vk[i];
        const double2 x = q[i];
        wr = fma(v.x, x.x, fma(v.y, x.y, wr));
        wi = fma(v.x, x.y, fma(-v.y, x.x, wi));
      }
      wr = warp_sum(wr);
      wi = warp_sum(wi);
      const double2 f = cmul(t, make_double2(wr, wi));
      for (int i = k + lane; i < m; i += 32) {
        const double2 v = i == k ? make_double2(1.0, 0.0) : vk[i];
        const double2 fv = cmul(v, f);
        q[i] = make_double2(q[i].x - fv.x, q[i].y - fv.y);
      }
      __syncwarp();
    }
    const double sg = beta[c] < 0.0 ? -1.0 : 1.0;
    for (int i = lane; i < m; i += 32) q[i] = make_double2(q[i].x * sg, q[i].y * sg);
    if (lane == 0) d.rdiag_host[c] = fabs(beta[c]);
  }
}

}  // namespace

// Launch KERNEL<N> with the smallest parameter block that holds the launch's descriptors, or the
// arena form (N = 16, nothing inline) when the descriptors were copied to the device. LAUNCH is a
// macro taking (kernel instantiation, parameter block, inline byte count).
#define BUG_WITH_BLOB(BLOB, LAUNCH)                                                        \
  do {                                                                                   \
    const Blob& b_ = (BLOB);                                                             \
    const int64_t nb_ = b_.host ? int64_t(b_.bytes) : 0;                                  \
    if (nb_ == 0) {                                                                      \
      ParamBlock<16> p_{};                                                               \
      LAUNCH(16, p_, 0);                                                                 \
    } else if (nb_ <= 512) {                                                             \
      ParamBlock<512> p_;                                                                \
      std::memcpy(p_.b, b_.host, size_t(nb_));                                           \
      LAUNCH(512, p_, nb_);                                                              \
    } else if (nb_ <= 2048) {                                                            \
      ParamBlock<2048> p_;                                                               \
      std::memcpy(p_.b, b_.host, size_t(nb_));                                           \
      LAUNCH(2048, p_, nb_);                                                             \
    } else if (nb_ <= 8192) {                                                            \
      ParamBlock<8192> p_;                                                               \
      std::memcpy(p_.b, b_.host, size_t(nb_));                                           \
      LAUNCH(8192, p_, nb_);                                                             \
    } else {                                                                             \
      ParamBlock<int(kInlineMax)> p_;                                                    \
      std::memcpy(p_.b, b_.host, size_t(nb_));                                           \
      LAUNCH(int(kInlineMax), p_, nb_);                                                  \
    }                                                                                    \
  } while (0)

int stage_items(const Stage& s) {
  switch (s.kind) {
    case kStageCopy:
    case kStageLincomb:
    case kStageScale: {
      const int64_t g = (s.total + kThreads - 1) / kThreads;
      return int(std::min<int64_t>(std::max<int64_t>(g, 1), int64_t(kSmCount) * 16));
    }
    case kStageGemm:
    case kStageDot:
      return std::max(s.n, 1);
    default:
      return 1;
  }
}

// Per-device launch facts shared by every host thread that launches (server workers included).
std::mutex g_launch_mu;

int stage_grid_limit() {
  static int limit[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  std::lock_guard<std::mutex> lk(g_launch_mu);
  if (limit[dev] == 0) {
    int per_sm = 0, sms = kSmCount;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, stage_kernel<int(kInlineMax)>, kThreads, 0);
    limit[dev] = std::max(1, per_sm) * std::max(1, sms);
  }
  return limit[dev];
}

void launch_stage(const Blob& b, const Stage& st, cudaStream_t s) {
  const int grid = std::min(stage_items(st), stage_grid_limit());
#define BUG_STAGE_LAUNCH(NB, P, NBYTES) \
  stage_kernel<NB><<<grid, kThreads, 0, s>>>(P, b.arena, (NBYTES), st)
  BUG_WITH_BLOB(b, BUG_STAGE_LAUNCH);
#undef BUG_STAGE_LAUNCH
}

namespace {
cudaLaunchConfig_t cluster_config(int cluster, int nclusters, cudaStream_t s, cudaLaunchAttribute* attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(cluster * nclusters), 1, 1);
  cfg.blockDim = dim3(kThreads, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = unsigned(cluster);
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

template <int N>
cudaError_t list_launch_n(const ParamBlock<N>& p, const char* arena, int64_t nb, const Stage* st,
                          int n, int cluster, cudaStream_t s) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = cluster_config(cluster, 1, s, attr);
  return cudaLaunchKernelEx(&cfg, stage_list_kernel<N>, p, arena, nb, st, n);
}

// Largest cluster (16, else 8) of which at least one can be resident, for one kernel.
template <class K>
int cluster_for(K kernel) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  for (int c : {16, 8}) {
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = cluster_config(c, 1, nullptr, attr);
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kernel, &cfg) == cudaSuccess && n >= 1) return c;
    cudaGetLastError();
  }
  return 0;
}
}  // namespace

int stage_list_cluster() {
  static int cl[64];
  static bool done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  std::lock_guard<std::mutex> lk(g_launch_mu);
  if (!done[dev]) {
    // every list kernel must allow the size used (they share one code path)
    cl[dev] = std::min({cluster_for(stage_list_kernel<16>), cluster_for(stage_list_kernel<512>),
                        cluster_for(stage_list_kernel<2048>), cluster_for(stage_list_kernel<8192>),
                        cluster_for(stage_list_kernel<int(kInlineMax)>), cluster_for(stage_lists_kernel)});
    done[dev] = true;
  }
  return cl[dev];
}

cudaError_t launch_stage_list(const Blob& b, const Stage* stages, int nstages, int cluster,
                              cudaStream_t s) {
  cudaError_t e = cudaSuccess;
#define BUG_LIST_LAUNCH(NB, P, NBYTES) \
  e = list_launch_n<NB>(P, b.arena, (NBYTES), stages, nstages, cluster, s)
  BUG_WITH_BLOB(b, BUG_LIST_LAUNCH);
#undef BUG_LIST_LAUNCH
  return e;
}

cudaError_t launch_stage_lists(const ListTable& lt, int nlists, int cluster, cudaStream_t s) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = cluster_config(cluster, nlists, s, attr);
  return cudaLaunchKernelEx(&cfg, stage_lists_kernel, lt);
}

void launch_qr(const Blob& b, const QrDesc* d_desc, int nprob, const CopyDesc* packs, int threads,
               cudaStream_t s) {
  if (nprob <= 0) return;
#define BUG_QR_LAUNCH(NB, P, NBYTES) \
  qr_kernel<NB><<<nprob, threads, 0, s>>>(P, b.arena, (NBYTES), d_desc, packs)
  BUG_WITH_BLOB(b, BUG_QR_LAUNCH);
#undef BUG_QR_LAUNCH
}

namespace {
// Opt the SVD kernel's instantiations into large dynamic shared memory once per device.
template <int N>
void svd_smem_optin(int bytes) {
  static int granted[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  std::lock_guard<std::mutex> lk(g_launch_mu);  // the attribute only ever grows
  if (bytes > granted[dev]) {
    cudaFuncSetAttribute(jacobi_svd_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    granted[dev] = bytes;
  }
}
}  // namespace

int svd_smem_limit() {
  static int limit[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  std::lock_guard<std::mutex> lk(g_launch_mu);
  if (limit[dev] == 0) {
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, jacobi_svd_kernel<int(kInlineMax)>);
    limit[dev] = std::max(0, optin - int(fa.sharedSizeBytes) - 1024);
  }
  return limit[dev];
}

void launch_svd(const Blob& b, const SvdDesc* d_desc, int nprob, const CopyDesc* packs,
                int max_smem_bytes, int threads, cudaStream_t s) {
  if (nprob <= 0) return;
  if (max_smem_bytes > 0) {
    const int64_t nb = b.host ? int64_t(b.bytes) : 0;
    if (nb == 0) svd_smem_optin<16>(max_smem_bytes);
    else if (nb <= 512) svd_smem_optin<512>(max_smem_bytes);
    else if (nb <= 2048) svd_smem_optin<2048>(max_smem_bytes);
    else if (nb <= 8192) svd_smem_optin<8192>(max_smem_bytes);
    else svd_smem_optin<int(kInlineMax)>(max_smem_bytes);
  }
#define BUG_SVD_LAUNCH(NB, P, NBYTES)                                                           \
  jacobi_svd_kernel<NB><<<nprob, threads, max_smem_bytes, s>>>(P, b.arena, (NBYTES), d_desc,    \
                                                                 packs, 2.220446049250313e-16)
  BUG_WITH_BLOB(b, BUG_SVD_LAUNCH);
#undef BUG_SVD_LAUNCH
}

}  // namespace bugk

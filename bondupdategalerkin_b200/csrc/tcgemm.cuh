// Mixed-precision grouped complex GEMM on the sm_100a tensor cores (tcgen05, TF32 split in three).
//
// Every output block C_g (m x n complex, row-major) is the sum over its block pairs of A_p B_p,
// which is one GEMM over the pairs' K extents laid end to end. The complex product is embedded in a
// real one: with A as its interleaved (re, im) reals (m x 2K) and B expanded to
//   B_r[2k][2j] = Re B[k][j],  B_r[2k+1][2j] = -Im B[k][j],
//   B_r[2k][2j+1] = Im B[k][j], B_r[2k+1][2j+1] = Re B[k][j]      (2K x 2n),
// A_r B_r is C with (re, im) interleaved, so the output tile is C's own memory layout.
//
// Each FP64 operand value x is split into two TF32 values hi = tf32(x), lo = tf32(x - hi) (about
// 22 significant bits together), and the product is accumulated in FP32 in tensor memory as
// lo*hi + hi*lo + hi*hi ("3xTF32"; the dropped lo*lo term is below the FP32 accumulation error).
// The result carries FP32-level relative error (about 1e-7 of sum |a||b|), not FP64's.
//
// Data path: a pack kernel writes the operands as 128-row slabs of 128-byte rows (32 reals of K),
// hi and lo slabs side by side; the GEMM kernel streams them with TMA (cp.async.bulk.tensor, 128-byte
// swizzle) through a 3-stage shared-memory ring into tcgen05.mma (M = 128, N = 128 reals = 64
// complex columns, K = 8 per instruction) with the accumulator in TMEM, and four warps move the
// finished tile out with tcgen05.ld, widen it to FP64 and store it. Only this GPU's own memory is
// read; no load uses cluster multicast.
#pragma once

#include "kernels.cuh"

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

struct bug_ctx;

namespace bugtc {

constexpr int kTileM = 128;   // output rows per tile (UMMA M)
constexpr int kTileNr = 128;  // real output columns per tile (UMMA N): 64 complex columns
constexpr int kTileN = kTileNr / 2;
constexpr int kSlotK = 32;    // reals of K per slab row: 128 bytes, one swizzle span

// One output block of the mixed path.
struct TcGroup {
  double2* C;        // row-major m x n, leading dimension n
  int m, n;
  int K;             // complex K: the pairs' k summed
  int ks;            // K slots: ceil(2K / 32)
  int pair_begin, pair_end;  // GemmPair range; pair_koff gives each pair's K offset
  int mtiles, ntiles;
  int64_t a_slab0;   // first A slab: tile (tm, slot s) holds hi at a_slab0 + 2 (tm ks + s), lo after it
  int64_t b_slab0;   // first B slab, likewise over (tn, s)
};

struct TcTile {
  int group, tm, tn;
};

// One pack work item: the hi and lo slabs of one (group, tile, K slot) of A (which = 0) or B (1).
struct TcPack {
  int group, tile, slot, which;
};

// True when the mixed path should take this output block (both sides at least min_dim).
inline bool mixed_block(int m, int n, int min_dim) { return m >= min_dim && n >= min_dim; }

// Runs C_g = sum_p A_p B_p for the given output blocks on the tensor cores. `outs` and `pairs` are
// the FP64 planner's host arrays; only the outputs listed in `sel` are computed. Launches the pack
// kernel and the GEMM kernel on the context stream (queued FP64 stages are launched first).
// Returns the algorithmic flops (8 m n k per pair) of the blocks it ran.
double run_mixed(bug_ctx* c, const std::vector<bugk::GemmOut>& outs,
                 const std::vector<bugk::GemmPair>& pairs, const std::vector<int>& sel);

}  // namespace bugtc

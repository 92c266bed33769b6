// Device kernels of the B200 block-sparse engine (sm_100a, complex FP64).
//
// Four kernel families carry every block-sparse operation of the BUG step:
//   * copy_kernel      -- batched strided gather/scatter (permutations, sector packing, direct
//                         sums, trims, conjugation, scaling): the reference's HPTT transposes
//                         (deps/Telum/src/contract.jl:27-167) folded into one launch per operation;
//   * gemm_kernel      -- segmented grouped complex GEMM: every output block is owned by one CTA
//                         tile that loops over all its contributing block pairs, so accumulation
//                         is deterministic and needs no atomics (contract.jl:952-1005);
//   * jacobi_svd_kernel-- batched one-sided (Hestenes) Jacobi SVD, one CTA per charge sector,
//                         sorted, with the engine's phase convention (replaces gesdd,
//                         deps/Telum/src/utils.jl:93-105);
//   * dot/lincomb/scale kernels -- deterministic two-phase reductions and block-union linear
//                         combinations (tensor_inner, norm, Telum's lazy +/-).
#pragma once

#include <cuComplex.h>
#include <cstdint>

namespace bugk {

constexpr int kMaxRank = 6;

struct CopyDesc {
  const double2* src;
  double2* dst;
  int64_t n;        // elements of this descriptor
  int64_t prefix;   // exclusive prefix sum of n over the launch
  int ndim;
  int conj;         // conjugate the source value
  int accumulate;   // dst += alpha*v instead of dst = alpha*v
  int pad_;
  double2 alpha;
  const double* w;  // optional per-index weight along dim `wdim` (singular values for U*S, S*Vd)
  int wdim;
  int pad2_;
  int dims[kMaxRank];
  int64_t sstr[kMaxRank];
  int64_t dstr[kMaxRank];
};

struct GemmOut {
  double2* C;       // row-major m x n, leading dimension n
  int m, n;
  int pair_begin, pair_end;
};

// A GEMM operand viewed as a matrix over two index groups (A: rows = free legs, cols = contracted
// legs in contraction order; B: rows = contracted legs, cols = free legs). Each group is up to
// kGroup dims (C order, last fastest) with element strides, so any leg order of a block is read
// in place -- no transpose pass.
constexpr int kGroup = 4;
struct Operand {
  const double2* p;
  int nr, nc;               // dims in the row / column group (0 = that extent is 1)
  int rd[kGroup], cd[kGroup];
  int64_t rs[kGroup], cs[kGroup];
  int conj;
  int row_fast;             // the row group holds the unit stride: let threads vary along rows
};

struct GemmPair {
  Operand A, B;
  int k;
  int pad_;
};

struct GemmTile {
  int out;
  int tm, tn;
};

struct SvdDesc {
  double2* work;    // mm x r column-major input (M or M^H), overwritten
  double2* vwork;   // r x r column-major scratch (right rotations)
  double2* U;       // m x r column-major output (left vectors of M)
  double2* V;       // n x r column-major output (right vectors of M): M = U diag(S) V^H
  double* S;        // r singular values, descending
  int* sweeps;      // sweeps used (or -1 if the bound was hit)
  int m, n;         // shape of M
  int trans;        // 1: work holds M^H (m < n)
  int use_smem;     // 1: the CTA copies work/vwork into shared memory
  int pack_begin, pack_end;  // gather descriptors that assemble `work` from the tensor's blocks
};

struct DotDesc {
  const double2* a;
  const double2* b;
  int64_t n;
  int out;          // output slot
  int pad_;
};

struct LinOut {
  double2* dst;
  int64_t n;
  int64_t prefix;
  int src_begin, src_end;
};

struct LinSrc {
  const double2* src;
  double2 coef;
};

struct ScaleDesc {
  const double2* src;
  double2* dst;
  int64_t n;
  int64_t prefix;
  int64_t leg_stride;
  int leg_dim;
  int pad_;
  const double* w;
};

void launch_copy(const CopyDesc* d_desc, int ndesc, int64_t total, cudaStream_t s);
void launch_gemm(const GemmOut* outs, const GemmPair* pairs, const GemmTile* tiles, int ntiles,
                 cudaStream_t s);
void launch_svd(const SvdDesc* d_desc, int nprob, const CopyDesc* packs, int max_smem_bytes,
                cudaStream_t s);
void launch_dot(const DotDesc* d_desc, int ndesc, double2* partial, cudaStream_t s);
void launch_dot_fused(const DotDesc* d_desc, int ndesc, double2* partial, const int* seg, int nout,
                      double2* out, unsigned int* counter, cudaStream_t s);
void launch_dot_reduce(const double2* partial, const int* seg_begin, int nout, double2* out,
                       cudaStream_t s);
void launch_lincomb(const LinOut* outs, int nout, const LinSrc* srcs, int64_t total,
                    cudaStream_t s);
void launch_scale(const ScaleDesc* d_desc, int ndesc, int64_t total, cudaStream_t s);

}  // namespace bugk

// Device kernels of the B200 block-sparse engine (sm_100a, complex FP64).
//
// Two kernels carry every block-sparse operation of the BUG step.
//
// stage_kernel runs one operation per launch; its stage kind selects the body:
//   * copy     -- batched strided gather/scatter (permutations, sector packing, direct sums, trims,
//                 conjugation, scaling, zero fills): the reference's HPTT transposes
//                 (deps/Telum/src/contract.jl:27-167) as one launch per operation;
//   * gemm     -- segmented grouped complex GEMM: every output block is owned by tiles that loop
//                 over all its contributing block pairs, so accumulation is deterministic and needs
//                 no atomics (contract.jl:952-1005);
//   * dot      -- deterministic inner products (tensor_inner, norm): partial sums per descriptor,
//                 and the last CTA sums each output's partials in index order into host-mapped
//                 memory;
//   * lincomb, scale -- linear combinations over a union of blocks (Telum's lazy +/-), leg scaling.
// The descriptors of a launch travel inside its kernel parameters when they fit (see Blob).
//
// jacobi_svd_kernel is the batched one-sided (Hestenes) Jacobi SVD, one CTA per charge sector,
// sorted, with the engine's phase convention (replaces gesdd, deps/Telum/src/utils.jl:93-105).
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
  int conj;         // conjugate the source value (a null src reads zeros: a fill)
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
  double* S_host;   // the same values written to host-mapped pinned memory (read after the sync)
  int* sweeps;      // sweeps used (or -1 if the bound was hit), host-mapped pinned memory
  int m, n;         // shape of M
  int trans;        // 1: work holds M^H (m < n)
  int use_smem;     // 1: the CTA keeps work in shared memory; 2: work and vwork
  int pack_begin, pack_end;  // gather descriptors that assemble `work` from the tensor's blocks
};

// One charge sector of a column-pivoted thin QR: `work` (m x n, column-major) is gathered from the
// tensor's blocks by packs [pack_begin, pack_end), overwritten by the reflectors; `Q` receives the
// first kq = min(m, n) columns of Q (column-major, m x kq), each with the phase that makes R_kk
// real non-negative; `rdiag_host` (host-mapped) receives |R_kk|.
struct QrDesc {
  double2* work;
  double2* Q;
  double* rdiag_host;
  int m, n;
  int pack_begin, pack_end;
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

// One source of a linear combination: coef * src, or with `cmode` != 0 a coefficient computed in
// the kernel from the real part x of a dot product the device wrote at `cref` (the recurrence
// coefficients of a Krylov chain that the host has not read back): 1 -> -x, 2 -> 1/sqrt(max(x,0)),
// 3 -> -sqrt(max(x,0)).
struct LinSrc {
  const double2* src;
  double2 coef;
  const double* cref;
  int cmode;
  int pad_;
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

// Where one launch finds its descriptor arrays. The engine forms every descriptor pointer against
// the context's device arena. A launch whose arrays total at most kInlineMax bytes carries them
// inside its kernel parameters (`host` set): no copy precedes the kernel, which rebases pointers
// that fall in [arena, arena + bytes) onto its parameter block. A larger launch reads them from
// the arena, filled by one host-to-device copy before the kernel (`host` null).
struct Blob {
  const void* host;
  size_t bytes;
  const char* arena;
};
constexpr size_t kInlineMax = 32000;  // kernel parameters are limited to 32764 bytes

enum StageKind {
  kStageCopy = 0,     // a: CopyDesc[n], total elements
  kStageGemm = 1,     // a: GemmOut[], b: GemmPair[], c: GemmTile[n]
  kStageDot = 2,      // a: DotDesc[n], b: int seg[total + 1]; p: n partials (scratch);
                      // q[o] = sum of p[seg[o] .. seg[o+1]) in index order (host-mapped)
  kStageLincomb = 4,  // a: LinOut[n], b: LinSrc[], total elements
  kStageScale = 5,    // a: ScaleDesc[n], total elements
};

struct Stage {
  int kind;
  int n;
  int64_t total;
  const void* a;
  const void* b;
  const void* c;
  double2* p;
  double2* q;
  unsigned int* counter;  // dot: the context's last-CTA counter (zero between launches)
};

constexpr int kStageThreads = 256;

// Work items of one stage: its CTA count (capped at the co-resident limit; loops stride).
int stage_items(const Stage& s);
int stage_grid_limit();
void launch_stage(const Blob& b, const Stage& st, cudaStream_t s);

// A list of small stages run in order by ONE launch of one thread-block cluster: every CTA of the
// cluster takes part in every stage (the stage bodies stride over the cluster's CTAs exactly as a
// single-stage launch strides over its grid), and a hardware cluster barrier (release/acquire at
// cluster scope) separates consecutive stages, so each stage sees every earlier stage's writes.
// The arithmetic of every element, tile and partial sum is the single-stage launch's, so results
// are bit-identical; the dot stage reduces its partials after a barrier instead of by a last-CTA
// counter. `stages` is an array in the descriptor blob.
cudaError_t launch_stage_list(const Blob& b, const Stage* stages, int nstages, int cluster,
                              cudaStream_t s);
// CTAs per cluster for stage lists on the current device (16 where the device allows the
// non-portable size, else 8; 0 if no cluster launch is possible).
int stage_list_cluster();

// Stage lists of several contexts launched together: cluster i (of `cluster` CTAs) runs the n[i]
// stages at stages[i], in order, with barriers as above. Their descriptors live in device memory
// (each context's arena), so the kernel rebases nothing.
constexpr int kMaxLists = 128;
struct ListTable {
  const Stage* stages[kMaxLists];
  int n[kMaxLists];
};
cudaError_t launch_stage_lists(const ListTable& lt, int nlists, int cluster, cudaStream_t s);
// Column-pivoted Householder QR, one CTA per sector (see QrDesc).
void launch_qr(const Blob& b, const QrDesc* d_desc, int nprob, const CopyDesc* packs, int threads,
               cudaStream_t s);
// Dynamic shared memory the SVD kernel may use per CTA on this device (opt-in maximum minus its
// static arrays).
int svd_smem_limit();
// `threads`: 256, or 1024 for wide sectors (one warp per column pair of a round).
void launch_svd(const Blob& b, const SvdDesc* d_desc, int nprob, const CopyDesc* packs,
                int max_smem_bytes, int threads, cudaStream_t s);

}  // namespace bugk

/*
 * bug_b200.h -- C-ABI of the B200 block-sparse engine behind the rank-adaptive BUG step.
 *
 * The reference (madhavmen/BondUpdateGalerkin, pure Julia) has no FFI: its hot path calls the
 * block-sparse library Telum, which calls MKL/HPTT per block. This library replaces that layer.
 * Every entry point below is what a Julia host that keeps the sweep logic of
 * `cbe_bug_step!` (src/BUG/TimeEvolution/bug_step.jl:17-513) would `ccall`; the reference
 * function each one stands in for is cited beside it.
 *
 * Conventions
 *   - Plain C types only. Complex numbers are interleaved (re, im) doubles.
 *   - A tensor is block-sparse under an abelian charge (U(1) 2*S^z, or one sector for :none):
 *     each leg has an arrow (+1 out, -1 in) and sorted (charge, dim) sectors; a block, keyed by one
 *     charge per leg, exists only if sum_i dir_i*q_i == 0. Blocks are C-ordered in leg order and
 *     stored in one HBM allocation, in ascending key order. Rank <= 6.
 *   - Tensors are opaque, immutable after creation (every operation returns a new handle; the
 *     reference's ops replace slots and never mutate, src/BUG/Core/Interfaces/state.jl:5-7).
 *   - Every function returns an int status; nothing throws across the ABI. Tolerance verdicts of
 *     the step are ledger fields, never errors (basis_budget.jl:284-299).
 *   - One context per host thread; all work of a context runs on its own CUDA stream.
 */
#ifndef BUG_B200_H
#define BUG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  BUG_OK = 0,
  BUG_EINVAL = 1,      /* bad argument, shape or arrow mismatch (ArgumentError/DimensionMismatch) */
  BUG_ENONFINITE = 2,  /* non-finite data where the reference throws (krylov.jl:80-86) */
  BUG_ENOMEM = 3,      /* device or host allocation failed */
  BUG_ETIMEOUT = 4,    /* a bounded device wait gave up */
  BUG_EDEVICE = 5,     /* CUDA error; bug_last_error() has the text */
  BUG_ENOTCONV = 6     /* an iterative kernel (Jacobi SVD) did not converge in its sweep bound */
};

#define BUG_MAX_RANK 6

typedef struct bug_ctx bug_ctx;
typedef struct bug_tensor bug_tensor;

/* Text of the last error on this thread. */
const char* bug_last_error(void);
/* Library version string. */
const char* bug_version(void);

/* ── context ───────────────────────────────────────────────────────────────────────────────── */
/* No reference counterpart (the reference is one CPU process); owns the stream and the HBM pool. */
int bug_ctx_create(int device, bug_ctx** out);
int bug_ctx_destroy(bug_ctx* ctx);
int bug_ctx_synchronize(bug_ctx* ctx);
/* Kernel launches issued by this context so far (for launch accounting). */
int64_t bug_ctx_launches(const bug_ctx* ctx);
/* Bytes currently held by tensors of this context. */
int64_t bug_ctx_bytes_in_use(const bug_ctx* ctx);
/* The context's CUDA stream (cudaStream_t), for callers that time it with their own events. */
void* bug_ctx_stream(bug_ctx* ctx);

/* Kernel families for bug_ctx_kernel_stats. No reference counterpart: the reference's
 * KernelCounters (src/BUG/Core/diagnostics.jl:17-53) count calls and seconds per kernel family on
 * the CPU; these count device launches, algorithmic flops/bytes and (when profiling) device time. */
enum {
  BUG_K_COPY = 0,     /* strided gathers: permutes, packing, direct sums, trims */
  BUG_K_GEMM = 1,     /* segmented grouped complex GEMM */
  BUG_K_SVD = 2,      /* batched Jacobi SVD */
  BUG_K_DOT = 3,      /* inner products and norms */
  BUG_K_LINCOMB = 4,  /* linear combinations */
  BUG_K_SCALE = 5,    /* leg scaling (U*S, S*Vd) */
  BUG_K_NFAMILIES = 6
};
/* Profiling on: every launch is bracketed by CUDA events on the context stream. */
int bug_ctx_set_profiling(bug_ctx* ctx, int on);
int bug_ctx_kernel_stats(bug_ctx* ctx, int family, int64_t* launches, double* flops, double* bytes,
                         double* device_ms);
int bug_ctx_reset_stats(bug_ctx* ctx);

/* ── tensors: create / upload / download / inspect ────────────────────────────────────────── */
/* A zero tensor with the given legs and block keys (TLArray construction,
 * deps/Telum/TELUM_QUICK_REFERENCE.md:20-60). `nsec[l]` sectors per leg, their charges and dims
 * concatenated leg by leg; `keys` is nblocks*rank charges. Keys are sorted and checked. */
int bug_tensor_create(bug_ctx* ctx, int rank, const int* dirs, const int* nsec,
                      const int* charges, const int* dims, int nblocks, const int* keys,
                      bug_tensor** out);
/* Copy `nelem` complex values (block order, C order within blocks) from host memory. */
int bug_tensor_upload(bug_ctx* ctx, bug_tensor* t, const double* host, int64_t nelem);
/* Copy the payload to host memory (same layout). Synchronises the context stream. */
int bug_tensor_download(bug_ctx* ctx, const bug_tensor* t, double* host, int64_t nelem);
int bug_tensor_free(bug_ctx* ctx, bug_tensor* t);
/* Metadata: rank, number of blocks, total elements, and the sizes `bug_tensor_meta` fills. */
int bug_tensor_shape(const bug_tensor* t, int* rank, int* nblocks, int64_t* nelem, int* total_sectors);
/* dirs[rank], nsec[rank], charges[total_sectors], dims[total_sectors], keys[nblocks*rank]. */
int bug_tensor_meta(const bug_tensor* t, int* dirs, int* nsec, int* charges, int* dims, int* keys);

/* ── algebra ──────────────────────────────────────────────────────────────────────────────── */
/* Telum `contract(A, ia, B, ib)` (deps/Telum/src/contract.jl:2686-2691): paired legs must have
 * opposite arrows after the optional conjugations; the result keeps A's free legs, then B's. Block
 * pairs matched by charge run as one segmented grouped complex-FP64 GEMM launch
 * (contract.jl:952-1005 does one zgemm per pair; HPTT transposes become strided gathers). */
int bug_contract(bug_ctx* ctx, const bug_tensor* a, int n, const int* ia, const bug_tensor* b,
                 const int* ib, int conja, int conjb, bug_tensor** out);
/* Block-sparse SVD over the split `left | rest` with Telum's selection (svd.jl:1825-1921): keep
 * sigma > cutoff*sigma_max, stable descending sort over sectors (ascending charge), then the nkeep
 * largest (nkeep < 0: no limit). U = (left legs.., bond:+1), Vd = (bond:-1, right legs..).
 * Every sector's singular vectors have their phase fixed so that sum_i U[i,k]/(i+phi) is real
 * positive (phi = golden ratio). `sv_all`/`sv_charge` receive every singular value computed (up
 * to `cap` entries, descending) and its sector; `nsv_all` the count, `nkept` how many are kept.
 * Replaces the per-sector LAPACK gesdd of Telum (utils.jl:93-105). */
int bug_svd(bug_ctx* ctx, const bug_tensor* t, int nleft, const int* left, double cutoff,
            int nkeep, bug_tensor** U, bug_tensor** Vd, double* sv_all, int* sv_charge,
            int cap, int* nsv_all, int* nkept);
/* Multiply leg `leg` by per-sector diagonal weights (the `U*S` / `S*Vd` of an SVD result): for
 * each sector charge q of that leg, `w` holds dim(q) reals, sectors in ascending order. */
int bug_scale_leg(bug_ctx* ctx, const bug_tensor* t, int leg, const double* w, bug_tensor** out);
/* sum_b ||block_b||^2 (norm, tlarray/algebra.jl:69-105). */
int bug_norm2(bug_ctx* ctx, const bug_tensor* t, double* out);
/* <a|b> over matching blocks (tensor_inner, symmetric_mps.jl:83-93); zero if none match. */
int bug_inner(bug_ctx* ctx, const bug_tensor* a, const bug_tensor* b, double* out_re_im);
/* <v_i|w> for i < n in one launch (the classical Gram-Schmidt passes, krylov.jl:321-332). */
int bug_inner_many(bug_ctx* ctx, int n, const bug_tensor* const* v, const bug_tensor* w,
                   double* out_re_im);
/* sum_i coef_i * t_i on the union of the blocks (Telum's lazy +/-, materialised once). */
int bug_lincomb(bug_ctx* ctx, int n, const double* coef_re_im, const bug_tensor* const* t,
                bug_tensor** out);
/* Leg permutation (permutedims). */
int bug_permute(bug_ctx* ctx, const bug_tensor* t, const int* perm, bug_tensor** out);
/* Complex conjugate with all arrows flipped (Telum's adjoint `t'`). */
int bug_conj(bug_ctx* ctx, const bug_tensor* t, bug_tensor** out);
/* The same tensor with leg `leg` re-expressed on the opposite arrow (labels negated; shares the
 * payload). The U(1) label of a leg depends on its arrow (sectors.jl:193-206). */
int bug_flip_leg(bug_ctx* ctx, const bug_tensor* t, int leg, bug_tensor** out);
/* Direct sum along `leg` (oplus, tlarray/oplus.jl:451-504). */
int bug_oplus(bug_ctx* ctx, int n, const bug_tensor* const* t, int leg, bug_tensor** out);
/* Keep the leading counts[s] entries of sector s (ascending sector order) of `leg`
 * (_trim_per_sector, truncation.jl:283-288). *out is NULL when nothing is kept. */
int bug_trim(bug_ctx* ctx, const bug_tensor* t, int leg, const int* counts, bug_tensor** out);

#ifdef __cplusplus
}
#endif

#endif /* BUG_B200_H */

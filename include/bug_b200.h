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
  BUG_K_MIXED = 6,    /* tensor-core (tcgen05, 3xTF32) grouped complex GEMM and its operand pack */
  BUG_K_NFAMILIES = 7
};
/* Profiling on: every launch is bracketed by CUDA events on the context stream. */
int bug_ctx_set_profiling(bug_ctx* ctx, int on);
int bug_ctx_kernel_stats(bug_ctx* ctx, int family, int64_t* launches, double* flops, double* bytes,
                         double* device_ms);
int bug_ctx_reset_stats(bug_ctx* ctx);
/* Mixed precision (the BUG step's contractions, bug_contract and everything built on them): an
 * output block whose row and column extents are both at least `min_dim` is computed on the tensor
 * cores as a 3xTF32 split product with FP32 accumulation (relative error about 1e-7 of
 * sum |a||b| instead of FP64's 1e-16); smaller blocks, the SVD/QR factorisations, the Krylov
 * recurrences' inner products and every reduction stay in FP64. min_dim <= 0 turns it off (the
 * default: everything in FP64). No reference counterpart (the reference computes in FP64 only,
 * deps/Telum/src/contract.jl:952-1005). */
int bug_ctx_set_mixed(bug_ctx* ctx, int min_dim);
/* Host-side accounting since the last reset: how many times the host waited for the stream to
 * read a result back (norms, inner products, singular values), the seconds spent waiting, the
 * seconds spent inside kernel-launch calls, and the seconds spent in the stream-ordered
 * allocator. No reference counterpart (the reference runs on the CPU and waits for nothing). */
int bug_ctx_host_stats(bug_ctx* ctx, int64_t* syncs, double* wait_s, double* launch_s,
                       double* alloc_s);

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
/* Many tensors through one flat host layout (no reference counterpart: the reference's tensors
 * live in host memory; a host that keeps an MPS and MPO there moves them with one call each way).
 * Tensor i's metadata sits at meta + meta_off[i]: rank r, r arrows, r sector counts, every
 * sector's charge (leg by leg, ascending within a leg), every sector's dimension (same order),
 * the block count nb and nb x r block keys (ascending); its payload, complex interleaved, blocks in
 * key order and each C-ordered, at payload_off[i] complex values into `payload`.
 * bug_tensors_from_host creates and uploads n tensors (through pinned staging, no wait);
 * bug_tensors_layout gives each tensor's metadata length (ints) and payload size (complex values);
 * bug_tensors_to_host writes n tensors' metadata and payloads with ONE synchronisation. */
int bug_tensors_from_host(bug_ctx* ctx, int n, const int* meta, const int64_t* meta_off,
                          const double* payload, const int64_t* payload_off, bug_tensor** out);
int bug_tensors_layout(int n, const bug_tensor* const* t, int64_t* meta_len, int64_t* nelem);
int bug_tensors_to_host(bug_ctx* ctx, int n, const bug_tensor* const* t, int* meta,
                        const int64_t* meta_off, double* payload, const int64_t* payload_off);

/* ── algebra ──────────────────────────────────────────────────────────────────────────────── */
/* Telum `contract(A, ia, B, ib)` (deps/Telum/src/contract.jl:2686-2691): paired legs must have
 * opposite arrows after the optional conjugations; the result keeps A's free legs, then B's. Block
 * pairs matched by charge run as one segmented grouped complex-FP64 GEMM launch
 * (contract.jl:952-1005 does one zgemm per pair; HPTT transposes become strided gathers). */
int bug_contract(bug_ctx* ctx, const bug_tensor* a, int n, const int* ia, const bug_tensor* b,
                 const int* ib, int conja, int conjb, bug_tensor** out);
/* Orthonormal basis of the span of the leg-`leg` columns of `t` (`_thin_qr`,
 * src/BUG/Randomised/dd_cbe.jl:184-259): per charge sector of that leg, the sector's blocks stacked
 * row-wise (ascending keys; rows = the other legs in C order) and a column-pivoted Householder QR
 * (LAPACK geqp3's pivot rule, as Julia's qr(A, ColumnNorm())); the leading Q columns whose |R_kk|
 * exceeds `thr` are kept, each with the phase that makes R_kk real positive. The new leg has arrow
 * `ref_dir` and keeps the charge (negated when the arrow flips). A sector is at most 1024 columns
 * wide (BUG_EINVAL otherwise). *out = NULL when nothing is kept. */
int bug_thin_qr(bug_ctx* ctx, const bug_tensor* t, int leg, int ref_dir, double thr,
                bug_tensor** out);
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

/* ── the whole step ───────────────────────────────────────────────────────────────────────── */
/* Keyword arguments of `cbe_bug_step!` (bug_step.jl:17-148); a non-positive value selects the
 * reference default noted beside it (TOL_DEFAULTS, basis_budget.jl:568; DDQRExpansion,
 * src/BUG/Randomised/cbe.jl:254-290). */
/* Saves (op 0) or restores (op 1) the caller's Gaussian stream: the outside-residual
 * measurement draws from a copy of the stream (the reference measures with `copy(rng)`,
 * bug_step_stages.jl:309-317), so the step's own draws continue from the saved state. */
typedef void (*bug_rng_ctl_fn)(void* user, int op);

/* Fills `n` standard normal reals; the step consumes them pairwise as (re, im) scaled by
 * sqrt(1/2), probe by probe: sectors in ascending charge, one C-ordered matrix over the fused
 * space per sector (the caller's seeded generator stands in for the reference's `rng`,
 * bug_step.jl:147). */
typedef void (*bug_normal_fn)(void* user, int64_t n, double* out);

/* parallel = true: the right half of a sweep draws from a stream of its own, seeded by ONE 64-bit
 * draw from the step's stream at the point the reference calls `MersenneTwister(rand(rng,
 * UInt64))` (bug_step.jl:225 for the half-sweeps, frontier_closure.jl:125 for each frontier
 * sweep). The callee takes that draw from the step's stream, makes the new stream and returns its
 * normal-draw callback in *draw / *draw_user (valid until the step returns; called from another
 * thread than the step's). Returns 0, or non-zero to fail the step. */
typedef int (*bug_rng_fork_fn)(void* user, bug_normal_fn* draw, void** draw_user);

typedef struct {
  double tol_basis;           /* <= 0: 1e-5 */
  double tol_trunc;           /* < 0: 1e-7 */
  double tol_expv;            /* <= 0: 1e-10 */
  double tol_krylov;          /* <= 0: tol_basis */
  int order;                  /* temporal order p >= 1 */
  int maxdim;                 /* <= 0: 128 */
  int hermitian;              /* 1: Lanczos root solve, 0: Arnoldi */
  int work_ceiling_rule;      /* 0: :bond, 1: :maxdim, 2: :bond_strict, 3: :frame_root */
  double bond_ceiling_factor; /* < 0: 1.2 under :bond, 0 under :maxdim */
  int root;                   /* root link; <= 0: L/2 */
  int reorth;                 /* re-orthogonalise the root Lanczos basis */
  int truncate;               /* run the final compression */
  int root_maxiter;           /* <= 0: 30 */
  int fixed_width;            /* DD sketch width (:rank_tail); <= 0: 8 */
  double tail_factor;         /* :rank_tail acceptance share; <= 0: 0.10 */
  int krylov_mode;            /* 0 :auto, 1 :lanczos, 2 :arnoldi */
  int krylov_fixed_depth;     /* 0: residual-controlled stop */
  int dd_mode;                /* DD expansion rule: 0 :rank_tail (tail_dd), 1 :adaptive
                                 (_dd_controller, dd_cbe_controller.jl:26-212) */
  int holdout_width;          /* :adaptive holdout columns; <= 0: 4 */
  int batch_blocks;           /* :adaptive blocks per holdout, 1..8; <= 0: 1 */
  int cap_selection;          /* :adaptive past the cap: 0 :storage (first sectors), 1 :svd */
  double acceptance_factor;   /* :adaptive acceptance, (0, 1]; <= 0: 1 */
  double eshift;              /* the generators are H - eshift (shift_h, effective_operators.jl:110-129) */
  int root_report;            /* fill the info's root report (_report_root!, bug_step_stages.jl:243-390) */
  int outside_residual;       /* with root_report: measure |tau| ||(I-P) H psi_1|| / ||psi_1|| and
                                 re-enrich on it (at most 2 order + 2 passes); needs rng_ctl */
  bug_rng_ctl_fn rng_ctl;
  void* rng_ctl_user;
  int closure_checks;         /* order > 1: measure every frontier first and close them in passes
                                 (_krylov_closure! with checks = true,
                                 krylov_closure_loop.jl:18-194) instead of the single pass */
  int root_method;            /* root integrator (root_methods.jl:12-345): 0 exp, 1 trapezoid,
                                 2 radau2, 3 radau3 (one implicit stage on the Krylov basis),
                                 4 radau2_gmres (the coupled stages by shifted GMRES) */
  int root_noshift;           /* 1: no imaginary-time spectral shift of the implicit roots
                                 (`root_shift = false`) */
  int parallel;               /* 1: parallel = true (:half_sweeps): the two half-sweeps, and the two
                                 halves of every frontier sweep, run at once on two streams driven
                                 by two host threads (bug_step.jl:222-268,
                                 frontier_closure.jl:121-145); needs rng_fork */
  bug_rng_fork_fn rng_fork;
  void* rng_fork_user;
  int exact;                  /* 1: exact = true, the deterministic reference: every DD expansion
                                 sketches the complete fused basis with the opposite frame projected
                                 out (_dd_probe(...; exact = true), dd_cbe.jl:140-161) and keeps what
                                 _dd_select's QR admits in one pass (dd_cbe_expand.jl:91,346-360) */
  int fold_omega;             /* 0: the reference's default, folded above order 1 unless exact
                                 (bug_step_stages.jl:67); 1: folded closures, sampled frontier leaks;
                                 2: the exact leak of the formed two-site action
                                 (krylov_frontier_bonds.jl:80-100) */
  int n_keep;                 /* keep_states: how many MPS the trial space must contain; each
                                 half-sweep unions their carried sites into its frames
                                 (_union_fresh, half_sweeps.jl:143-204) */
  const bug_tensor* const* keep_sites; /* n_keep x L borrowed site handles, state-major (state k's
                                 site i at [k L + i]), legs as psi's; read during the call only */
  const double* keep_tols;    /* n_keep entries or NULL (all 0): 0 contains the state exactly,
                                 > 0 admits only its directions carrying more than ~tol of it; under
                                 work_ceiling_rule :bond an admitted state fills a frame only up to
                                 its bond's ceiling */
  int frames_only;            /* 1: skip the root solve; the state comes back as psi in the frames
                                 (bug_step.jl:381-382); needs truncate = 0 and no root report */
  double root_ceiling_factor; /* :frame_root's root-bond factor, in (1, frame factor]; <= 0: 1.2 */
  bug_tensor** frames_out;    /* frames_report: NULL, or 2L slots the step fills with new handles
                                 owned by the caller (bug_step.jl:455-467): [b-1] the left frame of
                                 bond b for b <= root, [L-2+b] the right frame of bond b for
                                 b >= root (NULL elsewhere), [2L-2] and [2L-1] the root's left and
                                 right environments */
} bug_step_params;


#define BUG_MAX_SITES 1024

/* One bond visit of a sweep (the ledger's bond_log, basis_budget.jl:399-436). side 0 left, 1 right. */
typedef struct {
  int bond, side;
  double sample, tail, krylov_c, krylov_d;
  int64_t n_probes, n_selected, n_krylov, n_h1;
  int c_pass, d_after_c, workcap, met, unmet_mask, width, r_old, r_final;
  double discarded;
} bug_bond_log;

/* CBEBugSweepInfo + AdaptiveLedger fields (diagnostics.jl:209-255, basis_budget.jl:144-228).
 * status 0 = :met, 1 = :budget_unmet; unmet bits / unmet_order codes (1-based): 1 sample, 2 tail,
 * 3 krylov, 4 trunc, 5 projection, 6 expv, 7 closure. */
typedef struct {
  int status;
  int unmet_mask;
  int unmet_order[8];
  int root_link, root_rank, root_frame_width;
  double discarded;
  int64_t n_matvec;
  double max_sample, max_tail, max_krylov, max_krylov_c, max_krylov_d, ledger_discarded, expv_err;
  int64_t expv_iters, n_probes, n_selected, n_krylov, n_h1, n_c_pass, n_d_after_c;
  int workcap_reached, maxdim_reached;
  double proj_err;
  int64_t r_old, r_aug, r_final, n_passes, n_closure_sweeps;
  double defect;
  int64_t n_root_frontier, n_h1_closure, n_compress;
  double leak1;
  int expanded[BUG_MAX_SITES];
  int n_new[BUG_MAX_SITES];
  int workcap[BUG_MAX_SITES];
  int64_t n_holdout, n_targeted; /* holdout probe columns; sectors targeted (:adaptive) */
  /* root report (NaN where not measured): Rayleigh-quotient energies of the root start and
   * result (+ eshift), the outside defect before and after re-enrichment, its left/right parts
   * and bound relative to ||psi_1||, the re-enrichment passes and directions added */
  double e_pre, e_root, resid, resid_initial, outside, outside_left, outside_right;
  int outside_passes, outside_added;
  int64_t n_h2_leak; /* two-site applications that measured a frontier leak (fold_omega = false) */
} bug_step_info;

/* One rank-adaptive BUG step in place: `cbe_bug_step!(psi, mpo, tau; ...)`
 * (src/BUG/TimeEvolution/bug_step.jl:17-513), DD-QR :rank_tail, :adaptive or exact expansion,
 * Lanczos/Arnoldi local Krylov, order-p single-pass or checked closure with folded (sampled) or
 * exact frontier leaks, :exp or implicit root. `psi_io[L]` holds the
 * state's site handles on entry; on return each slot holds a new handle owned by the caller, or
 * NULL where the caller's handle is unchanged. The MPO handles are only read. */
int bug_mps_step(bug_ctx* ctx, int L, bug_tensor** psi_io, int* center_io,
                 const bug_tensor* const* mpo, double tau_re, double tau_im,
                 const bug_step_params* params, bug_normal_fn draw, void* user,
                 bug_step_info* info, bug_bond_log* bond_log, int bond_log_cap, int* n_bond_log);

/* ── kernel-granular entry points ─────────────────────────────────────────────────────────
 * The pieces of the step for a host that keeps the sweep logic itself (a Julia `ccall` shim).
 * Inputs are borrowed; each output is a new handle owned by the caller. Layouts follow the
 * engine's arrow conventions: MPS site (link_l:-1, site:-1, link_r:+1); MPO (w_l:-1, s_in:+1,
 * s_out:-1, w_r:+1); left environment (bra:-1, w:+1, ket:+1); right environment (bra:+1, w:-1,
 * ket:-1). */

/* Chain-end environments (the `nothing` ends of mpo_environments.jl:141-175, explicit here):
 * side 0 left (trivial), 1 right (carrying `charge`, the state's total charge). */
int bug_env_boundary(bug_ctx* ctx, int side, int charge, bug_tensor** out);
/* One environment push E -> A^dagger (E A W): side 0 `_mpo_left_step`, 1 `_mpo_right_step`
 * (mpo_environments.jl:65-108). */
int bug_env_step(bug_ctx* ctx, int side, const bug_tensor* env, const bug_tensor* A,
                 const bug_tensor* W, bug_tensor** out);
/* H1 x for the local Krylov (`apply_one_site`, effective_operators.jl:27-64). */
int bug_apply_one_site(bug_ctx* ctx, const bug_tensor* lenv, const bug_tensor* W,
                       const bug_tensor* renv, const bug_tensor* x, bug_tensor** out);
/* H0 S = sum_w L[w] S R[w] (`apply_zero_site`, effective_operators.jl:91-107); `lgen`/`rgen` are
 * the environments pushed through the bond's expanded left / right frames. */
int bug_apply_zero_site(bug_ctx* ctx, const bug_tensor* lgen, const bug_tensor* rgen,
                        const bug_tensor* core, bug_tensor** out);
/* The streamed two-site sketch X Om with Theta never formed (`_stream_left`/`_stream_right`,
 * mpo_environments.jl:409-481): side 0 with a = U0 S0 (l, s, b), b = V0 and a probe in V0's
 * layout (g, s_r, l_r), out (l_l, s_l, g); side 1 with a = U0, b = S0 V0 and a probe
 * (l_l, s_l, g), out (g, s_r, l_r). Wl, Wr: the bond's MPO sites. */
int bug_sketch_stream(bug_ctx* ctx, int side, const bug_tensor* a, const bug_tensor* b,
                      const bug_tensor* Wl, const bug_tensor* Wr, const bug_tensor* lenv,
                      const bug_tensor* renv, const bug_tensor* probe, bug_tensor** out);
/* (I - U U^dagger) K: side 0 `perp_component` (a left frame over legs 0, 1), 1
 * `perp_component_right` (a right frame over legs 1, 2) (sectors.jl:215-240). */
int bug_perp(bug_ctx* ctx, int side, const bug_tensor* frame, const bug_tensor* K,
             bug_tensor** out);
/* The root Galerkin exponential exp(tau H0) core (`expv`, root_methods.jl:359-402: `lanczos_expv`
 * krylov.jl:128-263 when `hermitian`, else `arnoldi_expv` :343-442) with the Saad tail against
 * `tol_expv` and adaptive substeps; `iters` = H0 applications, `err` = the accumulated tail. */
int bug_root_expv(bug_ctx* ctx, const bug_tensor* lgen, const bug_tensor* rgen,
                  const bug_tensor* core, double tau_re, double tau_im, int hermitian, int maxiter,
                  int reorth, double tol_expv, bug_tensor** out, int64_t* iters, double* err);
/* Normalised local populations of every site (`site_expval` of the diagonal projectors,
 * local_observables.jl:11-24): per site, the site leg's indices in leg order (sectors
 * ascending, then index); `n` = the total count (at most `cap` written). */
int bug_site_populations(bug_ctx* ctx, int L, const bug_tensor* const* psi, int center,
                         double* out, int cap, int* n);
/* <S^z_j> for every site of a spin-1/2 chain (`sz_expectation`/`magnetisation`,
 * local_observables.jl:11-24, bond_observables.jl:15): under U(1) the site charge is 2 S^z;
 * under :none the one charge-0 sector holds up (index 0) and down (index 1). */
int bug_observable_sz(bug_ctx* ctx, int L, const bug_tensor* const* psi, int center, double* out);

/* H Theta for a two-site tensor (l, s1, s2, r) (`apply_h_two_site`, mpo_environments.jl:316-344). */
int bug_apply_two_site(bug_ctx* ctx, const bug_tensor* lenv, const bug_tensor* Wl,
                       const bug_tensor* Wr, const bug_tensor* renv, const bug_tensor* theta,
                       bug_tensor** out);

/* ── two-site TDVP, the reference's matched-accuracy baseline ─────────────────────────────
 * `tdvp2_step!(psi, h, tau; ...)` (src/Baselines/TDVP/tdvp2.jl:229-297). Keyword defaults in
 * brackets are the reference's; a zero-initialised struct gets them except `substeps` and
 * `hermitian`, which the caller sets (the reference's defaults: 1 and 1). */
typedef struct {
  int maxdim;          /* <= 0: 200 */
  double trunc_thresh; /* Telum relative cutoff of each split (at least 1e-14); < 0: 1e-12 */
  int maxiter;         /* Krylov dimension per exponential; <= 0: 30 */
  double tol;          /* Krylov breakdown; <= 0: 1e-15 */
  int hermitian;       /* 1 Lanczos, 0 Arnoldi */
  double conv_tol;     /* Saad tail stop; 0: none */
  int substeps;        /* 1 one step of each tau, > 1 equal substeps, 0 adaptive */
  double weight_tol;   /* < 0: cut by trunc_thresh; >= 0: the BUG's budgeted cut
                          weight_tol ||Theta|| / (sqrt(r - 1) + sqrt(L - r)), r = root link + 1 */
  double eshift;       /* integrate H - eshift (imaginary time) */
} bug_tdvp2_params;

/* TDVP2Info (tdvp2.jl:17-24). */
typedef struct {
  int max_bond;
  int64_t theta_elements; /* largest two-site tensor formed (stored elements) */
  double discarded;       /* largest relative weight one split discarded */
  int64_t peak_elements;  /* state + largest two-site tensor */
  int64_t krylov_dims;    /* operator applications */
  double cumulative;      /* relative discarded norm, accounted as in truncate_recursive! */
} bug_tdvp2_info;

/* One symmetric two-site TDVP step of `tau` in place (forward sweep of exp(tau/2 H2) updates with
 * backward exp(-tau/2 H1) half-steps, then the mirror sweep). Handles as in bug_mps_step: each
 * slot of `psi_io` returns a new handle owned by the caller, or NULL where unchanged. */
int bug_tdvp2_step(bug_ctx* ctx, int L, bug_tensor** psi_io, int* center_io,
                   const bug_tensor* const* mpo, double tau_re, double tau_im,
                   const bug_tdvp2_params* params, bug_tdvp2_info* info);

/* ── serving: many jobs on one GPU ─────────────────────────────────────────────────────────
 * No reference counterpart: the reference calls cbe_bug_step! one chain at a time. A server owns
 * `workers` threads, each with its own context (stream, memory, staging); jobs wait in one FIFO
 * queue and start when a worker is idle and the running jobs' projected footprints plus the new
 * one fit `budget_bytes` (a job always starts when nothing runs). Running jobs overlap on the
 * device (one stream each) and on the host cores; a job's result is the same as alone. */
typedef struct bug_server bug_server;

enum { BUG_JOB_QUEUED = 0, BUG_JOB_RUNNING = 1, BUG_JOB_DONE = 2, BUG_JOB_FAILED = 3,
       BUG_JOB_CANCELLED = 4 };

/* Build the job's state (L site handles, centre) and MPO (L handles) on `ctx`, the worker's
 * context; the server owns the handles afterwards. Return BUG_OK or an error code. Called on the
 * worker thread. `psi` and `mpo` have room for BUG_MAX_SITES + 1 handles. */
typedef int (*bug_job_load_fn)(void* user, bug_ctx* ctx, int* L, bug_tensor** psi, int* center,
                               bug_tensor** mpo);
/* Read the job's final state (the handles stay the server's and are freed after the call).
 * `status` is BUG_OK or the failing step's code. Called on the worker thread. */
typedef void (*bug_job_done_fn)(void* user, bug_ctx* ctx, int status, int L,
                                bug_tensor* const* psi, int center);

typedef struct {
  double tau_re, tau_im;     /* step size */
  int nsteps;                /* steps of cbe_bug_step! */
  bug_step_params params;
  bug_normal_fn draw;        /* the job's own Gaussian stream */
  void* draw_user;
  bug_job_load_fn load;
  bug_job_done_fn done;      /* may be NULL */
  void* user;
  int64_t footprint_bytes;   /* projected HBM need at maxdim (bug_projected_footprint) */
} bug_job_spec;

typedef struct {
  int state;                 /* BUG_JOB_* */
  int status;                /* BUG_OK or the failing call's code */
  int worker;                /* the worker that ran it (-1: never started) */
  int steps_done;
  double t_submit, t_start, t_end;  /* seconds since the server started */
  double step_s_sum, step_s_max;    /* per-step latency (stream drained), sum and maximum */
} bug_job_stats;

int bug_server_create(int device, int workers, int64_t budget_bytes, bug_server** out);
int bug_server_submit(bug_server* s, const bug_job_spec* spec, int64_t* job_id);
/* A queued job leaves the queue at once; a running one stops after its current step. */
int bug_server_cancel(bug_server* s, int64_t job_id);
/* Wait until job `job_id` (or every job, job_id <= 0) has finished, or `timeout_s` passes
 * (negative: no limit). `finished` tells which. */
int bug_server_wait(bug_server* s, int64_t job_id, double timeout_s, int* finished);
int bug_server_job_stats(bug_server* s, int64_t job_id, bug_job_stats* out);
/* The job's per-step latencies in seconds (up to cap; n = how many there are). */
int bug_server_step_times(bug_server* s, int64_t job_id, double* out, int cap, int* n);
/* Cancels queued jobs, lets running ones stop after their step, joins the workers. */
int bug_server_destroy(bug_server* s);
/* The failing call's message of a failed job ("" otherwise), truncated to cap - 1 bytes. */
int bug_server_job_error(bug_server* s, int64_t job_id, char* buf, int cap);
/* Kernel launches issued by all workers so far. */
int64_t bug_server_launches(const bug_server* s);
/* Projected HBM bytes of one chain at bond dimension maxdim: state, environment stacks, one
 * bond's Krylov basis and probes and the two-site work tensors, doubled for temporaries. */
int64_t bug_projected_footprint(int L, int d, int maxdim, int mpo_dim);

/* ── batched steps ──────────────────────────────────────────────────────────────────────────
 * Many independent chains stepped together (the batched caller of `cbe_bug_step!`,
 * src/BUG/TimeEvolution/bug_step.jl:17-513, which the reference runs one chain at a time). A batch
 * owns n engine contexts and n host threads; each chain's sweep logic runs on its own thread and
 * context, so the chains' host work and their kernels overlap. With `combine` != 0 the contexts
 * share ONE stream and the small stages each chain queues between its read-backs are merged with
 * the other chains' into one launch (a thread-block cluster per chain); with 0 (recommended: on
 * B200 a stream per chain measured 3x the throughput) each context keeps its own stream. Every
 * chain's result is bit-identical to its own bug_mps_step either way (the kernels are
 * deterministic, each chain draws from its own generator). Build chain i's state and MPO on
 * bug_batch_context(b, i); a chain's tensors must stay on its context and be freed before
 * bug_batch_destroy. Up to 128 chains. */
typedef struct bug_batch bug_batch;
int bug_batch_create(int device, int n, int combine, bug_batch** out);
int bug_batch_context(bug_batch* b, int i, bug_ctx** out);
/* One step of chains 0..n-1 (n <= the batch's size), each argument indexed by chain as
 * bug_mps_step's; status[i] is chain i's return code, and the call returns the first failing code
 * (bug_last_error names the chain). */
int bug_step_batch(bug_batch* b, int n, const int* L, bug_tensor** const* psi_io, int* center_io,
                   const bug_tensor* const* const* mpo, const double* tau_re, const double* tau_im,
                   const bug_step_params* params, bug_normal_fn draw, void* const* draw_user,
                   bug_step_info* info, int* status);
/* Kernel launches issued for the batch so far (merged stage-list launches counted once). */
int64_t bug_batch_launches(const bug_batch* b);
int bug_batch_destroy(bug_batch* b);

/* ── host small-matrix routines of the step (no device work; usable without a GPU) ────────── */
/* exp(A) for a complex n x n row-major matrix (Pade-13 scaling and squaring); replaces Julia's
 * matrix `exp` in _kry_weight/_hess_coeffs (krylov_enrichment.jl:89-120, root_methods.jl:136-141). */
int bug_la_expm(int n, const double* a, double* out);
/* The step's per-bond work ceilings from the bond dimensions before it (bond_work_ceilings,
 * bond_work_ceilings_strict, bond_frame_root_ceilings, work_ceiling; basis_budget.jl:454-555):
 * rule 0 :bond, 1 :maxdim, 2 :bond_strict, 3 :frame_root; factor < 0 is bond_ceiling_factor's
 * default, root_factor <= 0 is root_ceiling_factor's (1.2); root_link is the root bond (1-based).
 * Writes nbonds ceilings to out; BUG_EINVAL with the reference's reason for a refused factor. */
int bug_work_ceilings(int rule, int nbonds, const int64_t* bonds, int64_t site_dim, int64_t maxdim,
                      double factor, int root_link, double root_factor, int64_t* out);
/* Eigen-decomposition of a real symmetric n x n matrix (cyclic Jacobi): ascending eigenvalues and
 * eigenvectors as columns (row-major n x n). */
int bug_la_eigh(int n, const double* a, double* vals, double* vecs);
/* Eigen-decomposition of the symmetric tridiagonal matrix with diagonal d (n) and off-diagonal e
 * (n - 1) by implicit QR steps with Wilkinson shifts: ascending eigenvalues and eigenvectors as
 * columns (row-major n x n); replaces syevr in _tridiag_eigen (krylov.jl:77-98), the step's
 * Lanczos tridiagonal. A non-finite entry returns BUG_ENONFINITE, as _tridiag_eigen throws. */
int bug_la_eigh_tridiag(int n, const double* d, const double* e, double* vals, double* vecs);
/* Eigenvalues of a complex upper-Hessenberg n x n matrix; replaces geev in _hess_coeffs. */
int bug_la_eigvals_hess(int n, const double* a, double* vals_re_im);
/* The Krylov weight of v_{k+1} in exp(tau H) v_1 for the n x n Hessenberg matrix H (row-major,
 * interleaved re/im): |H[k, k-1]| |tau| int_0^1 |(exp(s tau H_k) e_1)[k-1]| ds by composite Simpson
 * in log space, normalised by the propagated seed's norm when state_seed (_kry_weight and
 * _residual_integral, src/BUG/Core/RankAdaptation/krylov_enrichment.jl:58-120). k is 1-based,
 * 1 <= k < n. */
int bug_la_kry_weight(int n, const double* hm, int k, double tau_re, double tau_im, int state_seed,
                      double* out);

/* ── allocation-free inner product ──────────────────────────────────────────────────────── */
/* No counterpart in the reference: added for callers that cannot allocate GPU memory at the call
 * site -- a process whose device memory budget is fixed up front, a host callback or library hook
 * where cudaMalloc is forbidden, or code that must not create or use an engine context (contexts
 * allocate). Computes out[0] + i*out[1] = sum_i conj(a_i) * b_i for `n` interleaved complex
 * doubles at device pointers `a` and `b`, writing the result to the device pointer `out`, on
 * `stream` (a cudaStream_t; NULL is the default stream). a, b and out must be 16-byte aligned
 * (BUG_EINVAL otherwise, before anything runs). The reduction scratch is a static device array of
 * 64 KiB + 256 B (65,792 bytes) held by every device that loads this library until the process
 * exits; n may be at most 8,388,608 (larger n returns BUG_EINVAL). The first call on a device looks
 * the array up with cudaGetSymbolAddress and should come before any stream capture; the address is
 * kept for the process, so calls assume the device's primary context and no cudaDeviceReset in
 * between. Calls on one device share the array: calls whose kernels overlap on the GPU race, so
 * serialise them. No cudaMalloc, cudaFree or allocating library routine is called. */
int bug_inner_noalloc(const double* a, const double* b, int64_t n, double* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BUG_B200_H */

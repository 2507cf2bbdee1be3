/*
 * mfgpu.h -- B200 (sm_100a) numeric phase of CliqueTrees.jl's Multifrontal
 * submodule behind a plain C ABI (no torch or CUDA types in the signatures).
 *
 * The reference numeric phase is two Julia functions over flat arrays:
 *   chol_impl!(Mptr, Mval, Dptr, Dval, Lptr, Lval, d, Fval, res, rel, chd,
 *              uplo, S, R, diag)        src/Multifrontal.jl/src/cholesky.jl:361-392
 *   div_impl!(B, Mptr, Mval, Dptr, Dval, Lptr, Lval, Fval, res, rel, chd,
 *             tA, tB, uplo, side, diag) src/Multifrontal.jl/src/divide.jl:417-450
 * reached from factorize! (cholesky.jl:304-315) and ldiv! (divide.jl:167-199,
 * :1762-1764).  This library replaces both.  A Julia caller passes the
 * ChordalSymbolic arrays once (mf_create), then calls mf_chol_impl /
 * mf_div_impl with the same Dval/Lval/d/B arrays the reference uses.
 *
 * Conventions
 *   - every index array is 0-based int64 (a Julia shim subtracts 1);
 *   - matrices are column major, values float64;
 *   - Dval: per front nn x nn (lower triangle used) at Dptr[j];
 *     Lval: per front na x nn at Lptr[j]  (UPLO = :L layout,
 *     chordal_factorization.jl:146-167);
 *   - info follows the reference: 0 = success, k > 0 = 1-based column (in
 *     the elimination order) of the first rejected pivot (cholesky.jl:384-388);
 *     the caller maps it through perm as factorize! does (cholesky.jl:250-254);
 *   - return codes: 0 ok, -1 bad argument, -2 invalid symbolic input,
 *     -3 CUDA error, -4 out of device memory; mf_last_error() explains.
 *   - one handle = one pattern + its device factor; a handle is used by one
 *     host thread at a time; all work runs on the handle's stream.
 */
#ifndef MFGPU_H
#define MFGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mf_handle mf_handle;

/* Upload a ChordalSymbolic (chordal_symbolic.jl:15-28) and allocate the
 * device factor.  diag: 0 = Cholesky (ChordalCholesky, DIAG=:N),
 * 1 = LDLt (ChordalLDLt, DIAG=:U).  nrhs_cap: largest number of right-hand
 * sides solved per pass (<= 16; larger blocks are processed in chunks).
 * Arrays: resptr, sepptr, Dptr, Lptr: nfr+1; septgt, reltgt: sepptr[nfr];
 * chdptr: nfr+2; chdtgt: nfr (children ascending, roots in list nfr).
 * Replaces: ChordalFactorization(P, S) allocation, chordal_factorization.jl:146-167,
 * and the workspaces FactorizationWorkspace (cholesky.jl:15-24) and
 * DivisionWorkspace (divide.jl:13-18). */
int mf_create(int64_t n, int64_t nfr, const int64_t* resptr, const int64_t* sepptr, const int64_t* septgt,
              const int64_t* reltgt, const int64_t* chdptr, const int64_t* chdtgt, const int64_t* Dptr,
              const int64_t* Lptr, int diag, int nrhs_cap, int device, mf_handle** out);

void mf_destroy(mf_handle* h);

/* Run the work of a handle on a caller-owned CUDA stream (a cudaStream_t
 * passed as void*); NULL restores the handle's own stream. */
int mf_set_stream(mf_handle* h, void* stream);

/* Full reference-equivalent factorization with host arrays:
 * Dval/Lval hold the assembled matrix on entry and the factor on exit (in
 * place, as chol_impl! does); d receives the LDLt pivots (length n, may be
 * NULL for Cholesky); signs (length n, may be NULL) are the pivot signs S
 * of NoRegularization (no_regularization.jl:27-42): NULL means all ones for
 * Cholesky and all zeros for LDLt.
 * Replaces chol_impl!, cholesky.jl:361-392. */
int mf_chol_impl(mf_handle* h, double* Dval, double* Lval, double* d, const double* signs, int64_t* info);

/* Natural-factorization solve with host arrays: B (n x nrhs, leading
 * dimension ldb, elimination order) <- (L D L^T)^{-1} B, or (L L^T)^{-1} B.
 * Uses the factor left on the device by the last factorization.
 * Replaces ldiv!(W, NaturalFactorization(F), B) = div_impl! forward, D,
 * div_impl! backward, divide.jl:191-199, :417-450. */
int mf_div_impl(mf_handle* h, double* B, int64_t nrhs, int64_t ldb);

/* ---- device-resident path (pattern cached on the device) ---------------- */

/* Assembly map: slot[k] = flat 0-based index into [Dval; Lval] of the k-th
 * stored value the caller will pass to mf_assemble (flatindices,
 * chordal_symbolic.jl:731-752).  Uploaded once per pattern. */
int mf_set_assembly(mf_handle* h, int64_t nnz, const int64_t* slot);

/* Refill the device factor from nonzero values (host pointer), i.e.
 * fill!(F, 0); setflatindex!(F, v, slot) (chordal_factorization.jl:322-338). */
int mf_assemble(mf_handle* h, const double* nzval);

/* Same with a device pointer (values already in HBM). */
int mf_assemble_device(mf_handle* h, const double* nzval_dev);

/* Factor the device-resident values (chol_impl! without host copies).
 * info as above (host int64); signs may be NULL (see mf_chol_impl). */
int mf_factorize(mf_handle* h, const double* signs, int64_t* info);

/* x = A^{-1} b with the permutation applied on the device, host buffers:
 * B (n x nrhs, leading dimension ldb, ORIGINAL order) is overwritten with
 * the solution; perm (length n) is the elimination order (perm[i] = original
 * vertex at position i).  Replaces ldiv!!(C, F, B), divide.jl:1762-1764.
 * perm NULL reuses the permutation last passed to this handle (the identity
 * before any). */
int mf_solve(mf_handle* h, double* B, int64_t nrhs, int64_t ldb, const int64_t* perm);

/* Same with device pointers (B_dev n x nrhs, leading dimension ldb). */
int mf_solve_device(mf_handle* h, double* B_dev, int64_t nrhs, int64_t ldb, const int64_t* perm_dev);

/* ---- mixed precision (FP32 fronts, FP64 refinement) -------------------- */

/* Allocate the single-precision factor and the refinement workspace (after
 * mf_set_assembly).  From then on mf_assemble only stages the values.  The
 * FP64 factor storage (panels, update matrices, block inverses) is released
 * and allocated again only when a factorization needs it (mf_factorize, or a
 * mixed factorization that falls back to FP64); the FP64 solves and
 * mf_get_factor fail until then. */
int mf_enable_mixed(mf_handle* h);

/* Scale A symmetrically by diag(|a_ii|)^-1/2, factor it in FP32 (same plan,
 * single-precision kernels) and compute ||A||_inf.  Every front (nj <= 96)
 * and every 64 x 64 diagonal block of a larger front whose FP32 pivots are
 * rejected, lost more than five digits against their diagonal entry, or grew
 * beyond 1e7 times the block's largest diagonal entry is factored again in
 * FP64 on the GPU and stored rounded to FP32 (mf_rescued counts them).  If a
 * pivot is rejected even then (or in FP32 in a small front with nj > 67),
 * the matrix is refactored in FP64 and *used_fp64 = 1; info then follows the
 * FP64 factorization (the reference's convention). */
int mf_factorize_mixed(mf_handle* h, const double* signs, int64_t* info, int* used_fp64);

/* Fronts and diagonal blocks that the last factorization refactored in FP64
 * after the single-precision pivot check flagged them (see
 * mf_factorize_mixed).  No reference counterpart. */
int mf_rescued(mf_handle* h, int64_t* count);

/* Autotuning of the single-precision factorization (no reference
 * counterpart: the reference has one dense kernel per role).  For every tree
 * level, times the level's GEMM roles (left-looking, TRSM, trailing update;
 * and the SYRK of the update matrix) with the tcgen05 tensor-core tiles and
 * with the FFMA tiles on the handle's current values, `reps` timed runs
 * after one warm-up each, and keeps the faster variant per level and role.
 * The handle's factor is overwritten: call mf_factorize_mixed afterwards.
 * ms (may be NULL) receives 6 values: GEMM-role milliseconds with tcgen05
 * everywhere, with FFMA everywhere, with the tuned choice; levels that kept
 * tcgen05 for the panel steps, for the SYRK; number of levels. */
int mf_autotune(mf_handle* h, int reps, double* ms);
/* The per-level choice (1 = tcgen05, 0 = FFMA), one entry per tree level
 * (mf_info out[7] levels); either array may be NULL. */
int mf_kernel_choice(const mf_handle* h, int32_t* tc_steps, int32_t* tc_syrk);
int mf_set_kernel_choice(mf_handle* h, const int32_t* tc_steps, const int32_t* tc_syrk);

/* x = A^-1 b to normwise backward error <= tol in FP64 with the FP32 factor
 * as preconditioner: conjugate gradients (Cholesky) or GMRES (LDLt); when
 * segments are set (mf_set_segments) every segment runs its own recurrence
 * and is refined to its own backward error.  B (n x nrhs, ORIGINAL order)
 * is overwritten with x.  *iters and *eta report the worst right-hand side. */
int mf_solve_refined(mf_handle* h, double* B, int64_t nrhs, int64_t ldb, const int64_t* perm, double tol, int maxit,
                     int* iters, double* eta);
int mf_solve_refined_device(mf_handle* h, double* B_dev, int64_t nrhs, int64_t ldb, const int64_t* perm_dev,
                            double tol, int maxit, int* iters, double* eta);

/* The single-precision factor of the scaled matrix S A S (reference layout,
 * widened to double) and the scaling S (elimination order). */
int mf_get_factor_mixed(mf_handle* h, double* Dval, double* Lval, double* d, double* scale);

/* Copy the device factor out in the reference layout (any pointer may be NULL). */
int mf_get_factor(mf_handle* h, double* Dval, double* Lval, double* d);

/* Pivot rule of the FP64 factorizations (mf_factorize, mf_chol_impl):
 * mode 0 = NoRegularization (the default; no_regularization.jl:27-42),
 * mode 1 = DynamicRegularization (dynamic_regularization.jl:75-90): a pivot
 * d_j with s_j d_j < epsilon is replaced by delta s_j (s = the pivot signs;
 * ones for Cholesky); delta / epsilon < 0 take the reference defaults
 * cbrt(eps) and sqrt(eps).  mf_factorize_mixed refuses a handle with
 * mode 1.  Replaces the `reg` keyword of cholesky! / ldlt!
 * (src/Multifrontal.jl/src/cholesky.jl:80-229). */
int mf_set_regularization(mf_handle* h, int mode, double delta, double epsilon);

/* Selected inversion (Cholesky handles): after mf_factorize, replace the
 * FP64 factor on the device by the entries of A^{-1} on the sparsity pattern
 * of L (lower triangle of each diagonal block); mf_get_factor then returns
 * them in the reference layout, and the solves refuse until the next
 * factorization.  Replaces selinv!(F), src/Multifrontal.jl/src/selinv.jl:38-41.
 * Synchronises the handle's stream. */
int mf_selinv(mf_handle* h);

/* log|det A| and sign(det A) of the matrix last factored on this handle,
 * reduced on the device from the factor's diagonal: Cholesky 2 sum log L_jj
 * with sign +1, LDLt sum log|d_j| with the sign of prod d_j; a zero pivot
 * gives -inf and sign 0.  A mixed handle whose factor is single precision
 * uses it and the scaling (log|det A| = log|det S A S| - 2 sum log s_j), to
 * single-precision accuracy.  Replaces logabsdet / logdet / det of a
 * factorization, src/Multifrontal.jl/src/abstract_factorization.jl:156-179.
 * Synchronises the handle's stream. */
int mf_logdet(mf_handle* h, double* logabsdet, double* sign);

/* Wait for the handle's stream.  Returns -3 if a bounded device wait of
 * the work it ran timed out (the tensor-core pipeline, or the one-launch
 * super-block solve chain), so the result of the asynchronous calls
 * (mf_solve_device, mf_solve_device_static) is incomplete; mf_solve,
 * mf_div_impl and the refined solves check the same before they return. */
int mf_synchronize(mf_handle* h);

/* Sizes: out[0..8] = n, nfr, ndz, nlz, panel values, update values,
 * device bytes allocated, number of tree levels, execution fronts. */
int mf_info(const mf_handle* h, int64_t* out);

/* Residual and separator sizes of the execution fronts (mf_info out[8]
 * entries each), for flop accounting. */
int mf_exec_sizes(const mf_handle* h, int64_t* nn, int64_t* na);

/* Parent of every execution front (mf_info out[8] entries; -1 for roots),
 * for counting the algorithmic bytes of the extend-add. */
int mf_exec_parents(const mf_handle* h, int64_t* parent);

/* Host-only inspection of the execution plan a handle would use (no CUDA
 * call): out[0..6] = execution fronts after amalgamation, tree levels,
 * panel values, update-matrix pool values, solve-update pool rows, work
 * items, factorization launches.  Arguments as for mf_create. */
int mf_plan_info(int64_t n, int64_t nfr, const int64_t* resptr, const int64_t* sepptr, const int64_t* septgt,
                 const int64_t* reltgt, const int64_t* chdptr, const int64_t* chdtgt, const int64_t* Dptr,
                 const int64_t* Lptr, int nrhs_cap, int64_t* out);

/* Optional per-kernel timing (CUDA events around every launch, stream
 * synchronised after each: for profiling passes only).  mf_kernel_times
 * fills ms[18] and launches[18] in the order: assemble, small, extend-add,
 * panel TRSM, trailing update, syrk, solve-small, solve-gather, solve-fwd,
 * solve-bwd-l, solve-bwd, permute, other, diagonal blocks, left update,
 * residual; then two counters that are not kernels (ms 0): solve passes
 * and the right-hand-side columns they solved. */
int mf_profile(mf_handle* h, int enable);
int mf_kernel_times(const mf_handle* h, double* ms, int64_t* launches);

const char* mf_last_error(void);

/* ---- solve without device allocation ----------------------------------- */

/* mf_solve_device with its work buffers taken from one fixed 32 MiB device
 * region (a file-scope __device__ array) instead of the handle's: the call
 * allocates no device memory.  For callers that must not reach the device
 * allocator while solving, e.g. a serving loop whose device memory is already
 * fully committed under an admission cap, or one that keeps the handle's own
 * solve buffers busy on another stream.  No reference counterpart.
 *
 * A chunk of c = min(nrhs, 16) right-hand sides needs 2*n*c + R*c + 1024*P
 * doubles (R, P fixed by the plan; each part rounded up to 256 bytes); a solve
 * that needs more than 4,194,304 doubles returns -1 with the sizes in
 * mf_last_error() and does nothing.  Nothing in the region has to start at
 * zero.  The first call on a device looks up the region's address
 * (cudaGetSymbolAddress, which loads the module holding it); make that first
 * call before any stream capture.  There is one region per device shared by
 * every handle: two calls whose work overlaps on the device race and corrupt
 * each other's results, so serialise them (same stream, or an event between).
 * Work runs on the handle's stream and is not synchronised. */
int mf_solve_device_static(mf_handle* h, double* B_dev, int64_t nrhs, int64_t ldb, const int64_t* perm_dev);

/* ---- batches of independent matrices ------------------------------------ */

/* Split the rows (elimination order) into nseg independent segments,
 * segptr[0] = 0 <= segptr[1] <= ... <= segptr[nseg] = n.  Used when the
 * handle holds a batch of matrices as one block-diagonal forest (their
 * ChordalSymbolic arrays concatenated): the mixed refinement then measures
 * the normwise backward error of every segment separately, refines with
 * x += M^-1 (b - A x) so segments stay independent, and stops when the
 * worst segment meets the tolerance.  nseg = 0 removes the split.
 * No reference counterpart (the reference factors one matrix per object). */
int mf_set_segments(mf_handle* h, int64_t nseg, const int64_t* segptr);

/* Per-segment backward error (worst right-hand side) of the last refined
 * solve; eta has nseg entries. */
int mf_segment_errors(mf_handle* h, double* eta);

#ifdef __cplusplus
}
#endif

#endif

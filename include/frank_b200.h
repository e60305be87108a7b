/*
 * frank_b200.h -- C ABI of the B200 engine for FRANK's BLR-LU
 * factor-and-solve path.
 *
 * Plain pointers and sizes only; no torch or CUDA types cross this boundary
 * (streams are passed as `void*` holding a cudaStream_t, NULL = default).
 * Host buffers are ordinary host memory (pinned or not); `_device` variants
 * take device pointers.
 *
 * Each entry point names the FRANK interface it replaces (paths within the
 * FRANK project).  A plan ("frank_blr") is one block-low-rank matrix resident
 * on one GPU: the FP64 compressed matrix A_H (kept for the residual of
 * iterative refinement) plus a working copy in the factorization precision
 * that getrf overwrites with its L and U factors.
 *
 * Thread safety: a plan is not thread-safe; distinct plans may be used from
 * distinct host threads.  The library keeps no other mutable global state
 * apart from the per-thread error string.
 */
#ifndef FRANK_B200_H
#define FRANK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes returned by every entry point. */
enum {
  FRANK_OK = 0,
  FRANK_ERR_INVALID = 1,        /* bad argument (see frank_last_error) */
  FRANK_ERR_SINGULAR = 2,       /* a leaf getrf met an exactly zero pivot */
  FRANK_ERR_UNSUPPORTED = 3,    /* block-type combination not supported */
  FRANK_ERR_NOT_CONVERGED = 4,  /* refinement did not reach the tolerance */
  FRANK_ERR_TIMEOUT = 5,        /* a bounded device-side wait gave up */
  FRANK_ERR_CUDA = 6,           /* a CUDA runtime call failed */
  FRANK_ERR_RANK_OVERFLOW = 7,  /* a recompressed rank exceeded the capacity */
  FRANK_ERR_STATE = 8           /* call out of order (e.g. solve before getrf) */
};

/* Arithmetic of the factorization (the refinement residual is always FP64). */
enum {
  FRANK_PREC_FP64 = 0,   /* plain FP64 factor */
  FRANK_PREC_MIXED = 1   /* FP32 bulk factor, FP64 leaf getrf / core SVD */
};

/* Block types (classes/dense.h, classes/low_rank.h). */
enum { FRANK_BLOCK_DENSE = 0, FRANK_BLOCK_LOWRANK = 1 };

/* Kernel functions for on-device construction (functions.cpp:92-128 and the
 * two kernels of the batched / adjoint workloads). */
enum {
  FRANK_KERNEL_LAPLACE = 0,     /* 1/(r+1e-3)                  functions.cpp:92-109 */
  FRANK_KERNEL_HELMHOLTZ = 1,   /* exp(-r^2)/(r+1e-3)          functions.cpp:111-128 */
  FRANK_KERNEL_NEGLOG = 2,      /* -log(r+1e-3) + p0*delta_ij  */
  FRANK_KERNEL_EXP = 3          /* exp(-r/p0) + p1*delta_ij    */
};

typedef struct frank_blr frank_blr;

typedef struct frank_blr_desc {
  int64_t n;          /* matrix order */
  int32_t nb;         /* blocks per side; block sizes follow IndexRange::split
                         (index_range.cpp:15-24): ceil(n/nb), last takes the rest;
                         ceil(n/nb) <= 810 (the recompression keeps its
                         Householder panels in shared memory) */
  int32_t max_rank;   /* rank capacity of every low-rank block (0 = block size) */
  int32_t precision;  /* FRANK_PREC_* */
  int32_t fixed_rank; /* >0: recompress to this rank (LowRank fixed-rank mode);
                         0: truncate by eps (find_svd_truncation_rank, misc.cpp:133-146) */
  double eps;         /* truncation tolerance of the factorization */
  double admis;       /* position-based admissibility: block (i,j) is low rank
                         iff |i - j| > admis (matrix_initializer.cpp:51-58);
                         diagonal blocks are always dense */
} frank_blr_desc;

/* Text of the last error on the calling thread ("" if none). */
const char* frank_last_error(void);

/* Library / device information: compiled arch, device name, SM count. */
int frank_device_info(char* name, int name_len, int* sm_count, int* cc_major, int* cc_minor);

/* Create a plan on the current CUDA device.  Replaces the allocation side of
 * Hierarchical(n_row_blocks, n_col_blocks) (classes/hierarchical.cpp:46-47). */
int frank_blr_create(const frank_blr_desc* desc, frank_blr** out);

/* Create a plan whose admissibility is geometry-based: off-diagonal block
 * (i, j) is low rank iff admis^2 diam^2 < dist^2 for the bounding boxes of
 * its row and column points padded by 0.5 (AdmisType::GeometryBased,
 * classes/initialization_helpers/matrix_initializer.cpp:51-91).  points:
 * dim x n, axis-major (params[d][i], functions.h:34-38), host FP64; desc->admis
 * is the admissibility constant. */
int frank_blr_create_geometric(const frank_blr_desc* desc, const double* points, int dim, frank_blr** out);

/* Free all device memory of the plan. */
int frank_blr_destroy(frank_blr* plan);

/* Block geometry: offsets[nb+1] of the block rows/columns. */
int frank_blr_offsets(const frank_blr* plan, int64_t* offsets);

/* Set block (i, j) of A_H to a dense matrix (host, FP64).  `rowmajor` selects
 * the layout of `a` with leading dimension `ld`.  Replaces
 * MatrixInitializer::get_dense_representation (matrix_initializer.cpp:28-34). */
int frank_blr_set_dense(frank_blr* plan, int i, int j, const double* a, int64_t ld, int rowmajor);

/* Set block (i, j) of A_H to U (m x k) S (k x k) V (k x n), host FP64.
 * Replaces LowRank(U, S, V) (classes/low_rank.cpp:61-69). */
int frank_blr_set_lowrank(frank_blr* plan, int i, int j, int rank,
                          const double* U, int64_t ldu, const double* S, int64_t lds,
                          const double* V, int64_t ldv, int rowmajor);

/* Build A_H on the device from points (dim x n, axis-major like the
 * reference's params[d][i], functions.h:34-38): diagonal and inadmissible
 * blocks dense, admissible blocks compressed by truncated column-pivoted QR
 * + RQ (LowRank(Dense, eps), low_rank.cpp:50-59 with geqp3.cpp:71-192) when
 * eps > 0, or by randomized SVD to the plan's fixed rank when eps = 0
 * (LowRank(Dense, rank), low_rank.cpp:40-48 -> rsvd.cpp:17-29, with the
 * reference's Omega: uniform [0,1) from std::mt19937 seeded 0, functions.cpp:52-66).
 * Which blocks are low rank follows the plan's admissibility.
 * kparams: kernel parameters (see FRANK_KERNEL_*), may be NULL.  Replaces
 * Hierarchical(kernel, params, n, n, nleaf, eps, admis, nb, nb)
 * (classes/hierarchical.cpp:89-109) for one level. */
int frank_blr_build_kernel(frank_blr* plan, int kernel, const double* points, int dim,
                           const double* kparams, double eps, void* stream);

/* Block type and rank of block (i, j); which = 0: A_H, 1: working/factor. */
int frank_blr_block_info(const frank_blr* plan, int which, int i, int j, int* type, int* rank);

/* Copy block (i, j) of A_H (which=0) or of the factor (which=1) to host FP64.
 * Dense: a (rows x cols, ld).  Low rank: U (m x rank), S (rank x rank),
 * V (rank x n).  For which=1 after getrf: diagonal blocks hold the packed
 * pivoted LU (unit L below, U on and above the diagonal) with pivots from
 * frank_blr_get_pivots; blocks below the diagonal hold L, above hold U. */
int frank_blr_get_dense(const frank_blr* plan, int which, int i, int j, double* a, int64_t ld, int rowmajor);
int frank_blr_get_lowrank(const frank_blr* plan, int which, int i, int j,
                          double* U, int64_t ldu, double* S, int64_t lds,
                          double* V, int64_t ldv, int rowmajor);

/* LAPACK-style 1-based pivot rows of the diagonal block i (after getrf). */
int frank_blr_get_pivots(const frank_blr* plan, int i, int* ipiv);

/* Select the LowRank recompression of the factorization, like FRANK's
 * setGlobalValue("FRANK_LRA", name) (util/global_key_value.cpp:10-22, read at
 * operations/arithmetic/addition.cpp:194-201):
 *   "rounded_addition"       core SVD (one-sided Jacobi, FP64) truncated by
 *                            find_svd_truncation_rank -- the reference algorithm
 *                            selected by FRANK_LRA=rounded_addition;
 *   "fast_rounded_addition"  (default of fixed-rank plans, as in the reference
 *                            with FRANK_LRA unset, addition.cpp:133-189) the
 *                            update's bases projected out of the target's
 *                            orthonormal ones, QR of the remainders only, core
 *                            SVD; on tolerance plans it falls back to
 *                            "rounded_addition" like the reference;
 *   "rounded_addition_rrqr"  the reference's fixed-accuracy compressor
 *                            truncated_geqp3 + rq applied to the same core, with
 *                            tolerance core_scale * eps (core_scale <= 0: 0.1);
 *   "rounded_addition_rrqr_proj"  (default of tolerance plans) the same RRQR
 *                            core on projected bases: the target's orthonormal
 *                            U_C, V_C are kept and only the update's bases,
 *                            projected out of them (twice), are QR-factored
 *                            (fast_rounded_addition's bases, addition.cpp:
 *                            133-189, at a tolerance).  Low-rank blocks given
 *                            by frank_blr_set_lowrank get orthonormal bases
 *                            (U = Qu Ru, V^T = Qv Rv, S <- Ru S Rv^T: the same
 *                            matrix) before the next factorization;
 *   "rounded_addition_rrqr_gram"  mixed plans only: the same RRQR core, with the
 *                            stacked bases orthogonalised through their FP64
 *                            Gram matrices (pivoted Cholesky) instead of a
 *                            Householder QR along the block rows.
 * Fixed-rank plans use the core SVD under every value but
 * "fast_rounded_addition" and the default. */
int frank_blr_set_lra(frank_blr* plan, const char* name, double core_scale);

/* Right-looking block LU in place.  Replaces getrf(Hierarchical&)
 * (operations/LAPACK/getrf.cpp:40-65) with its leaf getrf (getrf.cpp:67-84,
 * here with partial pivoting applied), trsm (operations/BLAS/trsm.cpp:92-115),
 * gemm (operations/BLAS/gemm.cpp:180-272) and rounded LowRank addition
 * (operations/arithmetic/addition.cpp:93-127).  Resets the working copy from
 * A_H first, so it may be called repeatedly. */
int frank_blr_getrf(frank_blr* plan, void* stream);

/* x = U^{-1} L^{-1} P b for nrhs right-hand sides (column-major n x nrhs,
 * leading dimension ldb), in place.  Replaces trsm(L, b, Lower) followed by
 * trsm(U, b, Upper) (trsm.cpp:117-125, 40-90; examples/h_lu.cpp:45-48).
 * Every call on a plan (solve, matvec, refine, their _device and transposed
 * variants) writes plan-owned device workspace (the FP32 solve vector of a
 * mixed plan, the matvec partials, the refinement residual), so calls on the
 * same plan must be serialised.  The host-buffer calls (frank_blr_solve,
 * frank_blr_matvec, frank_blr_refine) additionally stage b, x and y in one
 * device buffer owned by the plan (allocated at the first call, grown when
 * nrhs grows); the _device variants only avoid that staging buffer. */
int frank_blr_solve(frank_blr* plan, double* b, int64_t ldb, int nrhs, void* stream);
int frank_blr_solve_device(frank_blr* plan, double* d_b, int64_t ldb, int nrhs, void* stream);

/* One of the two block substitutions of the solve on host buffers, in place:
 * uplo FRANK_LOWER: b = L^{-1} P b (trsm(L, b, Mode::Lower), the forward
 * sweep, trsm.cpp:163-174 with the leaf pivots applied); FRANK_UPPER:
 * b = U^{-1} b (trsm(U, b, Mode::Upper), the backward sweep,
 * trsm.cpp:136-145).  Replaces trsm(Hierarchical, Dense, Mode)
 * (operations/BLAS/trsm.cpp:117-125, 40-90). */
enum { FRANK_LOWER = 0, FRANK_UPPER = 1 };
int frank_blr_trsm(frank_blr* plan, int uplo, double* b, int64_t ldb, int nrhs, void* stream);

/* y = alpha A_H x + beta y in FP64 on host buffers (column-major, nrhs
 * columns).  Replaces gemm(Hierarchical, Dense, Dense, alpha, beta)
 * (operations/BLAS/gemm.cpp:581-615). */
int frank_blr_gemv(frank_blr* plan, double alpha, const double* x, int64_t ldx, double beta, double* y, int64_t ldy,
                   int nrhs, void* stream);

/* y = A_H x in FP64 (column-major, nrhs columns).  Replaces
 * gemm(Hierarchical, Dense, Dense, 1, 0) (gemm.cpp:581-615). */
int frank_blr_matvec(frank_blr* plan, const double* x, int64_t ldx, double* y, int64_t ldy,
                     int nrhs, void* stream);
int frank_blr_matvec_device(frank_blr* plan, const double* d_x, int64_t ldx, double* d_y,
                            int64_t ldy, int nrhs, void* stream);

/* Solve A_H x = b to a relative residual max_j ||b_j - A_H x_j|| / ||b_j|| <= tol
 * by iterative refinement preconditioned with the factor (getrf must have run):
 * x0 = (LU)^{-1} b, x += (LU)^{-1}(b - A_H x) with the residual in FP64.
 * Reports iterations and the final relative residual.  Returns
 * FRANK_ERR_NOT_CONVERGED if maxit is reached first. */
int frank_blr_refine(frank_blr* plan, const double* b, int64_t ldb, double* x, int64_t ldx,
                     int nrhs, double tol, int maxit, int* iters, double* resid, void* stream);
int frank_blr_refine_device(frank_blr* plan, const double* d_b, int64_t ldb, double* d_x,
                            int64_t ldx, int nrhs, double tol, int maxit, int* iters,
                            double* resid, void* stream);

/* Transposed solve x = (P^T L U)^{-T} b = A^{-T} b with the same factors, for
 * the adjoint of solve(A, b) (no reference counterpart; python/FRANK adjoint). */
int frank_blr_solve_transpose_device(frank_blr* plan, double* d_b, int64_t ldb, int nrhs, void* stream);

/* y = A_H^T x in FP64, and refinement of A_H^T x = b with the transposed
 * solve (the adjoint solve A^T lambda = g of solve(A, b)).  No reference
 * counterpart (python/FRANK adjoint). */
int frank_blr_matvec_transpose_device(frank_blr* plan, const double* d_x, int64_t ldx, double* d_y, int64_t ldy,
                                      int nrhs, void* stream);
int frank_blr_refine_transpose_device(frank_blr* plan, const double* d_b, int64_t ldb, double* d_x, int64_t ldx,
                                      int nrhs, double tol, int maxit, int* iters, double* resid, void* stream);

/* out = sum_h sum_ij lambda_ih (dA_ij / dtheta) x_jh for the exponential
 * kernel A_ij = exp(-r_ij / theta) + nugget delta_ij (kparams = {theta,
 * nugget}), evaluated on the fly from the device points (dim x n,
 * axis-major); the theta-gradient of a loss through solve(A(theta), b) is
 * -out with lambda the adjoint solution.  No reference counterpart. */
int frank_kernel_dtheta_contract(int kernel, const double* d_points, int dim, int64_t n, const double* kparams,
                                 const double* d_lambda, int64_t ldl, const double* d_x, int64_t ldx, int nrhs,
                                 double* out, void* stream);

/* Limit a plan's recompression / update grids to `ctas` thread blocks and
 * shrink its scratch accordingly, for plans that run concurrently in a batch. */
int frank_blr_set_grid(frank_blr* plan, int ctas);

/* A batch of independent plans (same precision): frank_batch_getrf factors
 * all of them in one captured CUDA graph (one branch per system, so systems
 * of uneven order run concurrently); frank_batch_refine_device refines every
 * system k (b d_b[k], solution d_x[k], column-major, nrhs <= 8) to tol, the
 * host synchronising once per iteration for the whole batch.  iters/resid
 * are per system.  Replaces a host loop of getrf/trsm over independent
 * Hierarchical matrices (no batched call in the reference). */
typedef struct frank_batch frank_batch;
int frank_batch_create(frank_blr* const* plans, int count, frank_batch** out);
int frank_batch_destroy(frank_batch* batch);
int frank_batch_getrf(frank_batch* batch, void* stream);
int frank_batch_refine_device(frank_batch* batch, const double* const* d_b, int64_t ldb, double* const* d_x,
                              int64_t ldx, int nrhs, double tol, int maxit, int* iters, double* resid);

/* Write the block tree of A_H (which = 0) or of the factor (which = 1, FP64
 * plans after getrf) as JSON in the layout of FRANK's write_JSON
 * (util/print.cpp:54-128, keys sorted as nlohmann::json prints them): the
 * Hierarchical root with "abs_pos", "children" (rows of blocks), "dim",
 * "level", "type"; every block with its "abs_pos", "dim", "level", "type",
 * its singular values "svalues" (min(m, n) of them, computed on the GPU;
 * those of a LowRank block beyond its rank are 0) and, for LowRank blocks,
 * "rank".  Replaces write_JSON(const Matrix&, filename)
 * (util/print.cpp:124-128). */
int frank_blr_write_json(const frank_blr* plan, int which, const char* path);

/* Autotuner of the plan's launch parameters: the rows per dense-update task
 * (64 / 128 / 256), the operand rank above which a band-1 recompression
 * target is split over two CTAs (never / 16 ... 96), and, for tolerance plans
 * with the RRQR core, stacked or projected bases.  Coordinate descent, one
 * parameter at a time, each candidate timed on the plan's own factorization
 * (device time of a captured-graph replay); the choice is cached for the
 * process per workload shape (n, nb, precision, rank / tolerance,
 * recompression) and reused by later calls unless `force`.  Leaves the plan
 * unfactored.  No reference counterpart. */
int frank_blr_autotune(frank_blr* plan, int force, void* stream);

/* Set the launch parameters by hand (band_rows >= 16; split_rank 0 = never
 * split; projected: bases of tolerance plans with the RRQR core). */
int frank_blr_set_tuning(frank_blr* plan, int band_rows, int split_rank, int projected);

/* The plan's current launch parameters (see frank_blr_autotune). */
int frank_blr_tuning(const frank_blr* plan, int* band_rows, int* split_rank, int* projected);

/* The largest recompression core (in doubles) kept in shared memory; larger
 * cores take the L2 paths (randomized block pivoting for the RRQR core,
 * blocked WY).  Chosen by frank_blr_autotune; 0 < value.  */
int frank_blr_core_smem(const frank_blr* plan, int* doubles);
int frank_blr_set_core_smem(frank_blr* plan, int doubles);

/* Counters of the last getrf: kernels launched by it plus those of every
 * solve / matvec / refine since, recompressions performed, the largest
 * recompressed rank and the number of ranks clamped at max_rank. */
int frank_blr_stats(const frank_blr* plan, int64_t* launches, int64_t* recompressions,
                    int64_t* max_rank_seen, int64_t* rank_overflows);

/* Record CUDA events around each launch class inside the factorization graph
 * (on = 1) for frank_blr_kernel_times; off by default because event-record
 * nodes serialise the graph's concurrent branches (the lookahead getrf). */
int frank_blr_set_timing(frank_blr* plan, int on);

/* Device time (ms, CUDA events recorded around each launch inside the
 * factorization graph when timing is on; zeros otherwise) and algorithmic
 * FLOPs of the last getrf, per kernel
 * class: [0] leaf getrf + inverses, [1] panel trsm, [2] dense-target updates,
 * [3] LowRank recompression.  The FLOPs count the reference's call sequence
 * with the LAWN 41 operation counts (no reference counterpart; reporting). */
int frank_blr_kernel_times(const frank_blr* plan, double* ms, double* flops);

/* ---------------------------------------------------------------------------
 * Per-operation entry points: FRANK's dense factorizations and low-rank
 * operations one block at a time, batched.  All matrices are FP64,
 * column-major, in device memory; matrix b of a batch starts at
 * ptr + b * stride.  m, n <= 4096 (<= 1024 for the SVD).  Synchronous on
 * `stream`; scratch comes from the stream-ordered pool.
 * ------------------------------------------------------------------------- */

/* Device buffers for callers of the per-operation entry points that do not
 * manage device memory themselves (the C++ layer): allocate, free, and copy
 * host <-> device (to_device != 0: host to device).  No reference
 * counterpart (the reference's matrices live in host memory). */
int frank_device_alloc(size_t bytes, void** out);
int frank_device_free(void* ptr);
int frank_copy(void* dst, const void* src, size_t bytes, int to_device);

/* C = alpha op(A) op(B) + beta C, op(A) m x k, op(B) k x n (trans_* != 0:
 * transposed).  Replaces gemm(Dense, Dense, Dense, alpha, beta, TransA,
 * TransB) (operations/BLAS/gemm.cpp:126-146: cblas_dgemm). */
int frank_gemm_batched(int m, int n, int k, int count, double alpha, const double* d_a, int64_t lda, int64_t stride_a,
                       int trans_a, const double* d_b, int64_t ldb, int64_t stride_b, int trans_b, double beta,
                       double* d_c, int64_t ldc, int64_t stride_c, void* stream);

/* Householder QR: Q (m x k, explicit), R (k x n, upper trapezoidal), k = min(m, n).
 * Replaces qr(A, Q, R) (operations/LAPACK/qr.cpp:65-90: dgeqrf + dorgqr). */
int frank_qr_batched(int m, int n, int count, const double* d_a, int64_t lda, int64_t stride_a, double* d_q,
                     int64_t ldq, int64_t stride_q, double* d_r, int64_t ldr, int64_t stride_r, void* stream);

/* RQ: A = R Q with R (m x k, upper trapezoidal) and Q (k x n, orthonormal
 * rows), k = min(m, n).  Replaces rq(A, R, Q) (operations/LAPACK/rq.cpp:43-70:
 * dgerqf + dorgrq); rows of Q (and columns of R) may differ in sign from
 * LAPACK's. */
int frank_rq_batched(int m, int n, int count, const double* d_a, int64_t lda, int64_t stride_a, double* d_r,
                     int64_t ldr, int64_t stride_r, double* d_q, int64_t ldq, int64_t stride_q, void* stream);

/* Thin SVD by one-sided Jacobi: A = U diag(s) Vt, U (m x k), s (k, descending),
 * Vt (k x n), k = min(m, n).  Replaces svd(A) (operations/LAPACK/svd.cpp:23-44:
 * dgesvd 'S','S'; singular vectors up to sign).  FRANK_ERR_NOT_CONVERGED if
 * the sweeps do not converge. */
int frank_svd_batched(int m, int n, int count, const double* d_a, int64_t lda, int64_t stride_a, double* d_u,
                      int64_t ldu, int64_t stride_u, double* d_s, int64_t stride_s, double* d_vt, int64_t ldvt,
                      int64_t stride_vt, void* stream);

/* Randomized SVD truncated to `rank`: U (m x rank), S (rank x rank, diagonal),
 * V (rank x n).  Sample rank + oversample (capped at min(m, n)) columns with
 * the reference's Omega (random_uniform: std::mt19937 seeded 0, uniform [0,1),
 * functions.cpp:52-66), `power_its` subspace iterations.  Replaces
 * LowRank(Dense, rank) (classes/low_rank.cpp:40-48: rsvd with oversample 5,
 * no power iteration, operations/randomized/rsvd.cpp:17-29). */
int frank_rsvd_batched(int m, int n, int count, int rank, int oversample, int power_its, const double* d_a,
                       int64_t lda, int64_t stride_a, double* d_u, int64_t ldu, int64_t stride_u, double* d_s,
                       int64_t lds, int64_t stride_s, double* d_v, int64_t ldv, int64_t stride_v, void* stream);

/* Interpolative decomposition at rank k: A ~= U S V with S = A(rows, cols)
 * (k x k), U (m x k), V (k x n), rows / cols the selected indices (0-based,
 * k per matrix), from column-pivoted QR (geqp3) and R11^{-1} R12.  Replaces
 * id(A, k) (operations/LAPACK/id.cpp:75-116, one_sided_id :49-73). */
int frank_id_batched(int m, int n, int count, int k, const double* d_a, int64_t lda, int64_t stride_a, double* d_u,
                     int64_t ldu, int64_t stride_u, double* d_s, int64_t lds, int64_t stride_s, double* d_v,
                     int64_t ldv, int64_t stride_v, int* d_rows, int* d_cols, void* stream);

/* Randomized ID: the ID of Q^T A at rank k, Q an orthonormal basis of
 * A Omega (sample columns, the reference's Omega), U = Q U_b.  Replaces
 * rid(A, sample, k) (operations/randomized/rid.cpp:18-31). */
int frank_rid_batched(int m, int n, int count, int sample, int k, const double* d_a, int64_t lda, int64_t stride_a,
                      double* d_u, int64_t ldu, int64_t stride_u, double* d_s, int64_t lds, int64_t stride_s,
                      double* d_v, int64_t ldv, int64_t stride_v, void* stream);

/* A += B for low-rank pairs, in place on A: A = Ua Sa Va (m x ka, ka x ka,
 * ka x n, capacity kmax), B = Ub Sb Vb (kb <= kb_max); ranks d_ka (in/out) and
 * d_kb per pair.  lra "rounded_addition" (addition.cpp:93-127: QR of both
 * stacked bases, core SVD, rank by find_svd_truncation_rank at eps, or ka when
 * eps = 0), "fast_rounded_addition" (addition.cpp:133-189: fixed rank, A's
 * bases orthonormal; falls back to rounded_addition when eps > 0) or "naive"
 * (also "naive_addition"; addition.cpp:68-89: ka + kb >= min(m, n) gives
 * LowRank(Dense(A) + Dense(B), ka) by rsvd with the reference's Omega, else
 * the bases and S are concatenated to rank ka + kb, which must fit kmax --
 * FRANK_ERR_RANK_OVERFLOW otherwise; reads the ranks to the host).  Replaces
 * operator+=(LowRank&, const LowRank&) (addition.cpp:191-203). */
int frank_lowrank_add_batched(int m, int n, int count, int kmax, const char* lra, double eps, double* d_ua,
                              int64_t ldua, int64_t stride_ua, double* d_sa, int64_t ldsa, int64_t stride_sa,
                              double* d_va, int64_t ldva, int64_t stride_va, int* d_ka, const double* d_ub,
                              int64_t ldub, int64_t stride_ub, const double* d_sb, int64_t ldsb, int64_t stride_sb,
                              const double* d_vb, int64_t ldvb, int64_t stride_vb, const int* d_kb, int kb_max,
                              void* stream);

/* Largest block order accepted by frank_getrf_dense_noalloc. */
#define FRANK_NOALLOC_MAX_N 256

/* Pivoted LU of one dense FP64 block that allocates no memory.  No
 * counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc, e.g. code running inside a custom device-memory allocator's
 * callback, on an out-of-memory recovery path where every byte is already
 * committed, or in a process whose memory pool forbids new allocations.
 * The plan-based entry points allocate device memory (the plan itself, and
 * staging buffers in the host-buffer calls); this one uses only the fixed
 * scratch described below and the caller's buffers.
 *
 * d_a: n x n input (device, column-major, lda >= n), left unchanged.
 * d_lu: n x n output (device, column-major, ldlu >= n): the packed LU of
 * P A (unit L below the diagonal, U on and above), the same factor as
 * frank_blr_getrf on a one-block plan.  d_ipiv: n ints (device), 1-based
 * LAPACK-style pivots.  n must be 1..FRANK_NOALLOC_MAX_N, else
 * FRANK_ERR_UNSUPPORTED; a zero pivot gives FRANK_ERR_SINGULAR.
 *
 * The scratch is one fixed 2 MB array in device memory (a file-scope
 * __device__ array of the library) that every GPU loading the library holds
 * until exit; all calls share it and it keeps the last call's contents.  The
 * first call on a device (and the first after the device's context has been
 * re-created, e.g. by cudaDeviceReset) does the set-up: it looks up the
 * array's device address and loads this entry point's kernels.  With CUDA's
 * default lazy module loading that loading can itself take device memory, so
 * make one warm-up call per device at start-up, while memory is still
 * available; later calls load and allocate nothing.  The call synchronises
 * `stream` and reads status words back to the host, so it cannot be made
 * inside a stream capture at all.  Calls that overlap on the GPU (from
 * several host threads or streams at once) race on the shared scratch:
 * serialise them. */
int frank_getrf_dense_noalloc(const double* d_a, int64_t lda, int n, double* d_lu, int64_t ldlu,
                              int* d_ipiv, void* stream);

/* ------------------------------------------------------------------------
 * Multi-level H-matrices: binary cluster tree, weak admissibility, fixed rank.
 *
 * The matrix Hierarchical(kernel, params, n, n, rank, nleaf, admis = 0, 2, 2)
 * (classes/hierarchical.cpp:49-109 with matrix_initializer.cpp:51-58): every
 * off-diagonal child at every level is LowRank of rank `rank`, every diagonal
 * child recurses until it is a dense leaf of order `leaf`.  n / leaf must be
 * a power of two (levels L = log2(n / leaf)).  Block (level l, index c),
 * l = 1..L, c = 0..2^l - 1, spans the rows of cluster c of level l and the
 * columns of its sibling c ^ 1; it is U (s x rank), S (rank x rank),
 * V (rank x s), s = n >> l, all column-major.  Leaf p (0 .. 2^L - 1) is the
 * dense diagonal block of rows and columns [p leaf, (p + 1) leaf).
 * ------------------------------------------------------------------------ */
typedef struct frank_hodlr frank_hodlr;

/* New H-matrix (all blocks zero); 8 <= leaf <= 512, 1 <= rank <= min(64, leaf). */
int frank_hodlr_create(int64_t n, int leaf, int rank, frank_hodlr** out);
int frank_hodlr_destroy(frank_hodlr* h);
int frank_hodlr_shape(const frank_hodlr* h, int64_t* n, int* leaf, int* rank, int* levels);

/* LowRank += LowRank of the factorization's updates: "fast_rounded_addition"
 * (the reference's default for fixed rank, addition.cpp:133-189, 191-203)
 * or "rounded_addition" (addition.cpp:93-127). */
int frank_hodlr_set_lra(frank_hodlr* h, const char* name);

/* Host blocks of A_H, column-major (leading dimension ld >= leaf for leaves;
 * U, S, V packed). */
int frank_hodlr_set_dense(frank_hodlr* h, int leaf, const double* a, int64_t ld);
int frank_hodlr_set_lowrank(frank_hodlr* h, int level, int index, const double* U, const double* S,
                            const double* V);
/* which = 0: A_H; 1: the factor (leaves: packed LU of dgetrf with the
 * interchanges applied; LowRank: L blocks (odd index) and U blocks (even)). */
int frank_hodlr_get_dense(const frank_hodlr* h, int which, int leaf, double* a, int64_t ld);
int frank_hodlr_get_lowrank(const frank_hodlr* h, int which, int level, int index, double* U, double* S,
                            double* V);
/* 0-based LAPACK-style pivots of leaf p's getrf. */
int frank_hodlr_get_pivots(const frank_hodlr* h, int leaf, int* ipiv);

/* Build A_H on the device from points (dim x n, axis-major): dense leaves by
 * kernel evaluation, every LowRank block by LowRank(Dense, rank)
 * (low_rank.cpp:40-48 -> rsvd.cpp:17-29, sample min(rank + 5, s), the
 * reference's Omega: uniform [0,1) from std::mt19937 seeded 0,
 * functions.cpp:52-66) without storing the block: A Omega and A^T Q are
 * evaluated tile by tile.  kparams as for frank_blr_build_kernel. */
int frank_hodlr_build_kernel(frank_hodlr* h, int kernel, const double* points, int dim, const double* kparams,
                             void* stream);

/* getrf(A) (operations/LAPACK/getrf.cpp:45-65, recursive): the factorization
 * is captured once into a CUDA graph and replayed from A_H on every call. */
int frank_hodlr_getrf(frank_hodlr* h, void* stream);
/* b <- (L U)^{-1} P b in place: trsm(L, b, Lower) then trsm(U, b, Upper)
 * (examples/h_lu.cpp:45-48); device buffer n x nrhs, ld ldb. */
int frank_hodlr_solve_device(frank_hodlr* h, double* d_b, int64_t ldb, int nrhs, void* stream);
/* One of the two: uplo FRANK_LOWER: b <- L^{-1} P b (trsm(L, b, Mode::Lower));
 * FRANK_UPPER: b <- U^{-1} b (trsm(U, b, Mode::Upper)); in either order. */
int frank_hodlr_trsm_device(frank_hodlr* h, int uplo, double* d_b, int64_t ldb, int nrhs, void* stream);
/* y = A_H x (FP64; gemm(H, x, y) over the leaves and every LowRank block). */
int frank_hodlr_matvec_device(frank_hodlr* h, const double* d_x, int64_t ldx, double* d_y, int64_t ldy, int nrhs,
                              void* stream);
/* x = solve(b), then x += solve(b - A_H x) until every column's
 * ||b - A_H x|| / ||b|| <= tol (or max_iter corrections). */
int frank_hodlr_refine_device(frank_hodlr* h, const double* d_b, int64_t ldb, double* d_x, int64_t ldx, int nrhs,
                              double tol, int max_iter, int* iters, double* relres, void* stream);
/* Kernel launches of one factorization and the device time of the last getrf (ms). */
int frank_hodlr_stats(const frank_hodlr* h, int64_t* launches, double* factor_ms);

#ifdef __cplusplus
}
#endif

#endif /* FRANK_B200_H */

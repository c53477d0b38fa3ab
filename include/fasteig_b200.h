/*
 * fasteig_b200 — C ABI of the B200 (sm_100a) backend for fasteig's sparse
 * symmetric eigensolver hot path.
 *
 * Conventions shared by every entry point:
 *   - Return value: 0 on success, a negative FE_ERR_* code on failure.
 *     fe_last_error() returns a message for the calling thread's last failure.
 *     Errors never abort the process.
 *   - Dense blocks ("multivectors") live in device memory ROW-MAJOR:
 *     element (row i, column j) of a block with leading dimension ld is at
 *     base[i * ld + j]. A column range is addressed by offsetting base.
 *     (The reference stores column-major n-by-k blocks, ld = n,
 *     src/gpu/CudaMultiVector.cpp:26-28; the row-major "slab" makes one CSR
 *     row's neighbours contiguous 128-bit loads for SpMM.)
 *   - Small matrices (Gram, rotation coefficients, Cholesky factors) are FP64,
 *     column-major, in device memory, matching Eigen's MatrixXd convention
 *     used by the reference's host-side small matrices.
 *   - Every compute call is asynchronous on the given CUDA stream (a
 *     cudaStream_t passed as void*, NULL = legacy default stream) and takes
 *     caller-owned device pointers. Calls that need scratch space take a
 *     caller-owned device workspace and report its size via *_workspace_bytes.
 */
#ifndef FASTEIG_B200_H
#define FASTEIG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FE_OK 0
#define FE_ERR_INVALID -1     /* invalid argument (shape, pointer, alignment) */
#define FE_ERR_CUDA -2        /* CUDA runtime / library failure */
#define FE_ERR_NOT_SPD -3     /* Cholesky rank loss (reference returns -1) */
#define FE_ERR_NONFINITE -4   /* non-finite Ritz data / residuals */
#define FE_ERR_ALLOC -5       /* device allocation failure */
#define FE_ERR_UNSUPPORTED -6 /* option not supported by this backend */
#define FE_PENDING 1          /* fe_server_wait: request not finished within the timeout */

typedef struct fe_csr* fe_csr_t;

/* Library identity and error reporting. */
const char* fe_version(void);
const char* fe_last_error(void);
int fe_device_count(int* count);
/* Kernel launches issued by this library since it was loaded (all threads). */
int64_t fe_launch_count(void);

/* ---------------------------------------------------------------------
 * CSR operator (replaces CudaCsrMatrix, src/gpu/CudaCsrMatrix.cpp:20-52,
 * constructed from core::CsrMatrixData, include/core/CsrMatrix.hpp:18-27).
 * The host arrays are validated exactly as validate_csr_matrix_data
 * (src/core/CsrMatrix.cpp:11-39) and uploaded; FP64 and FP32 value copies
 * are kept on the device.
 * ------------------------------------------------------------------- */
int fe_csr_create(int64_t rows, int64_t cols, int64_t nnz, const int32_t* rowptr,
                  const int32_t* colind, const double* values, fe_csr_t* out);
int fe_csr_destroy(fe_csr_t csr);
int fe_csr_info(fe_csr_t csr, int64_t* rows, int64_t* cols, int64_t* nnz);
/* Copies back the stored matrix (CsrMatrix::copy_to_host,
 * include/core/CsrMatrix.hpp:35). Arrays must hold rows+1 / nnz / nnz items. */
int fe_csr_copy_to_host(fe_csr_t csr, int32_t* rowptr, int32_t* colind, double* values);

/* CSR built on the device from triplets (replaces the host Eigen path
 * fasteig_problem::build_sparse_matrix_from_triplets, src/fasteig_problem.cpp:474-506,
 * followed by build_csr_from_sparse_matrix, :554-607). rows/cols/values are `count`
 * 0-based host triplets of an n-by-n matrix; duplicates are summed left to right in
 * input order (Eigen's setFromTriplets); expand = 0 keeps the matrix as given,
 * 1 adds the mirror (c, r, v) of every off-diagonal entry (a symmetric matrix
 * stored as one triangle), 2 adds (c, r, -v) (skew); positions that then hold two
 * values keep their sum. Rows come out sorted by column, explicit zeros are kept,
 * and the result is bit-identical to the reference's. Index errors give the
 * reference's messages ("Triplet index out of bounds.", "Invalid matrix
 * dimension n <= 0."). */
int fe_csr_create_from_triplets(int64_t n, int64_t count, const int32_t* rows,
                                const int32_t* cols, const double* values, int32_t expand,
                                fe_csr_t* out);
/* MatrixMarket coordinate file (real, integer or pattern; general, symmetric or
 * skew-symmetric; 1-based entries, as src/mmio.cpp reads them) parsed on the host
 * into triplets and built on the device as fe_csr_create_from_triplets does
 * (symmetric files expand their stored triangle). */
int fe_csr_create_from_matrix_market(const char* path, fe_csr_t* out);

/* ---------------------------------------------------------------------
 * Block SpMM (replaces LinearOperator::apply_block of a CSR matrix,
 * include/core/LinearOperator.hpp:32-37; GPU: CudaCsrMatrix::apply_block,
 * src/gpu/CudaCsrMatrix.cpp:196-223, a loop of ncols cuSPARSE SpMVs; CPU:
 * CpuCsrMatrix::apply_block, src/core/CsrMatrix.cpp:209-245):
 *     Y[:, 0:ncols] = alpha * A * X[:, 0:ncols] + beta * Y[:, 0:ncols]
 * beta == 0 overwrites Y (NaN-safe), as the reference's setZero branch.
 * X and Y must not overlap. _f32 computes with FP32 values and FP32
 * accumulation on FP32 blocks.
 * ------------------------------------------------------------------- */
int fe_spmm_csr_f64(fe_csr_t A, const double* X, int64_t ldx, double* Y, int64_t ldy,
                    int64_t ncols, double alpha, double beta, void* stream);
int fe_spmm_csr_f32(fe_csr_t A, const float* X, int64_t ldx, float* Y, int64_t ldy,
                    int64_t ncols, double alpha, double beta, void* stream);

/* ---------------------------------------------------------------------
 * Fused Chebyshev three-term step (replaces the per-step copy_from +
 * apply_block(2c, -1) + add_scaled_columns(2d) sequence of
 * ChebyshevSolver::chebyshev_filter, src/ChebyshevSolver.cpp:243-256):
 *     Yout = alpha * A * Ycur + gamma * Ycur + beta * Yprev
 * Step 1 of the filter is (alpha, gamma, beta) = (c, d, 0) with Yprev unused;
 * step k >= 2 is (2c, 2d, -1). Yout may alias Yprev (in-place update of the
 * k-2 block); Ycur must not overlap Yout.
 * ------------------------------------------------------------------- */
int fe_cheb_step_f64(fe_csr_t A, const double* Ycur, const double* Yprev, double* Yout,
                     int64_t ld, int64_t ncols, double alpha, double gamma, double beta,
                     void* stream);
int fe_cheb_step_f32(fe_csr_t A, const float* Ycur, const float* Yprev, float* Yout,
                     int64_t ld, int64_t ncols, double alpha, double gamma, double beta,
                     void* stream);
/* Whole filter of degree `degree` in place on X (ChebyshevSolver::chebyshev_filter,
 * src/ChebyshevSolver.cpp:223-258, with scaling (c, d) already computed);
 * `scratch` is a second block of the same shape. */
int fe_cheb_filter_f64(fe_csr_t A, double* X, double* scratch, int64_t ld, int64_t ncols,
                       int32_t degree, double c, double d, void* stream);
int fe_cheb_filter_f32(fe_csr_t A, float* X, float* scratch, int64_t ld, int64_t ncols,
                       int32_t degree, double c, double d, void* stream);

/* ---------------------------------------------------------------------
 * Gram G = X^T Y over all n rows (replaces MultiVector::transpose_multiply,
 * src/gpu/CudaMultiVector.cpp:361-406, and the Gram Dgemm of Cholesky QR,
 * src/core/Orthogonalization.cpp:202-209). X is n-by-k, Y is n-by-m; G is
 * k-by-m FP64 column-major with leading dimension ldg. Products of the inputs
 * are accumulated in FP64 (FP32 inputs: exact products, FP64 sums), split over
 * row chunks whose partial Grams are reduced in a fixed order (deterministic).
 * ------------------------------------------------------------------- */
size_t fe_gram_workspace_bytes(int64_t n, int64_t k, int64_t m);
int fe_gram_f64(const double* X, int64_t ldx, const double* Y, int64_t ldy, int64_t n,
                int64_t k, int64_t m, double* G, int64_t ldg, void* workspace,
                size_t workspace_bytes, void* stream);
int fe_gram_f32(const float* X, int64_t ldx, const float* Y, int64_t ldy, int64_t n,
                int64_t k, int64_t m, double* G, int64_t ldg, void* workspace,
                size_t workspace_bytes, void* stream);

/* FP64 Gram that allocates nothing (this entry point has no counterpart in the
 * reference). For callers that cannot allocate device memory at call time —
 * e.g. a program whose device memory is all owned by its own pool, or a
 * latency-critical path that must not call cudaMalloc — the split-K partial
 * sums go to a fixed 8 MiB array inside this library instead of a caller
 * workspace; every GPU that loads the library keeps that array until the
 * process exits. Same arguments, results and accuracy as fe_gram_f64; it
 * requires k*m <= fe_gram_f64_noalloc_max_entries() (1,048,576) and returns
 * FE_ERR_INVALID otherwise. The first call on a device looks up the array's
 * device address with that device current; make that first call before any
 * stream capture. The address belongs to the device's primary context (the one
 * the CUDA runtime uses); it is looked up again after cudaDeviceReset, and a
 * caller that makes a different context current through the driver API must not
 * call this entry point. All calls share the one array (each call overwrites the
 * part it uses, nothing needs clearing): calls that can overlap on the GPU —
 * on different streams, or from different host threads — race and must be
 * serialized by the caller. */
int fe_gram_f64_noalloc(const double* X, int64_t ldx, const double* Y, int64_t ldy, int64_t n,
                        int64_t k, int64_t m, double* G, int64_t ldg, void* stream);
int64_t fe_gram_f64_noalloc_max_entries(void);

/* Tensor-core Gram of FP32 blocks (tcgen05, 3xTF32 split products accumulated
 * in FP32 per row chunk, chunk partials summed in FP64): FP32-level accuracy
 * relative to |X|^T |Y|, for the mixed-precision path. Same shapes as
 * fe_gram_f32; workspace from fe_gram_tf32x3_workspace_bytes. */
size_t fe_gram_tf32x3_workspace_bytes(int64_t n, int64_t k, int64_t m);
int fe_gram_tf32x3(const float* X, int64_t ldx, const float* Y, int64_t ldy, int64_t n,
                   int64_t k, int64_t m, double* G, int64_t ldg, void* workspace,
                   size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------
 * Rotation Y = alpha * X * C + beta * Y (replaces
 * MultiVector::right_multiply_active_columns, src/gpu/CudaMultiVector.cpp:310-359,
 * the triangular solve of Cholesky QR, src/core/Orthogonalization.cpp:227-235,
 * applied as X * R^{-1}, and the X - V*H updates of block Gram-Schmidt,
 * :554-601). X is n-by-k, C is k-by-m FP64 column-major (ldc), Y is n-by-m.
 * _f32 rounds C to FP32 and accumulates in FP32. X and Y must not overlap.
 * ------------------------------------------------------------------- */
int fe_rotate_f64(const double* X, int64_t ldx, const double* C, int64_t ldc, double* Y,
                  int64_t ldy, int64_t n, int64_t k, int64_t m, double alpha, double beta,
                  void* stream);
int fe_rotate_f32(const float* X, int64_t ldx, const double* C, int64_t ldc, float* Y,
                  int64_t ldy, int64_t n, int64_t k, int64_t m, double alpha, double beta,
                  void* stream);
/* Tensor-core rotation of FP32 blocks (tcgen05, 3xTF32 split of X and of C,
 * FP32 accumulation). X must start 16-byte aligned with ldx a multiple of 4;
 * the workspace holds the split FP32 copies of C. */
size_t fe_rotate_tf32x3_workspace_bytes(int64_t k, int64_t m);
int fe_rotate_tf32x3(const float* X, int64_t ldx, const double* C, int64_t ldc, float* Y,
                     int64_t ldy, int64_t n, int64_t k, int64_t m, double alpha, double beta,
                     void* workspace, size_t workspace_bytes, void* stream);
/* First failure code recorded by a bounded device-side wait of the tensor-core
 * or pipelined SpMM kernels launched outside a solve (0 = none); clear != 0
 * resets it. Kernels launched by a solve record in that solve's own word. */
int fe_device_status(int32_t* status, int32_t clear);
/* Self-test of the bounded-wait failure path (this entry point has no counterpart
 * in the reference): launches one warp that waits on an mbarrier nothing arrives
 * on for limit_cycles SM clocks, then records `code` in the library's default
 * status word (read by fe_device_status) and returns. No copies are in flight and
 * the context stays usable. Solves (fe_solve, the server) record timeouts in a
 * status word of their own and fail with FE_ERR_CUDA instead; the fe_solve option
 * inject_wait_timeout=<code> runs the same probe on a solve's word (test hook). */
int fe_selftest_wait_timeout(int64_t limit_cycles, int32_t code, void* stream);
/* SpMM kernel selection for all later calls in the process (the numerics are
 * the same; the choice only changes the memory schedule): 0 = default
 * (row-batched register kernel for slabs of >= 32 128-bit vectors and rows of
 * <= 7 nonzeros, else the loop kernel), 1 = loop kernel, 2 = bulk-copy
 * pipelined kernel where it applies, 3 = row-batched kernel with narrower
 * column panels, 4 = mode 0 with each warp's next Z row prefetched into L2,
 * 5 = row-batched kernel with 16-byte lanes and up to 3 per lane, 6 = row-batched
 * kernel with 8-byte lanes and up to 3 per lane, 7 = mode 0 with X and Z read
 * through L2 only (ld.global.cg). */
int fe_set_spmm_kernel(int32_t mode);
/* Chebyshev filter schedule for all later filters in the process (fe_cheb_filter_*
 * and the Chebyshev solver; the numerics are the same bit for bit): 0 = default,
 * one SpMM launch per step; 1 = several filter steps per launch (levels of warps, each level one step, each
 * trailing the previous one by the operator's bandwidth so the block it gathers is
 * still in L2) where the operator is square with at least 4096 rows of <= 7 entries,
 * the block splits into 1, 2 or 4 column panels of 32..160 8-byte vectors and a
 * panel's window of 2 x bandwidth rows per level fits about 75% of L2 for at least
 * two levels (measured slower than one step per launch on B200 for the 128^3
 * well operator: the steps are bound by gather latency, not by DRAM bytes).
 * For measurements: 2..8 = that many
 * steps per launch whatever the L2 window, 9 = one step per launch through the
 * multi-step kernel, 12..18 = 2..8 steps per launch with L1-cached coherent loads,
 * 100 P + S = P column panels (1, 2 or 4) of S steps (1..8) per launch.
 * A timed-out wait in the multi-step kernel records status 13 (see
 * fe_device_status). */
int fe_set_cheb_wave_kernel(int32_t mode);
/* SpMM autotuner: times every SpMM kernel on operator A for an n-by-ncols block
 * in the Chebyshev-step form (precision 0 = FP64, 1 = FP32) on `stream` and
 * records the fastest on the handle (up to four widths per precision); later
 * SpMMs of that precision within a factor of two of a tuned width use it while
 * the process-wide mode is the default 0. Writes the chosen mode to *mode (may
 * be NULL). Not to be called while solves on the same handle are running. */
int fe_csr_autotune(fe_csr_t A, int64_t ncols, int32_t precision, void* stream, int32_t* mode);
/* FP64 Gram / rotation kernel selection for all later calls in the process:
 * 0 = default (FP64 tensor-core mma.sync.m8n8k4 kernels with a cp.async ring),
 * 1 = SIMT FP64-FMA kernels. Both accumulate every output in FP64; results
 * differ only in the order of the rounded additions. */
int fe_set_f64_gemm_kernel(int32_t mode);
/* 3xTF32 rotation kernel for 16-byte aligned outputs, for all later calls:
 * 0 = default (persistent, one CTA per SM looping over tiles with two TMEM
 * accumulators; X split into hi/lo in registers and read by the MMA from tensor
 * memory), 1 = one CTA per tile, 2 = persistent with X split in shared memory.
 * Same MMAs in the same order (bit-identical results); unaligned outputs always use
 * the one-CTA-per-tile kernel with its staged epilogue. */
int fe_set_tc_rotate_kernel(int32_t mode);
/* Tridiagonalization kernel of the symmetric eigensolver (process-wide): 0 (default)
 * by matrix size, 1 one CTA per matrix, 2 the 8-CTA cluster wherever it fits. The
 * eigenvalues and vectors agree to rounding between the kernels. */
int fe_set_syevd_kernel(int32_t mode);

/* ---------------------------------------------------------------------
 * One Lanczos step on the device (replaces KrylovSubspace::build_one,
 * src/core/KrylovSubspace.cpp:125-131, for a standard problem: its
 * normalize_residual_into_basis, apply_operator_to_basis_column, two-pass
 * orthogonalize_operator_result and residual_norm, and the T entries that
 * CudaLanczosKernels.cu:11-22 records):
 *     beta = *fnorm;  V[:, j] = f / beta;  w = A V[:, j];
 *     h = V_j^T w, w -= V_j h;  h2 = V_j^T w, w -= V_j h2  (V_j = V[:, 0..j]);
 *     T[j, j] = h[j] + h2[j];  T[j, j-1] = T[j-1, j] = beta (j > 0);
 *     f = w;  *fnorm = ||f||.
 * V is an n-by-m row-major device block (ldv >= m), f an n-vector, fnorm one
 * device double (||f|| on entry, the new ||f|| on exit), T m-by-m FP64
 * column-major (ldt >= m). All scalars stay on the device, so steps can be
 * queued (or graph-captured) back to back. A breakdown (*fnorm == 0) is the
 * caller's to handle (the reference restarts with a random vector,
 * normalize_or_restart). Workspace from fe_lanczos_workspace_bytes(n, m).
 * ------------------------------------------------------------------- */
size_t fe_lanczos_workspace_bytes(int64_t n, int64_t m);
int fe_lanczos_step(fe_csr_t A, double* V, int64_t ldv, int64_t m, int64_t j, double* f,
                    double* fnorm, double* T, int64_t ldt, void* workspace,
                    size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------
 * Ritz residuals and column norms (replaces the copy + add_scaled_columns +
 * 2 x column_norms sequence of extract_projected_ritz_pairs,
 * src/core/RitzExtraction.cpp:125-139, and evaluate_ritz_pairs, :49-62):
 *     R[:, j] = AX[:, j] - lambda[j] * MX[:, j]   (MX = X when BX is NULL)
 *     rnorm[j] = ||R[:, j]||,  xnorm[j] = ||MX[:, j]||,
 *     rel[j] = rnorm[j] / ((1 + |lambda[j]|) * xnorm[j])  (rnorm if the
 *     denominator is not positive, as src/core/RitzExtraction.cpp:131-139).
 * lambda, rnorm, xnorm, rel are FP64 device arrays of length m; R may be NULL
 * (norms only). Norms are accumulated in FP64.
 * ------------------------------------------------------------------- */
size_t fe_residual_workspace_bytes(int64_t n, int64_t m);
int fe_residual_norms_f64(const double* AX, const double* X, const double* BX, int64_t ld,
                          int64_t n, int64_t m, const double* lambda, double* R, int64_t ldr,
                          double* rnorm, double* xnorm, double* rel, void* workspace,
                          size_t workspace_bytes, void* stream);
int fe_residual_norms_f32(const float* AX, const float* X, const float* BX, int64_t ld,
                          int64_t n, int64_t m, const double* lambda, float* R, int64_t ldr,
                          double* rnorm, double* xnorm, double* rel, void* workspace,
                          size_t workspace_bytes, void* stream);
/* ||X[:, j]|| for j < m (MultiVector::column_norms, src/gpu/CudaMultiVector.cpp:435-474). */
int fe_column_norms_f64(const double* X, int64_t ld, int64_t n, int64_t m, double* norms,
                        void* workspace, size_t workspace_bytes, void* stream);
int fe_column_norms_f32(const float* X, int64_t ld, int64_t n, int64_t m, double* norms,
                        void* workspace, size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------
 * Small FP64 dense kernels (device-resident; replace cusolverDnDpotrf + its
 * info device-to-host sync and cublasDtrsm, src/core/Orthogonalization.cpp:211-235).
 * ------------------------------------------------------------------- */
/* In place: upper Cholesky factor R of the k-by-k SPD matrix G (G = R^T R);
 * the strictly lower part is zeroed. *info (device int) = 0 on success or
 * j+1 when the j-th pivot is not positive/finite (rank loss: the reference's
 * -1 return). */
int fe_potrf_upper_f64(double* G, int64_t k, int64_t ldg, int32_t* info, void* stream);
/* Rinv = R^{-1} for an upper-triangular k-by-k R (both column-major). */
int fe_trinv_upper_f64(const double* R, int64_t ldr, double* Rinv, int64_t ldi, int64_t k,
                       void* stream);
/* Cholesky and inverse in one launch for a batch of small SPD matrices (k <= 128,
 * matrix p column-major at G + p*ldg*k, upper triangle read): Rinv + p*ldi*k gets
 * chol(G_p)^{-1} (upper triangular, zero below), info[p] (device) 0 or the failed
 * pivot + 1. One CTA per matrix with the matrix in shared memory (the reference
 * factors and solves one projected matrix at a time, src/core/Orthogonalization.cpp:
 * 211-235). Asynchronous on `stream`. */
int fe_chol_inv_upper_batched_f64(int32_t count, const double* G, int64_t ldg, int64_t k,
                                  double* Rinv, int64_t ldi, int32_t* info, void* stream);
/* P = (P + P^T) / 2 in place (src/core/RitzExtraction.cpp:103). */
int fe_symmetrize_f64(double* P, int64_t k, int64_t ldp, void* stream);

/* ---------------------------------------------------------------------
 * Precision conversions between FP64 and FP32 blocks (row-major).
 * ------------------------------------------------------------------- */
int fe_convert_f64_to_f32(const double* src, int64_t lds, float* dst, int64_t ldd,
                          int64_t n, int64_t m, void* stream);
int fe_convert_f32_to_f64(const float* src, int64_t lds, double* dst, int64_t ldd,
                          int64_t n, int64_t m, void* stream);

/* ---------------------------------------------------------------------
 * Solver entry point (replaces fasteig_problem::solve for the Lanczos,
 * Chebyshev, LOBPCG, Davidson, Krylov-Schur and block Krylov-Schur solvers on the
 * CUDA executor, src/fasteig_problem.cpp:340-437, src/fasteig_solver.cpp:131-168).
 * The problem is given as host CSR (full symmetric storage, as
 * build_csr_from_sparse_matrix produces) and options as "key=value" lines
 * with the reference's keys (src/fasteig_options.cpp:51-112: nev, maxiter,
 * maxdim, maxblks, degree, which, solver, tol, seed, blksize, print_every:
 * the Lanczos convergence-check interval) plus
 * extensions (precision=fp64|mixed, block=<cols>, bounds=reference|ritz,
 * precond=none|jacobi, init=host|device, mixed_switch=<FP32 floor>,
 * locking=soft|hard: Chebyshev soft locking is the reference's, hard locking
 * keeps locked pairs final and orthonormalizes and projects only the active
 * block; for precision=mixed also tail_degree=<filter degree of the FP64 cycles>,
 * tail_guard=<columns past nev kept in the FP64 cycles>, tail_filter=refined|fp64,
 * tail_rr=split|fp64 (the FP64 cycles' projected operator Y^T A Y as
 * (Y^T Y) diag(theta) + Y^T (AY - Y diag(theta)) with the small second term on the
 * split-TF32 tensor cores, or as one FP64 Gram), rr=fused|cholqr). B != NULL makes the
 * problem
 * generalized (A x = l B x, B symmetric positive definite): LOBPCG and Davidson
 * then work in the B metric (extension; the reference's are standard-only), and
 * Krylov-Schur runs the reference's B-metric Lanczos on B^-1 A with B^-1
 * applied by conjugate gradients to 1e-14 (the reference factorizes B with
 * cuDSS); its status is 1 when the returned pairs miss tol.
 * Results: eigenvalues[nev], residual_norms[nev] (the reference's relative
 * residual), eigenvectors n-by-nev column-major (may be NULL), stats[12] (may
 * be NULL): iterations, status, solve seconds, SpMM launches, FP32 cycles, FP64
 * cycles, spectral lower and upper bounds, device ms in filter, in
 * orthogonalization, in Rayleigh-Ritz, and FP32 Cholesky passes redone with the
 * FP64-accumulated Gram.
 * ------------------------------------------------------------------- */
int fe_solve(fe_csr_t A, fe_csr_t B, const char* options, double* eigenvalues,
             double* residual_norms, double* eigenvectors, double* stats);

/* ---------------------------------------------------------------------
 * Batched Krylov-Schur (extension; the reference solves one problem per
 * process with KrylovSchurSolver::solve, src/KrylovSchurSolver.cpp:28-160):
 * `count` independent standard problems A[p] (all on one device) with nev[p]
 * wanted pairs each, solved together in lockstep on grouped kernels, one CUDA
 * graph per Lanczos step of the whole batch. Options as for fe_solve (which,
 * tol, maxiter, maxdim, seed, init); subspace dimension per problem
 * max(2 nev, 20, maxdim) capped at n and at 96. Each problem's arithmetic is
 * independent of the rest of the batch, so its results are the same alone.
 * Results concatenated in problem order: eigenvalues and residual_norms
 * (sum of nev), eigenvectors (may be NULL) as consecutive n[p]-by-nev[p]
 * column-major blocks, iterations[count] (restart cycles), status[count]
 * (0 = converged or at maxiter), stats[4] (may be NULL): seconds, restart
 * rounds, Lanczos steps, graph launches.
 * ------------------------------------------------------------------- */
int fe_batch_krylov_schur(int32_t count, const fe_csr_t* A, const int64_t* nev,
                          const char* options, double* eigenvalues, double* residual_norms,
                          double* eigenvectors, int32_t* iterations, int32_t* status,
                          double* stats);

/* ---------------------------------------------------------------------
 * Grouped Chebyshev (extension; the reference runs one ChebyshevSolver::solve
 * per problem, src/ChebyshevSolver.cpp:67-221): `count` standard problems A[p]
 * (one device) with their own option strings, solved together. Problems of one
 * subspace width (the solve's capacity rounded up to a multiple of 32) and
 * filter degree form a group; each cycle of a group runs every member's filter,
 * Cholesky QR and Rayleigh-Ritz in grouped kernels over the concatenated
 * block-diagonal operator (one CUDA graph per cycle once membership is
 * stable), and members leave as they converge. Eligible problems: solver
 * Chebyshev, precision fp64 or mixed, locking soft, which SR or LR, width <=
 * 512, one stored diagonal entry per row. Mixed problems filter in FP32 (the
 * rest of each cycle in FP64) in the FP32-filter group of their width until
 * their residuals reach the FP32 floor (mixed_switch) or stall, then continue in
 * the FP64 group. Each problem's arithmetic reads only its own rows, so its
 * result does not depend on the rest of the batch.
 * Results per problem: eigenvalues[p][nev_p], residual_norms[p][nev_p] (the
 * reference's relative residual), eigenvectors[p] (n_p-by-nev_p column-major;
 * the array or any entry may be NULL), stats[count * FE_GROUP_STATS] (may be
 * NULL): cycles, status (0 converged, 1 at maxiter), seconds in the group,
 * width, spectral lower and upper bounds, then the batch's total group cycles,
 * graph replays and repacks, the problem's status code, and its FP32-filter
 * cycles.
 * ------------------------------------------------------------------- */
#define FE_GROUP_STATS 11
int fe_grouped_chebyshev(int32_t count, const fe_csr_t* A, const char* const* options,
                         double* const* eigenvalues, double* const* residual_norms,
                         double* const* eigenvectors, double* stats);

/* Block-diagonal operator of `count` CSR handles on one device (part p's rows and
 * columns follow those of parts 0..p-1); an SpMM on it is the grouped SpMM of
 * all parts in one launch (the reference applies one operator per process).
 * The result is a new handle (release with fe_csr_destroy); parts stay valid. */
int fe_csr_block_diag(int32_t count, const fe_csr_t* parts, fe_csr_t* out);

/* Symmetric eigensolver for one small dense FP64 matrix on the device (replaces
 * the projected-matrix Dsyevd of src/gpu/CudaLanczosWorkspace.cpp:155-157 and the
 * host SelfAdjointEigenSolver of src/core/RitzExtraction.cpp:104): A (k-by-k,
 * column-major, lda >= k) is replaced by its orthonormal eigenvectors, W[k] gets
 * the eigenvalues in ascending order, *info (device int) is 0, or 1 for
 * non-finite input. Householder tridiagonalization in one CTA, bisection for the
 * eigenvalues, inverse iteration (clusters re-orthogonalized) for the vectors,
 * back-transformation; k <= 8192. Asynchronous on `stream`; workspace from
 * fe_syevd_f64_workspace_bytes(k). */
size_t fe_syevd_f64_workspace_bytes(int64_t k);
int fe_syevd_f64(double* A, int64_t lda, int64_t k, double* W, int32_t* info, void* workspace,
                 size_t workspace_bytes, void* stream);

/* Batched symmetric eigensolver for `count` small FP64 matrices (replaces one
 * Dsyevd per projected matrix, src/gpu/CudaLanczosWorkspace.cpp:155): sizes
 * m[count] (host array, each in [1, 8192]), matrix p column-major at
 * A + p*lda*lda on the device (lda >= max m; A is not modified); ascending
 * eigenvalues to W + p*lda, eigenvectors to Z + p*lda*lda. Batches of matrices
 * up to 96 run a parallel cyclic Jacobi kernel (one CTA per matrix), larger ones
 * the tridiagonal path of fe_syevd_f64 (one CTA per matrix per stage); returns
 * after the stream has finished. */
int fe_syevd_batched_f64(int32_t count, const int32_t* m, const double* A, int64_t lda,
                         double* W, double* Z, void* stream);

/* ---------------------------------------------------------------------
 * Request server (extension; the reference's fasteig_problem::solve,
 * src/fasteig_problem.cpp:340-437, is one blocking solve per call).
 * A server owns `slots` worker threads on `device`. Submitted requests are
 * admitted in arrival order as soon as a slot is free and the request's device
 * memory bound (its blocks and workspaces) fits the budget
 * (memory_budget_bytes, or 90 % of the free memory at creation when <= 0); a
 * request larger than the budget runs alone. Each admitted request runs the
 * fe_solve path on its own stream, so concurrent requests overlap on the GPU
 * and each result is the one fe_solve gives alone. The caller keeps A (and B)
 * alive until the request is collected.
 *   fe_server_submit: options as for fe_solve; returns a request id.
 *   fe_server_wait: blocks (timeout < 0) or up to timeout seconds; FE_PENDING
 *     if still queued or running, else the solve's status. On completion
 *     writes eigenvalues[nev], residual_norms[nev] and stats[18] (the 12
 *     fe_solve stats, then seconds queued, seconds running, latency from
 *     submission, admitted memory bytes, start and end in seconds since the
 *     server was created) and forgets the request.
 *   fe_server_destroy: finishes running requests, drops queued ones.
 * A request whose options carry group=1 and that fe_grouped_chebyshev accepts
 * runs in a grouped lane instead (one per width and degree, beside the
 * slots): it joins the lane's group at the next cycle boundary once its memory
 * fits, advances with the other admitted members in grouped kernels, and leaves
 * when it converges (continuous batching); its stats are the fe_solve layout
 * with iterations, status, seconds and bounds filled.
 * ------------------------------------------------------------------- */
typedef struct fe_server* fe_server_t;
int fe_server_create(int32_t device, int32_t slots, int64_t memory_budget_bytes,
                     fe_server_t* out);
int fe_server_submit(fe_server_t server, fe_csr_t A, fe_csr_t B, const char* options,
                     int64_t* request_id);
int fe_server_wait(fe_server_t server, int64_t request_id, double timeout_seconds,
                   double* eigenvalues, double* residual_norms, double* stats);
int fe_server_destroy(fe_server_t server);
/* Counters of the grouped lanes, out[count] (up to 6): requests served grouped,
 * group cycles, graph replays, repacks, lanes, largest group seen. */
int fe_server_stats(fe_server_t server, double* out, int32_t count);

#ifdef __cplusplus
}
#endif

#endif /* FASTEIG_B200_H */

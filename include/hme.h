/* hme -- a B200-native (sm_100a) exact modular matrix engine.  C ABI.
 *
 * Drop-in device layer for the matrix engine of drjanosch42/hacs 0.2.1.  Each
 * entry point names the reference interface it replaces (file:line in the
 * reference tree); the C++ seam files under integration/ install these behind
 * the reference's own seams (the device RREF hook, the Z/2^k device LU table,
 * the micro-bench GPU hooks, the tape's device kernels, the Z/2^k and Z/3^k
 * Smith / Howell calls).
 *
 * Conventions (the reference's, ENGINE_API.md Sec. 1-5):
 *   - matrices are row-major uint32 with an explicit leading dimension in
 *     elements; every residue is canonical, in [0, p);
 *   - moduli: 2 <= p < 2^32 (fields: p prime; rings: p = ell^k);
 *   - op: HME_SET (C = A*B), HME_ADD (C += A*B), HME_SUB (C -= A*B), mod p;
 *   - every call returns HME_OK (0) or a negative HME_E* code; the message of
 *     the last failure on the calling thread is hme_last_error().  No C++
 *     exception crosses this boundary;
 *   - "_dev" entry points take device pointers and are asynchronous on the
 *     context's stream; the others take host pointers, copy in, compute and
 *     copy out, and return when the result is in host memory;
 *   - one context per thread at a time (the reference's "one driver thread per
 *     backend", ENGINE_API.md:1332-1333); different contexts are independent.
 */
#ifndef HME_H
#define HME_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define HME_API __attribute__((visibility("default")))
#else
#define HME_API
#endif

#define HME_OK 0
#define HME_EINVAL (-1)       /* contract violation (shape, modulus, alignment, op) */
#define HME_ECUDA (-2)        /* CUDA runtime / driver error */
#define HME_ENOMEM (-3)       /* device memory exhausted */
#define HME_ETIMEOUT (-4)     /* a bounded device-side wait ran out (kernel returned early) */
#define HME_EUNSUPPORTED (-5) /* no sm_100 device, or a case outside the supported range */
#define HME_ENOTINSPAN (-6)   /* solve: a right-hand side is not in the column span */

#define HME_SET 0
#define HME_ADD 1
#define HME_SUB 2

typedef struct hme_ctx hme_ctx;

/* ---- context ---------------------------------------------------------------
 * Replaces engine::cuda::CudaCtx (src/Cuda/CudaCtx.h:51-256): device choice,
 * stream, device workspace (grown on demand and reused), device error word. */
HME_API int hme_ctx_create(int device, hme_ctx **out);
HME_API int hme_ctx_destroy(hme_ctx *ctx);
/* Run the context's work on a caller-owned cudaStream_t (NULL = the CUDA
 * legacy default stream); hme_ctx_own_stream() is the stream the context
 * created and uses until this is called. */
HME_API int hme_ctx_set_stream(hme_ctx *ctx, void *cuda_stream);
HME_API void *hme_ctx_own_stream(const hme_ctx *ctx);
/* Keep (on != 0) every device workspace allocation of the context alive until
 * hme_ctx_destroy, also after a larger call replaced it: kernels captured in a
 * CUDA graph keep the pointers of the workspace they were captured with, so a
 * caller that replays graphs of this context's asynchronous entry points turns
 * this on (the tape's device layer does).  Off by default. */
HME_API int hme_ctx_set_workspace_retain(hme_ctx *ctx, int on);
/* Wait for the context's stream; reports a device-side timeout as HME_ETIMEOUT. */
HME_API int hme_ctx_sync(hme_ctx *ctx);
/* Kernel launches issued by this library on the context so far (a counter). */
HME_API uint64_t hme_ctx_launches(const hme_ctx *ctx);
/* Per-kernel CUDA-event timing on the context's stream (bench / profiling
 * use): while on, each kernel launch is bracketed by two events;
 * hme_ctx_kernel_time sums the elapsed milliseconds and the launch count of
 * one kernel name ("limb_gemm", "split_a", "split_b", ...; NULL = all). */
HME_API int hme_ctx_set_timing(hme_ctx *ctx, int on);
HME_API int hme_ctx_kernel_time(hme_ctx *ctx, const char *name, double *total_ms, uint64_t *count);
HME_API int hme_ctx_timing_reset(hme_ctx *ctx);
HME_API const char *hme_last_error(void);
/* Library version string. */
HME_API const char *hme_version(void);

/* ---- dense mod-p GEMM ------------------------------------------------------
 * C op= A*B mod p; A m x k, B k x n, C m x n.  The INT8-limb tcgen05 GEMM:
 * each residue splits into L unsigned bytes (L = 1 for p <= 2^8, 2 for
 * p <= 2^16, 3 for p <= 2^24, 4 otherwise), the limb products run on the
 * tensor cores with exact int32 accumulation over K chunks with
 * L * 255 * 255 * K_chunk < 2^31, and the epilogue recombines and reduces.
 * Bit-exact with engine::kernels::gemm<uint32_t>.
 *
 * hme_gemm_u32: host pointers.  Replaces the GPU micro-bench hook
 *   micro::GpuHooks::gemm (src/ModArithmetic/PerformanceSmokeValidation.h:158-165,
 *   installed at src/Cuda/CudaBench.cpp:339) and serves the CPU entry
 *   engine::kernels::gemm<uint32_t> (src/ModArithmetic/Kernels.h:178-185).
 * hme_gemm_u32_dev: device pointers, asynchronous.  Replaces
 *   engine::cuda::gemm / schur_update (src/Cuda/CudaKernels.h:120-140,
 *   cuda_kernels.cu:815) as called by the tape's DeviceBackend
 *   (src/Engine/DeviceBackend.cpp:391-604). */
HME_API int hme_gemm_u32(hme_ctx *ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t *A, size_t lda,
                 const uint32_t *B, size_t ldb, uint32_t *C, size_t ldc, int op);
HME_API int hme_gemm_u32_dev(hme_ctx *ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t *A,
                     size_t lda, const uint32_t *B, size_t ldb, uint32_t *C, size_t ldc, int op);

/* ---- dense mod-p GEMM over u64 residues -----------------------------------
 * C op= A*B mod p for u64 residues, any modulus 2 <= p < 2^64; entries of A
 * and B must be canonical (< p).  Bit-exact with engine::kernels::gemm
 * <uint64_t> (src/ModArithmetic/Kernels.h:178-185) and the device u64 regime
 * engine::cuda::gemm<uint64_t> (src/Cuda/cuda_kernels.cu:151-163, 365-381).
 * Method: p < 2^32 runs the u32 limb GEMM directly; larger p runs t limb GEMMs
 * modulo primes below 2^16 (t chosen so that their product exceeds
 * 4 k (p-1)^2) and reconstructs each entry by the Chinese remainder theorem,
 * reduced mod p once (Montgomery for odd p < 2^63).  Device workspace:
 * t (2 m Kp + 4 n Kp + 4 m n) bytes, Kp = k rounded up to 32, 64 or a multiple of 128, t <= 12
 * (p < 2^32: 4 (mk + kn + mn) bytes plus the u32 GEMM's planes).
 * hme_gemm_u64: host pointers (synchronous); hme_gemm_u64_dev: device
 * pointers, asynchronous on the context's stream. */
HME_API int hme_gemm_u64(hme_ctx *ctx, uint64_t p, uint32_t m, uint32_t n, uint32_t k, const uint64_t *A, size_t lda,
                         const uint64_t *B, size_t ldb, uint64_t *C, size_t ldc, int op);
HME_API int hme_gemm_u64_dev(hme_ctx *ctx, uint64_t p, uint32_t m, uint32_t n, uint32_t k, const uint64_t *A,
                             size_t lda, const uint64_t *B, size_t ldb, uint64_t *C, size_t ldc, int op);

/* ---- device level-1 / level-2 operations ----------------------------------
 * The rest of the device layer the tape's DeviceBackend drives, on device
 * pointers, asynchronous on the context's stream.  A view is (pointer, rows,
 * cols, row stride, column stride), strides in elements, as the reference's
 * DeviceView; residues are canonical (< p) unless stated; every result is the
 * exact residue.  Semantics of engine::cuda::* (src/Cuda/CudaKernels.h):
 *
 * hme_gemm_nt_u32_dev       C op= A B^T, B given n x k row-major   (:126-129)
 * hme_schur_update_u32_dev  C -= L U                                (:131-134)
 * hme_gemv_u32_dev          y op= A x, x k x 1, y m x 1            (:189-192)
 * hme_axpy_u32_dev          y = y +/- alpha x, alpha canonical     (:194-197)
 * hme_scal_u32_dev          x = alpha x                             (:199-200)
 * hme_copy_u32_dev          dst = src, windows must not overlap     (:203-204)
 * hme_transpose_u32_dev     dst(i, j) = src(j, i); dst rows x cols  (:207-208)
 * hme_fill_u32_dev          x(i, j) = value                         (:212-213)
 * hme_axpy_identity_u32_dev y(i, i) +/-= alpha, i < min(rows, cols) (:218-219)
 * hme_gather_u32_dev        c(i, t) [+]= alpha [row_off + r(i) == col(t)]
 *                             + beta a(r(i), col(t)), r(i) = rows[i] or i,
 *                             col(t) = cols[t] or t; a (a_rows x a_cols)
 *                             may be NULL (beta ignored) and must not
 *                             overlap c; indices are not range-checked;
 *                             accumulate 0 = Set                (:228-231)
 * hme_canonicalise_u32_dev  v = v >= p ? v - p : v (Lazy2p form, 2p <= 2^32)
 *                                                                   (:233-234)
 * hme_canonicalise_acc64_u32_dev  dst = acc mod p, u64 accumulators (:237-238)
 * hme_trsm_unit_u32_dev     B <- T^-1 B in place, T m x m unit lower (lower
 *                             != 0) or unit upper, only the strict triangle
 *                             read; T and B row-major; T must not overlap B
 *                                                                   (:245-247)
 * Bodies of the reference: src/Cuda/cuda_kernels.cu:952-1130. */
HME_API int hme_gemm_nt_u32_dev(hme_ctx *ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t *A,
                                size_t lda, const uint32_t *B, size_t ldb, uint32_t *C, size_t ldc, int op);
HME_API int hme_schur_update_u32_dev(hme_ctx *ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t *L,
                                     size_t ldl, const uint32_t *U, size_t ldu, uint32_t *C, size_t ldc);
HME_API int hme_gemv_u32_dev(hme_ctx *ctx, uint32_t p, uint32_t m, uint32_t k, const uint32_t *A, size_t a_rs,
                             size_t a_cs, const uint32_t *x, size_t x_rs, uint32_t *y, size_t y_rs, int op);
HME_API int hme_axpy_u32_dev(hme_ctx *ctx, uint32_t p, uint32_t alpha, uint32_t rows, uint32_t cols, const uint32_t *x,
                             size_t x_rs, size_t x_cs, uint32_t *y, size_t y_rs, size_t y_cs, int subtract);
HME_API int hme_scal_u32_dev(hme_ctx *ctx, uint32_t p, uint32_t alpha, uint32_t rows, uint32_t cols, uint32_t *x,
                             size_t rs, size_t cs);
HME_API int hme_copy_u32_dev(hme_ctx *ctx, uint32_t rows, uint32_t cols, const uint32_t *src, size_t s_rs, size_t s_cs,
                             uint32_t *dst, size_t d_rs, size_t d_cs);
HME_API int hme_transpose_u32_dev(hme_ctx *ctx, uint32_t rows_dst, uint32_t cols_dst, const uint32_t *src,
                                  size_t s_rs, size_t s_cs, uint32_t *dst, size_t d_rs, size_t d_cs);
HME_API int hme_fill_u32_dev(hme_ctx *ctx, uint32_t rows, uint32_t cols, uint32_t *x, size_t rs, size_t cs,
                             uint32_t value);
HME_API int hme_axpy_identity_u32_dev(hme_ctx *ctx, uint32_t p, uint32_t alpha, uint32_t rows, uint32_t cols,
                                      uint32_t *y, size_t rs, size_t cs, int subtract);
HME_API int hme_gather_u32_dev(hme_ctx *ctx, uint32_t p, uint32_t alpha, uint32_t beta, const uint32_t *a,
                               uint32_t a_rows, uint32_t a_cols, size_t a_rs, size_t a_cs, uint32_t row_off,
                               const uint32_t *cols, const uint32_t *rows, uint32_t c_rows, uint32_t c_cols,
                               uint32_t *c, size_t c_rs, size_t c_cs, int accumulate);
HME_API int hme_canonicalise_u32_dev(hme_ctx *ctx, uint32_t p, uint32_t rows, uint32_t cols, uint32_t *v, size_t rs,
                                     size_t cs);
HME_API int hme_canonicalise_acc64_u32_dev(hme_ctx *ctx, uint32_t p, uint32_t rows, uint32_t cols,
                                           const uint64_t *acc, size_t a_rs, size_t a_cs, uint32_t *dst,
                                           size_t d_rs, size_t d_cs);
HME_API int hme_trsm_unit_u32_dev(hme_ctx *ctx, uint32_t p, int lower, uint32_t m, uint32_t n, const uint32_t *T,
                                  size_t ldt, uint32_t *B, size_t ldb);

/* The same level-1 operations over u64 residues (2 <= p < 2^64; entries and
 * scalars canonical below p), the uint64_t instantiations of
 * engine::cuda::axpy / scal / copy / transpose / fill / axpy_identity /
 * gather / canonicalise (src/Cuda/CudaKernels.h:194-234, bodies
 * cuda_kernels.cu:986-1088): products formed in 128 bits and reduced once;
 * the lazy form of hme_canonicalise_u64_dev needs 2p <= 2^64.  The u64 GEMM
 * is hme_gemm_u64_dev. */
HME_API int hme_axpy_u64_dev(hme_ctx *ctx, uint64_t p, uint64_t alpha, uint32_t rows, uint32_t cols,
                             const uint64_t *x, size_t x_rs, size_t x_cs, uint64_t *y, size_t y_rs, size_t y_cs,
                             int subtract);
HME_API int hme_scal_u64_dev(hme_ctx *ctx, uint64_t p, uint64_t alpha, uint32_t rows, uint32_t cols, uint64_t *x,
                             size_t rs, size_t cs);
HME_API int hme_copy_u64_dev(hme_ctx *ctx, uint32_t rows, uint32_t cols, const uint64_t *src, size_t s_rs,
                             size_t s_cs, uint64_t *dst, size_t d_rs, size_t d_cs);
HME_API int hme_transpose_u64_dev(hme_ctx *ctx, uint32_t rows_dst, uint32_t cols_dst, const uint64_t *src,
                                  size_t s_rs, size_t s_cs, uint64_t *dst, size_t d_rs, size_t d_cs);
HME_API int hme_fill_u64_dev(hme_ctx *ctx, uint32_t rows, uint32_t cols, uint64_t *x, size_t rs, size_t cs,
                             uint64_t value);
HME_API int hme_axpy_identity_u64_dev(hme_ctx *ctx, uint64_t p, uint64_t alpha, uint32_t rows, uint32_t cols,
                                      uint64_t *y, size_t rs, size_t cs, int subtract);
HME_API int hme_gather_u64_dev(hme_ctx *ctx, uint64_t p, uint64_t alpha, uint64_t beta, const uint64_t *a,
                               uint32_t a_rows, uint32_t a_cols, size_t a_rs, size_t a_cs, uint32_t row_off,
                               const uint32_t *cols, const uint32_t *rows, uint32_t c_rows, uint32_t c_cols,
                               uint64_t *c, size_t c_rs, size_t c_cs, int accumulate);
HME_API int hme_canonicalise_u64_dev(hme_ctx *ctx, uint64_t p, uint32_t rows, uint32_t cols, uint64_t *v, size_t rs,
                                     size_t cs);

/* ---- elimination over F_p (p prime, p < 2^32) --------------------------------
 * Device-resident blocked LU: a cooperative panel kernel (pivot = leftmost
 * column with a non-zero in the Schur complement, topmost such row), row
 * permutation, unit-lower TRSM and the limb GEMM for every trailing update;
 * RREF = U1^-1 U by a blocked backward substitution on the free columns.  The
 * RREF, pivots, rank and determinant are unique, so every output equals the
 * reference's bit for bit.  A composite p is refused with HME_EINVAL (the
 * reference's field-only rule, ENGINE_API.md Sec. 13.3).
 *
 * hme_rref_u32: in-place RREF of a host matrix (leading 1, zero rows at the
 *   bottom), pivot columns ascending into pivots[] (min(m, n) entries), rank.
 *   Replaces elim::DeviceRrefHook with want_rref = true
 *   (src/ModArithmetic/DenseElim.h:121-123, installed at src/Engine/TapeElim.cpp:250;
 *   the reference's own hook, cuda::imma_rref, serves p <= 127 only) and
 *   serves elim::rref (DenseElim.h:153-158, DenseElim.cpp:921).
 * hme_rref_u32_dev: the same on a device matrix (in place).
 * hme_rank_profile_u32: pivots and rank only; A untouched.  Replaces the hook's
 *   want_rref = false arm and elim::column_rank_profile (DenseElim.h:160-169).
 * hme_det_u32: det(A) mod p of a square matrix (sign of the row permutation
 *   times the product of the U diagonal; 0 when singular).  The reference has
 *   no determinant entry point; this is the restatement of its PLU
 *   (DenseElim.cpp:323-560).
 * hme_rref_det_u32: RREF, pivots, rank and determinant of a square matrix in
 *   one factorisation.
 * hme_kernel_basis_u32: the (n - rank) x n kernel basis of A, one row per free
 *   column ascending (1 there, -R[i][free] at pivot i): elim::kernel_basis of
 *   the RREF (DenseElim.h:171-179).  K needs n rows of capacity.
 * hme_inverse_u32: A^-1 through RREF([A | I]); *invertible = 0 when singular
 *   (elim::inverse, DenseElim.h:186-189).
 * hme_solve_u32: X (nb x ny) with B X = Y through RREF([B | Y]); column t of X
 *   is the reference's result[t] (elim::solve_multi_rhs, DenseElim.h:191-197);
 *   HME_ENOTINSPAN when a column of Y is outside the span of B's columns.
 * hme_ctx_set_elim_options: panel width (<= 128), rows per CTA of the panel
 *   kernel, cap on its grid, block of the backward substitution (0 = default).
 *   Tuning only: no option changes a value.
 * hme_ctx_set_panel_kernel: which kernel factors the LU panels: 0 automatic
 *   (over a field, the top-block path first: when the panel's top rows factor
 *   with non-zero diagonal entries they are its pivots and no search runs;
 *   otherwise, and over Z/ell^k, the thread-block-cluster kernel whenever the
 *   panel's active rows fit the shared memory of one cluster, else the
 *   cooperative grid kernel), 1 always
 *   the grid kernel, 2 the cluster kernel (HME_EINVAL from a factorisation
 *   whose panel does not fit), 3 the cluster kernel with 1024 threads per CTA
 *   (2 uses 512 while a CTA holds at most 512 rows).  Tuning only: every mode
 *   gives the same outputs. */
HME_API int hme_rref_u32(hme_ctx *ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t *A, size_t lda,
                         uint32_t *pivots, uint32_t *rank);
HME_API int hme_rref_u32_dev(hme_ctx *ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t *A, size_t lda,
                             uint32_t *pivots, uint32_t *rank);
HME_API int hme_rank_profile_u32(hme_ctx *ctx, uint32_t p, uint32_t m, uint32_t n, const uint32_t *A, size_t lda,
                                 uint32_t *pivots, uint32_t *rank);
HME_API int hme_det_u32(hme_ctx *ctx, uint32_t p, uint32_t n, const uint32_t *A, size_t lda, uint32_t *det);
HME_API int hme_rref_det_u32(hme_ctx *ctx, uint32_t p, uint32_t n, uint32_t *A, size_t lda, uint32_t *pivots,
                             uint32_t *rank, uint32_t *det);
HME_API int hme_kernel_basis_u32(hme_ctx *ctx, uint32_t p, uint32_t m, uint32_t n, const uint32_t *A, size_t lda,
                                 uint32_t *K, size_t ldk, uint32_t *nullity);
HME_API int hme_inverse_u32(hme_ctx *ctx, uint32_t p, uint32_t n, const uint32_t *A, size_t lda, uint32_t *Ainv,
                            size_t ldi, int *invertible);
HME_API int hme_solve_u32(hme_ctx *ctx, uint32_t p, uint32_t m, uint32_t nb, uint32_t ny, const uint32_t *B,
                          size_t ldb, const uint32_t *Y, size_t ldy, uint32_t *X, size_t ldx);
HME_API int hme_ctx_set_elim_options(hme_ctx *ctx, int panel, int rows_per_cta, int panel_ctas, int back_block);
/* hme_ctx_set_elim_lookahead: on (the default) factors the next panel on a
 * second stream while the rest of the current panel's trailing update runs
 * (its GEMM leaving the panel's SMs free); off factors each panel after the
 * whole update.  Tuning only: no setting changes a value. */
HME_API int hme_ctx_set_elim_lookahead(hme_ctx *ctx, int on);
HME_API int hme_ctx_set_panel_kernel(hme_ctx *ctx, int mode);
/* hme_ctx_elim_panel_stats: panels of this context's eliminations so far that
 * the top-block path settled (mode 0 over a field: the nb x w top block of the
 * panel factors with non-zero diagonal entries, so the pivots are its rows in
 * order and the rows below take x U^-1), and panels that a searching kernel
 * factored. */
HME_API int hme_ctx_elim_panel_stats(const hme_ctx *ctx, uint64_t *block_panels, uint64_t *search_panels);

/* ---- Howell and Smith forms over Z/ell^k (ell prime, ell^k < 2^32) ----------
 * Input canonical in [0, ell^k) (else HME_EINVAL, the reference's entry check).
 *
 * hme_howell_u32: the Howell form of rowspan(A) (ENGINE_API.md Sec. 13.5): h
 *   rows (h <= n, possibly > m), leading columns strictly increasing, row i
 *   leading with exactly ell^pivot_v[i], entries above each pivot reduced into
 *   [0, ell^v).  H needs n rows of capacity (ldh >= n).  Replaces
 *   elim::howell (src/ModArithmetic/DenseElim.h:248-249), ring2k::howell
 *   (src/ModArithmetic/Binary/Ring2k.h:960-969, the Z/2^k device-ops table
 *   ring2k::device::Ops of Binary/Ring2kDevice.h:64-83 serves its LU) and
 *   ring3k::howell (Binary/Ring3k.h:101, host-only in the reference).
 * hme_smith_u32: the Smith valuations sigma (ascending, each < k; the
 *   non-zero Smith diagonal entries ell^sigma), count <= min(m, n).  Replaces
 *   ring2k::smith (Ring2k.h:702) and ring3k::smith (Ring3k.h:100; host-only in
 *   the reference); elim::invariant_factors (DenseElim.h:613-617) is
 *   {k - sigma} descending. */
HME_API int hme_howell_u32(hme_ctx *ctx, uint32_t ell, uint32_t k, uint32_t m, uint32_t n, const uint32_t *A,
                           size_t lda, uint32_t *H, size_t ldh, uint32_t *pivots, uint32_t *pivot_v, uint32_t *h);
HME_API int hme_smith_u32(hme_ctx *ctx, uint32_t ell, uint32_t k, uint32_t m, uint32_t n, const uint32_t *A,
                          size_t lda, uint32_t *sigma, uint32_t *count);

/* ---- batched job stream ------------------------------------------------------
 * A job is C = A*B mod p (A m x k, B k x n, device pointers) and/or the rank
 * of C over F_p.  Thousands of uneven jobs run as one launch per phase: the
 * GEMMs in one grouped persistent tcgen05 launch per modulus (the reference's
 * GemmBatch, src/Cuda/CudaKernels.h:141-185, needs equal shapes), the ranks
 * as rounds of a batched blocked LU (one CTA per job per panel, one grouped
 * limb GEMM for every job's trailing update).  No reference caller uses the
 * batch API yet; it serves the tape's BATCHED_GEMM node
 * (src/Engine/DeviceBackend.cpp:416-439, 551-559) and per-job rank queries
 * (elim::column_rank_profile, DenseElim.h:160-169).
 * hme_batch_gemm_u32_dev: every C_j = A_j B_j mod p_j.
 * hme_batch_rank_u32_dev: ranks[j] = rank of C_j (m x n) over F_{p_j} (p_j
 *   prime); destroys C_j.
 * hme_batch_gemm_rank_u32_dev: both, in that order.
 * hme_gen_jobs_u32_dev: the seeded synthetic job-stream matrices on the
 *   device (family 0: banded sparse, |i - j| <= 8, 5 % density, values in
 *   [-3, 3] mod p; family 1: dense uniform mod p); element (r, c) is output
 *   r*cols + c of splitmix64(seed). */
typedef struct hme_job {
    uint32_t p, m, n, k;
    const uint32_t *A;
    size_t lda;
    const uint32_t *B;
    size_t ldb;
    uint32_t *C;
    size_t ldc;
} hme_job;
typedef struct hme_gen_spec {
    uint32_t *dst;
    size_t ld;
    uint32_t rows, cols, p;
    int family;
    uint64_t seed;
} hme_gen_spec;
HME_API int hme_batch_gemm_u32_dev(hme_ctx *ctx, uint32_t njobs, const hme_job *jobs);
/* The same with every job's GEMM schedule given: variants[j] is one of the
 * GEMM variants below (0, 1 tensor-core wide / half-width tiles; 2, 3
 * CUDA-core 32 / 64 tiles) or -1 (the batch rule: one tensor-core launch per
 * modulus, wide tiles unless they leave SMs idle); variants = NULL takes the
 * context's scheduler (a pinned variant, else under the learned policy the
 * planner's decision per job's shape class, else the batch rule).  Jobs run as
 * one launch per (modulus, schedule) group; no schedule changes a residue. */
HME_API int hme_batch_gemm_u32_dev_plan(hme_ctx *ctx, uint32_t njobs, const hme_job *jobs, const int *variants);
HME_API int hme_batch_gemm_rank_u32_dev_plan(hme_ctx *ctx, uint32_t njobs, const hme_job *jobs, const int *variants,
                                             uint32_t *ranks);
HME_API int hme_batch_rank_u32_dev(hme_ctx *ctx, uint32_t njobs, const hme_job *jobs, uint32_t *ranks);
HME_API int hme_batch_gemm_rank_u32_dev(hme_ctx *ctx, uint32_t njobs, const hme_job *jobs, uint32_t *ranks);
HME_API int hme_gen_jobs_u32_dev(hme_ctx *ctx, uint32_t nmat, const hme_gen_spec *specs);
/* The rank rounds' schedules (no counterpart in the reference, whose ranks of
 * p > 127 run on the host, elim::column_rank_profile, DenseElim.h:160-169).
 * rank_variants[j] picks, for job j's rounds, the trailing-update variant and
 * the widest last panel (a job whose remaining columns fit it finishes in that
 * one panel on one CTA; otherwise its rounds take 32 columns):
 *   0 the grouped tensor-core limb GEMM, last panel up to 128 columns,
 *   1 the grouped tensor-core limb GEMM, 32-column rounds to the end,
 *   2 the CUDA-core update (a list of 64 x 64 tiles over a persistent grid,
 *     exact dot products), last panel up to 128 columns,
 *   3 the CUDA-core update, 32-column rounds to the end,
 *  -1 the batch rule: 0 for jobs of at most 128 rows, else 1 (a taller job's
 *     last panel is a long serial chain on one CTA that the round waits for).
 * rank_variants = NULL takes the context's scheduler (under the learned policy
 * the rank planner's decision per job's shape class, recorded by
 * hme_sched_plan_rank; else the batch rule).  No schedule changes a rank.
 * hme_batch_gemm_rank_u32_dev_sched: the GEMM phase under gemm_variants (as
 * hme_batch_gemm_u32_dev_plan), then the rank phase under rank_variants. */
HME_API int hme_batch_rank_u32_dev_sched(hme_ctx *ctx, uint32_t njobs, const hme_job *jobs, const int *rank_variants,
                                         uint32_t *ranks);
HME_API int hme_batch_gemm_rank_u32_dev_sched(hme_ctx *ctx, uint32_t njobs, const hme_job *jobs,
                                              const int *gemm_variants, const int *rank_variants, uint32_t *ranks);

/* ---- scheduler: GEMM variants, exhaustive autotuner, learned MLP planner -------
 * Variants (every one computes the same residues; a schedule changes speed
 * only): 0 limb tcgen05 GEMM with wide tiles, 1 with half-width tiles, 2 the
 * CUDA-core GEMM with 32 x 32 tiles, 3 with 64 x 64 tiles.  The reference has
 * no autotuner and no learned scheduler (its static rules:
 * src/Engine/EngineCostModel.h:22-51, pick_tile src/Cuda/cuda_kernels.cu:354-359).
 * hme_gemm_u32_dev_variant: the GEMM with an explicit variant.
 * hme_ctx_set_gemm_variant: pin every GEMM of the context to one variant
 *   (-1 = the scheduler decides).
 * hme_ctx_set_sched_policy: 0 the shape heuristic, 1 the learned plan
 *   (decisions recorded by hme_sched_plan, heuristic for unplanned shapes).
 * hme_autotune_gemm: the exhaustive autotuner: the median device time (ms) of
 *   each variant on an m x k x n product mod p into ms[hme_gemm_variant_count()].
 * hme_mlp_*: the scheduler's MLP, 5 -> 64 -> 64 -> 64 -> 4, ReLU, trained on
 *   the GPU (FP32 forward + backward of the mean squared error, Adam) and run
 *   in BF16 for inference.  X rows are 5 normalised features, Y rows 4
 *   normalised log-times.  hme_mlp_loss_grad returns the loss and its full
 *   parameter gradient (for checks against a CPU reference).
 * hme_sched_plan: BF16 inference for n products (shapes rows: p, m, n, k;
 *   optional density), arg-min variant per product into variants[], recorded
 *   in the context's plan; norm holds the 5 feature means then 5 std devs. */
typedef struct hme_mlp hme_mlp;
HME_API int hme_gemm_variant_count(void);
HME_API int hme_gemm_u32_dev_variant(hme_ctx *ctx, int variant, uint32_t p, uint32_t m, uint32_t n, uint32_t k,
                                     const uint32_t *A, size_t lda, const uint32_t *B, size_t ldb, uint32_t *C,
                                     size_t ldc, int op);
HME_API int hme_ctx_set_gemm_variant(hme_ctx *ctx, int variant);
HME_API int hme_ctx_set_sched_policy(hme_ctx *ctx, int policy);
HME_API int hme_autotune_gemm(hme_ctx *ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, int reps, float *ms);
/* The exhaustive autotuner of the batched stream: a batch of `count` jobs of
 * one shape run with every job on each variant in turn
 * (hme_batch_gemm_u32_dev_plan); ms[v] = median batch time / count, the
 * per-job device time of variant v inside a batch. */
HME_API int hme_autotune_batch(hme_ctx *ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, uint32_t count, int reps,
                               float *ms);
/* The exhaustive autotuner of the rank rounds: `count` products C = A B of
 * one shape (m <= 1024, p prime) built like the stream's jobs (banded sparse
 * operands when density < 0.5, dense uniform ones otherwise) and one anchor
 * (a dense 1024 x 1024 product of full rank on the batch rule, whose rounds run
 * as long as the stream's largest jobs'); the batched rank of fresh copies of
 * them under each rank schedule in turn (hme_batch_rank_u32_dev_sched), and of
 * the anchor alone.  ms[v] = (median time with the jobs on schedule v - median
 * time of the anchor alone) / count: the device time a job on schedule v adds
 * to a stream whose rounds run anyway (floored at 1 us per batch).  Fails
 * (HME_EINVAL) if two schedules disagree on a rank. */
HME_API int hme_autotune_batch_rank(hme_ctx *ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, float density,
                                    uint32_t count, int reps, float *ms);
HME_API int hme_mlp_param_count(void);
HME_API int hme_mlp_create(hme_ctx *ctx, uint64_t seed, hme_mlp **out);
HME_API int hme_mlp_destroy(hme_mlp *mlp);
HME_API int hme_mlp_get_params(hme_mlp *mlp, float *params);
HME_API int hme_mlp_set_params(hme_mlp *mlp, const float *params);
HME_API int hme_mlp_loss_grad(hme_mlp *mlp, uint32_t n, const float *X, const float *Y, float *loss, float *grad);
HME_API int hme_mlp_train(hme_mlp *mlp, uint32_t n, const float *X, const float *Y, uint32_t epochs, uint32_t batch,
                          float lr, uint64_t seed, float *final_loss);
HME_API int hme_mlp_predict_bf16(hme_mlp *mlp, uint32_t n, const float *X, float *Y);
HME_API int hme_sched_plan(hme_ctx *ctx, hme_mlp *mlp, uint32_t n, const uint32_t *shapes, const float *density,
                           const float *norm, int *variants);
/* Decisions recorded directly in the context's plan (table 0: the GEMM plan,
 * table 1: the rank plan), one per shape row (p, m, n, k), replacing the
 * network's for that shape class: the exhaustive autotuner's choice where the
 * network is not confident (hacs_b200.sched.plan_with_fallback).  HME_EINVAL
 * (nothing recorded) for a schedule outside 0..3.  No counterpart in the
 * reference. */
HME_API int hme_sched_plan_set(hme_ctx *ctx, int table, uint32_t n, const uint32_t *shapes, const int *variants);
/* The same for the rank rounds: a network trained on hme_autotune_batch_rank
 * timings picks each job's rank schedule (0..3 above), recorded in the
 * context's rank plan (used by the batched calls under the learned policy). */
HME_API int hme_sched_plan_rank(hme_ctx *ctx, hme_mlp *mlp, uint32_t n, const uint32_t *shapes, const float *density,
                                const float *norm, int *variants);

/* ---- device-resident blocked LU over Z/2^32 and Z/2^64 (ring2k device ops) ----
 * The session behind engine::ring2k::device::Ops (src/ModArithmetic/Binary/
 * Ring2kDevice.h:64-83, installed by src/hacs/Integral/Descent/
 * DescentSmithGpu.cpp:160-178; its device side in the reference is
 * engine::cuda::ring2k, src/Cuda/CudaRing2k.h:27-45).  ring2k::echelon_blocked
 * (Ring2k.h:539-695, driver Ring2kDeviceLU.h) factors each panel on the host
 * and hands the device one step per panel; every entry is an exact value of
 * Z/2^W (W = 8 * elem), bit-identical to the host LU.
 *
 * hme_r2k_plan: the column window cw for an m x n matrix of elem-byte entries
 *   (4 or 8) with this panel width: n when the session fits the device's free
 *   memory (less a reserve of max(1 GiB, 2 % of the card), capped at vram_cap
 *   bytes when non-zero), a multiple of panel below n (tiled), or 0 (decline:
 *   the host LU runs).  Ops::plan.
 * hme_r2k_session_bytes: device bytes of a session (window, L store, planes).
 * hme_r2k_open: a session on `device` for m rows and a window of cw columns
 *   (Ops::open); its own stream pair and pinned staging.
 * hme_r2k_put / hme_r2k_get: synchronous copies between a host block (ld ldh
 *   elements) and the window's rows [r0, r0+rows) x columns [c0, c0+cols)
 *   (Ops::put / Ops::get).
 * hme_r2k_step: one panel step (Ops::step with StepArgs, Ring2kDevice.h:49-62):
 *   the factored panel (rows r .. m-1, columns [pc0, pc1), ld ldp; NULL = none)
 *   written into the window; the nswaps row pairs of `swaps` exchanged in order
 *   on every other window column of [0, w); the unit-lower solve with L's rows
 *   0 .. np-1 (L row 0 = matrix row r, ld ldl) on the pivot rows, columns
 *   [u0, w); C -= L21 U12 on rows r+np .. m-1, columns [u0, w); lookahead: rows
 *   r+np .. m-1 of the columns [la0, la1) are read back once updated (empty
 *   when la0 == la1).  w = 0 means the session's cw.  The host buffers are
 *   copied before the call returns; the device work is asynchronous.
 * hme_r2k_fetch: waits for the last step's lookahead block and copies it to a
 *   host block (ld ldh elements) (Ops::fetch).
 * hme_r2k_close: frees the session; reports a device-side timeout seen in it
 *   (Ops::close). */
typedef struct hme_r2k hme_r2k;
typedef struct hme_r2k_step_args {
    uint32_t m;
    uint32_t r, np;
    uint32_t pc0, pc1;
    const void *panel;
    size_t ldp;
    const uint32_t *swaps;
    uint32_t nswaps;
    const void *L;
    size_t ldl;
    uint32_t u0;
    uint32_t la0, la1;
    uint32_t w;
} hme_r2k_step_args;
HME_API uint32_t hme_r2k_plan(int device, uint32_t elem, uint32_t m, uint32_t n, uint32_t panel, uint64_t vram_cap);
HME_API size_t hme_r2k_session_bytes(uint32_t elem, uint32_t m, uint32_t cw, uint32_t panel);
HME_API int hme_r2k_open(int device, uint32_t elem, uint32_t m, uint32_t cw, uint32_t panel, hme_r2k **out);
HME_API int hme_r2k_put(hme_r2k *s, const void *host, size_t ldh, uint32_t r0, uint32_t rows, uint32_t c0,
                        uint32_t cols);
HME_API int hme_r2k_get(hme_r2k *s, void *host, size_t ldh, uint32_t r0, uint32_t rows, uint32_t c0, uint32_t cols);
HME_API int hme_r2k_step(hme_r2k *s, const hme_r2k_step_args *a);
HME_API int hme_r2k_fetch(hme_r2k *s, void *host, size_t ldh);
HME_API int hme_r2k_close(hme_r2k *s);

/* The GEMM above (same kernels, same result bits) for callers that cannot
 * allocate device memory when they call it -- a plugin inside another runtime
 * that owns the device-memory budget, or a latency-critical path where
 * cudaMalloc / cudaFree would synchronise the device.  It takes no context
 * and allocates nothing: the limb planes live in a 32 MiB scratch array
 * compiled into the library (every GPU that loads the library holds it until
 * the process exits).  It runs on the calling thread's current device, on
 * `cuda_stream` (NULL = the legacy default stream), and returns when C is
 * final.  The planes of one call, L*m*Kp + L*L*n*Kp bytes (each rounded up
 * to 256; Kp = k rounded up to 16; L limbs as above), must fit 32 MiB, else
 * HME_EINVAL before anything runs.  The first call on a device does that
 * device's set-up (scratch address lookup, kernel attributes).  The call
 * synchronises its stream, so it cannot run while any stream is being
 * captured into a CUDA graph: it then returns HME_EINVAL before doing
 * anything.  All calls share the one scratch array: calls
 * that overlap on the GPU race and give wrong results, so serialise them.
 * No counterpart in the reference: an addition of this library. */
HME_API int hme_gemm_u32_dev_noalloc(uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t *A, size_t lda,
                                     const uint32_t *B, size_t ldb, uint32_t *C, size_t ldc, int op,
                                     void *cuda_stream);

/* FNV-1a-64 of a host matrix over (rows, cols, entries), each fed as a 64-bit
 * word, low byte first: the checksum the reference's micro bench prints and
 * compares across backends (src/ModArithmetic/PerformanceSmokeValidation.cpp:
 * 104-120, src/ModArithmetic/Fnv.h). */
HME_API uint64_t hme_fnv1a_u32(const uint32_t *M, uint32_t rows, uint32_t cols, size_t ld);

#ifdef __cplusplus
}
#endif
#endif /* HME_H */

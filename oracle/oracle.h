/* ORACLE / TEST INFRASTRUCTURE ONLY -- the CPU checker of the exact modular
 * matrix engine.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg may load liboracle.so; the product never does.
 *
 * A plain-C restatement of the reference's algorithms (drjanosch42/hacs 0.2.1),
 * each function citing the reference file:line it follows.  Pinned against the
 * reference's own compiled CPU engine (oracle/_ref/libhacsref.so, built from
 * the reference sources by oracle/Makefile) and against committed golden
 * fixtures (tests/golden/) in tests/test_oracle.py.
 *
 * All matrices are row-major uint32 with an explicit leading dimension; all
 * residues canonical in [0, p).  Functions return 0 on success, < 0 on a
 * contract violation. */
#ifndef HME_ORACLE_H
#define HME_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* splitmix64 / SeedFor / RandomEntries: PerformanceSmokeValidation.cpp:64-88 */
uint64_t orc_splitmix64(uint64_t *state);
uint64_t orc_seed_for(uint32_t r, uint32_t c, uint32_t ell, uint64_t salt);
void orc_random_entries(uint32_t *out, uint64_t count, uint32_t ell, uint64_t seed);
/* FNV-1a-64 over (rows, cols, entries) as 64-bit words: PerformanceSmokeValidation.cpp:104-120, Fnv.h:60-90 */
uint64_t orc_fnv_matrix(const uint32_t *M, uint32_t rows, uint32_t cols, uint32_t ld);

/* C op= A*B mod p, op 0 Set / 1 Add / 2 Sub: Kernels.h:178-185 contract, delayed
 * u64 accumulation over k_max products (ModCtx.h:139-142, 233-235). */
int orc_gemm_u32(uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t *A, uint32_t lda,
                 const uint32_t *B, uint32_t ldb, uint32_t *C, uint32_t ldc, int op);
int orc_gemm_u64(uint64_t p, uint32_t m, uint32_t n, uint32_t k, const uint64_t *A, uint32_t lda,
                 const uint64_t *B, uint32_t ldb, uint64_t *C, uint32_t ldc, int op);

/* In-place RREF over F_p (leading 1, zero rows at the bottom); pivot columns
 * ascending into pivots[] (>= min(m,n) entries).  Returns the rank.
 * DenseElim.h:153-158 (definition), RefLinAlg.cpp:60-100 (Gauss-Jordan rule). */
int64_t orc_rref_u32(uint32_t p, uint32_t m, uint32_t n, uint32_t *A, uint32_t lda, uint32_t *pivots);

/* det(A) mod p for square A by PLU with the leftmost-column / topmost-row rule
 * (DenseElim.cpp:323-560): sign(P) * prod U_ii.  A is not modified. */
int64_t orc_det_u32(uint32_t p, uint32_t n, const uint32_t *A, uint32_t lda);

/* Kernel basis from an RREF: DenseElim.h:171-179.  K is (n - rank) x n, ld n. */
int orc_kernel_basis_u32(uint32_t p, uint32_t n, const uint32_t *R, uint32_t ldr, const uint32_t *pivots,
                         uint32_t rank, uint32_t *K);

/* Inverse via RREF([A | I]): DenseElim.h:186-189.  Returns 1 if invertible. */
int orc_inverse_u32(uint32_t p, uint32_t n, const uint32_t *A, uint32_t *Ainv);

/* Solve B X = Y (B m x nb, Y m x ny) via RREF([B | Y]): DenseElim.h:191-197.
 * X is nb x ny (row t of the reference's result[t][j] is column t of X).
 * Returns 0, or -3 when some column of Y is not in the span. */
int orc_solve_u32(uint32_t p, uint32_t m, uint32_t nb, uint32_t ny, const uint32_t *B, const uint32_t *Y,
                  uint32_t *X);

/* Howell form of rowspan(A) over Z/ell^k (ENGINE_API.md Sec. 13.5, the
 * valuation-pivoting pass with closure rows at the bottom of the active list,
 * then reduce-above; DenseElim.cpp:722-820).  H receives h rows of n entries
 * (capacity n rows); returns h. */
int64_t orc_howell_u32(uint32_t ell, uint32_t kexp, uint32_t m, uint32_t n, const uint32_t *A, uint32_t lda,
                       uint32_t *H, uint32_t *pivots, uint32_t *pivot_v);

/* Smith valuations sigma (ascending, each < k) of A over Z/ell^k by global
 * minimal-valuation pivoting (Ring2k.h smith_naive, Ring3k.h smith_naive).
 * sigma holds min(m,n) entries; returns the count. */
int64_t orc_smith_u32(uint32_t ell, uint32_t kexp, uint32_t m, uint32_t n, const uint32_t *A, uint32_t lda,
                      uint32_t *sigma);

/* Modular inverse of a unit (extended Euclid), 0 when none. */
uint32_t orc_inv_mod(uint32_t a, uint32_t p);

#ifdef __cplusplus
}
#endif
#endif

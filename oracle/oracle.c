/* ORACLE / TEST INFRASTRUCTURE ONLY -- see oracle.h.  Plain C restatement of
 * the reference engine's algorithms; the checker, never the thing measured. */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ---- generators: PerformanceSmokeValidation.cpp:64-88 ------------------ */
uint64_t orc_splitmix64(uint64_t *state) {
    uint64_t z = (*state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

uint64_t orc_seed_for(uint32_t r, uint32_t c, uint32_t ell, uint64_t salt) {
    uint64_t s = 0xC0FFEE123456789ull ^ salt;
    s = s * 0x100000001B3ull + r;
    s = s * 0x100000001B3ull + c;
    s = s * 0x100000001B3ull + ell;
    return s;
}

void orc_random_entries(uint32_t *out, uint64_t count, uint32_t ell, uint64_t seed) {
    uint64_t st = seed;
    for (uint64_t i = 0; i < count; ++i) out[i] = (uint32_t)(orc_splitmix64(&st) % ell);
}

/* FNV-1a-64 fed with 64-bit words, low byte first (Fnv.h FnvU64). */
static uint64_t fnv_u64(uint64_t h, uint64_t v) {
    for (int i = 0; i < 8; ++i) {
        h ^= (v >> (8 * i)) & 0xffu;
        h *= 0x100000001b3ull;
    }
    return h;
}

uint64_t orc_fnv_matrix(const uint32_t *M, uint32_t rows, uint32_t cols, uint32_t ld) {
    uint64_t h = 0xcbf29ce484222325ull;
    h = fnv_u64(h, rows);
    h = fnv_u64(h, cols);
    for (uint32_t i = 0; i < rows; ++i)
        for (uint32_t j = 0; j < cols; ++j) h = fnv_u64(h, M[(size_t)i * ld + j]);
    return h;
}

/* ---- scalar arithmetic -------------------------------------------------- */
static inline uint32_t mulm(uint32_t a, uint32_t b, uint32_t p) { return (uint32_t)(((uint64_t)a * b) % p); }
static inline uint32_t addm(uint32_t a, uint32_t b, uint32_t p) {
    uint64_t s = (uint64_t)a + b;
    return (uint32_t)(s >= p ? s - p : s);
}
static inline uint32_t subm(uint32_t a, uint32_t b, uint32_t p) { return a >= b ? a - b : (uint32_t)((uint64_t)a + p - b); }

uint32_t orc_inv_mod(uint32_t a, uint32_t p) {
    /* extended Euclid on (a, p); 0 when gcd(a, p) != 1 */
    int64_t t0 = 0, t1 = 1;
    int64_t r0 = p, r1 = a % p;
    while (r1 != 0) {
        int64_t q = r0 / r1, tmp;
        tmp = r0 - q * r1; r0 = r1; r1 = tmp;
        tmp = t0 - q * t1; t0 = t1; t1 = tmp;
    }
    if (r0 != 1) return 0;
    if (t0 < 0) t0 += p;
    return (uint32_t)t0;
}

/* ---- GEMM ----------------------------------------------------------------
 * Kernels.h:178-185 / RefLinAlg.cpp gemm: exact sum of k products mod p.  The
 * u64 row accumulator holds at most k_max = floor((2^64-1)/(p-1)^2) products
 * between reductions (ModCtx.h:233-235). */
int orc_gemm_u32(uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t *A, uint32_t lda,
                 const uint32_t *B, uint32_t ldb, uint32_t *C, uint32_t ldc, int op) {
    if (p < 2 || op < 0 || op > 2) return -1;
    const uint64_t d = (uint64_t)(p - 1) * (p - 1);
    uint64_t kmax = d == 0 ? ~0ull : (~0ull) / d;
    if (kmax > 4096) kmax = 4096;
    uint64_t *acc = (uint64_t *)malloc(sizeof(uint64_t) * (n ? n : 1));
    if (!acc) return -2;
    for (uint32_t i = 0; i < m; ++i) {
        memset(acc, 0, sizeof(uint64_t) * n);
        uint32_t since = 0;
        for (uint32_t t = 0; t < k; ++t) {
            const uint64_t a = A[(size_t)i * lda + t];
            const uint32_t *b = B + (size_t)t * ldb;
            for (uint32_t j = 0; j < n; ++j) acc[j] += a * b[j];
            if (++since == kmax) {
                for (uint32_t j = 0; j < n; ++j) acc[j] %= p;
                since = 0;
            }
        }
        for (uint32_t j = 0; j < n; ++j) {
            const uint32_t r = (uint32_t)(acc[j] % p);
            uint32_t *c = C + (size_t)i * ldc + j;
            *c = op == 0 ? r : op == 1 ? addm(*c, r, p) : subm(*c, r, p);
        }
    }
    free(acc);
    return 0;
}

/* C op= A*B mod p over u64 residues, any 2 <= p < 2^64 (engine::kernels::gemm
 * <uint64_t>, src/ModArithmetic/Kernels.h:178-185; the u64 regime of
 * ModCtx<uint64_t>, ModCtx.h:226-248): each product reduced with a 128-bit
 * remainder, summed mod p.  Canonical inputs. */
int orc_gemm_u64(uint64_t p, uint32_t m, uint32_t n, uint32_t k, const uint64_t *A, uint32_t lda,
                 const uint64_t *B, uint32_t ldb, uint64_t *C, uint32_t ldc, int op) {
    if (p < 2 || op < 0 || op > 2) return -1;
    for (uint32_t i = 0; i < m; ++i)
        for (uint32_t j = 0; j < n; ++j) {
            unsigned __int128 s = 0;
            for (uint32_t t = 0; t < k; ++t) {
                s += (unsigned __int128)A[(size_t)i * lda + t] * B[(size_t)t * ldb + j] % p;
                if (s >= p) s -= p;
            }
            const uint64_t r = (uint64_t)s;
            uint64_t *c = C + (size_t)i * ldc + j;
            if (op == 0) *c = r;
            else if (op == 1) { const unsigned __int128 x = (unsigned __int128)*c + r; *c = (uint64_t)(x >= p ? x - p : x); }
            else *c = *c >= r ? *c - r : (uint64_t)((unsigned __int128)*c + p - r);
        }
    return 0;
}

/* ---- RREF over F_p ------------------------------------------------------
 * Gauss-Jordan with the legacy pivot rule (RefLinAlg.cpp rref; DenseElim.h
 * header): leftmost column with a non-zero at or below the current row,
 * topmost such row swapped into place, scaled to 1, eliminated above and
 * below.  RREF is unique, so any correct elimination agrees entrywise. */
int64_t orc_rref_u32(uint32_t p, uint32_t m, uint32_t n, uint32_t *A, uint32_t lda, uint32_t *pivots) {
    uint32_t rank = 0;
    for (uint32_t c = 0; c < n && rank < m; ++c) {
        uint32_t r = rank;
        while (r < m && A[(size_t)r * lda + c] == 0) ++r;
        if (r == m) continue;
        if (r != rank) {
            uint32_t *x = A + (size_t)r * lda, *y = A + (size_t)rank * lda;
            for (uint32_t j = 0; j < n; ++j) { uint32_t t = x[j]; x[j] = y[j]; y[j] = t; }
        }
        uint32_t *prow = A + (size_t)rank * lda;
        const uint32_t inv = orc_inv_mod(prow[c], p);
        if (inv == 0) return -1; /* not a field */
        for (uint32_t j = c; j < n; ++j) prow[j] = mulm(prow[j], inv, p);
        for (uint32_t i = 0; i < m; ++i) {
            if (i == rank) continue;
            uint32_t *row = A + (size_t)i * lda;
            const uint32_t f = row[c];
            if (f == 0) continue;
            for (uint32_t j = c; j < n; ++j) row[j] = subm(row[j], mulm(f, prow[j], p), p);
        }
        pivots[rank++] = c;
    }
    return rank;
}

/* ---- determinant ---------------------------------------------------------
 * No engine entry point exists; this follows the field PLU of
 * DenseElim.cpp:323-560 (leftmost column, topmost non-zero row swapped into
 * place): det = sign(P) * prod of the pivots, 0 when a column has no pivot. */
int64_t orc_det_u32(uint32_t p, uint32_t n, const uint32_t *A, uint32_t lda) {
    uint32_t *W = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n * (n ? n : 1));
    if (!W) return -2;
    for (uint32_t i = 0; i < n; ++i) memcpy(W + (size_t)i * n, A + (size_t)i * lda, sizeof(uint32_t) * n);
    uint32_t det = 1 % p;
    int neg = 0;
    for (uint32_t c = 0; c < n; ++c) {
        uint32_t r = c;
        while (r < n && W[(size_t)r * n + c] == 0) ++r;
        if (r == n) { det = 0; break; }
        if (r != c) {
            neg ^= 1;
            for (uint32_t j = 0; j < n; ++j) {
                uint32_t t = W[(size_t)r * n + j]; W[(size_t)r * n + j] = W[(size_t)c * n + j]; W[(size_t)c * n + j] = t;
            }
        }
        const uint32_t piv = W[(size_t)c * n + c];
        det = mulm(det, piv, p);
        const uint32_t inv = orc_inv_mod(piv, p);
        for (uint32_t i = c + 1; i < n; ++i) {
            const uint32_t f = mulm(W[(size_t)i * n + c], inv, p);
            if (f == 0) continue;
            for (uint32_t j = c; j < n; ++j)
                W[(size_t)i * n + j] = subm(W[(size_t)i * n + j], mulm(f, W[(size_t)c * n + j], p), p);
        }
    }
    free(W);
    if (neg && det != 0) det = p - det;
    return det;
}

/* ---- kernel basis: DenseElim.h:171-179 ----------------------------------- */
int orc_kernel_basis_u32(uint32_t p, uint32_t n, const uint32_t *R, uint32_t ldr, const uint32_t *pivots,
                         uint32_t rank, uint32_t *K) {
    uint32_t row = 0, pi = 0;
    for (uint32_t f = 0; f < n; ++f) {
        if (pi < rank && pivots[pi] == f) { ++pi; continue; }
        uint32_t *k = K + (size_t)row * n;
        memset(k, 0, sizeof(uint32_t) * n);
        k[f] = 1 % p;
        for (uint32_t i = 0; i < rank; ++i) {
            const uint32_t v = R[(size_t)i * ldr + f];
            k[pivots[i]] = v == 0 ? 0 : p - v;
        }
        ++row;
    }
    return 0;
}

/* ---- inverse: RREF([A | I]), DenseElim.h:186-189 -------------------------- */
int orc_inverse_u32(uint32_t p, uint32_t n, const uint32_t *A, uint32_t *Ainv) {
    const uint32_t w = 2 * n;
    uint32_t *M = (uint32_t *)calloc((size_t)n * w + 1, sizeof(uint32_t));
    uint32_t *piv = (uint32_t *)malloc(sizeof(uint32_t) * (w + 1));
    if (!M || !piv) { free(M); free(piv); return -2; }
    for (uint32_t i = 0; i < n; ++i) {
        memcpy(M + (size_t)i * w, A + (size_t)i * n, sizeof(uint32_t) * n);
        M[(size_t)i * w + n + i] = 1 % p;
    }
    const int64_t rank = orc_rref_u32(p, n, w, M, w, piv);
    int ok = rank == (int64_t)n && (n == 0 || piv[n - 1] == n - 1);
    if (ok)
        for (uint32_t i = 0; i < n; ++i) memcpy(Ainv + (size_t)i * n, M + (size_t)i * w + n, sizeof(uint32_t) * n);
    free(M);
    free(piv);
    return ok;
}

/* ---- solve: RREF([B | Y]), DenseElim.h:191-197 ---------------------------- */
int orc_solve_u32(uint32_t p, uint32_t m, uint32_t nb, uint32_t ny, const uint32_t *B, const uint32_t *Y,
                  uint32_t *X) {
    const uint32_t w = nb + ny;
    uint32_t *M = (uint32_t *)calloc((size_t)m * w + 1, sizeof(uint32_t));
    uint32_t *piv = (uint32_t *)malloc(sizeof(uint32_t) * (w + 1));
    if (!M || !piv) { free(M); free(piv); return -2; }
    for (uint32_t i = 0; i < m; ++i) {
        memcpy(M + (size_t)i * w, B + (size_t)i * nb, sizeof(uint32_t) * nb);
        memcpy(M + (size_t)i * w + nb, Y + (size_t)i * ny, sizeof(uint32_t) * ny);
    }
    const int64_t rank = orc_rref_u32(p, m, w, M, w, piv);
    int rc = 0;
    for (int64_t i = 0; i < rank; ++i)
        if (piv[i] >= nb) rc = -3;
    if (rc == 0) {
        memset(X, 0, sizeof(uint32_t) * (size_t)nb * ny);
        for (int64_t i = 0; i < rank; ++i)
            for (uint32_t t = 0; t < ny; ++t) X[(size_t)piv[i] * ny + t] = M[(size_t)i * w + nb + t];
    }
    free(M);
    free(piv);
    return rc;
}

/* ---- Z/ell^k helpers: ModCtx.h:284-311 ----------------------------------- */
static uint32_t val_of(uint32_t x, uint32_t ell, uint32_t k) {
    if (x == 0) return k;
    uint32_t v = 0;
    while (v < k && x % ell == 0) { x /= ell; ++v; }
    return v;
}
static uint32_t unit_of(uint32_t x, uint32_t ell) {
    if (x == 0) return 1;
    while (x % ell == 0) x /= ell;
    return x;
}

/* ---- Howell form over Z/ell^k: ENGINE_API.md Sec. 13.5 -------------------
 * Forward pass over columns with an ordered active list (rows of A top to
 * bottom): minimal valuation, ties to the topmost; the pivot row leaves the
 * list scaled to lead with ell^v; the other active rows are eliminated by
 * divide_exact multiples; for v > 0 the closure row ell^(k-v) * pivot is
 * appended at the bottom.  Then reduce-above, pivot columns left to right,
 * with the integer quotient q = H[i'][j_i] / ell^(v_i). */
int64_t orc_howell_u32(uint32_t ell, uint32_t kexp, uint32_t m, uint32_t n, const uint32_t *A, uint32_t lda,
                       uint32_t *H, uint32_t *pivots, uint32_t *pivot_v) {
    uint64_t q64 = 1;
    for (uint32_t i = 0; i < kexp; ++i) q64 *= ell;
    if (q64 > 0xffffffffull) return -1;
    const uint32_t q = (uint32_t)q64;
    uint32_t *pw = (uint32_t *)malloc(sizeof(uint32_t) * (kexp + 1));
    pw[0] = 1;
    for (uint32_t i = 1; i <= kexp; ++i) pw[i] = pw[i - 1] * ell;
    /* active list: capacity m + n rows (each pivot adds at most one closure row) */
    const size_t cap = (size_t)m + n + 1;
    uint32_t *store = (uint32_t *)malloc(sizeof(uint32_t) * cap * (n ? n : 1));
    uint32_t *act = (uint32_t *)malloc(sizeof(uint32_t) * cap);
    uint32_t *act2 = (uint32_t *)malloc(sizeof(uint32_t) * cap);
    size_t nstore = 0, nact = 0;
    for (uint32_t i = 0; i < m; ++i) {
        uint32_t *r = store + nstore * n;
        for (uint32_t j = 0; j < n; ++j) r[j] = A[(size_t)i * lda + j] % q;
        act[nact++] = (uint32_t)nstore++;
    }
    uint32_t h = 0;
    for (uint32_t c = 0; c < n; ++c) {
        uint32_t best = kexp, bi = 0;
        for (size_t t = 0; t < nact; ++t) {
            const uint32_t x = store[(size_t)act[t] * n + c];
            if (x == 0) continue;
            const uint32_t v = val_of(x, ell, kexp);
            if (v < best) { best = v; bi = (uint32_t)t; }
        }
        if (best == kexp) continue;
        const uint32_t v = best;
        uint32_t *prow = store + (size_t)act[bi] * n;
        const uint32_t u = unit_of(prow[c], ell);
        const uint32_t uinv = orc_inv_mod(u % q, q);
        for (uint32_t j = 0; j < n; ++j) prow[j] = mulm(prow[j], uinv, q);
        /* eliminate the other active rows */
        size_t na = 0;
        for (size_t t = 0; t < nact; ++t) {
            if (t == bi) continue;
            uint32_t *row = store + (size_t)act[t] * n;
            const uint32_t x = row[c];
            if (x != 0) {
                const uint32_t f = x / pw[v];
                for (uint32_t j = c; j < n; ++j) row[j] = subm(row[j], mulm(f, prow[j], q), q);
            }
            act2[na++] = act[t];
        }
        if (v > 0) {
            uint32_t *cl = store + nstore * n;
            int nz = 0;
            for (uint32_t j = 0; j < n; ++j) { cl[j] = mulm(pw[kexp - v], prow[j], q); nz |= cl[j] != 0; }
            if (nz) act2[na++] = (uint32_t)nstore++;
        }
        memcpy(H + (size_t)h * n, prow, sizeof(uint32_t) * n);
        pivots[h] = c;
        pivot_v[h] = v;
        ++h;
        memcpy(act, act2, sizeof(uint32_t) * na);
        nact = na;
    }
    /* reduce above */
    for (uint32_t i = 0; i < h; ++i) {
        const uint32_t ji = pivots[i], d = pw[pivot_v[i]];
        const uint32_t *ri = H + (size_t)i * n;
        for (uint32_t i2 = 0; i2 < i; ++i2) {
            uint32_t *r2 = H + (size_t)i2 * n;
            const uint32_t f = r2[ji] / d;
            if (f == 0) continue;
            for (uint32_t j = ji; j < n; ++j) r2[j] = subm(r2[j], mulm(f, ri[j], q), q);
        }
    }
    free(pw);
    free(store);
    free(act);
    free(act2);
    return h;
}

/* ---- Smith valuations over Z/ell^k ---------------------------------------
 * Global minimal-valuation pivoting (Ring2k.h smith_naive, Ring3k.h
 * smith_naive): the entry of least valuation anywhere in the remaining block
 * is the pivot; its row clears the column exactly (divide_exact), the pivot
 * row and column leave, and v is one Smith valuation. */
int64_t orc_smith_u32(uint32_t ell, uint32_t kexp, uint32_t m, uint32_t n, const uint32_t *A, uint32_t lda,
                      uint32_t *sigma) {
    uint64_t q64 = 1;
    for (uint32_t i = 0; i < kexp; ++i) q64 *= ell;
    if (q64 > 0xffffffffull) return -1;
    const uint32_t q = (uint32_t)q64;
    uint32_t *W = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)m * (n ? n : 1) + 4);
    uint32_t *rows = (uint32_t *)malloc(sizeof(uint32_t) * (m + 1));
    uint32_t *cols = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1));
    for (uint32_t i = 0; i < m; ++i)
        for (uint32_t j = 0; j < n; ++j) W[(size_t)i * n + j] = A[(size_t)i * lda + j] % q;
    for (uint32_t i = 0; i < m; ++i) rows[i] = i;
    for (uint32_t j = 0; j < n; ++j) cols[j] = j;
    uint32_t nr = m, nc = n, cnt = 0;
    uint32_t pwv = 1;
    (void)pwv;
    while (nr > 0 && nc > 0) {
        uint32_t best = kexp, bi = 0, bj = 0;
        for (uint32_t a = 0; a < nr && best > 0; ++a)
            for (uint32_t b = 0; b < nc; ++b) {
                const uint32_t x = W[(size_t)rows[a] * n + cols[b]];
                if (x == 0) continue;
                const uint32_t v = val_of(x, ell, kexp);
                if (v < best) { best = v; bi = a; bj = b; if (v == 0) break; }
            }
        if (best == kexp) break;
        uint32_t d = 1;
        for (uint32_t t = 0; t < best; ++t) d *= ell;
        const uint32_t pr = rows[bi], pc = cols[bj];
        uint32_t *prow = W + (size_t)pr * n;
        const uint32_t uinv = orc_inv_mod(unit_of(prow[pc], ell) % q, q);
        for (uint32_t b = 0; b < nc; ++b) prow[cols[b]] = mulm(prow[cols[b]], uinv, q);
        for (uint32_t a = 0; a < nr; ++a) {
            if (a == bi) continue;
            uint32_t *row = W + (size_t)rows[a] * n;
            const uint32_t x = row[pc];
            if (x == 0) continue;
            const uint32_t f = x / d;
            for (uint32_t b = 0; b < nc; ++b) row[cols[b]] = subm(row[cols[b]], mulm(f, prow[cols[b]], q), q);
        }
        sigma[cnt++] = best;
        rows[bi] = rows[--nr];
        cols[bj] = cols[--nc];
    }
    /* ascending */
    for (uint32_t i = 1; i < cnt; ++i) {
        uint32_t x = sigma[i], j = i;
        while (j > 0 && sigma[j - 1] > x) { sigma[j] = sigma[j - 1]; --j; }
        sigma[j] = x;
    }
    free(W);
    free(rows);
    free(cols);
    return cnt;
}

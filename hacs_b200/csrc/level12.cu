// Level-1 / level-2 device operations of the engine's device layer, on strided
// device views: y op= A x, axpy, scal, copy, transpose, fill, identity axpy,
// the gather used by the tape's assembly nodes, canonicalisation (from the
// lazy [0, 2p) form and from 64-bit accumulators), unit-triangular solves,
// C op= A B^T and the Schur update.
//
// Reference semantics: engine::cuda::gemv / axpy / scal / copy / transpose /
// fill / axpy_identity / gather / canonicalise / trsm_unit / gemm_nt /
// schur_update (src/Cuda/CudaKernels.h:120-131, 186-247; bodies
// src/Cuda/cuda_kernels.cu:952-1130): every view has a row stride and a column
// stride in elements (the reference's DeviceView), residues are canonical
// u32 below p unless stated, and every result is the exact residue, so the
// outputs equal the reference's element for element.
//
// B200 layout.  The element-wise kernels cut the window into tiles of one
// "outer" index by 1024 "inner" elements, the inner dimension being the one
// with unit stride when it is long enough (else the longer one): one integer
// division per tile, consecutive threads on consecutive addresses, and four
// independent loads per thread issued before any store, so that each SM keeps
// enough bytes in flight to stream HBM.  y op= A x runs one warp per row of A
// when A's rows are contiguous (one thread per row otherwise), four loads in
// flight per lane, and sums the 64-bit products exactly as a 96-bit value
// (a carry count beside a 64-bit sum) reduced once per row.  The triangular
// solve is blocked by 128 rows: one kernel solves a 128-row diagonal block in
// shared memory (32-row sub-blocks by warp substitution, four right-hand-side
// columns interleaved per warp, the sub-block updates between them in shared
// memory) and the limb GEMM (tensor cores) applies the block to the rows
// below (above) it.
#include <cuda_runtime.h>

#include <algorithm>

#include "hme_internal.h"

namespace hme {
namespace {

constexpr int kEwThreads = 256;             // threads per element-wise CTA
constexpr int kEwU = 4;                     // elements per thread per tile
constexpr int kEwTile = kEwThreads * kEwU;  // inner elements per tile
constexpr uint32_t kTrsmNB = 128;           // rows per diagonal block of the solve

// Iteration space of an element-wise op: outer x inner, `tpr` tiles per outer
// index.  Each operand has a stride along outer (so) and inner (si).
struct Ew {
    uint32_t outer, inner, tpr;
    uint64_t ntiles;
};
struct Strides {
    uint64_t so, si;
};

// Inner dimension: the unit-stride one when it holds at least 64 elements,
// else the longer one.
inline bool inner_is_cols(uint32_t rows, uint32_t cols, uint64_t rs, uint64_t cs) {
    if (cs == 1 && cols >= 64) return true;
    if (rs == 1 && rows >= 64) return false;
    return cols >= rows;
}
inline Ew make_ew(uint32_t rows, uint32_t cols, bool icols) {
    Ew e;
    e.outer = icols ? rows : cols;
    e.inner = icols ? cols : rows;
    e.tpr = (e.inner + kEwTile - 1) / kEwTile;
    e.ntiles = static_cast<uint64_t>(e.outer) * e.tpr;
    return e;
}
inline Strides strides_of(uint64_t rs, uint64_t cs, bool icols) { return icols ? Strides{rs, cs} : Strides{cs, rs}; }

// Tile loop of the element-wise kernels: `o` the outer index, `jb` this
// thread's first inner index (the others follow at kEwThreads apart).
#define HME_EW_TILES(E)                                                \
    for (uint64_t t_ = blockIdx.x; t_ < (E).ntiles; t_ += gridDim.x) { \
        const uint32_t o = static_cast<uint32_t>(t_ / (E).tpr);        \
        const uint32_t jb = static_cast<uint32_t>(t_ - static_cast<uint64_t>(o) * (E).tpr) * kEwTile + threadIdx.x;

__device__ __forceinline__ uint32_t apply_op(uint32_t old, uint32_t v, int op, uint32_t p) {
    return op == HME_SET ? v : op == HME_ADD ? mod_add(old, v, p) : mod_sub(old, v, p);
}

// (hi * 2^64 + lo) mod p for a small carry count hi; r64 = 2^64 mod p
__device__ __forceinline__ uint32_t fold96(uint64_t lo, uint32_t hi, uint32_t p, uint64_t barrett, uint32_t r64) {
    const uint32_t a = reduce_u64(lo, p, barrett);
    return hi ? mod_add(a, reduce_u64(static_cast<uint64_t>(hi) * r64, p, barrett), p) : a;
}
__device__ __forceinline__ void mac96(uint64_t& lo, uint32_t& hi, uint32_t a, uint32_t b) {
    const uint64_t prod = static_cast<uint64_t>(a) * b;
    lo += prod;
    hi += lo < prod ? 1u : 0u;
}

__global__ void __launch_bounds__(kEwThreads) axpy_kernel(uint32_t alpha, const uint32_t* __restrict__ x, Strides xs,
                                                          uint32_t* __restrict__ y, Strides ys, Ew e, int subtract,
                                                          uint32_t p, uint64_t barrett) {
    HME_EW_TILES(e)
    uint32_t xv[kEwU], yv[kEwU];
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t j = jb + u * kEwThreads;
        if (j < e.inner) {
            xv[u] = x[o * xs.so + j * xs.si];
            yv[u] = y[o * ys.so + j * ys.si];
        }
    }
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t j = jb + u * kEwThreads;
        if (j < e.inner) {
            const uint32_t ax = mod_mul(alpha, xv[u], p, barrett);
            y[o * ys.so + j * ys.si] = subtract ? mod_sub(yv[u], ax, p) : mod_add(yv[u], ax, p);
        }
    }
    }
}

// mode 0: x = alpha x;  1: x = alpha (a fill);  2: x = x >= p ? x - p : x
__global__ void __launch_bounds__(kEwThreads) unary_kernel(uint32_t* __restrict__ x, Strides xs, Ew e, int mode,
                                                           uint32_t alpha, uint32_t p, uint64_t barrett) {
    HME_EW_TILES(e)
    uint32_t v[kEwU];
    if (mode != 1) {
#pragma unroll
        for (int u = 0; u < kEwU; ++u) {
            const uint32_t j = jb + u * kEwThreads;
            if (j < e.inner) v[u] = x[o * xs.so + j * xs.si];
        }
    }
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t j = jb + u * kEwThreads;
        if (j < e.inner) {
            const uint32_t r = mode == 0   ? mod_mul(alpha, v[u], p, barrett)
                               : mode == 1 ? alpha
                                           : (v[u] >= p ? v[u] - p : v[u]);
            x[o * xs.so + j * xs.si] = r;
        }
    }
    }
}

__global__ void __launch_bounds__(kEwThreads) copy_kernel(const uint32_t* __restrict__ s, Strides ss,
                                                          uint32_t* __restrict__ d, Strides ds, Ew e) {
    HME_EW_TILES(e)
    uint32_t v[kEwU];
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t j = jb + u * kEwThreads;
        if (j < e.inner) v[u] = s[o * ss.so + j * ss.si];
    }
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t j = jb + u * kEwThreads;
        if (j < e.inner) d[o * ds.so + j * ds.si] = v[u];
    }
    }
}

// dst = acc mod p for 64-bit accumulators
__global__ void __launch_bounds__(kEwThreads) canon64_kernel(const uint64_t* __restrict__ a, Strides as,
                                                             uint32_t* __restrict__ d, Strides ds, Ew e, uint32_t p,
                                                             uint64_t barrett) {
    HME_EW_TILES(e)
    uint64_t v[kEwU];
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t j = jb + u * kEwThreads;
        if (j < e.inner) v[u] = a[o * as.so + j * as.si];
    }
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t j = jb + u * kEwThreads;
        if (j < e.inner) d[o * ds.so + j * ds.si] = reduce_u64(v[u], p, barrett);
    }
    }
}

__global__ void axpy_identity_kernel(uint32_t alpha, uint32_t* __restrict__ y, uint64_t rs, uint64_t cs, uint32_t n,
                                     int subtract, uint32_t p) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t* yp = y + i * rs + i * cs;
        *yp = subtract ? mod_sub(*yp, alpha, p) : mod_add(*yp, alpha, p);
    }
}

// c(i, t) [+]= alpha [row_off + r(i) == col(t)] + beta a(r(i), col(t)),
// r(i) = rows ? rows[i] : i, col(t) = cols ? cols[t] : t; tiles over (i, t)
// with t inner
__global__ void __launch_bounds__(kEwThreads)
    gather_kernel(uint32_t alpha, uint32_t beta, const uint32_t* __restrict__ a, uint64_t a_rs, uint64_t a_cs,
                  uint32_t row_off, const uint32_t* __restrict__ cols, const uint32_t* __restrict__ rows,
                  uint32_t* __restrict__ c, uint64_t c_rs, uint64_t c_cs, Ew e, int accumulate, uint32_t p,
                  uint64_t barrett) {
    HME_EW_TILES(e)
    const uint32_t ar = rows ? rows[o] : o;
    uint32_t av[kEwU], cv[kEwU], col[kEwU];
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t t = jb + u * kEwThreads;
        if (t < e.inner) {
            col[u] = cols ? cols[t] : t;
            av[u] = a ? a[ar * a_rs + col[u] * a_cs] : 0u;
            cv[u] = accumulate ? c[o * c_rs + t * c_cs] : 0u;
        }
    }
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t t = jb + u * kEwThreads;
        if (t < e.inner) {
            uint32_t v = a ? mod_mul(beta, av[u], p, barrett) : 0u;
            if (alpha != 0 && row_off + ar == col[u]) v = mod_add(v, alpha, p);
            c[o * c_rs + t * c_cs] = accumulate ? mod_add(cv[u], v, p) : v;
        }
    }
    }
}

// dst(i, j) = src(j, i), 32 x 32 tiles through shared memory
__global__ void transpose_kernel(const uint32_t* __restrict__ src, uint64_t s_rs, uint64_t s_cs,
                                 uint32_t* __restrict__ dst, uint64_t d_rs, uint64_t d_cs, uint32_t rows_dst,
                                 uint32_t cols_dst) {
    __shared__ uint32_t tile[32][33];
    for (uint32_t ty = blockIdx.y; ty * 32 < rows_dst; ty += gridDim.y)
        for (uint32_t tx = blockIdx.x; tx * 32 < cols_dst; tx += gridDim.x) {
            const uint32_t i0 = ty * 32, j0 = tx * 32;  // dst tile
            __syncthreads();
#pragma unroll
            for (uint32_t r = threadIdx.y; r < 32; r += 8) {
                const uint32_t jj = j0 + r, ii = i0 + threadIdx.x;  // src row jj, column ii
                if (jj < cols_dst && ii < rows_dst) tile[r][threadIdx.x] = src[jj * s_rs + ii * s_cs];
            }
            __syncthreads();
#pragma unroll
            for (uint32_t r = threadIdx.y; r < 32; r += 8) {
                const uint32_t ii = i0 + r, jj = j0 + threadIdx.x;
                if (ii < rows_dst && jj < cols_dst) dst[ii * d_rs + jj * d_cs] = tile[threadIdx.x][r];
            }
        }
}

// y op= A x, one warp per row (A's rows contiguous): four loads in flight per
// lane, the products summed exactly (96 bits), one reduction per lane
__global__ void gemv_warp_kernel(const uint32_t* __restrict__ A, uint64_t a_rs, uint64_t a_cs,
                                 const uint32_t* __restrict__ x, uint64_t x_rs, uint32_t* __restrict__ y,
                                 uint64_t y_rs, uint32_t m, uint32_t k, int op, uint32_t p, uint64_t barrett,
                                 uint32_t r64) {
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < m; row += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t* a = A + row * a_rs;
        uint64_t lo = 0;
        uint32_t hi = 0;
        for (uint32_t kk = lane; kk < k; kk += 128) {
            uint32_t av[4], xv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t j = kk + 32 * u;
                av[u] = j < k ? a[j * a_cs] : 0u;
                xv[u] = j < k ? x[j * x_rs] : 0u;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) mac96(lo, hi, av[u], xv[u]);
        }
        uint32_t v = fold96(lo, hi, p, barrett, r64);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = mod_add(v, __shfl_xor_sync(0xffffffffu, v, off), p);
        if (lane == 0) y[row * y_rs] = apply_op(y[row * y_rs], v, op, p);
    }
}
// one thread per row (A's columns contiguous: consecutive rows, consecutive addresses)
__global__ void gemv_thread_kernel(const uint32_t* __restrict__ A, uint64_t a_rs, uint64_t a_cs,
                                   const uint32_t* __restrict__ x, uint64_t x_rs, uint32_t* __restrict__ y,
                                   uint64_t y_rs, uint32_t m, uint32_t k, int op, uint32_t p, uint64_t barrett,
                                   uint32_t r64) {
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < m; row += gridDim.x * blockDim.x) {
        uint64_t lo = 0;
        uint32_t hi = 0;
        for (uint32_t kk = 0; kk < k; kk += 4) {
            uint32_t av[4], xv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                av[u] = kk + u < k ? A[row * a_rs + (kk + u) * a_cs] : 0u;
                xv[u] = kk + u < k ? x[(kk + u) * x_rs] : 0u;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) mac96(lo, hi, av[u], xv[u]);
        }
        y[row * y_rs] = apply_op(y[row * y_rs], fold96(lo, hi, p, barrett, r64), op, p);
    }
}

// One diagonal block of a unit-triangular solve: rows [i0, i0 + nb) of B
// (nb <= 128) become T_bb^-1 B_b.  A CTA takes 32 right-hand-side columns at a
// time.  The strict triangle of T_bb (pitch tp, odd) and the nb x 32 tile of
// B sit in shared memory.  Per 32-row sub-block, in solve order: each warp
// substitutes four columns at once (lane l holds row l of the sub-block; at
// step t row t is final and a shuffle broadcasts it), then all threads apply
// the solved sub-block to the rows still to solve within the block (exact
// 96-bit dot products of at most 32 terms).  LOWER walks down, upper walks up.
template <bool LOWER>
__global__ void __launch_bounds__(256) trsm_diag_kernel(const uint32_t* __restrict__ T, size_t ldt,
                                                        uint32_t* __restrict__ B, size_t ldb, uint32_t i0,
                                                        uint32_t nb, uint32_t n, uint32_t p, uint64_t barrett,
                                                        uint32_t r64) {
    extern __shared__ uint32_t sm[];
    const uint32_t tp = nb | 1u;
    uint32_t* sT = sm;            // nb x tp
    uint32_t* sB = sm + nb * tp;  // nb x 33
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
        const uint32_t r = idx / nb, s = idx - r * nb;
        const bool keep = LOWER ? s < r : s > r;
        sT[r * tp + s] = keep ? T[(i0 + r) * ldt + (i0 + s)] : 0u;
    }
    const uint32_t nsub = (nb + 31) / 32;
    for (uint32_t c0 = blockIdx.x * 32; c0 < n; c0 += gridDim.x * 32) {
        __syncthreads();
        for (uint32_t r = warp; r < nb; r += 8) sB[r * 33 + lane] = c0 + lane < n ? B[(i0 + r) * ldb + c0 + lane] : 0u;
        __syncthreads();
        for (uint32_t q = 0; q < nsub; ++q) {
            const uint32_t sb = LOWER ? q : nsub - 1 - q;
            const uint32_t r0 = sb * 32, rn = min(32u, nb - r0);
            uint32_t x[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) x[u] = lane < rn ? sB[(r0 + lane) * 33 + warp + 8 * u] : 0u;
            for (uint32_t st = 0; st + 1 < rn; ++st) {
                const uint32_t t = LOWER ? st : rn - 1 - st;
                const bool upd = LOWER ? (lane > t && lane < rn) : (lane < t);
                const uint32_t l = upd ? sT[(r0 + lane) * tp + r0 + t] : 0u;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const uint32_t xt = __shfl_sync(0xffffffffu, x[u], t);
                    if (l) x[u] = reduce_u64(static_cast<uint64_t>(p - l) * xt + x[u], p, barrett);
                }
            }
            if (lane < rn) {
#pragma unroll
                for (int u = 0; u < 4; ++u) sB[(r0 + lane) * 33 + warp + 8 * u] = x[u];
            }
            __syncthreads();
            const uint32_t u0 = LOWER ? r0 + rn : 0, u1 = LOWER ? nb : r0;
            for (uint32_t idx = threadIdx.x; idx < (u1 - u0) * 32; idx += blockDim.x) {
                const uint32_t r = u0 + (idx >> 5), c = idx & 31;
                uint64_t lo = 0;
                uint32_t hi = 0;
                for (uint32_t s = 0; s < rn; ++s) mac96(lo, hi, sT[r * tp + r0 + s], sB[(r0 + s) * 33 + c]);
                sB[r * 33 + c] = mod_sub(sB[r * 33 + c], fold96(lo, hi, p, barrett, r64), p);
            }
            __syncthreads();
        }
        for (uint32_t r = warp; r < nb; r += 8)
            if (c0 + lane < n) B[(i0 + r) * ldb + c0 + lane] = sB[r * 33 + lane];
    }
}

size_t trsm_smem_bytes(uint32_t nb) { return 4ull * (nb * (nb | 1u) + nb * 33u); }

int ew_grid(uint64_t ntiles, int sms) {
    return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(ntiles, static_cast<uint64_t>(sms) * 8)));
}

uint32_t r64_of(uint32_t p) { return static_cast<uint32_t>((static_cast<unsigned __int128>(1) << 64) % p); }

// [lo, hi) byte range of a rows x cols view of `esz`-byte elements
void span_of(const void* base, uint32_t rows, uint32_t cols, uint64_t rs, uint64_t cs, size_t esz, uintptr_t& lo,
             uintptr_t& hi) {
    lo = reinterpret_cast<uintptr_t>(base);
    hi = lo + esz * ((rows ? (rows - 1) * rs : 0) + (cols ? (cols - 1) * cs : 0) + 1);
}
bool overlap(const void* a, uint32_t ar, uint32_t ac, uint64_t ars, uint64_t acs, const void* b, uint32_t br,
             uint32_t bc, uint64_t brs, uint64_t bcs, size_t aesz = 4) {
    if (!ar || !ac || !br || !bc) return false;
    uintptr_t a0, a1, b0, b1;
    span_of(a, ar, ac, ars, acs, aesz, a0, a1);
    span_of(b, br, bc, brs, bcs, 4, b0, b1);
    return a0 < b1 && b0 < a1;
}

void launch_unary(hme_ctx* ctx, const char* name, uint32_t* x, uint32_t rows, uint32_t cols, uint64_t rs, uint64_t cs,
                  int mode, uint32_t alpha, uint32_t p) {
    const bool ic = inner_is_cols(rows, cols, rs, cs);
    const Ew e = make_ew(rows, cols, ic);
    const uint64_t barrett = p >= 2 ? make_mod(p).barrett : 0;
    HME_TIMED(ctx, name, unary_kernel<<<ew_grid(e.ntiles, ctx->num_sms), kEwThreads, 0, ctx->stream>>>(
                             x, strides_of(rs, cs, ic), e, mode, alpha, p, barrett));
    HME_CUDA(cudaGetLastError());
}

}  // namespace
}  // namespace hme

using namespace hme;

extern "C" {

int hme_gemv_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t k, const uint32_t* A, size_t a_rs, size_t a_cs,
                     const uint32_t* x, size_t x_rs, uint32_t* y, size_t y_rs, int op) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2, "gemv: bad context or modulus");
        HME_REQUIRE(op == HME_SET || op == HME_ADD || op == HME_SUB, "gemv: bad op");
        if (m == 0) return;
        HME_REQUIRE(y && (k == 0 || (A && x)), "gemv: null pointer");
        HME_REQUIRE(!overlap(y, m, 1, y_rs, 1, A, m, k, a_rs, a_cs) && !overlap(y, m, 1, y_rs, 1, x, k, 1, x_rs, 1),
                    "gemv: y aliases an operand");
        bind(ctx);
        const ModParams mp = make_mod(p);
        if (a_cs == 1 || a_rs != 1) {
            const int grid = static_cast<int>(std::min<size_t>((static_cast<size_t>(m) + 7) / 8, ctx->num_sms * 16));
            HME_TIMED(ctx, "gemv", gemv_warp_kernel<<<grid, 256, 0, ctx->stream>>>(A, a_rs, a_cs, x, x_rs, y, y_rs, m,
                                                                                 k, op, p, mp.barrett, r64_of(p)));
        } else {
            const int grid = static_cast<int>(std::min<size_t>((static_cast<size_t>(m) + 255) / 256, ctx->num_sms * 8));
            HME_TIMED(ctx, "gemv", gemv_thread_kernel<<<grid, 256, 0, ctx->stream>>>(
                                       A, a_rs, a_cs, x, x_rs, y, y_rs, m, k, op, p, mp.barrett, r64_of(p)));
        }
        HME_CUDA(cudaGetLastError());
    });
}

int hme_axpy_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t alpha, uint32_t rows, uint32_t cols, const uint32_t* x,
                     size_t x_rs, size_t x_cs, uint32_t* y, size_t y_rs, size_t y_cs, int subtract) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2 && alpha < p, "axpy: bad context, modulus or alpha (must be canonical)");
        if (!rows || !cols) return;
        HME_REQUIRE(x && y, "axpy: null pointer");
        bind(ctx);
        const bool ic = inner_is_cols(rows, cols, x_rs, x_cs);
        const Ew e = make_ew(rows, cols, ic);
        HME_TIMED(ctx, "axpy", axpy_kernel<<<ew_grid(e.ntiles, ctx->num_sms), kEwThreads, 0, ctx->stream>>>(
                                   alpha, x, strides_of(x_rs, x_cs, ic), y, strides_of(y_rs, y_cs, ic), e,
                                   subtract ? 1 : 0, p, make_mod(p).barrett));
        HME_CUDA(cudaGetLastError());
    });
}

int hme_scal_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t alpha, uint32_t rows, uint32_t cols, uint32_t* x, size_t rs,
                     size_t cs) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2 && alpha < p, "scal: bad context, modulus or alpha (must be canonical)");
        if (!rows || !cols) return;
        HME_REQUIRE(x, "scal: null pointer");
        bind(ctx);
        launch_unary(ctx, "scal", x, rows, cols, rs, cs, 0, alpha, p);
    });
}

int hme_fill_u32_dev(hme_ctx* ctx, uint32_t rows, uint32_t cols, uint32_t* x, size_t rs, size_t cs, uint32_t value) {
    return guard([&] {
        HME_REQUIRE(ctx, "fill: null context");
        if (!rows || !cols) return;
        HME_REQUIRE(x, "fill: null pointer");
        bind(ctx);
        launch_unary(ctx, "fill", x, rows, cols, rs, cs, 1, value, 0);
    });
}

int hme_canonicalise_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t rows, uint32_t cols, uint32_t* v, size_t rs,
                             size_t cs) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2 && p <= 0x80000000u, "canonicalise: bad context or modulus (2p must fit 32 bits)");
        if (!rows || !cols) return;
        HME_REQUIRE(v, "canonicalise: null pointer");
        bind(ctx);
        launch_unary(ctx, "canonicalise", v, rows, cols, rs, cs, 2, 0, p);
    });
}

int hme_copy_u32_dev(hme_ctx* ctx, uint32_t rows, uint32_t cols, const uint32_t* src, size_t s_rs, size_t s_cs,
                     uint32_t* dst, size_t d_rs, size_t d_cs) {
    return guard([&] {
        HME_REQUIRE(ctx, "copy: null context");
        if (!rows || !cols) return;
        HME_REQUIRE(src && dst, "copy: null pointer");
        if (src == dst && s_rs == d_rs && s_cs == d_cs) return;
        HME_REQUIRE(!overlap(src, rows, cols, s_rs, s_cs, dst, rows, cols, d_rs, d_cs), "copy: overlapping windows");
        bind(ctx);
        const bool ic = inner_is_cols(rows, cols, s_rs, s_cs);
        const Ew e = make_ew(rows, cols, ic);
        HME_TIMED(ctx, "copy", copy_kernel<<<ew_grid(e.ntiles, ctx->num_sms), kEwThreads, 0, ctx->stream>>>(
                                   src, strides_of(s_rs, s_cs, ic), dst, strides_of(d_rs, d_cs, ic), e));
        HME_CUDA(cudaGetLastError());
    });
}

int hme_canonicalise_acc64_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t rows, uint32_t cols, const uint64_t* acc,
                                   size_t a_rs, size_t a_cs, uint32_t* dst, size_t d_rs, size_t d_cs) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2, "canonicalise: bad context or modulus");
        if (!rows || !cols) return;
        HME_REQUIRE(acc && dst, "canonicalise: null pointer");
        HME_REQUIRE(!overlap(acc, rows, cols, a_rs, a_cs, dst, rows, cols, d_rs, d_cs, 8),
                    "canonicalise: overlapping windows");
        bind(ctx);
        const bool ic = inner_is_cols(rows, cols, a_rs, a_cs);
        const Ew e = make_ew(rows, cols, ic);
        HME_TIMED(ctx, "canonicalise", canon64_kernel<<<ew_grid(e.ntiles, ctx->num_sms), kEwThreads, 0, ctx->stream>>>(
                                           acc, strides_of(a_rs, a_cs, ic), dst, strides_of(d_rs, d_cs, ic), e, p,
                                           make_mod(p).barrett));
        HME_CUDA(cudaGetLastError());
    });
}

int hme_transpose_u32_dev(hme_ctx* ctx, uint32_t rows_dst, uint32_t cols_dst, const uint32_t* src, size_t s_rs,
                          size_t s_cs, uint32_t* dst, size_t d_rs, size_t d_cs) {
    return guard([&] {
        HME_REQUIRE(ctx, "transpose: null context");
        if (!rows_dst || !cols_dst) return;
        HME_REQUIRE(src && dst, "transpose: null pointer");
        HME_REQUIRE(!overlap(src, cols_dst, rows_dst, s_rs, s_cs, dst, rows_dst, cols_dst, d_rs, d_cs),
                    "transpose: overlapping windows");
        bind(ctx);
        const dim3 grid(std::min<uint32_t>((cols_dst + 31) / 32, 1024), std::min<uint32_t>((rows_dst + 31) / 32, 1024));
        HME_TIMED(ctx, "transpose", transpose_kernel<<<grid, dim3(32, 8), 0, ctx->stream>>>(src, s_rs, s_cs, dst, d_rs,
                                                                                          d_cs, rows_dst, cols_dst));
        HME_CUDA(cudaGetLastError());
    });
}

int hme_axpy_identity_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t alpha, uint32_t rows, uint32_t cols, uint32_t* y,
                              size_t rs, size_t cs, int subtract) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2 && alpha < p, "axpy_identity: bad context, modulus or alpha (must be canonical)");
        const uint32_t n = std::min(rows, cols);
        if (!n) return;
        HME_REQUIRE(y, "axpy_identity: null pointer");
        bind(ctx);
        const int grid = static_cast<int>(std::min<uint32_t>((n + 255) / 256, ctx->num_sms * 8));
        HME_TIMED(ctx, "axpy_identity", axpy_identity_kernel<<<grid, 256, 0, ctx->stream>>>(alpha, y, rs, cs, n,
                                                                                           subtract ? 1 : 0, p));
        HME_CUDA(cudaGetLastError());
    });
}

int hme_gather_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t alpha, uint32_t beta, const uint32_t* a, uint32_t a_rows,
                       uint32_t a_cols, size_t a_rs, size_t a_cs, uint32_t row_off, const uint32_t* cols,
                       const uint32_t* rows, uint32_t c_rows, uint32_t c_cols, uint32_t* c, size_t c_rs, size_t c_cs,
                       int accumulate) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2 && alpha < p && beta < p, "gather: bad context, modulus or coefficients");
        if (!c_rows || !c_cols) return;
        HME_REQUIRE(c, "gather: null output");
        const bool has_a = a != nullptr && beta != 0;
        if (has_a) {
            HME_REQUIRE(rows != nullptr || a_rows == c_rows, "gather: row count mismatch");
            HME_REQUIRE(cols != nullptr || a_cols == c_cols, "gather: column count mismatch");
            HME_REQUIRE(!overlap(a, a_rows, a_cols, a_rs, a_cs, c, c_rows, c_cols, c_rs, c_cs),
                        "gather: output aliases the source");
        }
        bind(ctx);
        const Ew e = make_ew(c_rows, c_cols, true);
        HME_TIMED(ctx, "gather", gather_kernel<<<ew_grid(e.ntiles, ctx->num_sms), kEwThreads, 0, ctx->stream>>>(
                                     alpha, has_a ? beta : 0u, has_a ? a : nullptr, a_rs, a_cs, row_off, cols, rows, c,
                                     c_rs, c_cs, e, accumulate ? 1 : 0, p, make_mod(p).barrett));
        HME_CUDA(cudaGetLastError());
    });
}

int hme_trsm_unit_u32_dev(hme_ctx* ctx, uint32_t p, int lower, uint32_t m, uint32_t n, const uint32_t* T, size_t ldt,
                          uint32_t* B, size_t ldb) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2, "trsm_unit: bad context or modulus");
        if (!m || !n) return;
        HME_REQUIRE(T && B && ldt >= m && ldb >= n, "trsm_unit: bad buffers");
        HME_REQUIRE(!overlap(T, m, m, ldt, 1, B, m, n, ldb, 1), "trsm_unit: T aliases B");
        bind(ctx);
        const ModParams mp = make_mod(p);
        const uint32_t r64 = r64_of(p);
        // a 128-row block takes 84 KB of shared memory (set on the calling device)
        HME_CUDA(cudaFuncSetAttribute(lower ? trsm_diag_kernel<true> : trsm_diag_kernel<false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(trsm_smem_bytes(kTrsmNB))));
        const uint32_t nblocks = (m + kTrsmNB - 1) / kTrsmNB;
        const int grid = static_cast<int>(std::min<uint32_t>((n + 31) / 32, ctx->num_sms * 2));
        for (uint32_t bi = 0; bi < nblocks; ++bi) {
            const uint32_t i0 = lower ? bi * kTrsmNB : (nblocks - 1 - bi) * kTrsmNB;
            const uint32_t nb = std::min(kTrsmNB, m - i0);
            const size_t smem = trsm_smem_bytes(nb);
            if (lower)
                HME_TIMED(ctx, "trsm_diag", trsm_diag_kernel<true><<<grid, 256, smem, ctx->stream>>>(
                                                T, ldt, B, ldb, i0, nb, n, p, mp.barrett, r64));
            else
                HME_TIMED(ctx, "trsm_diag", trsm_diag_kernel<false><<<grid, 256, smem, ctx->stream>>>(
                                                T, ldt, B, ldb, i0, nb, n, p, mp.barrett, r64));
            HME_CUDA(cudaGetLastError());
            // the solved block applied to the rows still to solve (limb GEMM, Sub)
            if (lower && i0 + nb < m)
                gemm_u32_device(ctx, mp, m - i0 - nb, n, nb, T + static_cast<size_t>(i0 + nb) * ldt + i0, ldt,
                                B + static_cast<size_t>(i0) * ldb, ldb, B + static_cast<size_t>(i0 + nb) * ldb, ldb,
                                HME_SUB);
            if (!lower && i0 > 0)
                gemm_u32_device(ctx, mp, i0, n, nb, T + i0, ldt, B + static_cast<size_t>(i0) * ldb, ldb, B, ldb,
                                HME_SUB);
        }
    });
}

int hme_gemm_nt_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A, size_t lda,
                        const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc, int op) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2, "gemm_nt: bad context or modulus");
        if (!m || !n) return;
        HME_REQUIRE(k == 0 || (A && B && lda >= k && ldb >= k), "gemm_nt: bad A / B");
        bind(ctx);
        // B (n x k, row-major) -> B^T (k x n) in workspace, then the limb GEMM
        uint32_t* Bt = nullptr;
        if (k > 0) {
            Bt = static_cast<uint32_t*>(ctx->ws.get(kSlotStageB, sizeof(uint32_t) * static_cast<size_t>(k) * n));
            const dim3 grid(std::min<uint32_t>((n + 31) / 32, 1024), std::min<uint32_t>((k + 31) / 32, 1024));
            HME_TIMED(ctx, "transpose",
                      transpose_kernel<<<grid, dim3(32, 8), 0, ctx->stream>>>(B, ldb, 1, Bt, n, 1, k, n));
            HME_CUDA(cudaGetLastError());
        }
        gemm_u32_device(ctx, make_mod(p), m, n, k, A, lda, Bt, n, C, ldc, op);
    });
}

int hme_schur_update_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t* L,
                             size_t ldl, const uint32_t* U, size_t ldu, uint32_t* C, size_t ldc) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2, "schur_update: bad context or modulus");
        bind(ctx);
        gemm_u32_device(ctx, make_mod(p), m, n, k, L, ldl, U, ldu, C, ldc, HME_SUB);
    });
}

}  // extern "C"

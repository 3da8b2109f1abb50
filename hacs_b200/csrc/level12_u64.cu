// The level-1 device operations over u64 residues (any modulus 2 <= p < 2^64),
// on strided device views: axpy, scal, copy, transpose, fill, identity axpy,
// gather and the lazy-form canonicalisation.  They complete the u64 element
// type of the engine's device layer (engine::cuda::* instantiated for
// uint64_t, src/Cuda/CudaKernels.h:186-234; the u64 GEMM is gemm_u64.cu).
//
// Arithmetic: a product of two residues is formed exactly in 128 bits and
// reduced mod p once (a 128-by-64 remainder), sums use the carry of the 64-bit
// add, so every result is the exact canonical residue.  Layout: one thread per
// element with consecutive threads on the unit-stride dimension when there is
// one, grid-stride loops; the transpose moves 32 x 32 tiles through shared
// memory.  These operations are far from the engine's hot path (the u64
// regime of the tape), so they favour plain, obviously exact code.
#include <cuda_runtime.h>

#include <algorithm>

#include "hme_internal.h"

namespace hme {
namespace {

__device__ __forceinline__ uint64_t add64(uint64_t a, uint64_t b, uint64_t p) {
    const uint64_t s = a + b;
    return (s < a || s >= p) ? s - p : s;  // a, b < p: the true sum is below 2p
}
__device__ __forceinline__ uint64_t sub64(uint64_t a, uint64_t b, uint64_t p) { return a >= b ? a - b : a + (p - b); }
__device__ __forceinline__ uint64_t mul64(uint64_t a, uint64_t b, uint64_t p) {
    const unsigned __int128 t = static_cast<unsigned __int128>(a) * b;
    return static_cast<uint64_t>(t % p);
}

// Element (i, j) of a window: i over rows, j over columns; the launch's x
// dimension walks the unit-stride dimension of the first operand.
struct Win {
    uint64_t* base;
    uint64_t rs, cs;
};
struct CWin {
    const uint64_t* base;
    uint64_t rs, cs;
};

// flat index t -> (i, j) with the fast index on columns (cols_fast) or rows
__device__ __forceinline__ void ij_of(uint64_t t, uint32_t rows, uint32_t cols, bool cols_fast, uint32_t& i,
                                      uint32_t& j) {
    if (cols_fast) {
        i = static_cast<uint32_t>(t / cols);
        j = static_cast<uint32_t>(t - static_cast<uint64_t>(i) * cols);
    } else {
        j = static_cast<uint32_t>(t / rows);
        i = static_cast<uint32_t>(t - static_cast<uint64_t>(j) * rows);
    }
}

enum Op64 : int { kAxpy = 0, kAxpySub, kScal, kCopy, kFill, kCanon };

__global__ void ew64_kernel(int op, uint32_t rows, uint32_t cols, bool cols_fast, CWin x, Win y, uint64_t p,
                            uint64_t alpha) {
    const uint64_t total = static_cast<uint64_t>(rows) * cols;
    for (uint64_t t = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint32_t i, j;
        ij_of(t, rows, cols, cols_fast, i, j);
        uint64_t* yp = y.base + i * y.rs + j * y.cs;
        switch (op) {
            case kAxpy: *yp = add64(*yp, mul64(alpha, x.base[i * x.rs + j * x.cs], p), p); break;
            case kAxpySub: *yp = sub64(*yp, mul64(alpha, x.base[i * x.rs + j * x.cs], p), p); break;
            case kScal: *yp = mul64(alpha, *yp, p); break;
            case kCopy: *yp = x.base[i * x.rs + j * x.cs]; break;
            case kFill: *yp = alpha; break;
            default: {
                const uint64_t v = *yp;
                *yp = v >= p ? v - p : v;
            }
        }
    }
}

// dst (rows x cols) = src^T, src cols x rows; 32 x 32 tiles through shared memory
__global__ void transpose64_kernel(uint32_t rows, uint32_t cols, CWin src, Win dst) {
    __shared__ uint64_t tile[32][33];
    const uint32_t tiles_c = (cols + 31) / 32, tiles_r = (rows + 31) / 32;
    for (uint64_t tb = blockIdx.x; tb < static_cast<uint64_t>(tiles_c) * tiles_r; tb += gridDim.x) {
        const uint32_t ti = static_cast<uint32_t>(tb / tiles_c), tj = static_cast<uint32_t>(tb % tiles_c);
        const uint32_t i0 = ti * 32, j0 = tj * 32;
        // read src rows j0.. (dst columns), src columns i0.. (dst rows)
        for (uint32_t r = threadIdx.y; r < 32; r += blockDim.y) {
            const uint32_t sj = j0 + r, si = i0 + threadIdx.x;
            if (sj < cols && si < rows) tile[r][threadIdx.x] = src.base[sj * src.rs + si * src.cs];
        }
        __syncthreads();
        for (uint32_t r = threadIdx.y; r < 32; r += blockDim.y) {
            const uint32_t di = i0 + r, dj = j0 + threadIdx.x;
            if (di < rows && dj < cols) dst.base[di * dst.rs + dj * dst.cs] = tile[threadIdx.x][r];
        }
        __syncthreads();
    }
}

__global__ void axpy_identity64_kernel(uint32_t n, Win y, uint64_t p, uint64_t alpha, bool subtract) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint64_t* yp = y.base + i * y.rs + i * y.cs;
        *yp = subtract ? sub64(*yp, alpha, p) : add64(*yp, alpha, p);
    }
}

// c(i, t) [+]= alpha [row_off + r(i) == col(t)] + beta a(r(i), col(t))
__global__ void gather64_kernel(uint32_t rows, uint32_t cols, CWin a, bool have_a, uint32_t row_off,
                                const uint32_t* colv, const uint32_t* rowv, Win c, uint64_t p, uint64_t alpha,
                                uint64_t beta, bool accumulate) {
    const uint64_t total = static_cast<uint64_t>(rows) * cols;
    for (uint64_t t = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t i = static_cast<uint32_t>(t / cols), tt = static_cast<uint32_t>(t % cols);
        const uint32_t ri = rowv ? rowv[i] : i, ct = colv ? colv[tt] : tt;
        uint64_t v = (row_off + ri == ct) ? alpha : 0;
        if (have_a) v = add64(v, mul64(beta, a.base[ri * a.rs + ct * a.cs], p), p);
        uint64_t* cp = c.base + i * c.rs + tt * c.cs;
        *cp = accumulate ? add64(*cp, v, p) : v;
    }
}

int ew_grid(hme_ctx* ctx, uint64_t total) {
    return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((total + 255) / 256,
                                                                     static_cast<uint64_t>(ctx->num_sms) * 16)));
}
bool cols_fast_of(uint64_t rs, uint64_t cs) { return !(rs == 1 && cs != 1); }

void run_ew(hme_ctx* ctx, int op, uint32_t rows, uint32_t cols, const uint64_t* x, uint64_t x_rs, uint64_t x_cs,
            uint64_t* y, uint64_t y_rs, uint64_t y_cs, uint64_t p, uint64_t alpha, const char* name) {
    if (!rows || !cols) return;
    const uint64_t total = static_cast<uint64_t>(rows) * cols;
    HME_TIMED(ctx, name,
              ew64_kernel<<<ew_grid(ctx, total), 256, 0, ctx->stream>>>(op, rows, cols, cols_fast_of(y_rs, y_cs),
                                                                        CWin{x, x_rs, x_cs}, Win{y, y_rs, y_cs}, p,
                                                                        alpha));
    HME_CUDA(cudaGetLastError());
}

// the byte range [lo, hi) a window spans
void span(const void* b, uint32_t rows, uint32_t cols, uint64_t rs, uint64_t cs, uintptr_t& lo, uintptr_t& hi) {
    lo = reinterpret_cast<uintptr_t>(b);
    hi = lo + ((rows - 1) * rs + (cols - 1) * cs + 1) * sizeof(uint64_t);
}
bool may_overlap(const void* a, uint32_t ar, uint32_t ac, uint64_t ars, uint64_t acs, const void* b, uint32_t br,
                 uint32_t bc, uint64_t brs, uint64_t bcs) {
    if (!ar || !ac || !br || !bc) return false;
    uintptr_t a0, a1, b0, b1;
    span(a, ar, ac, ars, acs, a0, a1);
    span(b, br, bc, brs, bcs, b0, b1);
    return !(a1 <= b0 || b1 <= a0);
}

}  // namespace
}  // namespace hme

using namespace hme;

extern "C" {

int hme_axpy_u64_dev(hme_ctx* ctx, uint64_t p, uint64_t alpha, uint32_t rows, uint32_t cols, const uint64_t* x,
                     size_t x_rs, size_t x_cs, uint64_t* y, size_t y_rs, size_t y_cs, int subtract) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2 && alpha < p, "axpy_u64: bad context, modulus or alpha (alpha must be canonical)");
        if (!rows || !cols) return;
        HME_REQUIRE(x && y, "axpy_u64: null view");
        HME_REQUIRE(!may_overlap(x, rows, cols, x_rs, x_cs, y, rows, cols, y_rs, y_cs) || x == y,
                    "axpy_u64: x and y overlap");
        bind(ctx);
        run_ew(ctx, subtract ? kAxpySub : kAxpy, rows, cols, x, x_rs, x_cs, y, y_rs, y_cs, p, alpha, "axpy64");
    });
}

int hme_scal_u64_dev(hme_ctx* ctx, uint64_t p, uint64_t alpha, uint32_t rows, uint32_t cols, uint64_t* x, size_t rs,
                     size_t cs) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2 && alpha < p, "scal_u64: bad context, modulus or alpha");
        if (!rows || !cols) return;
        HME_REQUIRE(x, "scal_u64: null view");
        bind(ctx);
        run_ew(ctx, kScal, rows, cols, nullptr, 0, 0, x, rs, cs, p, alpha, "scal64");
    });
}

int hme_copy_u64_dev(hme_ctx* ctx, uint32_t rows, uint32_t cols, const uint64_t* src, size_t s_rs, size_t s_cs,
                     uint64_t* dst, size_t d_rs, size_t d_cs) {
    return guard([&] {
        HME_REQUIRE(ctx, "copy_u64: null context");
        if (!rows || !cols) return;
        HME_REQUIRE(src && dst, "copy_u64: null view");
        HME_REQUIRE(!may_overlap(src, rows, cols, s_rs, s_cs, dst, rows, cols, d_rs, d_cs),
                    "copy_u64: the windows overlap");
        bind(ctx);
        run_ew(ctx, kCopy, rows, cols, src, s_rs, s_cs, dst, d_rs, d_cs, 0, 0, "copy64");
    });
}

int hme_transpose_u64_dev(hme_ctx* ctx, uint32_t rows_dst, uint32_t cols_dst, const uint64_t* src, size_t s_rs,
                          size_t s_cs, uint64_t* dst, size_t d_rs, size_t d_cs) {
    return guard([&] {
        HME_REQUIRE(ctx, "transpose_u64: null context");
        if (!rows_dst || !cols_dst) return;
        HME_REQUIRE(src && dst, "transpose_u64: null view");
        HME_REQUIRE(!may_overlap(src, cols_dst, rows_dst, s_rs, s_cs, dst, rows_dst, cols_dst, d_rs, d_cs),
                    "transpose_u64: the windows overlap");
        bind(ctx);
        const uint64_t tiles = static_cast<uint64_t>((rows_dst + 31) / 32) * ((cols_dst + 31) / 32);
        const int grid = static_cast<int>(std::min<uint64_t>(tiles, static_cast<uint64_t>(ctx->num_sms) * 8));
        HME_TIMED(ctx, "transpose64",
                  transpose64_kernel<<<grid, dim3(32, 8), 0, ctx->stream>>>(rows_dst, cols_dst, CWin{src, s_rs, s_cs},
                                                                             Win{dst, d_rs, d_cs}));
        HME_CUDA(cudaGetLastError());
    });
}

int hme_fill_u64_dev(hme_ctx* ctx, uint32_t rows, uint32_t cols, uint64_t* x, size_t rs, size_t cs, uint64_t value) {
    return guard([&] {
        HME_REQUIRE(ctx, "fill_u64: null context");
        if (!rows || !cols) return;
        HME_REQUIRE(x, "fill_u64: null view");
        bind(ctx);
        run_ew(ctx, kFill, rows, cols, nullptr, 0, 0, x, rs, cs, 0, value, "fill64");
    });
}

int hme_axpy_identity_u64_dev(hme_ctx* ctx, uint64_t p, uint64_t alpha, uint32_t rows, uint32_t cols, uint64_t* y,
                              size_t rs, size_t cs, int subtract) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2 && alpha < p, "axpy_identity_u64: bad context, modulus or alpha");
        const uint32_t n = std::min(rows, cols);
        if (!n) return;
        HME_REQUIRE(y, "axpy_identity_u64: null view");
        bind(ctx);
        HME_TIMED(ctx, "axpy_identity64",
                  axpy_identity64_kernel<<<std::max(1u, std::min<uint32_t>((n + 255) / 256, 1024)), 256, 0,
                                           ctx->stream>>>(n, Win{y, rs, cs}, p, alpha, subtract != 0));
        HME_CUDA(cudaGetLastError());
    });
}

int hme_gather_u64_dev(hme_ctx* ctx, uint64_t p, uint64_t alpha, uint64_t beta, const uint64_t* a, uint32_t a_rows,
                       uint32_t a_cols, size_t a_rs, size_t a_cs, uint32_t row_off, const uint32_t* cols,
                       const uint32_t* rows, uint32_t c_rows, uint32_t c_cols, uint64_t* c, size_t c_rs, size_t c_cs,
                       int accumulate) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2 && alpha < p && (!a || beta < p), "gather_u64: bad context, modulus or scalars");
        if (!c_rows || !c_cols) return;
        HME_REQUIRE(c, "gather_u64: null output view");
        HME_REQUIRE(!a || !may_overlap(a, a_rows, a_cols, a_rs, a_cs, c, c_rows, c_cols, c_rs, c_cs),
                    "gather_u64: a and c overlap");
        bind(ctx);
        const uint64_t total = static_cast<uint64_t>(c_rows) * c_cols;
        HME_TIMED(ctx, "gather64",
                  gather64_kernel<<<ew_grid(ctx, total), 256, 0, ctx->stream>>>(
                      c_rows, c_cols, CWin{a, a_rs, a_cs}, a != nullptr, row_off, cols, rows, Win{c, c_rs, c_cs}, p,
                      alpha, a ? beta : 0, accumulate != 0));
        HME_CUDA(cudaGetLastError());
    });
}

int hme_canonicalise_u64_dev(hme_ctx* ctx, uint64_t p, uint32_t rows, uint32_t cols, uint64_t* v, size_t rs,
                             size_t cs) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2 && p <= (uint64_t(1) << 63), "canonicalise_u64: the lazy form needs 2p <= 2^64");
        if (!rows || !cols) return;
        HME_REQUIRE(v, "canonicalise_u64: null view");
        bind(ctx);
        run_ew(ctx, kCanon, rows, cols, nullptr, 0, 0, v, rs, cs, p, 0, "canonicalise64");
    });
}

}  // extern "C"

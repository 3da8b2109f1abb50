// C ABI of the device elimination over F_p (include/hme.h): RREF, column rank
// profile, determinant, kernel basis, inverse, solve.  Host-pointer entry
// points copy in, run elim_device on the context's stream and copy out.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "hme_elim.h"
#include "hme_internal.h"

namespace hme {

bool is_prime_u32(uint32_t p) {
    if (p < 2) return false;
    for (uint32_t q : {2u, 3u, 5u, 7u, 11u, 13u, 17u, 19u, 23u, 29u, 31u, 37u})
        if (p % q == 0) return p == q;
    uint32_t d = p - 1;
    int s = 0;
    while ((d & 1) == 0) {
        d >>= 1;
        ++s;
    }
    auto powmod = [p](uint64_t b, uint32_t e) {
        uint64_t r = 1;
        b %= p;
        while (e) {
            if (e & 1) r = r * b % p;
            b = b * b % p;
            e >>= 1;
        }
        return r;
    };
    for (uint32_t a : {2u, 7u, 61u}) {
        if (a % p == 0) continue;
        uint64_t x = powmod(a, d);
        if (x == 1 || x == p - 1) continue;
        bool comp = true;
        for (int r = 1; r < s; ++r) {
            x = x * x % p;
            if (x == p - 1) {
                comp = false;
                break;
            }
        }
        if (comp) return false;
    }
    return true;
}

namespace {

void require_field(uint32_t p) {
    if (!is_prime_u32(p))
        throw Error(HME_EINVAL, "field-only entry point: p = " + std::to_string(p) +
                                    " is not prime (use the Z/ell^k Howell / Smith entry points)");
}

__global__ void kernel_basis_kernel(const uint32_t* __restrict__ R, uint64_t ldr, int n, int rank,
                                    const int* __restrict__ piv, const int* __restrict__ freec, int f, uint32_t p,
                                    uint32_t* __restrict__ K, uint64_t ldk) {
    // K (f x n): row t = free column freec[t]: 1 there, -R[i][freec[t]] at pivot column piv[i], 0 elsewhere.
    const size_t total = static_cast<size_t>(f) * n;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int t = static_cast<int>(idx / n), j = static_cast<int>(idx % n);
        K[static_cast<size_t>(t) * ldk + j] = (j == freec[t]) ? 1u % p : 0u;
    }
}
__global__ void kernel_basis_fill_kernel(const uint32_t* __restrict__ R, uint64_t ldr, int rank,
                                         const int* __restrict__ piv, const int* __restrict__ freec, int f,
                                         uint32_t p, uint32_t* __restrict__ K, uint64_t ldk) {
    const size_t total = static_cast<size_t>(f) * rank;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int t = static_cast<int>(idx / rank), i = static_cast<int>(idx % rank);
        const uint32_t v = R[static_cast<size_t>(i) * ldr + freec[t]];
        K[static_cast<size_t>(t) * ldk + piv[i]] = v == 0 ? 0u : p - v;
    }
}

ElimOptions& opts(hme_ctx* ctx) { return ctx->elim; }

// Working leading dimension of a device matrix with `cols` columns: a multiple
// of 4 (16-byte rows for vector access) that is not a power-of-two multiple of
// the row size, so the rows a warp touches together spread over the memory
// partitions instead of camping on one.
size_t padded_ld(size_t cols) { return (cols + 15) / 16 * 16 + 16; }

// Device copy of a host matrix (rows x cols, ld) into workspace slot `slot`,
// with the padded leading dimension padded_ld(cols).
uint32_t* upload(hme_ctx* ctx, int slot, const uint32_t* H, size_t ldh, uint32_t rows, uint32_t cols) {
    const size_t w = padded_ld(cols);
    uint32_t* d = static_cast<uint32_t*>(ctx->ws.get(slot, sizeof(uint32_t) * std::max<size_t>(1, rows * w)));
    if (rows && cols)
        HME_CUDA(cudaMemcpy2DAsync(d, sizeof(uint32_t) * w, H, sizeof(uint32_t) * ldh, sizeof(uint32_t) * cols, rows,
                                   cudaMemcpyHostToDevice, ctx->stream));
    return d;
}

uint32_t det_from(const ElimResult& r, uint32_t n, uint32_t p) {
    if (static_cast<uint32_t>(r.rank) < n) return 0;
    uint64_t d = 1 % p;
    for (uint32_t x : r.diag) d = d * x % p;
    if (r.sign_negative && d != 0) d = p - d;
    return static_cast<uint32_t>(d);
}

int grid_for(size_t work, int sms) {
    return static_cast<int>(std::max<size_t>(1, std::min<size_t>((work + 255) / 256, static_cast<size_t>(sms) * 8)));
}

}  // namespace
}  // namespace hme

using namespace hme;

extern "C" {

int hme_ctx_set_elim_options(hme_ctx* ctx, int panel, int rows_per_cta, int panel_ctas, int back_block) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr, "null context");
        HME_REQUIRE(panel >= 0 && panel <= 128, "panel must be in [1, 128] (0 = default)");
        ElimOptions& o = opts(ctx);
        o.panel = panel > 0 ? panel : 64;
        o.rows_per_cta = rows_per_cta > 0 ? rows_per_cta : 32;
        o.panel_ctas = panel_ctas > 0 ? panel_ctas : 0;
        o.back_block = back_block > 0 ? back_block : 128;
    });
}

int hme_ctx_set_panel_kernel(hme_ctx* ctx, int mode) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr, "null context");
        HME_REQUIRE(mode >= 0 && mode <= 3,
                    "panel kernel mode must be 0 (automatic), 1 (grid), 2 (cluster) or 3 (cluster, 1024 threads)");
        opts(ctx).panel_kernel = mode;
    });
}

int hme_ctx_elim_panel_stats(const hme_ctx* ctx, uint64_t* block_panels, uint64_t* search_panels) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr && block_panels != nullptr && search_panels != nullptr, "null argument");
        *block_panels = ctx->elim_block_panels;
        *search_panels = ctx->elim_search_panels;
    });
}

int hme_ctx_set_elim_lookahead(hme_ctx* ctx, int on) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr, "null context");
        opts(ctx).no_lookahead = on == 0;
    });
}

int hme_rref_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t* A, size_t lda, uint32_t* pivots,
                     uint32_t* rank) {
    return guard([&] {
        HME_REQUIRE(ctx && rank, "null argument");
        require_field(p);
        HME_REQUIRE(lda >= n, "lda < n");
        bind(ctx);
        ElimOptions o = opts(ctx);
        const ElimResult r = elim_device(ctx, make_mod(p), A, lda, m, n, true, A, lda, o);
        check_device_error(ctx);
        *rank = r.rank;
        if (pivots)
            for (int t = 0; t < r.rank; ++t) pivots[t] = r.pivots[t];
    });
}

int hme_rref_u32(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t* A, size_t lda, uint32_t* pivots,
                 uint32_t* rank) {
    return guard([&] {
        HME_REQUIRE(ctx && rank, "null argument");
        require_field(p);
        HME_REQUIRE(m == 0 || n == 0 || (A && lda >= n), "bad A");
        bind(ctx);
        *rank = 0;
        if (m == 0 || n == 0) return;
        uint32_t* d = upload(ctx, kSlotStageA, A, lda, m, n);
        const size_t dl = padded_ld(n);
        ElimOptions o = opts(ctx);
        const ElimResult r = elim_device(ctx, make_mod(p), d, dl, m, n, true, d, dl, o);
        HME_CUDA(cudaMemcpy2DAsync(A, sizeof(uint32_t) * lda, d, sizeof(uint32_t) * dl, sizeof(uint32_t) * n, m,
                                   cudaMemcpyDeviceToHost, ctx->stream));
        check_device_error(ctx);
        *rank = r.rank;
        if (pivots)
            for (int t = 0; t < r.rank; ++t) pivots[t] = r.pivots[t];
    });
}

int hme_rank_profile_u32(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t n, const uint32_t* A, size_t lda,
                         uint32_t* pivots, uint32_t* rank) {
    return guard([&] {
        HME_REQUIRE(ctx && rank, "null argument");
        require_field(p);
        HME_REQUIRE(m == 0 || n == 0 || (A && lda >= n), "bad A");
        bind(ctx);
        *rank = 0;
        if (m == 0 || n == 0) return;
        uint32_t* d = upload(ctx, kSlotStageA, A, lda, m, n);
        ElimOptions o = opts(ctx);
        const ElimResult r = elim_device(ctx, make_mod(p), d, padded_ld(n), m, n, false, nullptr, 0, o);
        check_device_error(ctx);
        *rank = r.rank;
        if (pivots)
            for (int t = 0; t < r.rank; ++t) pivots[t] = r.pivots[t];
    });
}

int hme_det_u32(hme_ctx* ctx, uint32_t p, uint32_t n, const uint32_t* A, size_t lda, uint32_t* det) {
    return guard([&] {
        HME_REQUIRE(ctx && det, "null argument");
        require_field(p);
        bind(ctx);
        if (n == 0) {
            *det = 1 % p;
            return;
        }
        HME_REQUIRE(A && lda >= n, "bad A");
        uint32_t* d = upload(ctx, kSlotStageA, A, lda, n, n);
        ElimOptions o = opts(ctx);
        o.want_diag = true;
        const ElimResult r = elim_device(ctx, make_mod(p), d, padded_ld(n), n, n, false, nullptr, 0, o);
        check_device_error(ctx);
        *det = det_from(r, n, p);
    });
}

int hme_rref_det_u32(hme_ctx* ctx, uint32_t p, uint32_t n, uint32_t* A, size_t lda, uint32_t* pivots,
                     uint32_t* rank, uint32_t* det) {
    return guard([&] {
        HME_REQUIRE(ctx && rank && det, "null argument");
        require_field(p);
        bind(ctx);
        *rank = 0;
        *det = 1 % p;
        if (n == 0) return;
        HME_REQUIRE(A && lda >= n, "bad A");
        uint32_t* d = upload(ctx, kSlotStageA, A, lda, n, n);
        const size_t dl = padded_ld(n);
        ElimOptions o = opts(ctx);
        o.want_diag = true;
        const ElimResult r = elim_device(ctx, make_mod(p), d, dl, n, n, true, d, dl, o);
        HME_CUDA(cudaMemcpy2DAsync(A, sizeof(uint32_t) * lda, d, sizeof(uint32_t) * dl, sizeof(uint32_t) * n, n,
                                   cudaMemcpyDeviceToHost, ctx->stream));
        check_device_error(ctx);
        *rank = r.rank;
        if (pivots)
            for (int t = 0; t < r.rank; ++t) pivots[t] = r.pivots[t];
        *det = det_from(r, n, p);
    });
}

int hme_kernel_basis_u32(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t n, const uint32_t* A, size_t lda,
                         uint32_t* K, size_t ldk, uint32_t* nullity) {
    return guard([&] {
        HME_REQUIRE(ctx && nullity, "null argument");
        require_field(p);
        bind(ctx);
        *nullity = n;
        if (n == 0) return;
        HME_REQUIRE(K && ldk >= n, "bad K");
        std::vector<int> piv;
        uint32_t* d = nullptr;
        int rank = 0;
        if (m > 0) {
            HME_REQUIRE(A && lda >= n, "bad A");
            d = upload(ctx, kSlotStageA, A, lda, m, n);
            ElimOptions o = opts(ctx);
            const ElimResult r = elim_device(ctx, make_mod(p), d, padded_ld(n), m, n, true, d, padded_ld(n), o);
            piv = r.pivots;
            rank = r.rank;
        }
        const int f = static_cast<int>(n) - rank;
        *nullity = f;
        if (f == 0) {
            check_device_error(ctx);
            return;
        }
        std::vector<int> freec;
        {
            std::vector<char> isp(n, 0);
            for (int x : piv) isp[x] = 1;
            for (uint32_t j = 0; j < n; ++j)
                if (!isp[j]) freec.push_back(static_cast<int>(j));
        }
        int* d_idx = static_cast<int*>(ctx->ws.get(kSlotElim5, sizeof(int) * (static_cast<size_t>(n) + 16)));
        if (rank) HME_CUDA(cudaMemcpyAsync(d_idx, piv.data(), sizeof(int) * rank, cudaMemcpyHostToDevice, ctx->stream));
        HME_CUDA(cudaMemcpyAsync(d_idx + rank, freec.data(), sizeof(int) * f, cudaMemcpyHostToDevice, ctx->stream));
        uint32_t* dK = static_cast<uint32_t*>(ctx->ws.get(kSlotStageC, sizeof(uint32_t) * static_cast<size_t>(f) * n));
        HME_TIMED(ctx, "kernel_basis", kernel_basis_kernel<<<grid_for(static_cast<size_t>(f) * n, ctx->num_sms), 256, 0,
                                                             ctx->stream>>>(d, padded_ld(n), n, rank, d_idx, d_idx + rank,
                                                                            f, p, dK, n));
        if (rank)
            HME_TIMED(ctx, "kernel_basis",
                      kernel_basis_fill_kernel<<<grid_for(static_cast<size_t>(f) * rank, ctx->num_sms), 256, 0,
                                                 ctx->stream>>>(d, padded_ld(n), rank, d_idx, d_idx + rank, f, p, dK, n));
        HME_CUDA(cudaGetLastError());
        HME_CUDA(cudaMemcpy2DAsync(K, sizeof(uint32_t) * ldk, dK, sizeof(uint32_t) * n, sizeof(uint32_t) * n, f,
                                   cudaMemcpyDeviceToHost, ctx->stream));
        check_device_error(ctx);
    });
}

int hme_inverse_u32(hme_ctx* ctx, uint32_t p, uint32_t n, const uint32_t* A, size_t lda, uint32_t* Ainv,
                    size_t ldi, int* invertible) {
    return guard([&] {
        HME_REQUIRE(ctx && invertible, "null argument");
        require_field(p);
        bind(ctx);
        *invertible = 0;
        if (n == 0) {
            *invertible = 1;
            return;
        }
        HME_REQUIRE(A && Ainv && lda >= n && ldi >= n, "bad A / Ainv");
        // RREF([A | I]) (DenseElim.h:186-189): invertible iff the pivots are 0 .. n-1
        const size_t w = 2 * static_cast<size_t>(n);
        std::vector<uint32_t> aug(static_cast<size_t>(n) * w, 0);
        for (uint32_t i = 0; i < n; ++i) {
            std::memcpy(&aug[i * w], A + i * lda, sizeof(uint32_t) * n);
            aug[i * w + n + i] = 1 % p;
        }
        uint32_t* d = upload(ctx, kSlotStageA, aug.data(), w, n, static_cast<uint32_t>(w));
        const size_t dl = padded_ld(w);
        ElimOptions o = opts(ctx);
        const ElimResult r = elim_device(ctx, make_mod(p), d, dl, n, static_cast<int>(w), true, d, dl, o);
        check_device_error(ctx);
        bool ok = r.rank == static_cast<int>(n);
        for (int t = 0; ok && t < r.rank; ++t) ok = r.pivots[t] == t;
        if (!ok) return;
        HME_CUDA(cudaMemcpy2DAsync(Ainv, sizeof(uint32_t) * ldi, d + n, sizeof(uint32_t) * dl, sizeof(uint32_t) * n, n,
                                   cudaMemcpyDeviceToHost, ctx->stream));
        check_device_error(ctx);
        *invertible = 1;
    });
}

int hme_solve_u32(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t nb, uint32_t ny, const uint32_t* B, size_t ldb,
                  const uint32_t* Y, size_t ldy, uint32_t* X, size_t ldx) {
    return guard([&] {
        HME_REQUIRE(ctx, "null argument");
        require_field(p);
        bind(ctx);
        if (nb == 0 || ny == 0) return;
        HME_REQUIRE(X && ldx >= ny, "bad X");
        // RREF([B | Y]) (DenseElim.h:191-197): a pivot in the Y block means "not in the span"
        const size_t w = static_cast<size_t>(nb) + ny;
        std::vector<uint32_t> aug(static_cast<size_t>(m) * w, 0);
        for (uint32_t i = 0; i < m; ++i) {
            std::memcpy(&aug[i * w], B + i * ldb, sizeof(uint32_t) * nb);
            std::memcpy(&aug[i * w + nb], Y + i * ldy, sizeof(uint32_t) * ny);
        }
        std::vector<uint32_t> Xh(static_cast<size_t>(nb) * ny, 0);
        if (m > 0) {
            uint32_t* d = upload(ctx, kSlotStageA, aug.data(), w, m, static_cast<uint32_t>(w));
            const size_t dl = padded_ld(w);
            ElimOptions o = opts(ctx);
            const ElimResult r = elim_device(ctx, make_mod(p), d, dl, m, static_cast<int>(w), true, d, dl, o);
            for (int t = 0; t < r.rank; ++t)
                if (r.pivots[t] >= static_cast<int>(nb))
                    throw Error(HME_ENOTINSPAN, "solve: right-hand side " + std::to_string(r.pivots[t] - nb) +
                                                    " is not in the column span of B");
            std::vector<uint32_t> R(static_cast<size_t>(r.rank) * w);
            if (r.rank)
                HME_CUDA(cudaMemcpy2DAsync(R.data(), sizeof(uint32_t) * w, d, sizeof(uint32_t) * dl, sizeof(uint32_t) * w,
                                           r.rank, cudaMemcpyDeviceToHost, ctx->stream));
            check_device_error(ctx);
            for (int t = 0; t < r.rank; ++t)
                std::memcpy(&Xh[static_cast<size_t>(r.pivots[t]) * ny], &R[t * w + nb], sizeof(uint32_t) * ny);
        }
        for (uint32_t j = 0; j < nb; ++j) std::memcpy(X + j * ldx, &Xh[j * ny], sizeof(uint32_t) * ny);
    });
}

}  // extern "C"

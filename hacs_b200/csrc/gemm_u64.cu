// The mod-p GEMM for u64 residues (any modulus 2 <= p < 2^64): C op= A*B mod p.
//
// Reference semantics: engine::kernels::gemm<uint64_t> / engine::cuda::gemm
// <uint64_t> (src/ModArithmetic/Kernels.h:178-185; src/Cuda/cuda_kernels.cu
// :151-163 and the u64 tiles :365-381): the exact sum of k products, reduced
// to the canonical residue, combined by Set / Add / Sub.  The reference's u64
// regime multiplies in Montgomery form (odd p < 2^63) or with a wide mulmod
// (otherwise), one reduction per product, on CUDA cores.
//
// Method (residue number system).  With canonical inputs the exact integer
// X = sum_k a_ik b_kj lies in [0, k (p-1)^2].  Pick t primes q_0 > q_1 > ...
// just below 2^16 whose product M exceeds 4 k (p-1)^2.  Then:
//   1. A_t = A mod q_t, B_t = B mod q_t, written directly as the limb planes
//      the tensor-core GEMM reads (one pass over each operand for all t);
//   2. C_t = A_t B_t mod q_t: t products on the INT8-limb tensor-core GEMM
//      (two limbs each, 4 limb products: 4t in all, against the 64 an
//      8-limb u64 split would need);
//   3. the CRT, element by element (32-bit arithmetic throughout except the
//      final reduction): y_t = C_t (M/q_t)^-1 mod q_t gives
//      X = sum_t y_t M/q_t - w M with w = sum_t y_t / q_t - X/M, and since
//      X/M < 1/4, w = rint(sum_t y_t / q_t) computed in double precision
//      (error below 2^-45) is exact.  So X mod p = (sum_t y_t (M/q_t mod p)
//      + w (p - M mod p)) mod p: a sum below 2^20 p, accumulated in 128 bits
//      and reduced once (Montgomery REDC with the constants in Montgomery
//      form for odd p < 2^63, a 128-bit remainder otherwise).
// Moduli below 2^32 skip the RNS: the operands narrow to u32 and the u32 GEMM
// computes the product mod p directly.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "hme_internal.h"

namespace hme {
namespace {

constexpr int kMaxRns = 12;

// The primes, the CRT constants and p's constants, passed by value.  All the
// per-prime arithmetic is 32-bit: the primes are below 2^16, so x mod q_t
// for x < 2^32 is one 32-bit Barrett step (qm = floor(2^32 / q_t)), and the
// 64-bit constants enter as 32-bit halves.
struct RnsPlan {
    int t;
    uint32_t q[kMaxRns];
    uint32_t qm[kMaxRns];    // floor(2^32 / q_t)
    uint32_t c32[kMaxRns];   // 2^32 mod q_t
    uint32_t minv[kMaxRns];  // (M / q_t)^-1 mod q_t
    double qinv[kMaxRns];    // 1 / q_t
    uint32_t wlo[kMaxRns];   // W_t = (M / q_t) mod p (times 2^64 mod p when mont): low and high 32 bits
    uint32_t whi[kMaxRns];
    uint32_t nlo, nhi;       // (p - M mod p) mod p (times 2^64 mod p when mont): low and high 32 bits
    uint64_t p;
    uint64_t ninv;           // -p^-1 mod 2^64 (mont)
    int mont;
};

// x mod q for x < 2^32, q < 2^16, qm = floor(2^32 / q): the quotient estimate
// floor(x qm / 2^32) is floor(x / q) or one less, so one correction suffices.
__device__ __forceinline__ uint32_t red32(uint32_t x, uint32_t q, uint32_t qm) {
    const uint32_t r = x - __umulhi(x, qm) * q;
    return r >= q ? r - q : r;
}

using u128 = unsigned __int128;

// (hi 2^64 + lo) 2^-64 mod p for hi 2^64 + lo < p 2^64, p odd and < 2^63
__device__ __forceinline__ uint64_t redc(uint64_t lo, uint64_t hi, uint64_t p, uint64_t ninv) {
    const uint64_t m = lo * ninv;
    const uint64_t ml = m * p, mh = __umul64hi(m, p);
    const uint64_t c = (lo + ml) < lo ? 1u : 0u;  // lo + m p == 0 mod 2^64
    const uint64_t r = hi + mh + c;
    return r >= p ? r - p : r;
}

__device__ __forceinline__ uint64_t add_mod64(uint64_t a, uint64_t b, uint64_t p) {
    const uint64_t s = a + b;
    return (s < a || s >= p) ? s - p : s;
}
__device__ __forceinline__ uint64_t sub_mod64(uint64_t a, uint64_t b, uint64_t p) {
    return a >= b ? a - b : a + (p - b);
}
__device__ __forceinline__ uint64_t combine64(uint64_t old, uint64_t v, int op, uint64_t p) {
    return op == HME_SET ? v : op == HME_ADD ? add_mod64(old, v, p) : sub_mod64(old, v, p);
}

// x mod q from the 32-bit halves of x: (xh mod q)(2^32 mod q) + (xl mod q)
// <= (q-1)^2 + q - 1 < 2^32, one more Barrett step
__device__ __forceinline__ uint32_t res32(uint32_t xh, uint32_t xl, uint32_t q, uint32_t qm, uint32_t c32) {
    return red32(red32(xh, q, qm) * c32 + red32(xl, q, qm), q, qm);
}

// The limb planes of A mod every prime, straight from the u64 operand, in the
// layout the limb GEMM reads (two limbs per prime): prime t's planes start at
// pa + 2 t a_plane, plane j holds byte j of (a mod q_t), [m][Kp] K-major, zero
// for k in [K, Kp).  16 k per thread, one 16-byte store per plane.
template <int NT>
__global__ void __launch_bounds__(256) rns_split_a_kernel(const uint64_t* __restrict__ A, uint64_t lda, uint32_t m,
                                                          uint32_t k, uint32_t Kp, uint8_t* __restrict__ pa,
                                                          uint64_t a_plane, const __grid_constant__ RnsPlan P) {
    const uint32_t kch = Kp >> 4;
    const size_t total = static_cast<size_t>(m) * kch;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const uint32_t row = static_cast<uint32_t>(idx / kch);
        const uint32_t k0 = static_cast<uint32_t>(idx - static_cast<size_t>(row) * kch) << 4;
        const uint64_t* src = A + row * lda + k0;
        uint32_t xl[16], xh[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            const uint64_t v = k0 + e < k ? src[e] : 0u;
            xl[e] = static_cast<uint32_t>(v);
            xh[e] = static_cast<uint32_t>(v >> 32);
        }
        uint8_t* dst = pa + static_cast<size_t>(row) * Kp + k0;
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            uint32_t w0[4] = {0, 0, 0, 0}, w1[4] = {0, 0, 0, 0};
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                const uint32_t r = res32(xh[e], xl[e], P.q[t], P.qm[t], P.c32[t]);
                w0[e >> 2] |= (r & 0xffu) << (8 * (e & 3));
                w1[e >> 2] |= ((r >> 8) & 0xffu) << (8 * (e & 3));
            }
            *reinterpret_cast<uint4*>(dst + 2 * t * a_plane) = make_uint4(w0[0], w0[1], w0[2], w0[3]);
            *reinterpret_cast<uint4*>(dst + (2 * t + 1) * a_plane) = make_uint4(w1[0], w1[1], w1[2], w1[3]);
        }
    }
}

// The limb planes of B mod every prime: prime t's planes start at
// pb + 4 t b_plane, plane (i, j) holds byte j of (256^i (b mod q_t) mod q_t),
// [n][Kp] K-major (B transposed through shared memory, 64 k x 32 n per tile,
// 8 k per thread), zero for k in [K, Kp).
template <int NT>
__global__ void __launch_bounds__(256) rns_split_b_kernel(const uint64_t* __restrict__ B, uint64_t ldb, uint32_t k,
                                                          uint32_t n, uint32_t Kp, uint8_t* __restrict__ pb,
                                                          uint64_t b_plane, const __grid_constant__ RnsPlan P) {
    __shared__ uint64_t tile[64][33];
    const uint32_t bk = (Kp + 63) / 64, tiles = bk * ((n + 31) / 32);
    const uint32_t nn = threadIdx.x >> 3, kc = threadIdx.x & 7;
    for (uint32_t blk = blockIdx.x; blk < tiles; blk += gridDim.x) {
        const uint32_t k0 = (blk % bk) * 64, n0 = (blk / bk) * 32;
        uint64_t v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const uint32_t t = threadIdx.x + 256 * q, kk = k0 + (t >> 5), c = n0 + (t & 31);
            v[q] = (kk < k && c < n) ? B[kk * ldb + c] : 0u;
        }
        __syncthreads();  // the previous tile is out of shared memory
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const uint32_t t = threadIdx.x + 256 * q;
            tile[t >> 5][t & 31] = v[q];
        }
        __syncthreads();
        const uint32_t col = n0 + nn, kb = k0 + kc * 8;
        if (col >= n || kb >= Kp) continue;
        uint32_t xl[8], xh[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const uint64_t x = tile[kc * 8 + e][nn];
            xl[e] = static_cast<uint32_t>(x);
            xh[e] = static_cast<uint32_t>(x >> 32);
        }
        uint8_t* base = pb + static_cast<size_t>(col) * Kp + kb;
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            const uint32_t q = P.q[t], qm = P.qm[t];
            uint32_t o[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};  // [2 i + j][word]
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const uint32_t r = res32(xh[e], xl[e], q, qm, P.c32[t]);
                const uint32_t r2 = red32(r << 8, q, qm);  // 256 r mod q (r < 2^16)
                const int sh = 8 * (e & 3);
                o[0][e >> 2] |= (r & 0xffu) << sh;
                o[1][e >> 2] |= ((r >> 8) & 0xffu) << sh;
                o[2][e >> 2] |= (r2 & 0xffu) << sh;
                o[3][e >> 2] |= ((r2 >> 8) & 0xffu) << sh;
            }
#pragma unroll
            for (int ij = 0; ij < 4; ++ij)
                *reinterpret_cast<uint2*>(base + (4 * t + ij) * b_plane) = make_uint2(o[ij][0], o[ij][1]);
        }
    }
}

// C[r][c] op= CRT(R[.][r][c]) mod p
template <bool MONT, int NT>
__global__ void __launch_bounds__(256) rns_crt_kernel(const uint32_t* __restrict__ R, uint32_t rows, uint32_t cols,
                                                      uint64_t* __restrict__ C, uint64_t ldc, int op,
                                                      const __grid_constant__ RnsPlan P) {
    const size_t plane = static_cast<size_t>(rows) * cols;
    for (uint32_t r = blockIdx.y; r < rows; r += gridDim.y)
        for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x) {
            const uint32_t* src = R + static_cast<size_t>(r) * cols + c;
            // T = sum_t y_t W_t + w N = s0 + s1 2^32 with s0 = sum y (W mod 2^32), s1 = sum y (W >> 32):
            // each term below 2^48, at most 13 terms, so both sums stay below 2^52
            uint64_t s0 = 0, s1 = 0;
            double wf = 0.0;
            uint32_t rv[NT];
#pragma unroll
            for (int t = 0; t < NT; ++t) rv[t] = src[t * plane];
#pragma unroll
            for (int t = 0; t < NT; ++t) {
                const uint32_t y = red32(rv[t] * P.minv[t], P.q[t], P.qm[t]);  // both < 2^16
                wf = fma(static_cast<double>(y), P.qinv[t], wf);
                s0 += static_cast<uint64_t>(y) * P.wlo[t];
                s1 += static_cast<uint64_t>(y) * P.whi[t];
            }
            const uint32_t w = static_cast<uint32_t>(rint(wf));
            s0 += static_cast<uint64_t>(w) * P.nlo;
            s1 += static_cast<uint64_t>(w) * P.nhi;
            const uint64_t lo = s0 + (s1 << 32);
            const uint64_t hi = (s1 >> 32) + (lo < s0 ? 1u : 0u);
            uint64_t v;
            if constexpr (MONT)
                v = redc(lo, hi, P.p, P.ninv);
            else
                v = static_cast<uint64_t>(((static_cast<u128>(hi) << 64) | lo) % P.p);
            uint64_t* cp = C + r * ldc + c;
            *cp = combine64(op == HME_SET ? 0u : *cp, v, op, P.p);
        }
}

// u64 -> u32 (entries below p < 2^32)
__global__ void __launch_bounds__(256) narrow_kernel(const uint64_t* __restrict__ X, uint64_t ldx, uint32_t rows,
                                                     uint32_t cols, uint32_t* __restrict__ out) {
    for (uint32_t r = blockIdx.y; r < rows; r += gridDim.y)
        for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x)
            out[static_cast<size_t>(r) * cols + c] = static_cast<uint32_t>(X[r * ldx + c]);
}
// C[r][c] op= R[r][c]  mod p
__global__ void __launch_bounds__(256) widen_kernel(const uint32_t* __restrict__ R, uint32_t rows, uint32_t cols,
                                                    uint64_t* __restrict__ C, uint64_t ldc, int op, uint64_t p) {
    for (uint32_t r = blockIdx.y; r < rows; r += gridDim.y)
        for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x) {
            uint64_t* cp = C + r * ldc + c;
            *cp = combine64(op == HME_SET ? 0u : *cp, R[static_cast<size_t>(r) * cols + c], op, p);
        }
}
__global__ void zero64_kernel(uint64_t* C, uint64_t ldc, uint32_t rows, uint32_t cols) {
    for (uint32_t r = blockIdx.y; r < rows; r += gridDim.y)
        for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x)
            C[r * ldc + c] = 0;
}

// f(std::integral_constant<int, t>) for the plan's prime count t (5..12: p >= 2^32 needs
// at least 67 bits of M, and a plan holds at most kMaxRns primes)
template <class F>
void with_primes(int t, F&& f) {
    switch (t) {
        case 5: f(std::integral_constant<int, 5>{}); break;
        case 6: f(std::integral_constant<int, 6>{}); break;
        case 7: f(std::integral_constant<int, 7>{}); break;
        case 8: f(std::integral_constant<int, 8>{}); break;
        case 9: f(std::integral_constant<int, 9>{}); break;
        case 10: f(std::integral_constant<int, 10>{}); break;
        case 11: f(std::integral_constant<int, 11>{}); break;
        case 12: f(std::integral_constant<int, 12>{}); break;
        default: throw Error(HME_EINVAL, "gemm_u64: unsupported prime count");
    }
}

dim3 grid2d(uint32_t rows, uint32_t cols, int sms) {
    const uint32_t gx = std::min<uint32_t>((cols + 255) / 256, 64);
    const uint32_t gy = std::max<uint32_t>(1, std::min<uint32_t>(rows, static_cast<uint32_t>(sms) * 16 / gx + 1));
    return dim3(gx, std::min<uint32_t>(gy, 65535));
}

uint64_t mulmod_host(uint64_t a, uint64_t b, uint64_t p) { return static_cast<uint64_t>(static_cast<u128>(a) * b % p); }
uint32_t powmod32(uint32_t a, uint32_t e, uint32_t q) {
    uint64_t r = 1, b = a % q;
    for (; e; e >>= 1, b = b * b % q)
        if (e & 1) r = r * b % q;
    return static_cast<uint32_t>(r);
}

// The plan for modulus p >= 2^32 and inner dimension k.
RnsPlan make_plan(uint64_t p, uint32_t k) {
    RnsPlan P{};
    // bits needed: M > 4 k (p-1)^2, with one bit of margin on the double-precision logs
    const double need = std::log2(static_cast<double>(std::max<uint32_t>(k, 1))) +
                        2.0 * std::log2(static_cast<double>(p - 1)) + 3.0;
    double have = 0;
    for (uint32_t q = 65521; q > 40000 && have <= need; q -= 2) {
        if (!is_prime_u32(q)) continue;
        HME_REQUIRE(P.t < kMaxRns, "gemm_u64: inner dimension too large for the residue system");
        P.q[P.t++] = q;
        have += std::log2(static_cast<double>(q));
    }
    HME_REQUIRE(have > need, "gemm_u64: inner dimension too large for the residue system");
    P.p = p;
    P.mont = (p & 1) && p < (uint64_t(1) << 63);
    const uint64_t r64 = P.mont ? static_cast<uint64_t>((static_cast<u128>(1) << 64) % p) : 1;  // 2^64 mod p
    uint64_t m_mod_p = 1;
    for (int t = 0; t < P.t; ++t) m_mod_p = mulmod_host(m_mod_p, P.q[t], p);
    for (int t = 0; t < P.t; ++t) {
        const uint32_t q = P.q[t];
        uint64_t mt_p = 1;   // (M / q_t) mod p
        uint32_t mt_q = 1;   // (M / q_t) mod q_t
        for (int s = 0; s < P.t; ++s)
            if (s != t) {
                mt_p = mulmod_host(mt_p, P.q[s], p);
                mt_q = static_cast<uint32_t>(static_cast<uint64_t>(mt_q) * (P.q[s] % q) % q);
            }
        P.minv[t] = powmod32(mt_q, q - 2, q);
        P.qm[t] = static_cast<uint32_t>((uint64_t(1) << 32) / q);
        P.c32[t] = static_cast<uint32_t>((uint64_t(1) << 32) % q);
        P.qinv[t] = 1.0 / static_cast<double>(q);
        const uint64_t w = P.mont ? mulmod_host(mt_p, r64, p) : mt_p;
        P.wlo[t] = static_cast<uint32_t>(w);
        P.whi[t] = static_cast<uint32_t>(w >> 32);
    }
    const uint64_t neg = m_mod_p ? p - m_mod_p : 0;
    const uint64_t nm = P.mont ? mulmod_host(neg, r64, p) : neg;
    P.nlo = static_cast<uint32_t>(nm);
    P.nhi = static_cast<uint32_t>(nm >> 32);
    if (P.mont) {
        uint64_t inv = p;  // Newton: p inv == 1 mod 2^64
        for (int i = 0; i < 6; ++i) inv *= 2 - p * inv;
        P.ninv = 0 - inv;
    }
    return P;
}

// C op= A*B mod p, device pointers, on ctx->stream.
void gemm_u64_device(hme_ctx* ctx, uint64_t p, uint32_t m, uint32_t n, uint32_t k, const uint64_t* A, size_t lda,
                     const uint64_t* B, size_t ldb, uint64_t* C, size_t ldc, int op) {
    HME_REQUIRE(p >= 2, "gemm_u64: modulus must be >= 2");
    HME_REQUIRE(op == HME_SET || op == HME_ADD || op == HME_SUB, "gemm_u64: op must be HME_SET, HME_ADD or HME_SUB");
    if (m == 0 || n == 0) return;
    HME_REQUIRE(C && ldc >= n, "gemm_u64: bad C");
    if (k == 0) {
        if (op == HME_SET) {
            HME_TIMED(ctx, "zero64", zero64_kernel<<<grid2d(m, n, ctx->num_sms), 256, 0, ctx->stream>>>(C, ldc, m, n));
            HME_CUDA(cudaGetLastError());
        }
        return;
    }
    HME_REQUIRE(A && B && lda >= k && ldb >= n, "gemm_u64: bad A / B");
    const int sms = ctx->num_sms;
    if (p < (uint64_t(1) << 32)) {
        uint32_t* a32 = static_cast<uint32_t*>(ctx->ws.get(kSlotRns0, 4ull * m * k));
        uint32_t* b32 = static_cast<uint32_t*>(ctx->ws.get(kSlotRns1, 4ull * k * n));
        uint32_t* c32 = static_cast<uint32_t*>(ctx->ws.get(kSlotRns2, 4ull * m * n));
        HME_TIMED(ctx, "narrow", narrow_kernel<<<grid2d(m, k, sms), 256, 0, ctx->stream>>>(A, lda, m, k, a32));
        HME_TIMED(ctx, "narrow", narrow_kernel<<<grid2d(k, n, sms), 256, 0, ctx->stream>>>(B, ldb, k, n, b32));
        HME_CUDA(cudaGetLastError());
        gemm_u32_device(ctx, make_mod(static_cast<uint32_t>(p)), m, n, k, a32, k, b32, n, c32, n, HME_SET);
        HME_TIMED(ctx, "widen", widen_kernel<<<grid2d(m, n, sms), 256, 0, ctx->stream>>>(c32, m, n, C, ldc, op, p));
        HME_CUDA(cudaGetLastError());
        return;
    }
    const RnsPlan P = make_plan(p, k);
    // each prime's limb planes written straight from the u64 operands, then t limb GEMMs on them
    const int Kp = limb_kp(k);
    const uint64_t a_plane = static_cast<uint64_t>(m) * Kp, b_plane = static_cast<uint64_t>(n) * Kp;
    const size_t pc = static_cast<size_t>(m) * n;
    uint8_t* pa = static_cast<uint8_t*>(ctx->ws.get(kSlotRns0, 2 * a_plane * P.t));
    uint8_t* pb = static_cast<uint8_t*>(ctx->ws.get(kSlotRns1, 4 * b_plane * P.t));
    uint32_t* rc = static_cast<uint32_t*>(ctx->ws.get(kSlotRns2, 4 * pc * P.t));
    const int ga = static_cast<int>(std::min<size_t>((static_cast<size_t>(m) * (Kp / 16) + 255) / 256, sms * 8ull));
    const int gb = static_cast<int>(std::min<size_t>(static_cast<size_t>((Kp + 63) / 64) * ((n + 31) / 32), sms * 8ull));
    with_primes(P.t, [&](auto nt) {
        constexpr int NT = decltype(nt)::value;
        HME_TIMED(ctx, "rns_split", rns_split_a_kernel<NT><<<ga, 256, 0, ctx->stream>>>(A, lda, m, k, Kp, pa, a_plane, P));
        HME_TIMED(ctx, "rns_split", rns_split_b_kernel<NT><<<gb, 256, 0, ctx->stream>>>(B, ldb, k, n, Kp, pb, b_plane, P));
    });
    HME_CUDA(cudaGetLastError());
    for (int t = 0; t < P.t; ++t)
        gemm_u32_planes(ctx, make_mod(P.q[t]), m, n, k, Kp, pa + 2 * t * a_plane, a_plane, pb + 4 * t * b_plane,
                        rc + t * pc, n, HME_SET);
    with_primes(P.t, [&](auto nt) {
        constexpr int NT = decltype(nt)::value;
        if (P.mont)
            HME_TIMED(ctx, "rns_crt", rns_crt_kernel<true, NT><<<grid2d(m, n, sms), 256, 0, ctx->stream>>>(
                                          rc, m, n, C, ldc, op, P));
        else
            HME_TIMED(ctx, "rns_crt", rns_crt_kernel<false, NT><<<grid2d(m, n, sms), 256, 0, ctx->stream>>>(
                                          rc, m, n, C, ldc, op, P));
    });
    HME_CUDA(cudaGetLastError());
}

}  // namespace
}  // namespace hme

using namespace hme;

extern "C" {

int hme_gemm_u64_dev(hme_ctx* ctx, uint64_t p, uint32_t m, uint32_t n, uint32_t k, const uint64_t* A, size_t lda,
                     const uint64_t* B, size_t ldb, uint64_t* C, size_t ldc, int op) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr, "null context");
        bind(ctx);
        gemm_u64_device(ctx, p, m, n, k, A, lda, B, ldb, C, ldc, op);
    });
}

int hme_gemm_u64(hme_ctx* ctx, uint64_t p, uint32_t m, uint32_t n, uint32_t k, const uint64_t* A, size_t lda,
                 const uint64_t* B, size_t ldb, uint64_t* C, size_t ldc, int op) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr, "null context");
        HME_REQUIRE(op == HME_SET || op == HME_ADD || op == HME_SUB, "gemm_u64: op must be HME_SET, HME_ADD or HME_SUB");
        if (m == 0 || n == 0) return;
        HME_REQUIRE(C && ldc >= n && (k == 0 || (A && B && lda >= k && ldb >= n)), "gemm_u64: bad buffers");
        bind(ctx);
        uint64_t* dA = k ? static_cast<uint64_t*>(ctx->ws.get(kSlotStageA, 8ull * m * k)) : nullptr;
        uint64_t* dB = k ? static_cast<uint64_t*>(ctx->ws.get(kSlotStageB, 8ull * k * n)) : nullptr;
        uint64_t* dC = static_cast<uint64_t*>(ctx->ws.get(kSlotStageC, 8ull * m * n));
        if (k) {
            HME_CUDA(copy_rows_async(dA, 8ull * k, A, 8 * lda, 8ull * k, m, cudaMemcpyHostToDevice, ctx->stream));
            HME_CUDA(copy_rows_async(dB, 8ull * n, B, 8 * ldb, 8ull * n, k, cudaMemcpyHostToDevice, ctx->stream));
        }
        if (op != HME_SET)
            HME_CUDA(copy_rows_async(dC, 8ull * n, C, 8 * ldc, 8ull * n, m, cudaMemcpyHostToDevice, ctx->stream));
        gemm_u64_device(ctx, p, m, n, k, dA, k, dB, n, dC, n, op);
        if (op == HME_SET || k)
            HME_CUDA(copy_rows_async(C, 8 * ldc, dC, 8ull * n, 8ull * n, m, cudaMemcpyDeviceToHost, ctx->stream));
        HME_CUDA(cudaStreamSynchronize(ctx->stream));
        check_device_error(ctx);
    });
}

}  // extern "C"

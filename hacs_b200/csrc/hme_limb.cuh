// Shared pieces of the INT8-limb GEMM kernels (limb_gemm.cu, grouped_gemm.cu):
// tile configuration, and the limb-split device routines.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "hme_mod.h"
#include "hme_ptx.cuh"

namespace hme {
namespace limb {

constexpr int kBM = 128;     // UMMA M (rows of C per tile, one TMEM lane each)
constexpr int kBK = 128;     // bytes of K per pipeline stage: one 128-byte swizzle row
constexpr int kEpiWarps = 8;                 // epilogue warps: two per TMEM lane quarter
constexpr int kThreads = 64 + 32 * kEpiWarps;  // + the TMA warp and the MMA warp

// KB: bytes of K per pipeline stage = the width of one swizzle row (128, 64 or
// 32; products whose K fits a narrower row stream no zero padding).
template <int L, int BN, int KB = kBK>
struct Cfg {
    static_assert(KB == 128 || KB == 64 || KB == 32, "k-block of 128, 64 or 32 bytes");
    static constexpr int UN = L * BN;  // UMMA N: L accumulators of BN columns
    static_assert(UN % 16 == 0 && UN >= 16 && UN <= 256, "UMMA N must be a multiple of 16 in [16, 256]");
    static_assert(BN % 16 == 0, "the epilogue drains 16 columns at a time");
    static constexpr int A_BYTES = kBM * KB;
    static constexpr int B_BYTES = UN * KB;
    static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
    static constexpr int STAGES = (196608 / STAGE_BYTES) < 12 ? (196608 / STAGE_BYTES) : 12;
    static constexpr int ACC_STRIDE = UN <= 32 ? 32 : UN <= 64 ? 64 : UN <= 128 ? 128 : 256;
    static constexpr int TMEM_COLS = 2 * ACC_STRIDE;
    static constexpr int BAR_BYTES = 256;
    static constexpr int EPI_BYTES = kEpiWarps * 32 * 17 * 4;  // per-warp 32 x 16 staging chunk (+1 column of padding)
    static constexpr int SMEM = STAGES * STAGE_BYTES + 1024 + BAR_BYTES + EPI_BYTES;
    static constexpr uint32_t IDESC = idesc_u8(kBM, UN);
    static_assert((2 * STAGES + 5) * 8 + 8 <= BAR_BYTES, "barrier area too small");
};

// ---- limb split (one launch for both operands) ------------------------------------
// Blocks [0, a_blocks): A planes[i][m][k] = byte i of A[m][k], 16 k per thread
// (four 16-byte loads when A rows are 16-byte aligned).  Blocks [a_blocks, ..):
// B planes[i][j][n][k] = byte j of (256^i * B[k][n] mod p), B transposed to
// K-major through shared memory, 64 k x 32 n per block, 8 k per thread.
// k in [K, Kp) is written as zero in both.
struct SplitArgs {
    const uint32_t* A;
    uint64_t lda;
    const uint32_t* B;
    uint64_t ldb;
    int M, N, K, Kp;
    uint32_t p;
    uint64_t barrett;
    uint8_t* planesA;
    uint8_t* planesB;
    int a_blocks;        // blocks of the A part
    int b_blocks_k;      // B part: blocks along k (64 k each)
    bool a_vec;          // A rows 16-byte aligned: vector loads
    uint64_t a_plane;    // bytes between A limb planes (0: M * Kp)
    uint64_t b_plane;    // bytes between B limb planes (0: N * Kp)
};

template <int L>
__device__ __forceinline__ void split_a_part(const SplitArgs& s, int block) {
    const int kch = s.Kp >> 4;
    const size_t total = static_cast<size_t>(s.M) * kch;
    const size_t plane = s.a_plane ? s.a_plane : static_cast<size_t>(s.M) * s.Kp;
    for (size_t idx = static_cast<size_t>(block) * blockDim.x + threadIdx.x; idx < total;
         idx += static_cast<size_t>(s.a_blocks) * blockDim.x) {
        const int row = static_cast<int>(idx / kch);
        const int k0 = static_cast<int>(idx - static_cast<size_t>(row) * kch) << 4;
        const uint32_t* src = s.A + static_cast<size_t>(row) * s.lda + k0;
        uint32_t x[16];
        if (s.a_vec && k0 + 16 <= s.K) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint4 v = __ldg(reinterpret_cast<const uint4*>(src) + q);
                x[4 * q] = v.x; x[4 * q + 1] = v.y; x[4 * q + 2] = v.z; x[4 * q + 3] = v.w;
            }
        } else {
#pragma unroll
            for (int e = 0; e < 16; ++e) x[e] = (k0 + e < s.K) ? __ldg(src + e) : 0u;
        }
        uint8_t* dst = s.planesA + static_cast<size_t>(row) * s.Kp + k0;
#pragma unroll
        for (int j = 0; j < L; ++j) {
            uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
            for (int e = 0; e < 16; ++e) w[e >> 2] |= ((x[e] >> (8 * j)) & 0xffu) << (8 * (e & 3));
            *reinterpret_cast<uint4*>(dst + j * plane) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

template <int L>
__device__ __forceinline__ void split_b_part(const SplitArgs& s, int block, uint32_t (*tile)[33]) {
    const int k0 = (block % s.b_blocks_k) * 64, n0 = (block / s.b_blocks_k) * 32;
    // all eight loads of a thread in flight before the first shared-memory store
    // (blockDim.x == 256: 8 x 256 = the 64 x 32 tile)
    uint32_t v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int t = threadIdx.x + 256 * q;
        const int k = k0 + (t >> 5), n = n0 + (t & 31);
        v[q] = (k < s.K && n < s.N) ? __ldg(s.B + static_cast<size_t>(k) * s.ldb + n) : 0u;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int t = threadIdx.x + 256 * q;
        tile[t >> 5][t & 31] = v[q];
    }
    __syncthreads();
    const int nn = threadIdx.x >> 3, kc = threadIdx.x & 7;
    const int n = n0 + nn, kb = k0 + kc * 8;
    if (n >= s.N || kb >= s.Kp) return;
    uint32_t out[L][L][2];
#pragma unroll
    for (int i = 0; i < L; ++i)
#pragma unroll
        for (int j = 0; j < L; ++j) out[i][j][0] = out[i][j][1] = 0;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        uint32_t v = tile[kc * 8 + e][nn];
#pragma unroll
        for (int i = 0; i < L; ++i) {
            if (i) v = reduce_u64(static_cast<uint64_t>(v) << 8, s.p, s.barrett);
#pragma unroll
            for (int j = 0; j < L; ++j) out[i][j][e >> 2] |= ((v >> (8 * j)) & 0xffu) << (8 * (e & 3));
        }
    }
    const size_t plane = s.b_plane ? s.b_plane : static_cast<size_t>(s.N) * s.Kp;
#pragma unroll
    for (int i = 0; i < L; ++i)
#pragma unroll
        for (int j = 0; j < L; ++j)
            *reinterpret_cast<uint2*>(s.planesB + (i * L + j) * plane + static_cast<size_t>(n) * s.Kp + kb) =
                make_uint2(out[i][j][0], out[i][j][1]);
}

}  // namespace limb

// Host: encode a tiled uint8 TMA descriptor with 128-byte swizzle (limb planes).
void encode_tma_u8(CUtensorMap* map, void* base, int rank, const cuuint64_t* dims, const cuuint64_t* strides,
                   const cuuint32_t* box);
// The same with the swizzle matching a k-block of kb bytes (128, 64 or 32).
void encode_tma_u8_kb(CUtensorMap* map, void* base, int rank, const cuuint64_t* dims, const cuuint64_t* strides,
                      const cuuint32_t* box, int kb);

}  // namespace hme

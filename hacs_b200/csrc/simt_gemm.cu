// CUDA-core mod-p GEMM for small products: one launch, no limb planes.
//
// C op= A*B mod p with exact u64 accumulation, reduced (Barrett, the
// ModCtx<uint32_t>::reduce_u64 rule) every kmax products, where
// kmax = floor((2^64 - 1) / (p - 1)^2) is the reference's delayed-accumulation
// bound (src/ModArithmetic/ModCtx.h:139-142).  It is one of the schedules the
// scheduler chooses from: for shapes of a few tiles its single launch beats
// the tensor-core path's split + GEMM launches.  TILE x TILE outputs per CTA,
// (TILE/4)^2 threads, 4 x 4 outputs per thread, K staged through shared memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "hme_grouped.h"
#include "hme_internal.h"

namespace hme {
namespace {

// One TILE x TILE tile of C (rows row0.., columns col0..) by the calling CTA.
template <int TILE>
__device__ __forceinline__ void simt_tile(const uint32_t* __restrict__ A, uint64_t lda,
                                          const uint32_t* __restrict__ B, uint64_t ldb, uint32_t* __restrict__ C,
                                          uint64_t ldc, int M, int N, int K, uint32_t p, uint64_t barrett,
                                          uint32_t kmax, int op, int row0, int col0) {
    constexpr int KT = 16;
    constexpr int TPR = TILE / 4;  // threads per row of the thread grid
    __shared__ uint32_t sA[KT][TILE + 1];
    __shared__ uint32_t sB[KT][TILE + 1];
    const int tx = threadIdx.x % TPR, ty = threadIdx.x / TPR;
    uint64_t acc[4][4];
    uint32_t res[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            acc[i][j] = 0;
            res[i][j] = 0;
        }
    uint32_t since = 0;
    for (int k0 = 0; k0 < K; k0 += KT) {
        for (int idx = threadIdx.x; idx < KT * TILE; idx += blockDim.x) {
            const int kk = idx / TILE, t = idx % TILE;
            const int ra = row0 + t, ka = k0 + kk;
            sA[kk][t] = (ra < M && ka < K) ? A[static_cast<size_t>(ra) * lda + ka] : 0u;
            const int cb = col0 + t;
            sB[kk][t] = (ka < K && cb < N) ? B[static_cast<size_t>(ka) * ldb + cb] : 0u;
        }
        __syncthreads();
        const int kt = min(KT, K - k0);
        for (int kk = 0; kk < kt; ++kk) {
            uint32_t a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = sA[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = sB[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] += static_cast<uint64_t>(a[i]) * b[j];
            if (++since == kmax) {
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        res[i][j] = mod_add(res[i][j], reduce_u64(acc[i][j], p, barrett), p);
                        acc[i][j] = 0;
                    }
                since = 0;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = row0 + ty * 4 + i;
        if (r >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = col0 + tx * 4 + j;
            if (c >= N) continue;
            const uint32_t v = mod_add(res[i][j], reduce_u64(acc[i][j], p, barrett), p);
            uint32_t* dst = C + static_cast<size_t>(r) * ldc + c;
            *dst = op == HME_SET ? v : op == HME_ADD ? mod_add(*dst, v, p) : mod_sub(*dst, v, p);
        }
    }
}

template <int TILE>
__global__ void __launch_bounds__((TILE / 4) * (TILE / 4))
    simt_gemm_kernel(const uint32_t* __restrict__ A, uint64_t lda, const uint32_t* __restrict__ B, uint64_t ldb,
                     uint32_t* __restrict__ C, uint64_t ldc, int M, int N, int K, uint32_t p, uint64_t barrett,
                     uint32_t kmax, int op) {
    simt_tile<TILE>(A, lda, B, ldb, C, ldc, M, N, K, p, barrett, kmax, op, blockIdx.y * TILE, blockIdx.x * TILE);
}

// One problem of a batched CUDA-core launch (one modulus per launch).
struct SimtProblem {
    const uint32_t* A;
    uint64_t lda;
    const uint32_t* B;
    uint64_t ldb;
    uint32_t* C;
    uint64_t ldc;
    int M, N, K, op;
    int tiles_n, tile_begin;
};

// Every tile of every problem, one CTA per tile (a grid-stride loop over the
// tile table); tile_prob[t] is the problem of tile t.
template <int TILE>
__global__ void __launch_bounds__((TILE / 4) * (TILE / 4))
    batch_simt_gemm_kernel(const SimtProblem* __restrict__ probs, const int* __restrict__ tile_prob, int tiles,
                           uint32_t p, uint64_t barrett, uint32_t kmax) {
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const SimtProblem P = probs[tile_prob[t]];
        const int local = t - P.tile_begin, tm = local / P.tiles_n, tn = local - tm * P.tiles_n;
        simt_tile<TILE>(P.A, P.lda, P.B, P.ldb, P.C, P.ldc, P.M, P.N, P.K, p, barrett, kmax, P.op, tm * TILE,
                        tn * TILE);
        __syncthreads();  // the tile's shared-memory stages are reused by the next tile
    }
}

uint32_t simt_kmax(const ModParams& mp) {
    const uint64_t d = static_cast<uint64_t>(mp.p - 1) * (mp.p - 1);
    return static_cast<uint32_t>(std::min<uint64_t>(d == 0 ? 1024 : (~0ull) / d, 1024));
}

}  // namespace

void batch_simt_gemm_device(hme_ctx* ctx, const ModParams& mp, const std::vector<GemmJob>& jobs, int tile) {
    std::vector<SimtProblem> probs;
    std::vector<int> tile_prob;
    for (const GemmJob& j : jobs) {
        if (j.M == 0 || j.N == 0) continue;
        SimtProblem P{j.A, j.lda, j.B, j.ldb, j.C, j.ldc, static_cast<int>(j.M), static_cast<int>(j.N),
                      static_cast<int>(j.K), j.op, static_cast<int>((j.N + tile - 1) / tile),
                      static_cast<int>(tile_prob.size())};
        const int nt = static_cast<int>((j.M + tile - 1) / tile) * P.tiles_n;
        tile_prob.insert(tile_prob.end(), nt, static_cast<int>(probs.size()));
        probs.push_back(P);
    }
    if (probs.empty()) return;
    const size_t pb = (sizeof(SimtProblem) * probs.size() + 255) / 256 * 256;
    char* d = static_cast<char*>(ctx->ws.get(kSlotJobs7, pb + sizeof(int) * tile_prob.size()));
    HME_CUDA(cudaMemcpyAsync(d, probs.data(), sizeof(SimtProblem) * probs.size(), cudaMemcpyHostToDevice,
                             ctx->stream));
    HME_CUDA(cudaMemcpyAsync(d + pb, tile_prob.data(), sizeof(int) * tile_prob.size(), cudaMemcpyHostToDevice,
                             ctx->stream));
    const int tiles = static_cast<int>(tile_prob.size());
    const uint32_t kmax = simt_kmax(mp);
    const SimtProblem* dp = reinterpret_cast<const SimtProblem*>(d);
    const int* dt = reinterpret_cast<const int*>(d + pb);
    if (tile == 32) {
        const int grid = std::min(tiles, ctx->num_sms * 16);
        HME_TIMED(ctx, "batch_simt_gemm",
                  batch_simt_gemm_kernel<32><<<grid, 64, 0, ctx->stream>>>(dp, dt, tiles, mp.p, mp.barrett, kmax));
    } else {
        const int grid = std::min(tiles, ctx->num_sms * 8);
        HME_TIMED(ctx, "batch_simt_gemm",
                  batch_simt_gemm_kernel<64><<<grid, 256, 0, ctx->stream>>>(dp, dt, tiles, mp.p, mp.barrett, kmax));
    }
    HME_CUDA(cudaGetLastError());
    // the host tables are consumed by the copies above before the caller may rebuild them
    HME_CUDA(cudaStreamSynchronize(ctx->stream));
}

void simt_gemm_u32_device(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A,
                          size_t lda, const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc, int op, int tile) {
    if (m == 0 || n == 0) return;
    const uint32_t kmax = simt_kmax(mp);
    if (tile == 32) {
        const dim3 grid((n + 31) / 32, (m + 31) / 32);
        HME_TIMED(ctx, "simt_gemm", simt_gemm_kernel<32><<<grid, 64, 0, ctx->stream>>>(
                                        A, lda, B, ldb, C, ldc, m, n, k, mp.p, mp.barrett, kmax, op));
    } else {
        const dim3 grid((n + 63) / 64, (m + 63) / 64);
        HME_TIMED(ctx, "simt_gemm", simt_gemm_kernel<64><<<grid, 256, 0, ctx->stream>>>(
                                        A, lda, B, ldb, C, ldc, m, n, k, mp.p, mp.barrett, kmax, op));
    }
    HME_CUDA(cudaGetLastError());
}

}  // namespace hme

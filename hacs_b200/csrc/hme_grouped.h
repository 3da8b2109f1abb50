// The grouped (many-shape) limb GEMM (grouped_gemm.cu).
#pragma once
#include <cstdint>
#include <vector>

#include <cuda.h>

#include "hme_internal.h"
#include "hme_limb.cuh"

namespace hme {

// One problem of a grouped launch.  Problems with the same padded K share one
// stacked plane tensor per operand (their rows / columns at offsets a_row0 /
// b_col0); tiles that run past a problem's rows or columns read a neighbour's
// planes, which only reach accumulator rows and columns the epilogue does not
// store.
struct GroupedProblem {
    const CUtensorMap* tmA;  // stacked limb planes of the A operands: dims {Kp, rows, L}
    const CUtensorMap* tmB;  // stacked limb planes of 256^i B: dims {Kp, cols, L, L}
    uint32_t* C;
    uint64_t ldc;
    int M, N;
    int kblocks;
    int op;
    int tiles_n;
    int tile_begin;
    int a_row0, b_col0;
};

// One problem's limb split in the grouped split launch.
struct GroupedSplitJob {
    limb::SplitArgs s;
    int b_blocks;     // blocks of the B part
    int block_begin;  // prefix over all jobs (A part then B part)
};

// The wide tile width of the grouped GEMM for L limbs (L * BN close to 256).
constexpr int grouped_bn_wide(int L) { return L == 1 ? 256 : L == 2 ? 128 : L == 3 ? 80 : 64; }

// The grouped split + GEMM on tables built on the device (32-byte k-blocks, wide
// tiles): block and tile counts, the per-block job and per-tile problem indexes
// are read from device memory when the kernels run, so the launches have fixed
// shapes (persistent grids) and can be captured in a CUDA graph.
// Kernel attributes of those launches, set outside any stream capture.
void grouped_prepare_device_tables(uint32_t limbs);
void grouped_launch_device_tables(hme_ctx* ctx, const ModParams& mp, const GroupedSplitJob* d_split,
                                  const int* d_block_job, const int* d_nblocks, const GroupedProblem* d_probs,
                                  const int* d_tile_prob, const int* d_ntiles);

struct GemmJob {
    uint32_t M = 0, N = 0, K = 0;
    const uint32_t* A = nullptr;
    size_t lda = 0;
    const uint32_t* B = nullptr;
    size_t ldb = 0;
    uint32_t* C = nullptr;
    size_t ldc = 0;
    int op = HME_SET;
};

// C_j op= A_j * B_j mod mp.p for every job (device pointers), in one split
// launch and one persistent tensor-core launch on ctx->stream; returns after
// the launches are enqueued and their host-side tables consumed.  K_j must fit
// one exact-accumulation chunk (limb_k_chunk).  bn_choice: the tile width,
// 0 wide (L * BN close to 256), 1 half-width, -1 wide unless the launch's
// wide tiles leave SMs idle.
void grouped_gemm_u32_device(hme_ctx* ctx, const ModParams& mp, const std::vector<GemmJob>& jobs,
                             int bn_choice = -1);
// The same products on the CUDA cores: one launch over every tile of every
// job (TILE x TILE tiles, tile 32 or 64), exact u64 accumulation; returns after
// the launch is enqueued and its tables are on the device.
void batch_simt_gemm_device(hme_ctx* ctx, const ModParams& mp, const std::vector<GemmJob>& jobs, int tile);

// A device matrix of a batch (rank jobs).
struct BatchMatrix {
    uint32_t* A = nullptr;
    size_t ld = 0;
    uint32_t m = 0, n = 0, p = 0;
    int rank_variant = 0;  // the schedule of its rank rounds (RankVariant)
};

// The schedules of a job's rank rounds: the trailing-update variant (the
// grouped tensor-core limb GEMM or the CUDA-core update) and the widest last
// panel (a job whose remaining columns fit it finishes in that one panel, on
// one CTA, with no trailing update; otherwise its rounds take 32 columns).
// Every schedule computes the same rank; only the time changes.
enum RankVariant {
    kRankTensorLast128 = 0,  // grouped limb GEMM, last panel up to 128 columns (the batch rule)
    kRankTensorLast32 = 1,   // grouped limb GEMM, 32-column rounds to the end
    kRankSimtLast128 = 2,    // CUDA-core update, last panel up to 128 columns
    kRankSimtLast32 = 3,     // CUDA-core update, 32-column rounds to the end
    kRankVariants = 4
};
inline int rank_variant_last(int v) { return v == kRankTensorLast32 || v == kRankSimtLast32 ? 32 : 128; }
inline bool rank_variant_simt(int v) { return v == kRankSimtLast128 || v == kRankSimtLast32; }

// ranks[j] = rank of mats[j] over F_p (destroys the matrices).
void batch_rank_device(hme_ctx* ctx, const std::vector<BatchMatrix>& mats, std::vector<int>& ranks);

// One seeded matrix of the job-stream generator.
struct GenSpec {
    uint32_t* dst = nullptr;
    size_t ld = 0;
    uint32_t rows = 0, cols = 0, p = 0;
    int family = 1;  // 0 banded sparse, 1 dense
    uint64_t seed = 0;
};
void gen_jobs_device(hme_ctx* ctx, const std::vector<GenSpec>& specs);

}  // namespace hme

// The grouped (many-shape) limb GEMM (grouped_gemm.cu).
#pragma once
#include <cstdint>
#include <vector>

#include "hme_internal.h"

namespace hme {

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
// one exact-accumulation chunk (limb_k_chunk).
void grouped_gemm_u32_device(hme_ctx* ctx, const ModParams& mp, const std::vector<GemmJob>& jobs);

// A device matrix of a batch (rank jobs).
struct BatchMatrix {
    uint32_t* A = nullptr;
    size_t ld = 0;
    uint32_t m = 0, n = 0, p = 0;
};

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

// The batched job stream: thousands of uneven products and ranks mod p.
//
// A job is C = A * B mod p (A m x k, B k x n) followed by rank(C) over F_p.  The
// reference runs such work one launch per job (engine::cuda::gemm,
// src/Cuda/cuda_kernels.cu:815) or one launch per SAME-shape batch
// (GemmBatch, cuda_kernels.cu:831-946), and computes ranks of p > 127 on the
// host (elim::column_rank_profile, src/ModArithmetic/DenseElim.h:160-169).
// Here every phase is one launch over all jobs:
//   GEMM: the grouped limb GEMM (grouped_gemm.cu), one launch per modulus;
//   rank: a round-based blocked LU over all jobs at once -- per round, one
//     CTA per job factors that job's next panel of columns in shared memory,
//     then batched kernels move the pivot rows up and solve the pivot rows'
//     trailing block, and ONE grouped limb GEMM applies every job's trailing
//     update.  A job leaves the rounds when its columns or rows run out.
// Also here: the seeded device generator of the config-4 stream's matrices.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <mutex>
#include <vector>

#include "hme_grouped.h"
#include "hme_internal.h"
#include "hme_ptx.cuh"

namespace hme {
namespace {

constexpr int kRankThreads = 1024;
constexpr int kMaxBw = 32;
constexpr int kRankSmem = 200 * 1024;

__device__ __forceinline__ uint64_t splitmix_at(uint64_t seed, uint64_t i) {
    // the i-th output (0-based) of splitmix64 seeded with `seed`
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ uint32_t inv_xgcd(uint32_t u, uint32_t q) {
    if (u == 0) return 0;
    uint32_t a = u, b = q, x1 = 1, x2 = 0;
    for (int it = 0; a != 1 && b != 1; ++it) {
        if (a == 0 || b == 0 || it > 128) return 0;
        while ((a & 1) == 0) {
            a >>= 1;
            x1 = (x1 & 1) ? static_cast<uint32_t>((static_cast<uint64_t>(x1) + q) >> 1) : x1 >> 1;
        }
        while ((b & 1) == 0) {
            b >>= 1;
            x2 = (x2 & 1) ? static_cast<uint32_t>((static_cast<uint64_t>(x2) + q) >> 1) : x2 >> 1;
        }
        if (a >= b) {
            a -= b;
            x1 = x1 >= x2 ? x1 - x2 : static_cast<uint32_t>(static_cast<uint64_t>(x1) + q - x2);
        } else {
            b -= a;
            x2 = x2 >= x1 ? x2 - x1 : static_cast<uint32_t>(static_cast<uint64_t>(x2) + q - x1);
        }
    }
    return a == 1 ? x1 : x2;
}


// ---- generator ----------------------------------------------------------------------
struct GenJob {
    uint32_t* dst;
    uint64_t ld;
    int rows, cols;
    uint32_t p;
    int family;     // 0 banded sparse (|i - j| <= 8, 5 % density, values in [-3, 3]), 1 dense uniform mod p
    uint64_t seed;  // element (r, c) is output r*cols + c of splitmix64(seed)
};

__global__ void gen_jobs_kernel(const GenJob* __restrict__ jobs) {
    const GenJob J = jobs[blockIdx.y];
    const size_t total = static_cast<size_t>(J.rows) * J.cols;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int r = static_cast<int>(idx / J.cols), c = static_cast<int>(idx % J.cols);
        const uint64_t z = splitmix_at(J.seed, idx);
        uint32_t v;
        if (J.family == 1) {
            v = static_cast<uint32_t>(z % J.p);
        } else {
            v = 0;
            if (abs(r - c) <= 8 && (z % 100) < 5) {
                const int w = static_cast<int>((z >> 32) % 7) - 3;
                v = w < 0 ? J.p - static_cast<uint32_t>(-w) : static_cast<uint32_t>(w);
            }
        }
        J.dst[static_cast<size_t>(r) * J.ld + c] = v;
    }
}

// ---- batched rank: per-round state ------------------------------------------------------
struct RankJob {
    uint32_t* A;   // m x n, ld (device), destroyed
    uint64_t ld;
    int m, n;
    uint32_t p;
    uint64_t barrett;
    int r0, c0, w;  // active rows [r0, m), panel columns [c0, c0 + w)
    int slot;       // index of the job's output slot
};

struct RankOut {
    int k;
    int pivot_rows[kMaxBw];
    int pivot_cols[kMaxBw];
};

// One CTA per job: factor the panel A[r0:m, c0:c0+w) in shared memory (field
// elimination, pivot = the topmost active row with a non-zero; pivot rows stay
// in place and leave the active set; multipliers are stored in the pivot
// columns), then write the panel back.
__global__ void __launch_bounds__(kRankThreads) batch_panel_kernel(const RankJob* __restrict__ jobs,
                                                                   RankOut* __restrict__ outs) {
    extern __shared__ uint32_t sp[];  // rows x w panel, then flags
    __shared__ int s_piv;
    __shared__ uint32_t s_prow[kMaxBw];
    __shared__ uint32_t s_inv;
    __shared__ int s_k;
    const RankJob J = jobs[blockIdx.x];
    const int rows = J.m - J.r0, w = J.w;
    unsigned char* isp = reinterpret_cast<unsigned char*>(sp + static_cast<size_t>(rows) * w);
    for (int idx = threadIdx.x; idx < rows * w; idx += blockDim.x) {
        const int i = idx / w, j = idx % w;
        sp[idx] = J.A[static_cast<size_t>(J.r0 + i) * J.ld + J.c0 + j];
    }
    for (int i = threadIdx.x; i < rows; i += blockDim.x) isp[i] = 0;
    if (threadIdx.x == 0) s_k = 0;
    __syncthreads();
    for (int jc = 0; jc < w; ++jc) {
        if (threadIdx.x == 0) s_piv = INT_MAX;
        __syncthreads();
        for (int i = threadIdx.x; i < rows; i += blockDim.x)
            if (!isp[i] && sp[i * w + jc] != 0) atomicMin(&s_piv, i);
        __syncthreads();
        const int pr = s_piv;
        if (pr == INT_MAX) continue;
        for (int j = threadIdx.x; j < w; j += blockDim.x) s_prow[j] = sp[pr * w + j];
        if (threadIdx.x == 0) {
            isp[pr] = 1;
            s_inv = inv_xgcd(sp[pr * w + jc], J.p);
            RankOut& o = outs[J.slot];
            o.pivot_rows[s_k] = J.r0 + pr;
            o.pivot_cols[s_k] = J.c0 + jc;
            ++s_k;
        }
        __syncthreads();
        const uint32_t inv = s_inv;
        const int width = w - jc - 1;
        // multipliers, then the (row, column) updates
        for (int i = threadIdx.x; i < rows; i += blockDim.x) {
            if (isp[i]) continue;
            const uint32_t x = sp[i * w + jc];
            if (x != 0) sp[i * w + jc] = mod_mul(x, inv, J.p, J.barrett);
        }
        __syncthreads();
        if (width > 0) {
            for (int e = threadIdx.x; e < rows * width; e += blockDim.x) {
                const int i = e / width, j = jc + 1 + e % width;
                if (isp[i]) continue;
                const uint32_t l = sp[i * w + jc];
                if (l == 0) continue;
                sp[i * w + j] = mod_sub(sp[i * w + j], mod_mul(l, s_prow[j], J.p, J.barrett), J.p);
            }
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < rows * w; idx += blockDim.x) {
        const int i = idx / w, j = idx % w;
        J.A[static_cast<size_t>(J.r0 + i) * J.ld + J.c0 + j] = sp[idx];
    }
    if (threadIdx.x == 0) outs[J.slot].k = s_k;
}

// Row permutation of columns [c0, n) for rows [r0, m): pivot rows first (in
// pivot order), then the other rows in order.  Per job a permutation segment
// in `perm` (absolute row indices) and a scratch segment in `tmp`.
struct PermJob {
    uint32_t* A;
    uint64_t ld;
    int r0, rows, c0, cols;
    const int* perm;
    uint32_t* tmp;
};
__global__ void batch_gather_rows_kernel(const PermJob* __restrict__ jobs) {
    const PermJob J = jobs[blockIdx.y];
    const size_t total = static_cast<size_t>(J.rows) * J.cols;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(idx / J.cols), j = static_cast<int>(idx % J.cols);
        J.tmp[idx] = J.A[static_cast<size_t>(J.perm[i]) * J.ld + J.c0 + j];
    }
}
__global__ void batch_scatter_rows_kernel(const PermJob* __restrict__ jobs) {
    const PermJob J = jobs[blockIdx.y];
    const size_t total = static_cast<size_t>(J.rows) * J.cols;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(idx / J.cols), j = static_cast<int>(idx % J.cols);
        J.A[static_cast<size_t>(J.r0 + i) * J.ld + J.c0 + j] = J.tmp[idx];
    }
}

// U12 = L11^-1 A12 (unit lower L11 from the pivot rows' multipliers at the
// pivot columns; one thread per trailing column), and L21 gathered into a
// compact buffer for the grouped GEMM.
struct SolveJob {
    uint32_t* A;
    uint64_t ld;
    int r0, k, m, c1, ntrail;
    uint32_t p;
    uint64_t barrett;
    int pcols[kMaxBw];
    uint32_t* L21;  // (m - r0 - k) x k
};
__global__ void batch_trsm_kernel(const SolveJob* __restrict__ jobs) {
    __shared__ uint32_t sL[kMaxBw * kMaxBw];
    const SolveJob& J = jobs[blockIdx.y];
    const int k = J.k;
    for (int idx = threadIdx.x; idx < k * k; idx += blockDim.x) {
        const int t = idx / k, s = idx % k;
        sL[idx] = s < t ? J.A[static_cast<size_t>(J.r0 + t) * J.ld + J.pcols[s]] : 0u;
    }
    __syncthreads();
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < J.ntrail; j += gridDim.x * blockDim.x) {
        uint32_t* col = J.A + static_cast<size_t>(J.r0) * J.ld + J.c1 + j;
        for (int t = 1; t < k; ++t) {
            uint32_t sub = 0;
            for (int s = 0; s < t; ++s) {
                const uint32_t l = sL[t * k + s];
                if (l) sub = mod_add(sub, mod_mul(l, col[static_cast<size_t>(s) * J.ld], J.p, J.barrett), J.p);
            }
            uint32_t* x = col + static_cast<size_t>(t) * J.ld;
            *x = mod_sub(*x, sub, J.p);
        }
    }
}
__global__ void batch_gather_l21_kernel(const SolveJob* __restrict__ jobs) {
    const SolveJob& J = jobs[blockIdx.y];
    const int below = J.m - J.r0 - J.k;
    const size_t total = static_cast<size_t>(below) * J.k;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(idx / J.k), t = static_cast<int>(idx % J.k);
        J.L21[idx] = J.A[static_cast<size_t>(J.r0 + J.k + i) * J.ld + J.pcols[t]];
    }
}

size_t a256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

// ---------------------------------------------------------------------------------------
void batch_rank_device(hme_ctx* ctx, const std::vector<BatchMatrix>& mats, std::vector<int>& ranks) {
    static std::once_flag once;
    std::call_once(once, [] {
        cudaFuncSetAttribute(batch_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kRankSmem);
    });
    const int nj = static_cast<int>(mats.size());
    ranks.assign(nj, 0);
    std::vector<RankJob> st(nj);
    for (int j = 0; j < nj; ++j) {
        const BatchMatrix& M = mats[j];
        HME_REQUIRE(is_prime_u32(M.p), "batch rank: every modulus must be prime");
        RankJob& J = st[j];
        J.A = M.A;
        J.ld = M.ld;
        J.m = static_cast<int>(M.m);
        J.n = static_cast<int>(M.n);
        J.p = M.p;
        J.barrett = make_mod(M.p).barrett;
        J.r0 = 0;
        J.c0 = 0;
        // the panel (m - r0) x w must fit shared memory
        const int wmax = static_cast<int>(std::min<size_t>(kMaxBw, (kRankSmem - 4096) / (5 * std::max<size_t>(1, M.m))));
        HME_REQUIRE(wmax >= 1, "batch rank: matrix too tall for the shared-memory panel");
        J.w = wmax;
        J.slot = j;
    }
    RankOut* d_out = static_cast<RankOut*>(ctx->ws.get(kSlotJobs2, sizeof(RankOut) * static_cast<size_t>(nj) + 256));
    std::vector<RankOut> h_out(nj);
    std::vector<int> active;
    for (int j = 0; j < nj; ++j)
        if (st[j].m > 0 && st[j].n > 0) active.push_back(j);
    while (!active.empty()) {
        // (1) panels of every active job
        std::vector<RankJob> round;
        round.reserve(active.size());
        size_t max_smem = 0;
        for (int j : active) {
            RankJob J = st[j];
            J.w = std::min(J.w, J.n - J.c0);
            round.push_back(J);
            max_smem = std::max(max_smem, static_cast<size_t>(J.m - J.r0) * J.w * 4 + (J.m - J.r0) + 16);
        }
        RankJob* d_jobs = static_cast<RankJob*>(ctx->ws.get(kSlotJobs3, sizeof(RankJob) * round.size() + 256));
        HME_CUDA(cudaMemcpyAsync(d_jobs, round.data(), sizeof(RankJob) * round.size(), cudaMemcpyHostToDevice,
                                 ctx->stream));
        HME_TIMED(ctx, "batch_panel", batch_panel_kernel<<<static_cast<int>(round.size()), kRankThreads, max_smem,
                                                           ctx->stream>>>(d_jobs, d_out));
        HME_CUDA(cudaGetLastError());
        HME_CUDA(cudaMemcpyAsync(h_out.data(), d_out, sizeof(RankOut) * nj, cudaMemcpyDeviceToHost, ctx->stream));
        HME_CUDA(cudaStreamSynchronize(ctx->stream));
        // (2) row permutations, (3) solves, (4) trailing updates, per job with pivots
        std::vector<PermJob> perms;
        std::vector<int> perm_rows;
        std::vector<SolveJob> solves;
        size_t tmp_elems = 0, l21_elems = 0;
        std::vector<size_t> tmp_off, perm_off, l21_off;
        for (const RankJob& J : round) {
            const RankOut& o = h_out[J.slot];
            if (o.k == 0) continue;
            const int rows = J.m - J.r0, cols = J.n - J.c0;
            // pivot rows first, in pivot order; skipped when they already are
            bool identity = true;
            for (int t = 0; t < o.k; ++t) identity = identity && o.pivot_rows[t] == J.r0 + t;
            PermJob pj{};
            pj.A = J.A;
            pj.ld = J.ld;
            pj.r0 = J.r0;
            pj.rows = identity ? 0 : rows;
            pj.c0 = J.c0;
            pj.cols = cols;
            perm_off.push_back(perm_rows.size());
            tmp_off.push_back(tmp_elems);
            if (!identity) {
                std::vector<char> isp(rows, 0);
                for (int t = 0; t < o.k; ++t) {
                    perm_rows.push_back(o.pivot_rows[t]);
                    isp[o.pivot_rows[t] - J.r0] = 1;
                }
                for (int i = 0; i < rows; ++i)
                    if (!isp[i]) perm_rows.push_back(J.r0 + i);
                tmp_elems += a256(static_cast<size_t>(rows) * cols);
            }
            perms.push_back(pj);
            SolveJob sj{};
            sj.A = J.A;
            sj.ld = J.ld;
            sj.r0 = J.r0;
            sj.k = o.k;
            sj.m = J.m;
            sj.c1 = J.c0 + J.w;
            sj.ntrail = J.n - sj.c1;
            sj.p = J.p;
            sj.barrett = J.barrett;
            for (int t = 0; t < o.k; ++t) sj.pcols[t] = o.pivot_cols[t];
            solves.push_back(sj);
            l21_off.push_back(l21_elems);
            l21_elems += a256(static_cast<size_t>(J.m - J.r0 - o.k) * o.k);
        }
        if (!perms.empty()) {
            const int np = static_cast<int>(perms.size());
            int* d_perm = static_cast<int*>(ctx->ws.get(kSlotJobs4, sizeof(int) * perm_rows.size() + 256));
            uint32_t* d_tmp = static_cast<uint32_t*>(ctx->ws.get(kSlotJobs5, sizeof(uint32_t) * tmp_elems + 256));
            uint32_t* d_l21 = static_cast<uint32_t*>(ctx->ws.get(kSlotJobs6, sizeof(uint32_t) * l21_elems + 256));
            for (int t = 0; t < np; ++t) {
                perms[t].perm = d_perm + perm_off[t];
                perms[t].tmp = d_tmp + tmp_off[t];
                solves[t].L21 = d_l21 + l21_off[t];
            }
            uint8_t* tab = static_cast<uint8_t*>(ctx->ws.get(kSlotJobs7, a256(sizeof(PermJob) * np) + a256(sizeof(SolveJob) * np)));
            PermJob* d_pj = reinterpret_cast<PermJob*>(tab);
            SolveJob* d_sj = reinterpret_cast<SolveJob*>(tab + a256(sizeof(PermJob) * np));
            if (!perm_rows.empty())
                HME_CUDA(cudaMemcpyAsync(d_perm, perm_rows.data(), sizeof(int) * perm_rows.size(),
                                         cudaMemcpyHostToDevice, ctx->stream));
            HME_CUDA(cudaMemcpyAsync(d_pj, perms.data(), sizeof(PermJob) * np, cudaMemcpyHostToDevice, ctx->stream));
            HME_CUDA(cudaMemcpyAsync(d_sj, solves.data(), sizeof(SolveJob) * np, cudaMemcpyHostToDevice, ctx->stream));
            // grid.y = job (<= 65535 per launch: chunked)
            for (int b0 = 0; b0 < np; b0 += 65535) {
                const int nb = std::min(65535, np - b0);
                const dim3 g(32, nb);
                HME_TIMED(ctx, "batch_permute", batch_gather_rows_kernel<<<g, 256, 0, ctx->stream>>>(d_pj + b0));
                HME_TIMED(ctx, "batch_permute", batch_scatter_rows_kernel<<<g, 256, 0, ctx->stream>>>(d_pj + b0));
                HME_TIMED(ctx, "batch_trsm", batch_trsm_kernel<<<dim3(8, nb), 128, 0, ctx->stream>>>(d_sj + b0));
                HME_TIMED(ctx, "batch_gather", batch_gather_l21_kernel<<<dim3(16, nb), 256, 0, ctx->stream>>>(d_sj + b0));
            }
            HME_CUDA(cudaGetLastError());
            // one grouped GEMM per modulus: A22 -= L21 * U12
            std::vector<uint32_t> mods;
            for (const SolveJob& sj : solves)
                if (std::find(mods.begin(), mods.end(), sj.p) == mods.end()) mods.push_back(sj.p);
            for (uint32_t p : mods) {
                std::vector<GemmJob> gj;
                for (int t = 0; t < np; ++t) {
                    const SolveJob& sj = solves[t];
                    if (sj.p != p) continue;
                    const int below = sj.m - sj.r0 - sj.k;
                    if (below <= 0 || sj.ntrail <= 0) continue;
                    GemmJob g;
                    g.M = below;
                    g.N = sj.ntrail;
                    g.K = sj.k;
                    g.A = sj.L21;
                    g.lda = sj.k;
                    g.B = sj.A + static_cast<size_t>(sj.r0) * sj.ld + sj.c1;
                    g.ldb = sj.ld;
                    g.C = sj.A + static_cast<size_t>(sj.r0 + sj.k) * sj.ld + sj.c1;
                    g.ldc = sj.ld;
                    g.op = HME_SUB;
                    gj.push_back(g);
                }
                if (!gj.empty()) grouped_gemm_u32_device(ctx, make_mod(p), gj);
            }
        }
        // (5) advance
        std::vector<int> next;
        for (const RankJob& J : round) {
            RankJob& S = st[J.slot];
            const int k = h_out[J.slot].k;
            S.r0 += k;
            S.c0 += J.w;
            if (S.r0 < S.m && S.c0 < S.n) next.push_back(J.slot);
        }
        active.swap(next);
    }
    check_device_error(ctx);
    for (int j = 0; j < nj; ++j) ranks[j] = st[j].r0;
}

void gen_jobs_device(hme_ctx* ctx, const std::vector<GenSpec>& specs) {
    if (specs.empty()) return;
    std::vector<GenJob> g(specs.size());
    for (size_t t = 0; t < specs.size(); ++t) {
        g[t].dst = specs[t].dst;
        g[t].ld = specs[t].ld;
        g[t].rows = static_cast<int>(specs[t].rows);
        g[t].cols = static_cast<int>(specs[t].cols);
        g[t].p = specs[t].p;
        g[t].family = specs[t].family;
        g[t].seed = specs[t].seed;
    }
    GenJob* d = static_cast<GenJob*>(ctx->ws.get(kSlotJobs3, sizeof(GenJob) * g.size() + 256));
    HME_CUDA(cudaMemcpyAsync(d, g.data(), sizeof(GenJob) * g.size(), cudaMemcpyHostToDevice, ctx->stream));
    for (size_t b0 = 0; b0 < g.size(); b0 += 65535) {
        const int nb = static_cast<int>(std::min<size_t>(65535, g.size() - b0));
        HME_TIMED(ctx, "gen_jobs", gen_jobs_kernel<<<dim3(16, nb), 256, 0, ctx->stream>>>(d + b0));
    }
    HME_CUDA(cudaGetLastError());
    HME_CUDA(cudaStreamSynchronize(ctx->stream));
}

}  // namespace hme

// ---- C ABI ----------------------------------------------------------------------------
using namespace hme;

namespace {
void check_job(const hme_job& j) {
    HME_REQUIRE(j.p >= 2, "job: modulus must be >= 2");
    HME_REQUIRE(j.m == 0 || j.n == 0 || (j.C && j.ldc >= j.n), "job: bad C");
    HME_REQUIRE(j.k == 0 || j.m == 0 || j.n == 0 || (j.A && j.B && j.lda >= j.k && j.ldb >= j.n), "job: bad A / B");
}

void batch_gemm(hme_ctx* ctx, uint32_t njobs, const hme_job* jobs) {
    // one grouped launch per modulus; a K beyond the exact-accumulation chunk takes the single-job path
    std::vector<uint32_t> mods;
    for (uint32_t t = 0; t < njobs; ++t) {
        check_job(jobs[t]);
        if (std::find(mods.begin(), mods.end(), jobs[t].p) == mods.end()) mods.push_back(jobs[t].p);
    }
    for (uint32_t p : mods) {
        const ModParams mp = make_mod(p);
        std::vector<GemmJob> g;
        for (uint32_t t = 0; t < njobs; ++t) {
            const hme_job& j = jobs[t];
            if (j.p != p || j.m == 0 || j.n == 0) continue;
            if (j.k == 0 || j.k > limb_k_chunk(mp.limbs)) {
                gemm_u32_device(ctx, mp, j.m, j.n, j.k, j.A, j.lda, j.B, j.ldb, j.C, j.ldc, HME_SET);
                continue;
            }
            GemmJob x;
            x.M = j.m;
            x.N = j.n;
            x.K = j.k;
            x.A = j.A;
            x.lda = j.lda;
            x.B = j.B;
            x.ldb = j.ldb;
            x.C = j.C;
            x.ldc = j.ldc;
            x.op = HME_SET;
            g.push_back(x);
        }
        grouped_gemm_u32_device(ctx, mp, g);
    }
}

void batch_rank(hme_ctx* ctx, uint32_t njobs, const hme_job* jobs, uint32_t* ranks) {
    std::vector<BatchMatrix> mats(njobs);
    for (uint32_t t = 0; t < njobs; ++t) {
        mats[t].A = jobs[t].C;
        mats[t].ld = jobs[t].ldc;
        mats[t].m = jobs[t].m;
        mats[t].n = jobs[t].n;
        mats[t].p = jobs[t].p;
    }
    std::vector<int> r;
    batch_rank_device(ctx, mats, r);
    for (uint32_t t = 0; t < njobs; ++t) ranks[t] = static_cast<uint32_t>(r[t]);
}
}  // namespace

extern "C" {

int hme_batch_gemm_u32_dev(hme_ctx* ctx, uint32_t njobs, const hme_job* jobs) {
    return guard([&] {
        HME_REQUIRE(ctx && (njobs == 0 || jobs), "null argument");
        bind(ctx);
        batch_gemm(ctx, njobs, jobs);
        check_device_error(ctx);
    });
}

int hme_batch_rank_u32_dev(hme_ctx* ctx, uint32_t njobs, const hme_job* jobs, uint32_t* ranks) {
    return guard([&] {
        HME_REQUIRE(ctx && (njobs == 0 || (jobs && ranks)), "null argument");
        bind(ctx);
        batch_rank(ctx, njobs, jobs, ranks);
    });
}

int hme_batch_gemm_rank_u32_dev(hme_ctx* ctx, uint32_t njobs, const hme_job* jobs, uint32_t* ranks) {
    return guard([&] {
        HME_REQUIRE(ctx && (njobs == 0 || (jobs && ranks)), "null argument");
        bind(ctx);
        batch_gemm(ctx, njobs, jobs);
        batch_rank(ctx, njobs, jobs, ranks);
    });
}

int hme_gen_jobs_u32_dev(hme_ctx* ctx, uint32_t nmat, const hme_gen_spec* specs) {
    return guard([&] {
        HME_REQUIRE(ctx && (nmat == 0 || specs), "null argument");
        bind(ctx);
        std::vector<GenSpec> g(nmat);
        for (uint32_t t = 0; t < nmat; ++t) {
            HME_REQUIRE(specs[t].dst && specs[t].ld >= specs[t].cols && specs[t].p >= 2, "gen: bad spec");
            g[t].dst = specs[t].dst;
            g[t].ld = specs[t].ld;
            g[t].rows = specs[t].rows;
            g[t].cols = specs[t].cols;
            g[t].p = specs[t].p;
            g[t].family = specs[t].family;
            g[t].seed = specs[t].seed;
        }
        gen_jobs_device(ctx, g);
    });
}

}  // extern "C"

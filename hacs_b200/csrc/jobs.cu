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

#include "hme_elim.h"
#include "hme_grouped.h"
#include "hme_internal.h"
#include "hme_ptx.cuh"

namespace hme {
namespace {

constexpr int kMaxBw = 128;   // panel columns per round (at most: a job's last panel)
constexpr int kRoundBw = 32;  // panel columns of the rounds before a job's last panel
constexpr int kRankSmem = 200 * 1024;

__device__ __forceinline__ uint64_t splitmix_at(uint64_t seed, uint64_t i) {
    // the i-th output (0-based) of splitmix64 seeded with `seed`
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
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
    uint32_t qinv;  // p odd: -p^-1 mod 2^32 (Montgomery)
    uint32_t r2;    // p odd: 2^64 mod p
    int r0, c0, w;  // active rows [r0, m), panel columns [c0, c0 + w)
    int slot;       // the job's index
    int out;        // its output slot in this round (its position in the round's table)
};

struct RankOut {
    int k;
    int pivot_rows[kMaxBw];
    int pivot_cols[kMaxBw];
};

// One CTA per job: factor the panel A[r0:m, c0:c0+w) in shared memory over
// F_p (pivot = the topmost active row with a non-zero; pivot rows stay in place
// and leave the active set; multipliers are stored in the pivot columns), then
// write the panel back.  The panel is column-major in shared memory, rows over
// consecutive threads (g threads per row).  Row updates are fraction-free:
// row <- (w row - x pivot_row) * rho, w the pivot (rho = 2^-32 with one
// Montgomery reduction per element for odd p < 2^31, else rho = 1), so no
// column needs a modular inverse; every active row takes the same unit
// factor w rho per pivot, and the panel is brought back to the classical
// values once at the end (multipliers times w_t^-1, every other entry times
// the inverse of the scale in force when the row left the active set or the
// column was passed).  One CTA barrier per column: the candidate of column
// c + 1 collects in a triple-buffered slot.
__device__ __forceinline__ uint32_t batch_ff_update(bool mont, uint32_t w, uint32_t y, uint32_t xn, uint32_t pr,
                                                    const RankJob& J) {
    if (mont) {
        const uint64_t t = static_cast<uint64_t>(w) * y + static_cast<uint64_t>(xn) * pr;  // < 2^63
        const uint32_t mq = static_cast<uint32_t>(t) * J.qinv;
        const uint32_t r = static_cast<uint32_t>((t + static_cast<uint64_t>(mq) * J.p) >> 32);
        return r >= J.p ? r - J.p : r;
    }
    return mod_add(mod_mul(w, y, J.p, J.barrett), mod_mul(xn, pr, J.p, J.barrett), J.p);
}

template <int NT>
__global__ void __launch_bounds__(NT) batch_panel_kernel(const RankJob* __restrict__ jobs, RankOut* __restrict__ outs,
                                                         int* err) {
    extern __shared__ uint32_t sp[];  // [w][rs] column-major panel, then a step byte per row
    __shared__ int s_cand[3];
    __shared__ uint32_t s_w[kMaxBw], s_inv[kMaxBw], s_sinv[kMaxBw + 1];
    __shared__ int s_colstep[kMaxBw], s_prow[kMaxBw], s_pcol[kMaxBw];
    const RankJob J = jobs[blockIdx.x];
    const int rows = J.m - J.r0, w = J.w, rs = rows | 1;
    uint32_t* S = sp;
    unsigned char* s_step = reinterpret_cast<unsigned char*>(S + static_cast<size_t>(w) * rs);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = NT / 32;
    constexpr int NONE = INT_MAX;
    int lg = 0;
    while ((1 << lg) < rows) ++lg;
    if ((1 << lg) > NT) {  // the host never launches this; uniform for the CTA
        if (tid == 0) atomicCAS(err, 0, DERR_LAUNCH_SHAPE);
        return;
    }
    const int nslots = 1 << lg, g = NT >> lg;
    const int li = tid & (nslots - 1), sub = tid >> lg;
    const bool has_row = li < rows;
    const bool mont = (J.p & 1u) && J.p < (1u << 31);

    for (int r = warp; r < rows; r += NW) {
        const uint32_t* src = J.A + static_cast<size_t>(J.r0 + r) * J.ld + J.c0;
        for (int j = lane; j < w; j += 32) S[j * rs + r] = src[j];
    }
    for (int i = tid; i < rows; i += NT) s_step[i] = 0;
    if (tid < 3) s_cand[tid] = NONE;
    __syncthreads();
    {
        int key = (has_row && sub == 0 && S[li] != 0) ? li : NONE;
        key = __reduce_min_sync(0xffffffffu, key);
        if (lane == 0 && key != NONE) atomicMin(&s_cand[0], key);
    }
    __syncthreads();
    int k = 0;
    for (int it = 0; it < w; ++it) {
        const int cur = it % 3, nxt = (it + 1) % 3;
        const int piv = s_cand[cur];
        if (tid == 0) s_cand[(it + 2) % 3] = NONE;  // last read in step it - 1, next written in step it + 1
        int key = NONE;
        if (piv == NONE) {
            if (tid == 0) s_colstep[it] = -1 - k;
            if (it + 1 < w && has_row && sub == 0 && s_step[li] == 0 && S[(it + 1) * rs + li] != 0) key = li;
        } else {
            const uint32_t wt = S[it * rs + piv];
            if (tid == 0) {
                s_w[k] = wt;
                s_colstep[it] = k;
                s_prow[k] = piv;
                s_pcol[k] = it;
                s_step[piv] = static_cast<unsigned char>(k + 1);
            }
            if (has_row && li != piv && s_step[li] == 0) {
                const uint32_t xp = S[it * rs + li];
                const uint32_t xn = xp == 0 ? 0u : J.p - xp;
                for (int j = it + 1 + sub; j < w; j += g) {
                    const uint32_t y = batch_ff_update(mont, wt, S[j * rs + li], xn, S[j * rs + piv], J);
                    S[j * rs + li] = y;
                    if (j == it + 1 && y != 0) key = li;
                }
            }
            ++k;
        }
        key = __reduce_min_sync(0xffffffffu, key);
        if (lane == 0 && key != NONE) atomicMin(&s_cand[nxt], key);
        __syncthreads();
    }
    // ---- classical values back: w_t^-1 and the prefix products of (w_s rho)^-1
    for (int t = tid; t < k; t += NT) {
        // Fermat: w^(p-2) mod p (p prime)
        uint32_t b = s_w[t], e = J.p - 2, r = 1u % J.p;
        while (e) {
            if (e & 1u) r = mod_mul(r, b, J.p, J.barrett);
            b = mod_mul(b, b, J.p, J.barrett);
            e >>= 1;
        }
        s_inv[t] = r;
    }
    __syncthreads();
    if (warp == 0) {
        // exclusive prefix products of f_t = w_t^-1 rho^-1, four consecutive t per lane
        const uint32_t one = 1u % J.p;
        const uint32_t rinv = mont ? static_cast<uint32_t>((1ull << 32) % J.p) : one;  // rho^-1
        constexpr int per = kMaxBw / 32;
        uint32_t f[per];
        uint32_t run = one;
#pragma unroll
        for (int e = 0; e < per; ++e) {
            const int t = lane * per + e;
            f[e] = t < k ? mod_mul(s_inv[t], rinv, J.p, J.barrett) : one;
            run = mod_mul(run, f[e], J.p, J.barrett);
        }
        uint32_t incl = run;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl = mod_mul(incl, y, J.p, J.barrett);
        }
        uint32_t ex = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) ex = one;
#pragma unroll
        for (int e = 0; e < per; ++e) {
            s_sinv[lane * per + e] = ex;
            ex = mod_mul(ex, f[e], J.p, J.barrett);
        }
        if (lane == 31) s_sinv[kMaxBw] = ex;
    }
    __syncthreads();
    if (has_row) {
        const int st = s_step[li];
        const int tau = st ? st - 1 : k;
        const uint32_t sc = s_sinv[tau];
        for (int j = sub; j < w; j += g) {
            const int t = s_colstep[j];
            const uint32_t f = t >= 0 ? (t < tau ? s_inv[t] : sc) : s_sinv[min(tau, -1 - t)];
            S[j * rs + li] = mod_mul(S[j * rs + li], f, J.p, J.barrett);
        }
    }
    __syncthreads();
    for (int r = warp; r < rows; r += NW) {
        uint32_t* dst = J.A + static_cast<size_t>(J.r0 + r) * J.ld + J.c0;
        for (int j = lane; j < w; j += 32) dst[j] = S[j * rs + r];
    }
    if (tid == 0) {
        RankOut& o = outs[J.out];
        for (int t = 0; t < k; ++t) {
            o.pivot_rows[t] = J.r0 + s_prow[t];
            o.pivot_cols[t] = J.c0 + s_pcol[t];
        }
        o.k = k;
    }
}

// Row moves of columns [c0, n): the pivot rows go to rows r0 .. r0+k-1 by
// swaps (a rank needs no particular order of the other rows), so at most 2k
// rows move: row dst[i] receives the old row src[i].  Per job a segment of the
// src / dst lists and a scratch segment in `tmp`.
struct PermJob {
    uint32_t* A;
    uint64_t ld;
    int rows, c0, cols;  // rows = rows that move
    const int* src;
    const int* dst;
    uint32_t* tmp;
};
__global__ void batch_gather_rows_kernel(const PermJob* __restrict__ jobs) {
    const PermJob J = jobs[blockIdx.y];
    const size_t total = static_cast<size_t>(J.rows) * J.cols;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(idx / J.cols), j = static_cast<int>(idx % J.cols);
        J.tmp[idx] = J.A[static_cast<size_t>(J.src[i]) * J.ld + J.c0 + j];
    }
}
__global__ void batch_scatter_rows_kernel(const PermJob* __restrict__ jobs) {
    const PermJob J = jobs[blockIdx.y];
    const size_t total = static_cast<size_t>(J.rows) * J.cols;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(idx / J.cols), j = static_cast<int>(idx % J.cols);
        J.A[static_cast<size_t>(J.dst[i]) * J.ld + J.c0 + j] = J.tmp[idx];
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
    const int* pcols;  // the panel's pivot columns (in the device copy of the panel's output)
    uint32_t* L21;     // (m - r0 - k) x k
    uint32_t* Linv;    // k x k: L11^-1
    uint32_t kmax;     // products a 64-bit sum starting below p holds before a reduction
};
// U12 = L11^-1 A12 for every job with a pivot block, in two launches:
// batch_linv_kernel, one CTA per job: L11^-1 column by column (forward
// substitution on e_j, one warp per column, lane l holding rows l, l+32, ...;
// at step t row t is final and a shuffle broadcasts it), into the job's slot;
// batch_apply_kernel, one CTA per (job, 32 trailing columns): the product
// L11^-1 A12 with lane = column and warps over rows, each output a dot
// product accumulated in 64 bits and reduced once per kmax products -- no
// sequential dependency, so no idle lanes.
constexpr int kBatchTrsmCols = 32;
size_t batch_linv_smem(int k) { return sizeof(uint32_t) * static_cast<size_t>(k) * (k | 1); }
size_t batch_apply_smem(int k) {
    return sizeof(uint32_t) * (static_cast<size_t>(k) * (k | 1) + static_cast<size_t>(k) * (kBatchTrsmCols + 1));
}

__global__ void __launch_bounds__(256) batch_linv_kernel(const SolveJob* __restrict__ jobs) {
    extern __shared__ uint32_t smem_bl[];
    const SolveJob& J = jobs[blockIdx.x];
    const int k = J.k;
    if (k < 2 || J.ntrail <= 0) return;  // the test is the same for the whole CTA
    const int ls = k | 1;
    uint32_t* sL = smem_bl;
    for (int idx = threadIdx.x; idx < k * k; idx += blockDim.x) {
        const int t = idx / k, s = idx % k;
        sL[t * ls + s] = s < t ? J.A[static_cast<size_t>(J.r0 + t) * J.ld + J.pcols[s]] : 0u;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    constexpr int per = kMaxBw / 32;
    for (int j = warp; j < k; j += nw) {
        uint32_t x[per];
#pragma unroll
        for (int q = 0; q < per; ++q) x[q] = (lane + 32 * q == j) ? 1u % J.p : 0u;
#pragma unroll
        for (int qt = 0; qt < per; ++qt) {
            if (32 * qt >= k - 1) break;
            if (32 * qt + 31 < j) continue;  // rows above j stay zero
            for (int tt = 0; tt < 32; ++tt) {
                const int t = 32 * qt + tt;
                if (t >= k - 1) break;
                if (t < j) continue;
                const uint32_t xt = __shfl_sync(0xffffffffu, x[qt], tt);
#pragma unroll
                for (int q = qt; q < per; ++q) {
                    const int r = lane + 32 * q;
                    if (r > t && r < k) {
                        const uint32_t l = sL[r * ls + t];
                        if (l) x[q] = reduce_u64(static_cast<uint64_t>(J.p - l) * xt + x[q], J.p, J.barrett);
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < per; ++q) {
            const int r = lane + 32 * q;
            if (r < k) J.Linv[static_cast<size_t>(r) * k + j] = x[q];
        }
    }
}

__global__ void __launch_bounds__(256) batch_apply_kernel(const SolveJob* __restrict__ jobs) {
    extern __shared__ uint32_t smem_ba[];
    const SolveJob& J = jobs[blockIdx.y];
    const int k = J.k;
    // nothing to solve, or no columns for this CTA: the test is the same for the whole CTA
    if (k < 2 || static_cast<int>(blockIdx.x) * kBatchTrsmCols >= J.ntrail) return;
    const int ls = k | 1;
    constexpr int xs = kBatchTrsmCols + 1;
    uint32_t* Li = smem_ba;
    uint32_t* X = smem_ba + k * ls;
    for (int idx = threadIdx.x; idx < k * k; idx += blockDim.x) {
        const int r = idx / k, s = idx - r * k;
        Li[r * ls + s] = J.Linv[idx];
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int c0 = blockIdx.x * kBatchTrsmCols; c0 < J.ntrail; c0 += gridDim.x * kBatchTrsmCols) {
        const int nc = min(kBatchTrsmCols, J.ntrail - c0);
        __syncthreads();  // Li ready / the previous tile consumed
        for (int idx = threadIdx.x; idx < k * kBatchTrsmCols; idx += blockDim.x) {
            const int r = idx / kBatchTrsmCols, c = idx % kBatchTrsmCols;
            if (c < nc) X[r * xs + c] = J.A[static_cast<size_t>(J.r0 + r) * J.ld + J.c1 + c0 + c];
        }
        __syncthreads();
        if (lane < nc) {
            for (int r = warp; r < k; r += nw) {
                uint64_t acc = X[r * xs + lane];  // the unit diagonal
                uint32_t cnt = 0;
                const uint32_t* lr = Li + r * ls;
                for (int s = 0; s < r; ++s) {
                    acc += static_cast<uint64_t>(lr[s]) * X[s * xs + lane];
                    if (++cnt == J.kmax) {
                        acc = reduce_u64(acc, J.p, J.barrett);
                        cnt = 0;
                    }
                }
                J.A[static_cast<size_t>(J.r0 + r) * J.ld + J.c1 + c0 + lane] = reduce_u64(acc, J.p, J.barrett);
            }
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
        cudaFuncSetAttribute(batch_panel_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRankSmem);
        cudaFuncSetAttribute(batch_panel_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRankSmem);
        cudaFuncSetAttribute(batch_panel_kernel<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRankSmem);
        cudaFuncSetAttribute(batch_panel_kernel<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRankSmem);
        cudaFuncSetAttribute(batch_linv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(batch_linv_smem(kMaxBw)));
        cudaFuncSetAttribute(batch_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(batch_apply_smem(kMaxBw)));
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
        if (M.p & 1u) {
            uint32_t x = M.p;  // p^-1 mod 2^32 by Newton's iteration
            for (int i = 0; i < 5; ++i) x *= 2u - M.p * x;
            J.qinv = 0u - x;
            J.r2 = static_cast<uint32_t>((static_cast<unsigned __int128>(1) << 64) % M.p);
        }
        J.r0 = 0;
        J.c0 = 0;
        // the panel (m - r0) x w must fit shared memory
        J.w = 0;  // set per round from the active rows
        J.slot = j;
    }
    RankOut* d_out = static_cast<RankOut*>(ctx->ws.get(kSlotJobs2, sizeof(RankOut) * static_cast<size_t>(nj) + 256));
    // the per-round panel outputs come back into pinned host memory (up to ~1 KB per job)
    struct PinnedOut {
        RankOut* p = nullptr;
        ~PinnedOut() {
            if (p) cudaFreeHost(p);
        }
    } pinned;
    HME_CUDA(cudaMallocHost(reinterpret_cast<void**>(&pinned.p), sizeof(RankOut) * std::max(1, nj)));
    RankOut* h_out = pinned.p;
    std::vector<int> scratch_content, scratch_where;
    std::vector<int> active;
    for (int j = 0; j < nj; ++j)
        if (st[j].m > 1024 && st[j].n > 0) {
            // taller than one panel CTA holds: the single-matrix elimination (cluster / grid panels)
            ElimOptions o = ctx->elim;
            const ElimResult r = elim_device(ctx, make_mod(st[j].p), st[j].A, st[j].ld, st[j].m, st[j].n, false,
                                             nullptr, 0, o);
            st[j].r0 = r.rank;
        } else if (st[j].m > 0 && st[j].n > 0) {
            active.push_back(j);
        }
    while (!active.empty()) {
        // (1) panels of every active job, in buckets of active rows: each bucket
        // launches with the threads and shared memory its largest panel needs
        constexpr int kBuckets = 4;
        constexpr int bucket_threads[kBuckets] = {128, 256, 512, 1024};
        auto bucket_of = [&](int rows) { return rows <= 64 ? 0 : rows <= 128 ? 1 : rows <= 256 ? 2 : 3; };
        std::vector<RankJob> round;
        round.reserve(active.size());
        int bcount[kBuckets] = {0, 0, 0, 0};
        size_t bsmem[kBuckets] = {0, 0, 0, 0};
        for (int j : active) {
            RankJob J = st[j];
            const int rows = J.m - J.r0;
            // the job's remaining columns in one last panel when they fit the shared memory
            // (up to kMaxBw: no trailing update at all), else a kRoundBw-column panel (a
            // wider one would grow the CUDA-core panel and pivot-block solve work, which
            // scale with the width, faster than it saves trailing-update traffic)
            const size_t wfit = (kRankSmem - static_cast<size_t>(rows) - 16) / (sizeof(uint32_t) * (rows | 1));
            const size_t left = static_cast<size_t>(J.n - J.c0);
            J.w = static_cast<int>(left <= std::min<size_t>(kMaxBw, wfit) ? left
                                                                          : std::min<size_t>(kRoundBw, wfit));
            HME_REQUIRE(J.w >= 1 && rows <= 1024, "batch rank: matrix too tall for the shared-memory panel");
            const int b = bucket_of(rows);
            ++bcount[b];
            bsmem[b] = std::max(bsmem[b], sizeof(uint32_t) * static_cast<size_t>(J.w) * (rows | 1) + rows + 16);
            round.push_back(J);
        }
        std::stable_sort(round.begin(), round.end(), [&](const RankJob& x, const RankJob& y) {
            return bucket_of(x.m - x.r0) < bucket_of(y.m - y.r0);
        });
        for (size_t t = 0; t < round.size(); ++t) round[t].out = static_cast<int>(t);
        RankJob* d_jobs = static_cast<RankJob*>(ctx->ws.get(kSlotJobs3, sizeof(RankJob) * round.size() + 256));
        HME_CUDA(cudaMemcpyAsync(d_jobs, round.data(), sizeof(RankJob) * round.size(), cudaMemcpyHostToDevice,
                                 ctx->stream));
        for (int b = 0, off = 0; b < kBuckets; off += bcount[b], ++b) {
            if (!bcount[b]) continue;
            const RankJob* dj = d_jobs + off;
            switch (bucket_threads[b]) {
                case 128: HME_TIMED(ctx, "batch_panel", batch_panel_kernel<128><<<bcount[b], 128, bsmem[b], ctx->stream>>>(dj, d_out, ctx->d_err)); break;
                case 256: HME_TIMED(ctx, "batch_panel", batch_panel_kernel<256><<<bcount[b], 256, bsmem[b], ctx->stream>>>(dj, d_out, ctx->d_err)); break;
                case 512: HME_TIMED(ctx, "batch_panel", batch_panel_kernel<512><<<bcount[b], 512, bsmem[b], ctx->stream>>>(dj, d_out, ctx->d_err)); break;
                default: HME_TIMED(ctx, "batch_panel", batch_panel_kernel<1024><<<bcount[b], 1024, bsmem[b], ctx->stream>>>(dj, d_out, ctx->d_err)); break;
            }
            HME_CUDA(cudaGetLastError());
        }
        HME_CUDA(cudaMemcpyAsync(h_out, d_out, sizeof(RankOut) * round.size(), cudaMemcpyDeviceToHost,
                                 ctx->stream));
        HME_CUDA(cudaStreamSynchronize(ctx->stream));
        // (2) row permutations, (3) solves, (4) trailing updates, per job with pivots
        std::vector<PermJob> perms;
        std::vector<int> perm_rows, perm_dst;
        std::vector<SolveJob> solves;
        size_t tmp_elems = 0, l21_elems = 0;
        std::vector<size_t> tmp_off, perm_off, l21_off, linv_off;
        size_t linv_elems = 0;
        for (const RankJob& J : round) {
            const RankOut& o = h_out[J.out];
            // no pivots, or the job's last panel (no columns right of it): nothing to move or update
            if (o.k == 0 || J.c0 + J.w >= J.n) continue;
            const int rows = J.m - J.r0, cols = J.n - J.c0;
            // the pivot rows to r0 .. r0+k-1 by swaps; only rows whose content changes move
            PermJob pj{};
            pj.A = J.A;
            pj.ld = J.ld;
            pj.c0 = J.c0;
            pj.cols = cols;
            perm_off.push_back(perm_rows.size());
            tmp_off.push_back(tmp_elems);
            {
                // content[pos] = original row now at pos; where[orig] = its position (touched rows only)
                std::vector<int>& content = scratch_content;
                std::vector<int>& where = scratch_where;
                content.resize(rows);
                where.resize(rows);
                for (int t = 0; t < o.k; ++t) {
                    const int a = t, b0 = o.pivot_rows[t] - J.r0;
                    content[a] = a;
                    where[a] = a;
                    content[b0] = b0;
                    where[b0] = b0;
                }
                for (int t = 0; t < o.k; ++t) {
                    const int a = t, b = where[o.pivot_rows[t] - J.r0];
                    if (a == b) continue;
                    const int ca = content[a], cb = content[b];
                    content[a] = cb;
                    content[b] = ca;
                    where[cb] = a;
                    where[ca] = b;
                }
                int moved = 0;
                std::vector<int> touched;
                for (int t = 0; t < o.k; ++t) {
                    touched.push_back(t);
                    touched.push_back(o.pivot_rows[t] - J.r0);
                }
                std::sort(touched.begin(), touched.end());
                touched.erase(std::unique(touched.begin(), touched.end()), touched.end());
                for (int pos : touched)
                    if (content[pos] != pos) {
                        perm_rows.push_back(J.r0 + content[pos]);  // src
                        perm_dst.push_back(J.r0 + pos);             // dst
                        ++moved;
                    }
                pj.rows = moved;
                if (moved) tmp_elems += a256(static_cast<size_t>(moved) * cols);
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
            sj.pcols = d_out[J.out].pivot_cols;
            {
                const uint64_t d = static_cast<uint64_t>(J.p - 1) * (J.p - 1);
                const uint64_t km = d == 0 ? (1u << 20) : (~0ull - (J.p - 1)) / d;
                sj.kmax = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(km, 1u << 20)));
            }
            solves.push_back(sj);
            l21_off.push_back(l21_elems);
            l21_elems += a256(static_cast<size_t>(J.m - J.r0 - o.k) * o.k);
            linv_off.push_back(linv_elems);
            linv_elems += a256(static_cast<size_t>(o.k) * o.k);
        }
        if (!perms.empty()) {
            const int np = static_cast<int>(perms.size());
            int* d_perm = static_cast<int*>(ctx->ws.get(kSlotJobs4, 2 * sizeof(int) * perm_rows.size() + 256));
            int* d_dst = d_perm + perm_rows.size();
            uint32_t* d_tmp = static_cast<uint32_t*>(ctx->ws.get(kSlotJobs5, sizeof(uint32_t) * tmp_elems + 256));
            uint32_t* d_l21 = static_cast<uint32_t*>(ctx->ws.get(kSlotJobs6, sizeof(uint32_t) * l21_elems + 256));
            uint32_t* d_linv = static_cast<uint32_t*>(ctx->ws.get(kSlotJobs8, sizeof(uint32_t) * linv_elems + 256));
            for (int t = 0; t < np; ++t) {
                perms[t].src = d_perm + perm_off[t];
                perms[t].dst = d_dst + perm_off[t];
                perms[t].tmp = d_tmp + tmp_off[t];
                solves[t].L21 = d_l21 + l21_off[t];
                solves[t].Linv = d_linv + linv_off[t];
            }
            uint8_t* tab = static_cast<uint8_t*>(ctx->ws.get(kSlotJobs7, a256(sizeof(PermJob) * np) + a256(sizeof(SolveJob) * np)));
            PermJob* d_pj = reinterpret_cast<PermJob*>(tab);
            SolveJob* d_sj = reinterpret_cast<SolveJob*>(tab + a256(sizeof(PermJob) * np));
            if (!perm_rows.empty()) {
                perm_rows.insert(perm_rows.end(), perm_dst.begin(), perm_dst.end());
                HME_CUDA(cudaMemcpyAsync(d_perm, perm_rows.data(), sizeof(int) * perm_rows.size(),
                                         cudaMemcpyHostToDevice, ctx->stream));
            }
            HME_CUDA(cudaMemcpyAsync(d_pj, perms.data(), sizeof(PermJob) * np, cudaMemcpyHostToDevice, ctx->stream));
            HME_CUDA(cudaMemcpyAsync(d_sj, solves.data(), sizeof(SolveJob) * np, cudaMemcpyHostToDevice, ctx->stream));
            int kmax = 1;
            for (const SolveJob& sj : solves) kmax = std::max(kmax, sj.k);
            const size_t linv_smem = batch_linv_smem(kmax), apply_smem = batch_apply_smem(kmax);
            // grid.y = job (<= 65535 per launch: chunked)
            for (int b0 = 0; b0 < np; b0 += 65535) {
                const int nb = std::min(65535, np - b0);
                const dim3 g(32, nb);
                HME_TIMED(ctx, "batch_permute", batch_gather_rows_kernel<<<g, 256, 0, ctx->stream>>>(d_pj + b0));
                HME_TIMED(ctx, "batch_permute", batch_scatter_rows_kernel<<<g, 256, 0, ctx->stream>>>(d_pj + b0));
                HME_TIMED(ctx, "batch_trsm", batch_linv_kernel<<<nb, 256, linv_smem, ctx->stream>>>(d_sj + b0));
                HME_TIMED(ctx, "batch_trsm", batch_apply_kernel<<<dim3(32, nb), 256, apply_smem, ctx->stream>>>(d_sj + b0));
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
            const int k = h_out[J.out].k;
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

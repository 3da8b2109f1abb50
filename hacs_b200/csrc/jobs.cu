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
//     trailing block, and ONE grouped limb GEMM per modulus applies every
//     job's trailing update.  A job leaves the rounds when its columns or rows
//     run out.  The rounds are planned on the device (bucket lists, row moves,
//     solve entries, GEMM tile tables), so a round is a fixed launch sequence:
//     it is captured once in a CUDA graph and replayed, with no host round trip
//     between rounds.
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

// Per-job state of the device-driven rounds: the job's RankJob (r0, c0 and the
// round's w advance on the device) and its fixed buffers.
struct RankDev {
    RankJob J;
    int active;
    int group;            // modulus group
    int a_row0, b_col0;   // the job's rows / columns in its group's stacked plane tensors
    uint32_t* L21;        // m x 32: L21 of the round (ld = k)
    uint32_t* Linv;       // 32 x 32: L11^-1 of the round
    uint32_t* tmp;        // 64 x n: rows in flight during the row moves
    int* mv;              // 64 sources, then 64 destinations
    uint32_t kmax;        // delayed-reduction bound of p
    int last_max;         // the job's schedule: the widest last panel (columns; 32 or kMaxBw)
    int simt;             // the job's schedule: 1 = CUDA-core trailing update, 0 = the grouped limb GEMM
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
__global__ void __launch_bounds__(NT) batch_panel_kernel(const RankDev* __restrict__ devs,
                                                         const int* __restrict__ list, const int* __restrict__ count,
                                                         RankOut* __restrict__ outs, int* err) {
    extern __shared__ uint32_t sp[];  // [w][rs] column-major panel, then a step byte per row
    __shared__ int s_cand[3];
    __shared__ uint32_t s_w[kMaxBw], s_inv[kMaxBw], s_sinv[kMaxBw + 1];
    __shared__ int s_colstep[kMaxBw], s_prow[kMaxBw], s_pcol[kMaxBw];
    const int njobs = *count;
    for (int ji = blockIdx.x; ji < njobs; ji += gridDim.x) {
    __syncthreads();  // the previous job's shared state is no longer read
    const RankJob J = devs[list[ji]].J;
    const int rows = J.m - J.r0, w = J.w, rs = rows | 1;
    uint32_t* S = sp;
    unsigned char* s_step = reinterpret_cast<unsigned char*>(S + static_cast<size_t>(w) * rs);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = NT / 32;
    constexpr int NONE = INT_MAX;
    int lg = 0;
    while ((1 << lg) < rows) ++lg;
    if ((1 << lg) > NT) {  // the planner never lists this; uniform for the CTA
        if (tid == 0) atomicCAS(err, 0, DERR_LAUNCH_SHAPE);
        continue;
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
    }  // jobs of this CTA
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
    int simt;          // the trailing update A22 -= L21 U12 on CUDA cores (batch_simt_update_kernel)
    int simt_base;     // the job's first entry in the round's CUDA-core tile list
};
// U12 = L11^-1 A12 for every job with a pivot block, in two launches:
// batch_linv_kernel, one CTA per job: L11^-1 column by column (forward
// substitution on e_j, one warp per column, lane l holding rows l, l+32, ...;
// at step t row t is final and a shuffle broadcasts it), into the job's slot;
// batch_apply_kernel, one CTA per (job, 32 trailing columns): the product
// L11^-1 A12 with lane = column and warps over rows, each output an exact
// dot product in a 96-bit sum reduced once -- no sequential dependency, so no
// idle lanes.
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
    const SolveJob J = jobs[blockIdx.y];
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
                // the unit diagonal's term, then r exact products in a 96-bit sum, one reduction
                uint32_t a0 = X[r * xs + lane], a1 = 0, a2 = 0;
                const uint32_t* lr = Li + r * ls;
                for (int s = 0; s < r; ++s) mac96(a0, a1, a2, lr[s], X[s * xs + lane]);
                const uint64_t h = reduce_u64((static_cast<uint64_t>(a2) << 32) | a1, J.p, J.barrett);
                J.A[static_cast<size_t>(J.r0 + r) * J.ld + J.c1 + c0 + lane] =
                    reduce_u64((h << 32) | a0, J.p, J.barrett);
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

// The CUDA-core trailing update, for the jobs whose schedule takes it
// (SolveJob::simt): A22 -= L21 U12 mod p with L21 the compact (below x k)
// gather and U12 the pivot rows' trailing columns, k <= kRoundBw.  The work
// is a list of 64 x 64 tiles of A22 built by rank_post_kernel (each job
// appends its tiles; tile_job[t] = the job, t - simt_base its tile in row-major
// tile order), taken by a persistent grid, so a large job's tiles spread over
// the whole GPU and the launch has no idle CTAs for jobs on the other
// schedule.  A CTA copies the next tile's L21 rows and U12 columns into its
// second shared-memory buffer (cp.async) while it multiplies the current
// tile's, loads the current tile's old A22 values before the multiply-adds,
// and gives each thread 4 x 4 outputs (rows ty + 16a, columns tx + 16b,
// so a half warp writes 16 consecutive words of a row); each output is an
// exact dot product reduced once: a 64-bit sum when kRoundBw (p - 1)^2 fits
// 64 bits (one wide multiply-add per product), else a 96-bit sum
// (mad.lo.cc / madc.hi.cc / addc).  No limb planes, no split, no tensor map.
constexpr int kSimtTile = 64;
__host__ __device__ inline int simt_tiles(int rows, int cols) {
    return ((rows + kSimtTile - 1) / kSimtTile) * ((cols + kSimtTile - 1) / kSimtTile);
}
__global__ void __launch_bounds__(256, 2) batch_simt_update_kernel(const SolveJob* __restrict__ jobs,
                                                                   const int* __restrict__ tile_job,
                                                                   const int* __restrict__ count) {
    // two operand buffers: tile t's L21 rows / U12 columns are consumed while tile t + gridDim.x's are copied
    __shared__ uint32_t sL[2][kSimtTile][kRoundBw + 1];
    __shared__ uint32_t sU[2][kRoundBw][kSimtTile];
    const int total = *count;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    // the job of tile t and the tile's first row / column in the job's trailing block
    auto locate = [&](int t, int& i0, int& j0) -> const SolveJob& {
        const SolveJob& J = jobs[tile_job[t]];
        const int tc = (J.ntrail + kSimtTile - 1) / kSimtTile, local = t - J.simt_base;
        i0 = (local / tc) * kSimtTile;
        j0 = (local % tc) * kSimtTile;
        return J;
    };
    // tile t's operands into buffer b as one asynchronous copy group (zero-filled outside the block)
    auto stage = [&](int t, int b) {
        int i0, j0;
        const SolveJob& J = locate(t, i0, j0);
        const int k = J.k, below = J.m - J.r0 - k;
        const uint32_t* U = J.A + static_cast<size_t>(J.r0) * J.ld + J.c1;
        for (int idx = threadIdx.x; idx < kSimtTile * k; idx += blockDim.x) {
            const int i = idx / k, s = idx - i * k;
            const bool v = i0 + i < below;
            cp_async4(&sL[b][i][s], v ? J.L21 + static_cast<size_t>(i0 + i) * k + s : J.L21, v);
        }
        for (int idx = threadIdx.x; idx < k * kSimtTile; idx += blockDim.x) {
            const int s = idx / kSimtTile, j = idx % kSimtTile;
            const bool v = j0 + j < J.ntrail;
            cp_async4(&sU[b][s][j], v ? U + static_cast<size_t>(s) * J.ld + j0 + j : U, v);
        }
        cp_async_commit();
    };
    if (static_cast<int>(blockIdx.x) < total) stage(blockIdx.x, 0);
    int it = 0;
    for (int t = blockIdx.x; t < total; t += gridDim.x, ++it) {  // t is the same for the whole CTA
        const int b = it & 1;
        // the next tile's copies start now (an empty group when there is none, so the wait below
        // always leaves exactly the newest group in flight)
        if (t + static_cast<int>(gridDim.x) < total) stage(t + gridDim.x, b ^ 1);
        else cp_async_commit();
        int i0, j0;
        const SolveJob& J = locate(t, i0, j0);
        const int k = J.k, below = J.m - J.r0 - k;
        uint32_t* A22 = J.A + static_cast<size_t>(J.r0 + k) * J.ld + J.c1;
        // the old A22 values, in flight during the wait and the multiply-adds
        uint32_t old[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int i = i0 + ty + 16 * a, j = j0 + tx + 16 * c;
                old[a][c] = (i < below && j < J.ntrail) ? A22[static_cast<size_t>(i) * J.ld + j] : 0u;
            }
        cp_async_wait<1>();
        __syncthreads();  // every thread's copies of this tile's operands have landed
        auto sub = [&](int a, int c, uint32_t d) {  // A22(i, j) = old - d mod p
            const int i = i0 + ty + 16 * a, j = j0 + tx + 16 * c;
            if (i >= below || j >= J.ntrail) return;
            const uint32_t x = old[a][c];
            A22[static_cast<size_t>(i) * J.ld + j] = x >= d ? x - d : x + (J.p - d);
        };
        const uint64_t pm1 = J.p - 1u;
        if (pm1 * pm1 <= ~0ull / kRoundBw) {
            // k <= kRoundBw products below (p - 1)^2 sum exactly in 64 bits: one wide multiply-add each
            uint64_t acc[4][4];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[a][c] = 0u;
            for (int s = 0; s < k; ++s) {
                uint32_t l[4], u[4];
#pragma unroll
                for (int a = 0; a < 4; ++a) l[a] = sL[b][ty + 16 * a][s];
#pragma unroll
                for (int c = 0; c < 4; ++c) u[c] = sU[b][s][tx + 16 * c];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int c = 0; c < 4; ++c) acc[a][c] += static_cast<uint64_t>(l[a]) * u[c];
            }
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int c = 0; c < 4; ++c) sub(a, c, reduce_u64(acc[a][c], J.p, J.barrett));
        } else {
            uint32_t a0[4][4], a1[4][4], a2[4][4];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int c = 0; c < 4; ++c) a0[a][c] = a1[a][c] = a2[a][c] = 0u;
            for (int s = 0; s < k; ++s) {
                uint32_t l[4], u[4];
#pragma unroll
                for (int a = 0; a < 4; ++a) l[a] = sL[b][ty + 16 * a][s];
#pragma unroll
                for (int c = 0; c < 4; ++c) u[c] = sU[b][s][tx + 16 * c];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int c = 0; c < 4; ++c) mac96(a0[a][c], a1[a][c], a2[a][c], l[a], u[c]);
            }
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const uint64_t h =
                        reduce_u64((static_cast<uint64_t>(a2[a][c]) << 32) | a1[a][c], J.p, J.barrett);
                    sub(a, c, reduce_u64((h << 32) | a0[a][c], J.p, J.barrett));
                }
        }
        __syncthreads();  // buffer b is consumed before the next iteration copies into it
    }
    cp_async_wait<0>();  // no copy outlives the kernel
}

size_t a256(size_t x) { return (x + 255) / 256 * 256; }

// ---- device-driven rounds ----------------------------------------------------------------
// A modulus group: its jobs are the contiguous range [begin, end) of the job
// arrays; one grouped split + GEMM launch per round reads its tables.
struct RankGroup {
    const CUtensorMap* tmA;  // stacked A planes of the group: {32, sum_m, L}
    const CUtensorMap* tmB;  // stacked B planes: {32, sum_n, L, L}
    uint8_t* planesA;
    uint8_t* planesB;
    uint64_t sum_m, sum_n;
    int bn;                  // grouped GEMM tile width
    int begin, end;
    int* tile_prob;          // per tile: the job (index within the group)
    int* block_job;          // per split block: the job (index within the group)
    int* totals;             // [0] tiles, [1] split blocks of the round
};

constexpr int kRowClasses = 4;
constexpr int kBuckets2 = 2 * kRowClasses;  // row class x {a 32-column round, a job's last panel}
__host__ __device__ inline int row_class(int rows) { return rows <= 64 ? 0 : rows <= 128 ? 1 : rows <= 256 ? 2 : 3; }
__host__ __device__ inline int row_class_max(int c) { return c == 0 ? 64 : c == 1 ? 128 : c == 2 ? 256 : 1024; }
__host__ __device__ inline int row_class_threads(int c) { return c == 0 ? 128 : c == 1 ? 256 : c == 2 ? 512 : 1024; }

// Each active job: the round's panel width (its remaining columns in one last
// panel when they fit the shared memory, else kRoundBw) and its bucket.
__global__ void rank_plan_kernel(RankDev* __restrict__ devs, int nj, int* __restrict__ lists,
                                 int* __restrict__ counters) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nj; j += gridDim.x * blockDim.x) {
        RankDev& D = devs[j];
        if (!D.active) continue;
        const int rows = D.J.m - D.J.r0, left = D.J.n - D.J.c0;
        const int wfit = (kRankSmem - rows - 16) / (4 * (rows | 1));
        const bool last = left <= min(D.last_max, wfit);
        D.J.w = last ? left : min(kRoundBw, wfit);
        const int b = row_class(rows) + (last ? kRowClasses : 0);
        const int idx = atomicAdd(&counters[b], 1);
        lists[static_cast<size_t>(b) * nj + idx] = j;
    }
}

// After the panels: each job's row moves, solve, L21 gather, split and GEMM
// entries of this round (empty when it has nothing to do), its tile and split
// block counts, and its advance to the next round.
__global__ void rank_post_kernel(RankDev* __restrict__ devs, int nj, const RankOut* __restrict__ outs,
                                 PermJob* __restrict__ perms, SolveJob* __restrict__ solves,
                                 GroupedProblem* __restrict__ gprob, GroupedSplitJob* __restrict__ gsplit,
                                 int* __restrict__ tiles, int* __restrict__ blocks,
                                 const RankGroup* __restrict__ groups, int* __restrict__ simt_tile_job,
                                 int* __restrict__ simt_count) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nj; j += gridDim.x * blockDim.x) {
        RankDev& D = devs[j];
        RankJob& J = D.J;
        PermJob& pj = perms[j];
        SolveJob& sj = solves[j];
        pj.rows = 0;
        sj.k = 0;
        sj.m = 0;
        sj.r0 = 0;
        sj.ntrail = 0;
        sj.simt = 0;
        tiles[j] = 0;
        blocks[j] = 0;
        if (!D.active) continue;
        const RankOut& o = outs[j];
        const int k = o.k;
        const int c1 = J.c0 + J.w;
        const int below = J.m - J.r0 - k, ntrail = J.n - c1;
        if (k > 0 && ntrail > 0 && below > 0) {
            // the pivot rows to r0 .. r0+k-1 by swaps: positions relative to r0,
            // touched[] holds (position, original row now there) pairs
            int pos[2 * kRoundBw], cont[2 * kRoundBw];
            int nt = 0;
            auto find = [&](int x) {
                for (int i = 0; i < nt; ++i)
                    if (pos[i] == x) return i;
                pos[nt] = x;
                cont[nt] = x;
                return nt++;
            };
            for (int t = 0; t < k; ++t) {
                const int a = find(t);
                const int orig = o.pivot_rows[t] - J.r0;
                int b = -1;  // the position now holding original row `orig`
                for (int i = 0; i < nt; ++i)
                    if (cont[i] == orig) b = i;
                if (b < 0) b = find(orig);  // untouched so far: still at its own position
                if (a != b) {
                    const int ca = cont[a];
                    cont[a] = cont[b];
                    cont[b] = ca;
                }
            }
            int moved = 0;
            for (int i = 0; i < nt; ++i)
                if (cont[i] != pos[i]) {
                    D.mv[moved] = J.r0 + cont[i];
                    D.mv[2 * kRoundBw + moved] = J.r0 + pos[i];
                    ++moved;
                }
            pj.A = J.A;
            pj.ld = J.ld;
            pj.rows = moved;
            pj.c0 = J.c0;
            pj.cols = J.n - J.c0;
            pj.src = D.mv;
            pj.dst = D.mv + 2 * kRoundBw;
            pj.tmp = D.tmp;
            // U12 = L11^-1 A12, L21, and A22 -= L21 U12
            sj.A = J.A;
            sj.ld = J.ld;
            sj.r0 = J.r0;
            sj.k = k;
            sj.m = J.m;
            sj.c1 = c1;
            sj.ntrail = ntrail;
            sj.p = J.p;
            sj.barrett = J.barrett;
            sj.pcols = o.pivot_cols;
            sj.L21 = D.L21;
            sj.Linv = D.Linv;
            sj.kmax = D.kmax;
            sj.simt = D.simt;
            if (D.simt) {  // the job's tiles join the round's CUDA-core tile list
                const int nt = simt_tiles(below, ntrail);
                const int base = atomicAdd(simt_count, nt);
                sj.simt_base = base;
                for (int i = 0; i < nt; ++i) simt_tile_job[base + i] = j;
            }
        }
        if (k > 0 && ntrail > 0 && below > 0 && !D.simt) {
            // the trailing update as the group's grouped limb GEMM: split and GEMM entries
            const RankGroup& G = groups[D.group];
            const int jl = j - G.begin;
            GroupedProblem& gp = gprob[j];
            gp.tmA = G.tmA;
            gp.tmB = G.tmB;
            gp.C = J.A + static_cast<size_t>(J.r0 + k) * J.ld + c1;
            gp.ldc = J.ld;
            gp.M = below;
            gp.N = ntrail;
            gp.kblocks = 1;
            gp.op = HME_SUB;
            gp.tiles_n = (ntrail + G.bn - 1) / G.bn;
            gp.a_row0 = D.a_row0;
            gp.b_col0 = D.b_col0;
            tiles[j] = ((below + limb::kBM - 1) / limb::kBM) * gp.tiles_n;
            GroupedSplitJob& gs = gsplit[j];
            limb::SplitArgs& sa = gs.s;
            sa.A = D.L21;
            sa.lda = static_cast<uint64_t>(k);
            sa.B = J.A + static_cast<size_t>(J.r0) * J.ld + c1;
            sa.ldb = J.ld;
            sa.M = below;
            sa.N = ntrail;
            sa.K = k;
            sa.Kp = 32;
            sa.p = J.p;
            sa.barrett = J.barrett;
            sa.planesA = G.planesA + static_cast<size_t>(D.a_row0) * 32;
            sa.planesB = G.planesB + static_cast<size_t>(D.b_col0) * 32;
            sa.a_plane = G.sum_m * 32;
            sa.b_plane = G.sum_n * 32;
            sa.a_blocks = min(64, max(1, (below * 2 + 255) / 256));
            sa.b_blocks_k = 1;
            sa.a_vec = (k & 3) == 0;
            gs.b_blocks = (ntrail + 31) / 32;
            blocks[j] = sa.a_blocks + gs.b_blocks;
            (void)jl;
        }
        J.r0 += k;
        J.c0 = c1;
        D.active = J.r0 < J.m && J.c0 < J.n;
    }
}

// Per group (one CTA each): exclusive prefix sums of the jobs' tile and block
// counts into the GEMM and split tables, and the totals.
__global__ void __launch_bounds__(1024) rank_scan_kernel(const RankGroup* __restrict__ groups,
                                                         const int* __restrict__ tiles,
                                                         const int* __restrict__ blocks,
                                                         GroupedProblem* __restrict__ gprob,
                                                         GroupedSplitJob* __restrict__ gsplit) {
    __shared__ int w_t[32], w_b[32];
    const RankGroup& G = groups[blockIdx.x];
    const int n = G.end - G.begin;
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int i0 = G.begin + static_cast<int>(threadIdx.x) * per;
    const int i1 = min(G.end, i0 + per);
    int st = 0, sb = 0;
    for (int i = i0; i < i1; ++i) {
        st += tiles[i];
        sb += blocks[i];
    }
    // exclusive scan of (st, sb) over the threads
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int it = st, ib = sb;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int yt = __shfl_up_sync(0xffffffffu, it, off), yb = __shfl_up_sync(0xffffffffu, ib, off);
        if (lane >= off) {
            it += yt;
            ib += yb;
        }
    }
    if (lane == 31) {
        w_t[warp] = it;
        w_b[warp] = ib;
    }
    __syncthreads();
    if (warp == 0) {
        int vt = lane < static_cast<int>(blockDim.x >> 5) ? w_t[lane] : 0;
        int vb = lane < static_cast<int>(blockDim.x >> 5) ? w_b[lane] : 0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int yt = __shfl_up_sync(0xffffffffu, vt, off), yb = __shfl_up_sync(0xffffffffu, vb, off);
            if (lane >= off) {
                vt += yt;
                vb += yb;
            }
        }
        w_t[lane] = vt;  // inclusive prefix over warps
        w_b[lane] = vb;
    }
    __syncthreads();
    int bt = it - st + (warp > 0 ? w_t[warp - 1] : 0);
    int bb = ib - sb + (warp > 0 ? w_b[warp - 1] : 0);
    for (int i = i0; i < i1; ++i) {
        gprob[i].tile_begin = bt;
        gsplit[i].block_begin = bb;
        bt += tiles[i];
        bb += blocks[i];
    }
    if (threadIdx.x == blockDim.x - 1) {
        G.totals[0] = bt;
        G.totals[1] = bb;
    }
}

// The per-tile problem and per-block job indexes of every group.
__global__ void rank_fill_kernel(const RankGroup* __restrict__ groups, const RankDev* __restrict__ devs, int nj,
                                 const int* __restrict__ tiles, const int* __restrict__ blocks,
                                 const GroupedProblem* __restrict__ gprob, const GroupedSplitJob* __restrict__ gsplit) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nj; j += gridDim.x * blockDim.x) {
        const RankGroup& G = groups[devs[j].group];
        const int jl = j - G.begin;
        for (int t = 0; t < tiles[j]; ++t) G.tile_prob[gprob[j].tile_begin + t] = jl;
        for (int b = 0; b < blocks[j]; ++b) G.block_job[gsplit[j].block_begin + b] = jl;
    }
}

}  // namespace

// ---------------------------------------------------------------------------------------
// Batched rank with the rounds planned on the device: per-job state and every
// buffer live at offsets fixed before the first round, and small kernels build
// each round's bucket lists, row moves, solve entries and grouped-GEMM tables,
// so a round is a fixed sequence of launches with no host round trip.  The
// sequence is captured once in a CUDA graph and replayed until every job can
// have finished (the widest job's column count / 32 + 2 rounds; jobs that are
// done drop out of every kernel at once).  With per-kernel timing on, the
// rounds are launched directly instead, so each launch gets its events.
void batch_rank_device(hme_ctx* ctx, const std::vector<BatchMatrix>& mats, std::vector<int>& ranks) {
    const int nj_all = static_cast<int>(mats.size());
    ranks.assign(nj_all, 0);
    // jobs taller than one panel CTA holds: the single-matrix elimination
    std::vector<int> order;
    order.reserve(nj_all);
    for (int j = 0; j < nj_all; ++j) {
        const BatchMatrix& M = mats[j];
        HME_REQUIRE(is_prime_u32(M.p), "batch rank: every modulus must be prime");
        if (M.m == 0 || M.n == 0) continue;
        if (M.m > 1024) {
            ElimOptions o = ctx->elim;
            const ElimResult r = elim_device(ctx, make_mod(M.p), M.A, M.ld, static_cast<int>(M.m),
                                             static_cast<int>(M.n), false, nullptr, 0, o);
            ranks[j] = r.rank;
        } else {
            order.push_back(j);
        }
    }
    if (order.empty()) return;
    // modulus groups: jobs sorted by modulus (stable)
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return mats[x].p < mats[y].p; });
    const int nj = static_cast<int>(order.size());
    std::vector<uint32_t> gmod;
    std::vector<int> gbegin;
    for (int i = 0; i < nj; ++i)
        if (i == 0 || mats[order[i]].p != mats[order[i - 1]].p) {
            gmod.push_back(mats[order[i]].p);
            gbegin.push_back(i);
        }
    const int ng = static_cast<int>(gmod.size());
    gbegin.push_back(nj);

    // ---- fixed layout: per-job state and buffers, per-group planes and tables
    std::vector<RankDev> devs(nj);
    std::vector<RankGroup> groups(ng);
    size_t buf_bytes = 0, plane_bytes = 0;
    std::vector<size_t> off_l21(nj), off_linv(nj), off_tmp(nj), off_mv(nj), g_planes(ng);
    std::vector<size_t> g_tiles(ng, 0), g_blocks(ng, 0);
    bool any_simt = false;
    size_t simt_cap = 0;  // CUDA-core tiles the round's list can hold: every such job's first-round tile count
    uint32_t max_n = 0;
    for (int g = 0; g < ng; ++g) {
        const ModParams mp = make_mod(gmod[g]);
        const int L = static_cast<int>(mp.limbs);
        uint64_t sm = 0, sn = 0;
        for (int i = gbegin[g]; i < gbegin[g + 1]; ++i) {
            const BatchMatrix& M = mats[order[i]];
            RankDev& D = devs[i];
            D = RankDev{};
            RankJob& J = D.J;
            J.A = M.A;
            J.ld = M.ld;
            J.m = static_cast<int>(M.m);
            J.n = static_cast<int>(M.n);
            J.p = M.p;
            J.barrett = mp.barrett;
            if (M.p & 1u) {
                uint32_t x = M.p;  // p^-1 mod 2^32 by Newton's iteration
                for (int t = 0; t < 5; ++t) x *= 2u - M.p * x;
                J.qinv = 0u - x;
                J.r2 = static_cast<uint32_t>((static_cast<unsigned __int128>(1) << 64) % M.p);
            }
            J.slot = i;
            J.out = i;
            D.active = 1;
            D.group = g;
            D.last_max = rank_variant_last(M.rank_variant);
            D.simt = rank_variant_simt(M.rank_variant) ? 1 : 0;
            if (D.simt) {
                any_simt = true;
                simt_cap += static_cast<size_t>(simt_tiles(static_cast<int>(M.m), static_cast<int>(M.n)));
            }
            max_n = std::max(max_n, M.n);
            D.a_row0 = static_cast<int>(sm);
            D.b_col0 = static_cast<int>(sn);
            sm += M.m;
            sn += M.n;
            {
                const uint64_t d = static_cast<uint64_t>(M.p - 1) * (M.p - 1);
                const uint64_t km = d == 0 ? (1u << 20) : (~0ull - (M.p - 1)) / d;
                D.kmax = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(km, 1u << 20)));
            }
            off_l21[i] = buf_bytes;
            buf_bytes += a256(sizeof(uint32_t) * M.m * kRoundBw);
            off_linv[i] = buf_bytes;
            buf_bytes += a256(sizeof(uint32_t) * kRoundBw * kRoundBw);
            off_tmp[i] = buf_bytes;
            buf_bytes += a256(sizeof(uint32_t) * 2 * kRoundBw * M.n);
            off_mv[i] = buf_bytes;
            buf_bytes += a256(sizeof(int) * 4 * kRoundBw);
            const int bn = grouped_bn_wide(L);
            g_tiles[g] += static_cast<size_t>((M.m + limb::kBM - 1) / limb::kBM) * ((M.n + bn - 1) / bn);
            g_blocks[g] += 64 + (M.n + 31) / 32;
        }
        RankGroup& G = groups[g];
        G.sum_m = sm;
        G.sum_n = sn;
        G.bn = grouped_bn_wide(L);
        G.begin = gbegin[g];
        G.end = gbegin[g + 1];
        g_planes[g] = plane_bytes;
        plane_bytes += a256(static_cast<size_t>(L) * sm * 32) + a256(static_cast<size_t>(L) * L * sn * 32);
    }
    // tables: states, outputs, entries, counts, lists, groups, tensor maps, indexes
    size_t tb = 0;
    auto take = [&](size_t bytes) {
        const size_t o = tb;
        tb += a256(bytes);
        return o;
    };
    const size_t o_devs = take(sizeof(RankDev) * nj), o_outs = take(sizeof(RankOut) * nj);
    const size_t o_perm = take(sizeof(PermJob) * nj), o_solve = take(sizeof(SolveJob) * nj);
    const size_t o_gprob = take(sizeof(GroupedProblem) * nj), o_gsplit = take(sizeof(GroupedSplitJob) * nj);
    const size_t o_tiles = take(sizeof(int) * nj), o_blocks = take(sizeof(int) * nj);
    const size_t o_lists = take(sizeof(int) * kBuckets2 * static_cast<size_t>(nj));
    const size_t o_counters = take(sizeof(int) * (kBuckets2 + 1));  // the buckets' counts, the CUDA-core tiles'
    const size_t o_simt = take(sizeof(int) * std::max<size_t>(1, simt_cap));
    const size_t o_groups = take(sizeof(RankGroup) * ng), o_maps = take(sizeof(CUtensorMap) * 2 * ng);
    const size_t o_totals = take(sizeof(int) * 2 * ng);
    std::vector<size_t> o_tp(ng), o_bj(ng);
    for (int g = 0; g < ng; ++g) {
        o_tp[g] = take(sizeof(int) * std::max<size_t>(1, g_tiles[g]));
        o_bj[g] = take(sizeof(int) * std::max<size_t>(1, g_blocks[g]));
    }
    uint8_t* tables = static_cast<uint8_t*>(ctx->ws.get(kSlotJobs1, tb));
    uint8_t* bufs = static_cast<uint8_t*>(ctx->ws.get(kSlotJobs4, std::max<size_t>(256, buf_bytes)));
    uint8_t* planes = static_cast<uint8_t*>(ctx->ws.get(kSlotJobs0, std::max<size_t>(256, plane_bytes)));
    RankDev* d_devs = reinterpret_cast<RankDev*>(tables + o_devs);
    RankOut* d_outs = reinterpret_cast<RankOut*>(tables + o_outs);
    PermJob* d_perm = reinterpret_cast<PermJob*>(tables + o_perm);
    SolveJob* d_solve = reinterpret_cast<SolveJob*>(tables + o_solve);
    GroupedProblem* d_gprob = reinterpret_cast<GroupedProblem*>(tables + o_gprob);
    GroupedSplitJob* d_gsplit = reinterpret_cast<GroupedSplitJob*>(tables + o_gsplit);
    int* d_tiles = reinterpret_cast<int*>(tables + o_tiles);
    int* d_blocks = reinterpret_cast<int*>(tables + o_blocks);
    int* d_lists = reinterpret_cast<int*>(tables + o_lists);
    int* d_counters = reinterpret_cast<int*>(tables + o_counters);
    int* d_simt_count = d_counters + kBuckets2;
    int* d_simt_tiles = reinterpret_cast<int*>(tables + o_simt);
    RankGroup* d_groups = reinterpret_cast<RankGroup*>(tables + o_groups);
    CUtensorMap* d_maps = reinterpret_cast<CUtensorMap*>(tables + o_maps);
    int* d_totals = reinterpret_cast<int*>(tables + o_totals);
    for (int i = 0; i < nj; ++i) {
        devs[i].L21 = reinterpret_cast<uint32_t*>(bufs + off_l21[i]);
        devs[i].Linv = reinterpret_cast<uint32_t*>(bufs + off_linv[i]);
        devs[i].tmp = reinterpret_cast<uint32_t*>(bufs + off_tmp[i]);
        devs[i].mv = reinterpret_cast<int*>(bufs + off_mv[i]);
    }
    std::vector<CUtensorMap> maps(2 * static_cast<size_t>(ng));
    for (int g = 0; g < ng; ++g) {
        RankGroup& G = groups[g];
        const int L = static_cast<int>(make_mod(gmod[g]).limbs);
        G.planesA = planes + g_planes[g];
        G.planesB = G.planesA + a256(static_cast<size_t>(L) * G.sum_m * 32);
        {
            const cuuint64_t dims[3] = {32, G.sum_m, static_cast<cuuint64_t>(L)};
            const cuuint64_t strides[2] = {32, 32 * G.sum_m};
            const cuuint32_t box[3] = {32, limb::kBM, 1};
            encode_tma_u8_kb(&maps[2 * g], G.planesA, 3, dims, strides, box, 32);
        }
        {
            const cuuint64_t dims[4] = {32, G.sum_n, static_cast<cuuint64_t>(L), static_cast<cuuint64_t>(L)};
            const cuuint64_t strides[3] = {32, 32 * G.sum_n, 32 * G.sum_n * L};
            const cuuint32_t box[4] = {32, static_cast<cuuint32_t>(G.bn), static_cast<cuuint32_t>(L), 1};
            encode_tma_u8_kb(&maps[2 * g + 1], G.planesB, 4, dims, strides, box, 32);
        }
        G.tmA = d_maps + 2 * g;
        G.tmB = d_maps + 2 * g + 1;
        G.tile_prob = reinterpret_cast<int*>(tables + o_tp[g]);
        G.block_job = reinterpret_cast<int*>(tables + o_bj[g]);
        G.totals = d_totals + 2 * g;
    }
    HME_CUDA(cudaMemcpyAsync(d_devs, devs.data(), sizeof(RankDev) * nj, cudaMemcpyHostToDevice, ctx->stream));
    HME_CUDA(cudaMemcpyAsync(d_groups, groups.data(), sizeof(RankGroup) * ng, cudaMemcpyHostToDevice, ctx->stream));
    HME_CUDA(cudaMemcpyAsync(d_maps, maps.data(), sizeof(CUtensorMap) * 2 * ng, cudaMemcpyHostToDevice, ctx->stream));

    // ---- launch shapes of a round (fixed)
    static OncePerDevice attr;
    attr.run([](int) {
        HME_CUDA(cudaFuncSetAttribute(batch_panel_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRankSmem));
        HME_CUDA(cudaFuncSetAttribute(batch_panel_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRankSmem));
        HME_CUDA(cudaFuncSetAttribute(batch_panel_kernel<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRankSmem));
        HME_CUDA(cudaFuncSetAttribute(batch_panel_kernel<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRankSmem));
        HME_CUDA(cudaFuncSetAttribute(batch_linv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(batch_linv_smem(kMaxBw))));
        HME_CUDA(cudaFuncSetAttribute(batch_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(batch_apply_smem(kMaxBw))));
    });
    size_t bucket_smem[kBuckets2];
    int bucket_grid[kBuckets2];
    for (int b = 0; b < kBuckets2; ++b) {
        const int c = b % kRowClasses, R = row_class_max(c);
        const size_t w = b < kRowClasses ? kRoundBw : kMaxBw;
        bucket_smem[b] = std::min<size_t>(kRankSmem, sizeof(uint32_t) * (R | 1) * w + R + 16);
        int occ = 1;
        const int nt = row_class_threads(c);
        switch (nt) {
            case 128: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_panel_kernel<128>, nt, bucket_smem[b]); break;
            case 256: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_panel_kernel<256>, nt, bucket_smem[b]); break;
            case 512: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_panel_kernel<512>, nt, bucket_smem[b]); break;
            default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_panel_kernel<1024>, nt, bucket_smem[b]); break;
        }
        bucket_grid[b] = std::max(1, std::min(nj, ctx->num_sms * std::max(1, occ)));
    }
    int simt_grid = 1;
    if (any_simt) {  // persistent: every resident CTA of the GPU, no more than the list can hold
        int occ = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_simt_update_kernel, 256, 0);
        simt_grid = static_cast<int>(std::max<size_t>(1, std::min<size_t>(simt_cap, static_cast<size_t>(ctx->num_sms) *
                                                                                      std::max(1, occ))));
    }
    // with per-kernel timing on, every launch stays on the context's stream (the timer's events are there)
    const bool fork = any_simt && !ctx->timer.on;
    struct EventPair {
        cudaEvent_t a = nullptr, b = nullptr;
        ~EventPair() {
            if (a) cudaEventDestroy(a);
            if (b) cudaEventDestroy(b);
        }
    } evs;
    if (fork) {
        if (!ctx->aux_stream) {
            int lo = 0, hi = 0;
            HME_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            HME_CUDA(cudaStreamCreateWithPriority(&ctx->aux_stream, cudaStreamNonBlocking, hi));
        }
        HME_CUDA(cudaEventCreateWithFlags(&evs.a, cudaEventDisableTiming));
        HME_CUDA(cudaEventCreateWithFlags(&evs.b, cudaEventDisableTiming));
    }
    const cudaEvent_t ev_fork = evs.a, ev_join = evs.b;
    HME_CUDA(cudaGetLastError());
    const size_t linv_smem = batch_linv_smem(kRoundBw), apply_smem = batch_apply_smem(kRoundBw);
    const int small_grid = std::max(1, std::min((nj + 255) / 256, ctx->num_sms * 8));
    auto round = [&]() {
        HME_CUDA(cudaMemsetAsync(d_counters, 0, sizeof(int) * (kBuckets2 + 1), ctx->stream));
        HME_TIMED(ctx, "rank_plan", rank_plan_kernel<<<small_grid, 256, 0, ctx->stream>>>(d_devs, nj, d_lists, d_counters));
        for (int b = 0; b < kBuckets2; ++b) {
            const int* list = d_lists + static_cast<size_t>(b) * nj;
            const int* cnt = d_counters + b;
            const int nt = row_class_threads(b % kRowClasses);
            switch (nt) {
                case 128: HME_TIMED(ctx, "batch_panel", batch_panel_kernel<128><<<bucket_grid[b], 128, bucket_smem[b], ctx->stream>>>(d_devs, list, cnt, d_outs, ctx->d_err)); break;
                case 256: HME_TIMED(ctx, "batch_panel", batch_panel_kernel<256><<<bucket_grid[b], 256, bucket_smem[b], ctx->stream>>>(d_devs, list, cnt, d_outs, ctx->d_err)); break;
                case 512: HME_TIMED(ctx, "batch_panel", batch_panel_kernel<512><<<bucket_grid[b], 512, bucket_smem[b], ctx->stream>>>(d_devs, list, cnt, d_outs, ctx->d_err)); break;
                default: HME_TIMED(ctx, "batch_panel", batch_panel_kernel<1024><<<bucket_grid[b], 1024, bucket_smem[b], ctx->stream>>>(d_devs, list, cnt, d_outs, ctx->d_err)); break;
            }
        }
        HME_TIMED(ctx, "rank_post", rank_post_kernel<<<small_grid, 256, 0, ctx->stream>>>(
                                         d_devs, nj, d_outs, d_perm, d_solve, d_gprob, d_gsplit, d_tiles, d_blocks, d_groups,
                                         d_simt_tiles, d_simt_count));
        HME_TIMED(ctx, "rank_post", rank_scan_kernel<<<ng, 1024, 0, ctx->stream>>>(d_groups, d_tiles, d_blocks, d_gprob,
                                                                                  d_gsplit));
        HME_TIMED(ctx, "rank_post", rank_fill_kernel<<<small_grid, 256, 0, ctx->stream>>>(d_groups, d_devs, nj, d_tiles,
                                                                                         d_blocks, d_gprob, d_gsplit));
        for (int b0 = 0; b0 < nj; b0 += 65535) {
            const int nb = std::min(65535, nj - b0);
            HME_TIMED(ctx, "batch_permute", batch_gather_rows_kernel<<<dim3(8, nb), 256, 0, ctx->stream>>>(d_perm + b0));
            HME_TIMED(ctx, "batch_permute", batch_scatter_rows_kernel<<<dim3(8, nb), 256, 0, ctx->stream>>>(d_perm + b0));
            HME_TIMED(ctx, "batch_trsm", batch_linv_kernel<<<nb, 256, linv_smem, ctx->stream>>>(d_solve + b0));
            HME_TIMED(ctx, "batch_trsm", batch_apply_kernel<<<dim3(32, nb), 256, apply_smem, ctx->stream>>>(d_solve + b0));
            HME_TIMED(ctx, "batch_gather", batch_gather_l21_kernel<<<dim3(8, nb), 256, 0, ctx->stream>>>(d_solve + b0));
        }
        if (fork) {
            // the CUDA-core updates on the second stream, beside the grouped split + GEMM of the other
            // jobs (disjoint jobs, so disjoint data); joined before the round ends
            HME_CUDA(cudaEventRecord(ev_fork, ctx->stream));
            HME_CUDA(cudaStreamWaitEvent(ctx->aux_stream, ev_fork, 0));
            batch_simt_update_kernel<<<simt_grid, 256, 0, ctx->aux_stream>>>(d_solve, d_simt_tiles, d_simt_count);
            ++ctx->launches;
            HME_CUDA(cudaEventRecord(ev_join, ctx->aux_stream));
        } else if (any_simt) {
            HME_TIMED(ctx, "batch_simt_update",
                      batch_simt_update_kernel<<<simt_grid, 256, 0, ctx->stream>>>(d_solve, d_simt_tiles, d_simt_count));
        }
        for (int g = 0; g < ng; ++g) {
            const RankGroup& G = groups[g];
            grouped_launch_device_tables(ctx, make_mod(gmod[g]), d_gsplit + G.begin, G.block_job, G.totals + 1,
                                         d_gprob + G.begin, G.tile_prob, G.totals);
        }
        if (fork) HME_CUDA(cudaStreamWaitEvent(ctx->stream, ev_join, 0));
        HME_CUDA(cudaGetLastError());
    };
    for (int g = 0; g < ng; ++g) grouped_prepare_device_tables(make_mod(gmod[g]).limbs);
    const int rounds = static_cast<int>((max_n + kRoundBw - 1) / kRoundBw) + 2;
    if (ctx->timer.on) {
        for (int r = 0; r < rounds; ++r) round();
    } else {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        HME_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        try {
            round();
        } catch (...) {
            cudaStreamEndCapture(ctx->stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        HME_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
        struct GraphGuard {
            cudaGraph_t g;
            cudaGraphExec_t* e;
            ~GraphGuard() {
                if (*e) cudaGraphExecDestroy(*e);
                if (g) cudaGraphDestroy(g);
            }
        } guard{graph, &exec};
        HME_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        for (int r = 0; r < rounds; ++r) HME_CUDA(cudaGraphLaunch(exec, ctx->stream));
        HME_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    check_device_error(ctx);
    HME_CUDA(cudaMemcpy(devs.data(), d_devs, sizeof(RankDev) * nj, cudaMemcpyDeviceToHost));
    for (int i = 0; i < nj; ++i) ranks[order[i]] = devs[i].J.r0;
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

// The GEMM phase of a batch.  Every job's schedule is one of the GEMM variants
// (GemmVariant: tensor-core wide / half-width tiles, CUDA-core 32 / 64 tiles):
// from `variants` when given (-1 = the batch rule), else from the context: a
// pinned variant, or under the learned policy the planner's decision for the
// job's shape class (unplanned shapes: the batch rule).  The batch rule is one
// tensor-core launch with wide tiles unless the launch's wide tiles leave SMs
// idle.  Jobs run as one launch per (modulus, schedule) group, so a schedule
// changes only the launch a job's tiles belong to, never a residue.
constexpr int kBatchRule = -1;

void batch_gemm(hme_ctx* ctx, uint32_t njobs, const hme_job* jobs, const int* variants = nullptr) {
    std::vector<uint32_t> mods;
    for (uint32_t t = 0; t < njobs; ++t) {
        check_job(jobs[t]);
        if (variants) HME_REQUIRE(variants[t] >= kBatchRule && variants[t] < kGemmVariants, "job: unknown variant");
        if (std::find(mods.begin(), mods.end(), jobs[t].p) == mods.end()) mods.push_back(jobs[t].p);
    }
    for (uint32_t p : mods) {
        const ModParams mp = make_mod(p);
        // groups: the batch rule, then one per variant
        std::vector<GemmJob> g[1 + kGemmVariants];
        for (uint32_t t = 0; t < njobs; ++t) {
            const hme_job& j = jobs[t];
            if (j.p != p || j.m == 0 || j.n == 0) continue;
            if (j.k == 0 || j.k > limb_k_chunk(mp.limbs)) {
                // a K beyond the exact-accumulation chunk takes the single-job path
                gemm_u32_device(ctx, mp, j.m, j.n, j.k, j.A, j.lda, j.B, j.ldb, j.C, j.ldc, HME_SET);
                continue;
            }
            int v = kBatchRule;
            if (variants) v = variants[t];
            else if (ctx->fixed_variant >= 0) v = ctx->fixed_variant;
            else if (ctx->sched_policy == 1) v = sched_planned_variant(ctx, mp, j.m, j.n, j.k);
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
            g[v + 1].push_back(x);
        }
        grouped_gemm_u32_device(ctx, mp, g[0], -1);
        grouped_gemm_u32_device(ctx, mp, g[1 + kVariantWide], 0);
        grouped_gemm_u32_device(ctx, mp, g[1 + kVariantNarrow], 1);
        batch_simt_gemm_device(ctx, mp, g[1 + kVariantSimt32], 32);
        batch_simt_gemm_device(ctx, mp, g[1 + kVariantSimt64], 64);
    }
}

// The batch rule of the rank rounds (the method without the planner): the
// grouped tensor-core limb GEMM as the trailing update, and one last panel of
// up to 128 columns only for jobs of at most 128 rows -- a taller job's last
// panel is a long serial chain on one CTA that every job of the round waits
// for, so its rounds take 32 columns to the end.
int rank_rule(uint32_t m) { return m <= 128 ? kRankTensorLast128 : kRankTensorLast32; }

// The rank phase of a batch.  Every job's rank rounds follow one of the
// RankVariant schedules: from `rank_variants` when given (-1 = the batch rule),
// else under the learned policy the planner's decision for the job's shape
// class (unplanned shapes: the batch rule).  A schedule changes which kernels
// apply a job's trailing updates and how many columns a round takes, never a
// residue or the rank.
void batch_rank(hme_ctx* ctx, uint32_t njobs, const hme_job* jobs, uint32_t* ranks,
                const int* rank_variants = nullptr) {
    std::vector<BatchMatrix> mats(njobs);
    for (uint32_t t = 0; t < njobs; ++t) {
        if (rank_variants)
            HME_REQUIRE(rank_variants[t] >= kBatchRule && rank_variants[t] < kRankVariants,
                        "job: unknown rank schedule");
        mats[t].A = jobs[t].C;
        mats[t].ld = jobs[t].ldc;
        mats[t].m = jobs[t].m;
        mats[t].n = jobs[t].n;
        mats[t].p = jobs[t].p;
        int v = kBatchRule;
        if (rank_variants) {
            v = rank_variants[t];
        } else if (ctx->sched_policy == 1 && jobs[t].p >= 2) {
            v = sched_planned_rank_variant(ctx, make_mod(jobs[t].p), jobs[t].m, jobs[t].n, jobs[t].k);
        }
        mats[t].rank_variant = v < 0 ? rank_rule(jobs[t].m) : v;
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

int hme_batch_gemm_u32_dev_plan(hme_ctx* ctx, uint32_t njobs, const hme_job* jobs, const int* variants) {
    return guard([&] {
        HME_REQUIRE(ctx && (njobs == 0 || jobs), "null argument");
        bind(ctx);
        batch_gemm(ctx, njobs, jobs, variants);
        check_device_error(ctx);
    });
}

int hme_batch_gemm_rank_u32_dev_plan(hme_ctx* ctx, uint32_t njobs, const hme_job* jobs, const int* variants,
                                     uint32_t* ranks) {
    return guard([&] {
        HME_REQUIRE(ctx && (njobs == 0 || (jobs && ranks)), "null argument");
        bind(ctx);
        batch_gemm(ctx, njobs, jobs, variants);
        batch_rank(ctx, njobs, jobs, ranks);
    });
}

int hme_batch_rank_u32_dev_sched(hme_ctx* ctx, uint32_t njobs, const hme_job* jobs, const int* rank_variants,
                                 uint32_t* ranks) {
    return guard([&] {
        HME_REQUIRE(ctx && (njobs == 0 || (jobs && ranks)), "null argument");
        bind(ctx);
        batch_rank(ctx, njobs, jobs, ranks, rank_variants);
    });
}

int hme_batch_gemm_rank_u32_dev_sched(hme_ctx* ctx, uint32_t njobs, const hme_job* jobs, const int* gemm_variants,
                                      const int* rank_variants, uint32_t* ranks) {
    return guard([&] {
        HME_REQUIRE(ctx && (njobs == 0 || (jobs && ranks)), "null argument");
        bind(ctx);
        if (rank_variants)  // every argument checked before anything runs
            for (uint32_t t = 0; t < njobs; ++t)
                HME_REQUIRE(rank_variants[t] >= kBatchRule && rank_variants[t] < kRankVariants,
                            "job: unknown rank schedule");
        batch_gemm(ctx, njobs, jobs, gemm_variants);
        batch_rank(ctx, njobs, jobs, ranks, rank_variants);
    });
}

int hme_autotune_batch_rank(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, float density,
                            uint32_t count, int reps, float* ms) {
    return guard([&] {
        HME_REQUIRE(ctx && ms && m && n && k && count, "autotune_batch_rank: bad arguments");
        HME_REQUIRE(m <= 1024, "autotune_batch_rank: rows beyond 1024 take the single-matrix elimination");
        HME_REQUIRE(is_prime_u32(p), "autotune_batch_rank: the modulus must be prime");
        bind(ctx);
        // count products C = A B of the stream's construction (banded sparse operands below density 0.5,
        // dense uniform ones otherwise), so the rounds meet the ranks and pivot patterns such jobs have, and
        // one anchor: a dense 1024 x 1024 product of full rank on the batch rule, whose rounds run the whole
        // 34-round sequence as the stream's largest jobs do.  A schedule's cost is its jobs' MARGINAL time
        // beside the anchor (the batch with them minus the anchor alone): what the jobs add to a stream whose
        // rounds run anyway, not the latency of a small batch alone.
        constexpr uint32_t kAnchor = 1024;
        const size_t ea = static_cast<size_t>(m) * k, eb = static_cast<size_t>(k) * n, ec = static_cast<size_t>(m) * n;
        const size_t anc = static_cast<size_t>(kAnchor) * kAnchor;
        const size_t ab_all = (ea + eb) * count + 2 * anc, c_all = ec * count + anc;
        uint32_t* AB = static_cast<uint32_t*>(ctx->ws.get(kSlotSched0, sizeof(uint32_t) * ab_all));
        uint32_t* Cs = static_cast<uint32_t*>(ctx->ws.get(kSlotSched1, sizeof(uint32_t) * 2 * c_all));
        uint32_t* C0 = Cs + c_all;
        std::vector<GenSpec> specs(2 * static_cast<size_t>(count) + 2);
        std::vector<hme_job> jobs(count + 1);
        const int family = density < 0.5f ? 0 : 1;
        for (uint32_t t = 0; t < count; ++t) {
            uint32_t* A = AB + t * (ea + eb);
            uint32_t* B = A + ea;
            specs[2 * t] = GenSpec{A, k, m, k, p, family, 0x5EED0000ull + 2 * t};
            specs[2 * t + 1] = GenSpec{B, n, k, n, p, family, 0x5EED0001ull + 2 * t};
            jobs[t] = hme_job{p, m, n, k, A, k, B, n, C0 + t * ec, n};
        }
        uint32_t* Aa = AB + (ea + eb) * count;
        uint32_t* Ba = Aa + anc;
        specs[2 * count] = GenSpec{Aa, kAnchor, kAnchor, kAnchor, p, 1, 0xA5C40000ull};
        specs[2 * count + 1] = GenSpec{Ba, kAnchor, kAnchor, kAnchor, p, 1, 0xA5C40001ull};
        jobs[count] = hme_job{p, kAnchor, kAnchor, kAnchor, Aa, kAnchor, Ba, kAnchor, C0 + ec * count, kAnchor};
        gen_jobs_device(ctx, specs);
        batch_gemm(ctx, count + 1, jobs.data());
        for (uint32_t t = 0; t <= count; ++t) jobs[t].C = Cs + (jobs[t].C - C0);  // the copies the ranks destroy
        cudaEvent_t e0, e1;
        HME_CUDA(cudaEventCreate(&e0));
        HME_CUDA(cudaEventCreate(&e1));
        std::vector<int> var(count + 1, kBatchRule);
        std::vector<uint32_t> rk(count + 1), rk0(count + 1);
        // the median time of a batched rank of `nj` jobs starting at jobs[j0] (fresh copies every run)
        auto timed = [&](uint32_t j0, uint32_t nj, bool check) {
            std::vector<float> t;
            for (int r = -1; r < std::max(1, reps); ++r) {  // r = -1: warm
                HME_CUDA(cudaMemcpyAsync(Cs, C0, sizeof(uint32_t) * c_all, cudaMemcpyDeviceToDevice, ctx->stream));
                HME_CUDA(cudaEventRecord(e0, ctx->stream));
                batch_rank(ctx, nj, jobs.data() + j0, rk.data(), var.data() + j0);
                HME_CUDA(cudaEventRecord(e1, ctx->stream));
                HME_CUDA(cudaEventSynchronize(e1));
                float x = 0.f;
                HME_CUDA(cudaEventElapsedTime(&x, e0, e1));
                if (r >= 0) t.push_back(x);
                if (check) {
                    if (rk0[count] == 0) rk0 = rk;  // the anchor's rank is 1024: the first run's ranks are kept
                    // a schedule changes only the time: the same ranks under every schedule
                    HME_REQUIRE(rk == rk0, "autotune_batch_rank: schedules disagree on a rank");
                }
            }
            std::sort(t.begin(), t.end());
            return t[t.size() / 2];
        };
        try {
            const float t_anchor = timed(count, 1, false);
            for (int v = 0; v < kRankVariants; ++v) {
                std::fill(var.begin(), var.begin() + count, v);
                const float tv = timed(0, count + 1, true);
                // a marginal time at or below the anchor's noise is floored at 1 us per batch
                ms[v] = std::max(tv - t_anchor, 1e-3f) / static_cast<float>(count);
            }
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        check_device_error(ctx);
    });
}

int hme_autotune_batch(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, uint32_t count, int reps,
                       float* ms) {
    return guard([&] {
        HME_REQUIRE(ctx && ms && p >= 2 && m && n && k && count, "autotune_batch: bad arguments");
        bind(ctx);
        const size_t ea = static_cast<size_t>(m) * k, eb = static_cast<size_t>(k) * n, ec = static_cast<size_t>(m) * n;
        uint32_t* AB = static_cast<uint32_t*>(ctx->ws.get(kSlotSched0, sizeof(uint32_t) * (ea + eb) * count));
        uint32_t* Cs = static_cast<uint32_t*>(ctx->ws.get(kSlotSched1, sizeof(uint32_t) * ec * count));
        // operand values do not change any variant's timing; fill with a residue pattern
        HME_CUDA(cudaMemsetAsync(AB, 0x11, sizeof(uint32_t) * (ea + eb) * count, ctx->stream));
        std::vector<hme_job> jobs(count);
        for (uint32_t t = 0; t < count; ++t) {
            jobs[t] = hme_job{p, m, n, k, AB + t * (ea + eb), k, AB + t * (ea + eb) + ea, n, Cs + t * ec, n};
        }
        cudaEvent_t e0, e1;
        HME_CUDA(cudaEventCreate(&e0));
        HME_CUDA(cudaEventCreate(&e1));
        std::vector<int> var(count);
        for (int v = 0; v < kGemmVariants; ++v) {
            std::fill(var.begin(), var.end(), v);
            std::vector<float> t;
            batch_gemm(ctx, count, jobs.data(), var.data());  // warm
            for (int r = 0; r < std::max(1, reps); ++r) {
                HME_CUDA(cudaEventRecord(e0, ctx->stream));
                batch_gemm(ctx, count, jobs.data(), var.data());
                HME_CUDA(cudaEventRecord(e1, ctx->stream));
                HME_CUDA(cudaEventSynchronize(e1));
                float x = 0.f;
                HME_CUDA(cudaEventElapsedTime(&x, e0, e1));
                t.push_back(x);
            }
            std::sort(t.begin(), t.end());
            ms[v] = t[t.size() / 2] / static_cast<float>(count);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        check_device_error(ctx);
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

// Howell and Smith forms over Z/ell^k (ell prime, ell^k < 2^32) on the device.
//
// Reference semantics (drjanosch42/hacs 0.2.1): the Howell form of rowspan(A),
// ENGINE_API.md Sec. 13.5 (elim::howell, DenseElim.h:239-249;
// ring2k::howell, Binary/Ring2k.h:960-969 = minimal-valuation echelon
// echelon_blocked :539-695 + howell_pass :853-954; ring3k::howell,
// Binary/Ring3k.h:101), and the Smith valuations sigma (ring2k::smith,
// Ring2k.h:702-845; ring3k::smith / smith_levels, Ring3k.cpp:615-843).  Both
// outputs are unique functions of the input, so the device result equals the
// reference's bit for bit whatever pivot rows the blocked elimination picks.
//
// Smith by valuation levels (the reference's algorithm): at level s, over
// Z/ell^(k-s), the F_ell column rank profile of the current matrix (the field
// elimination on A mod ell) moves to the front; a unit-pivot LU of those r_s
// columns (the blocked device LU, pivots of valuation 0) leaves a Schur
// complement that is 0 mod ell; r_s valuations equal s; the Schur complement
// divided by ell is the next level.
//
// Howell: the blocked device LU with minimal-valuation pivots gives echelon
// rows with the same row span; the Sec. 13.5 pass (active rows in id order,
// closure rows appended at the bottom) runs on them in one CTA; the
// reduce-above runs in blocks of pivots, the floor quotients of the rows above
// a block by one kernel and their application by one limb GEMM (mod ell^k).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "hme_elim.h"
#include "hme_internal.h"
#include "hme_ptx.cuh"

namespace hme {
namespace {

constexpr int kHowellThreads = 1024;
constexpr int kReduceBlock = 64;
constexpr size_t kHowellLeadSmemMax = 192 * 1024;  // leading-column table of the Howell pass (48k rows)

struct RingK {
    uint32_t q, ell, k;
    uint64_t barrett;
    uint32_t unit_exp;
    uint32_t pw[33];
};

RingK make_ring(uint32_t ell, uint32_t k) {
    RingK r{};
    r.ell = ell;
    r.k = k;
    uint64_t pw = 1;
    for (uint32_t v = 0; v <= k; ++v) {
        r.pw[v] = static_cast<uint32_t>(pw);
        pw *= ell;
    }
    r.q = r.pw[k];
    r.barrett = make_mod(r.q).barrett;
    r.unit_exp = static_cast<uint32_t>(static_cast<uint64_t>(r.pw[k - 1]) * (ell - 1) - 1);
    return r;
}

__device__ __forceinline__ uint32_t pow_mod_d(uint32_t b, uint32_t e, uint32_t q, uint64_t barrett) {
    uint32_t r = 1 % q;
    while (e) {
        if (e & 1) r = mod_mul(r, b, q, barrett);
        b = mod_mul(b, b, q, barrett);
        e >>= 1;
    }
    return r;
}

// floor(2^64 / d) for 2 <= d < 2^32 (the Barrett constant of a small modulus)
__device__ __forceinline__ uint64_t make_barrett_d(uint32_t d) {
    const uint64_t q = ~0ull / d;  // floor((2^64 - 1) / d)
    return (q + 1) * d == 0 ? q + 1 : q;  // d divides 2^64 only for powers of two
}

__device__ __forceinline__ uint32_t val_k(uint32_t x, const RingK& R) {
    if (x == 0) return R.k;
    if (R.ell == 2) return min(static_cast<uint32_t>(__ffs(x) - 1), R.k);
    uint32_t v = 0;
    while (v < R.k && x % R.ell == 0) {
        x /= R.ell;
        ++v;
    }
    return v;
}

int grid_for(size_t work, int sms) {
    return static_cast<int>(std::max<size_t>(1, std::min<size_t>((work + 255) / 256, static_cast<size_t>(sms) * 8)));
}

// ---- small element-wise kernels --------------------------------------------------
__global__ void count_noncanonical_kernel(const uint32_t* __restrict__ A, uint64_t ld, int m, int n, uint32_t q,
                                          int* __restrict__ bad) {
    const size_t total = static_cast<size_t>(m) * n;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x)
        if (A[(idx / n) * ld + idx % n] >= q) atomicAdd(bad, 1);
}

// dst = src mod ell (compact m x n, ld dst_ld)
__global__ void mod_small_kernel(const uint32_t* __restrict__ src, uint64_t lds, int m, int n, uint32_t ell,
                                 uint32_t* __restrict__ dst, uint64_t ldd) {
    const size_t total = static_cast<size_t>(m) * n;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(idx / n), j = static_cast<int>(idx % n);
        dst[static_cast<size_t>(i) * ldd + j] = src[static_cast<size_t>(i) * lds + j] % ell;
    }
}

// dst[i][j] = src[row0 + i][colmap[col0 + j]] / div  (exact division; div = 1 copies)
__global__ void gather_div_kernel(const uint32_t* __restrict__ src, uint64_t lds, int row0, int rows,
                                  const int* __restrict__ colmap, int col0, int cols, uint32_t div,
                                  uint32_t* __restrict__ dst, uint64_t ldd) {
    const size_t total = static_cast<size_t>(rows) * cols;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(idx / cols), j = static_cast<int>(idx % cols);
        const uint32_t x = src[static_cast<size_t>(row0 + i) * lds + colmap[col0 + j]];
        dst[static_cast<size_t>(i) * ldd + j] = div == 1 ? x : x / div;
    }
}

__global__ void any_nonzero_kernel(const uint32_t* __restrict__ A, uint64_t ld, int m, int n, int* __restrict__ flag) {
    const size_t total = static_cast<size_t>(m) * n;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x)
        if (A[(idx / n) * ld + idx % n] != 0) {
            *flag = 1;
            return;
        }
}

// zero the stale multipliers left of each echelon row's pivot column
__global__ void clean_left_kernel(uint32_t* __restrict__ A, uint64_t ld, int rank, const int* __restrict__ pcols) {
    for (int i = blockIdx.x; i < rank; i += gridDim.x) {
        const int c = pcols[i];
        for (int j = threadIdx.x; j < c; j += blockDim.x) A[static_cast<size_t>(i) * ld + j] = 0;
    }
}

// ---- the Sec. 13.5 pass, one CTA ------------------------------------------------------
// W: row store (capacity cap rows x n, ld), rows [0, r) the echelon rows;
// closure rows are appended at r, r+1, ...  The active list is the alive rows
// in id order (echelon rows first, closure rows in creation order), which is
// the reference's list order, so "topmost" is the smallest id.
struct PassArgs {
    uint32_t* W;
    uint64_t ld;
    int n, r, cap;
    RingK R;
    unsigned char* alive;  // [cap]
    int* piv_id;           // [n] out: row id of each pivot
    int* piv_col;          // [n] out
    int* piv_v;            // [n] out
    int* h_out;
    int* nrows_out;        // rows used in the store
    int* err;
};

__global__ void __launch_bounds__(kHowellThreads) howell_pass_scan_kernel(const PassArgs a) {
    __shared__ unsigned long long s_best;
    __shared__ int s_nel;
    __shared__ int s_el[kHowellThreads];
    __shared__ uint32_t s_ui;
    __shared__ int s_nrows, s_h;
    __shared__ int s_closure_nz;
    const RingK& R = a.R;
    if (threadIdx.x == 0) {
        s_nrows = a.r;
        s_h = 0;
    }
    for (int i = threadIdx.x; i < a.cap; i += blockDim.x) a.alive[i] = i < a.r ? 1 : 0;
    __syncthreads();
    for (int c = 0; c < a.n; ++c) {
        if (threadIdx.x == 0) s_best = ~0ull;
        __syncthreads();
        const int nrows = s_nrows;
        for (int id = threadIdx.x; id < nrows; id += blockDim.x) {
            if (!a.alive[id]) continue;
            const uint32_t x = a.W[static_cast<size_t>(id) * a.ld + c];
            if (x == 0) continue;
            const unsigned long long key = (static_cast<unsigned long long>(val_k(x, R)) << 32) | static_cast<unsigned>(id);
            atomicMin(&s_best, key);
        }
        __syncthreads();
        const unsigned long long best = s_best;
        if (best == ~0ull) continue;
        const int pid = static_cast<int>(best & 0xffffffffu);
        const uint32_t v = static_cast<uint32_t>(best >> 32);
        uint32_t* P = a.W + static_cast<size_t>(pid) * a.ld;
        if (threadIdx.x == 0) {
            a.alive[pid] = 0;
            s_ui = pow_mod_d(P[c] / R.pw[v], R.unit_exp, R.q, R.barrett);
            s_nel = 0;
            s_closure_nz = 0;
        }
        __syncthreads();
        // scale the pivot row so that it leads with ell^v exactly
        const uint32_t ui = s_ui;
        for (int j = c + threadIdx.x; j < a.n; j += blockDim.x) P[j] = mod_mul(P[j], ui, R.q, R.barrett);
        __syncthreads();
        // the other alive rows with a non-zero in column c, in chunks of the CTA size
        for (int base = 0; base < nrows; base += blockDim.x) {
            const int id = base + threadIdx.x;
            if (id < nrows && a.alive[id] && a.W[static_cast<size_t>(id) * a.ld + c] != 0) {
                const int slot = atomicAdd(&s_nel, 1);
                s_el[slot] = id;
            }
            __syncthreads();
            const int nel = s_nel;
            // one warp per row: R -= (R[c] / ell^v) * P over columns [c, n)
            const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
            for (int t = warp; t < nel; t += nw) {
                uint32_t* Rw = a.W + static_cast<size_t>(s_el[t]) * a.ld;
                const uint32_t f = Rw[c] / R.pw[v];
                __syncwarp();
                for (int j = c + lane; j < a.n; j += 32)
                    Rw[j] = mod_sub(Rw[j], mod_mul(f, P[j], R.q, R.barrett), R.q);
            }
            __syncthreads();
            if (threadIdx.x == 0) s_nel = 0;
            __syncthreads();
        }
        // Howell closure: ell^(k - v) * P, zero in columns <= c, appended at the bottom
        if (v > 0) {
            const int nid = s_nrows;
            if (nid >= a.cap) {
                if (threadIdx.x == 0) atomicCAS(a.err, 0, 64);  // store exhausted: cannot happen (<= n closures)
                return;
            }
            uint32_t* Z = a.W + static_cast<size_t>(nid) * a.ld;
            const uint32_t f = R.pw[R.k - v];
            for (int j = threadIdx.x; j < a.n; j += blockDim.x) {
                const uint32_t z = j > c ? mod_mul(P[j], f, R.q, R.barrett) : 0u;
                Z[j] = z;
                if (z) s_closure_nz = 1;
            }
            __syncthreads();
            if (threadIdx.x == 0 && s_closure_nz) {
                a.alive[nid] = 1;
                s_nrows = nid + 1;
            }
        }
        if (threadIdx.x == 0) {
            a.piv_id[s_h] = pid;
            a.piv_col[s_h] = c;
            a.piv_v[s_h] = static_cast<int>(v);
            ++s_h;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *a.h_out = s_h;
        *a.nrows_out = s_nrows;
    }
}

// The inverse of a unit u of Z/ell^k by Newton's iteration x <- x (2 - u x),
// which doubles the ell-adic precision per step: in 32-bit wraparound from
// x = u (right to 3 bits) for ell = 2; from the inverse mod ell,
// u^(ell - 2) mod ell, for odd ell (1 -> 2 -> 4 -> ... >= k digits).
__device__ __forceinline__ uint32_t ring_unit_inverse(uint32_t u, const RingK& R) {
    if (R.ell == 2) {
        uint32_t x = u;
        for (int i = 0; i < 5; ++i) x *= 2u - u * x;
        return R.k >= 32 ? x : (x & (R.q - 1u));
    }
    const uint32_t u0 = u % R.ell;
    uint32_t x = pow_mod_d(u0, R.ell - 2, R.ell, make_barrett_d(R.ell));
    for (uint32_t prec = 1; prec < R.k; prec *= 2) {
        const uint32_t ux = mod_mul(u % R.q, x, R.q, R.barrett);
        x = mod_mul(x, mod_sub(2u % R.q, ux, R.q), R.q, R.barrett);
    }
    return x;
}

// The pass with a leading-column table in shared memory.  Every live row's
// first non-zero column is at least the current column c (eliminating column
// c' zeroes it in every row that had a non-zero there), so the rows with a
// non-zero in column c are exactly those whose leading column IS c: the scan
// per column reads the table, not the store.  A row reduced by the pivot gets
// its new leading column from the same warp pass that updates it; consumed
// pivot rows, zero rows and unused slots hold n (never a candidate).  On
// entry piv_col[0 .. r) holds the echelon rows' pivot columns (their leading
// columns: the entries left of them are zero).
__global__ void __launch_bounds__(kHowellThreads) howell_pass_kernel(const PassArgs a) {
    extern __shared__ int s_lead[];  // [cap]
    __shared__ unsigned long long s_best;
    __shared__ int s_nel, s_over;
    __shared__ int s_el[kHowellThreads];
    __shared__ uint32_t s_ui;
    __shared__ int s_nrows, s_h, s_zlead;
    const RingK& R = a.R;
    const int none = a.n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int i = threadIdx.x; i < a.cap; i += blockDim.x) s_lead[i] = i < a.r ? a.piv_col[i] : none;
    if (threadIdx.x == 0) {
        s_nrows = a.r;
        s_h = 0;
    }
    __syncthreads();
    for (int c = 0; c < a.n; ++c) {
        if (threadIdx.x == 0) {
            s_best = ~0ull;
            s_nel = 0;
            s_over = 0;
        }
        __syncthreads();
        const int nrows = s_nrows;
        // the candidates: smallest (valuation, id) and the list of all of them
        for (int id = threadIdx.x; id < nrows; id += blockDim.x) {
            if (s_lead[id] != c) continue;
            const uint32_t x = a.W[static_cast<size_t>(id) * a.ld + c];
            atomicMin(&s_best, (static_cast<unsigned long long>(val_k(x, R)) << 32) | static_cast<unsigned>(id));
            const int slot = atomicAdd(&s_nel, 1);
            if (slot < kHowellThreads) s_el[slot] = id;
            else s_over = 1;
        }
        __syncthreads();
        const unsigned long long best = s_best;
        if (best == ~0ull) continue;
        const int pid = static_cast<int>(best & 0xffffffffu);
        const uint32_t v = static_cast<uint32_t>(best >> 32);
        uint32_t* P = a.W + static_cast<size_t>(pid) * a.ld;
        if (threadIdx.x == 0) {
            s_lead[pid] = none;  // consumed
            s_ui = ring_unit_inverse(P[c] / R.pw[v], R);
            s_zlead = none;
        }
        __syncthreads();
        // scale the pivot row so that it leads with ell^v exactly
        const uint32_t ui = s_ui;
        for (int j = c + threadIdx.x; j < a.n; j += blockDim.x) P[j] = mod_mul(P[j], ui, R.q, R.barrett);
        __syncthreads();
        // R -= (R[c] / ell^v) * P over columns [c, n) for every other candidate,
        // one warp per row; more than one CTA-size of candidates: rescan
        for (;;) {
            const int nel = min(s_nel, kHowellThreads);
            for (int t = warp; t < nel; t += nw) {
                const int id = s_el[t];
                if (id == pid) continue;
                uint32_t* Rw = a.W + static_cast<size_t>(id) * a.ld;
                const uint32_t f = Rw[c] / R.pw[v];
                __syncwarp();
                int first = none;
                for (int j = c + lane; j < a.n; j += 32) {
                    const uint32_t y = mod_sub(Rw[j], mod_mul(f, P[j], R.q, R.barrett), R.q);
                    Rw[j] = y;
                    if (y != 0 && first == none) first = j;
                }
                first = __reduce_min_sync(0xffffffffu, first);
                if (lane == 0) s_lead[id] = first;
            }
            __syncthreads();
            if (!s_over) break;
            __syncthreads();
            if (threadIdx.x == 0) {
                s_nel = 0;
                s_over = 0;
            }
            __syncthreads();
            for (int id = threadIdx.x; id < nrows; id += blockDim.x) {
                if (s_lead[id] != c) continue;
                const int slot = atomicAdd(&s_nel, 1);
                if (slot < kHowellThreads) s_el[slot] = id;
                else s_over = 1;
            }
            __syncthreads();
        }
        // Howell closure: ell^(k - v) * P, zero in columns <= c, appended at the bottom
        if (v > 0) {
            const int nid = s_nrows;
            if (nid >= a.cap) {
                if (threadIdx.x == 0) atomicCAS(a.err, 0, 64);  // store exhausted: cannot happen (<= n closures)
                return;
            }
            uint32_t* Z = a.W + static_cast<size_t>(nid) * a.ld;
            const uint32_t f = R.pw[R.k - v];
            for (int j = threadIdx.x; j < a.n; j += blockDim.x) {
                const uint32_t z = j > c ? mod_mul(P[j], f, R.q, R.barrett) : 0u;
                Z[j] = z;
                if (z) atomicMin(&s_zlead, j);
            }
            __syncthreads();
            if (threadIdx.x == 0 && s_zlead != none) {
                s_lead[nid] = s_zlead;
                s_nrows = nid + 1;
            }
        }
        if (threadIdx.x == 0) {
            a.piv_id[s_h] = pid;
            a.piv_col[s_h] = c;
            a.piv_v[s_h] = static_cast<int>(v);
            ++s_h;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *a.h_out = s_h;
        *a.nrows_out = s_nrows;
    }
}

// ---- blocked reduce-above --------------------------------------------------------------
// For the pivot block [t0, t0+b): Q[i][t] (rows i < t0) are the floor quotients
// of row i against the block's pivots applied in order (each quotient on the
// canonical residue after the previous ones); one thread per row.
__global__ void reduce_quotients_kernel(const uint32_t* __restrict__ H, uint64_t ld, int t0, int b,
                                        const int* __restrict__ pcol, const int* __restrict__ pv, RingK R,
                                        uint32_t* __restrict__ Q) {
    __shared__ uint32_t sB[kReduceBlock * kReduceBlock];  // sB[t][t3] = H[t0+t][pcol[t0+t3]]
    __shared__ uint32_t sdiv[kReduceBlock];
    __shared__ int scol[kReduceBlock];
    for (int idx = threadIdx.x; idx < b * b; idx += blockDim.x) {
        const int t = idx / b, t3 = idx % b;
        sB[idx] = H[static_cast<size_t>(t0 + t) * ld + pcol[t0 + t3]];
    }
    for (int t = threadIdx.x; t < b; t += blockDim.x) {
        sdiv[t] = R.pw[pv[t0 + t]];
        scol[t] = pcol[t0 + t];
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t0) return;
    uint32_t vals[kReduceBlock];
    for (int t = 0; t < b; ++t) vals[t] = H[static_cast<size_t>(i) * ld + scol[t]];
    for (int t = 0; t < b; ++t) {
        const uint32_t qt = vals[t] / sdiv[t];
        Q[static_cast<size_t>(i) * b + t] = qt;
        if (qt == 0) continue;
        for (int t3 = t + 1; t3 < b; ++t3)
            vals[t3] = mod_sub(vals[t3], mod_mul(qt, sB[t * b + t3], R.q, R.barrett), R.q);
    }
}

// The triangle inside a block: for t = t0+1 .. t0+b-1, rows i in [t0, t) are
// reduced by pivot row t (one CTA, a warp per row).
__global__ void reduce_triangle_kernel(uint32_t* __restrict__ H, uint64_t ld, int n, int t0, int b,
                                       const int* __restrict__ pcol, const int* __restrict__ pv, RingK R) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int t = t0 + 1; t < t0 + b; ++t) {
        const int ct = pcol[t];
        const uint32_t div = R.pw[pv[t]];
        const uint32_t* Pt = H + static_cast<size_t>(t) * ld;
        for (int i = t0 + warp; i < t; i += nw) {
            uint32_t* Hi = H + static_cast<size_t>(i) * ld;
            const uint32_t qv = Hi[ct] / div;
            __syncwarp();
            if (qv == 0) continue;
            for (int j = ct + lane; j < n; j += 32) Hi[j] = mod_sub(Hi[j], mod_mul(qv, Pt[j], R.q, R.barrett), R.q);
        }
        __syncthreads();
    }
}

// H[i] = W[piv_id[i]]  (h x n)
__global__ void gather_rows_by_id_kernel(const uint32_t* __restrict__ W, uint64_t ldw, const int* __restrict__ ids,
                                         int h, int n, uint32_t* __restrict__ H, uint64_t ldh) {
    const size_t total = static_cast<size_t>(h) * n;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(idx / n), j = static_cast<int>(idx % n);
        H[static_cast<size_t>(i) * ldh + j] = W[static_cast<size_t>(ids[i]) * ldw + j];
    }
}

size_t pad_ld(size_t cols) { return (cols + 15) / 16 * 16 + 16; }

void check_input(hme_ctx* ctx, const uint32_t* A, size_t ld, int m, int n, uint32_t q) {
    int* bad = static_cast<int*>(ctx->ws.get(kSlotElim6, 64));
    HME_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), ctx->stream));
    HME_TIMED(ctx, "ring_check", count_noncanonical_kernel<<<grid_for(static_cast<size_t>(m) * n, ctx->num_sms), 256, 0,
                                                             ctx->stream>>>(A, ld, m, n, q, bad));
    int h = 0;
    HME_CUDA(cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    HME_CUDA(cudaStreamSynchronize(ctx->stream));
    if (h) throw Error(HME_EINVAL, "input is not canonical mod ell^k (" + std::to_string(h) + " entries >= ell^k)");
}

}  // namespace

// ---- Smith valuations ------------------------------------------------------------------
std::vector<uint32_t> smith_device(hme_ctx* ctx, uint32_t ell, uint32_t k, const uint32_t* A, size_t lda, int m,
                                   int n, const ElimOptions& opt) {
    std::vector<uint32_t> sigma;
    if (m == 0 || n == 0) return sigma;
    const RingK R0 = make_ring(ell, k);
    check_input(ctx, A, lda, m, n, R0.q);
    // ping-pong buffers for the level matrices, padded leading dimension
    const size_t ld = pad_ld(n);
    uint32_t* cur = static_cast<uint32_t*>(ctx->ws.get(kSlotRing0, sizeof(uint32_t) * static_cast<size_t>(m) * ld));
    uint32_t* nxt = static_cast<uint32_t*>(ctx->ws.get(kSlotRing1, sizeof(uint32_t) * static_cast<size_t>(m) * ld));
    uint32_t* tmp = static_cast<uint32_t*>(ctx->ws.get(kSlotRing2, sizeof(uint32_t) * static_cast<size_t>(m) * ld));
    int* d_map = static_cast<int*>(ctx->ws.get(kSlotRing3, sizeof(int) * (static_cast<size_t>(n) + 16)));
    int* d_flag = d_map + n;
    std::vector<int> identity(n);
    for (int j = 0; j < n; ++j) identity[j] = j;
    HME_CUDA(cudaMemcpyAsync(d_map, identity.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->stream));
    HME_TIMED(ctx, "ring_gather", gather_div_kernel<<<grid_for(static_cast<size_t>(m) * n, ctx->num_sms), 256, 0,
                                                      ctx->stream>>>(A, lda, 0, m, d_map, 0, n, 1, cur, ld));
    int rows = m, cols = n;
    for (uint32_t s = 0; s < k && rows > 0 && cols > 0; ++s) {
        const uint32_t kk = k - s;
        const RingK R = make_ring(ell, kk);
        // stop when the level matrix is zero: no further valuation < k
        HME_CUDA(cudaMemsetAsync(d_flag, 0, sizeof(int), ctx->stream));
        HME_TIMED(ctx, "ring_nonzero", any_nonzero_kernel<<<grid_for(static_cast<size_t>(rows) * cols, ctx->num_sms),
                                                            256, 0, ctx->stream>>>(cur, ld, rows, cols, d_flag));
        int nz = 0;
        HME_CUDA(cudaMemcpyAsync(&nz, d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        HME_CUDA(cudaStreamSynchronize(ctx->stream));
        if (!nz) break;
        // (1) the F_ell column rank profile of the level matrix
        HME_TIMED(ctx, "ring_mod", mod_small_kernel<<<grid_for(static_cast<size_t>(rows) * cols, ctx->num_sms), 256, 0,
                                                      ctx->stream>>>(cur, ld, rows, cols, ell, tmp, ld));
        ElimOptions o = opt;
        const ElimResult prof = elim_device(ctx, make_mod(ell), tmp, ld, rows, cols, false, nullptr, 0, o);
        const int r = prof.rank;
        if (r == 0) {
            // A = 0 mod ell: the level has no invariant; divide by ell
            HME_TIMED(ctx, "ring_gather", gather_div_kernel<<<grid_for(static_cast<size_t>(rows) * cols, ctx->num_sms), 256,
                                                              0, ctx->stream>>>(cur, ld, 0, rows, d_map, 0, cols, ell, nxt,
                                                                                ld));
            std::swap(cur, nxt);
            continue;
        }
        // (2) profile columns to the front, then the rest in order
        std::vector<int> cmap;
        cmap.reserve(cols);
        {
            std::vector<char> isp(cols, 0);
            for (int c : prof.pivots) {
                isp[c] = 1;
                cmap.push_back(c);
            }
            for (int c = 0; c < cols; ++c)
                if (!isp[c]) cmap.push_back(c);
        }
        HME_CUDA(cudaMemcpyAsync(d_map, cmap.data(), sizeof(int) * cols, cudaMemcpyHostToDevice, ctx->stream));
        HME_TIMED(ctx, "ring_gather", gather_div_kernel<<<grid_for(static_cast<size_t>(rows) * cols, ctx->num_sms), 256, 0,
                                                          ctx->stream>>>(cur, ld, 0, rows, d_map, 0, cols, 1, nxt, ld));
        // (3) unit-pivot LU of the first r columns over Z/ell^kk
        RingSpec rs;
        rs.ell = ell;
        rs.k = kk;
        rs.max_v = 0;
        rs.lu_cols = r;
        const ElimResult lu = elim_device(ctx, make_mod(R.q), nxt, ld, rows, cols, false, nullptr, 0, o, &rs);
        if (lu.rank != r)
            throw Error(HME_EINVAL, "smith: unit-pivot LU found " + std::to_string(lu.rank) + " pivots, expected " +
                                        std::to_string(r));
        for (int t = 0; t < r; ++t) sigma.push_back(s);
        // (4) the Schur complement divided by ell is the next level
        for (int j = 0; j < cols; ++j) identity[j] = j;
        HME_CUDA(cudaMemcpyAsync(d_map, identity.data(), sizeof(int) * cols, cudaMemcpyHostToDevice, ctx->stream));
        const int nr = rows - r, nc = cols - r;
        if (nr > 0 && nc > 0)
            HME_TIMED(ctx, "ring_gather", gather_div_kernel<<<grid_for(static_cast<size_t>(nr) * nc, ctx->num_sms), 256, 0,
                                                              ctx->stream>>>(nxt, ld, r, nr, d_map, r, nc, ell, cur, ld));
        rows = nr;
        cols = nc;
    }
    check_device_error(ctx);
    return sigma;
}

// ---- Howell form ----------------------------------------------------------------------
HowellOut howell_device(hme_ctx* ctx, uint32_t ell, uint32_t k, const uint32_t* A, size_t lda, int m, int n,
                        const ElimOptions& opt) {
    HowellOut out;
    if (m == 0 || n == 0) return out;
    const RingK R = make_ring(ell, k);
    check_input(ctx, A, lda, m, n, R.q);
    const size_t ld = pad_ld(n);
    const int cap = std::max(m, 0) + n;  // echelon rows (<= min(m, n)) plus at most one closure row per pivot
    uint32_t* W = static_cast<uint32_t*>(ctx->ws.get(kSlotRing0, sizeof(uint32_t) * static_cast<size_t>(cap) * ld));
    int* d_map = static_cast<int*>(ctx->ws.get(kSlotRing3, sizeof(int) * (static_cast<size_t>(n) + 16)));
    {
        std::vector<int> identity(n);
        for (int j = 0; j < n; ++j) identity[j] = j;
        HME_CUDA(cudaMemcpyAsync(d_map, identity.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->stream));
        HME_TIMED(ctx, "ring_gather", gather_div_kernel<<<grid_for(static_cast<size_t>(m) * n, ctx->num_sms), 256, 0,
                                                          ctx->stream>>>(A, lda, 0, m, d_map, 0, n, 1, W, ld));
    }
    // (1) minimal-valuation echelon (same row span)
    RingSpec rs;
    rs.ell = ell;
    rs.k = k;
    rs.max_v = k - 1;
    rs.lu_cols = n;
    ElimOptions o = opt;
    const ElimResult lu = elim_device(ctx, make_mod(R.q), W, ld, m, n, false, nullptr, 0, o, &rs);
    const int r = lu.rank;
    int* d_idx = static_cast<int*>(ctx->ws.get(kSlotRing2, sizeof(int) * (5 * static_cast<size_t>(n) + 64)));
    int* d_pid = d_idx;
    int* d_pcol = d_idx + n;
    int* d_pv = d_idx + 2 * n;
    int* d_cnt = d_idx + 3 * n;  // h, nrows
    unsigned char* alive = static_cast<unsigned char*>(ctx->ws.get(kSlotRing1, static_cast<size_t>(cap) + 64));
    if (r > 0) {
        HME_CUDA(cudaMemcpyAsync(d_pcol, lu.pivots.data(), sizeof(int) * r, cudaMemcpyHostToDevice, ctx->stream));
        HME_TIMED(ctx, "ring_clean", clean_left_kernel<<<std::min(r, ctx->num_sms * 4), 256, 0, ctx->stream>>>(
                                         W, ld, r, d_pcol));
    }
    // rows [r, m) of W are the (zero) Schur complement; the closure rows start at r
    // (2) the Sec. 13.5 pass
    PassArgs pa{};
    pa.W = W;
    pa.ld = ld;
    pa.n = n;
    pa.r = r;
    pa.cap = cap;
    pa.R = R;
    pa.alive = alive;
    pa.piv_id = d_pid;
    pa.piv_col = d_pcol;
    pa.piv_v = d_pv;
    pa.h_out = d_cnt;
    pa.nrows_out = d_cnt + 1;
    pa.err = ctx->d_err;
    // the leading-column table in shared memory when it fits, else the store-scanning pass
    const size_t lead_bytes = sizeof(int) * static_cast<size_t>(cap);
    if (lead_bytes <= kHowellLeadSmemMax) {
        HME_CUDA(cudaFuncSetAttribute(howell_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kHowellLeadSmemMax)));
        HME_TIMED(ctx, "howell_pass", howell_pass_kernel<<<1, kHowellThreads, lead_bytes, ctx->stream>>>(pa));
    } else {
        HME_TIMED(ctx, "howell_pass", howell_pass_scan_kernel<<<1, kHowellThreads, 0, ctx->stream>>>(pa));
    }
    HME_CUDA(cudaGetLastError());
    int hc[2] = {0, 0};
    HME_CUDA(cudaMemcpyAsync(hc, d_cnt, sizeof(int) * 2, cudaMemcpyDeviceToHost, ctx->stream));
    check_device_error(ctx);
    const int h = hc[0];
    out.pivots.resize(h);
    out.pivot_v.resize(h);
    out.H.assign(static_cast<size_t>(h) * n, 0);
    if (h == 0) return out;
    HME_CUDA(cudaMemcpyAsync(out.pivots.data(), d_pcol, sizeof(int) * h, cudaMemcpyDeviceToHost, ctx->stream));
    HME_CUDA(cudaMemcpyAsync(out.pivot_v.data(), d_pv, sizeof(int) * h, cudaMemcpyDeviceToHost, ctx->stream));
    // (3) H = the pivot rows in pivot order, then the blocked reduce-above
    const size_t ldh = ld;
    uint32_t* H = static_cast<uint32_t*>(ctx->ws.get(kSlotRing4, sizeof(uint32_t) * static_cast<size_t>(h) * ldh));
    HME_TIMED(ctx, "ring_gather", gather_rows_by_id_kernel<<<grid_for(static_cast<size_t>(h) * n, ctx->num_sms), 256, 0,
                                                             ctx->stream>>>(W, ld, d_pid, h, n, H, ldh));
    HME_CUDA(cudaStreamSynchronize(ctx->stream));
    uint32_t* Q = static_cast<uint32_t*>(ctx->ws.get(kSlotRing5, sizeof(uint32_t) * static_cast<size_t>(h) * kReduceBlock));
    const ModParams mq = make_mod(R.q);
    for (int t0 = 0; t0 < h; t0 += kReduceBlock) {
        const int b = std::min(kReduceBlock, h - t0);
        const int c0 = out.pivots[t0];
        if (t0 > 0) {
            HME_TIMED(ctx, "reduce_quot", reduce_quotients_kernel<<<(t0 + 127) / 128, 128, 0, ctx->stream>>>(
                                              H, ldh, t0, b, d_pcol, d_pv, R, Q));
            HME_CUDA(cudaGetLastError());
            gemm_u32_device(ctx, mq, t0, n - c0, b, Q, b, H + static_cast<size_t>(t0) * ldh + c0, ldh, H + c0, ldh,
                            HME_SUB);
        }
        if (b > 1)
            HME_TIMED(ctx, "reduce_tri", reduce_triangle_kernel<<<1, 1024, 0, ctx->stream>>>(H, ldh, n, t0, b, d_pcol,
                                                                                              d_pv, R));
        HME_CUDA(cudaGetLastError());
    }
    HME_CUDA(cudaMemcpy2DAsync(out.H.data(), sizeof(uint32_t) * n, H, sizeof(uint32_t) * ldh, sizeof(uint32_t) * n, h,
                               cudaMemcpyDeviceToHost, ctx->stream));
    check_device_error(ctx);
    return out;
}

}  // namespace hme

// ---- C ABI ---------------------------------------------------------------------------------
using namespace hme;

namespace {
void check_ring(uint32_t ell, uint32_t k) {
    HME_REQUIRE(k >= 1, "ring: k must be >= 1");
    HME_REQUIRE(ell >= 2 && is_prime_u32(ell), "ring: ell must be a prime");
    uint64_t q = 1;
    for (uint32_t i = 0; i < k; ++i) {
        q *= ell;
        HME_REQUIRE(q < (1ull << 32), "ring: ell^k must be < 2^32");
    }
}
}  // namespace

extern "C" {

int hme_howell_u32(hme_ctx* ctx, uint32_t ell, uint32_t k, uint32_t m, uint32_t n, const uint32_t* A, size_t lda,
                   uint32_t* H, size_t ldh, uint32_t* pivots, uint32_t* pivot_v, uint32_t* h) {
    return guard([&] {
        HME_REQUIRE(ctx && h, "null argument");
        check_ring(ell, k);
        bind(ctx);
        *h = 0;
        if (m == 0 || n == 0) return;
        HME_REQUIRE(A && lda >= n && H && ldh >= n && pivots && pivot_v, "bad buffers");
        uint32_t* d = static_cast<uint32_t*>(ctx->ws.get(kSlotStageA, sizeof(uint32_t) * static_cast<size_t>(m) * n));
        HME_CUDA(cudaMemcpy2DAsync(d, sizeof(uint32_t) * n, A, sizeof(uint32_t) * lda, sizeof(uint32_t) * n, m,
                                   cudaMemcpyHostToDevice, ctx->stream));
        const HowellOut r = howell_device(ctx, ell, k, d, n, m, n, ctx->elim);
        const uint32_t hh = static_cast<uint32_t>(r.pivots.size());
        HME_REQUIRE(hh <= n, "howell: more rows than columns");
        for (uint32_t i = 0; i < hh; ++i) {
            pivots[i] = r.pivots[i];
            pivot_v[i] = r.pivot_v[i];
            std::copy(r.H.begin() + static_cast<size_t>(i) * n, r.H.begin() + static_cast<size_t>(i + 1) * n,
                      H + static_cast<size_t>(i) * ldh);
        }
        *h = hh;
    });
}

int hme_smith_u32(hme_ctx* ctx, uint32_t ell, uint32_t k, uint32_t m, uint32_t n, const uint32_t* A, size_t lda,
                  uint32_t* sigma, uint32_t* count) {
    return guard([&] {
        HME_REQUIRE(ctx && count, "null argument");
        check_ring(ell, k);
        bind(ctx);
        *count = 0;
        if (m == 0 || n == 0) return;
        HME_REQUIRE(A && lda >= n && sigma, "bad buffers");
        uint32_t* d = static_cast<uint32_t*>(ctx->ws.get(kSlotStageA, sizeof(uint32_t) * static_cast<size_t>(m) * n));
        HME_CUDA(cudaMemcpy2DAsync(d, sizeof(uint32_t) * n, A, sizeof(uint32_t) * lda, sizeof(uint32_t) * n, m,
                                   cudaMemcpyHostToDevice, ctx->stream));
        const std::vector<uint32_t> s = smith_device(ctx, ell, k, d, n, m, n, ctx->elim);
        for (size_t i = 0; i < s.size(); ++i) sigma[i] = s[i];
        *count = static_cast<uint32_t>(s.size());
    });
}

}  // extern "C"

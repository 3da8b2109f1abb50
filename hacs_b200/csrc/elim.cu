// Device-resident elimination over F_p, p < 2^32 prime: RREF, rank, column
// rank profile, determinant (and, built on them, kernel basis, inverse, solve).
//
// Reference semantics: engine::elim::rref / column_rank_profile
// (src/ModArithmetic/DenseElim.h:153-169; Plu factor / trailing_update / to_rref
// DenseElim.cpp:323-560, rref :921).  RREF(A) is unique (leading 1, zero rows
// at the bottom) and its pivot columns are the column rank profile, so the pivot
// ROW choice cannot show in the output; this driver takes the reference's rule
// anyway (leftmost column with a non-zero in the Schur complement, topmost such
// row) because it is also the cheapest to find in parallel (a min over rows).
//
// Blocked right-looking LU, panels of `bw` columns.  Over a field the panel
// first takes the top-block path (panel_block_kernel, panel_binv_kernel,
// panel_w_kernel; the reasoning is at their definitions): when the panel's top
// bw rows factor with non-zero diagonal entries they are its pivots, no search
// runs, no row moves, and steps 2-4 below collapse into one limb GEMM
// [A12; A22] += [L^-1 - I; -A21 B^-1] A12.  Otherwise:
//   1. panel_cluster_kernel: the panel's active rows A[r0:m, c0:c0+bw) sit in
//      the shared memory of one thread-block cluster (up to 16 CTAs); per
//      column each CTA pushes its best (valuation, row) key and that row to
//      every CTA through distributed shared memory, one cluster barrier, a
//      warp min of the keys; fraction-free row updates, unit scales undone
//      once per panel.  Panels too tall for one cluster take
//      panel_factor_kernel instead: one cooperative launch over all SMs with
//      one bounded grid barrier per column.  Either way pivot rows are not
//      swapped during the panel (they leave the active set) and multipliers
//      are stored in the pivot columns of the active rows (packed L).
//   2. the panel's pivot rows move to rows r0 .. r0+k-1 in pivot order (columns
//      >= c0; columns left of the panel of non-U rows hold dead multipliers).
//   3. U12 = L11^-1 A12 in place: trsm_unit_lower_kernel, one warp per column
//      of A12 holding its k rows in registers (forward substitution with
//      shuffles), L11 in shared memory.
//   4. A22 -= L21 * U12: the INT8-limb tcgen05 GEMM (Sub), K = k pivots.
// Then RREF = U1^-1 U on the free columns only (the pivot columns of the RREF
// are the identity): every diagonal block of U1 is inverted in shared memory
// (one launch), and the blocked backward substitution is two limb GEMMs per
// block (X_B = U_BB^-1 W_B, then W_above -= U_above,B X_B).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "hme_elim.h"
#include "hme_internal.h"
#include "hme_ptx.cuh"

namespace hme {
namespace {

constexpr int kPanelThreads = 256;
constexpr int kPanelWarps = kPanelThreads / 32;
constexpr int kMaxPanel = 128;
constexpr int kPanelSmemMax = 160 * 1024;  // largest shared-memory row slice of the panel kernel
constexpr unsigned long long kNoKey = 0x7f7f7f7f7f7f7f7full;  // piv_slot sentinel (memset 0x7f)


// Inverse of a unit u of Z/q, q = ell^k, without divisions on the slow path:
//   ell = 2: Newton's iteration x <- x (2 - u x) in native 32-bit wraparound
//            (each step doubles the correct low bits), then reduced mod 2^k;
//   k > 1:   the inverse mod ell (binary extended gcd) lifted by the same
//            iteration mod q (Hensel), doubling the ell-adic precision;
//   k = 1:   the binary extended gcd mod the odd prime q.
__device__ __forceinline__ uint32_t inv_binary_xgcd(uint32_t u, uint32_t q) {
    // invariant: x1 * u == a (mod q), x2 * u == b (mod q), q odd.  Bounded:
    // each pass shrinks a + b by at least one bit position or a subtraction,
    // so 128 passes cover 32-bit operands; a non-unit (gcd > 1) returns 0.
    if (u == 0) return 0;
    uint32_t a = u, b = q, x1 = 1, x2 = 0;
    for (int guard_it = 0; a != 1 && b != 1; ++guard_it) {
        if (a == 0 || b == 0 || guard_it > 128) return 0;
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

// The ring Z/q, q = ell^k (k = 1: the field F_ell), as the elimination sees it.
struct Ring {
    uint32_t q;          // modulus
    uint64_t barrett;    // floor(2^64 / q)
    uint32_t ell, k;
    uint32_t unit_exp;   // phi(q) - 1: u^unit_exp is the inverse of a unit u
    uint32_t max_v;      // pivots of valuation <= max_v only (0: unit pivots)
    uint32_t mont_qinv;  // q odd: -q^-1 mod 2^32 (Montgomery reduction)
    uint32_t mont_r2;    // q odd: 2^64 mod q
    uint32_t pw[32];     // ell^0 .. ell^k
};

// Montgomery product x * y * 2^-32 mod q for odd q < 2^32 and x, y < q: the
// sum T + m q may carry out of 64 bits when q > 2^31, so the carry is kept.
__device__ __forceinline__ uint32_t mont_mul(uint32_t x, uint32_t y, uint32_t q, uint32_t qinv) {
    const uint64_t t = static_cast<uint64_t>(x) * y;
    const uint32_t mq = static_cast<uint32_t>(t) * qinv;
    const uint64_t u = t + static_cast<uint64_t>(mq) * q;
    const uint64_t r = (u >> 32) + (u < t ? (1ull << 32) : 0ull);  // < 2q
    return static_cast<uint32_t>(r >= q ? r - q : r);
}

// u^(q-2) mod q (Fermat) for an odd prime q, left-to-right square and
// multiply in the Montgomery domain: about 2 log2 q dependent products.
__device__ __forceinline__ uint32_t inv_fermat(uint32_t u, const Ring& R) {
    const uint32_t q = R.q, qi = R.mont_qinv;
    const uint32_t um = mont_mul(u, R.mont_r2, q, qi);  // u * 2^32 mod q
    const uint32_t e = q - 2;
    uint32_t r = um;
    for (int b = 30 - __clz(e); b >= 0; --b) {
        r = mont_mul(r, r, q, qi);
        if ((e >> b) & 1u) r = mont_mul(r, um, q, qi);
    }
    return mont_mul(r, 1u, q, qi);  // out of the Montgomery domain
}

__device__ __forceinline__ uint32_t unit_inverse(uint32_t u, const Ring& R) {
    if (R.k == 1 && R.ell != 2) return inv_fermat(u % R.q, R);
    if (R.ell == 2) {
        uint32_t x = u;  // correct to 3 bits for odd u
        for (int i = 0; i < 5; ++i) x *= 2u - u * x;
        return R.k >= 32 ? x : (x & (R.q - 1));
    }
    if (R.k == 1) return inv_binary_xgcd(u % R.q, R.q);
    uint32_t x = inv_binary_xgcd(u % R.ell, R.ell);  // inverse mod ell
    for (uint32_t prec = 1; prec < R.k; prec *= 2) {
        const uint32_t ux = mod_mul(u, x, R.q, R.barrett);
        x = mod_mul(x, mod_sub(2u % R.q, ux, R.q), R.q, R.barrett);
    }
    return x;
}

// ell-adic valuation of x != 0, capped at cap + 1 (enough to reject a candidate).
__device__ __forceinline__ uint32_t valuation(uint32_t x, const Ring& R, uint32_t cap) {
    if (R.ell == 2) return min(static_cast<uint32_t>(__ffs(x) - 1), cap + 1);
    uint32_t v = 0;
    while (v <= cap && x % R.ell == 0) {
        x /= R.ell;
        ++v;
    }
    return v;
}

// Pivot key of an entry: (valuation << 32 | row), or kNoKey when x is zero or
// its valuation exceeds the ring's max_v.
__device__ __forceinline__ unsigned long long pivot_key(uint32_t x, int row, const Ring& R) {
    if (x == 0) return kNoKey;
    const uint32_t v = R.k == 1 ? 0u : R.max_v == 0 ? (x % R.ell == 0 ? 1u : 0u) : valuation(x, R, R.max_v);
    if (v > R.max_v) return kNoKey;
    return (static_cast<unsigned long long>(v) << 32) | static_cast<unsigned>(row);
}

struct PanelArgs {
    uint32_t* A;
    uint64_t ld;
    int m;
    int c0, bw;  // panel columns [c0, c0 + bw)
    int r0;      // first active row
    Ring R;
    unsigned long long* piv_slot;  // [bw], kNoKey on entry: smallest (valuation, row) key per column
    uint32_t* cand;      // [2][grid][kMaxPanel]: candidate row values, by column parity
    int* pivot_rows;     // [bw] out
    int* pivot_cols;     // [bw] out
    int* k_out;          // out: pivots found
    unsigned* bar;       // [2]: arrival count, generation
    int* err;
    const int* skip;     // non-null and non-zero: the panel is settled already (top-block path)
};

// Bounded grid-wide barrier for a cooperative launch (all CTAs co-resident).
// Returns false on timeout or when another CTA already gave up.
__device__ bool grid_barrier(unsigned* bar, int* err, int* s_flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = bar + 1;
        volatile int* verr = err;
        const unsigned g = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u);
        int ok = 1;
        if (arrived == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            const uint64_t t0 = global_timer_ns();
            uint32_t spin = 0;
            while (*vgen == g) {
                if ((++spin & 63u) == 0) {
                    if (*verr != 0) { ok = 0; break; }
                    if (global_timer_ns() - t0 > HME_WAIT_LIMIT_NS) {
                        atomicCAS(err, 0, DERR_GRID_BARRIER);
                        ok = 0;
                        break;
                    }
                }
            }
        }
        __threadfence();
        *s_flag = ok;
    }
    __syncthreads();
    return *s_flag != 0;
}

// One cooperative launch per panel.  With smem_rows, every CTA copies its
// slice of the panel (rpc rows x bw columns) into shared memory first and
// writes it back at the end, so the per-column work never leaves the SM; the
// global-memory mode (slices too large for shared memory) works in place.
__global__ void __launch_bounds__(kPanelThreads) panel_factor_kernel(const PanelArgs a, int smem_rows) {
    extern __shared__ uint32_t s_slice[];
    __shared__ uint32_t s_prow[kMaxPanel];
    __shared__ unsigned long long s_cand;
    __shared__ int s_flag;
    __shared__ unsigned long long s_piv;
    __shared__ uint32_t s_inv, s_div;

    // settled by the top-block path: the same in every CTA, before any grid barrier
    if (a.skip != nullptr && *a.skip != 0) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int active_rows = a.m - a.r0;
    const int rpc = (active_rows + gridDim.x - 1) / gridDim.x;
    const int row_begin = a.r0 + blockIdx.x * rpc;
    const int row_end = min(a.m, row_begin + rpc);
    const int cend = a.c0 + a.bw;
    const size_t cand_stride = static_cast<size_t>(gridDim.x) * kMaxPanel;

    // row i of the panel, indexed by absolute column c in [c0, cend)
    auto rowp = [&](int i) -> uint32_t* {
        return smem_rows ? s_slice + static_cast<size_t>(i - row_begin) * a.bw - a.c0
                         : a.A + static_cast<size_t>(i) * a.ld;
    };
    if (smem_rows) {
        for (int i = row_begin + warp; i < row_end; i += kPanelWarps) {
            const uint32_t* src = a.A + static_cast<size_t>(i) * a.ld;
            uint32_t* dst = rowp(i);
            for (int j = a.c0 + lane; j < cend; j += 32) dst[j] = src[j];
        }
    }
    // per-row multiplier of the current column, and per-row flag: the row
    // became a pivot row of this panel
    uint32_t* s_l = s_slice + (smem_rows ? static_cast<size_t>(rpc) * a.bw : 0);
    unsigned char* s_isp = reinterpret_cast<unsigned char*>(s_l + rpc);
    for (int i = threadIdx.x; i < rpc; i += blockDim.x) s_isp[i] = 0;
    __syncthreads();
    auto is_pivot_row = [&](int i) { return s_isp[i - row_begin] != 0; };

    // Publish this CTA's best pivot candidate for column c (smallest
    // (valuation, row) key, already in s_cand): the row's values of columns
    // [c, cend) into the parity slot, the key by atomicMin.
    auto publish_candidate = [&](int c) {
        __syncthreads();
        if (c < cend && s_cand != kNoKey) {
            const uint32_t* src = rowp(static_cast<int>(s_cand & 0xffffffffu));
            uint32_t* dst = a.cand + static_cast<size_t>(c & 1) * cand_stride + static_cast<size_t>(blockIdx.x) * kMaxPanel;
            for (int j = c + threadIdx.x; j < cend; j += blockDim.x) dst[j - a.c0] = src[j];
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                atomicMin(&a.piv_slot[c - a.c0], s_cand);
            }
        }
    };
    auto find_candidate = [&](int c) {
        if (threadIdx.x == 0) s_cand = kNoKey;
        __syncthreads();
        if (c < cend) {
            for (int i = row_begin + threadIdx.x; i < row_end; i += blockDim.x) {
                const unsigned long long key = pivot_key(rowp(i)[c], i, a.R);
                if (key != kNoKey && !is_pivot_row(i)) atomicMin(&s_cand, key);
            }
        }
        publish_candidate(c);
    };

    find_candidate(a.c0);
    int k = 0;
    bool ok = true;
    for (int c = a.c0; c < cend; ++c) {
        if (!grid_barrier(a.bar, a.err, &s_flag)) {
            ok = false;
            break;
        }
        if (threadIdx.x == 0) s_piv = *reinterpret_cast<volatile unsigned long long*>(&a.piv_slot[c - a.c0]);
        __syncthreads();
        const unsigned long long pkey = s_piv;
        if (pkey == kNoKey) {
            // column c is not a pivot column: every active row is zero there
            find_candidate(c + 1);
            continue;
        }
        const int prow = static_cast<int>(pkey & 0xffffffffu);
        const uint32_t pv = static_cast<uint32_t>(pkey >> 32);
        const int owner = (prow - a.r0) / rpc;
        const uint32_t* src = a.cand + static_cast<size_t>(c & 1) * cand_stride + static_cast<size_t>(owner) * kMaxPanel;
        for (int j = c + threadIdx.x; j < cend; j += blockDim.x)
            s_prow[j - a.c0] = *reinterpret_cast<const volatile uint32_t*>(&src[j - a.c0]);
        if (threadIdx.x == 0) {
            if (prow >= row_begin && prow < row_end) s_isp[prow - row_begin] = 1;
            if (blockIdx.x == 0) {
                a.pivot_rows[k] = prow;
                a.pivot_cols[k] = c;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            // pivot x = ell^v * u: multipliers are (x_i / ell^v) * u^-1
            const uint32_t x = s_prow[c - a.c0];
            const uint32_t div = a.R.pw[pv];
            s_div = div;
            s_inv = unit_inverse(x / div, a.R);
        }
        __syncthreads();
        const uint32_t inv = s_inv, div = s_div;
        ++k;
        // eliminate column c from this CTA's active rows in two phases:
        // (1) one thread per row: multiplier l = (x / ell^v) * u^-1, stored in
        //     the pivot column (packed L); (2) all threads over the (row,
        //     column > c) elements, l * pivot row subtracted; the elements of
        //     column c + 1 feed the next column's pivot candidate on the way.
        const int nloc = row_end - row_begin;
        if (threadIdx.x == 0) s_cand = kNoKey;
        for (int li = threadIdx.x; li < nloc; li += blockDim.x) {
            const int i = row_begin + li;
            uint32_t l = 0;
            if (i != prow && !is_pivot_row(i)) {
                uint32_t* row = rowp(i);
                const uint32_t x = row[c];
                if (x != 0) {
                    l = mod_mul(div == 1 ? x : x / div, inv, a.R.q, a.R.barrett);
                    row[c] = l;
                }
            }
            s_l[li] = l;
        }
        __syncthreads();
        const int width = cend - c - 1;
        if (width > 0) {
            const int total = nloc * width;
            for (int e = threadIdx.x; e < total; e += blockDim.x) {
                const int li = e / width, j = c + 1 + (e - li * width);
                const int i = row_begin + li;
                uint32_t* row = rowp(i);
                uint32_t y = row[j];
                const uint32_t l = s_l[li];
                if (l != 0) {
                    y = mod_sub(y, mod_mul(l, s_prow[j - a.c0], a.R.q, a.R.barrett), a.R.q);
                    row[j] = y;
                }
                if (j == c + 1 && i != prow && !is_pivot_row(i)) {
                    const unsigned long long key = pivot_key(y, i, a.R);
                    if (key != kNoKey) atomicMin(&s_cand, key);
                }
            }
        }
        publish_candidate(c + 1);
    }
    if (smem_rows) {
        __syncthreads();
        for (int i = row_begin + warp; i < row_end; i += kPanelWarps) {
            uint32_t* dst = a.A + static_cast<size_t>(i) * a.ld;
            const uint32_t* srow = rowp(i);
            for (int j = a.c0 + lane; j < cend; j += 32) dst[j] = srow[j];
        }
    }
    if (ok && blockIdx.x == 0 && threadIdx.x == 0) *a.k_out = k;
}

// ---- the panel on one thread-block cluster ---------------------------------------
// The same factorisation as panel_factor_kernel, for panels whose active rows
// fit the shared memory of one cluster (up to kClusterMax CTAs).  Each CTA
// keeps its slice of rows in shared memory, column-major, for the whole panel;
// the per-column exchange goes through distributed shared memory.
//
// Fraction-free row updates.  A column step needs no modular inverse: with the
// pivot x_p = ell^v * w (w a unit) every other active row becomes
//     row <- (w * row - (x_i / ell^v) * pivot_row) * rho          (mod q)
// with rho = 2^-32 in the Montgomery arithmetic of odd q (one reduction per
// element) and rho = 1 for q = 2^k (wraparound).  Every active row, pivot-free
// or not, is multiplied by the same unit w * rho, so after step t the active
// rows hold S_t times the values of the classical elimination, S_t = prod of
// (w_s rho) over s < t, and (x_i / ell^v) is stored as the raw multiplier.  The
// classical multiplier is (x_i / ell^v) * w_t^-1 and the classical pivot row
// t is its frozen raw row times S_t^-1; valuations (and zero / non-zero) do
// not change under unit scaling, so the pivot sequence is the classical one.
// After the last column every CTA computes the w_t^-1 in parallel and the
// prefix products S_t^-1, and rescales its rows once: the panel leaves the
// kernel as panel_factor_kernel leaves it (entry for entry over a field and for
// unit pivots; for pivots of valuation v > 0 the multiplier x / ell^v is only
// defined mod ell^(k-v), and the kernel's lift, consistent with the row
// updates it made, may differ from that kernel's by a multiple of ell^(k-v)).
// Like that kernel it updates only the columns right of each pivot.
//
// Per column:
//   1. every CTA pushes its best pivot key and that row's values (columns
//      [c, cend)) into a receive slot of every CTA of the cluster;
//   2. one hardware cluster barrier (release / acquire), reached once per
//      column by every thread of every CTA whatever the data;
//   3. every warp takes the smallest key of the slots (a warp min), and the
//      CTA updates its rows with the pivot row from its own receive slot.
// Receive slots are double-buffered by column parity: a CTA writes slot parity
// (it & 1) of column it only after passing barrier it - 1, when every CTA has
// finished column it - 2.  A cluster barrier before the first push makes sure
// every CTA of the cluster runs before any shared memory of it is written;
// after the last barrier no CTA touches another's shared memory.
constexpr int kClusterThreads = 1024;  // threads per CTA: 512 or 1024 (template NT)
constexpr int kClusterMax = 16;
constexpr int kClusterSmemMax = 200 * 1024;
constexpr int kClusterRowsMax = kClusterThreads;  // rows per CTA: at most one row per thread
constexpr int kKeyRowBits = 27;                   // 32-bit pivot key: valuation << 27 | row
constexpr uint32_t kKeyRowMask = (1u << kKeyRowBits) - 1u;
constexpr uint32_t kNoKey32 = 0xffffffffu;

enum : int { kArithPow2 = 0, kArithMont31 = 1, kArithMont32 = 2 };

// column stride of the column-major slice: odd, so a warp storing one row's
// consecutive columns hits 32 different banks
__host__ __device__ constexpr int cluster_stride(int rows) { return rows | 1; }

__host__ __device__ constexpr size_t cluster_smem_bytes(int rows, int bw) {
    return sizeof(uint32_t) * static_cast<size_t>(cluster_stride(rows)) * bw + static_cast<size_t>(rows) + 16;
}

__device__ __forceinline__ void cluster_barrier_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t pivot_key32(uint32_t x, int row, const Ring& R) {
    if (x == 0) return kNoKey32;
    const uint32_t v = R.k == 1 ? 0u : R.max_v == 0 ? (x % R.ell == 0 ? 1u : 0u) : valuation(x, R, R.max_v);
    if (v > R.max_v) return kNoKey32;
    return (v << kKeyRowBits) | static_cast<uint32_t>(row);
}

// x / ell^v for x divisible by ell^v
__device__ __forceinline__ uint32_t div_pw(uint32_t x, uint32_t v, const Ring& R) {
    return v == 0 ? x : R.ell == 2 ? x >> v : x / R.pw[v];
}

// The negated multiplier as the row update wants it.
template <int ARITH>
__device__ __forceinline__ uint32_t ff_negate(uint32_t xp, const Ring& R) {
    if constexpr (ARITH == kArithPow2) return 0u - xp;
    else return xp == 0 ? 0u : R.q - xp;
}

// (w * y + xn * pr) * rho mod q, xn the negated multiplier (ff_negate)
template <int ARITH>
__device__ __forceinline__ uint32_t ff_update(uint32_t w, uint32_t y, uint32_t xn, uint32_t pr, const Ring& R) {
    if constexpr (ARITH == kArithPow2) {
        return (w * y + xn * pr) & (R.q - 1u);
    } else if constexpr (ARITH == kArithMont31) {
        // q < 2^31: both products < 2^62, t < 2^63, t + m q < 2^64
        const uint64_t t = static_cast<uint64_t>(w) * y + static_cast<uint64_t>(xn) * pr;
        const uint32_t mq = static_cast<uint32_t>(t) * R.mont_qinv;
        const uint32_t r = static_cast<uint32_t>((t + static_cast<uint64_t>(mq) * R.q) >> 32);
        return r >= R.q ? r - R.q : r;
    } else {
        return mod_add(mont_mul(w, y, R.q, R.mont_qinv), mont_mul(xn, pr, R.q, R.mont_qinv), R.q);
    }
}

// The scale tables of a fraction-free factorization with k pivots, raw pivots
// s_w[0..k): s_inv[t] = w_t^-1 and s_sinv[t] = S_t^-1 = prod_{s<t} (w_s rho)^-1
// for t <= kMaxPanel (rho = 2^-32 for the Montgomery forms, else 1).  Called by
// every thread of the CTA; ends with a CTA barrier.
template <int ARITH>
__device__ void ff_scale_tables(int k, const uint32_t* s_w, uint32_t* s_inv, uint32_t* s_sinv, const Ring& R) {
    const int lane = threadIdx.x & 31;
    for (int t = threadIdx.x; t < k; t += blockDim.x) s_inv[t] = unit_inverse(s_w[t], R);
    __syncthreads();
    if (threadIdx.x < 32) {
        const uint32_t q = R.q;
        const uint64_t bm = R.barrett;
        const uint32_t one = 1u % q;
        // rho^-1 = 2^32 mod q (Montgomery) or 1
        const uint32_t rinv = ARITH == kArithPow2 ? one : mont_mul(R.mont_r2, 1u, q, R.mont_qinv);
        uint32_t f[kMaxPanel / 32];
        uint32_t run = one;
#pragma unroll
        for (int e = 0; e < kMaxPanel / 32; ++e) {
            const int t = lane * (kMaxPanel / 32) + e;
            f[e] = t < k ? mod_mul(s_inv[t], rinv, q, bm) : one;
            run = mod_mul(run, f[e], q, bm);
        }
        // inclusive scan of the lane products, then exclusive per element
        uint32_t incl = run;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl = mod_mul(incl, y, q, bm);
        }
        uint32_t ex = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) ex = one;
#pragma unroll
        for (int e = 0; e < kMaxPanel / 32; ++e) {
            s_sinv[lane * (kMaxPanel / 32) + e] = ex;
            ex = mod_mul(ex, f[e], q, bm);
        }
        if (lane == 31) s_sinv[kMaxPanel] = ex;
    }
    __syncthreads();
}

template <int ARITH, int NT>
__global__ void __launch_bounds__(NT, 1) panel_cluster_kernel(const PanelArgs a) {
    extern __shared__ __align__(16) uint32_t s_dyn[];
    __shared__ uint32_t r_key[2][kClusterMax];               // pushed keys, by parity and sender
    __shared__ uint32_t r_row[2][kClusterMax][kMaxPanel];     // pushed candidate rows (from column c)
    __shared__ uint32_t s_cand[2];                            // this CTA's best key, by parity
    __shared__ uint32_t s_w[kMaxPanel];                       // unit part of each step's raw pivot
    __shared__ uint32_t s_inv[kMaxPanel];                     // its inverse
    __shared__ uint32_t s_sinv[kMaxPanel + 1];                // S_t^-1
    __shared__ int s_colstep[kMaxPanel];                      // step t of pivot column c0 + j; else -1 - pivots left of it

    // settled by the top-block path: the same in every CTA, before any cluster barrier
    if (a.skip != nullptr && *a.skip != 0) return;
    const uint32_t crank = cluster_ctarank(), csize = cluster_nctarank();
    const int rows = a.m - a.r0;
    const int rpc = (rows + static_cast<int>(csize) - 1) / static_cast<int>(csize);
    const int row_begin = a.r0 + static_cast<int>(crank) * rpc;
    const int nloc = max(0, min(a.m, row_begin + rpc) - row_begin);
    if (rpc > NT) {  // the host never launches this; the test is the same in every CTA, before any barrier
        if (crank == 0 && threadIdx.x == 0) atomicCAS(a.err, 0, DERR_LAUNCH_SHAPE);
        return;
    }
    const int bw = a.bw, rs = cluster_stride(rpc);
    uint32_t* S = s_dyn;                                                           // [bw][rs]
    unsigned char* s_step = reinterpret_cast<unsigned char*>(S + static_cast<size_t>(bw) * rs);  // [rpc]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int nwarps = NT / 32;
    // thread -> (row li, phase sub): consecutive threads take consecutive rows,
    // so a warp reads one column of consecutive rows; g threads share a row
    int lg = 0;
    while ((1 << lg) < nloc) ++lg;
    const int nslots = 1 << lg, g = NT >> lg;
    const int li = tid & (nslots - 1), sub = tid >> lg;
    const bool has_row = li < nloc;

    for (int r = warp; r < nloc; r += nwarps) {
        const uint32_t* src = a.A + static_cast<size_t>(row_begin + r) * a.ld + a.c0;
        for (int j = lane; j < bw; j += 32) S[j * rs + r] = src[j];
    }
    for (int i = tid; i < rpc; i += NT) s_step[i] = 0;
    for (int j = tid; j < bw; j += NT) s_colstep[j] = -1;
    if (tid == 0) s_cand[0] = s_cand[1] = kNoKey32;
    __syncthreads();
    {
        uint32_t key = kNoKey32;
        if (has_row && sub == 0) key = pivot_key32(S[li], row_begin + li, a.R);
        key = __reduce_min_sync(0xffffffffu, key);
        if (lane == 0 && key != kNoKey32) atomicMin(&s_cand[0], key);
    }
    // every CTA of the cluster runs (its shared memory may be written) and s_cand[0] is complete
    cluster_barrier_all();

    const uint32_t rkey_addr = smem_u32(&r_key[0][0]);
    const uint32_t rrow_addr = smem_u32(&r_row[0][0][0]);
    int k = 0;
    int pend_col = -1;  // ring mode: multiplier x / ell^v stored after the column's CTA barrier
    uint32_t pend_xp = 0;
    for (int it = 0; it < bw; ++it) {
        const int par = it & 1;
        if (pend_col >= 0) {
            S[pend_col * rs + li] = pend_xp;
            pend_col = -1;
        }
        // (1) push this CTA's candidate for column c0 + it to every CTA (itself included)
        {
            const uint32_t mine = s_cand[par];
            if (warp < static_cast<int>(csize)) {
                const uint32_t d = static_cast<uint32_t>(warp);
                const uint32_t slot = par * kClusterMax + crank;
                if (lane == 0) st_dsmem_u32(dsmem_addr(rkey_addr + 4u * slot, d), mine);
                if (mine != kNoKey32) {
                    const int lm = static_cast<int>(mine & kKeyRowMask) - row_begin;
                    const uint32_t dst = dsmem_addr(rrow_addr + 4u * slot * kMaxPanel, d);
                    for (int j = lane; j < bw - it; j += 32) st_dsmem_u32(dst + 4u * j, S[(it + j) * rs + lm]);
                }
            }
            if (tid == 0) s_cand[par ^ 1] = kNoKey32;  // collects column it + 1's candidate below
        }
        // (2) every push of this column lands before any CTA reads its slots
        cluster_barrier_all();
        // (3) the pivot: the smallest (valuation, row) key of the cluster
        const uint32_t kd = lane < static_cast<int>(csize) ? r_key[par][lane] : kNoKey32;
        const uint32_t pkey = __reduce_min_sync(0xffffffffu, kd);
        uint32_t key = kNoKey32;
        if (pkey == kNoKey32) {
            // no pivot in this column: every active row is unchanged; scan column it + 1
            if (tid == 0) s_colstep[it] = -1 - k;
            if (it + 1 < bw && has_row && sub == 0 && s_step[li] == 0)
                key = pivot_key32(S[(it + 1) * rs + li], row_begin + li, a.R);
        } else {
            const int owner = __ffs(__ballot_sync(0xffffffffu, kd == pkey)) - 1;
            const int prow = static_cast<int>(pkey & kKeyRowMask);
            const uint32_t v = pkey >> kKeyRowBits;
            const uint32_t* prv = r_row[par][owner];  // pivot row, column c0 + it at index 0
            const uint32_t w = div_pw(prv[0], v, a.R);
            const int oli = owner == static_cast<int>(crank) ? prow - row_begin : -1;
            if (tid == 0) {
                s_w[k] = w;
                s_colstep[it] = k;
                if (oli >= 0) s_step[oli] = static_cast<unsigned char>(k + 1);
                if (crank == 0) {
                    a.pivot_rows[k] = prow;
                    a.pivot_cols[k] = a.c0 + it;
                }
            }
            if (has_row && li != oli && s_step[li] == 0) {
                const uint32_t xp = div_pw(S[it * rs + li], v, a.R);
                const uint32_t xn = ff_negate<ARITH>(xp, a.R);
                int j = it + 1 + sub;
                uint32_t* sp = S + j * rs + li;
                const uint32_t* pp = prv + (j - it);
                const int sstep = g * rs;
                if (sub == 0 && j < bw) {  // column it + 1: the next column's candidate
                    const uint32_t y = ff_update<ARITH>(w, *sp, xn, *pp, a.R);
                    *sp = y;
                    key = pivot_key32(y, row_begin + li, a.R);
                    j += g;
                    sp += sstep;
                    pp += g;
                }
                for (; j + g < bw; j += 2 * g, sp += 2 * sstep, pp += 2 * g) {
                    const uint32_t y0 = ff_update<ARITH>(w, sp[0], xn, pp[0], a.R);
                    const uint32_t y1 = ff_update<ARITH>(w, sp[sstep], xn, pp[g], a.R);
                    sp[0] = y0;
                    sp[sstep] = y1;
                }
                if (j < bw) *sp = ff_update<ARITH>(w, *sp, xn, *pp, a.R);
                if (v != 0 && sub == 0) {
                    pend_col = it;
                    pend_xp = xp;
                }
            }
            ++k;
        }
        key = __reduce_min_sync(0xffffffffu, key);
        if (lane == 0 && key != kNoKey32) atomicMin(&s_cand[par ^ 1], key);
        __syncthreads();
    }
    if (pend_col >= 0) S[pend_col * rs + li] = pend_xp;

    // ---- back to the classical values: w_t^-1 and S_t^-1 = prod_{s<t} w_s^-1 rho^-1
    ff_scale_tables<ARITH>(k, s_w, s_inv, s_sinv, a.R);
    if (has_row) {
        const int st = s_step[li];
        const int tau = st ? st - 1 : k;  // the step that froze this row's scale
        const uint32_t sc = s_sinv[tau];
        for (int j = sub; j < bw; j += g) {
            // a multiplier of step t < tau: times w_t^-1; any other entry was last
            // scaled by the step before min(tau, pivots left of column j)
            const int t = s_colstep[j];
            const uint32_t f = t >= 0 ? (t < tau ? s_inv[t] : sc) : s_sinv[min(tau, -1 - t)];
            S[j * rs + li] = mod_mul(S[j * rs + li], f, a.R.q, a.R.barrett);
        }
    }
    __syncthreads();
    for (int r = warp; r < nloc; r += nwarps) {
        uint32_t* dst = a.A + static_cast<size_t>(row_begin + r) * a.ld + a.c0;
        for (int j = lane; j < bw; j += 32) dst[j] = S[j * rs + r];
    }
    if (crank == 0 && tid == 0) *a.k_out = k;
}

// ---- the top-block path of a field panel ---------------------------------------
// At step t of a panel the pivot is the topmost active row with a non-zero in
// column c0 + t.  If the first t steps took rows r0 .. r0+t-1, row r0 + t is
// the topmost active row, so it is the pivot exactly when its entry (after the
// first t steps) is non-zero -- and those entries depend only on the top
// rows.  Hence: when the nb x w top block B = A[r0 : r0+nb, c0 : c0+w) (nb =
// min(w, m - r0)) factors with non-zero diagonal entries, the panel's pivots
// are (r0 + t, c0 + t), t < nb, the same as the search finds, with no row
// moved.  The packed LU of the block is unique for that pivot sequence, and
// the rest of the elimination step is one product:
//   [A12; A22] += [L^-1 - I; -A21 B^-1] A12
// gives U12 = L^-1 A12 in the top rows and the Schur complement A22 - A21 B^-1
// A12 below (B = L U, nb = w whenever rows remain below).  When a diagonal
// entry is zero, nothing is written and the searching kernel factors the panel.
struct BlockArgs {
    uint32_t* A;
    uint64_t ld;
    int m, r0, c0, w;
    Ring R;
    int* pivot_rows;  // [w] out
    int* pivot_cols;  // [w] out
    int* k_out;       // out
    int* ok;          // out: 1 when the top block settled the panel, else 0
    uint32_t* lm;     // out: L's strict lower part, Montgomery form (nb x nb, row-major, zero elsewhere)
    uint32_t* um;     // out: U's strict upper part, Montgomery form (nb x nb, row-major, zero elsewhere)
    uint32_t* dm;     // out: U's inverse diagonal, Montgomery form (nb)
};
constexpr int kBlockThreads = 512;

__host__ __device__ constexpr int block_stride(int w) { return w | 1; }
__host__ __device__ constexpr size_t block_smem_bytes(int nb, int w) {
    return sizeof(uint32_t) * static_cast<size_t>(nb) * block_stride(w);  // T = B, nb x w
}

// x * y with y in the Montgomery form (y 2^32 mod q) for odd q: one Montgomery
// reduction gives x y mod q; plain products for q = 2^k.
template <int ARITH>
__device__ __forceinline__ uint32_t mul_mform(uint32_t x, uint32_t ym, const Ring& R) {
    if constexpr (ARITH == kArithPow2) return (x * ym) & (R.q - 1u);
    else return mont_mul(x, ym, R.q, R.mont_qinv);
}

// x -> its Montgomery form x 2^32 mod q (unchanged for q = 2^k)
template <int ARITH>
__device__ __forceinline__ uint32_t to_mform(uint32_t x, const Ring& R) {
    if constexpr (ARITH == kArithPow2) return x;
    else return mont_mul(x, R.mont_r2, R.q, R.mont_qinv);
}

// One CTA: the fraction-free LU of the top block without a search (row t
// pivots at step t), one CTA barrier per step.  Step t touches only the
// active block (rows t+1 .. nb-1, columns t+1 .. w-1): warps over rows, lanes
// over columns, each row's operands loaded before its updates are computed.
// The classical values are restored as in the cluster kernel and written
// back; L, U and U's inverse diagonal go out in Montgomery form for the row
// solves of panel_binv_kernel.  WMAX (64 or 128) bounds w.
template <int ARITH, int WMAX>
__global__ void __launch_bounds__(kBlockThreads) panel_block_kernel(const BlockArgs a) {
    extern __shared__ __align__(16) uint32_t s_blk[];
    __shared__ uint32_t s_w[kMaxPanel], s_inv[kMaxPanel], s_sinv[kMaxPanel + 1];
    const int w = a.w, nb = min(w, a.m - a.r0), ts = block_stride(w);
    uint32_t* T = s_blk;  // [nb][ts]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = kBlockThreads / 32;
    constexpr int CW = WMAX / 32;  // column slots per lane
    constexpr int RI = WMAX / NW;  // row slots per warp
    for (int r = warp; r < nb; r += NW) {
        const uint32_t* src = a.A + static_cast<size_t>(a.r0 + r) * a.ld + a.c0;
#pragma unroll
        for (int c = 0; c < CW; ++c) {
            const int j = lane + 32 * c;
            if (j < w) T[r * ts + j] = src[j];
        }
    }
    __syncthreads();
    bool fail = false;
    for (int t = 0; t < nb; ++t) {
        const uint32_t wt = T[t * ts + t];
        // the pivot must be a unit (over a field: non-zero); the same value in every thread: uniform
        if (wt == 0 || (a.R.k > 1 && wt % a.R.ell == 0)) {
            fail = true;
            break;
        }
        if (tid == 0) s_w[t] = wt;
        const int jb = t + 1;
        uint32_t pr[CW];
#pragma unroll
        for (int c = 0; c < CW; ++c) {
            const int j = jb + lane + 32 * c;
            pr[c] = j < w ? T[t * ts + j] : 0u;
        }
#pragma unroll
        for (int i = 0; i < RI; ++i) {
            const int r = jb + warp + NW * i;
            if (r >= nb) break;  // uniform in the warp
            const uint32_t xn = ff_negate<ARITH>(T[r * ts + t], a.R);
            uint32_t y[CW];
#pragma unroll
            for (int c = 0; c < CW; ++c) {
                const int j = jb + lane + 32 * c;
                y[c] = j < w ? T[r * ts + j] : 0u;
            }
#pragma unroll
            for (int c = 0; c < CW; ++c) y[c] = ff_update<ARITH>(wt, y[c], xn, pr[c], a.R);
#pragma unroll
            for (int c = 0; c < CW; ++c) {
                const int j = jb + lane + 32 * c;
                if (j < w) T[r * ts + j] = y[c];
            }
        }
        __syncthreads();
    }
    if (fail) {
        if (tid == 0) *a.ok = 0;
        return;
    }
    if (tid < nb) s_w[tid] = T[tid * ts + tid];
    __syncthreads();
    ff_scale_tables<ARITH>(nb, s_w, s_inv, s_sinv, a.R);
    // row r froze at step r: a multiplier of step j < r takes w_j^-1, the rest (U) S_r^-1
    for (int r = warp; r < nb; r += NW) {
        uint32_t* dst = a.A + static_cast<size_t>(a.r0 + r) * a.ld + a.c0;
        for (int j = lane; j < w; j += 32) {
            const uint32_t v = mod_mul(T[r * ts + j], j < r ? s_inv[j] : s_sinv[r], a.R.q, a.R.barrett);
            dst[j] = v;
            if (j < nb) {
                a.lm[static_cast<size_t>(r) * nb + j] = j < r ? to_mform<ARITH>(v, a.R) : 0u;
                a.um[static_cast<size_t>(r) * nb + j] = j > r ? to_mform<ARITH>(v, a.R) : 0u;
            }
            if (j == r) T[r * ts + r] = v;  // the classical diagonal, for its inverse below
        }
    }
    if (tid < nb) {
        a.pivot_rows[tid] = a.r0 + tid;
        a.pivot_cols[tid] = a.c0 + tid;
    }
    __syncthreads();
    if (tid < nb) a.dm[tid] = to_mform<ARITH>(unit_inverse(T[tid * ts + tid], a.R), a.R);
    if (tid == 0) {
        *a.k_out = nb;
        *a.ok = 1;
    }
}

// Row solves against the factored top block, one warp per row, lanes over
// columns: the forward solve y U = v (y_s = (v_s - sum_{t<s} y_t U[t][s]) /
// U[s][s]) and the backward solve z L = y (z_i = y_i - sum_{t>i} z_t L[t][i],
// unit diagonal).  L, U and U's inverse diagonal come in Montgomery form, so
// each product is one Montgomery reduction.  panel_binv_kernel runs 2 nb of
// them: row r of B^-1 = e_r U^-1 L^-1 (when rows remain below the block) and
// row t of L^-1 (stored as L^-1 - I, the top rows of the update's left
// factor).  Nothing runs unless the top block settled the panel.
constexpr int kSolveWarps = 4;

template <int ARITH, int WMAX>
__global__ void __launch_bounds__(32 * kSolveWarps) panel_binv_kernel(const uint32_t* __restrict__ lm,
                                                                       const uint32_t* __restrict__ um,
                                                                       const uint32_t* __restrict__ dm, int nb,
                                                                       int with_binv, const Ring R,
                                                                       const int* __restrict__ ok,
                                                                       uint32_t* __restrict__ binv,
                                                                       uint32_t* __restrict__ linv) {
    if (*ok == 0) return;
    extern __shared__ __align__(16) uint32_t s_sv[];
    uint32_t* Ls = s_sv;                                                      // [nb][nb]
    uint32_t* Us = s_sv + ((static_cast<size_t>(nb) * nb + 3) & ~size_t(3));  // [nb][nb]
    __shared__ uint32_t s_dm[kMaxPanel];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int CS = WMAX / 32;
    for (int idx = tid; idx < nb * nb; idx += 32 * kSolveWarps) {
        Ls[idx] = lm[idx];
        if (with_binv) Us[idx] = um[idx];
    }
    for (int t = tid; t < nb; t += 32 * kSolveWarps) s_dm[t] = dm[t];
    __syncthreads();
    const int v = static_cast<int>(blockIdx.x) * kSolveWarps + warp;  // virtual row
    const bool is_binv = v < nb;
    const int r = is_binv ? v : v - nb;
    if (r >= nb || (is_binv && !with_binv)) return;  // uniform in the warp; no barrier follows
    const uint32_t one = 1u % R.q;
    uint32_t a[CS];
#pragma unroll
    for (int c = 0; c < CS; ++c) a[c] = lane + 32 * c == r ? one : 0u;
    if (is_binv) {
        // forward solve from e_r: y_s = 0 for s < r
#pragma unroll
        for (int sc = 0; sc < CS; ++sc) {
            for (int sl = 0; sl < 32; ++sl) {
                const int s = 32 * sc + sl;
                if (s >= nb) break;
                if (s < r) continue;
                const uint32_t ys = mul_mform<ARITH>(__shfl_sync(0xffffffffu, a[sc], sl), s_dm[s], R);
                if (lane == sl) a[sc] = ys;
#pragma unroll
                for (int c = sc; c < CS; ++c) {
                    const int j = lane + 32 * c;
                    const uint32_t u = j > s && j < nb ? Us[s * nb + j] : 0u;
                    a[c] = mod_sub(a[c], mul_mform<ARITH>(ys, u, R), R.q);
                }
            }
        }
    }
    // backward solve z L = y
#pragma unroll
    for (int sc = CS - 1; sc >= 0; --sc) {
        for (int sl = 31; sl >= 0; --sl) {
            const int t = 32 * sc + sl;
            if (t >= nb || t == 0) continue;
            const uint32_t zt = __shfl_sync(0xffffffffu, a[sc], sl);
#pragma unroll
            for (int c = 0; c <= sc; ++c) {
                const int j = lane + 32 * c;
                const uint32_t l = j < t ? Ls[t * nb + j] : 0u;
                a[c] = mod_sub(a[c], mul_mform<ARITH>(zt, l, R), R.q);
            }
        }
    }
    uint32_t* dst = (is_binv ? binv : linv) + static_cast<size_t>(r) * nb;
#pragma unroll
    for (int c = 0; c < CS; ++c) {
        const int j = lane + 32 * c;
        if (j < nb) dst[j] = !is_binv && j == r ? mod_sub(a[c], one, R.q) : a[c];
    }
}

// The left factor of the fused update, W ((m - r0) x nb, row-major, ld nb):
// rows t < nb are L^-1 - I (from panel_binv_kernel); a row x below the block
// becomes -x B^-1 (x = the row's panel columns).  A warp takes four rows at
// once, lanes over output columns; each dot product runs exactly in a 96-bit
// carry chain (nb <= 128 products below 2^64) and is reduced once.
constexpr int kWRows = 32;
constexpr int kWRowsPerWarp = 4;

template <int WMAX>
__global__ void __launch_bounds__(256) panel_w_kernel(const uint32_t* __restrict__ A, uint64_t ld, int r0, int m,
                                                      int c0, int nb, const uint32_t* __restrict__ linv,
                                                      const uint32_t* __restrict__ binv, uint32_t q,
                                                      uint64_t barrett, uint32_t* __restrict__ W) {
    extern __shared__ __align__(16) uint32_t s_wk[];
    const int rb = r0 + static_cast<int>(blockIdx.x) * kWRows;  // first row of this CTA
    const int nr = min(kWRows, m - rb);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = 256 / 32;
    static_assert(NW * kWRowsPerWarp == kWRows, "one pass of the warps covers the CTA's rows");
    constexpr int CS = WMAX / 32;
    // the top rows: L^-1 - I
    for (int r = warp; r < nr; r += NW) {
        const int row = rb + r;
        if (row >= r0 + nb) break;
        for (int j = lane; j < nb; j += 32)
            W[static_cast<size_t>(row - r0) * nb + j] = linv[static_cast<size_t>(row - r0) * nb + j];
    }
    if (rb + nr <= r0 + nb) return;  // no row below the block in this CTA (uniform)
    uint32_t* Bi = s_wk;                                   // [nb][nb]
    uint32_t* Xr = s_wk + ((static_cast<size_t>(nb) * nb + 3) & ~size_t(3));  // [kWRows][nb]
    {
        // B^-1 in 16-byte pieces (its buffer is 16-byte aligned), four loads of a thread in flight
        const int n4 = (nb * nb) >> 2;
        const uint4* b4 = reinterpret_cast<const uint4*>(binv);
        uint4* d4 = reinterpret_cast<uint4*>(Bi);
        for (int base = 0; base < n4; base += 256 * 4) {
            uint4 v[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int idx = base + tid + 256 * e;
                if (idx < n4) v[e] = b4[idx];
            }
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int idx = base + tid + 256 * e;
                if (idx < n4) d4[idx] = v[e];
            }
        }
        for (int idx = 4 * n4 + tid; idx < nb * nb; idx += 256) Bi[idx] = binv[idx];
    }
    const int rl = warp * kWRowsPerWarp;  // this warp's rows: rl .. rl + 3 of the CTA
    {
        uint32_t v[kWRowsPerWarp][CS];
#pragma unroll
        for (int i = 0; i < kWRowsPerWarp; ++i) {
            const int row = rb + rl + i;
            const bool below = rl + i < nr && row >= r0 + nb;
            const uint32_t* src = A + static_cast<size_t>(below ? row : r0) * ld + c0;
#pragma unroll
            for (int c = 0; c < CS; ++c) {
                const int j = lane + 32 * c;
                v[i][c] = below && j < nb ? src[j] : 0u;
            }
        }
#pragma unroll
        for (int i = 0; i < kWRowsPerWarp; ++i)
#pragma unroll
            for (int c = 0; c < CS; ++c) {
                const int j = lane + 32 * c;
                if (j < nb) Xr[(rl + i) * nb + j] = v[i][c];
            }
    }
    __syncthreads();
    uint32_t a0[kWRowsPerWarp][CS], a1[kWRowsPerWarp][CS], a2[kWRowsPerWarp][CS];
#pragma unroll
    for (int i = 0; i < kWRowsPerWarp; ++i)
#pragma unroll
        for (int c = 0; c < CS; ++c) a0[i][c] = a1[i][c] = a2[i][c] = 0;
    for (int t = 0; t < nb; ++t) {
        uint32_t bt[CS];
#pragma unroll
        for (int c = 0; c < CS; ++c) {
            const int j = lane + 32 * c;
            bt[c] = j < nb ? Bi[t * nb + j] : 0u;
        }
#pragma unroll
        for (int i = 0; i < kWRowsPerWarp; ++i) {
            const uint32_t x = Xr[(rl + i) * nb + t];
#pragma unroll
            for (int c = 0; c < CS; ++c) mac96(a0[i][c], a1[i][c], a2[i][c], x, bt[c]);
        }
    }
#pragma unroll
    for (int i = 0; i < kWRowsPerWarp; ++i) {
        const int row = rb + rl + i;
        if (rl + i >= nr || row < r0 + nb) continue;
        uint32_t* dst = W + static_cast<size_t>(row - r0) * nb;
#pragma unroll
        for (int c = 0; c < CS; ++c) {
            const int j = lane + 32 * c;
            if (j < nb) {
                const uint64_t h = reduce_u64((static_cast<uint64_t>(a2[i][c]) << 32) | a1[i][c], q, barrett);
                const uint32_t v = static_cast<uint32_t>(reduce_u64((h << 32) | a0[i][c], q, barrett));
                dst[j] = v == 0 ? 0u : q - v;
            }
        }
    }
}

// ---- row permutation of columns [c0, n) for rows [r0, m) -------------------------
// tmp[i'][j'] = A[perm[i']][c0 + j']
__global__ void gather_rows_kernel(const uint32_t* __restrict__ A, uint64_t ld, const int* __restrict__ perm,
                                   int rows, int c0, int cols, uint32_t* __restrict__ tmp) {
    const size_t total = static_cast<size_t>(rows) * cols;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(idx / cols), j = static_cast<int>(idx % cols);
        tmp[idx] = A[static_cast<size_t>(perm[i]) * ld + c0 + j];
    }
}
__global__ void scatter_rows_kernel(uint32_t* __restrict__ A, uint64_t ld, int r0, int rows, int c0, int cols,
                                    const uint32_t* __restrict__ tmp) {
    const size_t total = static_cast<size_t>(rows) * cols;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(idx / cols), j = static_cast<int>(idx % cols);
        A[static_cast<size_t>(r0 + i) * ld + c0 + j] = tmp[idx];
    }
}

// dst[i][t] = A[row0 + i][cols[t]]  (rows x k, ld k)
__global__ void gather_cols_kernel(const uint32_t* __restrict__ A, uint64_t ld, int row0, int rows,
                                   const int* __restrict__ cols, int k, uint32_t* __restrict__ dst) {
    const size_t total = static_cast<size_t>(rows) * k;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(idx / k), t = static_cast<int>(idx % k);
        dst[idx] = A[static_cast<size_t>(row0 + i) * ld + cols[t]];
    }
}

// Inverses of triangular diagonal blocks, one CTA per block.  Block b covers
// rows [row0 + b*bb, row0 + b*bb + nb) of A and the pivot columns
// pcols[b*bb ..]: T(t, s) = A[row0 + b*bb + t][pcols[b*bb + s]].
//   UPPER: T upper triangular with non-zero diagonal (the U1 blocks of the RREF)
//   !UPPER: T unit lower triangular, strictly-lower part read (the L11 of a panel)
// out + b*bb*bb receives T^-1 (nb x nb, row-major, ld nb).
// UPPER is reduced to the unit case: T = D T' with D its diagonal, and
// T^-1 = T'^-1 D^-1 (columns of T'^-1 scaled on the way out).  The unit
// triangular inverse X = T'^-1 is built right-looking from X = I: at step t
// row t of X is final, and every later row r (earlier, for UPPER) takes
// X[r] -= T'[r][t] * X[t] over the non-zero columns of X[t] -- one rank-1
// update and one CTA barrier per step, lanes over columns, warps over rows.
template <bool UPPER>
__global__ void __launch_bounds__(1024) tri_inv_kernel(const uint32_t* __restrict__ A, uint64_t ld, int row0,
                                                       const int* __restrict__ pcols, int total, int bb, uint32_t p,
                                                       uint64_t barrett, uint32_t kmax, uint32_t* __restrict__ out) {
    extern __shared__ uint32_t smem_ti[];
    (void)kmax;
    const int i0 = blockIdx.x * bb;
    const int nb = min(bb, total - i0);
    uint32_t* T = smem_ti;             // nb x nb: T' (unit diagonal implied)
    uint32_t* X = smem_ti + nb * nb;   // nb x nb
    uint32_t* dinv = X + nb * nb;      // nb
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int t = threadIdx.x; t < nb; t += blockDim.x)
        dinv[t] = UPPER ? inv_binary_xgcd(A[static_cast<size_t>(row0 + i0 + t) * ld + pcols[i0 + t]], p) : 1u % p;
    __syncthreads();
    for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
        const int t = idx / nb, s2 = idx - t * nb;
        const bool keep = UPPER ? (s2 > t) : (s2 < t);
        uint32_t v = keep ? A[static_cast<size_t>(row0 + i0 + t) * ld + pcols[i0 + s2]] : 0u;
        if (UPPER && keep) v = mod_mul(v, dinv[t], p, barrett);
        T[idx] = v;
        X[idx] = s2 == t ? 1u % p : 0u;
    }
    __syncthreads();
    for (int st = 0; st + 1 < nb; ++st) {
        const int t = UPPER ? nb - 1 - st : st;
        // LOWER: rows r > t, columns j <= t;  UPPER: rows r < t, columns j >= t
        const int rbeg = UPPER ? 0 : t + 1, rend = UPPER ? t : nb;
        const int jbeg = UPPER ? t : 0, jend = UPPER ? nb : t + 1;
        const uint32_t* xt = X + t * nb;
        for (int r = rbeg + warp; r < rend; r += nw) {
            const uint32_t l = T[r * nb + t];
            if (l == 0) continue;
            const uint32_t nl = p - l;
            uint32_t* xr = X + r * nb;
            for (int j = jbeg + lane; j < jend; j += 32)
                xr[j] = reduce_u64(static_cast<uint64_t>(nl) * xt[j] + xr[j], p, barrett);
        }
        __syncthreads();
    }
    uint32_t* o = out + static_cast<size_t>(blockIdx.x) * bb * bb;
    for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
        const uint32_t v = X[idx];
        o[idx] = UPPER ? mod_mul(v, dinv[idx % nb], p, barrett) : v;
    }
}

// U12 = L11^-1 A12 in place.  L11: the unit-lower k x k block of the panel's
// pivot rows (rows row0 .. row0+k-1 of A) at the pivot columns pcols[0..k),
// strictly-lower part read; A12: the same rows at columns [c1, c1 + trail).
// Each CTA takes kTrsmCols columns into shared memory; forward substitution
// runs per column in one warp, lane l holding rows l, l+32, l+64, l+96 in
// registers: at step t the value of row t is final, a shuffle broadcasts it,
// and every later row r takes x_r -= L[r][t] x_t.  The columns are
// independent, so after the loads no block barrier is needed until the
// write-back.  L11 sits in shared memory with an odd row stride, so the 32
// lanes reading L[r][t] for 32 rows hit 32 banks.
constexpr int kTrsmCols = 32;

__global__ void __launch_bounds__(32 * kTrsmCols) trsm_unit_lower_kernel(uint32_t* __restrict__ A, uint64_t ld,
                                                                         int row0, const int* __restrict__ pcols,
                                                                         int k, int c1, int trail, uint32_t p,
                                                                         uint64_t barrett) {
    extern __shared__ uint32_t smem_tr[];
    const int ls = k | 1;
    constexpr int xs = kTrsmCols + 1;
    uint32_t* Ls = smem_tr;               // [k][ls]
    uint32_t* X = smem_tr + k * ls;       // [k][xs]
    const int cbase = c1 + static_cast<int>(blockIdx.x) * kTrsmCols;
    const int ncols = min(kTrsmCols, c1 + trail - cbase);
    for (int idx = threadIdx.x; idx < k * k; idx += blockDim.x) {
        const int r = idx / k, t = idx - r * k;
        Ls[r * ls + t] = t < r ? A[static_cast<size_t>(row0 + r) * ld + pcols[t]] : 0u;
    }
    for (int idx = threadIdx.x; idx < k * kTrsmCols; idx += blockDim.x) {
        const int r = idx / kTrsmCols, c = idx - r * kTrsmCols;
        X[r * xs + c] = c < ncols ? A[static_cast<size_t>(row0 + r) * ld + cbase + c] : 0u;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp < ncols) {
        uint32_t x[kMaxPanel / 32];
#pragma unroll
        for (int q = 0; q < kMaxPanel / 32; ++q) {
            const int r = lane + 32 * q;
            x[q] = r < k ? X[r * xs + warp] : 0u;
        }
#pragma unroll
        for (int qt = 0; qt < kMaxPanel / 32; ++qt) {
            if (32 * qt >= k - 1) break;
            for (int tt = 0; tt < 32; ++tt) {
                const int t = 32 * qt + tt;
                if (t >= k - 1) break;
                const uint32_t xt = __shfl_sync(0xffffffffu, x[qt], tt);
#pragma unroll
                for (int q = qt; q < kMaxPanel / 32; ++q) {
                    const int r = lane + 32 * q;
                    if (r > t && r < k) {
                        const uint32_t l = Ls[r * ls + t];
                        if (l) x[q] = reduce_u64(static_cast<uint64_t>(p - l) * xt + x[q], p, barrett);
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kMaxPanel / 32; ++q) {
            const int r = lane + 32 * q;
            if (r < k) X[r * xs + warp] = x[q];
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < k * kTrsmCols; idx += blockDim.x) {
        const int r = idx / kTrsmCols, c = idx - r * kTrsmCols;
        if (c < ncols) A[static_cast<size_t>(row0 + r) * ld + cbase + c] = X[r * xs + c];
    }
}

size_t trsm_smem_bytes(int k) {
    return sizeof(uint32_t) * (static_cast<size_t>(k) * (k | 1) + static_cast<size_t>(k) * (kTrsmCols + 1));
}

// R (m x n, ld ldr): rows < rank: identity at the pivot columns, X at the free
// columns; rows >= rank: zero.
__global__ void assemble_rref_kernel(uint32_t* __restrict__ R, uint64_t ldr, int m, int n, int rank,
                                     const int* __restrict__ colmap, const uint32_t* __restrict__ X, int f) {
    // colmap[j] >= 0: pivot index of pivot column j; colmap[j] = -1 - t: free column number t
    const size_t total = static_cast<size_t>(m) * n;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(idx / n), j = static_cast<int>(idx % n);
        uint32_t v = 0;
        if (i < rank) {
            const int cm = colmap[j];
            v = cm >= 0 ? (cm == i ? 1u : 0u) : X[static_cast<size_t>(i) * f + (-1 - cm)];
        }
        R[static_cast<size_t>(i) * ldr + j] = v;
    }
}

// diag[t] = A[t][pivots[t]]
__global__ void gather_diag_kernel(const uint32_t* __restrict__ A, uint64_t ld, const int* __restrict__ piv, int rank,
                                   uint32_t* __restrict__ diag) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < rank; t += gridDim.x * blockDim.x)
        diag[t] = A[static_cast<size_t>(t) * ld + piv[t]];
}

uint32_t kmax_for(uint32_t p) {
    const uint64_t d = static_cast<uint64_t>(p - 1) * (p - 1);
    uint64_t km = d == 0 ? 1024 : (~0ull) / d;
    return static_cast<uint32_t>(std::min<uint64_t>(km, 1024));
}

int grid_1d(size_t work, int sms) {
    return static_cast<int>(std::max<size_t>(1, std::min<size_t>((work + 255) / 256, static_cast<size_t>(sms) * 8)));
}

}  // namespace

// ---------------------------------------------------------------------------------
ElimResult elim_device(hme_ctx* ctx, const ModParams& mp, uint32_t* A, size_t ld, int m, int n, bool want_rref,
                       uint32_t* R, size_t ldr, const ElimOptions& opt, const RingSpec* ring) {
    HME_REQUIRE(m >= 0 && n >= 0, "elim: negative shape");
    HME_REQUIRE(!(want_rref && ring && ring->k > 1), "elim: the RREF is a field-only object");
    ElimResult res;
    res.sign_negative = false;
    if (m == 0 || n == 0) {
        if (want_rref && m > 0 && n > 0) HME_CUDA(cudaMemsetAsync(R, 0, 1, ctx->stream));
        return res;
    }
    const int bw = std::max(1, std::min<int>(opt.panel > 0 ? opt.panel : 64, kMaxPanel));
    const uint32_t p = mp.p;
    // the ring: F_p by default, Z/ell^k with a pivot valuation bound when given
    Ring rg{};
    rg.q = p;
    rg.barrett = mp.barrett;
    rg.ell = ring ? ring->ell : p;
    rg.k = ring ? ring->k : 1;
    rg.max_v = ring ? ring->max_v : 0;
    {
        uint64_t pw = 1;
        for (uint32_t v = 0; v <= rg.k && v < 32; ++v) {
            rg.pw[v] = static_cast<uint32_t>(pw);
            pw *= rg.ell;
        }
        HME_REQUIRE(static_cast<uint64_t>(rg.pw[rg.k]) == p || rg.k == 1, "elim: modulus is not ell^k");
        // phi(ell^k) - 1 = ell^(k-1) (ell - 1) - 1
        rg.unit_exp = static_cast<uint32_t>(static_cast<uint64_t>(rg.pw[rg.k - 1]) * (rg.ell - 1) - 1);
    }
    if (p & 1u) {
        uint32_t x = p;  // p^-1 mod 2^32 by Newton's iteration (x = p is right to 3 bits)
        for (int i = 0; i < 5; ++i) x *= 2u - p * x;
        rg.mont_qinv = 0u - x;
        rg.mont_r2 = static_cast<uint32_t>(((static_cast<unsigned __int128>(1) << 64)) % p);
    }
    const int lu_cols = ring && ring->lu_cols > 0 ? std::min(ring->lu_cols, n) : n;

    static OncePerDevice attr;
    // per device: the largest cluster the panel kernel can be launched with (0: none)
    static int cluster_caps[OncePerDevice::kMaxDevices] = {};
    attr.run([](int dev) {
        int& cluster_cap = cluster_caps[dev];
        cluster_cap = 0;
        HME_CUDA(cudaFuncSetAttribute(panel_factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPanelSmemMax));
        {
            const int bsm = static_cast<int>(block_smem_bytes(kMaxPanel, kMaxPanel));
            for (const void* fn : {reinterpret_cast<const void*>(panel_block_kernel<kArithPow2, 64>),
                                   reinterpret_cast<const void*>(panel_block_kernel<kArithMont31, 64>),
                                   reinterpret_cast<const void*>(panel_block_kernel<kArithMont32, 64>),
                                   reinterpret_cast<const void*>(panel_block_kernel<kArithPow2, 128>),
                                   reinterpret_cast<const void*>(panel_block_kernel<kArithMont31, 128>),
                                   reinterpret_cast<const void*>(panel_block_kernel<kArithMont32, 128>)})
                HME_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bsm));
            const int wsm = static_cast<int>(sizeof(uint32_t) * (kMaxPanel * kMaxPanel + kWRows * kMaxPanel));
            HME_CUDA(cudaFuncSetAttribute(panel_w_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, wsm));
            HME_CUDA(cudaFuncSetAttribute(panel_w_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, wsm));
            const int ssm = static_cast<int>(2 * sizeof(uint32_t) * kMaxPanel * kMaxPanel);
            for (const void* fn : {reinterpret_cast<const void*>(panel_binv_kernel<kArithPow2, 64>),
                                   reinterpret_cast<const void*>(panel_binv_kernel<kArithMont31, 64>),
                                   reinterpret_cast<const void*>(panel_binv_kernel<kArithMont32, 64>),
                                   reinterpret_cast<const void*>(panel_binv_kernel<kArithPow2, 128>),
                                   reinterpret_cast<const void*>(panel_binv_kernel<kArithMont31, 128>),
                                   reinterpret_cast<const void*>(panel_binv_kernel<kArithMont32, 128>)})
                HME_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, ssm));
        }
        bool attrs_ok = true;
        for (const void* fn : {reinterpret_cast<const void*>(panel_cluster_kernel<kArithPow2, 512>),
                               reinterpret_cast<const void*>(panel_cluster_kernel<kArithMont31, 512>),
                               reinterpret_cast<const void*>(panel_cluster_kernel<kArithMont32, 512>),
                               reinterpret_cast<const void*>(panel_cluster_kernel<kArithPow2, 1024>),
                               reinterpret_cast<const void*>(panel_cluster_kernel<kArithMont31, 1024>),
                               reinterpret_cast<const void*>(panel_cluster_kernel<kArithMont32, 1024>)}) {
            attrs_ok = attrs_ok &&
                       cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kClusterSmemMax) ==
                           cudaSuccess &&
                       cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess;
        }
        if (attrs_ok) {
            for (int cs = kClusterMax; cs >= 1 && cluster_cap == 0; cs /= 2) {
                cudaLaunchConfig_t cfg{};
                cfg.gridDim = dim3(cs);
                cfg.blockDim = dim3(kClusterThreads);
                cfg.dynamicSmemBytes = kClusterSmemMax;
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeClusterDimension;
                at[0].val.clusterDim.x = cs;
                at[0].val.clusterDim.y = 1;
                at[0].val.clusterDim.z = 1;
                cfg.attrs = at;
                cfg.numAttrs = 1;
                int n = 0;
                if (cudaOccupancyMaxActiveClusters(&n, panel_cluster_kernel<kArithMont31, 1024>, &cfg) == cudaSuccess &&
                    n >= 1)
                    cluster_cap = cs;
            }
        }
        cudaGetLastError();  // a refused query leaves no error behind
        const int smem2 = sizeof(uint32_t) * (2 * kMaxPanel * kMaxPanel + kMaxPanel);
        HME_CUDA(cudaFuncSetAttribute(tri_inv_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem2));
        HME_CUDA(cudaFuncSetAttribute(tri_inv_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem2));
        HME_CUDA(cudaFuncSetAttribute(trsm_unit_lower_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(trsm_smem_bytes(kMaxPanel))));
    });
    const int cluster_cap = cluster_caps[ctx->device];

    // device scratch: two sets (by panel parity), so that the next panel, factored ahead on the
    // second stream, never writes the pivot lists the current panel's update still reads
    const int grid_cap = std::max(1, std::min(ctx->num_sms, opt.panel_ctas > 0 ? opt.panel_ctas : ctx->num_sms));
    struct Scratch {
        unsigned long long piv_slot[kMaxPanel];
        int pivot_rows[kMaxPanel];
        int pivot_cols[kMaxPanel];
        int k;
        int err;       // the device error word as of the panel's end
        int block_ok;  // the top-block path settled the panel
        unsigned bar[2];
    };
    const size_t scratch_bytes = (sizeof(Scratch) + 255) / 256 * 256;
    const size_t cand_bytes = sizeof(uint32_t) * 2 * static_cast<size_t>(grid_cap) * kMaxPanel;
    const size_t perm_bytes = (sizeof(int) * static_cast<size_t>(m) + 255) / 256 * 256;
    const size_t uinv_bytes = sizeof(uint32_t) * (4 * kMaxPanel * kMaxPanel + kMaxPanel);  // L, U, B^-1, L^-1 - I, 1/diag U
    uint8_t* base = static_cast<uint8_t*>(
        ctx->ws.get(kSlotElim0, 2 * (scratch_bytes + cand_bytes) + 2 * perm_bytes + 2 * uinv_bytes + 256));
    // the L21 / W slot at its largest (every panel's rows x pivots fits), so no panel regrows it
    ctx->ws.get(kSlotElim2, sizeof(uint32_t) * static_cast<size_t>(m) * bw);
    Scratch* d_sb[2] = {reinterpret_cast<Scratch*>(base), reinterpret_cast<Scratch*>(base + scratch_bytes)};
    uint32_t* d_candb[2] = {reinterpret_cast<uint32_t*>(base + 2 * scratch_bytes),
                            reinterpret_cast<uint32_t*>(base + 2 * scratch_bytes + cand_bytes)};
    int* d_permb[2] = {reinterpret_cast<int*>(base + 2 * (scratch_bytes + cand_bytes)),
                       reinterpret_cast<int*>(base + 2 * (scratch_bytes + cand_bytes) + perm_bytes)};
    uint32_t* d_uinvb[2] = {reinterpret_cast<uint32_t*>(base + 2 * (scratch_bytes + cand_bytes + perm_bytes)),
                            reinterpret_cast<uint32_t*>(base + 2 * (scratch_bytes + cand_bytes + perm_bytes) + uinv_bytes)};
    HME_CUDA(cudaMemsetAsync(d_sb[0]->bar, 0, sizeof(unsigned) * 2, ctx->stream));
    HME_CUDA(cudaMemsetAsync(d_sb[1]->bar, 0, sizeof(unsigned) * 2, ctx->stream));
    // pinned copies of the two scratch sets (the host reads a panel's pivots without waiting for
    // the other stream's work), the second stream and the events of the lookahead
    // (and two pinned permutation buffers: the host queues a panel's update behind the previous
    // one's without waiting for it)
    const size_t pinned_bytes = 2 * sizeof(Scratch) + 2 * sizeof(int) * static_cast<size_t>(m);
    if (ctx->elim_pinned_bytes < pinned_bytes) {
        if (ctx->elim_pinned) {
            HME_CUDA(cudaDeviceSynchronize());
            HME_CUDA(cudaFreeHost(ctx->elim_pinned));
            ctx->elim_pinned = nullptr;
            ctx->elim_pinned_bytes = 0;
        }
        HME_CUDA(cudaMallocHost(&ctx->elim_pinned, pinned_bytes));
        ctx->elim_pinned_bytes = pinned_bytes;
    }
    Scratch* h_sb = static_cast<Scratch*>(ctx->elim_pinned);
    int* h_permb[2] = {reinterpret_cast<int*>(h_sb + 2), reinterpret_cast<int*>(h_sb + 2) + m};
    if (!ctx->aux_stream) {
        // the lookahead panel's stream at the highest priority: its cluster takes SMs as they free up
        int lo = 0, hi = 0;
        HME_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        HME_CUDA(cudaStreamCreateWithPriority(&ctx->aux_stream, cudaStreamNonBlocking, hi));
    }
    while (ctx->elim_ev.size() < 3) {
        cudaEvent_t e;
        HME_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->elim_ev.push_back(e);
    }
    cudaEvent_t ev_next = ctx->elim_ev[0], ev_panel[2] = {ctx->elim_ev[1], ctx->elim_ev[2]};
    const cudaStream_t s_main = ctx->stream, s_aux = ctx->aux_stream;
    // lookahead only where it can overlap: the cluster kernel (a few SMs), and not while the
    // per-kernel timer is on (its events assume one stream)
    const bool allow_lookahead = !opt.no_lookahead && !ctx->timer.on;

    // The cluster kernel when the active rows fit the shared memory of one cluster: the cluster
    // doubles (up to the largest the device runs) until each CTA holds at most rows_per_cta rows,
    // and further while a slice does not fit.  Returns the cluster size, 0 for the grid kernel.
    auto cluster_size = [&](int rows, int w) -> int {
        int cs = 0;
        if (opt.panel_kernel != 1 && cluster_cap > 0) {
            const size_t want = static_cast<size_t>(std::max(1, opt.rows_per_cta > 0 ? opt.rows_per_cta : 32));
            auto rpc_of = [&](int c) { return (static_cast<size_t>(rows) + c - 1) / c; };
            auto fits = [&](int c) {
                const size_t rpc = rpc_of(c);
                return rpc <= static_cast<size_t>(kClusterRowsMax) &&
                       cluster_smem_bytes(static_cast<int>(rpc), w) <= static_cast<size_t>(kClusterSmemMax);
            };
            int c = 1;
            while (c < cluster_cap && (rpc_of(c) > want || !fits(c))) c *= 2;
            if (fits(c)) cs = c;
        }
        return cs;
    };

    // The panel [c0, c0 + w) of the active rows [r0, m) on `st`: its pivots and the error word
    // land in h_sb[par] and ev_panel[par] is recorded.  Returns the cluster size (0: grid kernel).
    // the top-block path: in automatic mode, over a field
    // the top-block path in automatic mode, over fields of at least 256 elements (a random top block
    // of 64 steps meets a zero pivot with probability about 64/p, so over small fields and over rings,
    // where a non-unit pivot is as likely, the attempts would mostly fail); after a panel it did not
    // settle, the next three panels go straight to the search (rank-deficient tails)
    const bool use_block = opt.panel_kernel == 0 && rg.k == 1 && p >= 256;
    int block_rest = 0;
    bool block_tried[2] = {false, false};
    // The panel [c0, c0 + w) of the active rows [r0, m) on `st`: the top-block path when it is tried
    // (the host launches the search afterwards if the block did not settle the panel), else the
    // searching kernel.  Its pivots and the error word land in h_sb[par] and ev_panel[par] is
    // recorded.  Returns the cluster size the search takes (0: grid kernel), the SMs a GEMM beside
    // the panel leaves free.
    cudaStream_t panel_stream[2] = {s_main, s_main};
    auto launch_panel = [&](int c0, int w, int r0, int par, cudaStream_t st, bool search_only) -> int {
        Scratch* d_s = d_sb[par];
        const cudaStream_t saved = ctx->stream;
        ctx->stream = st;  // HME_TIMED brackets the launch on the launching stream
        panel_stream[par] = st;
        PanelArgs pa{};
        pa.A = A;
        pa.ld = ld;
        pa.m = m;
        pa.c0 = c0;
        pa.bw = w;
        pa.r0 = r0;
        pa.R = rg;
        pa.piv_slot = d_s->piv_slot;
        pa.cand = d_candb[par];
        pa.pivot_rows = d_s->pivot_rows;
        pa.pivot_cols = d_s->pivot_cols;
        pa.k_out = &d_s->k;
        pa.bar = d_s->bar;
        pa.err = ctx->d_err;
        const int rows = m - r0;
        // the top-block path first; the searching kernel below runs only when the block did not
        // settle the panel
        const bool try_block = !search_only && use_block && block_rest == 0;
        if (!search_only && use_block && block_rest > 0) --block_rest;
        block_tried[par] = try_block;
        if (try_block) {
            const int nb = std::min(w, rows);
            BlockArgs ba{};
            ba.A = A;
            ba.ld = ld;
            ba.m = m;
            ba.r0 = r0;
            ba.c0 = c0;
            ba.w = w;
            ba.R = rg;
            ba.pivot_rows = d_s->pivot_rows;
            ba.pivot_cols = d_s->pivot_cols;
            ba.k_out = &d_s->k;
            ba.ok = &d_s->block_ok;
            ba.lm = d_uinvb[par];
            ba.um = d_uinvb[par] + kMaxPanel * kMaxPanel;
            ba.dm = d_uinvb[par] + 4 * kMaxPanel * kMaxPanel;
            const size_t bsm = block_smem_bytes(nb, w);
            auto launch_block = [&](auto kern) {
                HME_TIMED(ctx, "panel_block", kern<<<1, kBlockThreads, bsm, st>>>(ba));
            };
            const bool w64 = w <= 64;
            if (rg.ell == 2) {
                if (w64) launch_block(panel_block_kernel<kArithPow2, 64>);
                else launch_block(panel_block_kernel<kArithPow2, 128>);
            } else if (p < (1u << 31)) {
                if (w64) launch_block(panel_block_kernel<kArithMont31, 64>);
                else launch_block(panel_block_kernel<kArithMont31, 128>);
            } else {
                if (w64) launch_block(panel_block_kernel<kArithMont32, 64>);
                else launch_block(panel_block_kernel<kArithMont32, 128>);
            }
            HME_CUDA(cudaGetLastError());
            {
                // B^-1 (when rows remain below) and L^-1 - I by row solves, one warp per row
                const int with_binv = rows > nb ? 1 : 0;
                const int gs = (2 * nb + kSolveWarps - 1) / kSolveWarps;
                const size_t ssm = 2 * sizeof(uint32_t) * ((static_cast<size_t>(nb) * nb + 3) & ~size_t(3));
                uint32_t* sb = d_uinvb[par];
                auto launch_solve = [&](auto kern) {
                    HME_TIMED(ctx, "panel_block", kern<<<gs, 32 * kSolveWarps, ssm, st>>>(
                                                      sb, sb + kMaxPanel * kMaxPanel, sb + 4 * kMaxPanel * kMaxPanel, nb,
                                                      with_binv, rg, &d_s->block_ok, sb + 2 * kMaxPanel * kMaxPanel,
                                                      sb + 3 * kMaxPanel * kMaxPanel));
                };
                if (rg.ell == 2) {
                    if (w64) launch_solve(panel_binv_kernel<kArithPow2, 64>);
                    else launch_solve(panel_binv_kernel<kArithPow2, 128>);
                } else if (p < (1u << 31)) {
                    if (w64) launch_solve(panel_binv_kernel<kArithMont31, 64>);
                    else launch_solve(panel_binv_kernel<kArithMont31, 128>);
                } else {
                    if (w64) launch_solve(panel_binv_kernel<kArithMont32, 64>);
                    else launch_solve(panel_binv_kernel<kArithMont32, 128>);
                }
                HME_CUDA(cudaGetLastError());
            }
        }
        const int cs = cluster_size(rows, w);
        HME_REQUIRE(opt.panel_kernel < 2 || cs > 0, "elim: the panel does not fit one cluster");
        if (try_block) {
            // no search behind the block: the host relaunches the panel with the search if needed
        } else if (cs > 0) {
            const int rpc = static_cast<int>((static_cast<size_t>(rows) + cs - 1) / cs);
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3(cs);
            cfg.blockDim = dim3(kClusterThreads);
            cfg.dynamicSmemBytes = cluster_smem_bytes(rpc, w);
            cfg.stream = st;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = cs;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            // q = 2^k: wraparound; odd q < 2^31: one Montgomery reduction per element; else two.
            // 512 threads per CTA while a CTA holds at most 512 rows (half the per-column
            // control work of 1024 threads), unless the panel-kernel setting asks for 1024
            const bool t512 = rpc <= 512 && opt.panel_kernel != 3;
            cfg.blockDim = dim3(t512 ? 512 : 1024);
            auto launch = [&](auto kern) {
                HME_TIMED(ctx, "panel_factor", HME_CUDA(cudaLaunchKernelEx(&cfg, kern, pa)));
            };
            if (rg.ell == 2) {
                if (t512) launch(panel_cluster_kernel<kArithPow2, 512>);
                else launch(panel_cluster_kernel<kArithPow2, 1024>);
            } else if (p < (1u << 31)) {
                if (t512) launch(panel_cluster_kernel<kArithMont31, 512>);
                else launch(panel_cluster_kernel<kArithMont31, 1024>);
            } else {
                if (t512) launch(panel_cluster_kernel<kArithMont32, 512>);
                else launch(panel_cluster_kernel<kArithMont32, 1024>);
            }
        } else {
            HME_CUDA(cudaMemsetAsync(d_s->piv_slot, 0x7f, sizeof(unsigned long long) * kMaxPanel, st));
            const int rpc_want = std::max(1, opt.rows_per_cta > 0 ? opt.rows_per_cta : 32);
            const int want_grid = std::max(1, std::min(grid_cap, (rows + rpc_want - 1) / rpc_want));
            const int rpc = (rows + want_grid - 1) / want_grid;
            const size_t slice_bytes = sizeof(uint32_t) * static_cast<size_t>(rpc) * w;
            const size_t extra = 5 * static_cast<size_t>(rpc) + 16;  // multipliers + pivot flags
            int smem_rows = slice_bytes + extra <= kPanelSmemMax ? 1 : 0;
            const size_t dyn = (smem_rows ? slice_bytes : 0) + extra;
            void* args[] = {&pa, &smem_rows};
            HME_TIMED(ctx, "panel_factor",
                      HME_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(panel_factor_kernel), want_grid,
                                                           kPanelThreads, args, dyn, st)));
        }
        // the panel's error word next to its pivots, then the pivots to pinned memory
        HME_CUDA(cudaMemcpyAsync(&d_s->err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToDevice, st));
        HME_CUDA(cudaMemcpyAsync(&h_sb[par], d_s, sizeof(Scratch), cudaMemcpyDeviceToHost, st));
        HME_CUDA(cudaEventRecord(ev_panel[par], st));
        ctx->stream = saved;
        return cs;
    };

    std::vector<int> pivots;
    pivots.reserve(std::min(m, n));
    std::vector<int> perm_host;
    int r0 = 0;
    int par = 0;
    bool launched = false;  // the panel at c0 was already factored ahead (on the second stream)
    for (int c0 = 0; c0 < lu_cols && r0 < m; c0 += bw) {
        const int w = std::min(bw, lu_cols - c0);
        if (!launched) launch_panel(c0, w, r0, par, s_main, false);
        launched = false;
        HME_CUDA(cudaEventSynchronize(ev_panel[par]));
        if (block_tried[par] && !h_sb[par].block_ok) {
            // the top block did not settle the panel (nothing was written): the search, on the
            // panel's stream; the main stream's later work waits for it too
            block_rest = 3;
            launch_panel(c0, w, r0, par, panel_stream[par], true);
            if (panel_stream[par] != s_main) HME_CUDA(cudaStreamWaitEvent(s_main, ev_panel[par], 0));
            HME_CUDA(cudaEventSynchronize(ev_panel[par]));
        }
        const Scratch& h_s = h_sb[par];
        if (h_s.err != 0) check_device_error(ctx);  // reports the timeout (and clears the word)
        if (block_tried[par]) ++ctx->elim_block_panels;
        else ++ctx->elim_search_panels;
        const int k = h_s.k;
        if (k == 0) continue;  // no pivot in the panel: nothing moved, the next panel starts at r0
        for (int t = 0; t < k; ++t) pivots.push_back(h_s.pivot_cols[t]);

        // (2) pivot rows first, in pivot order, the other active rows after them in order; the
        // identity when the pivots are rows r0 .. r0+k-1 in order (then nothing moves)
        const int rows = m - r0;
        bool identity = true;
        for (int t = 0; t < k && identity; ++t) identity = h_s.pivot_rows[t] == r0 + t;
        if (!identity) {
            perm_host.assign(rows, 0);
            std::vector<char> is_piv(rows, 0);
            for (int t = 0; t < k; ++t) {
                perm_host[t] = h_s.pivot_rows[t];
                is_piv[h_s.pivot_rows[t] - r0] = 1;
            }
            int q = k;
            for (int i = 0; i < rows; ++i)
                if (!is_piv[i]) perm_host[q++] = r0 + i;
            // permutation parity: the sequence is the pivot rows p_0 .. p_k-1 (relative to r0), then
            // the other rows ascending, so its inversions are the pivot pairs out of order plus, per
            // pivot p_t, the other rows below it (p_t minus the pivots below it): O(k^2), not O(rows)
            long long inv = 0;
            for (int t = 0; t < k; ++t) {
                const int pt = h_s.pivot_rows[t] - r0;
                int below_piv = 0;
                for (int u = 0; u < k; ++u) {
                    const int pu = h_s.pivot_rows[u] - r0;
                    if (pu < pt) {
                        ++below_piv;
                        if (u > t) ++inv;  // p_t before p_u in the sequence, p_t > p_u
                    }
                }
                inv += pt - below_piv;
            }
            if (inv & 1) res.sign_negative = !res.sign_negative;
            // pinned by parity: the copy of the panel two steps back has long completed (the host
            // waited for this panel, which follows that panel's update on the main stream)
            std::memcpy(h_permb[par], perm_host.data(), sizeof(int) * rows);
            HME_CUDA(cudaMemcpyAsync(d_permb[par], h_permb[par], sizeof(int) * rows, cudaMemcpyHostToDevice, s_main));
        }
        int* d_perm = d_permb[par];
        const int c1 = c0 + w;
        const int below = m - r0 - k;
        const int* d_pcols = d_sb[par]->pivot_cols;
        // the update of columns [ca, cb): row permutation (from c0 on), U12 = L11^-1 A12, A22 -= L21 U12
        uint32_t* L21 = nullptr;
        const bool blk = block_tried[par] && h_s.block_ok;
        uint32_t* Wf = nullptr;
        auto update = [&](int ca, int cb, int sm_cap) {
            if (cb <= ca) return;
            if (blk) {
                // settled by the top block (no row moved): [A12; A22] += W A12, W = [L^-1 - I; -A21 B^-1],
                // on a tensor-core variant (it reads A12 through its limb planes, so C may alias it)
                const int ua = std::max(ca, c1);
                if (cb <= ua) return;
                if (!Wf) {
                    Wf = static_cast<uint32_t*>(ctx->ws.get(kSlotElim2, sizeof(uint32_t) * static_cast<size_t>(rows) * k));
                    const int g = (rows + kWRows - 1) / kWRows;
                    const size_t wsm = sizeof(uint32_t) * (((static_cast<size_t>(k) * k + 3) & ~size_t(3)) +
                                                           static_cast<size_t>(kWRows) * k);
                    const uint32_t* binv = d_uinvb[par] + 2 * kMaxPanel * kMaxPanel;
                    const uint32_t* linv = d_uinvb[par] + 3 * kMaxPanel * kMaxPanel;
                    if (k <= 64)
                        HME_TIMED(ctx, "panel_w", panel_w_kernel<64><<<g, 256, wsm, s_main>>>(
                                                      A, ld, r0, m, c0, k, linv, binv, p, mp.barrett, Wf));
                    else
                        HME_TIMED(ctx, "panel_w", panel_w_kernel<128><<<g, 256, wsm, s_main>>>(
                                                      A, ld, r0, m, c0, k, linv, binv, p, mp.barrett, Wf));
                    HME_CUDA(cudaGetLastError());
                }
                ctx->gemm_sm_cap = sm_cap;
                uint32_t* C12 = A + static_cast<size_t>(r0) * ld + ua;
                gemm_u32_variant(ctx, mp, rows, cb - ua, k, Wf, k, C12, ld, C12, ld, HME_ADD,
                                 gemm_default_variant(ctx, mp, rows, cb - ua));
                ctx->gemm_sm_cap = 0;
                return;
            }
            if (!identity) {
                const int cols = cb - ca;
                uint32_t* tmp = static_cast<uint32_t*>(ctx->ws.get(kSlotElim1, sizeof(uint32_t) * static_cast<size_t>(rows) * (n - c0)));
                const int g = grid_1d(static_cast<size_t>(rows) * cols, ctx->num_sms);
                HME_TIMED(ctx, "row_permute", gather_rows_kernel<<<g, 256, 0, s_main>>>(A, ld, d_perm, rows, ca, cols, tmp));
                HME_TIMED(ctx, "row_permute", scatter_rows_kernel<<<g, 256, 0, s_main>>>(A, ld, r0, rows, ca, cols, tmp));
                HME_CUDA(cudaGetLastError());
            }
            const int ua = std::max(ca, c1);
            if (cb <= ua) return;
            const int cols = cb - ua;
            if (k > 1) {
                const int g = (cols + kTrsmCols - 1) / kTrsmCols;
                HME_TIMED(ctx, "trsm", trsm_unit_lower_kernel<<<g, 32 * kTrsmCols, trsm_smem_bytes(k), s_main>>>(
                                           A, ld, r0, d_pcols, k, ua, cols, p, mp.barrett));
                HME_CUDA(cudaGetLastError());
            }
            if (below > 0) {
                if (!L21) {
                    L21 = static_cast<uint32_t*>(ctx->ws.get(kSlotElim2, sizeof(uint32_t) * static_cast<size_t>(below) * k));
                    HME_TIMED(ctx, "gather_cols",
                              gather_cols_kernel<<<grid_1d(static_cast<size_t>(below) * k, ctx->num_sms), 256, 0, s_main>>>(
                                  A, ld, r0 + k, below, d_pcols, k, L21));
                    HME_CUDA(cudaGetLastError());
                }
                ctx->gemm_sm_cap = sm_cap;
                gemm_u32_device(ctx, mp, below, cols, k, L21, k, A + static_cast<size_t>(r0) * ld + ua, ld,
                                A + static_cast<size_t>(r0 + k) * ld + ua, ld, HME_SUB);
                ctx->gemm_sm_cap = 0;
            }
        };
        const int nw = std::min(bw, lu_cols - c1);
        // lookahead only when the next panel runs on the cluster kernel (a few SMs beside the GEMM;
        // the cooperative grid kernel would wait for the whole device anyway)
        const bool next = allow_lookahead && c1 < lu_cols && below > 0 && nw > 0 && cluster_size(below, nw) > 0;
        if (next) {
            // LOOKAHEAD: the next panel's columns first; that panel is factored on the second stream
            // while the rest of this update runs here, the GEMM leaving the cluster's SMs free
            update(c0, c1 + nw, 0);
            HME_CUDA(cudaEventRecord(ev_next, s_main));
            HME_CUDA(cudaStreamWaitEvent(s_aux, ev_next, 0));
            const int cs_next = launch_panel(c1, nw, r0 + k, par ^ 1, s_aux, false);
            update(c1 + nw, n, cs_next > 0 ? std::max(1, ctx->num_sms - cs_next) : 0);
            launched = true;
        } else {
            update(c0, n, 0);
        }
        // the main stream's later work (the next panel's update) follows the lookahead panel
        if (launched) HME_CUDA(cudaStreamWaitEvent(s_main, ev_panel[par ^ 1], 0));
        r0 += k;
        par ^= 1;
    }
    HME_CUDA(cudaStreamSynchronize(s_aux));
    res.rank = r0;
    res.pivots = pivots;

    // determinant factors: the U diagonal
    if (opt.want_diag && res.rank > 0) {
        int* d_pv = static_cast<int*>(ctx->ws.get(kSlotElim3, sizeof(int) * (2 * static_cast<size_t>(n) + 16)));
        uint32_t* d_diag = reinterpret_cast<uint32_t*>(d_pv + n);
        HME_CUDA(cudaMemcpyAsync(d_pv, pivots.data(), sizeof(int) * res.rank, cudaMemcpyHostToDevice, ctx->stream));
        HME_TIMED(ctx, "gather_diag", gather_diag_kernel<<<grid_1d(res.rank, ctx->num_sms), 256, 0, ctx->stream>>>(
                                          A, ld, d_pv, res.rank, d_diag));
        HME_CUDA(cudaGetLastError());
        res.diag.resize(res.rank);
        HME_CUDA(cudaMemcpyAsync(res.diag.data(), d_diag, sizeof(uint32_t) * res.rank, cudaMemcpyDeviceToHost,
                                 ctx->stream));
        HME_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    if (!want_rref) return res;

    // ---- RREF = U1^-1 U on the free columns ------------------------------------------
    const int rank = res.rank;
    const int f = n - rank;
    std::vector<int> colmap(n);
    std::vector<int> free_cols;
    {
        std::vector<char> isp(n, 0);
        for (int t = 0; t < rank; ++t) {
            isp[pivots[t]] = 1;
            colmap[pivots[t]] = t;
        }
        for (int j = 0; j < n; ++j)
            if (!isp[j]) {
                colmap[j] = -1 - static_cast<int>(free_cols.size());
                free_cols.push_back(j);
            }
    }
    int* d_cols = static_cast<int*>(ctx->ws.get(kSlotElim3, sizeof(int) * (2 * static_cast<size_t>(n) + 16)));
    int* d_piv = d_cols + n;  // pivots, then free columns at d_cols
    uint32_t* X = nullptr;
    if (rank > 0) {
        HME_CUDA(cudaMemcpyAsync(d_piv, pivots.data(), sizeof(int) * rank, cudaMemcpyHostToDevice, ctx->stream));
    }
    if (rank > 0 && f > 0) {
        HME_CUDA(cudaMemcpyAsync(d_cols, free_cols.data(), sizeof(int) * f, cudaMemcpyHostToDevice, ctx->stream));
        X = static_cast<uint32_t*>(ctx->ws.get(kSlotElim1, sizeof(uint32_t) * static_cast<size_t>(rank) * f));
        HME_TIMED(ctx, "gather_cols",
                  gather_cols_kernel<<<grid_1d(static_cast<size_t>(rank) * f, ctx->num_sms), 256, 0, ctx->stream>>>(
                      A, ld, 0, rank, d_cols, f, X));
        HME_CUDA(cudaGetLastError());
        const int bb = std::max(16, std::min(opt.back_block > 0 ? opt.back_block : 128, 128));
        const int nblk = (rank + bb - 1) / bb;
        // all diagonal blocks of U1 inverted at once, one CTA each
        uint32_t* Uinv = static_cast<uint32_t*>(ctx->ws.get(kSlotElim5, sizeof(uint32_t) * static_cast<size_t>(nblk) * bb * bb));
        {
            const size_t sm = sizeof(uint32_t) * (2 * static_cast<size_t>(bb) * bb + bb);
            HME_TIMED(ctx, "tri_inv", tri_inv_kernel<true><<<nblk, 1024, sm, ctx->stream>>>(
                                          A, ld, 0, d_piv, rank, bb, p, mp.barrett, kmax_for(p), Uinv));
            HME_CUDA(cudaGetLastError());
        }
        // W (rank x f) in X's slot; the solution accumulates in Xs
        uint32_t* Xs = static_cast<uint32_t*>(ctx->ws.get(kSlotElim6, sizeof(uint32_t) * static_cast<size_t>(rank) * f));
        for (int blk = nblk - 1; blk >= 0; --blk) {
            const int i0 = blk * bb, nb = std::min(bb, rank - i0);
            // X_B = U_BB^-1 W_B
            gemm_u32_device(ctx, mp, nb, f, nb, Uinv + static_cast<size_t>(blk) * bb * bb, nb,
                            X + static_cast<size_t>(i0) * f, f, Xs + static_cast<size_t>(i0) * f, f, HME_SET);
            if (i0 > 0) {
                // W[0:i0] -= U1[0:i0, block pivots] * X_B
                uint32_t* Ub = static_cast<uint32_t*>(ctx->ws.get(kSlotElim2, sizeof(uint32_t) * static_cast<size_t>(i0) * nb));
                HME_TIMED(ctx, "gather_cols",
                          gather_cols_kernel<<<grid_1d(static_cast<size_t>(i0) * nb, ctx->num_sms), 256, 0, ctx->stream>>>(
                              A, ld, 0, i0, d_piv + i0, nb, Ub));
                HME_CUDA(cudaGetLastError());
                gemm_u32_device(ctx, mp, i0, f, nb, Ub, nb, Xs + static_cast<size_t>(i0) * f, f, X, f, HME_SUB);
            }
        }
        X = Xs;
    }
    int* d_colmap = static_cast<int*>(ctx->ws.get(kSlotElim4, sizeof(int) * (static_cast<size_t>(n) + 16)));
    HME_CUDA(cudaMemcpyAsync(d_colmap, colmap.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->stream));
    HME_TIMED(ctx, "assemble_rref",
              assemble_rref_kernel<<<grid_1d(static_cast<size_t>(m) * n, ctx->num_sms), 256, 0, ctx->stream>>>(
                  R, ldr, m, n, rank, d_colmap, X, std::max(f, 1)));
    HME_CUDA(cudaGetLastError());
    HME_CUDA(cudaStreamSynchronize(ctx->stream));
    return res;
}

}  // namespace hme

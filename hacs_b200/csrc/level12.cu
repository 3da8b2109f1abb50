// Level-1 / level-2 device operations of the engine's device layer, on strided
// device views: y op= A x, axpy, scal, copy, transpose, fill, identity axpy,
// the gather used by the tape's assembly nodes, canonicalisation (from the
// lazy [0, 2p) form and from 64-bit accumulators), unit-triangular solves,
// C op= A B^T and the Schur update.
//
// Reference semantics: engine::cuda::gemv / axpy / scal / copy / transpose /
// fill / axpy_identity / gather / canonicalise / trsm_unit / gemm_nt /
// schur_update (src/Cuda/CudaKernels.h:120-131, 186-247; bodies
// src/Cuda/cuda_kernels.cu:952-1130): every view has a row stride and a column
// stride in elements (the reference's DeviceView), residues are canonical
// u32 below p unless stated, and every result is the exact residue, so the
// outputs equal the reference's element for element.
//
// B200 layout.  The element-wise kernels cut the window into tiles of one
// "outer" index by 1024 "inner" vectors, the inner dimension being the one
// with unit stride when it is long enough (else the longer one): one integer
// division per tile, consecutive threads on consecutive addresses, and four
// independent loads per thread issued before any store, so that each SM keeps
// enough bytes in flight to stream HBM.  Where every operand is unit-stride
// along the inner dimension with 16-byte aligned rows, a vector is 4 residues
// moved by one 16-byte access; otherwise it is one residue.  y op= A x runs
// one warp per row of A when A's rows are contiguous (one thread per row
// otherwise), four (vector) loads in flight per lane, and sums the 64-bit
// products exactly as a 96-bit value (a carry count beside a 64-bit sum)
// reduced once per row.  The transpose moves 64 x 64 tiles through shared
// memory, sixteen loads in flight per thread.  The triangular solve is blocked
// by 128 rows: one kernel solves a 128-row diagonal block (the block's
// triangle in shared memory, one right-hand-side column per warp, the
// column's 128 rows in registers, four per lane) and the limb GEMM (tensor
// cores) applies the block to the rows below (above) it.
#include <cuda_runtime.h>

#include <algorithm>
#include <initializer_list>

#include "hme_internal.h"

namespace hme {
namespace {

constexpr int kEwThreads = 256;             // threads per element-wise CTA
constexpr int kEwU = 4;                     // vectors per thread per tile
constexpr int kEwTile = kEwThreads * kEwU;  // inner vectors per tile
constexpr uint32_t kTrsmNB = 128;           // rows per diagonal block of the solve

// Iteration space of an element-wise op: outer x inner (inner counted in
// vectors), `tpr` tiles per outer index.  Each operand has a stride along
// outer (so) and inner (si), in elements.
struct Ew {
    uint32_t outer, inner, tpr;
    uint64_t ntiles;
};
struct Strides {
    uint64_t so, si;
};

// Inner dimension: the unit-stride one when it holds at least 64 elements,
// else the longer one.
inline bool inner_is_cols(uint32_t rows, uint32_t cols, uint64_t rs, uint64_t cs) {
    if (cs == 1 && cols >= 64) return true;
    if (rs == 1 && rows >= 64) return false;
    return cols >= rows;
}
inline Ew make_ew(uint32_t rows, uint32_t cols, bool icols, int V) {
    Ew e;
    e.outer = icols ? rows : cols;
    e.inner = (icols ? cols : rows) / V;
    e.tpr = (e.inner + kEwTile - 1) / kEwTile;
    e.ntiles = static_cast<uint64_t>(e.outer) * e.tpr;
    return e;
}
inline Strides strides_of(uint64_t rs, uint64_t cs, bool icols) { return icols ? Strides{rs, cs} : Strides{cs, rs}; }

// One operand of an element-wise op, for the choice of the vector width.
struct Operand {
    const void* p;
    uint64_t rs, cs;
};
// 4 when every operand is unit-stride along the inner dimension, its rows
// start 16-byte aligned, and the inner extent is a multiple of 4; else 1.
inline int vec_width(bool icols, uint32_t rows, uint32_t cols, std::initializer_list<Operand> ops) {
    const uint32_t inner = icols ? cols : rows, outer = icols ? rows : cols;
    if (inner % 4) return 1;
    for (const Operand& q : ops) {
        const Strides s = strides_of(q.rs, q.cs, icols);
        if (s.si != 1 || (outer > 1 && s.so % 4) || reinterpret_cast<uintptr_t>(q.p) % 16) return 1;
    }
    return 4;
}

template <int V>
struct VW {
    uint32_t v[V];
};
template <int V>
__device__ __forceinline__ VW<V> ldv(const uint32_t* p) {
    VW<V> r;
    if constexpr (V == 4) {
        const uint4 t = *reinterpret_cast<const uint4*>(p);
        r.v[0] = t.x, r.v[1] = t.y, r.v[2] = t.z, r.v[3] = t.w;
    } else {
        r.v[0] = *p;
    }
    return r;
}
template <int V>
__device__ __forceinline__ void stv(uint32_t* p, const VW<V>& r) {
    if constexpr (V == 4)
        *reinterpret_cast<uint4*>(p) = make_uint4(r.v[0], r.v[1], r.v[2], r.v[3]);
    else
        *p = r.v[0];
}
// element offset of vector (o, j)
template <int V>
__device__ __forceinline__ uint64_t offv(const Strides& s, uint32_t o, uint32_t j) {
    return o * s.so + (V == 1 ? j * s.si : static_cast<uint64_t>(j) * V);
}

// Tile loop of the element-wise kernels: `o` the outer index, `jb` this
// thread's first inner vector (the others follow at kEwThreads apart).
#define HME_EW_TILES(E)                                                \
    for (uint64_t t_ = blockIdx.x; t_ < (E).ntiles; t_ += gridDim.x) { \
        const uint32_t o = static_cast<uint32_t>(t_ / (E).tpr);        \
        const uint32_t jb = static_cast<uint32_t>(t_ - static_cast<uint64_t>(o) * (E).tpr) * kEwTile + threadIdx.x;

__device__ __forceinline__ uint32_t apply_op(uint32_t old, uint32_t v, int op, uint32_t p) {
    return op == HME_SET ? v : op == HME_ADD ? mod_add(old, v, p) : mod_sub(old, v, p);
}

// (hi * 2^64 + lo) mod p for a small carry count hi; r64 = 2^64 mod p
__device__ __forceinline__ uint32_t fold96(uint64_t lo, uint32_t hi, uint32_t p, uint64_t barrett, uint32_t r64) {
    const uint32_t a = reduce_u64(lo, p, barrett);
    return hi ? mod_add(a, reduce_u64(static_cast<uint64_t>(hi) * r64, p, barrett), p) : a;
}
__device__ __forceinline__ void mac96(uint64_t& lo, uint32_t& hi, uint32_t a, uint32_t b) {
    const uint64_t prod = static_cast<uint64_t>(a) * b;
    lo += prod;
    hi += lo < prod ? 1u : 0u;
}
// acc += a b, a 2^64 wraparound folded back as r64 = 2^64 mod p: acc stays
// congruent to the exact sum.  After a wrap acc < a b <= (2^32 - 1)^2, so
// adding r64 < 2^32 cannot wrap again.
__device__ __forceinline__ void mac_fold(uint64_t& acc, uint32_t a, uint32_t b, uint32_t r64) {
    const uint64_t prod = static_cast<uint64_t>(a) * b;
    acc += prod;
    acc += acc < prod ? r64 : 0u;
}

template <int V>
__global__ void __launch_bounds__(kEwThreads) axpy_kernel(uint32_t alpha, const uint32_t* __restrict__ x, Strides xs,
                                                          uint32_t* __restrict__ y, Strides ys, Ew e, int subtract,
                                                          uint32_t p, uint64_t barrett) {
    HME_EW_TILES(e)
    VW<V> xv[kEwU], yv[kEwU];
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t j = jb + u * kEwThreads;
        if (j < e.inner) {
            xv[u] = ldv<V>(x + offv<V>(xs, o, j));
            yv[u] = ldv<V>(y + offv<V>(ys, o, j));
        }
    }
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t j = jb + u * kEwThreads;
        if (j < e.inner) {
            VW<V> r;
#pragma unroll
            for (int c = 0; c < V; ++c) {
                const uint32_t ax = mod_mul(alpha, xv[u].v[c], p, barrett);
                r.v[c] = subtract ? mod_sub(yv[u].v[c], ax, p) : mod_add(yv[u].v[c], ax, p);
            }
            stv<V>(y + offv<V>(ys, o, j), r);
        }
    }
    }
}

// mode 0: x = alpha x;  1: x = alpha (a fill);  2: x = x >= p ? x - p : x
template <int V>
__global__ void __launch_bounds__(kEwThreads) unary_kernel(uint32_t* __restrict__ x, Strides xs, Ew e, int mode,
                                                           uint32_t alpha, uint32_t p, uint64_t barrett) {
    HME_EW_TILES(e)
    VW<V> v[kEwU];
    if (mode != 1) {
#pragma unroll
        for (int u = 0; u < kEwU; ++u) {
            const uint32_t j = jb + u * kEwThreads;
            if (j < e.inner) v[u] = ldv<V>(x + offv<V>(xs, o, j));
        }
    }
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t j = jb + u * kEwThreads;
        if (j < e.inner) {
            VW<V> r;
#pragma unroll
            for (int c = 0; c < V; ++c)
                r.v[c] = mode == 0   ? mod_mul(alpha, v[u].v[c], p, barrett)
                         : mode == 1 ? alpha
                                     : (v[u].v[c] >= p ? v[u].v[c] - p : v[u].v[c]);
            stv<V>(x + offv<V>(xs, o, j), r);
        }
    }
    }
}

template <int V>
__global__ void __launch_bounds__(kEwThreads) copy_kernel(const uint32_t* __restrict__ s, Strides ss,
                                                          uint32_t* __restrict__ d, Strides ds, Ew e) {
    HME_EW_TILES(e)
    VW<V> v[kEwU];
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t j = jb + u * kEwThreads;
        if (j < e.inner) v[u] = ldv<V>(s + offv<V>(ss, o, j));
    }
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t j = jb + u * kEwThreads;
        if (j < e.inner) stv<V>(d + offv<V>(ds, o, j), v[u]);
    }
    }
}

// dst = acc mod p for 64-bit accumulators (V = 4: two 16-byte loads per vector)
template <int V>
__global__ void __launch_bounds__(kEwThreads) canon64_kernel(const uint64_t* __restrict__ a, Strides as,
                                                             uint32_t* __restrict__ d, Strides ds, Ew e, uint32_t p,
                                                             uint64_t barrett) {
    HME_EW_TILES(e)
    uint64_t v[kEwU][V];
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t j = jb + u * kEwThreads;
        if (j < e.inner) {
            const uint64_t* src = a + offv<V>(as, o, j);
            if constexpr (V == 4) {
                const ulonglong2 t0 = reinterpret_cast<const ulonglong2*>(src)[0];
                const ulonglong2 t1 = reinterpret_cast<const ulonglong2*>(src)[1];
                v[u][0] = t0.x, v[u][1] = t0.y, v[u][2] = t1.x, v[u][3] = t1.y;
            } else {
                v[u][0] = *src;
            }
        }
    }
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t j = jb + u * kEwThreads;
        if (j < e.inner) {
            VW<V> r;
#pragma unroll
            for (int c = 0; c < V; ++c) r.v[c] = reduce_u64(v[u][c], p, barrett);
            stv<V>(d + offv<V>(ds, o, j), r);
        }
    }
    }
}

__global__ void axpy_identity_kernel(uint32_t alpha, uint32_t* __restrict__ y, uint64_t rs, uint64_t cs, uint32_t n,
                                     int subtract, uint32_t p) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t* yp = y + i * rs + i * cs;
        *yp = subtract ? mod_sub(*yp, alpha, p) : mod_add(*yp, alpha, p);
    }
}

// c(i, t) [+]= alpha [row_off + r(i) == col(t)] + beta a(r(i), col(t)),
// r(i) = rows ? rows[i] : i, col(t) = cols ? cols[t] : t; tiles over (i, t)
// with t inner.  V = 4 (no column list, a's and c's rows unit-stride and
// 16-byte aligned) moves 4 consecutive columns per access.
template <int V>
__global__ void __launch_bounds__(kEwThreads)
    gather_kernel(uint32_t alpha, uint32_t beta, const uint32_t* __restrict__ a, uint64_t a_rs, uint64_t a_cs,
                  uint32_t row_off, const uint32_t* __restrict__ cols, const uint32_t* __restrict__ rows,
                  uint32_t* __restrict__ c, uint64_t c_rs, uint64_t c_cs, Ew e, int accumulate, uint32_t p,
                  uint64_t barrett) {
    HME_EW_TILES(e)
    const uint32_t ar = rows ? rows[o] : o;
    VW<V> av[kEwU], cv[kEwU];
    uint32_t col[kEwU];
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t t = jb + u * kEwThreads;
        if (t < e.inner) {
            if constexpr (V == 4) {
                col[u] = 4 * t;
                if (a) av[u] = ldv<4>(a + ar * a_rs + col[u]);
                if (accumulate) cv[u] = ldv<4>(c + o * c_rs + col[u]);
            } else {
                col[u] = cols ? cols[t] : t;
                av[u].v[0] = a ? a[ar * a_rs + col[u] * a_cs] : 0u;
                cv[u].v[0] = accumulate ? c[o * c_rs + t * c_cs] : 0u;
            }
        }
    }
#pragma unroll
    for (int u = 0; u < kEwU; ++u) {
        const uint32_t t = jb + u * kEwThreads;
        if (t < e.inner) {
            VW<V> r;
#pragma unroll
            for (int q = 0; q < V; ++q) {
                uint32_t v = a ? mod_mul(beta, av[u].v[q], p, barrett) : 0u;
                if (alpha != 0 && row_off + ar == col[u] + q) v = mod_add(v, alpha, p);
                r.v[q] = accumulate ? mod_add(cv[u].v[q], v, p) : v;
            }
            if constexpr (V == 4)
                stv<4>(c + o * c_rs + col[u], r);
            else
                c[o * c_rs + t * c_cs] = r.v[0];
        }
    }
    }
}

// dst(i, j) = src(j, i): 64 x 64 tiles through shared memory, 256 threads as
// 64 x 4, sixteen loads in flight per thread; coalesced on both sides when
// src and dst are row-major
__global__ void __launch_bounds__(256) transpose_kernel(const uint32_t* __restrict__ src, uint64_t s_rs, uint64_t s_cs,
                                                        uint32_t* __restrict__ dst, uint64_t d_rs, uint64_t d_cs,
                                                        uint32_t rows_dst, uint32_t cols_dst) {
    __shared__ uint32_t tile[64][65];
    const uint32_t tx = threadIdx.x & 63, ty = threadIdx.x >> 6;
    for (uint32_t by = blockIdx.y; by * 64 < rows_dst; by += gridDim.y)
        for (uint32_t bx = blockIdx.x; bx * 64 < cols_dst; bx += gridDim.x) {
            const uint32_t i0 = by * 64, j0 = bx * 64;  // dst tile origin
            uint32_t v[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const uint32_t jj = j0 + ty + 4 * q, ii = i0 + tx;  // src row jj, column ii
                v[q] = (jj < cols_dst && ii < rows_dst) ? src[jj * s_rs + ii * s_cs] : 0u;
            }
            __syncthreads();  // the previous tile's reads of `tile` are done
#pragma unroll
            for (int q = 0; q < 16; ++q) tile[ty + 4 * q][tx] = v[q];
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const uint32_t r = ty + 4 * q, ii = i0 + r, jj = j0 + tx;
                if (ii < rows_dst && jj < cols_dst) dst[ii * d_rs + jj * d_cs] = tile[tx][r];
            }
        }
}

// y op= A x, one warp per row (A's rows contiguous): four vector loads in
// flight per lane, the products summed exactly (96 bits), one reduction per
// lane.  V = 4 needs A and x unit-stride, 16-byte aligned rows, k % 4 == 0.
template <int V>
__global__ void gemv_warp_kernel(const uint32_t* __restrict__ A, uint64_t a_rs, uint64_t a_cs,
                                 const uint32_t* __restrict__ x, uint64_t x_rs, uint32_t* __restrict__ y,
                                 uint64_t y_rs, uint32_t m, uint32_t k, int op, uint32_t p, uint64_t barrett,
                                 uint32_t r64) {
    const uint32_t lane = threadIdx.x & 31, kv = k / V;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < m; row += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t* a = A + row * a_rs;
        uint64_t lo = 0;
        uint32_t hi = 0;
        for (uint32_t kk = lane; kk < kv; kk += 128) {
            VW<V> av[4], xv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t j = kk + 32 * u;
                if (j < kv) {
                    av[u] = ldv<V>(a + (V == 1 ? j * a_cs : static_cast<uint64_t>(j) * V));
                    xv[u] = ldv<V>(x + (V == 1 ? j * x_rs : static_cast<uint64_t>(j) * V));
                } else {
#pragma unroll
                    for (int c = 0; c < V; ++c) av[u].v[c] = xv[u].v[c] = 0u;
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int c = 0; c < V; ++c) mac96(lo, hi, av[u].v[c], xv[u].v[c]);
        }
        uint32_t v = fold96(lo, hi, p, barrett, r64);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = mod_add(v, __shfl_xor_sync(0xffffffffu, v, off), p);
        if (lane == 0) y[row * y_rs] = apply_op(y[row * y_rs], v, op, p);
    }
}
// y op= A x for long rows: a CTA per row at a time (rows striped over a
// persistent grid), its 8 warps splitting the row, four vector loads in flight
// per thread, the 8 warp sums combined in shared memory.
template <int V>
__global__ void __launch_bounds__(256) gemv_block_kernel(const uint32_t* __restrict__ A, uint64_t a_rs, uint64_t a_cs,
                                                         const uint32_t* __restrict__ x, uint64_t x_rs,
                                                         uint32_t* __restrict__ y, uint64_t y_rs, uint32_t m,
                                                         uint32_t k, int op, uint32_t p, uint64_t barrett,
                                                         uint32_t r64) {
    __shared__ uint32_t part[8];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, kv = k / V;
    for (uint32_t row = blockIdx.x; row < m; row += gridDim.x) {
        const uint32_t* a = A + row * a_rs;
        uint64_t lo = 0;
        uint32_t hi = 0;
        for (uint32_t kk = threadIdx.x; kk < kv; kk += 1024) {
            VW<V> av[4], xv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t j = kk + 256 * u;
                if (j < kv) {
                    av[u] = ldv<V>(a + (V == 1 ? j * a_cs : static_cast<uint64_t>(j) * V));
                    xv[u] = ldv<V>(x + (V == 1 ? j * x_rs : static_cast<uint64_t>(j) * V));
                } else {
#pragma unroll
                    for (int c = 0; c < V; ++c) av[u].v[c] = xv[u].v[c] = 0u;
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int c = 0; c < V; ++c) mac96(lo, hi, av[u].v[c], xv[u].v[c]);
        }
        uint32_t v = fold96(lo, hi, p, barrett, r64);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = mod_add(v, __shfl_xor_sync(0xffffffffu, v, off), p);
        if (lane == 0) part[warp] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t s = part[0];
#pragma unroll
            for (int w = 1; w < 8; ++w) s = mod_add(s, part[w], p);
            y[row * y_rs] = apply_op(y[row * y_rs], s, op, p);
        }
        __syncthreads();
    }
}

// one thread per row (A's columns contiguous: consecutive rows, consecutive addresses)
__global__ void gemv_thread_kernel(const uint32_t* __restrict__ A, uint64_t a_rs, uint64_t a_cs,
                                   const uint32_t* __restrict__ x, uint64_t x_rs, uint32_t* __restrict__ y,
                                   uint64_t y_rs, uint32_t m, uint32_t k, int op, uint32_t p, uint64_t barrett,
                                   uint32_t r64) {
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < m; row += gridDim.x * blockDim.x) {
        uint64_t lo = 0;
        uint32_t hi = 0;
        for (uint32_t kk = 0; kk < k; kk += 4) {
            uint32_t av[4], xv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                av[u] = kk + u < k ? A[row * a_rs + (kk + u) * a_cs] : 0u;
                xv[u] = kk + u < k ? x[(kk + u) * x_rs] : 0u;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) mac96(lo, hi, av[u], xv[u]);
        }
        y[row * y_rs] = apply_op(y[row * y_rs], fold96(lo, hi, p, barrett, r64), op, p);
    }
}

// One diagonal block of a unit-triangular solve: rows [i0, i0 + nb) of B
// (nb <= 128) become T_bb^-1 B_b.  A CTA takes 8 right-hand-side columns at a
// time, one per warp.  Shared memory holds nT(r, s) = p - T(r, s) on the
// strict triangle and 0 elsewhere, for all 128 x 128 positions (pitch 129:
// the 32 lanes' rows fall in 32 different banks), and the nb x 8 tile of B.
// Lane l of a warp keeps rows l, l + 32, l + 64, l + 96 of its column as
// 64-bit words congruent to b_r + sum_t nT(r, t) x_t (no reduction per
// update, wraparounds folded back as 2^64 mod p; no branch: entries outside
// the triangle are 0).  At step t the row-t sum is
// reduced, broadcast by a shuffle, and added into every row; LOWER walks t up,
// upper walks it down; at the end every row is reduced once.
template <bool LOWER>
__global__ void __launch_bounds__(256) trsm_diag_kernel(const uint32_t* __restrict__ T, size_t ldt,
                                                        uint32_t* __restrict__ B, size_t ldb, uint32_t i0,
                                                        uint32_t nb, uint32_t n, uint32_t p, uint64_t barrett,
                                                        uint32_t r64) {
    extern __shared__ uint32_t sm[];
    constexpr uint32_t tp = kTrsmNB + 1;
    uint32_t* sT = sm;                  // 128 x tp
    uint32_t* sB = sm + kTrsmNB * tp;   // 128 x 9
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t rb = 0; rb < kTrsmNB; rb += 32) {
        uint32_t v[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t r = rb + warp + 8 * i, s = lane + 32 * q;
                const bool keep = r < nb && s < nb && (LOWER ? s < r : s > r);
                v[i][q] = keep ? T[(i0 + r) * ldt + (i0 + s)] : 0u;
            }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int q = 0; q < 4; ++q) sT[(rb + warp + 8 * i) * tp + lane + 32 * q] = v[i][q] ? p - v[i][q] : 0u;
    }
    const uint32_t nsub = (nb + 31) / 32;
    const uint32_t cc = threadIdx.x & 7, rr = threadIdx.x >> 3;  // tile load / store: column, first row
    for (uint32_t c0 = blockIdx.x * 8; c0 < n; c0 += gridDim.x * 8) {
        const bool col_ok = c0 + cc < n;
        {
            uint32_t v[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const uint32_t r = rr + 32 * i;
                v[i] = (r < nb && col_ok) ? B[(i0 + r) * ldb + c0 + cc] : 0u;
            }
            __syncthreads();  // sT is complete; the previous tile is out of sB
#pragma unroll
            for (int i = 0; i < 4; ++i) sB[(rr + 32 * i) * 9 + cc] = v[i];
        }
        __syncthreads();
        uint64_t acc[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[i] = sB[(lane + 32 * i) * 9 + warp];
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) {
            const int q = LOWER ? qq : 3 - qq;  // the 32-row group holding the rows t of this pass
            if (static_cast<uint32_t>(q) < nsub) {
                const uint32_t tn = min(32u, nb - 32 * q);
                for (uint32_t st = 0; st < tn; ++st) {
                    const uint32_t tt = LOWER ? st : tn - 1 - st, t = 32 * q + tt;
                    const uint32_t xt = __shfl_sync(0xffffffffu, reduce_u64(acc[q], p, barrett), tt);
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        if (LOWER ? i < q : i > q) continue;  // rows already final
                        mac_fold(acc[i], sT[(lane + 32 * i) * tp + t], xt, r64);
                    }
                }
            }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) sB[(lane + 32 * i) * 9 + warp] = reduce_u64(acc[i], p, barrett);
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t r = rr + 32 * i;
            if (r < nb && col_ok) B[(i0 + r) * ldb + c0 + cc] = sB[r * 9 + cc];
        }
    }
}

constexpr size_t kTrsmSmem = 4ull * (kTrsmNB * (kTrsmNB + 1) + kTrsmNB * 9);

int ew_grid(uint64_t ntiles, int sms) {
    return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(ntiles, static_cast<uint64_t>(sms) * 8)));
}

uint32_t r64_of(uint32_t p) { return static_cast<uint32_t>((static_cast<unsigned __int128>(1) << 64) % p); }

// [lo, hi) byte range of a rows x cols view of `esz`-byte elements
void span_of(const void* base, uint32_t rows, uint32_t cols, uint64_t rs, uint64_t cs, size_t esz, uintptr_t& lo,
             uintptr_t& hi) {
    lo = reinterpret_cast<uintptr_t>(base);
    hi = lo + esz * ((rows ? (rows - 1) * rs : 0) + (cols ? (cols - 1) * cs : 0) + 1);
}
bool overlap(const void* a, uint32_t ar, uint32_t ac, uint64_t ars, uint64_t acs, const void* b, uint32_t br,
             uint32_t bc, uint64_t brs, uint64_t bcs, size_t aesz = 4) {
    if (!ar || !ac || !br || !bc) return false;
    uintptr_t a0, a1, b0, b1;
    span_of(a, ar, ac, ars, acs, aesz, a0, a1);
    span_of(b, br, bc, brs, bcs, 4, b0, b1);
    return a0 < b1 && b0 < a1;
}

void launch_transpose(hme_ctx* ctx, const uint32_t* src, uint64_t s_rs, uint64_t s_cs, uint32_t* dst, uint64_t d_rs,
                      uint64_t d_cs, uint32_t rows_dst, uint32_t cols_dst) {
    const dim3 grid(std::min<uint32_t>((cols_dst + 63) / 64, 4096), std::min<uint32_t>((rows_dst + 63) / 64, 4096));
    HME_TIMED(ctx, "transpose", transpose_kernel<<<grid, 256, 0, ctx->stream>>>(src, s_rs, s_cs, dst, d_rs, d_cs,
                                                                                rows_dst, cols_dst));
    HME_CUDA(cudaGetLastError());
}

void launch_unary(hme_ctx* ctx, const char* name, uint32_t* x, uint32_t rows, uint32_t cols, uint64_t rs, uint64_t cs,
                  int mode, uint32_t alpha, uint32_t p) {
    const bool ic = inner_is_cols(rows, cols, rs, cs);
    const int V = vec_width(ic, rows, cols, {{x, rs, cs}});
    const Ew e = make_ew(rows, cols, ic, V);
    const uint64_t barrett = p >= 2 ? make_mod(p).barrett : 0;
    const Strides xs = strides_of(rs, cs, ic);
    const int grid = ew_grid(e.ntiles, ctx->num_sms);
    if (V == 4)
        HME_TIMED(ctx, name, unary_kernel<4><<<grid, kEwThreads, 0, ctx->stream>>>(x, xs, e, mode, alpha, p, barrett));
    else
        HME_TIMED(ctx, name, unary_kernel<1><<<grid, kEwThreads, 0, ctx->stream>>>(x, xs, e, mode, alpha, p, barrett));
    HME_CUDA(cudaGetLastError());
}

}  // namespace
}  // namespace hme

using namespace hme;

extern "C" {

int hme_gemv_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t k, const uint32_t* A, size_t a_rs, size_t a_cs,
                     const uint32_t* x, size_t x_rs, uint32_t* y, size_t y_rs, int op) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2, "gemv: bad context or modulus");
        HME_REQUIRE(op == HME_SET || op == HME_ADD || op == HME_SUB, "gemv: bad op");
        if (m == 0) return;
        HME_REQUIRE(y && (k == 0 || (A && x)), "gemv: null pointer");
        HME_REQUIRE(!overlap(y, m, 1, y_rs, 1, A, m, k, a_rs, a_cs) && !overlap(y, m, 1, y_rs, 1, x, k, 1, x_rs, 1),
                    "gemv: y aliases an operand");
        bind(ctx);
        const ModParams mp = make_mod(p);
        const uint32_t r64 = r64_of(p);
        const bool v4 = a_cs == 1 && x_rs == 1 && k % 4 == 0 && (m == 1 || a_rs % 4 == 0) &&
                        reinterpret_cast<uintptr_t>(A) % 16 == 0 && reinterpret_cast<uintptr_t>(x) % 16 == 0;
        if ((a_cs == 1 || a_rs != 1) && k >= 2048) {
            // long rows: a CTA per row, the grid one wave of resident CTAs
            int per_sm = 1;
            HME_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, v4 ? gemv_block_kernel<4> : gemv_block_kernel<1>, 256, 0));
            const int grid = static_cast<int>(std::min<size_t>(m, static_cast<size_t>(std::max(1, per_sm)) * ctx->num_sms));
            if (v4)
                HME_TIMED(ctx, "gemv", gemv_block_kernel<4><<<grid, 256, 0, ctx->stream>>>(
                                           A, a_rs, a_cs, x, x_rs, y, y_rs, m, k, op, p, mp.barrett, r64));
            else
                HME_TIMED(ctx, "gemv", gemv_block_kernel<1><<<grid, 256, 0, ctx->stream>>>(
                                           A, a_rs, a_cs, x, x_rs, y, y_rs, m, k, op, p, mp.barrett, r64));
        } else if (a_cs == 1 || a_rs != 1) {
            const int grid = static_cast<int>(std::min<size_t>((static_cast<size_t>(m) + 7) / 8, ctx->num_sms * 16));
            if (v4)
                HME_TIMED(ctx, "gemv", gemv_warp_kernel<4><<<grid, 256, 0, ctx->stream>>>(
                                           A, a_rs, a_cs, x, x_rs, y, y_rs, m, k, op, p, mp.barrett, r64));
            else
                HME_TIMED(ctx, "gemv", gemv_warp_kernel<1><<<grid, 256, 0, ctx->stream>>>(
                                           A, a_rs, a_cs, x, x_rs, y, y_rs, m, k, op, p, mp.barrett, r64));
        } else {
            const int grid = static_cast<int>(std::min<size_t>((static_cast<size_t>(m) + 255) / 256, ctx->num_sms * 8));
            HME_TIMED(ctx, "gemv", gemv_thread_kernel<<<grid, 256, 0, ctx->stream>>>(A, a_rs, a_cs, x, x_rs, y, y_rs, m,
                                                                                   k, op, p, mp.barrett, r64));
        }
        HME_CUDA(cudaGetLastError());
    });
}

int hme_axpy_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t alpha, uint32_t rows, uint32_t cols, const uint32_t* x,
                     size_t x_rs, size_t x_cs, uint32_t* y, size_t y_rs, size_t y_cs, int subtract) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2 && alpha < p, "axpy: bad context, modulus or alpha (must be canonical)");
        if (!rows || !cols) return;
        HME_REQUIRE(x && y, "axpy: null pointer");
        bind(ctx);
        const bool ic = inner_is_cols(rows, cols, x_rs, x_cs);
        const int V = vec_width(ic, rows, cols, {{x, x_rs, x_cs}, {y, y_rs, y_cs}});
        const Ew e = make_ew(rows, cols, ic, V);
        const Strides xs = strides_of(x_rs, x_cs, ic), ys = strides_of(y_rs, y_cs, ic);
        const int grid = ew_grid(e.ntiles, ctx->num_sms);
        const uint64_t bar = make_mod(p).barrett;
        if (V == 4)
            HME_TIMED(ctx, "axpy", axpy_kernel<4><<<grid, kEwThreads, 0, ctx->stream>>>(alpha, x, xs, y, ys, e,
                                                                                       subtract ? 1 : 0, p, bar));
        else
            HME_TIMED(ctx, "axpy", axpy_kernel<1><<<grid, kEwThreads, 0, ctx->stream>>>(alpha, x, xs, y, ys, e,
                                                                                       subtract ? 1 : 0, p, bar));
        HME_CUDA(cudaGetLastError());
    });
}

int hme_scal_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t alpha, uint32_t rows, uint32_t cols, uint32_t* x, size_t rs,
                     size_t cs) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2 && alpha < p, "scal: bad context, modulus or alpha (must be canonical)");
        if (!rows || !cols) return;
        HME_REQUIRE(x, "scal: null pointer");
        bind(ctx);
        launch_unary(ctx, "scal", x, rows, cols, rs, cs, 0, alpha, p);
    });
}

int hme_fill_u32_dev(hme_ctx* ctx, uint32_t rows, uint32_t cols, uint32_t* x, size_t rs, size_t cs, uint32_t value) {
    return guard([&] {
        HME_REQUIRE(ctx, "fill: null context");
        if (!rows || !cols) return;
        HME_REQUIRE(x, "fill: null pointer");
        bind(ctx);
        launch_unary(ctx, "fill", x, rows, cols, rs, cs, 1, value, 0);
    });
}

int hme_canonicalise_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t rows, uint32_t cols, uint32_t* v, size_t rs,
                             size_t cs) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2 && p <= 0x80000000u, "canonicalise: bad context or modulus (2p must fit 32 bits)");
        if (!rows || !cols) return;
        HME_REQUIRE(v, "canonicalise: null pointer");
        bind(ctx);
        launch_unary(ctx, "canonicalise", v, rows, cols, rs, cs, 2, 0, p);
    });
}

int hme_copy_u32_dev(hme_ctx* ctx, uint32_t rows, uint32_t cols, const uint32_t* src, size_t s_rs, size_t s_cs,
                     uint32_t* dst, size_t d_rs, size_t d_cs) {
    return guard([&] {
        HME_REQUIRE(ctx, "copy: null context");
        if (!rows || !cols) return;
        HME_REQUIRE(src && dst, "copy: null pointer");
        if (src == dst && s_rs == d_rs && s_cs == d_cs) return;
        HME_REQUIRE(!overlap(src, rows, cols, s_rs, s_cs, dst, rows, cols, d_rs, d_cs), "copy: overlapping windows");
        bind(ctx);
        const bool ic = inner_is_cols(rows, cols, s_rs, s_cs);
        const int V = vec_width(ic, rows, cols, {{src, s_rs, s_cs}, {dst, d_rs, d_cs}});
        const Ew e = make_ew(rows, cols, ic, V);
        const Strides ss = strides_of(s_rs, s_cs, ic), ds = strides_of(d_rs, d_cs, ic);
        const int grid = ew_grid(e.ntiles, ctx->num_sms);
        if (V == 4)
            HME_TIMED(ctx, "copy", copy_kernel<4><<<grid, kEwThreads, 0, ctx->stream>>>(src, ss, dst, ds, e));
        else
            HME_TIMED(ctx, "copy", copy_kernel<1><<<grid, kEwThreads, 0, ctx->stream>>>(src, ss, dst, ds, e));
        HME_CUDA(cudaGetLastError());
    });
}

int hme_canonicalise_acc64_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t rows, uint32_t cols, const uint64_t* acc,
                                   size_t a_rs, size_t a_cs, uint32_t* dst, size_t d_rs, size_t d_cs) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2, "canonicalise: bad context or modulus");
        if (!rows || !cols) return;
        HME_REQUIRE(acc && dst, "canonicalise: null pointer");
        HME_REQUIRE(!overlap(acc, rows, cols, a_rs, a_cs, dst, rows, cols, d_rs, d_cs, 8),
                    "canonicalise: overlapping windows");
        bind(ctx);
        const bool ic = inner_is_cols(rows, cols, a_rs, a_cs);
        const int V = vec_width(ic, rows, cols, {{acc, a_rs, a_cs}, {dst, d_rs, d_cs}});
        const Ew e = make_ew(rows, cols, ic, V);
        const Strides as = strides_of(a_rs, a_cs, ic), ds = strides_of(d_rs, d_cs, ic);
        const int grid = ew_grid(e.ntiles, ctx->num_sms);
        const uint64_t bar = make_mod(p).barrett;
        if (V == 4)
            HME_TIMED(ctx, "canonicalise",
                      canon64_kernel<4><<<grid, kEwThreads, 0, ctx->stream>>>(acc, as, dst, ds, e, p, bar));
        else
            HME_TIMED(ctx, "canonicalise",
                      canon64_kernel<1><<<grid, kEwThreads, 0, ctx->stream>>>(acc, as, dst, ds, e, p, bar));
        HME_CUDA(cudaGetLastError());
    });
}

int hme_transpose_u32_dev(hme_ctx* ctx, uint32_t rows_dst, uint32_t cols_dst, const uint32_t* src, size_t s_rs,
                          size_t s_cs, uint32_t* dst, size_t d_rs, size_t d_cs) {
    return guard([&] {
        HME_REQUIRE(ctx, "transpose: null context");
        if (!rows_dst || !cols_dst) return;
        HME_REQUIRE(src && dst, "transpose: null pointer");
        HME_REQUIRE(!overlap(src, cols_dst, rows_dst, s_rs, s_cs, dst, rows_dst, cols_dst, d_rs, d_cs),
                    "transpose: overlapping windows");
        bind(ctx);
        launch_transpose(ctx, src, s_rs, s_cs, dst, d_rs, d_cs, rows_dst, cols_dst);
    });
}

int hme_axpy_identity_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t alpha, uint32_t rows, uint32_t cols, uint32_t* y,
                              size_t rs, size_t cs, int subtract) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2 && alpha < p, "axpy_identity: bad context, modulus or alpha (must be canonical)");
        const uint32_t n = std::min(rows, cols);
        if (!n) return;
        HME_REQUIRE(y, "axpy_identity: null pointer");
        bind(ctx);
        const int grid = static_cast<int>(std::min<uint32_t>((n + 255) / 256, ctx->num_sms * 8));
        HME_TIMED(ctx, "axpy_identity", axpy_identity_kernel<<<grid, 256, 0, ctx->stream>>>(alpha, y, rs, cs, n,
                                                                                           subtract ? 1 : 0, p));
        HME_CUDA(cudaGetLastError());
    });
}

int hme_gather_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t alpha, uint32_t beta, const uint32_t* a, uint32_t a_rows,
                       uint32_t a_cols, size_t a_rs, size_t a_cs, uint32_t row_off, const uint32_t* cols,
                       const uint32_t* rows, uint32_t c_rows, uint32_t c_cols, uint32_t* c, size_t c_rs, size_t c_cs,
                       int accumulate) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2 && alpha < p && beta < p, "gather: bad context, modulus or coefficients");
        if (!c_rows || !c_cols) return;
        HME_REQUIRE(c, "gather: null output");
        const bool has_a = a != nullptr && beta != 0;
        if (has_a) {
            HME_REQUIRE(rows != nullptr || a_rows == c_rows, "gather: row count mismatch");
            HME_REQUIRE(cols != nullptr || a_cols == c_cols, "gather: column count mismatch");
            HME_REQUIRE(!overlap(a, a_rows, a_cols, a_rs, a_cs, c, c_rows, c_cols, c_rs, c_cs),
                        "gather: output aliases the source");
        }
        bind(ctx);
        const uint32_t* as = has_a ? a : nullptr;
        const bool v4 = cols == nullptr && c_cols % 4 == 0 && c_cs == 1 && (c_rows == 1 || c_rs % 4 == 0) &&
                        reinterpret_cast<uintptr_t>(c) % 16 == 0 &&
                        (as == nullptr || (a_cs == 1 && a_rs % 4 == 0 && reinterpret_cast<uintptr_t>(as) % 16 == 0));
        const Ew e = make_ew(c_rows, c_cols, true, v4 ? 4 : 1);
        const int grid = ew_grid(e.ntiles, ctx->num_sms);
        const uint64_t bar = make_mod(p).barrett;
        if (v4)
            HME_TIMED(ctx, "gather", gather_kernel<4><<<grid, kEwThreads, 0, ctx->stream>>>(
                                         alpha, has_a ? beta : 0u, as, a_rs, a_cs, row_off, cols, rows, c, c_rs, c_cs, e,
                                         accumulate ? 1 : 0, p, bar));
        else
            HME_TIMED(ctx, "gather", gather_kernel<1><<<grid, kEwThreads, 0, ctx->stream>>>(
                                         alpha, has_a ? beta : 0u, as, a_rs, a_cs, row_off, cols, rows, c, c_rs, c_cs, e,
                                         accumulate ? 1 : 0, p, bar));
        HME_CUDA(cudaGetLastError());
    });
}

int hme_trsm_unit_u32_dev(hme_ctx* ctx, uint32_t p, int lower, uint32_t m, uint32_t n, const uint32_t* T, size_t ldt,
                          uint32_t* B, size_t ldb) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2, "trsm_unit: bad context or modulus");
        if (!m || !n) return;
        HME_REQUIRE(T && B && ldt >= m && ldb >= n, "trsm_unit: bad buffers");
        HME_REQUIRE(!overlap(T, m, m, ldt, 1, B, m, n, ldb, 1), "trsm_unit: T aliases B");
        bind(ctx);
        const ModParams mp = make_mod(p);
        // the diagonal-block kernel takes 70 KB of shared memory (set on the calling device)
        HME_CUDA(cudaFuncSetAttribute(lower ? trsm_diag_kernel<true> : trsm_diag_kernel<false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kTrsmSmem)));
        const uint32_t r64 = r64_of(p);
        const uint32_t nblocks = (m + kTrsmNB - 1) / kTrsmNB;
        const int grid = static_cast<int>(std::min<uint32_t>((n + 7) / 8, ctx->num_sms * 3));
        for (uint32_t bi = 0; bi < nblocks; ++bi) {
            const uint32_t i0 = lower ? bi * kTrsmNB : (nblocks - 1 - bi) * kTrsmNB;
            const uint32_t nb = std::min(kTrsmNB, m - i0);
            if (lower)
                HME_TIMED(ctx, "trsm_diag", trsm_diag_kernel<true><<<grid, 256, kTrsmSmem, ctx->stream>>>(
                                                T, ldt, B, ldb, i0, nb, n, p, mp.barrett, r64));
            else
                HME_TIMED(ctx, "trsm_diag", trsm_diag_kernel<false><<<grid, 256, kTrsmSmem, ctx->stream>>>(
                                                T, ldt, B, ldb, i0, nb, n, p, mp.barrett, r64));
            HME_CUDA(cudaGetLastError());
            // the solved block applied to the rows still to solve (limb GEMM, Sub)
            if (lower && i0 + nb < m)
                gemm_u32_device(ctx, mp, m - i0 - nb, n, nb, T + static_cast<size_t>(i0 + nb) * ldt + i0, ldt,
                                B + static_cast<size_t>(i0) * ldb, ldb, B + static_cast<size_t>(i0 + nb) * ldb, ldb,
                                HME_SUB);
            if (!lower && i0 > 0)
                gemm_u32_device(ctx, mp, i0, n, nb, T + i0, ldt, B + static_cast<size_t>(i0) * ldb, ldb, B, ldb,
                                HME_SUB);
        }
    });
}

int hme_gemm_nt_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A, size_t lda,
                        const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc, int op) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2, "gemm_nt: bad context or modulus");
        if (!m || !n) return;
        HME_REQUIRE(k == 0 || (A && B && lda >= k && ldb >= k), "gemm_nt: bad A / B");
        bind(ctx);
        // B (n x k, row-major) -> B^T (k x n) in workspace, then the limb GEMM
        uint32_t* Bt = nullptr;
        if (k > 0) {
            Bt = static_cast<uint32_t*>(ctx->ws.get(kSlotStageB, sizeof(uint32_t) * static_cast<size_t>(k) * n));
            launch_transpose(ctx, B, ldb, 1, Bt, n, 1, k, n);
        }
        gemm_u32_device(ctx, make_mod(p), m, n, k, A, lda, Bt, n, C, ldc, op);
    });
}

int hme_schur_update_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t* L,
                             size_t ldl, const uint32_t* U, size_t ldu, uint32_t* C, size_t ldc) {
    return guard([&] {
        HME_REQUIRE(ctx && p >= 2, "schur_update: bad context or modulus");
        bind(ctx);
        gemm_u32_device(ctx, make_mod(p), m, n, k, L, ldl, U, ldu, C, ldc, HME_SUB);
    });
}

}  // extern "C"

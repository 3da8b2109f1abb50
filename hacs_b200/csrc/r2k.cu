// The device side of the Z/2^W blocked LU's operations table (W = 32 or 64):
// the session of engine::ring2k::device::Ops (reference
// src/ModArithmetic/Binary/Ring2kDevice.h:49-83, driven by ring2k::echelon_blocked
// through Ring2kDeviceLU.h; the reference's own device side is
// src/Cuda/CudaRing2k.h:27-45 with plain SIMT kernels).
//
// A session holds a column window [0, cw) of an m x n matrix over Z/2^W on the
// device (row-major, ld = cw rounded up to 16 bytes), the L store of the
// current panel and pinned staging.  One step() applies one factored panel to
// the window, all asynchronous on the session's compute stream:
//   1. the factored panel (rows r .. m-1, the panel's columns) is written into
//      the window (it carries its own row swaps);
//   2. the panel's row swaps, in order, on every other column of [0, w);
//   3. the unit-lower solve on the pivot rows r .. r+np-1, columns [u0, w)
//      (row r+t -= sum_{t2<t} L[t][t2] row r+t2, rows already final);
//   4. the trailing update C -= L21 U12 on rows r+np .. m-1, columns [u0, w):
//      W = 32 on the INT8-limb tcgen05 GEMM in its wraparound mode (4 limbs,
//      every reduction the truncation to 32 bits), W = 64 on a CUDA-core
//      kernel with 64-bit wraparound multiply-adds;
//   lookahead: the columns [la0, la1) of step 4 are updated first and their
//   rows r+np .. m-1 copied back to pinned memory on a second stream while the
//   rest of the update runs; fetch() waits for that copy only.
// Every entry is an exact value of Z/2^W computed by ring operations, so each
// one equals the host code's (echelon_blocked's axpy / gemm_sub in native
// wraparound arithmetic) whatever the summation order or tiling.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "hme_internal.h"

namespace hme {
namespace {

constexpr int kSwapThreads = 256;
constexpr int kTrsmThreads = 256;
constexpr uint32_t kMaxSwapsSmem = 4096;  // swap pairs held in shared memory by the swap kernel

// Rows a and b of the window exchanged, pair by pair in list order, in every
// column of [0, w) outside [pc0, pc1).  One thread per column: the pairs are
// applied sequentially, so a row named by several pairs moves exactly as the
// host code moves it.
template <class E>
__global__ void r2k_swap_kernel(E* W, size_t ld, uint32_t w, uint32_t pc0, uint32_t pc1, const uint32_t* swaps,
                                uint32_t nswaps) {
    __shared__ uint32_t sw[2 * kMaxSwapsSmem];
    for (uint32_t i = threadIdx.x; i < 2 * nswaps; i += blockDim.x) sw[i] = swaps[i];
    __syncthreads();
    const uint32_t other = w - (pc1 - pc0);  // columns outside the panel
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < other; t += gridDim.x * blockDim.x) {
        const uint32_t c = t < pc0 ? t : t + (pc1 - pc0);
        for (uint32_t s = 0; s < nswaps; ++s) {
            E* a = W + static_cast<size_t>(sw[2 * s]) * ld + c;
            E* b = W + static_cast<size_t>(sw[2 * s + 1]) * ld + c;
            const E x = *a;
            *a = *b;
            *b = x;
        }
    }
}

// Forward substitution with the unit lower L11 (rows 0 .. np-1 of L, ld ldl)
// on the pivot rows r .. r+np-1 of the window, columns [c0, c1): one thread per
// column walks t = 1 .. np-1 in order, each row reading the rows above it that
// this same thread has already made final.
template <class E>
__global__ void r2k_trsm_kernel(E* W, size_t ld, uint32_t r, uint32_t np, uint32_t c0, uint32_t c1, const E* L,
                                size_t ldl) {
    for (uint32_t c = c0 + blockIdx.x * blockDim.x + threadIdx.x; c < c1; c += gridDim.x * blockDim.x) {
        E* col = W + static_cast<size_t>(r) * ld + c;
        for (uint32_t t = 1; t < np; ++t) {
            const E* lt = L + static_cast<size_t>(t) * ldl;
            E acc = col[static_cast<size_t>(t) * ld];
            for (uint32_t t2 = 0; t2 < t; ++t2) acc -= __ldg(lt + t2) * col[static_cast<size_t>(t2) * ld];
            col[static_cast<size_t>(t) * ld] = acc;
        }
    }
}

// C -= A B in native 64-bit wraparound arithmetic (A m x k, B k x n, row-major):
// 64 x 64 tiles, 256 threads with 4 x 4 outputs each, k in slices of 16
// through shared memory.
constexpr int kWT = 64, kWK = 16;
__global__ void r2k_gemm_sub_u64_kernel(uint64_t* C, size_t ldc, const uint64_t* A, size_t lda, const uint64_t* B,
                                        size_t ldb, uint32_t m, uint32_t n, uint32_t k) {
    __shared__ uint64_t As[kWK][kWT + 1];
    __shared__ uint64_t Bs[kWK][kWT + 1];
    const uint32_t tm = blockIdx.y * kWT, tn = blockIdx.x * kWT;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    uint64_t acc[4][4] = {};
    for (uint32_t k0 = 0; k0 < k; k0 += kWK) {
        for (int i = threadIdx.x; i < kWK * kWT; i += blockDim.x) {
            const int kk = i % kWK, rr = i / kWK;  // A tile: rows of the tile, kWK values of k each
            const uint32_t gr = tm + rr, gk = k0 + kk;
            As[kk][rr] = (gr < m && gk < k) ? A[static_cast<size_t>(gr) * lda + gk] : 0ull;
            const int cc = i % kWT, kb = i / kWT;  // B tile: kWK rows of k, kWT columns
            const uint32_t gc = tn + cc, gk2 = k0 + kb;
            Bs[kb][cc] = (gc < n && gk2 < k) ? B[static_cast<size_t>(gk2) * ldb + gc] : 0ull;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kWK; ++kk) {
            uint64_t a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint32_t gr = tm + ty + 16 * i;
        if (gr >= m) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t gc = tn + tx + 16 * j;
            if (gc < n) C[static_cast<size_t>(gr) * ldc + gc] -= acc[i][j];
        }
    }
}

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace
}  // namespace hme

using namespace hme;

struct hme_r2k {
    hme_ctx* ctx = nullptr;
    uint32_t elem = 4, m = 0, cw = 0, panel = 0;
    size_t ldw = 0, ldl = 0;            // elements
    void* d_win = nullptr;              // m x ldw
    void* d_L = nullptr;                // m x ldl: the step's L store, row 0 = global row r
    uint32_t* d_swaps = nullptr;        // 2 x panel
    void* h_panel = nullptr;            // pinned: m x panel
    void* h_L = nullptr;                // pinned: m x panel
    uint32_t* h_swaps = nullptr;        // pinned: 2 x panel
    void* h_la = nullptr;               // pinned: m x panel (lookahead block)
    int* h_err_la = nullptr;            // pinned: the error word as of the lookahead block
    cudaStream_t s_copy = nullptr;      // lookahead copies
    cudaEvent_t ev_staged = nullptr;    // the last step's host-to-device copies are done
    cudaEvent_t ev_la_ready = nullptr;  // the lookahead columns are updated (compute stream)
    cudaEvent_t ev_la = nullptr;        // the lookahead block is in h_la (copy stream)
    bool staged_pending = false, la_pending = false;
    uint32_t la_rows = 0, la_cols = 0;
};

namespace hme {
namespace {

size_t r2k_bytes(uint32_t elem, uint32_t m, uint32_t cw, uint32_t panel) {
    const size_t ldw = round_up(std::max<uint32_t>(cw, 1), 16 / elem), ldl = round_up(std::max<uint32_t>(panel, 1), 16 / elem);
    size_t b = static_cast<size_t>(elem) * m * (ldw + ldl) + 8ull * panel + 4096;
    if (elem == 4) {  // the limb GEMM's planes: 4 limbs of L21, 16 of U12, k <= panel rounded to a k-block
        const size_t kp = round_up(std::max<uint32_t>(panel, 1), panel <= 32 ? 32 : panel <= 64 ? 64 : 128);
        b += 4 * static_cast<size_t>(m) * kp + 16 * static_cast<size_t>(cw) * kp;
    }
    return b;
}

void r2k_free(hme_r2k* s) {
    if (!s) return;
    if (s->ctx) cudaSetDevice(s->ctx->device);
    if (s->ctx) cudaStreamSynchronize(s->ctx->stream);
    if (s->s_copy) cudaStreamSynchronize(s->s_copy);
    if (s->d_win) cudaFree(s->d_win);
    if (s->d_L) cudaFree(s->d_L);
    if (s->d_swaps) cudaFree(s->d_swaps);
    if (s->h_panel) cudaFreeHost(s->h_panel);
    if (s->h_L) cudaFreeHost(s->h_L);
    if (s->h_swaps) cudaFreeHost(s->h_swaps);
    if (s->h_la) cudaFreeHost(s->h_la);
    if (s->h_err_la) cudaFreeHost(s->h_err_la);
    if (s->ev_staged) cudaEventDestroy(s->ev_staged);
    if (s->ev_la_ready) cudaEventDestroy(s->ev_la_ready);
    if (s->ev_la) cudaEventDestroy(s->ev_la);
    if (s->s_copy) cudaStreamDestroy(s->s_copy);
    if (s->ctx) hme_ctx_destroy(s->ctx);
    delete s;
}

// Copy `rows` rows of `cols` elements between two pitched host buffers.
void host_copy_rows(void* dst, size_t ldd, const void* src, size_t lds, uint32_t rows, uint32_t cols, uint32_t elem) {
    const size_t w = static_cast<size_t>(cols) * elem;
    if (ldd == cols && lds == cols) {
        std::memcpy(dst, src, w * rows);
        return;
    }
    for (uint32_t i = 0; i < rows; ++i)
        std::memcpy(static_cast<char*>(dst) + i * ldd * elem, static_cast<const char*>(src) + i * lds * elem, w);
}

// C (rows x cols at window (r0, c0)) -= L21 (rows x np, ld ldl) U12 (np rows from window row ru, columns c0..)
void r2k_update(hme_r2k* s, uint32_t ru, uint32_t r0, uint32_t rows, uint32_t np, uint32_t c0, uint32_t c1,
                const void* L21) {
    if (c1 <= c0 || rows == 0 || np == 0) return;
    hme_ctx* ctx = s->ctx;
    const uint32_t cols = c1 - c0;
    if (s->elem == 4) {
        uint32_t* W = static_cast<uint32_t*>(s->d_win);
        gemm_u32_wrap_device(ctx, rows, cols, np, static_cast<const uint32_t*>(L21), s->ldl,
                             W + static_cast<size_t>(ru) * s->ldw + c0, s->ldw,
                             W + static_cast<size_t>(r0) * s->ldw + c0, s->ldw, HME_SUB);
    } else {
        uint64_t* W = static_cast<uint64_t*>(s->d_win);
        const dim3 grid((cols + kWT - 1) / kWT, (rows + kWT - 1) / kWT);
        HME_TIMED(ctx, "r2k_gemm64",
                  r2k_gemm_sub_u64_kernel<<<grid, 256, 0, ctx->stream>>>(
                      W + static_cast<size_t>(r0) * s->ldw + c0, s->ldw, static_cast<const uint64_t*>(L21), s->ldl,
                      W + static_cast<size_t>(ru) * s->ldw + c0, s->ldw, rows, cols, np));
        HME_CUDA(cudaGetLastError());
    }
}

template <class E>
void r2k_step_kernels(hme_r2k* s, const hme_r2k_step_args& a, uint32_t w) {
    hme_ctx* ctx = s->ctx;
    E* W = static_cast<E*>(s->d_win);
    const E* L = static_cast<const E*>(s->d_L);
    if (a.nswaps > 0 && w > a.pc1 - a.pc0) {
        const uint32_t other = w - (a.pc1 - a.pc0);
        const int grid = static_cast<int>(std::min<uint32_t>((other + kSwapThreads - 1) / kSwapThreads,
                                                             static_cast<uint32_t>(ctx->num_sms) * 4));
        HME_TIMED(ctx, "r2k_swap",
                  r2k_swap_kernel<E><<<grid, kSwapThreads, 0, ctx->stream>>>(W, s->ldw, w, a.pc0, a.pc1, s->d_swaps,
                                                                             a.nswaps));
        HME_CUDA(cudaGetLastError());
    }
    if (a.np == 0 || a.u0 >= w) return;
    if (a.np > 1) {
        const uint32_t cols = w - a.u0;
        const int grid = static_cast<int>(std::min<uint32_t>((cols + kTrsmThreads - 1) / kTrsmThreads,
                                                             static_cast<uint32_t>(ctx->num_sms) * 8));
        HME_TIMED(ctx, "r2k_trsm",
                  r2k_trsm_kernel<E><<<grid, kTrsmThreads, 0, ctx->stream>>>(W, s->ldw, a.r, a.np, a.u0, w, L,
                                                                             s->ldl));
        HME_CUDA(cudaGetLastError());
    }
}

}  // namespace
}  // namespace hme

extern "C" {

size_t hme_r2k_session_bytes(uint32_t elem, uint32_t m, uint32_t cw, uint32_t panel) {
    if (elem != 4 && elem != 8) return 0;
    return r2k_bytes(elem, m, cw, panel);
}

uint32_t hme_r2k_plan(int device, uint32_t elem, uint32_t m, uint32_t n, uint32_t panel, uint64_t vram_cap) {
    if ((elem != 4 && elem != 8) || m == 0 || n == 0 || panel == 0) return 0;
    try {
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
            cudaGetLastError();
            return 0;
        }
        cudaDeviceProp prop{};
        if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) return 0;
        int cur = 0;
        cudaGetDevice(&cur);
        size_t free_b = 0, total_b = 0;
        cudaSetDevice(device);
        const cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
        cudaSetDevice(cur);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        // keep 1 GiB or 2 % of the card (whichever is larger) free for everyone else on the device
        const size_t reserve = std::max<size_t>(size_t(1) << 30, total_b / 50);
        size_t budget = free_b > reserve ? free_b - reserve : 0;
        if (vram_cap != 0 && budget > vram_cap) budget = static_cast<size_t>(vram_cap);
        if (r2k_bytes(elem, m, n, panel) <= budget) return n;
        const size_t base = r2k_bytes(elem, m, 0, panel);
        const size_t per_col = r2k_bytes(elem, m, 1024, panel) - base;  // bytes per 1024 window columns
        if (budget <= base) return 0;
        size_t cw = (budget - base) / per_col * 1024;
        cw -= cw % panel;
        // a window of fewer than four panels re-streams the columns right of it too often: decline
        if (cw < 4ull * panel) return 0;
        return static_cast<uint32_t>(std::min<size_t>(cw, n));
    } catch (...) {
        return 0;
    }
}

int hme_r2k_open(int device, uint32_t elem, uint32_t m, uint32_t cw, uint32_t panel, hme_r2k** out) {
    return guard([&] {
        HME_REQUIRE(out != nullptr, "hme_r2k_open: out is null");
        *out = nullptr;
        HME_REQUIRE(elem == 4 || elem == 8, "hme_r2k_open: elem must be 4 (Z/2^32) or 8 (Z/2^64)");
        HME_REQUIRE(m > 0 && cw > 0 && panel > 0, "hme_r2k_open: empty session");
        HME_REQUIRE(m < (1u << 30) && cw < (1u << 30) && panel <= (1u << 16), "hme_r2k_open: session too large");
        hme_r2k* s = new hme_r2k();
        try {
            const int rc = hme_ctx_create(device, &s->ctx);
            if (rc != HME_OK) throw Error(rc, hme_last_error());
            bind(s->ctx);
            s->elem = elem;
            s->m = m;
            s->cw = cw;
            s->panel = panel;
            s->ldw = round_up(cw, 16 / elem);
            s->ldl = round_up(panel, 16 / elem);
            HME_CUDA(cudaMalloc(&s->d_win, static_cast<size_t>(elem) * m * s->ldw));
            HME_CUDA(cudaMalloc(&s->d_L, static_cast<size_t>(elem) * m * s->ldl));
            HME_CUDA(cudaMalloc(&s->d_swaps, 8ull * panel));
            HME_CUDA(cudaMallocHost(&s->h_panel, static_cast<size_t>(elem) * m * panel));
            HME_CUDA(cudaMallocHost(&s->h_L, static_cast<size_t>(elem) * m * panel));
            HME_CUDA(cudaMallocHost(&s->h_swaps, 8ull * panel));
            HME_CUDA(cudaMallocHost(&s->h_la, static_cast<size_t>(elem) * m * panel));
            HME_CUDA(cudaMallocHost(&s->h_err_la, sizeof(int)));
            *s->h_err_la = 0;
            HME_CUDA(cudaStreamCreateWithFlags(&s->s_copy, cudaStreamNonBlocking));
            HME_CUDA(cudaEventCreateWithFlags(&s->ev_staged, cudaEventDisableTiming));
            HME_CUDA(cudaEventCreateWithFlags(&s->ev_la_ready, cudaEventDisableTiming));
            HME_CUDA(cudaEventCreateWithFlags(&s->ev_la, cudaEventDisableTiming));
        } catch (...) {
            r2k_free(s);
            throw;
        }
        *out = s;
    });
}

int hme_r2k_put(hme_r2k* s, const void* host, size_t ldh, uint32_t r0, uint32_t rows, uint32_t c0, uint32_t cols) {
    return guard([&] {
        HME_REQUIRE(s != nullptr, "hme_r2k_put: null session");
        HME_REQUIRE(static_cast<uint64_t>(r0) + rows <= s->m && static_cast<uint64_t>(c0) + cols <= s->cw,
                    "hme_r2k_put: block outside the window");
        if (rows == 0 || cols == 0) return;
        HME_REQUIRE(host != nullptr && ldh >= cols, "hme_r2k_put: bad host block");
        bind(s->ctx);
        const cudaStream_t st = s->ctx->stream;
        if (s->la_pending) HME_CUDA(cudaStreamWaitEvent(st, s->ev_la, 0));  // the readback of these columns first
        const size_t e = s->elem;
        HME_CUDA(cudaMemcpy2DAsync(static_cast<char*>(s->d_win) + (r0 * s->ldw + c0) * e, s->ldw * e, host, ldh * e,
                                   cols * e, rows, cudaMemcpyHostToDevice, st));
        HME_CUDA(cudaStreamSynchronize(st));
    });
}

int hme_r2k_get(hme_r2k* s, void* host, size_t ldh, uint32_t r0, uint32_t rows, uint32_t c0, uint32_t cols) {
    return guard([&] {
        HME_REQUIRE(s != nullptr, "hme_r2k_get: null session");
        HME_REQUIRE(static_cast<uint64_t>(r0) + rows <= s->m && static_cast<uint64_t>(c0) + cols <= s->cw,
                    "hme_r2k_get: block outside the window");
        bind(s->ctx);
        check_device_error(s->ctx);  // synchronises the compute stream
        if (rows == 0 || cols == 0) return;
        HME_REQUIRE(host != nullptr && ldh >= cols, "hme_r2k_get: bad host block");
        const size_t e = s->elem;
        HME_CUDA(cudaMemcpy2DAsync(host, ldh * e, static_cast<const char*>(s->d_win) + (r0 * s->ldw + c0) * e,
                                   s->ldw * e, cols * e, rows, cudaMemcpyDeviceToHost, s->ctx->stream));
        HME_CUDA(cudaStreamSynchronize(s->ctx->stream));
    });
}

int hme_r2k_step(hme_r2k* s, const hme_r2k_step_args* ap) {
    return guard([&] {
        HME_REQUIRE(s != nullptr && ap != nullptr, "hme_r2k_step: null argument");
        const hme_r2k_step_args& a = *ap;
        const uint32_t w = a.w ? a.w : s->cw;
        HME_REQUIRE(a.m == s->m, "hme_r2k_step: m differs from the session's");
        HME_REQUIRE(w <= s->cw, "hme_r2k_step: w beyond the window");
        HME_REQUIRE(static_cast<uint64_t>(a.r) + a.np <= s->m, "hme_r2k_step: pivot rows outside the matrix");
        HME_REQUIRE(a.pc0 <= a.pc1 && a.pc1 <= w, "hme_r2k_step: panel columns outside the window");
        HME_REQUIRE(a.pc1 - a.pc0 <= s->panel, "hme_r2k_step: panel wider than the session's");
        HME_REQUIRE(a.np <= s->panel, "hme_r2k_step: more pivots than the panel width");
        HME_REQUIRE(a.nswaps <= s->panel && a.nswaps <= hme::kMaxSwapsSmem, "hme_r2k_step: too many swaps");
        HME_REQUIRE(a.la0 <= a.la1 && a.la1 <= w && a.la1 - a.la0 <= s->panel, "hme_r2k_step: bad lookahead block");
        const uint32_t rows = s->m - a.r;
        const uint32_t pw = a.pc1 - a.pc0;
        const bool write_panel = a.panel != nullptr && pw > 0 && rows > 0;
        const bool update = a.np > 0 && a.u0 < w;
        HME_REQUIRE(!write_panel || a.ldp >= pw, "hme_r2k_step: ldp < panel width");
        HME_REQUIRE(!update || (a.L != nullptr && a.ldl >= a.np), "hme_r2k_step: missing L store");
        HME_REQUIRE(a.nswaps == 0 || a.swaps != nullptr, "hme_r2k_step: missing swap list");
        HME_REQUIRE(!(a.la1 > a.la0) || (a.la0 >= a.u0 || !update), "hme_r2k_step: lookahead block left of u0");
        for (uint32_t i = 0; i < 2 * a.nswaps; ++i)
            HME_REQUIRE(a.swaps[i] < s->m, "hme_r2k_step: swap row outside the matrix");
        bind(s->ctx);
        hme_ctx* ctx = s->ctx;
        const cudaStream_t st = ctx->stream;
        const size_t e = s->elem;
        // the staging buffers are reused: wait until the previous step's copies out of them are done
        if (s->staged_pending) HME_CUDA(cudaEventSynchronize(s->ev_staged));
        if (write_panel) host_copy_rows(s->h_panel, pw, a.panel, a.ldp, rows, pw, s->elem);
        if (update) host_copy_rows(s->h_L, a.np, a.L, a.ldl, rows, a.np, s->elem);
        if (a.nswaps) std::memcpy(s->h_swaps, a.swaps, 8ull * a.nswaps);
        // the previous lookahead readback must be done before this step writes those columns
        if (s->la_pending) HME_CUDA(cudaStreamWaitEvent(st, s->ev_la, 0));
        if (write_panel)
            HME_CUDA(cudaMemcpy2DAsync(static_cast<char*>(s->d_win) + (static_cast<size_t>(a.r) * s->ldw + a.pc0) * e,
                                       s->ldw * e, s->h_panel, pw * e, pw * e, rows, cudaMemcpyHostToDevice, st));
        if (update)
            HME_CUDA(cudaMemcpy2DAsync(s->d_L, s->ldl * e, s->h_L, a.np * e, a.np * e, rows, cudaMemcpyHostToDevice,
                                       st));
        if (a.nswaps) HME_CUDA(cudaMemcpyAsync(s->d_swaps, s->h_swaps, 8ull * a.nswaps, cudaMemcpyHostToDevice, st));
        HME_CUDA(cudaEventRecord(s->ev_staged, st));
        s->staged_pending = true;
        if (s->elem == 4) r2k_step_kernels<uint32_t>(s, a, w);
        else r2k_step_kernels<uint64_t>(s, a, w);
        // the trailing update, lookahead columns first
        const uint32_t r1 = a.r + a.np, below = s->m - r1;
        const char* L21 = static_cast<const char*>(s->d_L) + static_cast<size_t>(a.np) * s->ldl * e;
        const bool la = a.la1 > a.la0;
        const bool gemm = update && below > 0;
        if (gemm) r2k_update(s, a.r, r1, below, a.np, la ? a.la0 : a.u0, la ? a.la1 : w, L21);
        s->la_pending = false;
        if (la) {
            // rows r+np .. m-1 of the lookahead columns, read back on the copy stream
            HME_CUDA(cudaEventRecord(s->ev_la_ready, st));
            HME_CUDA(cudaStreamWaitEvent(s->s_copy, s->ev_la_ready, 0));
            s->la_rows = below;
            s->la_cols = a.la1 - a.la0;
            if (below > 0)
                HME_CUDA(cudaMemcpy2DAsync(s->h_la, s->la_cols * e,
                                           static_cast<const char*>(s->d_win) + (static_cast<size_t>(r1) * s->ldw + a.la0) * e,
                                           s->ldw * e, s->la_cols * e, below, cudaMemcpyDeviceToHost, s->s_copy));
            HME_CUDA(cudaMemcpyAsync(s->h_err_la, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, s->s_copy));
            HME_CUDA(cudaEventRecord(s->ev_la, s->s_copy));
            s->la_pending = true;
            // the rest of the update while the block travels
            if (gemm) {
                r2k_update(s, a.r, r1, below, a.np, a.u0, a.la0, L21);
                r2k_update(s, a.r, r1, below, a.np, a.la1, w, L21);
            }
        }
        HME_CUDA(cudaGetLastError());
    });
}

int hme_r2k_fetch(hme_r2k* s, void* host, size_t ldh) {
    return guard([&] {
        HME_REQUIRE(s != nullptr, "hme_r2k_fetch: null session");
        HME_REQUIRE(s->la_pending, "hme_r2k_fetch: the last step asked for no lookahead block");
        HME_REQUIRE(host != nullptr && ldh >= s->la_cols, "hme_r2k_fetch: bad host block");
        bind(s->ctx);
        HME_CUDA(cudaEventSynchronize(s->ev_la));
        if (*static_cast<volatile int*>(s->h_err_la) != 0)
            throw Error(HME_ETIMEOUT, "hme_r2k_fetch: a bounded device-side wait ran out in the lookahead update");
        host_copy_rows(host, ldh, s->h_la, s->la_cols, s->la_rows, s->la_cols, s->elem);
    });
}

int hme_r2k_close(hme_r2k* s) {
    return guard([&] {
        if (!s) return;
        int code = 0;
        if (s->ctx) {
            cudaSetDevice(s->ctx->device);
            if (cudaStreamSynchronize(s->ctx->stream) == cudaSuccess &&
                cudaMemcpy(&code, s->ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
                code = 0;
        }
        r2k_free(s);
        if (code != 0) throw Error(HME_ETIMEOUT, "hme_r2k_close: a bounded device-side wait ran out in the session");
    });
}

}  // extern "C"

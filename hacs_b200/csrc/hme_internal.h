// Host-side internals shared by the translation units of libhme: the context,
// error plumbing and the device workspace.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/hme.h"
#include "hme_mod.h"

namespace hme {

// Thrown inside the library, turned into a status code at the C boundary.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);

#define HME_CUDA(call)                                                                                  \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            throw ::hme::Error(e_ == cudaErrorMemoryAllocation ? HME_ENOMEM : HME_ECUDA,                \
                               std::string(#call) + ": " + cudaGetErrorString(e_));                     \
    } while (0)

#define HME_REQUIRE(cond, msg)                                        \
    do {                                                              \
        if (!(cond)) throw ::hme::Error(HME_EINVAL, (msg));           \
    } while (0)

// Grow-only device scratch arena: one region per purpose ("slot") so that a
// caller holding slot 0 (limb planes of A) can also hold slot 1 (planes of B).
enum WorkspaceSlot : int {
    kSlotPlanesA = 0,  // limb planes of the left GEMM operand
    kSlotPlanesB = 1,  // limb planes of 256^i * right operand
    kSlotStageA = 2,   // device copies made by the host-pointer entry points
    kSlotStageB = 3,
    kSlotStageC = 4,
    kSlotElim0 = 5,    // elimination / ring drivers
    kSlotElim1 = 6,
    kSlotElim2 = 7,
    kSlotElim3 = 8,
    kSlotElim4 = 9,
    kSlotElim5 = 10,
    kSlotElim6 = 11,
    kSlotRing0 = 12,   // Howell / Smith drivers
    kSlotRing1 = 13,
    kSlotRing2 = 14,
    kSlotRing3 = 15,
    kSlotRing4 = 16,
    kSlotRing5 = 17,
    kSlotJobs0 = 18,   // batched job stream
    kSlotJobs1 = 19,
    kSlotJobs2 = 20,
    kSlotJobs3 = 21,
    kSlotJobs4 = 22,
    kSlotJobs5 = 23,
    kSlotJobs6 = 24,
    kSlotJobs7 = 25,
    kSlotSched0 = 26,  // scheduler / autotuner
    kSlotSched1 = 27,
    kSlotJobs8 = 28,   // batched job stream: the pivot blocks' inverses
    kSlotRns0 = 29,    // u64 GEMM: residues of A, B and the products mod the RNS primes
    kSlotRns1 = 30,
    kSlotRns2 = 31,
};

struct Workspace {
    static constexpr int kSlots = 32;
    void* ptr[kSlots] = {};
    size_t size[kSlots] = {};
    // keep a slot's previous allocation alive when it grows (freed by release()), so that CUDA
    // graphs captured with the old pointers stay valid (hme_ctx_set_workspace_retain)
    bool retain = false;
    std::vector<void*> retired;
    void* get(int slot, size_t bytes);
    void release();
};

}  // namespace hme

namespace hme {
// Tunables of the device elimination (elim.cu); none of them changes a value.
struct ElimOptions {
    int panel = 64;         // LU panel width (columns, <= 128)
    int rows_per_cta = 32;  // active rows per CTA of the cooperative panel kernel
    int panel_ctas = 0;     // cap on the panel kernel's grid (0 = one CTA per SM)
    int back_block = 128;   // block of the RREF backward substitution
    bool want_diag = false; // return the U diagonal (determinant)
    int panel_kernel = 0;   // 0 automatic, 1 cooperative grid kernel, 2 cluster kernel where the panel fits
    bool no_lookahead = false;  // factor each panel only after the previous update (no second stream)
};

// Optional per-kernel CUDA-event timing (bench / profiling use): when enabled,
// every launch of a named kernel is bracketed by two events on the launching
// stream; hme_ctx_kernel_time() sums the elapsed times per name.
struct KernelTimer {
    bool on = false;
    struct Rec {
        const char* name;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t take();
    void begin(const char* name, cudaStream_t s);
    void end(cudaStream_t s);
    void clear();
};
}  // namespace hme

struct hme_ctx {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;      // active stream
    cudaStream_t own_stream = nullptr;  // created by the context
    int* d_err = nullptr;               // device error word written by bounded waits
    int* h_err = nullptr;               // pinned host copy of d_err (read after each synchronising call)
    cudaStream_t copy_in = nullptr;     // host-pointer GEMM: host -> device copies (created on first use)
    cudaStream_t copy_out = nullptr;    // host-pointer GEMM: device -> host copies
    std::vector<cudaEvent_t> pipe_ev;   // events of the host-pointer GEMM pipeline (reused)
    uint64_t launches = 0;
    hme::Workspace ws;
    hme::KernelTimer timer;
    hme::ElimOptions elim;
    int fixed_variant = -1;          // >= 0: every GEMM of this context uses that variant
    int sched_policy = 0;            // 0 shape heuristic, 1 learned planner table
    void* sched_table = nullptr;     // planner decisions by shape class (sched.cu)
    void* sched_rank_table = nullptr;  // the rank rounds' planner decisions by shape class (sched.cu)
    int gemm_sm_cap = 0;             // > 0: persistent GEMM grids use at most this many SMs
    cudaStream_t aux_stream = nullptr;   // elimination: the lookahead panel's stream (created on first use)
    void* elim_pinned = nullptr;         // elimination: pinned copies of the panel scratch, permutations
    size_t elim_pinned_bytes = 0;
    std::vector<cudaEvent_t> elim_ev;    // elimination: lookahead events
    uint64_t elim_block_panels = 0;      // field panels settled by the top-block path
    uint64_t elim_search_panels = 0;     // panels factored by a searching kernel
};

// Bracket one kernel launch with timing events when the context's timer is on.
#define HME_TIMED(ctx, name, ...)                                   \
    do {                                                            \
        if ((ctx)->timer.on) (ctx)->timer.begin(name, (ctx)->stream); \
        __VA_ARGS__;                                                \
        if ((ctx)->timer.on) (ctx)->timer.end((ctx)->stream);       \
        ++(ctx)->launches;                                          \
    } while (0)

namespace hme {

// Copy `rows` rows of `width` bytes between pitched buffers: one linear copy
// when both sides are contiguous (the DMA engines stream a linear copy at full
// PCIe rate), a pitched 2D copy otherwise.
inline cudaError_t copy_rows_async(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                                   size_t rows, cudaMemcpyKind kind, cudaStream_t st) {
    if (dpitch == width && spitch == width) return cudaMemcpyAsync(dst, src, width * rows, kind, st);
    return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, kind, st);
}

// Fails with HME_ETIMEOUT (and clears the word) when a kernel on this context
// recorded a device-side wait that ran out.  Synchronises the stream.
void check_device_error(hme_ctx* ctx);

// Make the context's device current on the calling thread.
void bind(hme_ctx* ctx);

// Run f, turning every exception into a status code and hme_last_error().
template <class F>
inline int guard(F&& f) {
    try {
        f();
        return HME_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return HME_ENOMEM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return HME_EINVAL;
    } catch (...) {
        set_last_error("unknown exception");
        return HME_EINVAL;
    }
}

// Kernel attributes (the dynamic shared-memory limit, cluster permissions)
// belong to one device: a process that drives several GPUs must set them on
// each.  OncePerDevice runs its set-up once per device id on the calling
// thread's current device; a set-up that throws is retried on the next call.
class OncePerDevice {
  public:
    static constexpr int kMaxDevices = 64;
    template <class F>
    void run(F&& f) {
        int dev = 0;
        HME_CUDA(cudaGetDevice(&dev));
        HME_REQUIRE(dev >= 0 && dev < kMaxDevices, "device id out of range");
        const uint64_t bit = uint64_t(1) << dev;
        if (done_.load(std::memory_order_acquire) & bit) return;
        std::lock_guard<std::mutex> lock(mu_);
        if (done_.load(std::memory_order_relaxed) & bit) return;
        f(dev);
        done_.fetch_or(bit, std::memory_order_release);
    }

  private:
    std::mutex mu_;
    std::atomic<uint64_t> done_{0};
};

// Deterministic primality for 32-bit moduli (Miller-Rabin, bases 2, 7, 61).
bool is_prime_u32(uint32_t p);

// ---- the GEMM variants (limb_gemm.cu, simt_gemm.cu) -----------------------
// The schedules of one product; every variant computes the same residues.
enum GemmVariant : int {
    kVariantWide = 0,    // INT8-limb tcgen05 GEMM, wide tiles (L*BN ~ 256)
    kVariantNarrow = 1,  // INT8-limb tcgen05 GEMM, half-width tiles (twice the tiles)
    kVariantSimt32 = 2,  // CUDA-core GEMM, 32 x 32 tiles, one launch
    kVariantSimt64 = 3,  // CUDA-core GEMM, 64 x 64 tiles, one launch
    kGemmVariants = 4,
};
// C op= A*B mod p with device pointers, on ctx->stream; the variant comes from
// the context's scheduler (sched.cu) unless a fixed variant is set.
void gemm_u32_device(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A,
                     size_t lda, const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc, int op);
void gemm_u32_variant(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A,
                      size_t lda, const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc, int op, int variant);
// C op= A*B mod p with HOST pointers: copies in, product, copy out, with the
// copies of row chunks pipelined against the GEMMs of the chunks before them
// (limb_gemm.cu).  Synchronous; tensor-core variants only.
void gemm_u32_host(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A,
                   size_t lda, const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc, int op, int variant);
void simt_gemm_u32_device(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A,
                          size_t lda, const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc, int op, int tile);
// The limb GEMM on planes that are already split (A: [L][m][Kp] with a_plane
// bytes between limb planes; B: [L][L][n][Kp], byte j of 256^i * B mod p,
// K-major), K padded to limb_kp(k) with zeros; the shape heuristic's tile.
int limb_kp(uint32_t k);
void gemm_u32_planes(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k, int Kp, uint8_t* pa,
                     uint64_t a_plane, uint8_t* pb, uint32_t* C, size_t ldc, int op);
// C op= A*B mod 2^32 (native wraparound u32 arithmetic, any u32 words) on the
// same limb-split + tcgen05 kernels: with the modulus constants p = 0 and
// Barrett m = 0 every reduction of the split and the epilogue is the
// truncation to 32 bits (x - mulhi(x, 0) * 0 = x), and 256^i * B "mod p" is
// B << 8i truncated, so sum_j 256^j D_j truncated is A*B mod 2^32.  Device
// pointers, on ctx->stream.
void gemm_u32_wrap_device(hme_ctx* ctx, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A, size_t lda,
                          const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc, int op);
// The shape heuristic (the method without a learned model).
int gemm_default_variant(const hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n);
// The scheduler's choice for one product (sched.cu), and its tear-down.
int sched_variant(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k);
// The learned plan's decision for one product's shape class, or -1 when the
// plan holds none (sched.cu).
int sched_planned_variant(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k);
// The same for the schedule of a batched job's rank rounds (RankVariant).
int sched_planned_rank_variant(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k);
void sched_release(hme_ctx* ctx);

}  // namespace hme

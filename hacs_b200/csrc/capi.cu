// The C ABI of libhme (include/hme.h): contexts, error plumbing, workspace and
// the GEMM entry points.  No C++ exception crosses this boundary.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "hme_internal.h"
#include "hme_ptx.cuh"

namespace hme {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

void* Workspace::get(int slot, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (size[slot] < bytes) {
        if (ptr[slot] && retain) retired.push_back(ptr[slot]);
        else if (ptr[slot]) HME_CUDA(cudaFree(ptr[slot]));
        ptr[slot] = nullptr;
        size[slot] = 0;
        // grow with headroom so a sequence of slightly larger calls does not reallocate every time
        const size_t want = bytes + bytes / 8;
        HME_CUDA(cudaMalloc(&ptr[slot], want));
        size[slot] = want;
    }
    return ptr[slot];
}

void Workspace::release() {
    for (int s = 0; s < kSlots; ++s) {
        if (ptr[s]) cudaFree(ptr[s]);
        ptr[s] = nullptr;
        size[s] = 0;
    }
    for (void* q : retired) cudaFree(q);
    retired.clear();
}

cudaEvent_t KernelTimer::take() {
    if (!pool.empty()) {
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    HME_CUDA(cudaEventCreate(&e));
    return e;
}
void KernelTimer::begin(const char* name, cudaStream_t s) {
    Rec r{name, take(), take()};
    HME_CUDA(cudaEventRecord(r.a, s));
    recs.push_back(r);
}
void KernelTimer::end(cudaStream_t s) { HME_CUDA(cudaEventRecord(recs.back().b, s)); }
void KernelTimer::clear() {
    for (auto& r : recs) {
        pool.push_back(r.a);
        pool.push_back(r.b);
    }
    recs.clear();
}

void bind(hme_ctx* ctx) { HME_CUDA(cudaSetDevice(ctx->device)); }

void check_device_error(hme_ctx* ctx) {
    // one stream-ordered read of the error word into pinned memory, one synchronisation
    HME_CUDA(cudaMemcpyAsync(ctx->h_err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    HME_CUDA(cudaStreamSynchronize(ctx->stream));
    const int code = *static_cast<volatile int*>(ctx->h_err);
    if (code != 0) {
        const int zero = 0;
        HME_CUDA(cudaMemcpy(ctx->d_err, &zero, sizeof(int), cudaMemcpyHostToDevice));
        if (code == DERR_LAUNCH_SHAPE)
            throw Error(HME_ECUDA, "a kernel was launched with a shape it does not support and did nothing");
        throw Error(HME_ETIMEOUT, "a bounded device-side wait ran out (device code " + std::to_string(code) +
                                      "); the kernel returned early and its output is incomplete");
    }
}



const char* last_error_cstr() { return g_last_error.c_str(); }

}  // namespace hme

using namespace hme;

extern "C" {

const char* hme_last_error(void) { return last_error_cstr(); }

const char* hme_version(void) { return "hme 0.1 (sm_100a)"; }

int hme_ctx_create(int device, hme_ctx** out) {
    return guard([&] {
        HME_REQUIRE(out != nullptr, "hme_ctx_create: out is null");
        *out = nullptr;
        int count = 0;
        HME_CUDA(cudaGetDeviceCount(&count));
        HME_REQUIRE(device >= 0 && device < count, "hme_ctx_create: no such device");
        cudaDeviceProp prop{};
        HME_CUDA(cudaGetDeviceProperties(&prop, device));
        if (prop.major != 10 || prop.minor != 0)
            throw Error(HME_EUNSUPPORTED, std::string("hme needs an sm_100 (B200) device; found ") + prop.name +
                                              " sm_" + std::to_string(prop.major) + std::to_string(prop.minor));
        auto* c = new hme_ctx();
        c->device = device;
        c->num_sms = prop.multiProcessorCount;
        try {
            HME_CUDA(cudaSetDevice(device));
            HME_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
            c->stream = c->own_stream;
            HME_CUDA(cudaMalloc(&c->d_err, sizeof(int)));
            HME_CUDA(cudaMemset(c->d_err, 0, sizeof(int)));
            HME_CUDA(cudaMallocHost(&c->h_err, sizeof(int)));
            *c->h_err = 0;
        } catch (...) {
            if (c->own_stream) cudaStreamDestroy(c->own_stream);
            if (c->d_err) cudaFree(c->d_err);
            if (c->h_err) cudaFreeHost(c->h_err);
            delete c;
            throw;
        }
        *out = c;
    });
}

int hme_ctx_destroy(hme_ctx* ctx) {
    return guard([&] {
        if (!ctx) return;
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        ctx->ws.release();
        sched_release(ctx);
        ctx->timer.clear();
        for (cudaEvent_t e : ctx->timer.pool) cudaEventDestroy(e);
        if (ctx->copy_in) cudaStreamSynchronize(ctx->copy_in);
        if (ctx->copy_out) cudaStreamSynchronize(ctx->copy_out);
        for (cudaEvent_t e : ctx->pipe_ev) cudaEventDestroy(e);
        if (ctx->copy_in) cudaStreamDestroy(ctx->copy_in);
        if (ctx->copy_out) cudaStreamDestroy(ctx->copy_out);
        if (ctx->aux_stream) {
            cudaStreamSynchronize(ctx->aux_stream);
            cudaStreamDestroy(ctx->aux_stream);
        }
        for (cudaEvent_t e : ctx->elim_ev) cudaEventDestroy(e);
        if (ctx->elim_pinned) cudaFreeHost(ctx->elim_pinned);
        if (ctx->d_err) cudaFree(ctx->d_err);
        if (ctx->h_err) cudaFreeHost(ctx->h_err);
        if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
        delete ctx;
    });
}

int hme_ctx_set_stream(hme_ctx* ctx, void* stream) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr, "null context");
        ctx->stream = static_cast<cudaStream_t>(stream);
    });
}

void* hme_ctx_own_stream(const hme_ctx* ctx) { return ctx ? static_cast<void*>(ctx->own_stream) : nullptr; }

int hme_ctx_set_workspace_retain(hme_ctx* ctx, int on) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr, "null context");
        ctx->ws.retain = on != 0;
    });
}

int hme_ctx_sync(hme_ctx* ctx) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr, "null context");
        bind(ctx);
        check_device_error(ctx);
    });
}

uint64_t hme_ctx_launches(const hme_ctx* ctx) { return ctx ? ctx->launches : 0; }

int hme_ctx_set_timing(hme_ctx* ctx, int on) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr, "null context");
        ctx->timer.on = on != 0;
    });
}

int hme_ctx_kernel_time(hme_ctx* ctx, const char* name, double* total_ms, uint64_t* count) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr && total_ms && count, "hme_ctx_kernel_time: null argument");
        bind(ctx);
        HME_CUDA(cudaStreamSynchronize(ctx->stream));
        double t = 0.0;
        uint64_t c = 0;
        for (auto& r : ctx->timer.recs) {
            if (name && std::strcmp(name, r.name) != 0) continue;
            float ms = 0.f;
            HME_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
            t += ms;
            ++c;
        }
        *total_ms = t;
        *count = c;
    });
}

int hme_ctx_timing_reset(hme_ctx* ctx) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr, "null context");
        bind(ctx);
        HME_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->timer.clear();
    });
}

int hme_gemm_u32_dev(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A, size_t lda,
                     const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc, int op) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr, "null context");
        HME_REQUIRE(p >= 2, "gemm: modulus must be >= 2");
        bind(ctx);
        gemm_u32_device(ctx, make_mod(p), m, n, k, A, lda, B, ldb, C, ldc, op);
    });
}

int hme_gemm_u32(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A, size_t lda,
                 const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc, int op) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr, "null context");
        HME_REQUIRE(p >= 2, "gemm: modulus must be >= 2");
        HME_REQUIRE(op == HME_SET || op == HME_ADD || op == HME_SUB, "gemm: bad op");
        if (m == 0 || n == 0) return;
        HME_REQUIRE(C != nullptr && ldc >= n, "gemm: bad C");
        HME_REQUIRE(k == 0 || (A && B && lda >= k && ldb >= n), "gemm: bad A/B");
        bind(ctx);
        const ModParams mp = make_mod(p);
        if (k > 0) {
            int v = ctx->fixed_variant;
            if (v < 0) v = sched_variant(ctx, mp, m, n, k);
            if (v == kVariantWide || v == kVariantNarrow) {
                gemm_u32_host(ctx, mp, m, n, k, A, lda, B, ldb, C, ldc, op, v);
                check_device_error(ctx);
                return;
            }
        }
        // compact device copies (row-major, ld = cols) in the context's staging slots
        uint32_t* dA = static_cast<uint32_t*>(ctx->ws.get(kSlotStageA, sizeof(uint32_t) * static_cast<size_t>(m) * k));
        uint32_t* dB = static_cast<uint32_t*>(ctx->ws.get(kSlotStageB, sizeof(uint32_t) * static_cast<size_t>(k) * n));
        uint32_t* dC = static_cast<uint32_t*>(ctx->ws.get(kSlotStageC, sizeof(uint32_t) * static_cast<size_t>(m) * n));
        if (k) {
            HME_CUDA(copy_rows_async(dA, sizeof(uint32_t) * k, A, sizeof(uint32_t) * lda, sizeof(uint32_t) * k, m,
                                       cudaMemcpyHostToDevice, ctx->stream));
            HME_CUDA(copy_rows_async(dB, sizeof(uint32_t) * n, B, sizeof(uint32_t) * ldb, sizeof(uint32_t) * n, k,
                                       cudaMemcpyHostToDevice, ctx->stream));
        }
        if (op != HME_SET)
            HME_CUDA(copy_rows_async(dC, sizeof(uint32_t) * n, C, sizeof(uint32_t) * ldc, sizeof(uint32_t) * n, m,
                                       cudaMemcpyHostToDevice, ctx->stream));
        gemm_u32_device(ctx, mp, m, n, k, dA, k, dB, n, dC, n, op);
        HME_CUDA(copy_rows_async(C, sizeof(uint32_t) * ldc, dC, sizeof(uint32_t) * n, sizeof(uint32_t) * n, m,
                                   cudaMemcpyDeviceToHost, ctx->stream));
        check_device_error(ctx);
    });
}

}  // extern "C"

extern "C" HME_API uint64_t hme_fnv1a_u32(const uint32_t* M, uint32_t rows, uint32_t cols, size_t ld) {
    uint64_t h = 0xcbf29ce484222325ull;
    auto feed = [&h](uint64_t v) {
        for (int i = 0; i < 8; ++i) {
            h ^= (v >> (8 * i)) & 0xffu;
            h *= 0x100000001b3ull;
        }
    };
    feed(rows);
    feed(cols);
    for (uint32_t i = 0; i < rows; ++i)
        for (uint32_t j = 0; j < cols; ++j) feed(M[static_cast<size_t>(i) * ld + j]);
    return h;
}

// The scheduler: exhaustive GEMM autotuner and a learned MLP planner.
//
// Schedules are the GEMM variants (hme_internal.h GemmVariant); every variant
// computes the same residues, so the scheduler can change only speed, never a
// value.  The reference has no autotuner and no learned scheduler: its
// placement and tiling are static rules (src/Engine/EngineCostModel.h:22-51,
// pick_tile src/Cuda/cuda_kernels.cu:354-359).
//
// The MLP maps 5 normalised features (log2 m, log2 n, log2 k, log2 p,
// density) through three hidden layers of 64 ReLU units to one normalised
// log-time per variant; the planner takes the arg-min.  Training runs on the
// GPU with this file's FP32 kernels (forward + backward of the mean squared
// error, shared-memory gradient accumulation, Adam); inference with the BF16
// kernel (bf16 weights and activations, fp32 accumulation).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <random>
#include <unordered_map>
#include <vector>

#include "hme_grouped.h"
#include "hme_internal.h"

namespace hme {
namespace {

constexpr int kIn = 5, kH = 64, kOut = kGemmVariants;
// one network shape serves both planners: its outputs are the GEMM variants or the rank schedules
static_assert(static_cast<int>(kRankVariants) == kOut, "the rank planner reuses the GEMM planner's network shape");
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kIn * kH;
constexpr int kOffW2 = kOffB1 + kH;
constexpr int kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH;
constexpr int kOffB3 = kOffW3 + kH * kH;
constexpr int kOffW4 = kOffB3 + kH;
constexpr int kOffB4 = kOffW4 + kH * kOut;
constexpr int kParams = kOffB4 + kOut;
constexpr int kWarps = 8;

// ---- FP32 forward + backward of the mean squared error ---------------------------------
// Samples idx[0 .. n) of X (rows of kIn) / Y (rows of kOut); one warp per
// sample; gradients accumulate in shared memory, then once per CTA into grad.
// loss receives sum((y - t)^2) / (total * kOut); grad the gradient of that mean.
__global__ void __launch_bounds__(kWarps * 32)
    mlp_fwd_bwd_kernel(const float* __restrict__ P, const float* __restrict__ X, const float* __restrict__ Y,
                       const int* __restrict__ idx, int n, int total, float* __restrict__ grad,
                       float* __restrict__ loss) {
    extern __shared__ float sm[];
    float* sP = sm;                  // parameters
    float* sG = sm + kParams;        // gradient accumulators
    float* act = sG + kParams;       // per warp: x[kIn] h1 h2 h3 [kH each] dh[kH] dh2[kH]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) {
        sP[i] = P[i];
        sG[i] = 0.f;
    }
    __syncthreads();
    float* x = act + warp * (kIn + 5 * kH);
    float* h1 = x + kIn;
    float* h2 = h1 + kH;
    float* h3 = h2 + kH;
    float* d3 = h3 + kH;
    float* d2 = d3 + kH;
    float lsum = 0.f;
    const float inv_count = 1.f / (static_cast<float>(total) * kOut);
    for (int s = blockIdx.x * kWarps + warp; s < n; s += gridDim.x * kWarps) {
        const int r = idx ? idx[s] : s;
        if (lane < kIn) x[lane] = X[static_cast<size_t>(r) * kIn + lane];
        __syncwarp();
        // forward
        for (int u = lane; u < kH; u += 32) {
            float a = sP[kOffB1 + u];
            for (int i = 0; i < kIn; ++i) a += x[i] * sP[kOffW1 + i * kH + u];
            h1[u] = fmaxf(a, 0.f);
        }
        __syncwarp();
        for (int u = lane; u < kH; u += 32) {
            float a = sP[kOffB2 + u];
            for (int v = 0; v < kH; ++v) a += h1[v] * sP[kOffW2 + v * kH + u];
            h2[u] = fmaxf(a, 0.f);
        }
        __syncwarp();
        for (int u = lane; u < kH; u += 32) {
            float a = sP[kOffB3 + u];
            for (int v = 0; v < kH; ++v) a += h2[v] * sP[kOffW3 + v * kH + u];
            h3[u] = fmaxf(a, 0.f);
        }
        __syncwarp();
        float dy = 0.f;
        if (lane < kOut) {
            float yv = sP[kOffB4 + lane];
            for (int v = 0; v < kH; ++v) yv += h3[v] * sP[kOffW4 + v * kOut + lane];
            const float e = yv - Y[static_cast<size_t>(r) * kOut + lane];
            lsum += e * e;
            dy = 2.f * e * inv_count;
        }
        // backward: output layer
        float dyo[kOut];
#pragma unroll
        for (int o = 0; o < kOut; ++o) dyo[o] = __shfl_sync(0xffffffffu, dy, o);
        for (int v = lane; v < kH; v += 32) {
            float g = 0.f;
#pragma unroll
            for (int o = 0; o < kOut; ++o) {
                atomicAdd(&sG[kOffW4 + v * kOut + o], h3[v] * dyo[o]);
                g += sP[kOffW4 + v * kOut + o] * dyo[o];
            }
            d3[v] = h3[v] > 0.f ? g : 0.f;
        }
        if (lane < kOut) atomicAdd(&sG[kOffB4 + lane], dy);
        __syncwarp();
        // layer 3
        for (int u = lane; u < kH; u += 32) {
            const float du = d3[u];
            atomicAdd(&sG[kOffB3 + u], du);
            if (du != 0.f)
                for (int v = 0; v < kH; ++v) atomicAdd(&sG[kOffW3 + v * kH + u], h2[v] * du);
        }
        for (int v = lane; v < kH; v += 32) {
            float g = 0.f;
            for (int u = 0; u < kH; ++u) g += sP[kOffW3 + v * kH + u] * d3[u];
            d2[v] = h2[v] > 0.f ? g : 0.f;
        }
        __syncwarp();
        // layer 2
        for (int u = lane; u < kH; u += 32) {
            const float du = d2[u];
            atomicAdd(&sG[kOffB2 + u], du);
            if (du != 0.f)
                for (int v = 0; v < kH; ++v) atomicAdd(&sG[kOffW2 + v * kH + u], h1[v] * du);
        }
        for (int v = lane; v < kH; v += 32) {
            float g = 0.f;
            for (int u = 0; u < kH; ++u) g += sP[kOffW2 + v * kH + u] * d2[u];
            d3[v] = h1[v] > 0.f ? g : 0.f;  // dh1, reusing d3
        }
        __syncwarp();
        // layer 1
        for (int u = lane; u < kH; u += 32) {
            const float du = d3[u];
            atomicAdd(&sG[kOffB1 + u], du);
            for (int i = 0; i < kIn; ++i) atomicAdd(&sG[kOffW1 + i * kH + u], x[i] * du);
        }
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if (lane == 0 && lsum != 0.f) atomicAdd(loss, lsum * inv_count);
    __syncthreads();
    for (int i = threadIdx.x; i < kParams; i += blockDim.x)
        if (sG[i] != 0.f) atomicAdd(&grad[i], sG[i]);
}

__global__ void adam_kernel(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M,
                            float* __restrict__ V, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    const float g = G[i];
    const float m = b1 * M[i] + (1.f - b1) * g;
    const float v = b2 * V[i] + (1.f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

__global__ void to_bf16_kernel(const float* __restrict__ P, __nv_bfloat16* __restrict__ Q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kParams) Q[i] = __float2bfloat16_rn(P[i]);
}

// ---- BF16 inference: one warp per sample ---------------------------------------------------
__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__global__ void __launch_bounds__(kWarps * 32)
    mlp_predict_bf16_kernel(const __nv_bfloat16* __restrict__ Q, const float* __restrict__ X, int n,
                            float* __restrict__ Y) {
    __shared__ float sQ[kParams];  // bf16 values held as floats (exactly representable)
    __shared__ float act[kWarps][kIn + 3 * kH];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) sQ[i] = __bfloat162float(Q[i]);
    __syncthreads();
    float* x = act[warp];
    float* h1 = x + kIn;
    float* h2 = h1 + kH;
    float* h3 = h2 + kH;
    for (int s = blockIdx.x * kWarps + warp; s < n; s += gridDim.x * kWarps) {
        if (lane < kIn) x[lane] = bf(X[static_cast<size_t>(s) * kIn + lane]);
        __syncwarp();
        for (int u = lane; u < kH; u += 32) {
            float a = sQ[kOffB1 + u];
            for (int i = 0; i < kIn; ++i) a += x[i] * sQ[kOffW1 + i * kH + u];
            h1[u] = bf(fmaxf(a, 0.f));
        }
        __syncwarp();
        for (int u = lane; u < kH; u += 32) {
            float a = sQ[kOffB2 + u];
            for (int v = 0; v < kH; ++v) a += h1[v] * sQ[kOffW2 + v * kH + u];
            h2[u] = bf(fmaxf(a, 0.f));
        }
        __syncwarp();
        for (int u = lane; u < kH; u += 32) {
            float a = sQ[kOffB3 + u];
            for (int v = 0; v < kH; ++v) a += h2[v] * sQ[kOffW3 + v * kH + u];
            h3[u] = bf(fmaxf(a, 0.f));
        }
        __syncwarp();
        if (lane < kOut) {
            float yv = sQ[kOffB4 + lane];
            for (int v = 0; v < kH; ++v) yv += h3[v] * sQ[kOffW4 + v * kOut + lane];
            Y[static_cast<size_t>(s) * kOut + lane] = yv;
        }
        __syncwarp();
    }
}

size_t fwd_bwd_smem() { return sizeof(float) * (2 * kParams + kWarps * (kIn + 5 * kH)); }

// ---- the learned planner's decisions, by shape class ----------------------------------------
struct ShapeKey {
    uint64_t v;
    bool operator==(const ShapeKey& o) const { return v == o.v; }
};
struct ShapeHash {
    size_t operator()(const ShapeKey& k) const { return std::hash<uint64_t>()(k.v); }
};
using PlanTable = std::unordered_map<ShapeKey, int, ShapeHash>;

ShapeKey shape_key(uint32_t m, uint32_t n, uint32_t k, uint32_t limbs) {
    // quarter-octave classes of each dimension, and the limb count
    auto q = [](uint32_t x) { return static_cast<uint64_t>(std::lround(4.0 * std::log2(std::max(1u, x)))); };
    return ShapeKey{(q(m) << 40) | (q(n) << 24) | (q(k) << 8) | limbs};
}

}  // namespace

int sched_planned_variant(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k) {
    if (!ctx->sched_table) return -1;
    const PlanTable& t = *static_cast<PlanTable*>(ctx->sched_table);
    auto it = t.find(shape_key(m, n, k, mp.limbs));
    return it == t.end() ? -1 : it->second;
}

int sched_planned_rank_variant(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k) {
    if (!ctx->sched_rank_table) return -1;
    const PlanTable& t = *static_cast<PlanTable*>(ctx->sched_rank_table);
    auto it = t.find(shape_key(m, n, k, mp.limbs));
    return it == t.end() ? -1 : it->second;
}

int sched_variant(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k) {
    if (ctx->sched_policy == 1 && ctx->sched_table) {
        const PlanTable& t = *static_cast<PlanTable*>(ctx->sched_table);
        auto it = t.find(shape_key(m, n, k, mp.limbs));
        if (it != t.end()) return it->second;
    }
    return gemm_default_variant(ctx, mp, m, n);
}

void sched_release(hme_ctx* ctx) {
    delete static_cast<PlanTable*>(ctx->sched_table);
    ctx->sched_table = nullptr;
    delete static_cast<PlanTable*>(ctx->sched_rank_table);
    ctx->sched_rank_table = nullptr;
}

}  // namespace hme

struct hme_mlp {
    hme_ctx* ctx = nullptr;
    float* P = nullptr;  // device parameters, fp32
    float* G = nullptr;  // gradient
    float* M = nullptr;  // Adam moments
    float* V = nullptr;
    __nv_bfloat16* Q = nullptr;  // bf16 copy for inference
    float* loss = nullptr;
    uint64_t adam_t = 0;
};

using namespace hme;

namespace {

void init_params(std::vector<float>& w, uint64_t seed) {
    // He-uniform weights, zero biases, from a fixed-seed generator
    std::mt19937_64 g(seed);
    auto fill = [&](int off, int fan_in, int count) {
        const float lim = std::sqrt(6.0f / fan_in);
        std::uniform_real_distribution<float> U(-lim, lim);
        for (int i = 0; i < count; ++i) w[off + i] = U(g);
    };
    w.assign(kParams, 0.f);
    fill(kOffW1, kIn, kIn * kH);
    fill(kOffW2, kH, kH * kH);
    fill(kOffW3, kH, kH * kH);
    fill(kOffW4, kH, kH * kOut);
}

struct DevBuf {
    void* p = nullptr;
    explicit DevBuf(size_t b) { HME_CUDA(cudaMalloc(&p, b ? b : 16)); }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    template <class T>
    T* as() {
        return static_cast<T*>(p);
    }
};

void fwd_bwd(hme_mlp* mlp, const float* dX, const float* dY, const int* didx, int n, int total) {
    static OncePerDevice attr;
    attr.run([](int) {
        HME_CUDA(cudaFuncSetAttribute(mlp_fwd_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(fwd_bwd_smem())));
    });
    hme_ctx* ctx = mlp->ctx;
    HME_CUDA(cudaMemsetAsync(mlp->G, 0, sizeof(float) * kParams, ctx->stream));
    HME_CUDA(cudaMemsetAsync(mlp->loss, 0, sizeof(float), ctx->stream));
    const int grid = std::max(1, std::min(ctx->num_sms, (n + kWarps - 1) / kWarps));
    HME_TIMED(ctx, "mlp_fwd_bwd", mlp_fwd_bwd_kernel<<<grid, kWarps * 32, fwd_bwd_smem(), ctx->stream>>>(
                                      mlp->P, dX, dY, didx, n, total, mlp->G, mlp->loss));
    HME_CUDA(cudaGetLastError());
}

}  // namespace

namespace {
// BF16 inference of a planner network over the shapes (p, m, n, k), the
// arg-min per shape into `variants`, and the decisions recorded by shape class
// in the context's table `*table` (created on first use).
void sched_plan_into(hme_ctx* ctx, hme_mlp* m, uint32_t n, const uint32_t* shapes, const float* density,
                     const float* norm, int* variants, void** table) {
    if (n == 0) return;
    // features (log2 m, log2 n, log2 k, log2 p, density), normalised by norm[0..4] (mean), norm[5..9] (std)
    std::vector<float> X(static_cast<size_t>(n) * kIn), Y(static_cast<size_t>(n) * kOut);
    for (uint32_t t = 0; t < n; ++t) {
        const uint32_t* s = shapes + 4 * static_cast<size_t>(t);
        const float f[kIn] = {std::log2(static_cast<float>(std::max(1u, s[1]))),
                              std::log2(static_cast<float>(std::max(1u, s[2]))),
                              std::log2(static_cast<float>(std::max(1u, s[3]))),
                              std::log2(static_cast<float>(std::max(2u, s[0]))), density ? density[t] : 1.0f};
        for (int i = 0; i < kIn; ++i) X[t * kIn + i] = (f[i] - norm[i]) / norm[kIn + i];
    }
    const int rc = hme_mlp_predict_bf16(m, n, X.data(), Y.data());
    if (rc != HME_OK) throw Error(rc, hme_last_error());
    if (!*table) *table = new PlanTable();
    PlanTable& tab = *static_cast<PlanTable*>(*table);
    for (uint32_t t = 0; t < n; ++t) {
        int best = 0;
        for (int v = 1; v < kOut; ++v)
            if (Y[t * kOut + v] < Y[t * kOut + best]) best = v;
        variants[t] = best;
        const uint32_t* s = shapes + 4 * static_cast<size_t>(t);
        const uint32_t limbs = s[0] <= 256u ? 1u : s[0] <= 65536u ? 2u : s[0] <= (1u << 24) ? 3u : 4u;  // as make_mod
        tab[shape_key(s[1], s[2], s[3], limbs)] = best;
    }
}
}  // namespace

extern "C" {

int hme_gemm_variant_count(void) { return kGemmVariants; }

int hme_gemm_u32_dev_variant(hme_ctx* ctx, int variant, uint32_t p, uint32_t m, uint32_t n, uint32_t k,
                             const uint32_t* A, size_t lda, const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc,
                             int op) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr, "null context");
        HME_REQUIRE(p >= 2, "gemm: modulus must be >= 2");
        bind(ctx);
        gemm_u32_variant(ctx, make_mod(p), m, n, k, A, lda, B, ldb, C, ldc, op, variant);
    });
}

int hme_ctx_set_gemm_variant(hme_ctx* ctx, int variant) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr, "null context");
        HME_REQUIRE(variant >= -1 && variant < kGemmVariants, "unknown variant");
        ctx->fixed_variant = variant;
    });
}

int hme_ctx_set_sched_policy(hme_ctx* ctx, int policy) {
    return guard([&] {
        HME_REQUIRE(ctx != nullptr, "null context");
        HME_REQUIRE(policy == 0 || policy == 1, "policy: 0 heuristic, 1 learned plan");
        ctx->sched_policy = policy;
    });
}

int hme_sched_plan_set(hme_ctx* ctx, int table, uint32_t n, const uint32_t* shapes, const int* variants) {
    return guard([&] {
        HME_REQUIRE(ctx && (n == 0 || (shapes && variants)), "null argument");
        HME_REQUIRE(table == 0 || table == 1, "plan table: 0 the GEMM plan, 1 the rank plan");
        const int nv = table == 0 ? static_cast<int>(kGemmVariants) : static_cast<int>(kRankVariants);
        for (uint32_t t = 0; t < n; ++t)  // every decision checked before any is recorded
            HME_REQUIRE(variants[t] >= 0 && variants[t] < nv, "plan: unknown schedule");
        void** tp = table == 0 ? &ctx->sched_table : &ctx->sched_rank_table;
        if (!*tp) *tp = new PlanTable();
        PlanTable& tab = *static_cast<PlanTable*>(*tp);
        for (uint32_t t = 0; t < n; ++t) {
            const uint32_t* s = shapes + 4 * static_cast<size_t>(t);
            const uint32_t limbs = s[0] <= 256u ? 1u : s[0] <= 65536u ? 2u : s[0] <= (1u << 24) ? 3u : 4u;  // as make_mod
            tab[shape_key(s[1], s[2], s[3], limbs)] = variants[t];
        }
    });
}

int hme_autotune_gemm(hme_ctx* ctx, uint32_t p, uint32_t m, uint32_t n, uint32_t k, int reps, float* ms) {
    return guard([&] {
        HME_REQUIRE(ctx && ms && p >= 2 && m && n && k, "autotune: bad arguments");
        bind(ctx);
        const ModParams mp = make_mod(p);
        const size_t ld_a = k, ld_b = n, ld_c = n;
        uint32_t* A = static_cast<uint32_t*>(ctx->ws.get(kSlotSched0, sizeof(uint32_t) * (static_cast<size_t>(m) * k + static_cast<size_t>(k) * n)));
        uint32_t* B = A + static_cast<size_t>(m) * k;
        uint32_t* C = static_cast<uint32_t*>(ctx->ws.get(kSlotSched1, sizeof(uint32_t) * static_cast<size_t>(m) * n));
        // operand values do not change any variant's timing; fill with a residue pattern
        HME_CUDA(cudaMemsetAsync(A, 0x11, sizeof(uint32_t) * (static_cast<size_t>(m) * k + static_cast<size_t>(k) * n),
                                 ctx->stream));
        HME_CUDA(cudaMemsetAsync(C, 0, sizeof(uint32_t) * static_cast<size_t>(m) * n, ctx->stream));
        cudaEvent_t e0, e1;
        HME_CUDA(cudaEventCreate(&e0));
        HME_CUDA(cudaEventCreate(&e1));
        for (int v = 0; v < kGemmVariants; ++v) {
            std::vector<float> t;
            gemm_u32_variant(ctx, mp, m, n, k, A, ld_a, B, ld_b, C, ld_c, HME_SET, v);  // warm
            for (int r = 0; r < std::max(1, reps); ++r) {
                HME_CUDA(cudaEventRecord(e0, ctx->stream));
                gemm_u32_variant(ctx, mp, m, n, k, A, ld_a, B, ld_b, C, ld_c, HME_SET, v);
                HME_CUDA(cudaEventRecord(e1, ctx->stream));
                HME_CUDA(cudaEventSynchronize(e1));
                float x = 0.f;
                HME_CUDA(cudaEventElapsedTime(&x, e0, e1));
                t.push_back(x);
            }
            std::sort(t.begin(), t.end());
            ms[v] = t[t.size() / 2];
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        check_device_error(ctx);
    });
}

int hme_mlp_param_count(void) { return kParams; }

int hme_mlp_create(hme_ctx* ctx, uint64_t seed, hme_mlp** out) {
    return guard([&] {
        HME_REQUIRE(ctx && out, "null argument");
        bind(ctx);
        auto* m = new hme_mlp();
        m->ctx = ctx;
        try {
            HME_CUDA(cudaMalloc(&m->P, sizeof(float) * kParams * 4 + 64));
            m->G = m->P + kParams;
            m->M = m->G + kParams;
            m->V = m->M + kParams;
            m->loss = m->V + kParams;
            HME_CUDA(cudaMalloc(&m->Q, sizeof(__nv_bfloat16) * kParams));
            std::vector<float> w;
            init_params(w, seed);
            HME_CUDA(cudaMemcpy(m->P, w.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice));
            HME_CUDA(cudaMemset(m->M, 0, sizeof(float) * kParams * 2));
        } catch (...) {
            if (m->P) cudaFree(m->P);
            if (m->Q) cudaFree(m->Q);
            delete m;
            throw;
        }
        *out = m;
    });
}

int hme_mlp_destroy(hme_mlp* m) {
    return guard([&] {
        if (!m) return;
        cudaFree(m->P);
        cudaFree(m->Q);
        delete m;
    });
}

int hme_mlp_get_params(hme_mlp* m, float* w) {
    return guard([&] {
        HME_REQUIRE(m && w, "null argument");
        bind(m->ctx);
        HME_CUDA(cudaMemcpy(w, m->P, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
    });
}

int hme_mlp_set_params(hme_mlp* m, const float* w) {
    return guard([&] {
        HME_REQUIRE(m && w, "null argument");
        bind(m->ctx);
        HME_CUDA(cudaMemcpy(m->P, w, sizeof(float) * kParams, cudaMemcpyHostToDevice));
        HME_CUDA(cudaMemset(m->M, 0, sizeof(float) * kParams * 2));
        m->adam_t = 0;
    });
}

int hme_mlp_loss_grad(hme_mlp* m, uint32_t n, const float* X, const float* Y, float* loss, float* grad) {
    return guard([&] {
        HME_REQUIRE(m && X && Y && loss && n > 0, "null argument");
        bind(m->ctx);
        DevBuf dX(sizeof(float) * n * kIn), dY(sizeof(float) * n * kOut);
        HME_CUDA(cudaMemcpyAsync(dX.p, X, sizeof(float) * n * kIn, cudaMemcpyHostToDevice, m->ctx->stream));
        HME_CUDA(cudaMemcpyAsync(dY.p, Y, sizeof(float) * n * kOut, cudaMemcpyHostToDevice, m->ctx->stream));
        fwd_bwd(m, dX.as<float>(), dY.as<float>(), nullptr, static_cast<int>(n), static_cast<int>(n));
        HME_CUDA(cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->ctx->stream));
        if (grad)
            HME_CUDA(cudaMemcpyAsync(grad, m->G, sizeof(float) * kParams, cudaMemcpyDeviceToHost, m->ctx->stream));
        check_device_error(m->ctx);
    });
}

int hme_mlp_train(hme_mlp* m, uint32_t n, const float* X, const float* Y, uint32_t epochs, uint32_t batch, float lr,
                  uint64_t seed, float* final_loss) {
    return guard([&] {
        HME_REQUIRE(m && X && Y && n > 0 && batch > 0, "bad arguments");
        bind(m->ctx);
        hme_ctx* ctx = m->ctx;
        DevBuf dX(sizeof(float) * n * kIn), dY(sizeof(float) * n * kOut), dI(sizeof(int) * n);
        HME_CUDA(cudaMemcpyAsync(dX.p, X, sizeof(float) * n * kIn, cudaMemcpyHostToDevice, ctx->stream));
        HME_CUDA(cudaMemcpyAsync(dY.p, Y, sizeof(float) * n * kOut, cudaMemcpyHostToDevice, ctx->stream));
        std::vector<int> idx(n);
        for (uint32_t i = 0; i < n; ++i) idx[i] = static_cast<int>(i);
        std::mt19937_64 g(seed);
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        for (uint32_t e = 0; e < epochs; ++e) {
            std::shuffle(idx.begin(), idx.end(), g);
            HME_CUDA(cudaMemcpyAsync(dI.p, idx.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->stream));
            for (uint32_t b0 = 0; b0 < n; b0 += batch) {
                const int nb = static_cast<int>(std::min(batch, n - b0));
                fwd_bwd(m, dX.as<float>(), dY.as<float>(), dI.as<int>() + b0, nb, nb);
                ++m->adam_t;
                const float c1 = 1.f - std::pow(b1, static_cast<float>(m->adam_t));
                const float c2 = 1.f - std::pow(b2, static_cast<float>(m->adam_t));
                HME_TIMED(ctx, "mlp_adam", adam_kernel<<<(kParams + 255) / 256, 256, 0, ctx->stream>>>(
                                               m->P, m->G, m->M, m->V, lr, b1, b2, eps, c1, c2));
            }
            // the host index vector is reshuffled next epoch: wait for its upload to be consumed
            HME_CUDA(cudaStreamSynchronize(ctx->stream));
        }
        // loss over the whole training set
        fwd_bwd(m, dX.as<float>(), dY.as<float>(), nullptr, static_cast<int>(n), static_cast<int>(n));
        float l = 0.f;
        HME_CUDA(cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        check_device_error(ctx);
        if (final_loss) *final_loss = l;
    });
}

int hme_mlp_predict_bf16(hme_mlp* m, uint32_t n, const float* X, float* Y) {
    return guard([&] {
        HME_REQUIRE(m && X && Y, "null argument");
        bind(m->ctx);
        if (n == 0) return;
        hme_ctx* ctx = m->ctx;
        // features and scores in the context's scheduler slots: no allocation (and no device-wide
        // synchronisation of a free) per call
        float* dX = static_cast<float*>(ctx->ws.get(kSlotSched0, sizeof(float) * n * kIn));
        float* dY = static_cast<float*>(ctx->ws.get(kSlotSched1, sizeof(float) * n * kOut));
        HME_CUDA(cudaMemcpyAsync(dX, X, sizeof(float) * n * kIn, cudaMemcpyHostToDevice, ctx->stream));
        HME_TIMED(ctx, "mlp_to_bf16", to_bf16_kernel<<<(kParams + 255) / 256, 256, 0, ctx->stream>>>(m->P, m->Q));
        const int grid = std::max(1, std::min(ctx->num_sms * 4, static_cast<int>((n + kWarps - 1) / kWarps)));
        HME_TIMED(ctx, "mlp_predict_bf16",
                  mlp_predict_bf16_kernel<<<grid, kWarps * 32, 0, ctx->stream>>>(m->Q, dX, n, dY));
        HME_CUDA(cudaGetLastError());
        HME_CUDA(cudaMemcpyAsync(Y, dY, sizeof(float) * n * kOut, cudaMemcpyDeviceToHost, ctx->stream));
        check_device_error(ctx);
    });
}


int hme_sched_plan(hme_ctx* ctx, hme_mlp* m, uint32_t n, const uint32_t* shapes, const float* density,
                   const float* norm, int* variants) {
    return guard([&] {
        HME_REQUIRE(ctx && m && shapes && norm && variants, "null argument");
        bind(ctx);
        sched_plan_into(ctx, m, n, shapes, density, norm, variants, &ctx->sched_table);
    });
}

int hme_sched_plan_rank(hme_ctx* ctx, hme_mlp* m, uint32_t n, const uint32_t* shapes, const float* density,
                        const float* norm, int* variants) {
    return guard([&] {
        HME_REQUIRE(ctx && m && shapes && norm && variants, "null argument");
        bind(ctx);
        sched_plan_into(ctx, m, n, shapes, density, norm, variants, &ctx->sched_rank_table);
    });
}

}  // extern "C"

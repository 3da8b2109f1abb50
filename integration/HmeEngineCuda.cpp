// The reference engine's device layer (engine::cuda, drjanosch42/hacs 0.2.1: src/Cuda/CudaCtx.h,
// CudaKernels.h, DeviceBuf.h) implemented over libhme, with the reference's own C++ names and
// signatures, so that the tape's DeviceBackend (src/Engine/DeviceBackend.cpp), TapeElim and every
// other consumer link against it unchanged in place of the reference's libEngineCuda
// (CudaCtx.cpp + cuda_kernels.cu).
//
// What is where:
//   * CudaCtx: one device (ENGINE_CUDA_DEVICE, default 0), three streams, a caching arena over
//     cudaMalloc (exact-size free lists), a pinned staging pool of 8 MiB chunks up to 128 MiB
//     for the pageable uploads / downloads, transfer counters; GraphCapture over the runtime's
//     stream capture (thread-local mode).
//   * kernels: every operation runs in libhme on the caller's stream.  u32: the INT8-limb
//     tcgen05 GEMM (gemm / gemm_nt / schur_update; operands that are not row-contiguous are
//     first laid out row-major in scratch by hme's copy / transpose), gemv, axpy, scal, copy,
//     transpose, fill, axpy_identity, gather, canonicalise (both forms), trsm_unit.  u64: the
//     residue-number-system GEMM (hme_gemm_u64_dev) and the u64 level-1 operations; gemv is a
//     one-column GEMM.  GemmBatch: one GEMM per instance (capturable; hme's grouped launch for
//     uneven batches is the batched stream's API, which synchronises the host).
//   * imma_rref (the reference's device RREF for p <= 127): hme's device elimination, for every
//     field p < 2^32; pivot_rows (the row rank profile) is the column rank profile of A^T.
//
// Errors: a failed hme call throws CudaError (std::runtime_error) with hme's message, as the
// reference's layer does for launch errors; contract violations hme reports (bad shapes,
// overlapping windows, non-canonical alpha) are thrown the same way.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "CudaCtx.h"
#include "CudaKernels.h"
#include "DeviceBuf.h"
#include "hme.h"

namespace engine {
namespace cuda {

namespace {

[[noreturn]] void fail_hme(const char* what) { throw CudaError(std::string(what) + ": " + hme_last_error()); }
void chk(int rc, const char* what) {
    if (rc != HME_OK) fail_hme(what);
}
void cu(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

int env_device() {
    const char* e = std::getenv("ENGINE_CUDA_DEVICE");
    return (e && *e) ? std::atoi(e) : 0;
}

struct Avail {
    bool ok = false;
    std::string why;
};
const Avail& avail() {
    static const Avail a = [] {
        Avail r;
        const char* dis = std::getenv("ENGINE_CUDA_DISABLE");
        if (dis && dis[0] == '1') {
            r.why = "ENGINE_CUDA_DISABLE=1";
            return r;
        }
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            cudaGetLastError();
            r.why = "no CUDA device";
            return r;
        }
        const int d = env_device();
        cudaDeviceProp pr{};
        if (d < 0 || d >= n || cudaGetDeviceProperties(&pr, d) != cudaSuccess) {
            r.why = "ENGINE_CUDA_DEVICE out of range";
            return r;
        }
        if (pr.major != 10) {
            r.why = "libhme needs an sm_100 device";
            return r;
        }
        r.ok = true;
        return r;
    }();
    return a;
}

std::atomic<uint64_t> g_launches{0}, g_gemms{0}, g_batched{0};
cudaStream_t st(Stream s) { return static_cast<cudaStream_t>(s.h); }
thread_local int t_capturing = 0;
thread_local const char* t_tag = "";
std::atomic<bool> g_ctx_created{false};

// One hme context per host thread, on the engine's device, its stream set to the caller's for each
// call.  The calls of one thread share the context's workspace, so they are chained across streams:
// before a call on stream s, s waits for the thread's previous call (an event recorded after it on
// whichever stream it ran), and the call records that event again.  Events and waits are captured
// into a graph like any launch, and the chain restarts at every capture's begin and end (a wait
// never crosses a capture boundary).  Every workspace allocation stays alive
// (hme_ctx_set_workspace_retain), so the workspace a graph was captured with stays valid after a
// later, larger call grew it; the direct first run of a program grows the workspace to what its
// captured replays need, so no allocation happens inside a capture.
struct ThreadHme {
    hme_ctx* h = nullptr;
    cudaEvent_t done = nullptr;  // recorded after the thread's last call
    void* last = nullptr;        // the stream it was recorded on
    bool valid = false;
    ~ThreadHme() {
        if (done) cudaEventDestroy(done);
        if (h) hme_ctx_destroy(h);
    }
};
ThreadHme& thread_hme() {
    thread_local ThreadHme t;
    return t;
}
void chain_restart() { thread_hme().valid = false; }

// A call of the thread's hme context on stream s: ordered after the thread's previous call.
class HmeCall {
  public:
    explicit HmeCall(Stream s) : t_(thread_hme()), s_(s) {
        if (!t_.h) {
            chk(hme_ctx_create(env_device(), &t_.h), "hme_ctx_create");
            chk(hme_ctx_set_workspace_retain(t_.h, 1), "hme_ctx_set_workspace_retain");
            cu(cudaEventCreateWithFlags(&t_.done, cudaEventDisableTiming), "cudaEventCreate");
        }
        if (t_.valid && t_.last != s.h) cu(cudaStreamWaitEvent(st(s), t_.done, 0), "cudaStreamWaitEvent");
        chk(hme_ctx_set_stream(t_.h, s.h), "hme_ctx_set_stream");
        g_launches.fetch_add(1, std::memory_order_relaxed);
    }
    ~HmeCall() {
        if (cudaEventRecord(t_.done, st(s_)) == cudaSuccess) {
            t_.last = s_.h;
            t_.valid = true;
        } else {
            cudaGetLastError();
            t_.valid = false;
        }
        // between calls the context holds its own stream, never a caller's (which may be destroyed)
        hme_ctx_set_stream(t_.h, hme_ctx_own_stream(t_.h));
    }
    hme_ctx* ctx() const { return t_.h; }

  private:
    ThreadHme& t_;
    Stream s_;
};

}  // namespace

// ---- availability / policy ----------------------------------------------------------------
bool available() { return avail().ok; }
const char* unavailable_reason() { return avail().ok ? "" : avail().why.c_str(); }
Device requested_device() {
    static const Device d = [] {
        const char* e = std::getenv("ENGINE_DEVICE");
        if (e && std::strcmp(e, "gpu") == 0) return Device::Gpu;
        if (e && std::strcmp(e, "hybrid") == 0) return Device::Hybrid;
        return Device::Cpu;
    }();
    return d;
}
bool device_enabled() { return available() && requested_device() != Device::Cpu; }

DeviceInfo device_info() {
    if (!available()) throw CudaError(std::string("device_info: ") + unavailable_reason());
    DeviceInfo i;
    cudaDeviceProp pr{};
    cu(cudaGetDeviceProperties(&pr, env_device()), "cudaGetDeviceProperties");
    i.name = pr.name;
    i.index = env_device();
    i.cc_major = pr.major;
    i.cc_minor = pr.minor;
    i.sms = pr.multiProcessorCount;
    i.total_mem = pr.totalGlobalMem;
    size_t fr = 0, to = 0;
    cudaSetDevice(i.index);
    if (cudaMemGetInfo(&fr, &to) == cudaSuccess) i.free_mem = fr;
    cudaDriverGetVersion(&i.driver_version);
    cudaRuntimeGetVersion(&i.runtime_version);
    return i;
}
bool capturing_now() { return t_capturing > 0; }
void set_trace_tag(const char* tag) { t_tag = tag ? tag : ""; }
const char* trace_tag() { return t_tag; }

// ---- CudaCtx ----------------------------------------------------------------------------------
struct CudaCtx::Impl {
    int device = 0;
    std::vector<cudaStream_t> streams;
    std::mutex mu;
    std::unordered_map<size_t, std::vector<void*>> free_blocks;  // exact-size free lists
    std::unordered_map<void*, size_t> live;
    ArenaStats arena;
    struct Chunk {
        void* p = nullptr;
        cudaEvent_t ev = nullptr;
        bool used = false;
    };
    std::vector<Chunk> chunks;
    size_t chunk_bytes = size_t(8) << 20, cap_bytes = size_t(128) << 20;
    PinnedPoolStats pinned;
    TransferStats xfer;
    size_t next_chunk = 0;

    Chunk& take_chunk() {
        // round robin over the pool; a chunk is free again once its last copy's event completed
        if (chunks.size() * chunk_bytes < cap_bytes) {
            Chunk c;
            cu(cudaMallocHost(&c.p, chunk_bytes), "cudaMallocHost");
            cu(cudaEventCreateWithFlags(&c.ev, cudaEventDisableTiming), "cudaEventCreate");
            chunks.push_back(c);
            pinned.allocated_bytes += chunk_bytes;
            pinned.peak_bytes = std::max(pinned.peak_bytes, pinned.allocated_bytes);
            ++pinned.acquisitions;
            return chunks.back();
        }
        Chunk& c = chunks[next_chunk++ % chunks.size()];
        if (c.used && cudaEventQuery(c.ev) == cudaErrorNotReady) ++pinned.waits;
        if (c.used) cu(cudaEventSynchronize(c.ev), "cudaEventSynchronize");
        ++pinned.acquisitions;
        return c;
    }
};

CudaCtx::CudaCtx() : impl_(new Impl()) {
    impl_->device = env_device();
    cu(cudaSetDevice(impl_->device), "cudaSetDevice");
    for (int i = 0; i < 3; ++i) {
        cudaStream_t s;
        cu(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
        impl_->streams.push_back(s);
    }
    impl_->pinned.chunk_bytes = impl_->chunk_bytes;
    impl_->pinned.cap_bytes = impl_->cap_bytes;
    g_ctx_created.store(true);
}
CudaCtx::~CudaCtx() {}  // the singleton lives until the process exits

CudaCtx& CudaCtx::get() {
    if (!available()) throw CudaError(std::string("CudaCtx: ") + unavailable_reason());
    static CudaCtx* c = new CudaCtx();
    cudaSetDevice(c->impl_->device);
    return *c;
}
bool context_created() { return g_ctx_created.load(); }

int CudaCtx::num_streams() const { return static_cast<int>(impl_->streams.size()); }
Stream CudaCtx::stream(int i) const { return Stream{impl_->streams.at(static_cast<size_t>(i))}; }
Stream CudaCtx::create_stream() {
    cudaStream_t s;
    cu(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    return Stream{s};
}
void CudaCtx::destroy_stream(Stream s) {
    if (s.h) cudaStreamDestroy(st(s));
}
void CudaCtx::sync(Stream s) const { cu(cudaStreamSynchronize(st(s)), "cudaStreamSynchronize"); }
void CudaCtx::sync_all() const { cu(cudaDeviceSynchronize(), "cudaDeviceSynchronize"); }
Event CudaCtx::create_event() const {
    cudaEvent_t e;
    cu(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    return Event{e};
}
Event CudaCtx::create_timing_event() const {
    cudaEvent_t e;
    cu(cudaEventCreate(&e), "cudaEventCreate");
    return Event{e};
}
void CudaCtx::record(Event e, Stream s) const {
    cu(cudaEventRecord(static_cast<cudaEvent_t>(e.h), st(s)), "cudaEventRecord");
}
void CudaCtx::wait(Stream s, Event e) const {
    cu(cudaStreamWaitEvent(st(s), static_cast<cudaEvent_t>(e.h), 0), "cudaStreamWaitEvent");
}
void CudaCtx::sync(Event e) const { cu(cudaEventSynchronize(static_cast<cudaEvent_t>(e.h)), "cudaEventSynchronize"); }
void CudaCtx::destroy(Event e) const {
    if (e.h) cudaEventDestroy(static_cast<cudaEvent_t>(e.h));
}
float CudaCtx::elapsed_ms(Event a, Event b) const {
    float ms = 0.f;
    cu(cudaEventElapsedTime(&ms, static_cast<cudaEvent_t>(a.h), static_cast<cudaEvent_t>(b.h)), "cudaEventElapsedTime");
    return ms;
}

void* CudaCtx::dalloc(size_t bytes) {
    if (bytes == 0) bytes = 256;
    bytes = (bytes + 255) / 256 * 256;
    std::lock_guard<std::mutex> lk(impl_->mu);
    auto it = impl_->free_blocks.find(bytes);
    void* p = nullptr;
    if (it != impl_->free_blocks.end() && !it->second.empty()) {
        p = it->second.back();
        it->second.pop_back();
        ++impl_->arena.reuses;
    } else {
        if (capturing_now()) throw CudaError("CudaCtx::dalloc: a new device allocation inside a graph capture");
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            ++impl_->arena.oom_retries;
            for (auto& kv : impl_->free_blocks)
                for (void* q : kv.second) {
                    cudaFree(q);
                    impl_->arena.reserved_bytes -= kv.first;
                    ++impl_->arena.cuda_frees;
                }
            impl_->free_blocks.clear();
            cu(cudaMalloc(&p, bytes), "cudaMalloc");
        }
        impl_->arena.reserved_bytes += bytes;
        impl_->arena.peak_reserved_bytes = std::max(impl_->arena.peak_reserved_bytes, impl_->arena.reserved_bytes);
        ++impl_->arena.cuda_mallocs;
    }
    impl_->live[p] = bytes;
    impl_->arena.live_bytes += bytes;
    impl_->arena.peak_live_bytes = std::max(impl_->arena.peak_live_bytes, impl_->arena.live_bytes);
    return p;
}
void CudaCtx::dfree(void* p, size_t) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(impl_->mu);
    auto it = impl_->live.find(p);
    if (it == impl_->live.end()) return;
    impl_->arena.live_bytes -= it->second;
    impl_->free_blocks[it->second].push_back(p);
    impl_->live.erase(it);
}
ArenaStats CudaCtx::arena_stats() const {
    std::lock_guard<std::mutex> lk(impl_->mu);
    return impl_->arena;
}
size_t CudaCtx::arena_idle_slack() const { return size_t(1) << 30; }
ReleaseStats CudaCtx::release_cached(bool pinned) {
    ReleaseStats r;
    cu(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    std::lock_guard<std::mutex> lk(impl_->mu);
    for (auto& kv : impl_->free_blocks)
        for (void* q : kv.second) {
            cudaFree(q);
            r.arena_bytes_freed += kv.first;
            ++r.slabs_freed;
            impl_->arena.reserved_bytes -= kv.first;
            ++impl_->arena.cuda_frees;
        }
    impl_->free_blocks.clear();
    r.slabs_kept = impl_->live.size();
    if (pinned) {
        for (auto& c : impl_->chunks) {
            cudaEventDestroy(c.ev);
            cudaFreeHost(c.p);
            r.pinned_bytes_freed += impl_->chunk_bytes;
        }
        impl_->chunks.clear();
        impl_->pinned.allocated_bytes = 0;
    }
    return r;
}
ReleaseStats release_device_caches() {
    if (!context_created() || !available()) return ReleaseStats{};
    return CudaCtx::get().release_cached(true);
}

void CudaCtx::upload(const void* host, void* dev, size_t bytes, Stream s) {
    if (capturing_now()) throw CudaError("CudaCtx::upload: a staged copy inside a graph capture");
    std::lock_guard<std::mutex> lk(impl_->mu);
    const char* h = static_cast<const char*>(host);
    char* d = static_cast<char*>(dev);
    for (size_t off = 0; off < bytes; off += impl_->chunk_bytes) {
        const size_t n = std::min(impl_->chunk_bytes, bytes - off);
        Impl::Chunk& c = impl_->take_chunk();
        std::memcpy(c.p, h + off, n);
        cu(cudaMemcpyAsync(d + off, c.p, n, cudaMemcpyHostToDevice, st(s)), "cudaMemcpyAsync");
        cu(cudaEventRecord(c.ev, st(s)), "cudaEventRecord");
        c.used = true;
    }
    impl_->xfer.h2d_bytes += bytes;
    ++impl_->xfer.h2d_calls;
}
void CudaCtx::download(void* host, const void* dev, size_t bytes, Stream s) {
    if (capturing_now()) throw CudaError("CudaCtx::download: a staged copy inside a graph capture");
    std::lock_guard<std::mutex> lk(impl_->mu);
    char* h = static_cast<char*>(host);
    const char* d = static_cast<const char*>(dev);
    for (size_t off = 0; off < bytes; off += impl_->chunk_bytes) {
        const size_t n = std::min(impl_->chunk_bytes, bytes - off);
        Impl::Chunk& c = impl_->take_chunk();
        cu(cudaMemcpyAsync(c.p, d + off, n, cudaMemcpyDeviceToHost, st(s)), "cudaMemcpyAsync");
        cu(cudaEventRecord(c.ev, st(s)), "cudaEventRecord");
        cu(cudaEventSynchronize(c.ev), "cudaEventSynchronize");
        std::memcpy(h + off, c.p, n);
        c.used = true;
    }
    impl_->xfer.d2h_bytes += bytes;
    ++impl_->xfer.d2h_calls;
}
void CudaCtx::copy_d2d(void* dst, const void* src, size_t bytes, Stream s) {
    cu(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st(s)), "cudaMemcpyAsync");
    impl_->xfer.d2d_bytes += bytes;
}
void CudaCtx::memset_d(void* dst, int value, size_t bytes, Stream s) {
    cu(cudaMemsetAsync(dst, value, bytes, st(s)), "cudaMemsetAsync");
}
void CudaCtx::upload_pageable(const void* host, void* dev, size_t bytes) {
    cu(cudaMemcpy(dev, host, bytes, cudaMemcpyHostToDevice), "cudaMemcpy");
    ++impl_->xfer.pageable_copies;
}
void CudaCtx::download_pageable(void* host, const void* dev, size_t bytes) {
    cu(cudaMemcpy(host, dev, bytes, cudaMemcpyDeviceToHost), "cudaMemcpy");
    ++impl_->xfer.pageable_copies;
}
void* CudaCtx::pinned_alloc(size_t bytes) {
    void* p = nullptr;
    cu(cudaMallocHost(&p, bytes), "cudaMallocHost");
    return p;
}
void CudaCtx::pinned_free(void* p) {
    if (p) cudaFreeHost(p);
}
PinnedPoolStats CudaCtx::pinned_stats() const { return impl_->pinned; }
TransferStats CudaCtx::transfer_stats() const { return impl_->xfer; }
void CudaCtx::reset_transfer_stats() { impl_->xfer = TransferStats{}; }
size_t CudaCtx::pinned_cap_bytes() const { return impl_->cap_bytes; }
size_t CudaCtx::pinned_chunk_bytes() const { return impl_->chunk_bytes; }
int CudaCtx::copy_threads() const { return 0; }

// ---- GraphCapture -------------------------------------------------------------------------------
struct GraphCapture::Impl {
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool capturing = false;
    size_t nodes = 0;
};
GraphCapture::GraphCapture() : impl_(new Impl()) {}
GraphCapture::~GraphCapture() {
    if (impl_) {
        if (impl_->capturing) {  // abandoned mid-capture (an exception): end it, discard the graph
            cudaGraph_t g = nullptr;
            if (cudaStreamEndCapture(impl_->stream, &g) == cudaSuccess && g) cudaGraphDestroy(g);
            cudaGetLastError();
            --t_capturing;
            chain_restart();
        }
        if (impl_->exec) cudaGraphExecDestroy(impl_->exec);
        if (impl_->graph) cudaGraphDestroy(impl_->graph);
        delete impl_;
    }
}
void GraphCapture::begin(Stream s) {
    if (impl_->capturing) throw CudaError("GraphCapture::begin: already capturing");
    impl_->stream = st(s);
    chain_restart();
    cu(cudaStreamBeginCapture(impl_->stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    impl_->capturing = true;
    ++t_capturing;
}
void GraphCapture::end() {
    if (!impl_->capturing) throw CudaError("GraphCapture::end: not capturing");
    impl_->capturing = false;
    --t_capturing;
    chain_restart();
    cudaGraph_t g = nullptr;
    cu(cudaStreamEndCapture(impl_->stream, &g), "cudaStreamEndCapture");
    if (impl_->exec) cudaGraphExecDestroy(impl_->exec);
    if (impl_->graph) cudaGraphDestroy(impl_->graph);
    impl_->graph = g;
    cu(cudaGraphGetNodes(g, nullptr, &impl_->nodes), "cudaGraphGetNodes");
    cu(cudaGraphInstantiate(&impl_->exec, g, 0), "cudaGraphInstantiate");
}
void GraphCapture::launch(Stream s) const {
    if (!impl_->exec) throw CudaError("GraphCapture::launch: nothing captured");
    cu(cudaGraphLaunch(impl_->exec, st(s)), "cudaGraphLaunch");
}
bool GraphCapture::instantiated() const { return impl_->exec != nullptr; }
size_t GraphCapture::num_nodes() const { return impl_->nodes; }
Stream GraphCapture::captured_stream() const { return Stream{impl_->stream}; }
bool GraphCapture::capturing() const { return impl_->capturing; }

// ---- kernels ------------------------------------------------------------------------------------
namespace {

int op_of(GemmOp op) { return op == GemmOp::Set ? HME_SET : op == GemmOp::Add ? HME_ADD : HME_SUB; }

// Scratch of the calling thread for operands that are not row-contiguous (grow-only; never
// grown inside a capture).
struct Scratch {
    void* p[3] = {};
    size_t n[3] = {};
    ~Scratch() {
        for (void* q : p)
            if (q) cudaFree(q);
    }
    void* get(int i, size_t bytes) {
        if (n[i] < bytes) {
            if (capturing_now()) throw CudaError("engine::cuda (hme): scratch growth inside a graph capture");
            if (p[i]) cudaFree(p[i]);
            p[i] = nullptr;
            cu(cudaMalloc(&p[i], bytes), "cudaMalloc");
            n[i] = bytes;
        }
        return p[i];
    }
};
Scratch& scratch() {
    thread_local Scratch s;
    return s;
}

// A row-major (unit column stride) view of `v`: v itself, or a copy in scratch slot `slot`.
template <class Elt>
const Elt* row_major(hme_ctx* h, DeviceView<const Elt> v, int slot, size_t& ld) {
    if (v.cs == 1) {
        ld = std::max<size_t>(v.rs, v.cols);
        return v.base;
    }
    if (v.cols == 1) {  // a column: row-major with the row stride as leading dimension
        ld = std::max<size_t>(v.rs, 1);
        return v.base;
    }
    Elt* t = static_cast<Elt*>(scratch().get(slot, sizeof(Elt) * static_cast<size_t>(v.rows) * v.cols));
    ld = v.cols;
    if constexpr (sizeof(Elt) == 4)
        chk(hme_copy_u32_dev(h, v.rows, v.cols, reinterpret_cast<const uint32_t*>(v.base), v.rs, v.cs,
                             reinterpret_cast<uint32_t*>(t), v.cols, 1), "hme_copy_u32_dev");
    else
        chk(hme_copy_u64_dev(h, v.rows, v.cols, reinterpret_cast<const uint64_t*>(v.base), v.rs, v.cs,
                             reinterpret_cast<uint64_t*>(t), v.cols, 1), "hme_copy_u64_dev");
    return t;
}

template <class Elt>
void copy_any(hme_ctx* h, DeviceView<const Elt> s, DeviceView<Elt> d) {
    if constexpr (sizeof(Elt) == 4)
        chk(hme_copy_u32_dev(h, s.rows, s.cols, reinterpret_cast<const uint32_t*>(s.base), s.rs, s.cs,
                             reinterpret_cast<uint32_t*>(d.base), d.rs, d.cs), "hme_copy_u32_dev");
    else
        chk(hme_copy_u64_dev(h, s.rows, s.cols, reinterpret_cast<const uint64_t*>(s.base), s.rs, s.cs,
                             reinterpret_cast<uint64_t*>(d.base), d.rs, d.cs), "hme_copy_u64_dev");
}

template <class Elt>
void gemm_rowmajor(hme_ctx* h, const ModCtx<Elt>& ctx, uint32_t m, uint32_t n, uint32_t k, const Elt* A, size_t lda,
                   const Elt* B, size_t ldb, Elt* C, size_t ldc, int op) {
    if constexpr (sizeof(Elt) == 4)
        chk(hme_gemm_u32_dev(h, ctx.p, m, n, k, A, lda, B, ldb, C, ldc, op), "hme_gemm_u32_dev");
    else
        chk(hme_gemm_u64_dev(h, ctx.p, m, n, k, A, lda, B, ldb, C, ldc, op), "hme_gemm_u64_dev");
}

template <class Elt>
void gemm_views(const ModCtx<Elt>& ctx, DeviceView<const Elt> A, DeviceView<const Elt> B, DeviceView<Elt> C,
                GemmOp op, Stream s) {
    if (A.rows != C.rows || B.cols != C.cols || A.cols != B.rows) throw std::logic_error("gemm: shape mismatch");
    if (C.empty()) return;
    if (windows_overlap(A, DeviceView<const Elt>(C)) || windows_overlap(B, DeviceView<const Elt>(C)))
        throw std::logic_error("gemm: C overlaps an operand");
    HmeCall hc(s);
    hme_ctx* h = hc.ctx();
    g_gemms.fetch_add(1, std::memory_order_relaxed);
    const uint32_t m = C.rows, n = C.cols, k = A.cols;
    // u32 with B stored column-contiguous: hme's C op= A B^T on B as given
    if constexpr (sizeof(Elt) == 4) {
        if (C.cs == 1 && k > 0 && B.rs == 1 && B.cs != 1 && n > 1) {
            size_t lda;
            const Elt* a = row_major(h, A, 0, lda);
            chk(hme_gemm_nt_u32_dev(h, ctx.p, m, n, k, a, lda, B.base, B.cs, C.base, C.rs, op_of(op)),
                "hme_gemm_nt_u32_dev");
            return;
        }
    }
    size_t lda = 0, ldb = 0;
    const Elt* a = k ? row_major(h, A, 0, lda) : nullptr;
    const Elt* b = k ? row_major(h, B, 1, ldb) : nullptr;
    if (!k) lda = ldb = 1;
    lda = std::max<size_t>(lda, k);
    ldb = std::max<size_t>(ldb, n);
    if (C.cs == 1 || C.cols == 1) {
        gemm_rowmajor<Elt>(h, ctx, m, n, k, a, lda, b, ldb, C.base, std::max<size_t>(C.rs, n), op_of(op));
        return;
    }
    // C not row-contiguous: through a row-major copy
    Elt* t = static_cast<Elt*>(scratch().get(2, sizeof(Elt) * static_cast<size_t>(m) * n));
    DeviceView<Elt> tv(t, n, 1, m, n);
    if (op != GemmOp::Set) copy_any<Elt>(h, DeviceView<const Elt>(C), tv);
    gemm_rowmajor<Elt>(h, ctx, m, n, k, a, lda, b, ldb, t, n, op_of(op));
    copy_any<Elt>(h, DeviceView<const Elt>(tv), C);
}

}  // namespace

size_t gemm_workspace_bytes(uint32_t, uint32_t, uint32_t, size_t) { return 0; }
uint32_t suggest_splits(uint32_t, uint32_t, uint32_t) { return 1; }
bool imma_supported() { return available(); }
bool imma_policy() { return true; }

template <class Elt>
void gemm(const ModCtx<Elt>& ctx, DeviceView<const Elt> A, DeviceView<const Elt> B, DeviceView<Elt> C, GemmOp op,
          Stream s, const GemmOpts&) {
    gemm_views<Elt>(ctx, A, B, C, op, s);
}
template <class Elt>
void gemm_nt(const ModCtx<Elt>& ctx, DeviceView<const Elt> A, DeviceView<const Elt> B, DeviceView<Elt> C, GemmOp op,
             Stream s, const GemmOpts&) {
    gemm_views<Elt>(ctx, A, B.transposed_view(), C, op, s);
}
template <class Elt>
void schur_update(const ModCtx<Elt>& ctx, DeviceView<const Elt> L, DeviceView<const Elt> U, DeviceView<Elt> C,
                  Stream s, const GemmOpts&) {
    gemm_views<Elt>(ctx, L, U, C, GemmOp::Sub, s);
}

template <class Elt>
void gemv(const ModCtx<Elt>& ctx, DeviceView<const Elt> A, DeviceView<const Elt> x, DeviceView<Elt> y, GemmOp op,
          Stream s) {
    if (x.cols != 1 || y.cols != 1 || A.cols != x.rows || A.rows != y.rows) throw std::logic_error("gemv: shape mismatch");
    if (y.rows == 0) return;
    if constexpr (sizeof(Elt) == 4) {
        HmeCall hc(s);
        chk(hme_gemv_u32_dev(hc.ctx(), ctx.p, A.rows, A.cols, A.base, A.rs, A.cs, x.base, x.rs, y.base, y.rs,
                             op_of(op)), "hme_gemv_u32_dev");
    } else {
        gemm_views<Elt>(ctx, A, x, y, op, s);  // a one-column GEMM
    }
}

template <class Elt>
void axpy(const ModCtx<Elt>& ctx, Elt alpha, DeviceView<const Elt> x, DeviceView<Elt> y, bool subtract, Stream s) {
    if (x.rows != y.rows || x.cols != y.cols) throw std::logic_error("axpy: shape mismatch");
    if constexpr (sizeof(Elt) == 4)
        chk(hme_axpy_u32_dev(HmeCall(s).ctx(), ctx.p, alpha, y.rows, y.cols, x.base, x.rs, x.cs, y.base, y.rs, y.cs,
                             subtract), "hme_axpy_u32_dev");
    else
        chk(hme_axpy_u64_dev(HmeCall(s).ctx(), ctx.p, alpha, y.rows, y.cols, x.base, x.rs, x.cs, y.base, y.rs, y.cs,
                             subtract), "hme_axpy_u64_dev");
}

template <class Elt>
void scal(const ModCtx<Elt>& ctx, Elt alpha, DeviceView<Elt> x, Stream s) {
    if constexpr (sizeof(Elt) == 4)
        chk(hme_scal_u32_dev(HmeCall(s).ctx(), ctx.p, alpha, x.rows, x.cols, x.base, x.rs, x.cs), "hme_scal_u32_dev");
    else
        chk(hme_scal_u64_dev(HmeCall(s).ctx(), ctx.p, alpha, x.rows, x.cols, x.base, x.rs, x.cs), "hme_scal_u64_dev");
}

template <class Elt>
void copy(DeviceView<const Elt> src, DeviceView<Elt> dst, Stream s) {
    if (src.rows != dst.rows || src.cols != dst.cols) throw std::logic_error("copy: shape mismatch");
    copy_any<Elt>(HmeCall(s).ctx(), src, dst);
}

template <class Elt>
void transpose(DeviceView<const Elt> src, DeviceView<Elt> dst, Stream s) {
    if (src.rows != dst.cols || src.cols != dst.rows) throw std::logic_error("transpose: shape mismatch");
    if constexpr (sizeof(Elt) == 4)
        chk(hme_transpose_u32_dev(HmeCall(s).ctx(), dst.rows, dst.cols, src.base, src.rs, src.cs, dst.base, dst.rs, dst.cs),
            "hme_transpose_u32_dev");
    else
        chk(hme_transpose_u64_dev(HmeCall(s).ctx(), dst.rows, dst.cols, src.base, src.rs, src.cs, dst.base, dst.rs, dst.cs),
            "hme_transpose_u64_dev");
}

template <class Elt>
void fill(DeviceView<Elt> x, Elt value, Stream s) {
    if constexpr (sizeof(Elt) == 4)
        chk(hme_fill_u32_dev(HmeCall(s).ctx(), x.rows, x.cols, x.base, x.rs, x.cs, value), "hme_fill_u32_dev");
    else
        chk(hme_fill_u64_dev(HmeCall(s).ctx(), x.rows, x.cols, x.base, x.rs, x.cs, value), "hme_fill_u64_dev");
}

template <class Elt>
void axpy_identity(const ModCtx<Elt>& ctx, Elt alpha, DeviceView<Elt> y, bool subtract, Stream s) {
    if constexpr (sizeof(Elt) == 4)
        chk(hme_axpy_identity_u32_dev(HmeCall(s).ctx(), ctx.p, alpha, y.rows, y.cols, y.base, y.rs, y.cs, subtract),
            "hme_axpy_identity_u32_dev");
    else
        chk(hme_axpy_identity_u64_dev(HmeCall(s).ctx(), ctx.p, alpha, y.rows, y.cols, y.base, y.rs, y.cs, subtract),
            "hme_axpy_identity_u64_dev");
}

template <class Elt>
void gather(const ModCtx<Elt>& ctx, Elt alpha, Elt beta, DeviceView<const Elt> a, uint32_t row_off,
            const uint32_t* cols, DeviceView<Elt> c, bool accumulate, Stream s, const uint32_t* rows) {
    const bool have_a = !a.empty();
    if constexpr (sizeof(Elt) == 4)
        chk(hme_gather_u32_dev(HmeCall(s).ctx(), ctx.p, alpha, beta, have_a ? a.base : nullptr, a.rows, a.cols, a.rs, a.cs,
                               row_off, cols, rows, c.rows, c.cols, c.base, c.rs, c.cs, accumulate),
            "hme_gather_u32_dev");
    else
        chk(hme_gather_u64_dev(HmeCall(s).ctx(), ctx.p, alpha, beta, have_a ? a.base : nullptr, a.rows, a.cols, a.rs, a.cs,
                               row_off, cols, rows, c.rows, c.cols, c.base, c.rs, c.cs, accumulate),
            "hme_gather_u64_dev");
}

template <class Elt>
void canonicalise(const ModCtx<Elt>& ctx, DeviceView<Elt> v, Stream s) {
    if constexpr (sizeof(Elt) == 4)
        chk(hme_canonicalise_u32_dev(HmeCall(s).ctx(), ctx.p, v.rows, v.cols, v.base, v.rs, v.cs), "hme_canonicalise_u32_dev");
    else
        chk(hme_canonicalise_u64_dev(HmeCall(s).ctx(), ctx.p, v.rows, v.cols, v.base, v.rs, v.cs), "hme_canonicalise_u64_dev");
}

void canonicalise(const ModCtx<uint32_t>& ctx, DeviceView<const uint64_t> acc, DeviceView<uint32_t> dst, Stream s) {
    chk(hme_canonicalise_acc64_u32_dev(HmeCall(s).ctx(), ctx.p, dst.rows, dst.cols, acc.base, acc.rs, acc.cs, dst.base,
                                       dst.rs, dst.cs), "hme_canonicalise_acc64_u32_dev");
}

template <class Elt>
void trsm_unit(const ModCtx<Elt>& ctx, DeviceView<const Elt> T, DeviceView<Elt> B, Stream s, const GemmOpts&) {
    if (T.rows != T.cols || T.rows != B.rows) throw std::logic_error("trsm_unit: shape mismatch");
    if (B.empty()) return;
    if constexpr (sizeof(Elt) == 4) {
        const bool lower = T.structure == Structure::LowerUnitri;
        if (!lower && T.structure != Structure::UpperUnitri)
            throw std::logic_error("trsm_unit: T must be LowerUnitri or UpperUnitri");
        HmeCall hc(s);
        hme_ctx* h = hc.ctx();
        size_t ldt;
        const Elt* t = row_major(h, T, 0, ldt);
        if (B.cs == 1) {
            chk(hme_trsm_unit_u32_dev(h, ctx.p, lower, T.rows, B.cols, t, ldt, B.base, B.rs), "hme_trsm_unit_u32_dev");
            return;
        }
        Elt* b = static_cast<Elt*>(scratch().get(2, sizeof(Elt) * static_cast<size_t>(B.rows) * B.cols));
        DeviceView<Elt> bv(b, B.cols, 1, B.rows, B.cols);
        copy_any<Elt>(h, DeviceView<const Elt>(B), bv);
        chk(hme_trsm_unit_u32_dev(h, ctx.p, lower, T.rows, B.cols, t, ldt, b, B.cols), "hme_trsm_unit_u32_dev");
        copy_any<Elt>(h, DeviceView<const Elt>(bv), B);
    } else {
        (void)ctx;
        (void)T;
        (void)s;
        throw CudaError("trsm_unit: the u64 unit-triangular solve is not on the device in this layer");
    }
}

// ---- GemmBatch --------------------------------------------------------------------------------
template <class Elt>
GemmBatch<Elt>::~GemmBatch() {
    if (d_entries_) cudaFree(d_entries_);
}
template <class Elt>
void GemmBatch<Elt>::set_shape(uint32_t m, uint32_t n, uint32_t k, size_t a_rs, size_t a_cs, size_t b_rs, size_t b_cs,
                               size_t c_rs, size_t c_cs) {
    m_ = m, n_ = n, k_ = k;
    a_rs_ = a_rs, a_cs_ = a_cs, b_rs_ = b_rs, b_cs_ = b_cs, c_rs_ = c_rs, c_cs_ = c_cs;
    shape_set_ = true;
}
template <class Elt>
void GemmBatch<Elt>::set_shape(DeviceView<const Elt> A, DeviceView<const Elt> B, DeviceView<Elt> C) {
    set_shape(A.rows, C.cols, A.cols, A.rs, A.cs, B.rs, B.cs, C.rs, C.cs);
}
template <class Elt>
void GemmBatch<Elt>::push(DeviceView<const Elt> A, DeviceView<const Elt> B, DeviceView<Elt> C) {
    if (!shape_set_) set_shape(A, B, C);
    if (A.rows != m_ || A.cols != k_ || B.cols != n_ || C.rows != m_ || C.cols != n_ || A.rs != a_rs_ ||
        A.cs != a_cs_ || B.rs != b_rs_ || B.cs != b_cs_ || C.rs != c_rs_ || C.cs != c_cs_)
        throw std::logic_error("GemmBatch::push: shape or strides differ from the batch's");
    entries_.push_back(GemmBatchEntry<Elt>{A.base, B.base, C.base});
}
template <class Elt>
void GemmBatch<Elt>::upload(Stream) {
    // the instances stay on the host: the grouped launch builds its device tables itself
    uploaded_ = entries_.size();
}
template <class Elt>
bool GemmBatch<Elt>::prepare_imma(const ModCtx<Elt>&) {
    return false;  // no separate int8 workspace: every product runs on the limb GEMM
}
template <class Elt>
size_t GemmBatch<Elt>::imma_bytes_needed() const {
    return 0;
}
template <class Elt>
void GemmBatch<Elt>::run(const ModCtx<Elt>& ctx, GemmOp op, Stream s, int, int, void*, size_t) const {
    if (entries_.empty() || m_ == 0 || n_ == 0) return;
    g_batched.fetch_add(entries_.size(), std::memory_order_relaxed);
    // One GEMM per instance, in both of DeviceBackend's modes (direct launches and graph capture), so
    // the captured run uses exactly the workspace the direct run grew.  (hme's grouped launch for
    // uneven batches, hme_batch_gemm_u32_dev, synchronises the host and is not capturable.)
    for (const GemmBatchEntry<Elt>& e : entries_)
        gemm_views<Elt>(ctx, DeviceView<const Elt>(e.A, a_rs_, a_cs_, m_, k_),
                        DeviceView<const Elt>(e.B, b_rs_, b_cs_, k_, n_), DeviceView<Elt>(e.C, c_rs_, c_cs_, m_, n_),
                        op, s);
}

template class GemmBatch<uint32_t>;
template class GemmBatch<uint64_t>;

// ---- the device RREF (the reference's p <= 127 route) ---------------------------------------------
namespace {
ImmaElimStats g_elim_stats;
std::mutex g_elim_mu;
}  // namespace

ImmaRrefResult imma_rref(const ModCtx<uint32_t>& ctx, uint32_t m, uint32_t n, const ImmaRowSource& src,
                         const ImmaRowSink& sink, uint32_t slab_rows, uint32_t) {
    if (!ctx.is_field()) throw std::logic_error("imma_rref: a field modulus is required");
    ImmaRrefResult res;
    if (m == 0 || n == 0) return res;
    std::vector<uint32_t> A(static_cast<size_t>(m) * n);
    const uint32_t slab = slab_rows ? slab_rows : std::max<uint32_t>(1, static_cast<uint32_t>((size_t(64) << 20) / (4ull * n)));
    for (uint32_t r0 = 0; r0 < m; r0 += slab) {
        const uint32_t nr = std::min(slab, m - r0);
        const DenseView<const uint32_t> v = src(r0, nr);
        for (uint32_t i = 0; i < nr; ++i)
            for (uint32_t j = 0; j < n; ++j) A[(static_cast<size_t>(r0) + i) * n + j] = v.at(i, j);
    }
    HmeCall hc(Stream{nullptr});
    hme_ctx* h = hc.ctx();
    // the row rank profile: the column rank profile of A^T
    std::vector<uint32_t> At(static_cast<size_t>(n) * m);
    for (uint32_t i = 0; i < m; ++i)
        for (uint32_t j = 0; j < n; ++j) At[static_cast<size_t>(j) * m + i] = A[static_cast<size_t>(i) * n + j];
    std::vector<uint32_t> piv(std::min(m, n)), rows(std::min(m, n));
    uint32_t rank = 0, rrank = 0;
    chk(hme_rank_profile_u32(h, ctx.p, n, m, At.data(), m, rows.data(), &rrank), "hme_rank_profile_u32");
    if (sink) {
        chk(hme_rref_u32(h, ctx.p, m, n, A.data(), n, piv.data(), &rank), "hme_rref_u32");
        if (rank > 0) {
            DenseView<uint32_t> out = sink(rank);
            for (uint32_t i = 0; i < rank; ++i)
                for (uint32_t j = 0; j < n; ++j) out.at(i, j) = A[static_cast<size_t>(i) * n + j];
        }
    } else {
        chk(hme_rank_profile_u32(h, ctx.p, m, n, A.data(), n, piv.data(), &rank), "hme_rank_profile_u32");
    }
    if (rank != rrank) throw CudaError("imma_rref: row and column rank differ");
    res.rank = rank;
    res.pivots.assign(piv.begin(), piv.begin() + rank);
    res.pivot_rows.assign(rows.begin(), rows.begin() + rank);
    std::lock_guard<std::mutex> lk(g_elim_mu);
    ++g_elim_stats.calls;
    g_elim_stats.h2d_bytes += 8ull * m * n;
    return res;
}
ImmaElimStats imma_elim_stats() {
    std::lock_guard<std::mutex> lk(g_elim_mu);
    return g_elim_stats;
}
void reset_imma_elim_stats() {
    std::lock_guard<std::mutex> lk(g_elim_mu);
    g_elim_stats = ImmaElimStats{};
}
size_t imma_rref_device_bytes(uint32_t m, uint32_t n, uint32_t) { return 8ull * m * n; }

LaunchStats launch_stats() {
    LaunchStats s;
    s.kernel_launches = g_launches.load(std::memory_order_relaxed);
    s.gemm_launches = g_gemms.load(std::memory_order_relaxed);
    s.batched_instances = g_batched.load(std::memory_order_relaxed);
    return s;
}
void reset_launch_stats() {
    g_launches = 0;
    g_gemms = 0;
    g_batched = 0;
}
const char* kernel_layer_version() { return "engine::cuda over libhme (B200, sm_100a: INT8-limb tcgen05 GEMM)"; }

// ---- explicit instantiations: the set the reference's layer provides ----
#define HME_INST(Elt)                                                                                                  \
    template void gemm<Elt>(const ModCtx<Elt>&, DeviceView<const Elt>, DeviceView<const Elt>, DeviceView<Elt>, GemmOp, \
                            Stream, const GemmOpts&);                                                                  \
    template void gemm_nt<Elt>(const ModCtx<Elt>&, DeviceView<const Elt>, DeviceView<const Elt>, DeviceView<Elt>,      \
                               GemmOp, Stream, const GemmOpts&);                                                       \
    template void schur_update<Elt>(const ModCtx<Elt>&, DeviceView<const Elt>, DeviceView<const Elt>, DeviceView<Elt>, \
                                    Stream, const GemmOpts&);                                                          \
    template void gemv<Elt>(const ModCtx<Elt>&, DeviceView<const Elt>, DeviceView<const Elt>, DeviceView<Elt>, GemmOp, \
                            Stream);                                                                                   \
    template void axpy<Elt>(const ModCtx<Elt>&, Elt, DeviceView<const Elt>, DeviceView<Elt>, bool, Stream);            \
    template void scal<Elt>(const ModCtx<Elt>&, Elt, DeviceView<Elt>, Stream);                                         \
    template void canonicalise<Elt>(const ModCtx<Elt>&, DeviceView<Elt>, Stream);                                      \
    template void copy<Elt>(DeviceView<const Elt>, DeviceView<Elt>, Stream);                                           \
    template void transpose<Elt>(DeviceView<const Elt>, DeviceView<Elt>, Stream);                                      \
    template void fill<Elt>(DeviceView<Elt>, Elt, Stream);                                                             \
    template void axpy_identity<Elt>(const ModCtx<Elt>&, Elt, DeviceView<Elt>, bool, Stream);                          \
    template void gather<Elt>(const ModCtx<Elt>&, Elt, Elt, DeviceView<const Elt>, uint32_t, const uint32_t*,          \
                              DeviceView<Elt>, bool, Stream, const uint32_t*);                                         \
    template void trsm_unit<Elt>(const ModCtx<Elt>&, DeviceView<const Elt>, DeviceView<Elt>, Stream, const GemmOpts&);
HME_INST(uint32_t)
HME_INST(uint64_t)
#undef HME_INST

}  // namespace cuda
}  // namespace engine

// The seams of the reference's matrix engine (drjanosch42/hacs 0.2.1) served by libhme.
//
// A maintainer adds this file to the reference's build (it includes the reference's own headers
// and links libhme.so) and calls hme_seams::install() once at start-up; the callers stay as they
// are:
//
//   * engine::ring2k::device::Ops (src/ModArithmetic/Binary/Ring2kDevice.h:64-83; the reference
//     installs its own table in src/hacs/Integral/Descent/DescentSmithGpu.cpp:160-178):
//     ring2k::echelon_blocked (Ring2k.h:539-695) -- so ring2k::smith / howell / kernel_module of
//     the u32 and u64 rungs, the integral descent (DescentAssembly.cpp:386-392) and the orbifold
//     census (CampaignOrbifold.cpp:451-462) -- runs its LU on the device through hme_r2k_*.
//   * engine::elim::DeviceRrefHook (src/ModArithmetic/DenseElim.h:121-123; the reference's hook
//     is TapeElim.cpp:208-250 and serves p <= 127): every u32 in-place RREF of DenseElim.cpp
//     (rref, rref_with_transform, inverse, solve_multi_rhs, complement_basis) and
//     column_rank_profile run on hme_rref_u32 / hme_rank_profile_u32 for every prime p < 2^32.
//
// Errors: the table's functions throw std::runtime_error on a failed call (the reference's
// CudaError derives from it), so echelon_blocked falls back to the host LU when the failure
// comes before its first host write, as with the reference's own table.  The RREF hook returns
// false (the host elimination runs, A untouched) when hme declines or fails.
//
// Levers (environment, read once): HME_R2K=0 turns the device LU off; HME_R2K_MIN (entries,
// default 65536) is the size floor of the device LU; HME_R2K_VRAM_MB caps a session's device
// bytes; HME_R2K_HOST_MB (default 4096) is the host budget of one phase's L store on the tiled
// route; HME_R2K_VERIFY=1 re-runs every device LU on the host and compares (the reference's
// ENGINE_VERIFY_DEVICE twin).  HME_RREF=0 turns the RREF hook off; HME_RREF_MIN (entries,
// default 65536) is its size floor.  HME_DEVICE (default 0) is the GPU both use.
#include "HmeSeams.h"

#include <atomic>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "Binary/Ring2kDevice.h"
#include "DenseElim.h"
#include "ModCtx.h"
#include "hme.h"

namespace hme_seams {
namespace {

namespace dev = engine::ring2k::device;

uint64_t env_u64(const char* name, uint64_t dflt) {
    const char* e = std::getenv(name);
    return (e && *e) ? static_cast<uint64_t>(std::strtoull(e, nullptr, 10)) : dflt;
}
bool env_off(const char* name) {
    const char* e = std::getenv(name);
    return e && std::strcmp(e, "0") == 0;
}

std::atomic<int> g_device{0};
std::atomic<uint32_t> g_max_cols{0};
std::atomic<uint64_t> g_store_bytes{0};
std::atomic<int> g_verify{-1};
std::atomic<uint64_t> g_r2k_min{0}, g_rref_min{0};
std::atomic<uint64_t> g_sessions{0}, g_rref_calls{0};

[[noreturn]] void fail(const char* what) {
    throw std::runtime_error(std::string(what) + ": " + hme_last_error());
}

// ---- the ring2k device LU table ----
uint32_t op_plan(uint32_t elem, uint32_t m, uint32_t n, uint32_t panel) {
    static const bool off = env_off("HME_R2K");
    if (off) return 0;
    static const uint64_t min_env = env_u64("HME_R2K_MIN", 65536);
    const uint64_t mn = g_r2k_min.load(std::memory_order_relaxed);
    if (static_cast<uint64_t>(m) * n < (mn ? mn : min_env)) return 0;
    static const uint64_t cap = env_u64("HME_R2K_VRAM_MB", 0) << 20;
    uint32_t cw = hme_r2k_plan(g_device.load(std::memory_order_relaxed), elem, m, n, panel, cap);
    const uint32_t mc = g_max_cols.load(std::memory_order_relaxed);
    if (cw > 0 && mc > 0 && mc < n && cw > mc) cw = mc - mc % panel < panel ? panel : mc - mc % panel;
    return cw;
}
void* op_open(uint32_t elem, uint32_t m, uint32_t cw, uint32_t panel) {
    hme_r2k* s = nullptr;
    if (hme_r2k_open(g_device.load(std::memory_order_relaxed), elem, m, cw, panel, &s) != HME_OK) fail("hme_r2k_open");
    g_sessions.fetch_add(1, std::memory_order_relaxed);
    return s;
}
void op_put(void* s, const void* host, size_t ldh, uint32_t r0, uint32_t rows, uint32_t c0, uint32_t cols) {
    if (hme_r2k_put(static_cast<hme_r2k*>(s), host, ldh, r0, rows, c0, cols) != HME_OK) fail("hme_r2k_put");
}
void op_get(void* s, void* host, size_t ldh, uint32_t r0, uint32_t rows, uint32_t c0, uint32_t cols) {
    if (hme_r2k_get(static_cast<hme_r2k*>(s), host, ldh, r0, rows, c0, cols) != HME_OK) fail("hme_r2k_get");
}
void op_step(void* s, const dev::StepArgs& a) {
    hme_r2k_step_args b{};
    b.m = a.m;
    b.r = a.r;
    b.np = a.np;
    b.pc0 = a.pc0;
    b.pc1 = a.pc1;
    b.panel = a.panel;
    b.ldp = a.ldp;
    b.swaps = a.swaps;
    b.nswaps = a.nswaps;
    b.L = a.L;
    b.ldl = a.ldl;
    b.u0 = a.u0;
    b.la0 = a.la0;
    b.la1 = a.la1;
    b.w = a.w;
    if (hme_r2k_step(static_cast<hme_r2k*>(s), &b) != HME_OK) fail("hme_r2k_step");
}
void op_fetch(void* s, void* host, size_t ldh) {
    if (hme_r2k_fetch(static_cast<hme_r2k*>(s), host, ldh) != HME_OK) fail("hme_r2k_fetch");
}
void op_close(void* s) { hme_r2k_close(static_cast<hme_r2k*>(s)); }
bool op_verify() {
    const int v = g_verify.load(std::memory_order_relaxed);
    if (v >= 0) return v != 0;
    static const bool env = [] {
        const char* e = std::getenv("HME_R2K_VERIFY");
        return e && e[0] == '1';
    }();
    return env;
}
uint64_t op_store_budget() {
    const uint64_t o = g_store_bytes.load(std::memory_order_relaxed);
    if (o) return o;
    static const uint64_t mb = env_u64("HME_R2K_HOST_MB", 4096);
    return (mb ? mb : 4096) << 20;
}

const dev::Ops& table() {
    static const dev::Ops t = [] {
        dev::Ops o;
        o.plan = &op_plan;
        o.open = &op_open;
        o.put = &op_put;
        o.get = &op_get;
        o.step = &op_step;
        o.fetch = &op_fetch;
        o.close = &op_close;
        o.verify = &op_verify;
        o.store_budget = &op_store_budget;
        return o;
    }();
    return t;
}

// ---- the device RREF hook ----
// One hme context per thread that calls the hook (the reference's "one driver thread per backend").
struct ThreadCtx {
    hme_ctx* ctx = nullptr;
    int device = -1;
    ~ThreadCtx() {
        if (ctx) hme_ctx_destroy(ctx);
    }
};
hme_ctx* thread_ctx() {
    thread_local ThreadCtx tc;
    const int d = g_device.load(std::memory_order_relaxed);
    if (tc.ctx && tc.device != d) {
        hme_ctx_destroy(tc.ctx);
        tc.ctx = nullptr;
    }
    if (!tc.ctx) {
        if (hme_ctx_create(d, &tc.ctx) != HME_OK) {
            tc.ctx = nullptr;
            return nullptr;
        }
        tc.device = d;
    }
    return tc.ctx;
}

bool rref_hook(const engine::ModCtx<uint32_t>& ctx, engine::DenseView<uint32_t> A, bool want_rref,
               engine::elim::RrefResult& res) {
    static const bool off = env_off("HME_RREF");
    if (off || !ctx.is_field()) return false;
    const uint32_t m = A.rows(), n = A.cols();
    static const uint64_t min_env = env_u64("HME_RREF_MIN", 65536);
    const uint64_t mn = g_rref_min.load(std::memory_order_relaxed);
    if (static_cast<uint64_t>(m) * n < (mn ? mn : min_env) || m == 0 || n == 0) return false;
    if (!A.row_contiguous()) return false;
    hme_ctx* c = thread_ctx();
    if (!c) return false;
    std::vector<uint32_t> piv(std::min(m, n));
    uint32_t rank = 0;
    const int rc = want_rref ? hme_rref_u32(c, ctx.p, m, n, A.data(), A.row_stride(), piv.data(), &rank)
                             : hme_rank_profile_u32(c, ctx.p, m, n, A.data(), A.row_stride(), piv.data(), &rank);
    if (rc != HME_OK) return false;  // A is written only by a successful call: the host elimination runs
    res.rank = rank;
    res.pivots.assign(piv.begin(), piv.begin() + rank);
    g_rref_calls.fetch_add(1, std::memory_order_relaxed);
    return true;
}

}  // namespace

void install(int device) {
    g_device.store(device, std::memory_order_relaxed);
    dev::set_ops(&table());
    engine::elim::set_device_rref_hook(&rref_hook);
}

void uninstall() {
    dev::set_ops(nullptr);
    engine::elim::set_device_rref_hook(nullptr);
}

void set_r2k_max_cols(uint32_t cols) { g_max_cols.store(cols, std::memory_order_relaxed); }
void set_r2k_store_bytes(uint64_t bytes) { g_store_bytes.store(bytes, std::memory_order_relaxed); }
void set_r2k_verify(int on) { g_verify.store(on, std::memory_order_relaxed); }
void set_min_entries(uint64_t r2k, uint64_t rref) {
    g_r2k_min.store(r2k, std::memory_order_relaxed);
    g_rref_min.store(rref, std::memory_order_relaxed);
}
uint64_t r2k_sessions() { return g_sessions.load(std::memory_order_relaxed); }
uint64_t rref_calls() { return g_rref_calls.load(std::memory_order_relaxed); }

}  // namespace hme_seams

// TEST PROGRAM.  The reference's tape (drjanosch42/hacs 0.2.1: Recorder, compile, Executor and its
// DeviceBackend, compiled unchanged from the reference sources) linked against HmeEngineCuda.cpp --
// the reference's engine::cuda device layer implemented over libhme -- instead of the
// reference's libEngineCuda.  Each program runs with the device policy (its GEMM / Schur / AXPY /
// SCAL / TRANSPOSE / GATHER nodes on the GPU; twice, so the second run replays the captured
// CUDA graph) and again with the CPU policy, and every output must be equal entry for entry.
// Also: the executor's own device verify twin (ENGINE_VERIFY_DEVICE: every GPU node re-run on the
// CPU and compared) on one program.  Prints one line per check; exits 0 when all pass.
// Built by integration/Makefile; run by tests/test_integration_gpu.py.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

#include "CudaKernels.h"
#include "DenseBuf.h"
#include "Engine/Executor.h"
#include "Engine/Passes.h"
#include "Engine/Recorder.h"
#include "Engine/ThreadPool.h"
#include "ModCtx.h"

using namespace engine;
using namespace engine::tape;
using kernels::GemmOp;

namespace {

int g_checks = 0, g_fails = 0;
void check(bool ok, const std::string& what) {
    ++g_checks;
    if (!ok) ++g_fails;
    std::printf("%s %s\n", ok ? "ok" : "FAIL", what.c_str());
    std::fflush(stdout);
}

template <class Elt>
DenseBuf<Elt> rnd(uint32_t r, uint32_t c, Elt p, uint64_t seed, Layout lay = Layout::RowMajor) {
    std::mt19937_64 g(seed);
    DenseBuf<Elt> b(r, c, lay);
    for (uint32_t i = 0; i < r; ++i)
        for (uint32_t j = 0; j < c; ++j) b.at(i, j) = static_cast<Elt>(g() % p);
    return b;
}

template <class Elt>
bool same(const DenseBuf<Elt>& a, const DenseBuf<Elt>& b) {
    if (a.rows != b.rows || a.cols != b.cols) return false;
    for (uint32_t i = 0; i < a.rows; ++i)
        for (uint32_t j = 0; j < a.cols; ++j)
            if (a.at(i, j) != b.at(i, j)) return false;
    return true;
}

// One program: inputs A (m x k), B (k x n), E (m x k2), F (k2 x n); outputs
//   C = A B, D = C - E F (Schur update) + alpha C, then D scaled by beta, T = C^T,
//   G(i, t) = gamma [r(i) == col(t)] + delta C(r(i), col(t)) (a row-list gather).
template <class Elt>
struct Case {
    DenseBuf<Elt> A, B, E, F, C, D, T, G;
};

template <class Elt>
Case<Elt> make_case(Elt p, uint32_t m, uint32_t k, uint32_t n, uint32_t k2, Layout lay, uint64_t seed) {
    Case<Elt> c;
    c.A = rnd<Elt>(m, k, p, seed + 1, lay);
    c.B = rnd<Elt>(k, n, p, seed + 2);
    c.E = rnd<Elt>(m, k2, p, seed + 3);
    c.F = rnd<Elt>(k2, n, p, seed + 4, lay);
    c.C = DenseBuf<Elt>(m, n, lay);
    c.D = DenseBuf<Elt>(m, n);
    c.T = DenseBuf<Elt>(n, m);
    c.G = DenseBuf<Elt>(m / 2, n / 3, lay);
    return c;
}

template <class Elt>
void run_case(Case<Elt>& c, const ModCtx<Elt>& ctx, Executor<Elt>& ex, DevicePolicy pol, int runs) {
    Recorder<Elt> rec(ctx);
    const BufId a = rec.input(cview(c.A)), b = rec.input(cview(c.B)), e = rec.input(cview(c.E)),
                f = rec.input(cview(c.F));
    const BufId bc = rec.output(view(c.C)), bd = rec.output(view(c.D)), bt = rec.output(view(c.T)),
                bg = rec.output(view(c.G));
    const Elt alpha = static_cast<Elt>(5 % ctx.p), beta = static_cast<Elt>(3 % ctx.p);
    rec.gemm(rec.whole(a), rec.whole(b), rec.whole(bc), GemmOp::Set);
    rec.gemm(rec.whole(a), rec.whole(b), rec.whole(bd), GemmOp::Set);
    rec.schur_update(rec.whole(e), rec.whole(f), rec.whole(bd));
    rec.axpy(alpha, rec.whole(bc), rec.whole(bd));
    rec.scal(beta, rec.whole(bd));
    rec.transpose(rec.view(bc, 0, c.C.rows, 0, c.C.cols, /*transposed=*/true), rec.whole(bt));
    std::vector<uint32_t> rows, cols;
    for (uint32_t i = 0; i < c.G.rows; ++i) rows.push_back((7 * i + 3) % c.C.rows);
    for (uint32_t t = 0; t < c.G.cols; ++t) cols.push_back((5 * t + 1) % c.C.cols);
    const uint32_t rl = rec.index_list(rows), cl = rec.index_list(cols);
    rec.gather_rows(static_cast<Elt>(2), static_cast<Elt>(9), rec.whole(bc), 0, rl, cl, rec.whole(bg));
    Program<Elt> prog = rec.finish();
    PassOptions opts;
    opts.policy = pol;
    compile(prog, opts);
    const Bindings<Elt> bind = rec.bindings();
    for (int r = 0; r < runs; ++r) ex.run(prog, bind);
}

// graphs: 0 = direct launches only (ENGINE_CUDA_GRAPH=0, one run); 1 = the default (the second run
// of a program captured and replayed; three runs)
template <class Elt>
void check_program(const char* name, Elt p, uint32_t m, uint32_t k, uint32_t n, uint32_t k2, Layout lay,
                   uint64_t seed, int graphs, bool verify = false) {
    setenv("ENGINE_CUDA_GRAPH", graphs ? "1" : "0", 1);
    const ModCtx<Elt> ctx(p);
    ThreadPool pool(4);
    Executor<Elt> dev_ex(&pool), host_ex(&pool);
    dev_ex.set_verify_device(verify);
    Case<Elt> d = make_case<Elt>(p, m, k, n, k2, lay, seed), h = make_case<Elt>(p, m, k, n, k2, lay, seed);
    const std::string tag = std::string(name) + (graphs ? " [graph replay]" : " [direct]");
    try {
        run_case<Elt>(d, ctx, dev_ex, DevicePolicy::Gpu, graphs ? 3 : 1);
    } catch (const std::exception& e) {
        check(false, tag + ": " + e.what());
        return;
    }
    const auto& ds = dev_ex.device_stats();
    run_case<Elt>(h, ctx, host_ex, DevicePolicy::Cpu, 1);
    check(ds.gpu_nodes > 0 && (graphs == 0 || ds.graph_launches > 0),
          tag + ": GPU nodes ran (" + std::to_string(ds.gpu_nodes) + "), graph launches " +
              std::to_string(ds.graph_launches));
    check(same(d.C, h.C) && same(d.D, h.D) && same(d.T, h.T) && same(d.G, h.G),
          tag + ": GEMM, Schur update, AXPY, SCAL, TRANSPOSE and GATHER outputs equal the CPU run's");
}

}  // namespace

int main() {
    if (!cuda::available()) {
        std::printf("FAIL no device: %s\n", cuda::unavailable_reason());
        return 1;
    }
    try {
        for (int graphs : {0, 1}) {
            check_program<uint32_t>("u32 p=2^31-19 row-major 300x200x250", 2147483629u, 300, 200, 250, 64,
                                    Layout::RowMajor, 1, graphs);
            check_program<uint32_t>("u32 p=65521 column-major operands 257x130x300", 65521u, 257, 130, 300, 33,
                                    Layout::ColMajor, 2, graphs);
            check_program<uint64_t>("u64 p=2^61-1 row-major 160x90x120", (uint64_t(1) << 61) - 1, 160, 90, 120, 40,
                                    Layout::RowMajor, 3, graphs);
            check_program<uint64_t>("u64 p=2^64-59 column-major operands 96x70x64", static_cast<uint64_t>(-59), 96,
                                    70, 64, 17, Layout::ColMajor, 4, graphs);
        }
        check_program<uint32_t>("u32 p=4294967291 with the executor's device verify twin", 4294967291u, 200, 180,
                                150, 48, Layout::RowMajor, 5, 0, true);
        const cuda::LaunchStats ls = cuda::launch_stats();
        check(ls.gemm_launches > 0, "engine::cuda GEMMs served by libhme: " + std::to_string(ls.gemm_launches));
    } catch (const std::exception& e) {
        check(false, std::string("exception: ") + e.what());
    }
    std::printf("tape_check: %d checks, %d failed\n", g_checks, g_fails);
    return g_fails == 0 ? 0 : 1;
}

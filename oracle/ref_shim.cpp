// ORACLE / TEST INFRASTRUCTURE ONLY.  Never linked by the product library.
//
// A C-ABI shim over the reference's own CPU engine (drjanosch42/hacs 0.2.1,
// src/ModArithmetic and src/ModArithmetic/Binary), compiled from the reference
// sources where they lie by oracle/Makefile into oracle/_ref/libhacsref.so.
// Tests use it to pin the C restatement (oracle.c) and bench.py's cpu_baseline
// leg uses it as the reference CPU path.  Every entry point returns 0 on
// success and a negative code when the reference threw (message via
// ref_last_error()).
//
// Reference entry points bound here:
//   kernels::gemm<uint32_t>             src/ModArithmetic/Kernels.h:178-185 (Kernels.cpp:1418)
//   kernels::gemm_nt / gemv / axpy / scal / trmm / transpose / canonicalise (both forms)
//                                       src/ModArithmetic/Kernels.h:188-259
//   elim::rref / column_rank_profile    src/ModArithmetic/DenseElim.h:158-169 (DenseElim.cpp:921)
//   elim::kernel_basis                  src/ModArithmetic/DenseElim.h:176-179
//   elim::inverse                       src/ModArithmetic/DenseElim.h:188-189
//   elim::howell                        src/ModArithmetic/DenseElim.h:248-249
//   ring2k::howell / smith              src/ModArithmetic/Binary/Ring2k.h:702, :960
//   ring3k::smith / howell              src/ModArithmetic/Binary/Ring3k.h:100-101
//   smithpar::ScopedEnable              src/ModArithmetic/Binary/SmithPar.h:160
//   tape::Recorder::gemm + Executor::run src/Engine/Recorder.h:147, Executor.h:79 (the reference's
//                                       multi-thread GEMM path, EngineCoreScalingValidation.cpp:87-98)
//   tape::ScopedHostElimHook            src/Engine/EngineRuntime.h:260 (host eliminations split over
//                                       the consumer pool, ENGINE_API.md:1047-1059)
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "ModCtx.h"
#include "DenseBuf.h"
#include "DenseView.h"
#include "Kernels.h"
#include "DenseElim.h"
#include "Binary/Ring2k.h"
#include "Binary/Ring3k.h"
#include "Binary/SmithPar.h"
#include "Engine/EngineRuntime.h"
#include "Engine/Executor.h"
#include "Engine/Passes.h"
#include "Engine/Recorder.h"
#include "Engine/ThreadPool.h"

using namespace engine;

namespace {
thread_local std::string g_err;

template <class F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    } catch (...) {
        g_err = "unknown exception";
        return -2;
    }
}

DenseBuf<uint32_t> wrap(uint32_t* p, uint32_t rows, uint32_t cols, uint32_t ld) {
    return DenseBuf<uint32_t>(p, static_cast<size_t>(rows) * ld, rows, cols, Layout::RowMajor, ld);
}
}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// C op= A*B mod p (op 0 Set, 1 Add, 2 Sub), row-major with leading dims.
// threads > 1 splits C into row blocks, one kernels::gemm per block: the way
// the reference's tape executor parallelises a GEMM node (tiles of C, one
// kernels::gemm each).
int ref_gemm_u32(uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A, uint32_t lda,
                 const uint32_t* B, uint32_t ldb, uint32_t* C, uint32_t ldc, int op, int threads) {
    return guarded([&] {
        const ModCtx<uint32_t> ctx(p);
        const auto gop = op == 0 ? kernels::GemmOp::Set : op == 1 ? kernels::GemmOp::Add : kernels::GemmOp::Sub;
        DenseBuf<uint32_t> bA = wrap(const_cast<uint32_t*>(A), m, k, lda);
        DenseBuf<uint32_t> bB = wrap(const_cast<uint32_t*>(B), k, n, ldb);
        DenseBuf<uint32_t> bC = wrap(C, m, n, ldc);
        if (threads <= 1 || m < 64) {
            kernels::gemm<uint32_t>(ctx, cview(bA), cview(bB), DenseView<uint32_t>(bC), gop);
            return;
        }
        const uint32_t nt = static_cast<uint32_t>(threads);
        uint32_t rb = (m + nt - 1) / nt;
        rb = (rb + 7) / 8 * 8;
        std::vector<std::thread> pool;
        std::vector<std::string> errs(nt);
        for (uint32_t t = 0; t < nt; ++t) {
            const uint32_t r0 = t * rb;
            if (r0 >= m) break;
            const uint32_t r1 = std::min(m, r0 + rb);
            pool.emplace_back([&, r0, r1, t] {
                try {
                    DenseView<const uint32_t> a(bA, r0, r1 - r0, 0, k);
                    DenseView<uint32_t> c(bC, r0, r1 - r0, 0, n);
                    kernels::gemm<uint32_t>(ctx, a, cview(bB), c, gop);
                } catch (const std::exception& e) {
                    errs[t] = e.what();
                }
            });
        }
        for (auto& th : pool) th.join();
        for (auto& e : errs)
            if (!e.empty()) throw std::runtime_error(e);
    });
}

// C op= A*B mod p over u64 residues (ModCtx<uint64_t>: Montgomery for odd
// p < 2^63, wide otherwise).
int ref_gemm_u64(uint64_t p, uint32_t m, uint32_t n, uint32_t k, const uint64_t* A, uint32_t lda,
                 const uint64_t* B, uint32_t ldb, uint64_t* C, uint32_t ldc, int op) {
    return guarded([&] {
        const ModCtx<uint64_t> ctx(p);
        const auto gop = op == 0 ? kernels::GemmOp::Set : op == 1 ? kernels::GemmOp::Add : kernels::GemmOp::Sub;
        DenseBuf<uint64_t> bA(const_cast<uint64_t*>(A), static_cast<size_t>(m) * lda, m, k, Layout::RowMajor, lda);
        DenseBuf<uint64_t> bB(const_cast<uint64_t*>(B), static_cast<size_t>(k) * ldb, k, n, Layout::RowMajor, ldb);
        DenseBuf<uint64_t> bC(C, static_cast<size_t>(m) * ldc, m, n, Layout::RowMajor, ldc);
        kernels::gemm<uint64_t>(ctx, cview(bA), cview(bB), DenseView<uint64_t>(bC), gop);
    });
}

// Level-1 / level-2 CPU kernels of the reference, row-major with leading dims.
// C op= A * B^T with B given n x k.
int ref_gemm_nt_u32(uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A, uint32_t lda,
                    const uint32_t* B, uint32_t ldb, uint32_t* C, uint32_t ldc, int op) {
    return guarded([&] {
        const ModCtx<uint32_t> ctx(p);
        const auto gop = op == 0 ? kernels::GemmOp::Set : op == 1 ? kernels::GemmOp::Add : kernels::GemmOp::Sub;
        DenseBuf<uint32_t> bA = wrap(const_cast<uint32_t*>(A), m, k, lda);
        DenseBuf<uint32_t> bB = wrap(const_cast<uint32_t*>(B), n, k, ldb);
        DenseBuf<uint32_t> bC = wrap(C, m, n, ldc);
        kernels::gemm_nt<uint32_t>(ctx, cview(bA), cview(bB), DenseView<uint32_t>(bC), gop);
    });
}

// y op= A x; x and y contiguous vectors.
int ref_gemv_u32(uint32_t p, uint32_t m, uint32_t k, const uint32_t* A, uint32_t lda, const uint32_t* x,
                 uint32_t* y, int op) {
    return guarded([&] {
        const ModCtx<uint32_t> ctx(p);
        const auto gop = op == 0 ? kernels::GemmOp::Set : op == 1 ? kernels::GemmOp::Add : kernels::GemmOp::Sub;
        DenseBuf<uint32_t> bA = wrap(const_cast<uint32_t*>(A), m, k, lda);
        DenseBuf<uint32_t> bx = wrap(const_cast<uint32_t*>(x), k, 1, 1);
        DenseBuf<uint32_t> by = wrap(y, m, 1, 1);
        kernels::gemv<uint32_t>(ctx, cview(bA), cview(bx), DenseView<uint32_t>(by), gop);
    });
}

// y = y +/- alpha x (subtract != 0), or x = alpha x when y is null (scal).
int ref_axpy_scal_u32(uint32_t p, uint32_t alpha, uint32_t rows, uint32_t cols, uint32_t* x, uint32_t ldx,
                      uint32_t* y, uint32_t ldy, int subtract) {
    return guarded([&] {
        const ModCtx<uint32_t> ctx(p);
        DenseBuf<uint32_t> bx = wrap(x, rows, cols, ldx);
        if (y == nullptr) {
            kernels::scal<uint32_t>(ctx, alpha, DenseView<uint32_t>(bx));
            return;
        }
        DenseBuf<uint32_t> by = wrap(y, rows, cols, ldy);
        kernels::axpy<uint32_t>(ctx, alpha, cview(bx), DenseView<uint32_t>(by), subtract != 0);
    });
}

// C = T B with T m x m unit lower (lower != 0) or unit upper triangular.
int ref_trmm_unit_u32(uint32_t p, int lower, uint32_t m, uint32_t n, const uint32_t* T, uint32_t ldt,
                      const uint32_t* B, uint32_t ldb, uint32_t* C, uint32_t ldc) {
    return guarded([&] {
        const ModCtx<uint32_t> ctx(p);
        DenseBuf<uint32_t> bT = wrap(const_cast<uint32_t*>(T), m, m, ldt);
        bT.structure = lower ? Structure::LowerUnitri : Structure::UpperUnitri;
        DenseBuf<uint32_t> bB = wrap(const_cast<uint32_t*>(B), m, n, ldb);
        DenseBuf<uint32_t> bC = wrap(C, m, n, ldc);
        kernels::trmm<uint32_t>(ctx, cview(bT), cview(bB), DenseView<uint32_t>(bC));
    });
}

// dst (cols x rows) = src (rows x cols) transposed.
int ref_transpose_u32(uint32_t rows, uint32_t cols, const uint32_t* src, uint32_t lds, uint32_t* dst, uint32_t ldd) {
    return guarded([&] {
        DenseBuf<uint32_t> bs = wrap(const_cast<uint32_t*>(src), rows, cols, lds);
        DenseBuf<uint32_t> bd = wrap(dst, cols, rows, ldd);
        kernels::transpose<uint32_t>(cview(bs), DenseView<uint32_t>(bd));
    });
}

// v (entries below 2p) -> canonical in place.
int ref_canonicalise_u32(uint32_t p, uint32_t rows, uint32_t cols, uint32_t* v, uint32_t ld) {
    return guarded([&] {
        const ModCtx<uint32_t> ctx(p);
        DenseBuf<uint32_t> bv = wrap(v, rows, cols, ld);
        bv.invariant = Invariant::Lazy2p;
        kernels::canonicalise<uint32_t>(ctx, DenseView<uint32_t>(bv));
    });
}

// dst = acc mod p for 64-bit accumulators.
int ref_canonicalise_acc64_u32(uint32_t p, uint32_t rows, uint32_t cols, const uint64_t* acc, uint32_t lda,
                               uint32_t* dst, uint32_t ldd) {
    return guarded([&] {
        const ModCtx<uint32_t> ctx(p);
        DenseBuf<uint64_t> ba(const_cast<uint64_t*>(acc), static_cast<size_t>(rows) * lda, rows, cols,
                              Layout::RowMajor, lda, Invariant::Accum64);
        DenseBuf<uint32_t> bd = wrap(dst, rows, cols, ldd);
        kernels::canonicalise(ctx, cview(ba), DenseView<uint32_t>(bd));
    });
}

// In-place RREF over F_p; pivots must hold min(m, n) entries.
int ref_rref_u32(uint32_t p, uint32_t m, uint32_t n, uint32_t* A, uint32_t lda, uint32_t* pivots,
                 uint32_t* rank) {
    return guarded([&] {
        const ModCtx<uint32_t> ctx(p);
        DenseBuf<uint32_t> b = wrap(A, m, n, lda);
        const elim::RrefResult r = elim::rref<uint32_t>(ctx, DenseView<uint32_t>(b));
        *rank = r.rank;
        for (uint32_t i = 0; i < r.rank; ++i) pivots[i] = r.pivots[i];
    });
}

// Column rank profile (A destroyed).
int ref_rank_profile_u32(uint32_t p, uint32_t m, uint32_t n, uint32_t* A, uint32_t lda, uint32_t* pivots,
                         uint32_t* rank) {
    return guarded([&] {
        const ModCtx<uint32_t> ctx(p);
        DenseBuf<uint32_t> b = wrap(A, m, n, lda);
        const elim::RrefResult r = elim::column_rank_profile<uint32_t>(ctx, DenseView<uint32_t>(b));
        *rank = r.rank;
        for (uint32_t i = 0; i < r.rank; ++i) pivots[i] = r.pivots[i];
    });
}

// Kernel basis ((n - rank) x n rows) of an RREF R (rows x n) with its pivots.
int ref_kernel_basis_u32(uint32_t p, uint32_t rows, uint32_t n, const uint32_t* R, uint32_t ldr,
                         const uint32_t* pivots, uint32_t rank, uint32_t* K) {
    return guarded([&] {
        const ModCtx<uint32_t> ctx(p);
        DenseBuf<uint32_t> b = wrap(const_cast<uint32_t*>(R), rows, n, ldr);
        std::vector<uint32_t> pv(pivots, pivots + rank);
        DenseBuf<uint32_t> kb = elim::kernel_basis<uint32_t>(ctx, cview(b), pv);
        for (uint32_t i = 0; i < kb.rows; ++i)
            for (uint32_t j = 0; j < kb.cols; ++j) K[static_cast<size_t>(i) * n + j] = kb.at(i, j);
    });
}

// Inverse of a square matrix; *ok = 0 when singular.
int ref_inverse_u32(uint32_t p, uint32_t n, const uint32_t* A, uint32_t* Ainv, int* ok) {
    return guarded([&] {
        const ModCtx<uint32_t> ctx(p);
        DenseBuf<uint32_t> a = wrap(const_cast<uint32_t*>(A), n, n, n);
        DenseBuf<uint32_t> x = wrap(Ainv, n, n, n);
        *ok = elim::inverse<uint32_t>(ctx, cview(a), DenseView<uint32_t>(x)) ? 1 : 0;
    });
}

// Howell form over Z/ell^k by the generic engine route (elim::howell).  H must
// hold n*n entries; pivots/pivot_v n entries; *h receives the row count.
int ref_elim_howell_u32(uint32_t ell, uint32_t kexp, uint32_t m, uint32_t n, const uint32_t* A, uint32_t* H,
                        uint32_t* pivots, uint32_t* pivot_v, uint32_t* h) {
    return guarded([&] {
        const ModCtx<uint32_t> ctx = ModCtx<uint32_t>::prime_power(ell, kexp);
        DenseBuf<uint32_t> a = wrap(const_cast<uint32_t*>(A), m, n, n);
        const elim::HowellResult<uint32_t> r = elim::howell<uint32_t>(ctx, cview(a));
        *h = r.rows();
        for (uint32_t i = 0; i < r.rows(); ++i) {
            pivots[i] = r.pivots[i];
            pivot_v[i] = r.pivot_v[i];
            for (uint32_t j = 0; j < n; ++j) H[static_cast<size_t>(i) * n + j] = r.H.at(i, j);
        }
    });
}

// Howell form over Z/2^k (k <= 32) by the ring2k ladder (u32 rung).
int ref_howell_2k_u32(uint32_t kexp, uint32_t m, uint32_t n, const uint32_t* A, uint32_t* H, uint32_t* pivots,
                      uint32_t* pivot_v, uint32_t* h, int threads) {
    return guarded([&] {
        using Tr = ring2k::Traits<uint32_t>;
        ring2k::Mat<uint32_t> M(m, n);
        std::memcpy(M.a.data(), A, sizeof(uint32_t) * static_cast<size_t>(m) * n);
        std::unique_ptr<smithpar::ScopedEnable> par;
        if (threads > 1) par.reset(new smithpar::ScopedEnable());
        const ring2k::HowellForm<uint32_t> r = ring2k::howell<Tr>(std::move(M), kexp);
        *h = static_cast<uint32_t>(r.pivots.size());
        for (uint32_t i = 0; i < *h; ++i) {
            pivots[i] = r.pivots[i];
            pivot_v[i] = r.pivot_v[i];
            for (uint32_t j = 0; j < n; ++j) H[static_cast<size_t>(i) * n + j] = r.H.at(i, j);
        }
    });
}

// Smith valuations over Z/2^k (u32 rung); sigma holds min(m, n) entries.
int ref_smith_2k_u32(uint32_t kexp, uint32_t m, uint32_t n, const uint32_t* A, uint32_t* sigma, uint32_t* count,
                     int threads) {
    return guarded([&] {
        using Tr = ring2k::Traits<uint32_t>;
        ring2k::Mat<uint32_t> M(m, n);
        std::memcpy(M.a.data(), A, sizeof(uint32_t) * static_cast<size_t>(m) * n);
        std::unique_ptr<smithpar::ScopedEnable> par;
        if (threads > 1) par.reset(new smithpar::ScopedEnable());
        const ring2k::SmithResult r = ring2k::smith<Tr>(std::move(M), kexp);
        *count = static_cast<uint32_t>(r.sigma.size());
        for (uint32_t i = 0; i < *count; ++i) sigma[i] = r.sigma[i];
    });
}

// Smith valuations over Z/3^k, k <= 19.
int ref_smith_3k_u32(uint32_t kexp, uint32_t m, uint32_t n, const uint32_t* A, uint32_t* sigma, uint32_t* count,
                     int threads) {
    return guarded([&] {
        DenseBuf<uint32_t> a(m, n);
        for (uint32_t i = 0; i < m; ++i)
            for (uint32_t j = 0; j < n; ++j) a.at(i, j) = A[static_cast<size_t>(i) * n + j];
        std::unique_ptr<smithpar::ScopedEnable> par;
        if (threads > 1) par.reset(new smithpar::ScopedEnable());
        const ring3k::SmithResult r = ring3k::smith(std::move(a), kexp);
        *count = static_cast<uint32_t>(r.sigma.size());
        for (uint32_t i = 0; i < *count; ++i) sigma[i] = r.sigma[i];
    });
}

// Howell form over Z/3^k, k <= 19.
int ref_howell_3k_u32(uint32_t kexp, uint32_t m, uint32_t n, const uint32_t* A, uint32_t* H, uint32_t* pivots,
                      uint32_t* pivot_v, uint32_t* h, int threads) {
    return guarded([&] {
        DenseBuf<uint32_t> a(m, n);
        for (uint32_t i = 0; i < m; ++i)
            for (uint32_t j = 0; j < n; ++j) a.at(i, j) = A[static_cast<size_t>(i) * n + j];
        std::unique_ptr<smithpar::ScopedEnable> par;
        if (threads > 1) par.reset(new smithpar::ScopedEnable());
        const ring3k::HowellForm r = ring3k::howell(std::move(a), kexp);
        *h = static_cast<uint32_t>(r.pivots.size());
        for (uint32_t i = 0; i < *h; ++i) {
            pivots[i] = r.pivots[i];
            pivot_v[i] = r.pivot_v[i];
            for (uint32_t j = 0; j < n; ++j) H[static_cast<size_t>(i) * n + j] = r.H.at(i, j);
        }
    });
}

// C = A*B mod p (row-major, dense) through the reference's tape: one Recorder::gemm node, compiled,
// then run `reps` times by an Executor on a ThreadPool of `threads` workers (the executor tiles the
// node's C over the pool).  *seconds = the mean wall time of one Executor::run.
int ref_tape_gemm_u32(uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A, const uint32_t* B,
                      uint32_t* C, int threads, int reps, double* seconds) {
    return guarded([&] {
        const ModCtx<uint32_t> ctx(p);
        DenseBuf<uint32_t> bA = wrap(const_cast<uint32_t*>(A), m, k, k);
        DenseBuf<uint32_t> bB = wrap(const_cast<uint32_t*>(B), k, n, n);
        DenseBuf<uint32_t> bC = wrap(C, m, n, n);
        tape::ThreadPool pool(static_cast<uint32_t>(threads < 1 ? 1 : threads));
        tape::Executor<uint32_t> ex(&pool);
        tape::Recorder<uint32_t> rec(ctx);
        const tape::BufId a = rec.input(cview(bA)), b = rec.input(cview(bB)), c = rec.output(DenseView<uint32_t>(bC));
        rec.gemm(rec.whole(a), rec.whole(b), rec.whole(c), kernels::GemmOp::Set);
        tape::Program<uint32_t> prog = rec.finish();
        tape::compile(prog, tape::PassOptions());
        const tape::Bindings<uint32_t> bind = rec.bindings();
        const int r = reps < 1 ? 1 : reps;
        const auto t0 = std::chrono::steady_clock::now();
        for (int i = 0; i < r; ++i) ex.run(prog, bind);
        const auto t1 = std::chrono::steady_clock::now();
        *seconds = std::chrono::duration<double>(t1 - t0).count() / r;
    });
}

// elim::rref of A (in place) with the host elimination hook of the tape bound to a pool of `threads`
// workers: the reference's multi-thread host elimination.
int ref_rref_par_u32(uint32_t p, uint32_t m, uint32_t n, uint32_t* A, uint32_t lda, uint32_t* pivots,
                     uint32_t* rank, int threads) {
    return guarded([&] {
        const ModCtx<uint32_t> ctx(p);
        DenseBuf<uint32_t> a = wrap(A, m, n, lda);
        tape::ThreadPool pool(static_cast<uint32_t>(threads < 1 ? 1 : threads));
        tape::ScopedConsumerPool scp(&pool);
        tape::ScopedHostElimHook hook;
        const elim::RrefResult r = elim::rref<uint32_t>(ctx, DenseView<uint32_t>(a));
        *rank = r.rank;
        for (uint32_t i = 0; i < r.rank; ++i) pivots[i] = r.pivots[i];
    });
}

}  // extern "C"

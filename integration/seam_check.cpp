// TEST PROGRAM.  The reference's own callers (drjanosch42/hacs 0.2.1, its CPU engine compiled from
// the reference sources) with libhme installed behind their seams by HmeSeams.cpp, checked entry
// for entry against the same callers on the host route:
//
//   ring2k::echelon_blocked / smith / howell of the u32 and u64 rungs with the device LU table
//   (resident and tiled windows, serial and threaded routes, both pivot rules through smith and
//   howell, the reference's own verify twin on some runs);
//   elim::rref / column_rank_profile / inverse / solve_multi_rhs with the device RREF hook.
//
// Prints one line per check and a summary; exits 0 when every check passed.  Built by
// integration/Makefile; run by tests/test_integration_gpu.py.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "Binary/Ring2k.h"
#include "Binary/Ring2kDevice.h"
#include "Binary/SmithPar.h"
#include "DenseBuf.h"
#include "DenseElim.h"
#include "ModCtx.h"
#include "HmeSeams.h"

using namespace engine;
namespace r2 = engine::ring2k;

namespace {

int g_checks = 0, g_fails = 0;

void check(bool ok, const std::string& what) {
    ++g_checks;
    if (!ok) ++g_fails;
    std::printf("%s %s\n", ok ? "ok" : "FAIL", what.c_str());
    std::fflush(stdout);
}

template <class E>
E mask(E x, uint32_t k) {
    return k >= sizeof(E) * 8 ? x : static_cast<E>(x & ((E(1) << k) - 1));
}

// U D V over Z/2^k: D = diag(2^e_i) (e_i geometric(1/2) truncated at k: e_i = k gives 0), U and V
// each the product of `ops` random elementary operations with multipliers in [-5, 5]; entries
// masked to k bits (canonical).  The Smith valuations are sorted{e_i : e_i < k}.
template <class E>
r2::Mat<E> planted(uint32_t m, uint32_t n, uint32_t k, uint32_t ops, uint64_t seed, std::vector<uint32_t>& sigma) {
    std::mt19937_64 g(seed);
    r2::Mat<E> M(m, n);
    sigma.clear();
    for (uint32_t i = 0; i < std::min(m, n); ++i) {
        uint32_t e = 0;
        while (e < k && (g() & 1)) ++e;
        if (e < k) sigma.push_back(e);
        M.at(i, i) = mask<E>(E(1) << (e < sizeof(E) * 8 ? e : 0), k) * (e < k ? 1 : 0);
    }
    std::sort(sigma.begin(), sigma.end());
    for (uint32_t t = 0; t < ops; ++t) {  // row_i += c row_j
        const uint32_t i = g() % m, j = (i + 1 + g() % (m - 1)) % m;
        const E c = static_cast<E>(static_cast<int64_t>(g() % 11) - 5);
        for (uint32_t col = 0; col < n; ++col) M.at(i, col) = mask<E>(M.at(i, col) + c * M.at(j, col), k);
    }
    for (uint32_t t = 0; t < ops; ++t) {  // col_i += c col_j
        const uint32_t i = g() % n, j = (i + 1 + g() % (n - 1)) % n;
        const E c = static_cast<E>(static_cast<int64_t>(g() % 11) - 5);
        for (uint32_t row = 0; row < m; ++row) M.at(row, i) = mask<E>(M.at(row, i) + c * M.at(row, j), k);
    }
    return M;
}

template <class E>
r2::Mat<E> planted_mat(uint32_t m, uint32_t n, uint32_t k, uint64_t seed) {
    std::vector<uint32_t> sigma;
    return planted<E>(m, n, k, 64, seed, sigma);
}

template <class E>
r2::Mat<E> random_mat(uint32_t m, uint32_t n, uint32_t k, uint64_t seed) {
    std::mt19937_64 g(seed);
    r2::Mat<E> M(m, n);
    for (auto& x : M.a) x = mask<E>(static_cast<E>(g()), k);
    return M;
}

bool same_info(const r2::EchelonInfo& a, const r2::EchelonInfo& b) {
    return a.rank == b.rank && a.pivots == b.pivots && a.pivot_v == b.pivot_v;
}

// echelon_blocked on the device route vs the host route: every entry, rank, pivots, valuations.
template <class Tr>
void check_echelon(const char* name, r2::Mat<typename Tr::E> A, uint32_t k, r2::PivotRule rule, uint32_t panel) {
    r2::Mat<typename Tr::E> H = A;
    const uint64_t dev0 = r2::device::stats().device;
    const r2::EchelonInfo di = r2::echelon_blocked<Tr>(A, k, rule, panel);
    const bool took = r2::device::stats().device > dev0;
    r2::EchelonInfo hi;
    {
        const r2::device::ScopedHostOnly host;
        hi = r2::echelon_blocked<Tr>(H, k, rule, panel);
    }
    check(took, std::string(name) + ": the device route ran");
    check(same_info(di, hi) && A.a == H.a, std::string(name) + ": matrix, rank " + std::to_string(di.rank) +
                                               ", pivots and valuations equal the host LU's");
}

template <class Tr>
void check_smith_howell(const char* name, uint32_t m, uint32_t n, uint32_t k, uint64_t seed) {
    using E = typename Tr::E;
    std::vector<uint32_t> sigma;
    const r2::Mat<E> M = planted<E>(m, n, k, 64, seed, sigma);
    const uint64_t dev0 = r2::device::stats().device;
    const r2::SmithResult ds = r2::smith<Tr>(M, k);
    const r2::HowellForm<E> dh = r2::howell<Tr>(M, k);
    const bool took = r2::device::stats().device > dev0;
    r2::SmithResult hs;
    r2::HowellForm<E> hh;
    {
        const r2::device::ScopedHostOnly host;
        hs = r2::smith<Tr>(M, k);
        hh = r2::howell<Tr>(M, k);
    }
    check(took, std::string(name) + ": the device route ran");
    check(ds.sigma == hs.sigma && ds.level_ranks == hs.level_ranks && ds.sigma == sigma,
          std::string(name) + ": Smith valuations equal the host route's and the planted ones (" +
              std::to_string(ds.sigma.size()) + ")");
    check(dh.H.a == hh.H.a && dh.pivots == hh.pivots && dh.pivot_v == hh.pivot_v && dh.length() == ds.length(),
          std::string(name) + ": Howell form equals the host route's (" + std::to_string(dh.pivots.size()) + " rows)");
}

DenseBuf<uint32_t> ranked(uint32_t m, uint32_t n, uint32_t r, uint32_t p, uint64_t seed) {
    std::mt19937_64 g(seed);
    std::vector<uint64_t> L(static_cast<size_t>(m) * r), R(static_cast<size_t>(r) * n);
    for (auto& x : L) x = g() % p;
    for (auto& x : R) x = g() % p;
    DenseBuf<uint32_t> A(m, n);
    for (uint32_t i = 0; i < m; ++i)
        for (uint32_t j = 0; j < n; ++j) {
            unsigned __int128 s = 0;
            for (uint32_t t = 0; t < r; ++t) s += static_cast<unsigned __int128>(L[i * r + t]) * R[t * n + j];
            A.at(i, j) = static_cast<uint32_t>(s % p);
        }
    return A;
}

bool same_buf(const DenseBuf<uint32_t>& a, const DenseBuf<uint32_t>& b) {
    if (a.rows != b.rows || a.cols != b.cols) return false;
    for (uint32_t i = 0; i < a.rows; ++i)
        for (uint32_t j = 0; j < a.cols; ++j)
            if (a.at(i, j) != b.at(i, j)) return false;
    return true;
}

void check_rref_hook(uint32_t p, uint32_t m, uint32_t n, uint32_t r, uint64_t seed) {
    const ModCtx<uint32_t> ctx(p);
    const DenseBuf<uint32_t> A0 = ranked(m, n, r, p, seed);
    const std::string tag = std::to_string(m) + "x" + std::to_string(n) + " rank " + std::to_string(r) + " p=" +
                            std::to_string(p);
    DenseBuf<uint32_t> D = A0, H = A0, Dp = A0, Hp = A0;
    const uint64_t calls0 = hme_seams::rref_calls();
    const elim::RrefResult dr = elim::rref<uint32_t>(ctx, view(D));
    const elim::RrefResult dp = elim::column_rank_profile<uint32_t>(ctx, view(Dp));
    const bool took = hme_seams::rref_calls() >= calls0 + 2;
    hme_seams::uninstall();
    const elim::RrefResult hr = elim::rref<uint32_t>(ctx, view(H));
    const elim::RrefResult hp = elim::column_rank_profile<uint32_t>(ctx, view(Hp));
    hme_seams::install(0);
    check(took, "elim::rref / column_rank_profile " + tag + ": the device hook served both");
    check(dr.rank == hr.rank && dr.pivots == hr.pivots && same_buf(D, H),
          "elim::rref " + tag + ": RREF, rank and pivots equal the host elimination's");
    check(dp.rank == hp.rank && dp.pivots == hp.pivots, "elim::column_rank_profile " + tag + ": equal the host's");
}

void check_inverse_solve(uint32_t p, uint32_t n, uint64_t seed) {
    const ModCtx<uint32_t> ctx(p);
    const DenseBuf<uint32_t> A = ranked(n, n, n, p, seed);
    DenseBuf<uint32_t> Di(n, n), Hi(n, n);
    const DenseBuf<uint32_t> Y = ranked(n, 7, 7, p, seed + 1);
    const uint64_t calls0 = hme_seams::rref_calls();
    const bool dok = elim::inverse<uint32_t>(ctx, cview(A), view(Di));
    const auto dsol = elim::solve_multi_rhs<uint32_t>(ctx, cview(A), cview(Y));
    const bool took = hme_seams::rref_calls() >= calls0 + 2;
    hme_seams::uninstall();
    const bool hok = elim::inverse<uint32_t>(ctx, cview(A), view(Hi));
    const auto hsol = elim::solve_multi_rhs<uint32_t>(ctx, cview(A), cview(Y));
    hme_seams::install(0);
    const std::string tag = std::to_string(n) + "^2 p=" + std::to_string(p);
    check(took, "elim::inverse / solve_multi_rhs " + tag + ": served by the device hook");
    check(dok == hok && dok && same_buf(Di, Hi), "elim::inverse " + tag + ": equal the host's");
    check(dsol == hsol, "elim::solve_multi_rhs " + tag + ": equal the host's");
}

}  // namespace

int main() {
    hme_seams::install(0);
    hme_seams::set_min_entries(1, 1);
    using T32 = r2::Traits<uint32_t>;
    using T64 = r2::Traits<uint64_t>;
    try {
        // ---- the ring2k device LU, u32 rung ----
        check_echelon<T32>("echelon_blocked u32 700x600 Z/2^16 MinValuation panel 64",
                           planted_mat<uint32_t>(700, 600, 16, 1), 16,
                           r2::PivotRule::MinValuation, 64);
        check_echelon<T32>("echelon_blocked u32 513x777 Z/2^32 random panel 128",
                           random_mat<uint32_t>(513, 777, 32, 2), 32, r2::PivotRule::MinValuation, 128);
        check_echelon<T32>("echelon_blocked u32 300x300 Z/2^5 random panel 48", random_mat<uint32_t>(300, 300, 5, 3),
                           5, r2::PivotRule::MinValuation, 48);
        hme_seams::set_r2k_verify(1);
        check_echelon<T32>("echelon_blocked u32 400x500 Z/2^20 (reference verify twin on)",
                           planted_mat<uint32_t>(400, 500, 20, 4), 20,
                           r2::PivotRule::MinValuation, 64);
        hme_seams::set_r2k_verify(0);
        // tiled route: a window of 4 panels, L-store budget of ~3 panels (phase breaks)
        hme_seams::set_r2k_max_cols(256);
        hme_seams::set_r2k_store_bytes(3ull * 600 * 64 * 4);
        check_echelon<T32>("echelon_blocked u32 600x1000 Z/2^16 tiled (4-panel window, phase breaks)",
                           planted_mat<uint32_t>(600, 1000, 16, 5), 16,
                           r2::PivotRule::MinValuation, 64);
        hme_seams::set_r2k_max_cols(0);
        hme_seams::set_r2k_store_bytes(0);
        check_smith_howell<T32>("smith/howell u32 512x512 Z/2^16 serial", 512, 512, 16, 11);
        check_smith_howell<T32>("smith/howell u32 300x420 Z/2^32 serial", 300, 420, 32, 12);
        {
            const engine::smithpar::ScopedEnable par;
            check_smith_howell<T32>("smith/howell u32 640x640 Z/2^16 threaded (device panel 128)", 640, 640, 16, 13);
        }
        // ---- u64 rung ----
        check_echelon<T64>("echelon_blocked u64 300x400 Z/2^64 random panel 64", random_mat<uint64_t>(300, 400, 64, 6),
                           64, r2::PivotRule::MinValuation, 64);
        check_smith_howell<T64>("smith/howell u64 256x320 Z/2^40 serial", 256, 320, 40, 14);
        check(hme_seams::r2k_sessions() > 0, "device LU sessions opened: " + std::to_string(hme_seams::r2k_sessions()));
        // ---- the device RREF hook ----
        check_rref_hook(2147483629u, 300, 400, 250, 21);
        check_rref_hook(65521u, 520, 300, 300, 22);
        check_rref_hook(4294967291u, 257, 257, 200, 23);
        check_inverse_solve(2147483629u, 200, 24);
    } catch (const std::exception& e) {
        check(false, std::string("exception: ") + e.what());
    }
    std::printf("seam_check: %d checks, %d failed\n", g_checks, g_fails);
    hme_seams::uninstall();
    return g_fails == 0 ? 0 : 1;
}

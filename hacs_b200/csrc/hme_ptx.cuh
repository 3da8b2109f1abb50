// Inline-PTX building blocks for sm_100a: mbarriers with bounded waits, TMA
// tensor loads (each CTA loads only into its own shared memory), and the tcgen05
// tensor-core / tensor-memory instructions.
//
// Every spin on an mbarrier is bounded by wall time (%globaltimer): when the
// limit passes, the waiting thread records an error code in the kernel's
// global error word, raises the CTA's abort flag and returns false, so a
// kernel never hangs the device; the host reads the error word after the
// launch and reports HME_ETIMEOUT.
#pragma once
#include <cstdint>
#include <cuda.h>

namespace hme {

#ifndef HME_WAIT_LIMIT_NS
#define HME_WAIT_LIMIT_NS 2000000000ull  // 2 s per wait: far above any legitimate stage wait
#endif

enum DeviceErr : int {
    DERR_NONE = 0,
    DERR_WAIT_FULL = 1,       // consumer waited too long for a TMA stage
    DERR_WAIT_EMPTY = 2,      // producer waited too long for a free stage
    DERR_WAIT_ACCUM = 3,      // epilogue waited too long for an accumulator
    DERR_WAIT_ACCUM_FREE = 4, // MMA issuer waited too long for a drained accumulator
    DERR_WAIT_DRAIN = 5,      // tear-down wait for in-flight copies / MMAs ran out
    DERR_TMEM_ADDR = 6,       // tensor-memory allocation returned an unusable address
    DERR_GRID_BARRIER = 7,    // a cooperative kernel's grid barrier waited too long
    DERR_LAUNCH_SHAPE = 8,    // a kernel found its launch shape outside what it supports and did nothing
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- asynchronous 4-byte global -> shared copies (cp.async) ------------------------
// When !valid no byte is read (src-size 0) and the word is zero-filled; src must
// still be a valid global address.
__device__ __forceinline__ void cp_async4(uint32_t* dst, const uint32_t* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(valid ? 4 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// wait until at most N of this thread's committed groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---- mbarrier --------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, P;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase with the given parity to complete.  Returns false when
// the CTA's abort flag is up or the wall-time limit passed (then the error
// word receives `code` and the abort flag is raised for the whole CTA).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int* err,
                                          int code) {
    const uint32_t a = smem_u32(bar);
    if (mbar_try_wait(a, parity)) return true;
    const uint64_t t0 = global_timer_ns();
    for (uint32_t spin = 1;; ++spin) {
        if (mbar_try_wait(a, parity)) return true;
        if ((spin & 31u) == 0) {
            if (*abort_flag) return false;
            if (global_timer_ns() - t0 > HME_WAIT_LIMIT_NS) {
                *abort_flag = 1;
                atomicCAS(err, 0, code);
                return false;
            }
        }
    }
}

// ---- exact dot products ---------------------------------------------------------
// (a2:a1:a0) += x * y as one 96-bit unsigned sum (mad.lo.cc / madc.hi.cc / addc):
// up to 2^32 products below 2^64 stay exact; reduce the sum once at the end.
__device__ __forceinline__ void mac96(uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t x, uint32_t y) {
    asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
        "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
        "addc.u32 %2, %2, 0;"
        : "+r"(a0), "+r"(a1), "+r"(a2)
        : "r"(x), "r"(y));
}

// ---- L2 prefetch ----------------------------------------------------------------
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
// Prefetch into L2 the 128-byte lines of w u32 values at p (one row segment).
__device__ __forceinline__ void prefetch_l2_span(const uint32_t* p, int w) {
    if (w <= 0) return;
    const uintptr_t b = reinterpret_cast<uintptr_t>(p) & ~uintptr_t(127);
    const uintptr_t e = reinterpret_cast<uintptr_t>(p + w);
    for (uintptr_t q = b; q < e; q += 128) prefetch_l2(reinterpret_cast<const void*>(q));
}

// ---- thread-block clusters: ranks and distributed shared memory ----
__device__ __forceinline__ uint32_t cluster_ctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_nctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
// The shared::cluster address of `local_addr` (a shared::cta address) in CTA `rank`'s shared memory.
__device__ __forceinline__ uint32_t dsmem_addr(uint32_t local_addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local_addr), "r"(rank));
    return r;
}
__device__ __forceinline__ uint32_t ld_dsmem_u32(uint32_t addr) {
    uint32_t v;
    asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_dsmem_u64(uint32_t addr) {
    unsigned long long v;
    asm volatile("ld.shared::cluster.u64 %0, [%1];" : "=l"(v) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ void st_dsmem_u32(uint32_t addr, uint32_t v) {
    asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
__device__ __forceinline__ void st_dsmem_u64(uint32_t addr, unsigned long long v) {
    asm volatile("st.shared::cluster.u64 [%0], %1;" ::"r"(addr), "l"(v) : "memory");
}

// ---- TMA (tiled tensor loads into this CTA's shared memory) -----------------
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
        "[%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2, int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, "
        "%6}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}
__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// ---- programmatic dependent launch ------------------------------------------------
// A kernel launched with programmatic stream serialisation may start while the
// kernel before it in the stream is still running; grid_dep_wait() blocks until
// that kernel has completed and its memory operations are visible (it returns
// at once for a kernel launched without the attribute).  grid_dep_launch() lets
// the next kernel's CTAs start being scheduled.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// ---- tcgen05: tensor memory ----------------------------------------------------
// Allocation / deallocation are warp-collective (.sync.aligned): call from one full warp.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// ---- tcgen05: MMA ------------------------------------------------------------------
// D[tmem] (+)= A[smem desc] x B[smem desc], u8 x u8 -> s32, one elected thread.
__device__ __forceinline__ void mma_u8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// Arrive (once) on a CTA-local mbarrier when every tcgen05 op issued so far by this thread is done.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// ---- tcgen05: tensor memory -> registers ----------------------------------------------
// 32 lanes x 32 bits, 16 consecutive columns per thread (thread t of the warp reads lane base+t).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ---- descriptors --------------------------------------------------------------------------
// Shared-memory matrix descriptor for a K-major operand written by TMA with
// 128-byte swizzle: rows of 128 bytes, 8-row atoms 1024 bytes apart (SBO),
// LBO unused for swizzled K-major layouts (encoded 1), version 1 (sm_100),
// layout type 2 = SWIZZLE_128B.  The tile base must be 1024-byte aligned.
__device__ __forceinline__ uint64_t smem_desc_k128(uint32_t smem_addr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((smem_addr & 0x3FFFFu) >> 4);
    d |= static_cast<uint64_t>(1) << 16;
    d |= static_cast<uint64_t>(1024 >> 4) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    d |= static_cast<uint64_t>(2) << 61;
    return d;
}
// The same for a K-major operand written by TMA with KB-byte swizzle (KB = 128,
// 64 or 32): rows of KB bytes, 8-row atoms 8*KB bytes apart, layout type 2
// (SWIZZLE_128B), 4 (SWIZZLE_64B) or 6 (SWIZZLE_32B).  Tile base aligned to the
// atom (8*KB bytes).
template <int KB>
__device__ __forceinline__ uint64_t smem_desc_kmajor(uint32_t smem_addr) {
    static_assert(KB == 128 || KB == 64 || KB == 32, "swizzle width");
    constexpr uint64_t layout = KB == 128 ? 2 : KB == 64 ? 4 : 6;
    uint64_t d = 0;
    d |= static_cast<uint64_t>((smem_addr & 0x3FFFFu) >> 4);
    d |= static_cast<uint64_t>(1) << 16;
    d |= static_cast<uint64_t>((8 * KB) >> 4) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    d |= layout << 61;
    return d;
}
// Instruction descriptor, kind::i8: s32 accumulator, unsigned 8-bit A and B,
// both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_u8(uint32_t M, uint32_t N) {
    return (2u << 4) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

}  // namespace hme

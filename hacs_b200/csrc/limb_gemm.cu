// The INT8-limb tcgen05 mod-p GEMM: C op= A*B mod p, u32 residues, p < 2^32.
//
// Reference semantics: engine::kernels::gemm<uint32_t> (src/ModArithmetic/
// Kernels.h:178-185, Kernels.cpp:1418-1483) and its device twin
// engine::cuda::gemm (src/Cuda/cuda_kernels.cu:195-299, 474-519): the exact sum
// of k products reduced to the canonical residue, combined by Set/Add/Sub.
//
// Method.  Write a = sum_i a_i 256^i with unsigned bytes a_i (i < L).  Then
//     A*B = sum_i a_i * B^(i)  (mod p),   B^(i) = 256^i * B mod p,
// and with B^(i) = sum_j b^(i)_j 256^j:
//     A*B = sum_j 256^j D_j (mod p),      D_j = sum_i a_i * b^(i)_j.
// D_j is a plain u8 x u8 -> s32 GEMM over the virtual K' = L*K; for fixed
// output columns the L matrices D_j sit side by side in one accumulator of
// L*BN columns, so a CTA runs ONE integer GEMM of 128 x (L*BN) x (L*K) on the
// tensor cores (tcgen05.mma kind::i8, M=128, N=L*BN, K=32 per instruction),
// then recombines sum_j 256^j D_j in u64 and reduces once (Barrett, the
// ModCtx<uint32_t>::reduce_u64 rule).  Exactness: every D_j is a sum of at
// most L*K_chunk products below 255^2, and K is cut into chunks with
// L * 255^2 * K_chunk < 2^31 (later chunks accumulate with Add).
//
// Layout in HBM (workspace): A limb planes [i][m][k] (L x M x Kp bytes) and
// B planes [i][j][n][k] (L x L x N x Kp bytes), K contiguous (K-major for both
// tensor-core operands), Kp = K rounded up to 16 bytes for TMA strides.
//
// Kernel: persistent, one CTA per SM, 10 warps: warp 0 issues TMA loads
// (128-byte swizzle, each CTA loads its own tiles), warp 1 owns tensor memory and issues the
// MMAs, warps 2-9 (two per TMEM lane quarter, alternate 16-column chunks)
// drain the double-buffered accumulator (2 x L*BN columns of
// TMEM) into C while the next tile's MMAs run.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "hme_internal.h"
#include "hme_limb.cuh"
#include "hme_ptx.cuh"

namespace hme {
namespace {

using namespace limb;

struct GemmArgs {
    uint32_t* C;
    uint64_t ldc;
    int M, N;
    int k_begin;  // first k of this chunk (multiple of kBK)
    int kblocks;  // k-blocks of kBK bytes in this chunk
    int op;
    uint32_t p;
    uint64_t barrett;
    int tiles_m, tiles_n, group_m;
    int* err;
};

__device__ __forceinline__ void tile_coords(int tile, const GemmArgs& g, int& tm, int& tn) {
    // Grouped raster: group_m tile-rows share the B tiles they stream, so a
    // wave of CTAs re-reads each K-slice of A and B from L2, not HBM.
    const int per_group = g.group_m * g.tiles_n;
    const int grp = tile / per_group;
    const int first_m = grp * g.group_m;
    const int gm = min(g.tiles_m - first_m, g.group_m);
    const int local = tile - grp * per_group;
    tm = first_m + local % gm;
    tn = local / gm;
}

// Time-bounded wait that ignores the abort flag: used while tearing down, to
// let in-flight copies and MMAs land before shared / tensor memory is released.
__device__ __forceinline__ void drain_wait(uint64_t* bar, uint32_t parity, int* err) {
    int never = 0;
    mbar_wait(bar, parity, &never, err, DERR_WAIT_DRAIN);
}

template <int L, int BN, int KB = kBK>
__global__ void __launch_bounds__(kThreads, 1)
    limb_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     const GemmArgs g) {
    using CF = Cfg<L, BN, KB>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = smem;
    uint8_t* sB = smem + CF::STAGES * CF::A_BYTES;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + CF::STAGES * CF::STAGE_BYTES);
    uint64_t* empty = full + CF::STAGES;
    uint64_t* acc_full = empty + CF::STAGES;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* drain = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    uint32_t* epi_stage = reinterpret_cast<uint32_t*>(smem + CF::STAGES * CF::STAGE_BYTES + CF::BAR_BYTES);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int total_tiles = g.tiles_m * g.tiles_n;

    if (threadIdx.x == 0) {
        for (int s = 0; s < CF::STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], 32 * kEpiWarps);
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        fence_mbar_init();
        fence_proxy_async_smem();
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, CF::TMEM_COLS);
        tmem_relinquish();
    }
    if (warp == 0 && lane == 0) {
        prefetch_tmap(&tmA);
        prefetch_tmap(&tmB);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    // the set-up above overlaps the tail of the limb split when this grid is a
    // programmatic dependent of it; the planes are read only after this point
    grid_dep_wait();

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            int it = 0;
            bool ok = true;
            for (int tile = blockIdx.x; ok && tile < total_tiles; tile += gridDim.x) {
                int tm, tn;
                tile_coords(tile, g, tm, tn);
                for (int i = 0; ok && i < L; ++i) {
                    for (int kb = 0; kb < g.kblocks; ++kb, ++it) {
                        const int s = it % CF::STAGES;
                        const uint32_t ph = (it / CF::STAGES) & 1;
                        if (!mbar_wait(&empty[s], ph ^ 1, abort_flag, g.err, DERR_WAIT_EMPTY)) {
                            ok = false;
                            break;
                        }
                        mbar_arrive_expect_tx(&full[s], CF::STAGE_BYTES);
                        const int kx = g.k_begin + kb * KB;
                        tma_load_3d(sA + s * CF::A_BYTES, &tmA, &full[s], kx, tm * kBM, i);
                        tma_load_4d(sB + s * CF::B_BYTES, &tmB, &full[s], kx, tn * BN, 0, i);
                    }
                }
            }
            if (!ok) {
                // let every copy issued into shared memory land before the CTA exits
                for (int t = max(0, it - CF::STAGES); t < it; ++t)
                    drain_wait(&full[t % CF::STAGES], (t / CF::STAGES) & 1, g.err);
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int it = 0, lt = 0;
            bool ok = true, issued_any = false;
            for (int tile = blockIdx.x; ok && tile < total_tiles; tile += gridDim.x, ++lt) {
                const int a = lt & 1;
                const uint32_t aph = (lt >> 1) & 1;
                if (!mbar_wait(&acc_empty[a], aph ^ 1, abort_flag, g.err, DERR_WAIT_ACCUM_FREE)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem_base + a * CF::ACC_STRIDE;
                for (int i = 0; ok && i < L; ++i) {
                    for (int kb = 0; kb < g.kblocks; ++kb, ++it) {
                        const int s = it % CF::STAGES;
                        const uint32_t ph = (it / CF::STAGES) & 1;
                        if (!mbar_wait(&full[s], ph, abort_flag, g.err, DERR_WAIT_FULL)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint64_t adesc = smem_desc_kmajor<KB>(smem_u32(sA + s * CF::A_BYTES));
                        const uint64_t bdesc = smem_desc_kmajor<KB>(smem_u32(sB + s * CF::B_BYTES));
#pragma unroll
                        for (int kk = 0; kk < KB / 32; ++kk) {
                            // +32 bytes along K inside the swizzle atom = +2 in the 16-byte address field
                            mma_u8(d, adesc + 2 * kk, bdesc + 2 * kk, CF::IDESC, (i | kb | kk) != 0);
                        }
                        issued_any = true;
                        mma_commit(&empty[s]);
                    }
                }
                if (ok) mma_commit(&acc_full[a]);
            }
            if (!ok && issued_any) {
                mma_commit(drain);
                drain_wait(drain, 0, g.err);
            }
        }
    } else {
        // ---------------- epilogue: TMEM -> registers -> shared -> C ----------------
        // Each thread owns one accumulator row (its TMEM lane); the reduced
        // 16-column chunk goes through a per-warp shared-memory stage so that
        // C is read and written along rows: two rows x 64 contiguous bytes
        // per warp instruction instead of 32 rows x 16 bytes.
        const int q = warp & 3;  // the TMEM lane quarter this warp may read
        const uint32_t lane_base = static_cast<uint32_t>(q * 32) << 16;
        uint32_t (*stage)[17] = reinterpret_cast<uint32_t (*)[17]>(epi_stage + (warp - 2) * 32 * 17);
        const int chalf = (warp - 2) >> 2;  // the two warps of a lane quarter take alternate 16-column chunks
        const int half = lane >> 4, col_in = lane & 15;
        // Add / Sub read C: each lane prefetches its row of this warp's quarter of
        // a tile into L2 one tile ahead (the first tile before its accumulator is
        // ready), so the old values come from L2 when the drain reads them
        auto prefetch_tile = [&](int t) {
            if (g.op == HME_SET || t >= total_tiles) return;
            int qm, qn;
            tile_coords(t, g, qm, qn);
            const int row = qm * kBM + q * 32 + lane;
            if (chalf == 0 && row < g.M) prefetch_l2_span(g.C + static_cast<size_t>(row) * g.ldc + qn * BN, min(BN, g.N - qn * BN));
        };
        prefetch_tile(blockIdx.x);
        int lt = 0;
        for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x, ++lt) {
            prefetch_tile(tile + gridDim.x);
            const int a = lt & 1;
            const uint32_t aph = (lt >> 1) & 1;
            if (!mbar_wait(&acc_full[a], aph, abort_flag, g.err, DERR_WAIT_ACCUM)) break;
            tc_fence_after();
            int tm, tn;
            tile_coords(tile, g, tm, tn);
            const int row0 = tm * kBM + q * 32;
#pragma unroll 1
            for (int c0 = 16 * chalf; c0 < BN; c0 += 32) {
                uint32_t v[L][16];
#pragma unroll
                for (int j = 0; j < L; ++j)
                    tmem_ld16(tmem_base + lane_base + a * CF::ACC_STRIDE + j * BN + c0, v[j]);
                tmem_wait_ld();
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    uint64_t s = v[0][e];
                    if (L > 1) s += static_cast<uint64_t>(v[L > 1 ? 1 : 0][e]) << 8;
                    if (L > 2) s += static_cast<uint64_t>(v[L > 2 ? 2 : 0][e]) << 16;
                    if (L > 3) s += static_cast<uint64_t>(v[L > 3 ? 3 : 0][e]) << 24;
                    stage[lane][e] = reduce_u64(s, g.p, g.barrett);
                }
                __syncwarp();
                const int col = tn * BN + c0 + col_in;
                if (col < g.N) {
                    // all 16 rows' C values in flight at once, then combine and store
                    const int rlim = min(32, g.M - row0);
                    uint32_t old[16];
                    if (g.op != HME_SET) {
#pragma unroll
                        for (int t = 0; t < 16; ++t) {
                            const int rr = half + 2 * t;
                            old[t] = rr < rlim ? g.C[static_cast<size_t>(row0 + rr) * g.ldc + col] : 0u;
                        }
                    }
#pragma unroll
                    for (int t = 0; t < 16; ++t) {
                        const int rr = half + 2 * t;
                        if (rr >= rlim) break;
                        uint32_t o = stage[rr][col_in];
                        if (g.op == HME_ADD) o = mod_add(old[t], o, g.p);
                        else if (g.op == HME_SUB) o = mod_sub(old[t], o, g.p);
                        g.C[static_cast<size_t>(row0 + rr) * g.ldc + col] = o;
                    }
                }
                __syncwarp();
            }
            tc_fence_before();
            mbar_arrive(&acc_empty[a]);
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, CF::TMEM_COLS);
    }
}

template <int L>
__global__ void __launch_bounds__(256) limb_split_kernel(const SplitArgs s) {
    __shared__ uint32_t tile[64][33];
    grid_dep_launch();  // the GEMM that follows may start its set-up
    if (static_cast<int>(blockIdx.x) < s.a_blocks)
        split_a_part<L>(s, blockIdx.x);
    else
        split_b_part<L>(s, blockIdx.x - s.a_blocks, tile);
}

// ---- host side ---------------------------------------------------------------------
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    if (!fn) throw Error(HME_ECUDA, "cuTensorMapEncodeTiled is not available from the driver");
    return fn;
}

void encode_u8(CUtensorMap* map, void* base, int rank, const cuuint64_t* dims, const cuuint64_t* strides,
               const cuuint32_t* box, int kb = 128) {
    cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const CUtensorMapSwizzle sw = kb == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                                  : kb == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                                             : CU_TENSOR_MAP_SWIZZLE_32B;
    if (kb != 128 && kb != 64 && kb != 32) throw Error(HME_EINVAL, "tensor map: k-block must be 128, 64 or 32 bytes");
    const CUresult r = encode_fn()(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, rank, base, dims, strides, box, estr,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(HME_ECUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(r) + ")");
}

// a_plane: bytes between consecutive A limb planes (M * Kp for planes of
// exactly these m rows; larger when the m rows are a slice of taller planes).
// pdl: the launch directly follows the limb split on the same stream, so the
// first K chunk may be a programmatic dependent of it (off while per-kernel
// timing events sit between launches).
template <int L, int BN, int KB = kBK>
void launch_gemm(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k, int Kp,
                 uint8_t* planesA, uint64_t a_plane, uint8_t* planesB, uint32_t* C, size_t ldc, int op,
                 bool pdl) {
    using CF = Cfg<L, BN, KB>;
    static OncePerDevice attr;
    attr.run([](int) {
        HME_CUDA(cudaFuncSetAttribute(limb_gemm_kernel<L, BN, KB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      CF::SMEM));
    });
    CUtensorMap tmA, tmB;
    {
        const cuuint64_t dims[3] = {static_cast<cuuint64_t>(Kp), m, static_cast<cuuint64_t>(L)};
        const cuuint64_t strides[2] = {static_cast<cuuint64_t>(Kp), static_cast<cuuint64_t>(a_plane)};
        const cuuint32_t box[3] = {KB, kBM, 1};
        encode_u8(&tmA, planesA, 3, dims, strides, box, KB);
    }
    {
        const cuuint64_t dims[4] = {static_cast<cuuint64_t>(Kp), n, static_cast<cuuint64_t>(L),
                                    static_cast<cuuint64_t>(L)};
        const cuuint64_t strides[3] = {static_cast<cuuint64_t>(Kp), static_cast<cuuint64_t>(Kp) * n,
                                       static_cast<cuuint64_t>(Kp) * n * L};
        const cuuint32_t box[4] = {KB, BN, static_cast<cuuint32_t>(L), 1};
        encode_u8(&tmB, planesB, 4, dims, strides, box, KB);
    }
    GemmArgs g{};
    g.C = C;
    g.ldc = ldc;
    g.M = static_cast<int>(m);
    g.N = static_cast<int>(n);
    g.p = mp.p;
    g.barrett = mp.barrett;
    g.tiles_m = static_cast<int>((m + kBM - 1) / kBM);
    g.tiles_n = static_cast<int>((n + BN - 1) / BN);
    g.group_m = 16;
    g.err = ctx->d_err;
    const int total = g.tiles_m * g.tiles_n;
    const int grid = std::min(total, ctx->gemm_sm_cap > 0 ? std::min(ctx->gemm_sm_cap, ctx->num_sms) : ctx->num_sms);
    const uint32_t chunk = limb_k_chunk(L);
    for (uint32_t kb0 = 0; kb0 < k; kb0 += chunk) {
        const uint32_t kc = std::min(chunk, k - kb0);
        g.k_begin = static_cast<int>(kb0);
        g.kblocks = static_cast<int>((kc + KB - 1) / KB);
        g.op = kb0 == 0 ? op : (op == HME_SET ? HME_ADD : op);
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = CF::SMEM;
        cfg.stream = ctx->stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = (pdl && kb0 == 0 && !ctx->timer.on) ? 1 : 0;
        HME_TIMED(ctx, "limb_gemm", HME_CUDA(cudaLaunchKernelEx(&cfg, limb_gemm_kernel<L, BN, KB>, tmA, tmB, g)));
    }
}

__global__ void fill_zero_kernel(uint32_t* C, uint64_t ldc, int m, int n) {
    const size_t total = static_cast<size_t>(m) * n;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        C[(i / n) * ldc + (i % n)] = 0;
}

}  // namespace

void encode_tma_u8(CUtensorMap* map, void* base, int rank, const cuuint64_t* dims, const cuuint64_t* strides,
                   const cuuint32_t* box) {
    encode_u8(map, base, rank, dims, strides, box);
}
void encode_tma_u8_kb(CUtensorMap* map, void* base, int rank, const cuuint64_t* dims, const cuuint64_t* strides,
                      const cuuint32_t* box, int kb) {
    encode_u8(map, base, rank, dims, strides, box, kb);
}

namespace {

// Limb split of A (m rows, when do_a) and/or B (n columns, when do_b) in one launch.
// a_plane: bytes between A limb planes (0: m * Kp).
void launch_split(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k, int Kp, const uint32_t* A,
                  size_t lda, const uint32_t* B, size_t ldb, uint8_t* pa, uint64_t a_plane, uint8_t* pb, bool do_a,
                  bool do_b) {
    SplitArgs sa{};
    sa.A = A; sa.lda = lda; sa.B = B; sa.ldb = ldb;
    sa.M = static_cast<int>(m); sa.N = static_cast<int>(n); sa.K = static_cast<int>(k); sa.Kp = Kp;
    sa.p = mp.p; sa.barrett = mp.barrett;
    sa.planesA = pa; sa.planesB = pb;
    sa.a_plane = a_plane;
    const size_t work = static_cast<size_t>(m) * (Kp / 16);
    sa.a_blocks = do_a ? static_cast<int>(std::min<size_t>((work + 255) / 256, static_cast<size_t>(ctx->num_sms) * 8))
                       : 0;
    sa.b_blocks_k = (Kp + 63) / 64;
    sa.a_vec = do_a && ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && ((lda & 3) == 0);
    const int grid = sa.a_blocks + (do_b ? sa.b_blocks_k * static_cast<int>((n + 31) / 32) : 0);
    if (grid == 0) return;
    switch (mp.limbs) {
        case 1: HME_TIMED(ctx, "limb_split", limb_split_kernel<1><<<grid, 256, 0, ctx->stream>>>(sa)); break;
        case 2: HME_TIMED(ctx, "limb_split", limb_split_kernel<2><<<grid, 256, 0, ctx->stream>>>(sa)); break;
        case 3: HME_TIMED(ctx, "limb_split", limb_split_kernel<3><<<grid, 256, 0, ctx->stream>>>(sa)); break;
        default: HME_TIMED(ctx, "limb_split", limb_split_kernel<4><<<grid, 256, 0, ctx->stream>>>(sa)); break;
    }
    HME_CUDA(cudaGetLastError());
}

// kb: the k-block (swizzle row) width the planes were padded to: 32, 64 or 128
template <int KB>
void launch_gemm_variant_kb(hme_ctx* ctx, const ModParams& mp, bool narrow, uint32_t m, uint32_t n, uint32_t k,
                            int Kp, uint8_t* pa, uint64_t a_plane, uint8_t* pb, uint32_t* C, size_t ldc, int op,
                            bool pdl) {
    switch (mp.limbs) {
        case 1: if (narrow) launch_gemm<1, 128, KB>(ctx, mp, m, n, k, Kp, pa, a_plane, pb, C, ldc, op, pdl);
                else launch_gemm<1, 256, KB>(ctx, mp, m, n, k, Kp, pa, a_plane, pb, C, ldc, op, pdl); break;
        case 2: if (narrow) launch_gemm<2, 64, KB>(ctx, mp, m, n, k, Kp, pa, a_plane, pb, C, ldc, op, pdl);
                else launch_gemm<2, 128, KB>(ctx, mp, m, n, k, Kp, pa, a_plane, pb, C, ldc, op, pdl); break;
        case 3: if (narrow) launch_gemm<3, 32, KB>(ctx, mp, m, n, k, Kp, pa, a_plane, pb, C, ldc, op, pdl);
                else launch_gemm<3, 80, KB>(ctx, mp, m, n, k, Kp, pa, a_plane, pb, C, ldc, op, pdl); break;
        default: if (narrow) launch_gemm<4, 32, KB>(ctx, mp, m, n, k, Kp, pa, a_plane, pb, C, ldc, op, pdl);
                else launch_gemm<4, 64, KB>(ctx, mp, m, n, k, Kp, pa, a_plane, pb, C, ldc, op, pdl); break;
    }
}

// The narrowest k-block that holds K (products with a short K, like the
// elimination's trailing updates with K = the panel's pivots, stream and
// multiply no zero padding); longer K use the 128-byte row.
int kblock_for(uint32_t k) { return k <= 32 ? 32 : k <= 64 ? 64 : kBK; }

void launch_gemm_variant(hme_ctx* ctx, const ModParams& mp, bool narrow, uint32_t m, uint32_t n, uint32_t k, int Kp,
                         uint8_t* pa, uint64_t a_plane, uint8_t* pb, uint32_t* C, size_t ldc, int op, bool pdl) {
    switch (kblock_for(k)) {
        case 32: launch_gemm_variant_kb<32>(ctx, mp, narrow, m, n, k, Kp, pa, a_plane, pb, C, ldc, op, pdl); break;
        case 64: launch_gemm_variant_kb<64>(ctx, mp, narrow, m, n, k, Kp, pa, a_plane, pb, C, ldc, op, pdl); break;
        default: launch_gemm_variant_kb<kBK>(ctx, mp, narrow, m, n, k, Kp, pa, a_plane, pb, C, ldc, op, pdl); break;
    }
}

}  // namespace

int gemm_default_variant(const hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n) {
    // Wide tiles (L*BN = 256 columns of TMEM per accumulator) unless that leaves
    // SMs idle; then half-width tiles, which double the tile count.
    const uint32_t L = mp.limbs;
    const uint32_t tiles_m = (m + kBM - 1) / kBM;
    const uint32_t bn = 256 / L > 64 ? 256 / L : 64;
    const size_t tiles = static_cast<size_t>(tiles_m) * ((n + bn - 1) / bn);
    return 4 * tiles < 3 * static_cast<size_t>(ctx->num_sms) ? kVariantNarrow : kVariantWide;
}

int limb_kp(uint32_t k) { return static_cast<int>((k + kblock_for(k) - 1) / kblock_for(k) * kblock_for(k)); }

void gemm_u32_planes(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k, int Kp, uint8_t* pa,
                     uint64_t a_plane, uint8_t* pb, uint32_t* C, size_t ldc, int op) {
    const bool narrow = gemm_default_variant(ctx, mp, m, n) == kVariantNarrow;
    launch_gemm_variant(ctx, mp, narrow, m, n, k, Kp, pa, a_plane, pb, C, ldc, op, true);
}

void gemm_u32_device(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A,
                     size_t lda, const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc, int op) {
    int v = ctx->fixed_variant;
    if (v < 0) v = sched_variant(ctx, mp, m, n, k);
    gemm_u32_variant(ctx, mp, m, n, k, A, lda, B, ldb, C, ldc, op, v);
}

void gemm_u32_variant(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A,
                      size_t lda, const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc, int op, int variant) {
    HME_REQUIRE(op == HME_SET || op == HME_ADD || op == HME_SUB, "gemm: op must be HME_SET, HME_ADD or HME_SUB");
    HME_REQUIRE(variant >= 0 && variant < kGemmVariants, "gemm: unknown variant");
    HME_REQUIRE(mp.p >= 2, "gemm: modulus must be >= 2");
    HME_REQUIRE(m < (1u << 30) && n < (1u << 30) && k < (1u << 30), "gemm: dimension too large");
    if (m == 0 || n == 0) return;
    HME_REQUIRE(ldc >= n, "gemm: ldc < n");
    if (k == 0) {
        if (op == HME_SET) {
            HME_TIMED(ctx, "fill_zero",
                      fill_zero_kernel<<<std::min<size_t>(1024, (static_cast<size_t>(m) * n + 255) / 256), 256, 0,
                                         ctx->stream>>>(C, ldc, m, n));
            HME_CUDA(cudaGetLastError());
        }
        return;
    }
    HME_REQUIRE(A && B && C, "gemm: null pointer");
    HME_REQUIRE(lda >= k && ldb >= n, "gemm: leading dimension too small");
    if (variant == kVariantSimt32 || variant == kVariantSimt64) {
        simt_gemm_u32_device(ctx, mp, m, n, k, A, lda, B, ldb, C, ldc, op, variant == kVariantSimt32 ? 32 : 64);
        return;
    }
    const int L = static_cast<int>(mp.limbs);
    // K padded to whole k-blocks of the width kblock_for picks (the split kernel
    // writes the pad as zeros), so no TMA box ever reaches past the planes' K extent
    const int Kp = static_cast<int>((k + kblock_for(k) - 1) / kblock_for(k) * kblock_for(k));
    uint8_t* pa = static_cast<uint8_t*>(ctx->ws.get(kSlotPlanesA, static_cast<size_t>(L) * m * Kp));
    uint8_t* pb = static_cast<uint8_t*>(ctx->ws.get(kSlotPlanesB, static_cast<size_t>(L) * L * n * Kp));
    launch_split(ctx, mp, m, n, k, Kp, A, lda, B, ldb, pa, 0, pb, true, true);
    launch_gemm_variant(ctx, mp, variant == kVariantNarrow, m, n, k, Kp, pa, static_cast<uint64_t>(Kp) * m, pb, C,
                        ldc, op, true);
}

void gemm_u32_wrap_device(hme_ctx* ctx, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A, size_t lda,
                          const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc, int op) {
    HME_REQUIRE(op == HME_SET || op == HME_ADD || op == HME_SUB, "gemm: op must be HME_SET, HME_ADD or HME_SUB");
    HME_REQUIRE(m < (1u << 30) && n < (1u << 30) && k < (1u << 30), "gemm: dimension too large");
    if (m == 0 || n == 0) return;
    HME_REQUIRE(ldc >= n, "gemm: ldc < n");
    if (k == 0) {
        if (op == HME_SET) {
            HME_TIMED(ctx, "fill_zero",
                      fill_zero_kernel<<<std::min<size_t>(1024, (static_cast<size_t>(m) * n + 255) / 256), 256, 0,
                                         ctx->stream>>>(C, ldc, m, n));
            HME_CUDA(cudaGetLastError());
        }
        return;
    }
    HME_REQUIRE(A && B && C && lda >= k && ldb >= n, "gemm: bad operands");
    ModParams mp;  // p = 0, m = 0: every reduction is the truncation to 32 bits
    mp.p = 0;
    mp.limbs = 4;
    mp.barrett = 0;
    const int Kp = static_cast<int>((k + kblock_for(k) - 1) / kblock_for(k) * kblock_for(k));
    uint8_t* pa = static_cast<uint8_t*>(ctx->ws.get(kSlotPlanesA, static_cast<size_t>(4) * m * Kp));
    uint8_t* pb = static_cast<uint8_t*>(ctx->ws.get(kSlotPlanesB, static_cast<size_t>(16) * n * Kp));
    launch_split(ctx, mp, m, n, k, Kp, A, lda, B, ldb, pa, 0, pb, true, true);
    launch_gemm_variant(ctx, mp, gemm_default_variant(ctx, mp, m, n) == kVariantNarrow, m, n, k, Kp, pa,
                        static_cast<uint64_t>(Kp) * m, pb, C, ldc, op, true);
}

void gemm_u32_host(hme_ctx* ctx, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A,
                   size_t lda, const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc, int op, int variant) {
    // Pipeline over row chunks of A and C (multiples of the 128-row tile, 1 to
    // 8 chunks): B is copied and split first; then chunk i's rows of A
    // (and of C for Add/Sub) are copied on copy_in while chunk i-1 is split
    // and multiplied on the context stream and chunk i-2's rows of C go back on
    // copy_out.  The host<->device copies run in both directions at once and
    // hide the compute; what is left is the copy of B and one chunk's tail.
    HME_REQUIRE(variant == kVariantWide || variant == kVariantNarrow, "gemm_u32_host: tensor-core variants only");
    HME_REQUIRE(m > 0 && n > 0 && k > 0, "gemm_u32_host: empty product");
    const int L = static_cast<int>(mp.limbs);
    const int Kp = static_cast<int>((k + kblock_for(k) - 1) / kblock_for(k) * kblock_for(k));
    const uint32_t tiles_m = (m + kBM - 1) / kBM;
    // chunks of >= 2 MiB of C: every copy carries a fixed cost on the PCIe
    // path, so small chunks lose more than their overlap gains (measured on
    // B200: 1024^3 runs fastest with two chunks)
    const size_t c_bytes = sizeof(uint32_t) * static_cast<size_t>(m) * n;
    const uint32_t by_size = static_cast<uint32_t>(std::min<size_t>(8, std::max<size_t>(1, c_bytes >> 21)));
    const uint32_t chunks_max = std::min<uint32_t>(by_size, tiles_m);
    const uint32_t rows_per = (tiles_m + chunks_max - 1) / chunks_max * kBM;
    const int nc = static_cast<int>((m + rows_per - 1) / rows_per);

    uint32_t* dA = static_cast<uint32_t*>(ctx->ws.get(kSlotStageA, sizeof(uint32_t) * static_cast<size_t>(m) * k));
    uint32_t* dB = static_cast<uint32_t*>(ctx->ws.get(kSlotStageB, sizeof(uint32_t) * static_cast<size_t>(k) * n));
    uint32_t* dC = static_cast<uint32_t*>(ctx->ws.get(kSlotStageC, sizeof(uint32_t) * static_cast<size_t>(m) * n));
    uint8_t* pa = static_cast<uint8_t*>(ctx->ws.get(kSlotPlanesA, static_cast<size_t>(L) * m * Kp));
    uint8_t* pb = static_cast<uint8_t*>(ctx->ws.get(kSlotPlanesB, static_cast<size_t>(L) * L * n * Kp));

    if (!ctx->copy_in) HME_CUDA(cudaStreamCreateWithFlags(&ctx->copy_in, cudaStreamNonBlocking));
    if (!ctx->copy_out) HME_CUDA(cudaStreamCreateWithFlags(&ctx->copy_out, cudaStreamNonBlocking));
    const size_t nev = 2 * static_cast<size_t>(nc) + 3;
    while (ctx->pipe_ev.size() < nev) {
        cudaEvent_t e;
        HME_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->pipe_ev.push_back(e);
    }
    cudaEvent_t ev_start = ctx->pipe_ev[0], ev_b = ctx->pipe_ev[1], ev_out = ctx->pipe_ev[2];
    cudaEvent_t* ev_a = ctx->pipe_ev.data() + 3;
    cudaEvent_t* ev_c = ev_a + nc;
    const cudaStream_t s0 = ctx->stream;

    // the copies start after earlier work on the context stream (it may still use the staging buffers)
    HME_CUDA(cudaEventRecord(ev_start, s0));
    HME_CUDA(cudaStreamWaitEvent(ctx->copy_in, ev_start, 0));
    HME_CUDA(cudaStreamWaitEvent(ctx->copy_out, ev_start, 0));
    const size_t w = sizeof(uint32_t);
    HME_CUDA(copy_rows_async(dB, w * n, B, w * ldb, w * n, k, cudaMemcpyHostToDevice, ctx->copy_in));
    HME_CUDA(cudaEventRecord(ev_b, ctx->copy_in));
    for (int i = 0; i < nc; ++i) {
        const uint32_t r0 = static_cast<uint32_t>(i) * rows_per, mc = std::min(rows_per, m - r0);
        HME_CUDA(copy_rows_async(dA + static_cast<size_t>(r0) * k, w * k, A + static_cast<size_t>(r0) * lda,
                                   w * lda, w * k, mc, cudaMemcpyHostToDevice, ctx->copy_in));
        if (op != HME_SET)
            HME_CUDA(copy_rows_async(dC + static_cast<size_t>(r0) * n, w * n, C + static_cast<size_t>(r0) * ldc,
                                       w * ldc, w * n, mc, cudaMemcpyHostToDevice, ctx->copy_in));
        HME_CUDA(cudaEventRecord(ev_a[i], ctx->copy_in));
    }
    HME_CUDA(cudaStreamWaitEvent(s0, ev_b, 0));
    launch_split(ctx, mp, 0, n, k, Kp, nullptr, 0, dB, n, nullptr, 0, pb, false, true);
    const uint64_t a_plane = static_cast<uint64_t>(Kp) * m;
    for (int i = 0; i < nc; ++i) {
        const uint32_t r0 = static_cast<uint32_t>(i) * rows_per, mc = std::min(rows_per, m - r0);
        HME_CUDA(cudaStreamWaitEvent(s0, ev_a[i], 0));
        uint8_t* pa_i = pa + static_cast<size_t>(r0) * Kp;
        launch_split(ctx, mp, mc, 0, k, Kp, dA + static_cast<size_t>(r0) * k, k, nullptr, 0, pa_i, a_plane, nullptr,
                     true, false);
        const bool narrow = ctx->fixed_variant >= 0 ? variant == kVariantNarrow
                                                    : gemm_default_variant(ctx, mp, mc, n) == kVariantNarrow;
        launch_gemm_variant(ctx, mp, narrow, mc, n, k, Kp, pa_i, a_plane, pb, dC + static_cast<size_t>(r0) * n, n,
                            op, true);
        HME_CUDA(cudaEventRecord(ev_c[i], s0));
        // enqueued right behind the chunk's GEMM, so the copy back starts as soon as the chunk is done
        HME_CUDA(cudaStreamWaitEvent(ctx->copy_out, ev_c[i], 0));
        HME_CUDA(copy_rows_async(C + static_cast<size_t>(r0) * ldc, w * ldc, dC + static_cast<size_t>(r0) * n, w * n,
                                   w * n, mc, cudaMemcpyDeviceToHost, ctx->copy_out));
    }
    HME_CUDA(cudaEventRecord(ev_out, ctx->copy_out));
    HME_CUDA(cudaStreamWaitEvent(s0, ev_out, 0));
}

}  // namespace hme

// ---- allocation-free GEMM entry point ---------------------------------------------
//
// Some callers cannot allocate device memory at the point where they need a
// GEMM: a plugin running inside another runtime that owns the whole device
// budget and forbids allocations after start-up, or a latency-critical path
// where cudaMalloc / cudaFree would synchronise the device.  For them,
// hme_gemm_u32_dev_noalloc runs the same limb-split and limb-GEMM kernels as
// hme_gemm_u32_dev, with the limb planes in a fixed scratch array that lives
// in this library's device image (held by every GPU that loads the library,
// until the process exits), and with no context.  It never calls cudaMalloc,
// cudaFree or any allocating routine.
//
// Limits and sharing: the planes of one call (L*m*Kp + L*L*n*Kp bytes, each
// rounded up to 256, Kp = k rounded up to 16) must fit the 32 MiB array, else
// the call fails with HME_EINVAL before launching anything.  Every call on a
// device shares the one array and leaves its planes behind; each call writes
// all plane bytes it reads before reading them, and clears the device error
// word it uses at its start.  Calls that overlap on the GPU (on different
// streams, or from several host threads at once) race on the array and give
// wrong results: serialise them.
namespace hme {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];
static __device__ int g_noalloc_err;

struct NoAllocDevice {
    bool ready = false;
    uint8_t* scratch = nullptr;  // device address of g_noalloc_scratch on this device
    int* err = nullptr;          // device address of g_noalloc_err on this device
    int num_sms = 0;
};
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];

template <int L, int BN>
void noalloc_smem_attr() {
    HME_CUDA(cudaFuncSetAttribute(limb_gemm_kernel<L, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  Cfg<L, BN>::SMEM));
}

// Once per device, with that device current: resolve the device addresses of
// the scratch array and the error word (the host-side names of __device__
// variables are not device addresses) and set the kernels' shared-memory limit.
const NoAllocDevice& noalloc_setup(int dev) {
    HME_REQUIRE(dev >= 0 && dev < kNoAllocMaxDevices, "hme_gemm_u32_dev_noalloc: device id out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoAllocDevice& d = g_noalloc_dev[dev];
    if (d.ready) return d;
    void* ptr = nullptr;
    HME_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    d.scratch = static_cast<uint8_t*>(ptr);
    ptr = nullptr;
    HME_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_err));
    d.err = static_cast<int*>(ptr);
    HME_CUDA(cudaDeviceGetAttribute(&d.num_sms, cudaDevAttrMultiProcessorCount, dev));
    noalloc_smem_attr<1, 128>(); noalloc_smem_attr<1, 256>();
    noalloc_smem_attr<2, 64>();  noalloc_smem_attr<2, 128>();
    noalloc_smem_attr<3, 32>();  noalloc_smem_attr<3, 80>();
    noalloc_smem_attr<4, 32>();  noalloc_smem_attr<4, 64>();
    d.ready = true;
    return d;
}

template <int L, int BN>
void noalloc_gemm(const NoAllocDevice& d, cudaStream_t st, const ModParams& mp, uint32_t m, uint32_t n, uint32_t k,
                  int Kp, uint8_t* pa, uint8_t* pb, uint32_t* C, size_t ldc, int op) {
    using CF = Cfg<L, BN>;
    CUtensorMap tmA, tmB;
    {
        const cuuint64_t dims[3] = {k, m, static_cast<cuuint64_t>(L)};
        const cuuint64_t strides[2] = {static_cast<cuuint64_t>(Kp), static_cast<cuuint64_t>(Kp) * m};
        const cuuint32_t box[3] = {kBK, kBM, 1};
        encode_u8(&tmA, pa, 3, dims, strides, box);
    }
    {
        const cuuint64_t dims[4] = {k, n, static_cast<cuuint64_t>(L), static_cast<cuuint64_t>(L)};
        const cuuint64_t strides[3] = {static_cast<cuuint64_t>(Kp), static_cast<cuuint64_t>(Kp) * n,
                                       static_cast<cuuint64_t>(Kp) * n * L};
        const cuuint32_t box[4] = {kBK, BN, static_cast<cuuint32_t>(L), 1};
        encode_u8(&tmB, pb, 4, dims, strides, box);
    }
    GemmArgs g{};
    g.C = C;
    g.ldc = ldc;
    g.M = static_cast<int>(m);
    g.N = static_cast<int>(n);
    g.p = mp.p;
    g.barrett = mp.barrett;
    g.tiles_m = static_cast<int>((m + kBM - 1) / kBM);
    g.tiles_n = static_cast<int>((n + BN - 1) / BN);
    g.group_m = 16;
    g.err = d.err;
    const int grid = std::min(g.tiles_m * g.tiles_n, d.num_sms);
    const uint32_t chunk = limb_k_chunk(L);
    for (uint32_t kb0 = 0; kb0 < k; kb0 += chunk) {
        const uint32_t kc = std::min(chunk, k - kb0);
        g.k_begin = static_cast<int>(kb0);
        g.kblocks = static_cast<int>((kc + kBK - 1) / kBK);
        g.op = kb0 == 0 ? op : (op == HME_SET ? HME_ADD : op);
        limb_gemm_kernel<L, BN><<<grid, kThreads, CF::SMEM, st>>>(tmA, tmB, g);
        HME_CUDA(cudaGetLastError());
    }
}

size_t round256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace
}  // namespace hme

extern "C" HME_API int hme_gemm_u32_dev_noalloc(uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A,
                                                size_t lda, const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc,
                                                int op, void* cuda_stream) {
    using namespace hme;
    try {
        HME_REQUIRE(op == HME_SET || op == HME_ADD || op == HME_SUB, "gemm: op must be HME_SET, HME_ADD or HME_SUB");
        HME_REQUIRE(p >= 2, "gemm: modulus must be >= 2");
        HME_REQUIRE(m < (1u << 30) && n < (1u << 30) && k < (1u << 30), "gemm: dimension too large");
        const ModParams mp = make_mod(p);
        const int L = static_cast<int>(mp.limbs);
        const size_t Kp = (static_cast<size_t>(k) + 15) / 16 * 16;
        const size_t bytes_a = round256(static_cast<size_t>(L) * m * Kp);
        const size_t need = bytes_a + round256(static_cast<size_t>(L) * L * n * Kp);
        if (need > kNoAllocScratchBytes)
            throw Error(HME_EINVAL, "hme_gemm_u32_dev_noalloc: this GEMM needs " + std::to_string(need) +
                                        " bytes of limb planes; the allocation-free entry point holds " +
                                        std::to_string(kNoAllocScratchBytes) +
                                        " (32 MiB). Use hme_gemm_u32_dev for larger products.");
        if (m == 0 || n == 0) return HME_OK;
        HME_REQUIRE(C != nullptr && ldc >= n, "gemm: bad C");
        HME_REQUIRE(k == 0 || (A && B && lda >= k && ldb >= n), "gemm: bad A/B");
        cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
        {
            // the call waits for its stream and reads the error word back: neither may happen inside a capture
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            const cudaError_t e = cudaStreamIsCapturing(st, &cs);
            if (e != cudaSuccess) cudaGetLastError();
            HME_REQUIRE(e == cudaSuccess && cs == cudaStreamCaptureStatusNone,
                        "hme_gemm_u32_dev_noalloc: cannot be called while a stream capture is in progress (it "
                        "synchronises its stream)");
        }
        int dev = 0;
        HME_CUDA(cudaGetDevice(&dev));
        const NoAllocDevice& d = noalloc_setup(dev);
        HME_CUDA(cudaMemsetAsync(d.err, 0, sizeof(int), st));
        if (k == 0) {
            if (op == HME_SET)
                fill_zero_kernel<<<std::min<size_t>(1024, (static_cast<size_t>(m) * n + 255) / 256), 256, 0, st>>>(
                    C, ldc, m, n);
            HME_CUDA(cudaGetLastError());
            HME_CUDA(cudaStreamSynchronize(st));
            return HME_OK;
        }
        uint8_t* pa = d.scratch;
        uint8_t* pb = d.scratch + bytes_a;
        SplitArgs sa{};
        sa.A = A; sa.lda = lda; sa.B = B; sa.ldb = ldb;
        sa.M = static_cast<int>(m); sa.N = static_cast<int>(n); sa.K = static_cast<int>(k);
        sa.Kp = static_cast<int>(Kp);
        sa.p = mp.p; sa.barrett = mp.barrett;
        sa.planesA = pa; sa.planesB = pb;
        const size_t work = static_cast<size_t>(m) * (Kp / 16);
        sa.a_blocks = static_cast<int>(std::min<size_t>((work + 255) / 256, static_cast<size_t>(d.num_sms) * 8));
        sa.b_blocks_k = static_cast<int>((Kp + 63) / 64);
        sa.a_vec = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && ((lda & 3) == 0);
        const int grid = sa.a_blocks + sa.b_blocks_k * static_cast<int>((n + 31) / 32);
        const uint32_t tiles_m = (m + kBM - 1) / kBM;
        auto tiles_for = [&](uint32_t bn) { return static_cast<size_t>(tiles_m) * ((n + bn - 1) / bn); };
        const bool narrow = 4 * tiles_for(256 / L > 64 ? 256 / L : 64) < 3 * static_cast<size_t>(d.num_sms);
        const int kpi = static_cast<int>(Kp);
        switch (L) {
            case 1:
                limb_split_kernel<1><<<grid, 256, 0, st>>>(sa);
                if (narrow) noalloc_gemm<1, 128>(d, st, mp, m, n, k, kpi, pa, pb, C, ldc, op);
                else noalloc_gemm<1, 256>(d, st, mp, m, n, k, kpi, pa, pb, C, ldc, op);
                break;
            case 2:
                limb_split_kernel<2><<<grid, 256, 0, st>>>(sa);
                if (narrow) noalloc_gemm<2, 64>(d, st, mp, m, n, k, kpi, pa, pb, C, ldc, op);
                else noalloc_gemm<2, 128>(d, st, mp, m, n, k, kpi, pa, pb, C, ldc, op);
                break;
            case 3:
                limb_split_kernel<3><<<grid, 256, 0, st>>>(sa);
                if (narrow) noalloc_gemm<3, 32>(d, st, mp, m, n, k, kpi, pa, pb, C, ldc, op);
                else noalloc_gemm<3, 80>(d, st, mp, m, n, k, kpi, pa, pb, C, ldc, op);
                break;
            default:
                limb_split_kernel<4><<<grid, 256, 0, st>>>(sa);
                if (narrow) noalloc_gemm<4, 32>(d, st, mp, m, n, k, kpi, pa, pb, C, ldc, op);
                else noalloc_gemm<4, 64>(d, st, mp, m, n, k, kpi, pa, pb, C, ldc, op);
                break;
        }
        HME_CUDA(cudaGetLastError());
        HME_CUDA(cudaStreamSynchronize(st));
        int code = 0;
        HME_CUDA(cudaMemcpyFromSymbol(&code, g_noalloc_err, sizeof(int)));
        if (code != 0)
            throw Error(HME_ETIMEOUT, "hme_gemm_u32_dev_noalloc: a bounded device-side wait ran out (device code " +
                                          std::to_string(code) + "); C is incomplete");
        return HME_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return HME_EINVAL;
    }
}

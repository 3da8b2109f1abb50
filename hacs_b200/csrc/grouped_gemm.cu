// Grouped INT8-limb GEMM: many independent mod-p products of different shapes
// (C_j op= A_j * B_j mod p, one modulus per launch) in ONE persistent tcgen05
// launch, plus one launch that splits every operand into limb planes.
//
// The per-problem table lives in device memory: the TMA descriptors of each
// problem's planes (CUtensorMap objects in global memory), C, ldc, the shape
// and the op.  A CTA walks global tile indices; a per-tile table gives each
// tile's problem in one load (a search over thousands of problems would be a
// chain of dependent loads per tile, longer than a one-k-block tile's work).  Warp roles, pipeline, tensor-memory
// double buffer and epilogue are those of limb_gemm_kernel.  This is the
// batched path the reference lacks: its GemmBatch (src/Cuda/CudaKernels.h:
// 141-185, cuda_kernels.cu:831-946) runs one launch per SAME-shape batch, so
// uneven shapes each cost a launch.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "hme_grouped.h"
#include "hme_internal.h"
#include "hme_limb.cuh"
#include "hme_ptx.cuh"

namespace hme {
namespace {

using namespace limb;

__device__ __forceinline__ void grouped_drain(uint64_t* bar, uint32_t parity, int* err) {
    int never = 0;
    mbar_wait(bar, parity, &never, err, DERR_WAIT_DRAIN);
}

template <int L, int BN, int KB>
__global__ void __launch_bounds__(kThreads, 1)
    grouped_limb_gemm_kernel(const GroupedProblem* __restrict__ probs, const int* __restrict__ tile_prob,
                             int total_tiles_arg, const int* __restrict__ d_total, uint32_t p, uint64_t barrett,
                             int* err) {
    // the tile count: a launch argument, or read from device memory (tables built on the device)
    const int total_tiles = d_total ? *d_total : total_tiles_arg;
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
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            int it = 0;
            bool ok = true;
            for (int tile = blockIdx.x; ok && tile < total_tiles; tile += gridDim.x) {
                const int pi = tile_prob[tile];
                const GroupedProblem& P = probs[pi];
                const int local = tile - P.tile_begin;
                const int tm = local / P.tiles_n, tn = local - tm * P.tiles_n;
                for (int i = 0; ok && i < L; ++i) {
                    for (int kb = 0; kb < P.kblocks; ++kb, ++it) {
                        const int s = it % CF::STAGES;
                        const uint32_t ph = (it / CF::STAGES) & 1;
                        if (!mbar_wait(&empty[s], ph ^ 1, abort_flag, err, DERR_WAIT_EMPTY)) {
                            ok = false;
                            break;
                        }
                        mbar_arrive_expect_tx(&full[s], CF::STAGE_BYTES);
                        tma_load_3d(sA + s * CF::A_BYTES, P.tmA, &full[s], kb * KB, P.a_row0 + tm * kBM, i);
                        tma_load_4d(sB + s * CF::B_BYTES, P.tmB, &full[s], kb * KB, P.b_col0 + tn * BN, 0, i);
                    }
                }
            }
            if (!ok)
                for (int t = max(0, it - CF::STAGES); t < it; ++t)
                    grouped_drain(&full[t % CF::STAGES], (t / CF::STAGES) & 1, err);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int it = 0, lt = 0;
            bool ok = true, issued_any = false;
            for (int tile = blockIdx.x; ok && tile < total_tiles; tile += gridDim.x, ++lt) {
                const int kblocks = probs[tile_prob[tile]].kblocks;
                const int a = lt & 1;
                const uint32_t aph = (lt >> 1) & 1;
                if (!mbar_wait(&acc_empty[a], aph ^ 1, abort_flag, err, DERR_WAIT_ACCUM_FREE)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem_base + a * CF::ACC_STRIDE;
                for (int i = 0; ok && i < L; ++i) {
                    for (int kb = 0; kb < kblocks; ++kb, ++it) {
                        const int s = it % CF::STAGES;
                        const uint32_t ph = (it / CF::STAGES) & 1;
                        if (!mbar_wait(&full[s], ph, abort_flag, err, DERR_WAIT_FULL)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint64_t adesc = smem_desc_kmajor<KB>(smem_u32(sA + s * CF::A_BYTES));
                        const uint64_t bdesc = smem_desc_kmajor<KB>(smem_u32(sB + s * CF::B_BYTES));
#pragma unroll
                        for (int kk = 0; kk < KB / 32; ++kk)
                            mma_u8(d, adesc + 2 * kk, bdesc + 2 * kk, CF::IDESC, (i | kb | kk) != 0);
                        issued_any = true;
                        mma_commit(&empty[s]);
                    }
                }
                if (ok) mma_commit(&acc_full[a]);
            }
            if (!ok && issued_any) {
                mma_commit(drain);
                grouped_drain(drain, 0, err);
            }
        }
    } else {
        const int q = warp & 3;
        const uint32_t lane_base = static_cast<uint32_t>(q * 32) << 16;
        uint32_t (*stage)[17] = reinterpret_cast<uint32_t (*)[17]>(epi_stage + (warp - 2) * 32 * 17);
        const int chalf = (warp - 2) >> 2;  // the two warps of a lane quarter take alternate 16-column chunks
        const int half = lane >> 4, col_in = lane & 15;
        // Add / Sub read C: each lane prefetches its row of this warp's quarter of
        // a tile into L2 one tile ahead, so the old values come from L2 and the
        // HBM reads of the next tile overlap this tile's drain
        auto prefetch_tile = [&](int t) {
            if (t >= total_tiles) return;
            const GroupedProblem& Q = probs[tile_prob[t]];
            if (Q.op == HME_SET) return;
            const int lq = t - Q.tile_begin;
            const int qm = lq / Q.tiles_n, qn = lq - qm * Q.tiles_n;
            const int row = qm * kBM + q * 32 + lane;
            if (chalf == 0 && row < Q.M) prefetch_l2_span(Q.C + static_cast<size_t>(row) * Q.ldc + qn * BN, min(BN, Q.N - qn * BN));
        };
        prefetch_tile(blockIdx.x);
        int lt = 0;
        for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x, ++lt) {
            prefetch_tile(tile + gridDim.x);
            const int a = lt & 1;
            const uint32_t aph = (lt >> 1) & 1;
            if (!mbar_wait(&acc_full[a], aph, abort_flag, err, DERR_WAIT_ACCUM)) break;
            tc_fence_after();
            const GroupedProblem& P = probs[tile_prob[tile]];
            const int local = tile - P.tile_begin;
            const int tm = local / P.tiles_n, tn = local - tm * P.tiles_n;
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
                    stage[lane][e] = reduce_u64(s, p, barrett);
                }
                __syncwarp();
                const int col = tn * BN + c0 + col_in;
                if (col < P.N) {
                    // all 16 rows' C values in flight at once, then combine and store
                    const int rlim = min(32, P.M - row0);
                    uint32_t old[16];
                    if (P.op != HME_SET) {
#pragma unroll
                        for (int t = 0; t < 16; ++t) {
                            const int rr = half + 2 * t;
                            old[t] = rr < rlim ? P.C[static_cast<size_t>(row0 + rr) * P.ldc + col] : 0u;
                        }
                    }
#pragma unroll
                    for (int t = 0; t < 16; ++t) {
                        const int rr = half + 2 * t;
                        if (rr >= rlim) break;
                        uint32_t o = stage[rr][col_in];
                        if (P.op == HME_ADD) o = mod_add(old[t], o, p);
                        else if (P.op == HME_SUB) o = mod_sub(old[t], o, p);
                        P.C[static_cast<size_t>(row0 + rr) * P.ldc + col] = o;
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
__global__ void __launch_bounds__(256) grouped_split_kernel(const GroupedSplitJob* __restrict__ jobs,
                                                            const int* __restrict__ block_job, int nblocks_arg,
                                                            const int* __restrict__ d_nblocks) {
    __shared__ uint32_t tile[64][33];
    const int nblocks = d_nblocks ? *d_nblocks : nblocks_arg;
    for (int b = blockIdx.x; b < nblocks; b += gridDim.x) {
        __syncthreads();  // the previous block's use of the tile is over
        const GroupedSplitJob& J = jobs[block_job[b]];
        const int local = b - J.block_begin;
        if (local < J.s.a_blocks)
            split_a_part<L>(J.s, local);
        else
            split_b_part<L>(J.s, local - J.s.a_blocks, tile);
    }
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

template <int L, int BN, int KB>
void ensure_grouped_attr() {
    static OncePerDevice attr;
    attr.run([](int) {
        HME_CUDA(cudaFuncSetAttribute(grouped_limb_gemm_kernel<L, BN, KB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      Cfg<L, BN, KB>::SMEM));
    });
}

template <int L, int BN, int KB>
void launch_grouped(hme_ctx* ctx, const ModParams& mp, const GroupedProblem* d_probs, const int* d_tile_prob,
                    int total_tiles, const int* d_total = nullptr) {
    using CF = Cfg<L, BN, KB>;
    ensure_grouped_attr<L, BN, KB>();
    const int grid = d_total ? ctx->num_sms : std::min(total_tiles, ctx->num_sms);
    HME_TIMED(ctx, "grouped_gemm", grouped_limb_gemm_kernel<L, BN, KB><<<grid, kThreads, CF::SMEM, ctx->stream>>>(
                                       d_probs, d_tile_prob, total_tiles, d_total, mp.p, mp.barrett, ctx->d_err));
    HME_CUDA(cudaGetLastError());
}

template <int L>
void run_grouped(hme_ctx* ctx, const ModParams& mp, const std::vector<GemmJob>& jobs_in, int bn_choice) {
    std::vector<GemmJob> jobs;
    jobs.reserve(jobs_in.size());
    for (const GemmJob& j : jobs_in) {
        if (j.M == 0 || j.N == 0) continue;
        HME_REQUIRE(j.K > 0 && j.K <= limb_k_chunk(L), "grouped gemm: K must be in [1, the exact-accumulation chunk]");
        jobs.push_back(j);
    }
    if (jobs.empty()) return;
    const int nj = static_cast<int>(jobs.size());
    // tile width: wide (L*BN close to 256) unless the whole group leaves SMs idle
    constexpr int BNw = grouped_bn_wide(L);
    constexpr int BNn = L == 1 ? 128 : L == 2 ? 64 : 32;
    size_t tiles_wide = 0;
    for (const GemmJob& j : jobs) tiles_wide += static_cast<size_t>((j.M + kBM - 1) / kBM) * ((j.N + BNw - 1) / BNw);
    const bool narrow = bn_choice == 1 || (bn_choice < 0 && tiles_wide < static_cast<size_t>(ctx->num_sms));
    const int BN = narrow ? BNn : BNw;
    // k-block: the narrowest swizzle row (32, 64 or 128 bytes) that holds every
    // K of the launch (the rank rounds' updates have K = the round's pivots), so
    // no zero padding is streamed or multiplied
    uint32_t kmax = 0;
    for (const GemmJob& j : jobs) kmax = std::max(kmax, j.K);
    const int KBsel = kmax <= 32 ? 32 : kmax <= 64 ? 64 : kBK;

    // plane layout: problems bucketed by padded K; per bucket one stacked tensor
    // for the A planes (rows of all problems) and one for the B planes
    std::vector<int> kp_of(nj), bucket_of(nj);
    std::vector<int> bucket_kp;
    for (int t = 0; t < nj; ++t) {
        kp_of[t] = static_cast<int>((jobs[t].K + KBsel - 1) / KBsel * KBsel);
        auto it = std::find(bucket_kp.begin(), bucket_kp.end(), kp_of[t]);
        if (it == bucket_kp.end()) {
            bucket_of[t] = static_cast<int>(bucket_kp.size());
            bucket_kp.push_back(kp_of[t]);
        } else {
            bucket_of[t] = static_cast<int>(it - bucket_kp.begin());
        }
    }
    const int nb = static_cast<int>(bucket_kp.size());
    std::vector<size_t> b_rows(nb, 0), b_cols(nb, 0);
    std::vector<int> row0(nj), col0(nj);
    for (int t = 0; t < nj; ++t) {
        row0[t] = static_cast<int>(b_rows[bucket_of[t]]);
        col0[t] = static_cast<int>(b_cols[bucket_of[t]]);
        b_rows[bucket_of[t]] += jobs[t].M;
        b_cols[bucket_of[t]] += jobs[t].N;
    }
    std::vector<size_t> offA(nb), offB(nb);
    size_t bytes = 0;
    for (int b = 0; b < nb; ++b) {
        offA[b] = bytes;
        bytes += align256(static_cast<size_t>(L) * b_rows[b] * bucket_kp[b]);
        offB[b] = bytes;
        bytes += align256(static_cast<size_t>(L) * L * b_cols[b] * bucket_kp[b]);
    }
    HME_REQUIRE(static_cast<double>(bytes) < 1.0e11, "grouped gemm: plane tensors too large");
    uint8_t* planes = static_cast<uint8_t*>(ctx->ws.get(kSlotJobs0, bytes));
    std::vector<GroupedSplitJob> split(nj);
    int blocks = 0;
    for (int t = 0; t < nj; ++t) {
        const GemmJob& j = jobs[t];
        const int b = bucket_of[t];
        const int Kp = kp_of[t];
        SplitArgs& s = split[t].s;
        s = SplitArgs{};
        s.A = j.A;
        s.lda = j.lda;
        s.B = j.B;
        s.ldb = j.ldb;
        s.M = static_cast<int>(j.M);
        s.N = static_cast<int>(j.N);
        s.K = static_cast<int>(j.K);
        s.Kp = Kp;
        s.p = mp.p;
        s.barrett = mp.barrett;
        s.planesA = planes + offA[b] + static_cast<size_t>(row0[t]) * Kp;
        s.planesB = planes + offB[b] + static_cast<size_t>(col0[t]) * Kp;
        s.a_plane = static_cast<uint64_t>(b_rows[b]) * Kp;
        s.b_plane = static_cast<uint64_t>(b_cols[b]) * Kp;
        const size_t work = static_cast<size_t>(j.M) * (Kp / 16);
        s.a_blocks = static_cast<int>(std::max<size_t>(1, std::min<size_t>((work + 255) / 256, 64)));
        s.b_blocks_k = (Kp + 63) / 64;
        s.a_vec = ((reinterpret_cast<uintptr_t>(j.A) & 15) == 0) && ((j.lda & 3) == 0);
        split[t].b_blocks = s.b_blocks_k * static_cast<int>((j.N + 31) / 32);
        split[t].block_begin = blocks;
        blocks += s.a_blocks + split[t].b_blocks;
    }
    // tensor maps (64-byte aligned objects, two per bucket) and the problem table
    const size_t maps_bytes = sizeof(CUtensorMap) * 2 * static_cast<size_t>(nb);
    const size_t probs_bytes = sizeof(GroupedProblem) * static_cast<size_t>(nj);
    const size_t split_bytes = sizeof(GroupedSplitJob) * static_cast<size_t>(nj);
    // per-tile problem and per-split-block job (tile counts known only after the layout)
    size_t total_tiles = 0;
    for (const GemmJob& j : jobs) total_tiles += static_cast<size_t>((j.M + kBM - 1) / kBM) * ((j.N + BN - 1) / BN);
    HME_REQUIRE(total_tiles < (1u << 31) && static_cast<size_t>(blocks) < (1u << 31), "grouped gemm: too many tiles");
    const size_t index_bytes = sizeof(int) * (total_tiles + static_cast<size_t>(blocks));
    uint8_t* tables = static_cast<uint8_t*>(ctx->ws.get(kSlotJobs1, align256(maps_bytes) + align256(probs_bytes) +
                                                                         align256(split_bytes) + align256(index_bytes)));
    CUtensorMap* d_maps = reinterpret_cast<CUtensorMap*>(tables);
    GroupedProblem* d_probs = reinterpret_cast<GroupedProblem*>(tables + align256(maps_bytes));
    GroupedSplitJob* d_split = reinterpret_cast<GroupedSplitJob*>(tables + align256(maps_bytes) + align256(probs_bytes));
    int* d_tile_prob = reinterpret_cast<int*>(tables + align256(maps_bytes) + align256(probs_bytes) +
                                              align256(split_bytes));
    int* d_block_job = d_tile_prob + total_tiles;
    std::vector<CUtensorMap> maps(2 * static_cast<size_t>(nb));
    for (int b = 0; b < nb; ++b) {
        const cuuint64_t Kp = static_cast<cuuint64_t>(bucket_kp[b]);
        {
            const cuuint64_t dims[3] = {Kp, b_rows[b], static_cast<cuuint64_t>(L)};
            const cuuint64_t strides[2] = {Kp, Kp * b_rows[b]};
            const cuuint32_t box[3] = {static_cast<cuuint32_t>(KBsel), kBM, 1};
            encode_tma_u8_kb(&maps[2 * b], planes + offA[b], 3, dims, strides, box, KBsel);
        }
        {
            const cuuint64_t dims[4] = {Kp, b_cols[b], static_cast<cuuint64_t>(L), static_cast<cuuint64_t>(L)};
            const cuuint64_t strides[3] = {Kp, Kp * b_cols[b], Kp * b_cols[b] * L};
            const cuuint32_t box[4] = {static_cast<cuuint32_t>(KBsel), static_cast<cuuint32_t>(BN),
                                       static_cast<cuuint32_t>(L), 1};
            encode_tma_u8_kb(&maps[2 * b + 1], planes + offB[b], 4, dims, strides, box, KBsel);
        }
    }
    std::vector<GroupedProblem> probs(nj);
    int tiles = 0;
    for (int t = 0; t < nj; ++t) {
        const GemmJob& j = jobs[t];
        GroupedProblem& P = probs[t];
        P.tmA = d_maps + 2 * bucket_of[t];
        P.tmB = d_maps + 2 * bucket_of[t] + 1;
        P.C = j.C;
        P.ldc = j.ldc;
        P.M = static_cast<int>(j.M);
        P.N = static_cast<int>(j.N);
        P.kblocks = kp_of[t] / KBsel;
        P.op = j.op;
        P.tiles_n = static_cast<int>((j.N + BN - 1) / BN);
        P.tile_begin = tiles;
        P.a_row0 = row0[t];
        P.b_col0 = col0[t];
        tiles += static_cast<int>((j.M + kBM - 1) / kBM) * P.tiles_n;
    }
    HME_CUDA(cudaMemcpyAsync(d_maps, maps.data(), maps_bytes, cudaMemcpyHostToDevice, ctx->stream));
    HME_CUDA(cudaMemcpyAsync(d_probs, probs.data(), probs_bytes, cudaMemcpyHostToDevice, ctx->stream));
    HME_CUDA(cudaMemcpyAsync(d_split, split.data(), split_bytes, cudaMemcpyHostToDevice, ctx->stream));
    std::vector<int> index(total_tiles + static_cast<size_t>(blocks));
    for (int t = 0; t < nj; ++t) {
        const int nt = static_cast<int>((jobs[t].M + kBM - 1) / kBM) * probs[t].tiles_n;
        std::fill(index.begin() + probs[t].tile_begin, index.begin() + probs[t].tile_begin + nt, t);
        const int nbk = split[t].s.a_blocks + split[t].b_blocks;
        std::fill(index.begin() + total_tiles + split[t].block_begin,
                  index.begin() + total_tiles + split[t].block_begin + nbk, t);
    }
    HME_REQUIRE(static_cast<size_t>(tiles) == total_tiles, "grouped gemm: tile count mismatch");
    HME_CUDA(cudaMemcpyAsync(d_tile_prob, index.data(), index_bytes, cudaMemcpyHostToDevice, ctx->stream));
    HME_TIMED(ctx, "grouped_split",
              grouped_split_kernel<L><<<blocks, 256, 0, ctx->stream>>>(d_split, d_block_job, blocks, nullptr));
    HME_CUDA(cudaGetLastError());
    if (KBsel == 32) {
        if (narrow) launch_grouped<L, BNn, 32>(ctx, mp, d_probs, d_tile_prob, tiles);
        else launch_grouped<L, BNw, 32>(ctx, mp, d_probs, d_tile_prob, tiles);
    } else if (KBsel == 64) {
        if (narrow) launch_grouped<L, BNn, 64>(ctx, mp, d_probs, d_tile_prob, tiles);
        else launch_grouped<L, BNw, 64>(ctx, mp, d_probs, d_tile_prob, tiles);
    } else {
        if (narrow) launch_grouped<L, BNn, kBK>(ctx, mp, d_probs, d_tile_prob, tiles);
        else launch_grouped<L, BNw, kBK>(ctx, mp, d_probs, d_tile_prob, tiles);
    }
    // the host tables must outlive the asynchronous uploads
    HME_CUDA(cudaStreamSynchronize(ctx->stream));
}

template <int L>
void launch_device_tables(hme_ctx* ctx, const ModParams& mp, const GroupedSplitJob* d_split, const int* d_block_job,
                          const int* d_nblocks, const GroupedProblem* d_probs, const int* d_tile_prob,
                          const int* d_ntiles) {
    const int split_grid = ctx->num_sms * 8;
    HME_TIMED(ctx, "grouped_split", grouped_split_kernel<L><<<split_grid, 256, 0, ctx->stream>>>(d_split, d_block_job,
                                                                                              0, d_nblocks));
    HME_CUDA(cudaGetLastError());
    launch_grouped<L, grouped_bn_wide(L), 32>(ctx, mp, d_probs, d_tile_prob, 0, d_ntiles);
}

}  // namespace

void grouped_prepare_device_tables(uint32_t limbs) {
    switch (limbs) {
        case 1: ensure_grouped_attr<1, grouped_bn_wide(1), 32>(); break;
        case 2: ensure_grouped_attr<2, grouped_bn_wide(2), 32>(); break;
        case 3: ensure_grouped_attr<3, grouped_bn_wide(3), 32>(); break;
        default: ensure_grouped_attr<4, grouped_bn_wide(4), 32>(); break;
    }
}

void grouped_launch_device_tables(hme_ctx* ctx, const ModParams& mp, const GroupedSplitJob* d_split,
                                  const int* d_block_job, const int* d_nblocks, const GroupedProblem* d_probs,
                                  const int* d_tile_prob, const int* d_ntiles) {
    switch (mp.limbs) {
        case 1: launch_device_tables<1>(ctx, mp, d_split, d_block_job, d_nblocks, d_probs, d_tile_prob, d_ntiles); break;
        case 2: launch_device_tables<2>(ctx, mp, d_split, d_block_job, d_nblocks, d_probs, d_tile_prob, d_ntiles); break;
        case 3: launch_device_tables<3>(ctx, mp, d_split, d_block_job, d_nblocks, d_probs, d_tile_prob, d_ntiles); break;
        default: launch_device_tables<4>(ctx, mp, d_split, d_block_job, d_nblocks, d_probs, d_tile_prob, d_ntiles); break;
    }
}

void grouped_gemm_u32_device(hme_ctx* ctx, const ModParams& mp, const std::vector<GemmJob>& jobs, int bn_choice) {
    switch (mp.limbs) {
        case 1: run_grouped<1>(ctx, mp, jobs, bn_choice); break;
        case 2: run_grouped<2>(ctx, mp, jobs, bn_choice); break;
        case 3: run_grouped<3>(ctx, mp, jobs, bn_choice); break;
        default: run_grouped<4>(ctx, mp, jobs, bn_choice); break;
    }
}

}  // namespace hme

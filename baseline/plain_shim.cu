// The PLAIN METHOD: the reference's own CUDA-core mod-p GEMM
// (drjanosch42/hacs 0.2.1, src/Cuda/cuda_kernels.cu gemm_kernel :195-299,
// launch :328-382, entry engine::cuda::gemm :815), compiled unchanged for
// sm_100a from the reference sources by baseline/Makefile into
// baseline/_ref/libplain.so.  This shim only exposes it through a C ABI so that
// bench.py can time it beside the INT8-limb tensor-core GEMM on the same
// device buffers.  The IMMA route is switched off (GemmOpts::imma = 0): it
// covers p <= 127 only, and the plain method is the u32 CUDA-core kernel.
#include <cuda_runtime.h>

#include <exception>
#include <string>

#include "CudaKernels.h"

using namespace engine;

namespace {
thread_local std::string g_err;
}

extern "C" {

const char* plain_last_error() { return g_err.c_str(); }

// C op= A*B mod p, device pointers, row-major, on `stream` (cudaStream_t).
int plain_gemm_u32_dev(uint32_t p, uint32_t m, uint32_t n, uint32_t k, const uint32_t* A, size_t lda,
                       const uint32_t* B, size_t ldb, uint32_t* C, size_t ldc, int op, void* stream) {
    try {
        const ModCtx<uint32_t> ctx(p);
        cuda::DeviceView<const uint32_t> a(A, lda, 1, m, k);
        cuda::DeviceView<const uint32_t> b(B, ldb, 1, k, n);
        cuda::DeviceView<uint32_t> c(C, ldc, 1, m, n);
        cuda::GemmOpts o;
        o.imma = 0;
        const auto gop = op == 0 ? kernels::GemmOp::Set : op == 1 ? kernels::GemmOp::Add : kernels::GemmOp::Sub;
        cuda::gemm<uint32_t>(ctx, a, b, c, gop, cuda::Stream{stream}, o);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// The same for u64 residues (ModCtx<uint64_t>: Montgomery for odd p < 2^63, wide otherwise).
int plain_gemm_u64_dev(uint64_t p, uint32_t m, uint32_t n, uint32_t k, const uint64_t* A, size_t lda,
                       const uint64_t* B, size_t ldb, uint64_t* C, size_t ldc, int op, void* stream) {
    try {
        const ModCtx<uint64_t> ctx(p);
        cuda::DeviceView<const uint64_t> a(A, lda, 1, m, k);
        cuda::DeviceView<const uint64_t> b(B, ldb, 1, k, n);
        cuda::DeviceView<uint64_t> c(C, ldc, 1, m, n);
        cuda::GemmOpts o;
        o.imma = 0;
        const auto gop = op == 0 ? kernels::GemmOp::Set : op == 1 ? kernels::GemmOp::Add : kernels::GemmOp::Sub;
        cuda::gemm<uint64_t>(ctx, a, b, c, gop, cuda::Stream{stream}, o);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

}  // extern "C"

// Modulus constants shared by host and device code.
//
// A u32 modulus 2 <= p < 2^32 (a prime for the field routes, ell^k for the
// ring routes) with the Barrett constant of the reference's
// ModCtx<uint32_t>::init (src/ModArithmetic/ModCtx.h:202-250): m =
// floor(2^64 / p), and reduce(x) = x - mulhi(x, m) * p, corrected once, is x
// mod p for EVERY x < 2^64 (ModCtx.h:323-329).  Limb count L: the number of
// unsigned bytes a residue in [0, p) needs (p <= 256^L).
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define HME_HD __host__ __device__ __forceinline__
#else
#define HME_HD inline
#endif

namespace hme {

struct ModParams {
    uint32_t p = 0;
    uint32_t limbs = 0;    // unsigned 8-bit limbs per residue
    uint64_t barrett = 0;  // floor(2^64 / p)
};

inline ModParams make_mod(uint32_t p) {
    ModParams mp;
    mp.p = p;
    mp.limbs = p <= 256u ? 1u : p <= 65536u ? 2u : p <= (1u << 24) ? 3u : 4u;
    mp.barrett = static_cast<uint64_t>((static_cast<unsigned __int128>(1) << 64) / p);
    return mp;
}

HME_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return static_cast<uint64_t>((static_cast<unsigned __int128>(a) * b) >> 64);
#endif
}

HME_HD uint32_t reduce_u64(uint64_t x, uint32_t p, uint64_t m) {
    const uint64_t q = mulhi64(x, m);
    uint64_t r = x - q * p;
    if (r >= p) r -= p;
    return static_cast<uint32_t>(r);
}
HME_HD uint32_t mod_add(uint32_t a, uint32_t b, uint32_t p) {
    const uint64_t s = static_cast<uint64_t>(a) + b;
    return static_cast<uint32_t>(s >= p ? s - p : s);
}
HME_HD uint32_t mod_sub(uint32_t a, uint32_t b, uint32_t p) {
    return a >= b ? a - b : static_cast<uint32_t>(static_cast<uint64_t>(a) + p - b);
}
HME_HD uint32_t mod_mul(uint32_t a, uint32_t b, uint32_t p, uint64_t m) {
    return reduce_u64(static_cast<uint64_t>(a) * b, p, m);
}

// Largest K chunk (a multiple of 128) such that L limb products of two
// unsigned bytes, summed over the chunk, stay below 2^31:
// L * 255 * 255 * K_chunk < 2^31.
inline uint32_t limb_k_chunk(uint32_t L) {
    const uint64_t lim = ((1ull << 31) - 1) / (static_cast<uint64_t>(L) * 255u * 255u);
    return static_cast<uint32_t>(lim / 128u * 128u);
}

}  // namespace hme

// The device elimination driver over F_p (elim.cu) and its options.
#pragma once
#include <cstdint>
#include <vector>

#include "hme_internal.h"

namespace hme {


struct ElimResult {
    int rank = 0;
    std::vector<int> pivots;      // pivot columns, ascending (the column rank profile)
    std::vector<uint32_t> diag;   // U[t][pivots[t]] when ElimOptions::want_diag
    bool sign_negative = false;   // parity of the row permutation applied
};

// Elimination over Z/q, q = ell^k (mp.p == q): pivots of valuation <= max_v
// (0: unit pivots; k - 1: any non-zero entry, the minimal valuation first),
// LU restricted to the first lu_cols columns (0 = all) with the trailing
// updates still covering every column.  Absent: the field F_p.
struct RingSpec {
    uint32_t ell = 0, k = 1;
    uint32_t max_v = 0;
    int lu_cols = 0;
};

// Factor A (m x n, row-major, ld, device memory; destroyed) and, when
// want_rref (fields only), write RREF(A) into R (m x n, ldr; R may equal A).
// After the call rows [0, rank) of A hold the echelon rows (pivot rows in
// pivot order; entries left of a row's pivot column are stale multipliers)
// and rows [rank, m) the Schur complement of the factored columns.
ElimResult elim_device(hme_ctx* ctx, const ModParams& mp, uint32_t* A, size_t ld, int m, int n, bool want_rref,
                       uint32_t* R, size_t ldr, const ElimOptions& opt, const RingSpec* ring = nullptr);

}  // namespace hme

namespace hme {

struct HowellOut {
    std::vector<uint32_t> H;  // h x n, row-major
    std::vector<int> pivots;
    std::vector<int> pivot_v;
};

// Smith valuations (ascending) of A (m x n, device, canonical mod ell^k).
std::vector<uint32_t> smith_device(hme_ctx* ctx, uint32_t ell, uint32_t k, const uint32_t* A, size_t lda, int m,
                                   int n, const ElimOptions& opt);
// Howell form of rowspan(A) (m x n, device, canonical mod ell^k).
HowellOut howell_device(hme_ctx* ctx, uint32_t ell, uint32_t k, const uint32_t* A, size_t lda, int m, int n,
                        const ElimOptions& opt);

}  // namespace hme

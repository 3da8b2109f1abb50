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

// Factor A (m x n, row-major, ld, device memory; destroyed) and, when
// want_rref, write RREF(A) into R (m x n, ldr; R may equal A).
ElimResult elim_device(hme_ctx* ctx, const ModParams& mp, uint32_t* A, size_t ld, int m, int n, bool want_rref,
                       uint32_t* R, size_t ldr, const ElimOptions& opt);

}  // namespace hme
